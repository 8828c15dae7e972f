"""GPU: the reactive gradient on z-slabs (slab.ReactiveSlabGradient over the
lbm_reactive_slab_* entries) against the whole-box lbm_reactive_gradient_async.

The slabs of one box run in this process in lockstep (slab.run_local: the
exchanges are device copies, the all-reduces sums in rank order), from 1 to 8
ranks (8 ranks of an 8-plane box leaves one plane per slab, whose pulls and
scatters cross both faces). Every cell of a slab does the whole box's
arithmetic on the same inputs, so:
* mean-product objective (the seed is -1/N_c on every cell): dJ/dA0, dJ/dB0
  and dJ/du0 assembled from the slabs equal the whole box's bit for bit;
* segregation intensity: the seed depends on the FP64 statistics, which the
  slabs add in another order, so the fields agree to 1e-12 (FP64) / 1e-6
  (FP32) relative L2;
* J, dJ/dk, dJ/dtau, dJ/dtau_c: the per-warp FP64 slot sums are the same
  numbers, added in another order: relative 1e-10.
The step count is not a multiple of the checkpoint interval (a partial last
segment, and recomputed segments before it). With 16-bit stored states (each
format once; the slabs exchange faces of codes and the adjoint's FP32 scatter
faces) the same bars hold against the whole-box 16-bit gradient.
"""
import numpy as np
import pytest
import torch

import _util as U
import lbcube as E
import slab
from test_gpu_adjoint_reactive import fields

pytestmark = pytest.mark.gpu

TAU, TAU_C, K = 0.8, 0.7, 0.6
C0 = 0.5  # shift of 16-bit scalar states


def whole_box(fl, real, op, obj, rho, u, a, b, dims, steps, interval, storage=None):
    nx, ny, nz = dims
    nb = E.reactive_gradient_workspace_bytes(fl, real, nx, ny, nz, steps, interval, storage=storage)
    ws = torch.empty(nb, dtype=torch.uint8, device=a.device)
    res = torch.zeros(4, dtype=torch.float64, device=a.device)
    ga, gb, gu = torch.empty_like(a), torch.empty_like(b), torch.empty_like(u)
    E.check(E.reactive_gradient_async(fl, real, op, obj, rho, u, a, b, nx, ny, nz, TAU, TAU_C, K, steps, interval,
                                      ws, nb, res, ga, gb, gu, storage=storage, c0=C0))
    torch.cuda.synchronize()
    return res.cpu().numpy(), ga.cpu().numpy(), gb.cpu().numpy(), gu.cpu().numpy()


def slabs(fl, real, op, obj, rho, u, a, b, dims, steps, interval, world, storage=None):
    nx, ny, nz = dims
    grads = [slab.ReactiveSlabGradient(torch, fl, real, op, obj, nx, ny, nz, TAU, TAU_C, K, steps, interval, r, world,
                                       a.device, storage=storage, c0=C0) for r in range(world)]
    inputs = []
    for g in grads:
        sl = slice(g.z0, g.z0 + g.nz)
        inputs.append((rho[sl].contiguous(), u[:, sl].contiguous(), a[sl].contiguous(), b[sl].contiguous()))
    slab.run_local(grads, inputs)
    torch.cuda.synchronize()
    results = [g.result.cpu().numpy() for g in grads]
    ga = np.concatenate([g.grad_a0.cpu().numpy() for g in grads], axis=0)
    gb = np.concatenate([g.grad_b0.cpu().numpy() for g in grads], axis=0)
    gu = np.concatenate([g.grad_u0.cpu().numpy() for g in grads], axis=1)
    return results, ga, gb, gu


CASES = [
    ("D3Q19", "double", "BGK", "mean_product", (12, 6, 8), 7, 3, 2, None),
    ("D3Q19", "double", "TRT", "segregation", (12, 6, 8), 7, 3, 4, None),
    ("D3Q19", "double", "MRT", "mean_product", (12, 6, 8), 5, 2, 2, None),
    ("D3Q19", "double", "BGK", "mean_product", (10, 4, 8), 5, 3, 8, None),
    ("D3Q19", "float", "TRT", "mean_product", (16, 6, 6), 7, 3, 1, None),
    ("D3Q27", "float", "TRT", "mean_product", (12, 6, 8), 7, 3, 2, None),
    ("D3Q27", "double", "BGK", "segregation", (12, 6, 8), 6, 4, 2, None),
    # 16-bit stored states (the forward of the C5 configuration)
    ("D3Q19", "float", "TRT", "mean_product", (12, 6, 8), 7, 3, 2, "f16s"),
    ("D3Q19", "float", "MRT", "segregation", (12, 6, 8), 6, 3, 4, "q15s"),
    ("D3Q19", "float", "BGK", "mean_product", (16, 6, 6), 7, 3, 1, "bf16s"),
    ("D3Q27", "float", "TRT", "mean_product", (10, 4, 8), 5, 2, 8, "e3m12s"),
]


@pytest.mark.parametrize("fl,real,op,obj,dims,steps,interval,world,storage", CASES)
def test_slab_gradient_matches_whole_box(engine, dev, fl, real, op, obj, dims, steps, interval, world, storage):
    nx, ny, nz = dims
    dtype = torch.float32 if real == "float" else torch.float64
    rho, u, a, b = fields(fl, (nz, ny, nx), dev, dtype, seed=91)
    want = whole_box(fl, real, op, obj, rho, u, a, b, dims, steps, interval, storage)
    results, ga, gb, gu = slabs(fl, real, op, obj, rho, u, a, b, dims, steps, interval, world, storage)
    for r in results[1:]:
        assert np.array_equal(r, results[0]), "ranks disagree on the all-reduced scalars"
    w = want[0]
    assert np.all(np.abs(results[0] - w) <= 1e-10 * np.abs(w) + 1e-300), (results[0], w)
    for name, got, ref in (("dJ/dA0", ga, want[1]), ("dJ/dB0", gb, want[2]), ("dJ/du0", gu, want[3])):
        if obj == "mean_product":
            assert U.same_bits(got, ref), name
        else:
            assert U.rel_l2(got, ref) <= (1e-6 if real == "float" else 1e-12), name


def test_slab_gradient_rejects_bad_arguments(engine, dev):
    nx, ny, nz = 8, 4, 4
    t = torch.zeros((3, nz, ny, nx), dtype=torch.float64, device=dev)
    lib = E.load()
    args = dict(nx=nx, ny=ny, nz=nz)
    # D2Q9 has no slab form; D3Q27 MRT has no adjoint
    assert lib.lbm_reactive_slab_slots_bytes(E.LATTICES["D2Q9"], nx, ny, nz) == 0
    p = t.data_ptr()
    rc = lib.lbm_reactive_slab_forward_async(E.LATTICES["D3Q27"], E.REALS["double"], 0, C0, E.COLLISIONS["MRT"], p,
                                             p, p, p, p, p, None, args["nx"], args["ny"], args["nz"], TAU, TAU_C, K,
                                             p, p, p, p, None)
    assert rc != 0
    # 16-bit states need FP32
    rc = lib.lbm_reactive_slab_forward_async(E.LATTICES["D3Q19"], E.REALS["double"], E.FORMATS["f16s"], C0,
                                             E.COLLISIONS["BGK"], p, p, p, p, p, p, None, args["nx"], args["ny"],
                                             args["nz"], TAU, TAU_C, K, p, p, p, p, None)
    assert rc != 0
    # tau at the stability limit
    f = [torch.zeros((q, nz, ny, nx), dtype=torch.float64, device=dev) for q in (19, 19, 7, 7, 7, 7)]
    n = lib.lbm_fluid_reaction_slab_face_elems(E.LATTICES["D3Q19"], nx, ny)
    h = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(4)]
    rc = lib.lbm_reactive_slab_forward_async(E.LATTICES["D3Q19"], E.REALS["double"], 0, C0, E.COLLISIONS["BGK"],
                                             f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), f[3].data_ptr(),
                                             f[4].data_ptr(), f[5].data_ptr(), None, nx, ny, nz, 0.5, TAU_C, K,
                                             h[0].data_ptr(), h[1].data_ptr(), h[2].data_ptr(), h[3].data_ptr(), None)
    assert rc != 0
    # a send buffer aliasing a halo buffer
    rc = lib.lbm_reactive_slab_forward_async(E.LATTICES["D3Q19"], E.REALS["double"], 0, C0, E.COLLISIONS["BGK"],
                                             f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), f[3].data_ptr(),
                                             f[4].data_ptr(), f[5].data_ptr(), None, nx, ny, nz, TAU, TAU_C, K,
                                             h[0].data_ptr(), h[1].data_ptr(), h[0].data_ptr(), h[3].data_ptr(), None)
    assert rc != 0
    # a slots buffer smaller than lbm_reactive_slab_slots_bytes
    sb = lib.lbm_reactive_slab_slots_bytes(E.LATTICES["D3Q19"], nx, ny, nz)
    slots = torch.zeros(sb // 8, dtype=torch.float64, device=dev)
    lam = [torch.zeros((q, nz, ny, nx), dtype=torch.float64, device=dev) for q in (19, 7, 7, 19, 7, 7)]
    rc = lib.lbm_reactive_slab_adjoint_step_async(
        E.LATTICES["D3Q19"], E.REALS["double"], 0, C0, E.COLLISIONS["BGK"], f[0].data_ptr(), f[2].data_ptr(),
        f[3].data_ptr(), h[0].data_ptr(), h[1].data_ptr(), t.data_ptr(), lam[0].data_ptr(), lam[1].data_ptr(),
        lam[2].data_ptr(), lam[3].data_ptr(), lam[4].data_ptr(), lam[5].data_ptr(), f[1].data_ptr(), h[2].data_ptr(),
        h[3].data_ptr(), nx, ny, nz, TAU, TAU_C, K, slots.data_ptr(), sb - 8, None)
    assert rc != 0
    torch.cuda.synchronize()

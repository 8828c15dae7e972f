"""GPU: the z-slab decomposition on one device. W ranks are emulated in one
process (LocalExchange copies the face buffers between slabs, standing in for
the point-to-point transfers); stepping the slabs is bit-identical to
stepping the whole periodic box with lbm_step_async, for W = 1..4 including
one-plane slabs, and the same holds for the coupled fluid + A + B -> C step
with its statistics. The single-rank path of SlabDomain.step (exchange on a
second stream, overlapped with the interior planes) is bit-identical too.
tests/test_gpu_slab_mp.py runs the ranks as separate processes."""
import numpy as np
import pytest
import torch

import _util as U
import lbcube as E
import slab

pytestmark = pytest.mark.gpu

CASES = [("D3Q19", "float", "TRT", (16, 6, 8)), ("D3Q19", "double", "BGK", (10, 5, 6)),
         ("D3Q27", "float", "MRT", (8, 4, 4)), ("D3Q19", "float", "RLBM", (12, 3, 4)),
         ("D3Q27", "double", "TRT", (6, 4, 8))]


def whole_box(lat, dn, op, f, dims, steps, dev):
    nx, ny, nz = dims
    a = torch.from_numpy(f).to(dev)
    b = torch.empty_like(a)
    for _ in range(steps):
        E.check(E.step_async(lat, dn, op, a, b, nx, ny, nz, 1 / 0.6))
        a, b = b, a
    torch.cuda.synchronize()
    return a.cpu().numpy()


@pytest.mark.parametrize("lat,dn,op,dims", CASES)
@pytest.mark.parametrize("world", [1, 2, 4])
def test_slabs_match_whole_box(engine, dev, lat, dn, op, dims, world):
    nx, ny, nz = dims
    if nz % world:
        pytest.skip("nz not divisible")
    steps = 7
    f = U.random_state(lat, nx, ny, nz, np.float32 if dn == "float" else np.float64, seed=21)
    want = whole_box(lat, dn, op, f, dims, steps, dev)
    Q = f.shape[0]
    f4 = f.reshape(Q, nz, ny, nx)
    doms = [slab.SlabDomain(torch, lat, dn, op, nx, ny, nz, 1 / 0.6, r, world, dev) for r in range(world)]
    cur = [torch.from_numpy(np.ascontiguousarray(f4[:, d.z0:d.z0 + d.nz])).to(dev) for d in doms]
    nxt = [torch.empty_like(c) for c in cur]
    ex = slab.LocalExchange(doms)
    for d, c in zip(doms, cur):
        d.pack(c)
    ex.exchange_all()
    for _ in range(steps):
        for d, c, n in zip(doms, cur, nxt):
            d.compute(c, n)
        ex.exchange_all()
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    got = np.concatenate([c.cpu().numpy() for c in cur], axis=1).reshape(Q, -1)
    assert U.same_bits(got, want)


def test_one_plane_slabs(engine, dev):
    nx, ny, nz = 8, 4, 4
    f = U.random_state("D3Q19", nx, ny, nz, np.float32, seed=22)
    want = whole_box("D3Q19", "float", "TRT", f, (nx, ny, nz), 5, dev)
    doms = [slab.SlabDomain(torch, "D3Q19", "float", "TRT", nx, ny, nz, 1 / 0.6, r, 4, dev) for r in range(4)]
    f4 = f.reshape(19, nz, ny, nx)
    cur = [torch.from_numpy(np.ascontiguousarray(f4[:, r:r + 1])).to(dev) for r in range(4)]
    nxt = [torch.empty_like(c) for c in cur]
    ex = slab.LocalExchange(doms)
    for d, c in zip(doms, cur):
        d.pack(c)
    ex.exchange_all()
    for _ in range(5):
        for d, c, n in zip(doms, cur, nxt):
            assert d.ranges() == ([], [(0, 1)])
            d.compute(c, n)
        ex.exchange_all()
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    got = np.concatenate([c.cpu().numpy() for c in cur], axis=1).reshape(19, -1)
    assert U.same_bits(got, want)


def test_overlapped_single_rank_step(engine, dev):
    import torch.distributed as dist

    nx, ny, nz = 32, 8, 12
    f = U.random_state("D3Q19", nx, ny, nz, np.float32, seed=23)
    want = whole_box("D3Q19", "float", "TRT", f, (nx, ny, nz), 9, dev)
    d = slab.SlabDomain(torch, "D3Q19", "float", "TRT", nx, ny, nz, 1 / 0.6, 0, 1, dev)
    ex = slab.DistributedExchange(dist)
    a = torch.from_numpy(f).to(dev).view(19, nz, ny, nx)
    b = torch.empty_like(a)
    d.prime(a, ex)
    for _ in range(9):
        d.step(a, b, ex)
        a, b = b, a
    d.finish()
    torch.cuda.synchronize()
    assert U.same_bits(a.cpu().numpy().reshape(19, -1), want)


def test_slab_validation(engine, dev):
    d = slab.SlabDomain(torch, "D3Q19", "float", "TRT", 8, 4, 6, 1.6, 0, 2, dev)
    a = torch.zeros((19, 3, 4, 8), device=dev)
    b = torch.zeros_like(a)
    lib = E.load()
    args = lambda z0, z1, hl, hh, sl, sh: lib.lbm_step_slab_async(  # noqa: E731
        1, 0, 1, a.data_ptr(), b.data_ptr(), 8, 4, 3, 1.6, hl, hh, sl, sh, z0, z1, None)
    p = [d.halo_lo.data_ptr(), d.halo_hi.data_ptr(), d.send_lo.data_ptr(), d.send_hi.data_ptr()]
    assert args(0, 4, *p) == E.cudaErrorInvalidValue          # range past the slab
    assert args(2, 2, *p) == E.cudaErrorInvalidValue          # empty range
    assert args(0, 1, None, p[1], p[2], p[3]) == E.cudaErrorInvalidDevicePointer
    assert args(2, 3, p[0], None, p[2], p[3]) == E.cudaErrorInvalidDevicePointer
    assert args(1, 2, None, None, None, None) == 0             # interior plane: no face buffer needed
    assert args(0, 1, p[0], p[1], b.data_ptr(), p[3]) == E.cudaErrorInvalidValue  # send overlaps the output
    torch.cuda.synchronize()


REACTIVE_CASES = [("D3Q19", "float", "TRT", (16, 6, 6)), ("D3Q19", "double", "MRT", (8, 4, 6)),
                  ("D3Q27", "float", "BGK", (8, 4, 6))]


def _reactive_state(lat, dt, dims, seed):
    nx, ny, nz = dims
    f = U.random_state(lat, nx, ny, nz, dt, seed=seed)
    a = U.random_scalar("D3Q7", nx, ny, nz, dt, seed=seed + 1)
    b = U.random_scalar("D3Q7", nx, ny, nz, dt, seed=seed + 2)
    return f, a, b


@pytest.mark.parametrize("lat,dn,op,dims", REACTIVE_CASES)
@pytest.mark.parametrize("world", [1, 2, 3])
def test_coupled_slabs_match_whole_box(engine, dev, lat, dn, op, dims, world):
    """The coupled fluid + A + B -> C step as slabs (face buffers carrying the
    fluid's crossing populations and one D3Q7 plane per species) is
    bit-identical to the whole box stepped with lbm_fluid_reaction_ab_async, and
    the statistics from the ranks' summed partials equal the whole box's: bit
    for bit on one rank, to 1e-12 across ranks (the sums are added in another
    order)."""
    nx, ny, nz = dims
    dt = np.float32 if dn == "float" else np.float64
    steps, omega, omega_c, k = 6, 1 / 0.6, 1 / 0.8, 0.3
    f, a, b = _reactive_state(lat, dt, dims, seed=31)
    whole = [torch.from_numpy(x).to(dev) for x in (f, a, b)]
    wnext = [torch.empty_like(x) for x in whole]
    pb = E.stats_partials_bytes(lat, nx, ny, nz)
    part = torch.empty(pb // 8, dtype=torch.float64, device=dev)
    want_stats = torch.empty(8, dtype=torch.float64, device=dev)
    for s in range(steps):
        last = s == steps - 1
        E.check(E.fluid_reaction_ab_async(lat, dn, op, whole[0], wnext[0], whole[1], wnext[1], whole[2], wnext[2],
                                          nx, ny, nz, omega, omega_c, k, part if last else None, pb if last else 0))
        whole, wnext = wnext, whole
    E.check(E.reactive_stats_finalize_async(lat, dn, nx, ny, nz, k, part, pb, want_stats))

    doms = [slab.ReactiveSlabDomain(torch, lat, dn, op, nx, ny, nz, omega, omega_c, k, r, world, dev)
            for r in range(world)]
    q = E.Q_OF[lat]

    def split(x, qq):
        x4 = x.reshape(qq, nz, ny, nx)
        return [torch.from_numpy(np.ascontiguousarray(x4[:, d.z0:d.z0 + d.nz])).to(dev) for d in doms]

    cur = list(zip(split(f, q), split(a, 7), split(b, 7)))
    nxt = [tuple(torch.empty_like(t) for t in c) for c in cur]
    ex = slab.LocalExchange(doms)
    for d, c in zip(doms, cur):
        d.pack(c)
    ex.exchange_all()
    for s in range(steps):
        for d, c, n in zip(doms, cur, nxt):
            d.compute(c, n, stats=s == steps - 1)
        ex.exchange_all()
        cur, nxt = nxt, cur
    sums = sum(d.rank_sums() for d in doms) if world > 1 else doms[0].rank_sums()
    got_stats = slab.diagnostics_from_sums(torch, dn, sums, nx * ny * nz, k)
    torch.cuda.synchronize()
    for idx, (qq, ref) in enumerate(((q, whole[0]), (7, whole[1]), (7, whole[2]))):
        got = np.concatenate([c[idx].cpu().numpy() for c in cur], axis=1).reshape(qq, -1)
        assert U.same_bits(got, ref.cpu().numpy().reshape(qq, -1)), ("fluid", "A", "B")[idx]
    g, w = got_stats.cpu().numpy(), want_stats.cpu().numpy()
    if world == 1:
        assert U.same_bits(g, w)
    else:
        assert np.all(np.abs(g - w) <= 1e-12 * np.maximum(np.abs(w), 1e-300)), (g, w)


CASES16 = [("D3Q19", "f16s", "TRT", (32, 6, 8)), ("D3Q19", "q15s", "MRT", (16, 4, 8)),
           ("D3Q19", "bf16s", "BGK", (12, 4, 4)), ("D3Q27", "e3m12s", "TRT", (16, 4, 4)),
           ("D3Q19", "f16s", "RLBM", (16, 4, 4))]


@pytest.mark.parametrize("lat,fmt,op,dims", CASES16)
@pytest.mark.parametrize("world", [1, 2, 4])
def test_16bit_slabs_match_whole_box(engine, dev, lat, fmt, op, dims, world):
    """16-bit storage (lbm_step_slab_shifted_async, face buffers of codes):
    the slabs give the codes of the whole box stepped with
    lbm_step_shifted_async, bit for bit. Rows of a multiple of 8 cells run the
    row-staged kernel on every plane (its copies read the halo rows at the
    faces); 12-cell rows and the operators that decode to populations run the
    vectorised kernel and its SLAB form."""
    nx, ny, nz = dims
    steps = 6
    f = torch.from_numpy(U.random_state(lat, nx, ny, nz, np.float32, seed=23)).to(dev)
    Q = f.shape[0]
    h = torch.empty(f.shape, dtype=torch.int16, device=dev)
    E.check(E.encode_shifted_async(lat, fmt, "float", f, h, nx, ny, nz, 1.0))
    a, b = h.clone(), torch.empty_like(h)
    for _ in range(steps):
        E.check(E.step_shifted_async(lat, fmt, op, a, b, nx, ny, nz, 1 / 0.6, 1.0))
        a, b = b, a
    torch.cuda.synchronize()
    want = a.cpu().numpy().reshape(Q, -1)
    h4 = h.view(Q, nz, ny, nx)
    doms = [slab.SlabDomain(torch, lat, "float", op, nx, ny, nz, 1 / 0.6, r, world, dev, storage=fmt)
            for r in range(world)]
    cur = [h4[:, d.z0:d.z0 + d.nz].contiguous() for d in doms]
    nxt = [torch.empty_like(c) for c in cur]
    ex = slab.LocalExchange(doms)
    for d, c in zip(doms, cur):
        d.pack(c)
    ex.exchange_all()
    for _ in range(steps):
        for d, c, n in zip(doms, cur, nxt):
            d.compute(c, n)
        ex.exchange_all()
        cur, nxt = nxt, cur
    assert E.stage_timeouts(reset=True) == 0
    torch.cuda.synchronize()
    got = np.concatenate([c.cpu().numpy() for c in cur], axis=1).reshape(Q, -1)
    assert np.array_equal(got, want)

"""GPU: the engine's kernels, called through the C ABI, against the CPU oracle.

Parity bars (floating point, stated per test):
* fluid collide-stream, scalar step, equilibrium init, fused fluid step:
  bit-identical to the oracle (which is bit-identical to the reference build);
* steps that call exp() (the A + B -> C source): relative L2 <= 1e-13 (double)
  and <= 1e-5 (float) after the given number of steps. CUDA's exp and glibc's
  may differ in the last bit, and the source's denominator b - a e^{-k(b-a)}
  cancels, so a one-ulp difference in a few cells grows to ~1e-6 in the field;
* FP64-accumulated statistics: relative error <= 1e-12 per field against the
  oracle's FP64-accumulated sums.
"""
import math

import numpy as np
import pytest
import torch

import _util as U
import oracle as O

pytestmark = pytest.mark.gpu

LATS = ("D2Q9", "D3Q19", "D3Q27")
OPS = ("BGK", "TRT", "MRT", "RLBM")
REALS = {"float": np.float32, "double": np.float64}
# odd extents (no tile multiple) and an x-extent above one block (128)
SIZES = {"D2Q9": [(37, 23, 1), (150, 3, 1)], "D3Q19": [(13, 11, 7), (150, 3, 2)],
         "D3Q27": [(9, 7, 5), (131, 2, 3)]}


FUSED_SIZES = {"D2Q9": [(37, 23, 1), (150, 3, 1)], "D3Q19": [(13, 11, 7), (150, 3, 2)],
               "D3Q27": [(9, 7, 5), (64, 3, 2)]}


def _run_steps(E, lat, real, op, f0, nx, ny, nz, omega, steps, dev):
    cur = torch.from_numpy(f0).to(dev)
    nxt = torch.empty_like(cur)
    for _ in range(steps):
        E.check(E.launch_step_gpu(lat, real, op, cur, nxt, nx, ny, nz, omega))
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    return cur.cpu().numpy()


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("real", ["float", "double"])
@pytest.mark.parametrize("op", OPS)
def test_step_bitwise(engine, dev, lat, real, op):
    for k, (nx, ny, nz) in enumerate(SIZES[lat]):
        f0 = U.random_state(lat, nx, ny, nz, REALS[real], seed=100 + k)
        got = _run_steps(engine, lat, real, op, f0, nx, ny, nz, 1 / 0.6, 5, dev)
        want = O.step(f0, lat, op, nx, ny, nz, 1 / 0.6, steps=5)
        assert U.same_bits(got, want), f"{lat} {real} {op} {nx}x{ny}x{nz}: max |d| {np.abs(got - want).max()}"


@pytest.mark.parametrize("scale", [1e-24, 1e-33, 1e-38, 1e-42])
def test_d3q27_mrt_float_tiny_states_bitwise(engine, dev, scale):
    """D3Q27 MRT in FP32 divides by 3 and 6 without a division instruction and
    falls back to IEEE division for a cell whose dividends come near the
    subnormal range. Every other x cell is scaled down (1e-24 keeps nearly all
    cells on the fast path, 1e-33 .. 1e-42 send them to the fallback, the last
    with subnormal populations), so warps mix both paths; five steps stream
    tiny and normal populations into the same cells. Bit-identical throughout."""
    nx, ny, nz = 40, 7, 5
    f0 = U.random_state("D3Q27", nx, ny, nz, np.float32, seed=31).reshape(27, nz, ny, nx)
    f0[..., ::2] *= np.float32(scale)
    f0 = np.ascontiguousarray(f0.reshape(27, -1))
    got = _run_steps(engine, "D3Q27", "float", "MRT", f0, nx, ny, nz, 1 / 0.6, 5, dev)
    want = O.step(f0, "D3Q27", "MRT", nx, ny, nz, 1 / 0.6, steps=5)
    assert U.same_bits(got, want), f"max |d| {np.abs(got - want).max()}"


@pytest.mark.parametrize("real", ["float", "double"])
def test_d3q27_mrt_nonfinite_cells(engine, dev, real):
    """Cells holding an infinite or NaN population (a blown-up run): the FP32
    fast transform hands them to the IEEE fallback, so inf and NaN land where
    the reference puts them; the finite cells stay bit-identical."""
    nx, ny, nz = 9, 7, 5
    f0 = U.random_state("D3Q27", nx, ny, nz, REALS[real], seed=32)
    f0[3, 10] = np.inf
    f0[0, 40] = -np.inf
    f0[12, 77] = np.nan
    got = _run_steps(engine, "D3Q27", real, "MRT", f0, nx, ny, nz, 1 / 0.6, 1, dev)
    want = O.step(f0, "D3Q27", "MRT", nx, ny, nz, 1 / 0.6, steps=1)
    assert U.same_bits(got, want)


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("real", ["float", "double"])
def test_rlbm_tiny_and_nonfinite_cells_bitwise(engine, dev, lat, real):
    """RLBM on cells scaled to tiny and subnormal magnitudes (some products
    underflow to zero, so signed zeros meet in the sums) and on cells holding
    an infinite or NaN population (a blown-up run): bit-identical to the
    reference, NaN where it has NaN."""
    nx, ny, nz = SIZES[lat][0]
    f0 = U.random_state(lat, nx, ny, nz, REALS[real], seed=41)
    n = U.cells(lat, nx, ny, nz)
    tiny = np.float32(1e-36) if real == "float" else np.float64(1e-300)
    f0[:, 0:n:3] *= tiny
    f0[2, 7] = np.inf
    f0[0, 11] = -np.inf
    f0[5, 13] = np.nan
    got = _run_steps(engine, lat, real, "RLBM", f0, nx, ny, nz, 1 / 0.6, 1, dev)
    want = O.step(f0, lat, "RLBM", nx, ny, nz, 1 / 0.6, steps=1)
    assert U.same_bits(got, want)


def test_tgv_d3q19_fp64_bgk_64cube(engine, dev):
    """The C1 workload shape: D3Q19 BGK FP64 64^3 Taylor-Green (u0 0.05, rho 1,
    tau 0.6), 100 steps, bit-identical; KE decays."""
    n = 64
    k = 2 * math.pi / n
    x = np.arange(n, dtype=np.float64)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.stack([0.05 * np.sin(k * X) * np.cos(k * Y) * np.cos(k * Z),
                  -0.05 * np.cos(k * X) * np.sin(k * Y) * np.cos(k * Z),
                  np.zeros_like(X)]).reshape(3, -1)
    f0 = O.init_equilibrium("D3Q19", np.ones(n ** 3), u, n, n, n)
    got = _run_steps(engine, "D3Q19", "double", "BGK", f0, n, n, n, 1 / 0.6, 100, dev)
    want = O.step(f0, "D3Q19", "BGK", n, n, n, 1 / 0.6, steps=100)
    assert U.same_bits(got, want)
    _, u1 = O.macro_fields(got, "D3Q19", n, n, n)
    assert (u1 ** 2).sum() < (u ** 2).sum()


def test_step_async_matches_reference_launcher(engine, dev):
    nx, ny, nz = 40, 12, 6
    f0 = U.random_state("D3Q19", nx, ny, nz, np.float32, seed=5)
    a = torch.from_numpy(f0).to(dev)
    b1, b2 = torch.empty_like(a), torch.empty_like(a)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        engine.check(engine.step_async("D3Q19", torch.float32, "MRT", a, b1, nx, ny, nz, 1.7, stream=s))
    s.synchronize()
    engine.check(engine.launch_step_gpu("D3Q19", "float", "MRT", a, b2, nx, ny, nz, 1.7))
    torch.cuda.synchronize()
    assert torch.equal(b1, b2)


def test_2d_z_extent_forced_to_one(engine, dev):
    """For D==2 the reference forces z_extent = 1 (src/lattice_cuda.cu:496-499):
    a 2D launch with z_extent 0 or 5 behaves as z_extent 1."""
    nx, ny = 17, 9
    f0 = U.random_state("D2Q9", nx, ny, 1, np.float64, seed=9)
    want = O.step(f0, "D2Q9", "TRT", nx, ny, 1, 1.3)
    for nz in (0, 5):
        cur = torch.from_numpy(f0).to(dev)
        nxt = torch.empty_like(cur)
        assert engine.launch_step_gpu("D2Q9", "double", "TRT", cur, nxt, nx, ny, nz, 1.3) == 0
        torch.cuda.synchronize()
        assert U.same_bits(nxt.cpu().numpy(), want)


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("real", ["float", "double"])
def test_scalar_step_bitwise(engine, dev, lat, real):
    nx, ny, nz = SIZES[lat][0]
    sl = O.SCALAR_OF[lat]
    f = U.random_state(lat, nx, ny, nz, REALS[real], seed=21)
    g0 = U.random_scalar(sl, nx, ny, nz, REALS[real], seed=22)
    tf = torch.from_numpy(f).to(dev)
    cur = torch.from_numpy(g0).to(dev)
    nxt = torch.empty_like(cur)
    for _ in range(4):
        engine.check(engine.launch_scalar_step_gpu(lat, real, cur, nxt, tf, nx, ny, nz, 1 / 0.8, 2e-3))
        cur, nxt = nxt, cur
    torch.cuda.synchronize()
    want = O.scalar_step(g0, f, lat, nx, ny, nz, 1 / 0.8, 2e-3, steps=4)
    assert U.same_bits(cur.cpu().numpy(), want)


def _reaction_tol(real):
    return 1e-13 if real == "double" else 1e-5


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("real", ["float", "double"])
def test_reaction_ab(engine, dev, lat, real):
    nx, ny, nz = SIZES[lat][0]
    sl = O.SCALAR_OF[lat]
    dt = REALS[real]
    f = U.random_state(lat, nx, ny, nz, dt, seed=31)
    a0 = U.random_scalar(sl, nx, ny, nz, dt, seed=32)
    b0 = U.random_scalar(sl, nx, ny, nz, dt, seed=33)
    tf = torch.from_numpy(f).to(dev)
    ta, tb = torch.from_numpy(a0).to(dev), torch.from_numpy(b0).to(dev)
    na, nb = torch.empty_like(ta), torch.empty_like(tb)
    for _ in range(5):
        engine.check(engine.launch_reaction_AB_gpu(lat, real, ta, na, tb, nb, tf, nx, ny, nz, 1 / 0.8, 0.05))
        ta, na, tb, nb = na, ta, nb, tb
    torch.cuda.synchronize()
    wa, wb = O.reaction_ab(a0, b0, f, lat, nx, ny, nz, 1 / 0.8, 0.05, steps=5)
    assert U.rel_l2(ta.cpu().numpy(), wa) <= _reaction_tol(real)
    assert U.rel_l2(tb.cpu().numpy(), wb) <= _reaction_tol(real)


def test_reaction_equal_species_branch_bitwise(engine, dev):
    """A == B everywhere takes the exp-free branch A/(1+kA) (lattice_physics.hpp:726-729):
    bit-identical, and it matches the batch solution C0/(1+C0 k t) (test_validation.cpp:1655-1702)."""
    nx = ny = 16
    n = nx * ny
    fl = O.init_equilibrium("D2Q9", np.ones(n), np.zeros((2, n)), nx, ny, 1)
    g = O.init_equilibrium("D2Q5", np.ones(n), np.zeros((2, n)), nx, ny, 1)
    tf = torch.from_numpy(fl).to(dev)
    ta, tb = torch.from_numpy(g).to(dev), torch.from_numpy(g.copy()).to(dev)
    na, nb = torch.empty_like(ta), torch.empty_like(tb)
    for _ in range(200):
        engine.check(engine.launch_reaction_AB_gpu("D2Q9", "double", ta, na, tb, nb, tf, nx, ny, 1, 1 / 0.8, 0.005))
        ta, na, tb, nb = na, ta, nb, tb
    torch.cuda.synchronize()
    wa, _ = O.reaction_ab(g, g, fl, "D2Q9", nx, ny, 1, 1 / 0.8, 0.005, steps=200)
    assert U.same_bits(ta.cpu().numpy(), wa)
    assert abs(ta[:, 0].sum().item() - 1.0 / (1.0 + 0.005 * 200)) <= 1e-4


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("real", ["float", "double"])
@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT"])
@pytest.mark.parametrize("size", [0, 1])
def test_fused_fluid_reaction(engine, dev, lat, real, op, size):
    """One fused launch == the reference driver's two launches
    (src/simulate_reaction.cpp:518-543): fluid bit-identical to the oracle,
    scalars bit-identical to the engine's own two-launch sequence and within
    the exp tolerance of the oracle's coupled loop; at two extents (odd and
    even x)."""
    nx, ny, nz = FUSED_SIZES[lat][size]
    sl = O.SCALAR_OF[lat]
    dt = REALS[real]
    f0 = U.random_state(lat, nx, ny, nz, dt, seed=41)
    a0 = U.random_scalar(sl, nx, ny, nz, dt, seed=42)
    b0 = U.random_scalar(sl, nx, ny, nz, dt, seed=43)
    om, omc, k, steps = 1 / 0.6, 1 / 0.8, 0.05, 4

    tf, ta, tb = (torch.from_numpy(x).to(dev) for x in (f0, a0, b0))
    nf, na, nb = (torch.empty_like(x) for x in (tf, ta, tb))
    for _ in range(steps):
        engine.check(engine.fluid_reaction_ab_async(lat, real, op, tf, nf, ta, na, tb, nb, nx, ny, nz, om, omc, k))
        tf, nf, ta, na, tb, nb = nf, tf, na, ta, nb, tb
    # the two-launch sequence, as the reference driver issues it
    sf, sa, sb = (torch.from_numpy(x).to(dev) for x in (f0, a0, b0))
    mf, ma, mb = (torch.empty_like(x) for x in (sf, sa, sb))
    for _ in range(steps):
        engine.check(engine.launch_step_gpu(lat, real, op, sf, mf, nx, ny, nz, om))
        sf, mf = mf, sf
        engine.check(engine.launch_reaction_AB_gpu(lat, real, sa, ma, sb, mb, sf, nx, ny, nz, omc, k))
        sa, ma, sb, mb = ma, sa, mb, sb
    torch.cuda.synchronize()
    assert torch.equal(tf, sf) and torch.equal(ta, sa) and torch.equal(tb, sb)
    wf, wa, wb = O.coupled_reaction(f0, a0, b0, lat, op, nx, ny, nz, om, omc, k, steps=steps)
    assert U.same_bits(tf.cpu().numpy(), wf)
    assert U.rel_l2(ta.cpu().numpy(), wa) <= _reaction_tol(real)
    assert U.rel_l2(tb.cpu().numpy(), wb) <= _reaction_tol(real)


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("real", ["float", "double"])
def test_reactive_stats(engine, dev, lat, real):
    nx, ny, nz = SIZES[lat][1]
    sl = O.SCALAR_OF[lat]
    dt = REALS[real]
    a = U.random_scalar(sl, nx, ny, nz, dt, seed=51)
    b = U.random_scalar(sl, nx, ny, nz, dt, seed=52)
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    nbytes = engine.stats_partials_bytes(lat, nx, ny, nz)
    part = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
    out = torch.empty(8, dtype=torch.float64, device=dev)
    engine.check(engine.reactive_stats_async(sl, real, ta, tb, nx, ny, nz, 0.03, part, nbytes, out))
    torch.cuda.synchronize()
    want = O.reactive_stats(a, b, sl, nx, ny, nz, 0.03, accumulate_f64=True)
    got = out.cpu().numpy()
    for name, g, w in zip(O.STATS_FIELDS, got, want):
        assert abs(g - w) <= 1e-12 * max(abs(w), 1e-6), name
    # deterministic run to run
    out2 = torch.empty_like(out)
    engine.check(engine.reactive_stats_async(sl, real, ta, tb, nx, ny, nz, 0.03, part, nbytes, out2))
    torch.cuda.synchronize()
    assert torch.equal(out, out2)


@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19"])
def test_fused_stats_epilogue(engine, dev, lat):
    """Statistics accumulated inside the fused launch equal a separate
    statistics pass over the fields that launch wrote."""
    nx, ny, nz = SIZES[lat][1]
    sl = O.SCALAR_OF[lat]
    f0 = U.random_state(lat, nx, ny, nz, np.float32, seed=61)
    a0 = U.random_scalar(sl, nx, ny, nz, np.float32, seed=62)
    b0 = U.random_scalar(sl, nx, ny, nz, np.float32, seed=63)
    tf, ta, tb = (torch.from_numpy(x).to(dev) for x in (f0, a0, b0))
    nf, na, nb = (torch.empty_like(x) for x in (tf, ta, tb))
    nbytes = engine.stats_partials_bytes(lat, nx, ny, nz)
    part = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
    d1 = torch.empty(8, dtype=torch.float64, device=dev)
    d2 = torch.empty_like(d1)
    engine.check(engine.fluid_reaction_ab_async(lat, "float", "TRT", tf, nf, ta, na, tb, nb, nx, ny, nz,
                                                1 / 0.6, 1 / 0.8, 0.05, part, nbytes))
    engine.check(engine.reactive_stats_finalize_async(lat, "float", nx, ny, nz, 0.05, part, nbytes, d1))
    engine.check(engine.reactive_stats_async(sl, "float", na, nb, nx, ny, nz, 0.05, part, nbytes, d2))
    torch.cuda.synchronize()
    assert torch.equal(d1, d2)


@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19", "D3Q27", "D2Q5", "D3Q7"])
@pytest.mark.parametrize("real", ["float", "double"])
def test_init_equilibrium_bitwise(engine, dev, lat, real):
    nx, ny, nz = (19, 6, 1) if O.D_OF[lat] == 2 else (9, 6, 5)
    n = U.cells(lat, nx, ny, nz)
    rng = np.random.default_rng(71)
    dt = REALS[real]
    rho = (1 + 0.05 * rng.standard_normal(n)).astype(dt)
    u = (0.04 * rng.standard_normal((O.D_OF[lat], n))).astype(dt)
    out = torch.empty((O.Q_OF[lat], n), dtype=torch.float32 if real == "float" else torch.float64, device=dev)
    engine.check(engine.init_equilibrium_async(lat, real, torch.from_numpy(rho).to(dev),
                                               torch.from_numpy(u).to(dev), out, nx, ny, nz))
    torch.cuda.synchronize()
    want = O.init_equilibrium(lat, rho.astype(np.float64), u.astype(np.float64), nx, ny, nz, dt)
    assert U.same_bits(out.cpu().numpy(), want)

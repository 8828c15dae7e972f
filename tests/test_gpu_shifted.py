"""GPU: shifted 16-bit population storage (FP16 / BF16 / E3M12 / Q15) with FP32 collision.

* encode/decode round trip: the error of every population is within half a
  16-bit ulp of its stored deviation (f/w - rho0);
* one 16-bit step against encode(FP32 step(decode(h))): the two differ only in
  FP32 rounding before the final 16-bit rounding (BGK/TRT collide on the
  deviations; the FP32 path works on f ~ w and carries a few FP32 ulps of 1 of
  absolute error in f/w after cancelling rho0, more for D3Q27's 1/216 weights
  and 27-term MRT sums), so every value is within one 16-bit step plus 2e-6
  of the other; with nearest rounding at least 95 % of the codes agree, and
  where FP16 / BF16 round stochastically every value is one of the two 16-bit
  neighbours of the FP32 result with an average signed error of 0;
* Q15 covers |f/w - rho0| < 1 only, so its round trip uses a state inside
  that range (|u| ~ 0.03) and out-of-range values saturate;
* 2000 steps of the D3Q19 256^3 Taylor-Green + noise case (tau 0.55): the
  velocity rel-L2 against the FP64 run (the FP64 kernel is bit-identical to
  the reference CPU path, tests/test_gpu_parity.py), held to the 1e-3 target
  for every format that meets it: E3M12 (1.0e-4 / 8.4e-5 measured), IEEE FP16
  with stochastic rounding (3.7e-4 TRT, 3.5e-4 MRT; 1.96e-3 TRT with nearest
  rounding, whose correlated errors TRT's slowly relaxed odd modes keep) and
  Q15 for TRT (2.6e-4); Q15 MRT <= 3e-3 (1.45e-3 measured); BF16 <= 0.15
  (8-bit significand).
"""
import math

import numpy as np
import pytest
import torch

import _util as U
import oracle as O

pytestmark = pytest.mark.gpu

FMTS = ("f16s", "bf16s", "e3m12s", "q15s")
ULP = {"f16s": 2.0 ** -10, "bf16s": 2.0 ** -7, "e3m12s": 2.0 ** -12, "q15s": 0.0}  # relative spacing
ABS_FLOOR = {"f16s": 0.0, "bf16s": 0.0, "e3m12s": 2.0 ** -18, "q15s": 2.0 ** -16}  # half the uniform grid
BARS = {("e3m12s", "TRT"): 1e-3, ("e3m12s", "MRT"): 1e-3, ("f16s", "MRT"): 1e-3,
        ("f16s", "TRT"): 1e-3, ("bf16s", "TRT"): 0.15, ("bf16s", "MRT"): 0.15,
        ("q15s", "TRT"): 1e-3, ("q15s", "MRT"): 3e-3}


def _w(lat):
    import lbcube  # noqa: F401

    return torch.tensor({"D2Q9": [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4,
                         "D3Q19": [1 / 3] + [1 / 18] * 6 + [1 / 36] * 12,
                         "D3Q27": [8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8}[lat],
                        dtype=torch.float64)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19", "D3Q27"])
def test_encode_decode_round_trip(engine, dev, fmt, lat):
    nx, ny, nz = (64, 12, 1) if lat == "D2Q9" else (32, 6, 5)
    u_amp = 0.03 if fmt == "q15s" else 0.08
    f = torch.from_numpy(U.random_state(lat, nx, ny, nz, np.float32, seed=5, u_amp=u_amp)).to(dev)
    h = torch.empty(f.shape, dtype=torch.int16, device=dev)
    back = torch.empty_like(f)
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f, h, nx, ny, nz, 1.0))
    engine.check(engine.decode_shifted_async(lat, fmt, "float", h, back, nx, ny, nz, 1.0))
    torch.cuda.synchronize()
    w = _w(lat).to(dev).view(-1, 1)
    dev_in = f.double() / w - 1.0
    err = (back.double() - f.double()).abs() / w
    # half an ulp of the stored deviation (x2 for the binade), the E3M12 uniform-grid floor, FP32 arithmetic
    bound = 0.5 * ULP[fmt] * dev_in.abs() * 2 + ABS_FLOOR[fmt] + 1e-7
    assert bool((err <= bound).all()), float((err - bound).max())


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19", "D3Q27", "D3Q7"])
def test_encode_decode_vector_path_matches_scalar_path(engine, dev, fmt, lat):
    """FP32 fields with planes of a multiple of 4 cells in 16-byte aligned buffers
    convert four cells per thread; any other layout one cell per thread. The
    same field converted both ways (the second copy one element off the
    alignment) gives the same codes and the same decoded values, bit for bit."""
    nx, ny, nz = (64, 12, 1) if lat == "D2Q9" else (32, 6, 5)
    q = {"D2Q9": 9, "D3Q19": 19, "D3Q27": 27, "D3Q7": 7}[lat]
    n = nx * ny * nz
    if lat == "D3Q7":
        f = torch.from_numpy(U.random_scalar(lat, nx, ny, nz, np.float32, seed=6)).to(dev)
        ref = 0.5
    else:
        f = torch.from_numpy(U.random_state(lat, nx, ny, nz, np.float32, seed=6, u_amp=0.03)).to(dev)
        ref = 1.0
    f = f.reshape(q, n)
    f_off = torch.empty(q * n + 1, dtype=torch.float32, device=dev)[1:].view(q, n)  # 4 bytes off
    f_off.copy_(f)
    h = torch.empty((q, n), dtype=torch.int16, device=dev)
    h_off = torch.empty(q * n + 1, dtype=torch.int16, device=dev)[1:].view(q, n)  # 2 bytes off
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f, h, nx, ny, nz, ref))
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f_off, h_off, nx, ny, nz, ref))
    back = torch.empty_like(f)
    back_off = torch.empty(q * n + 1, dtype=torch.float32, device=dev)[1:].view(q, n)
    engine.check(engine.decode_shifted_async(lat, fmt, "float", h, back, nx, ny, nz, ref))
    engine.check(engine.decode_shifted_async(lat, fmt, "float", h_off, back_off, nx, ny, nz, ref))
    torch.cuda.synchronize()
    assert torch.equal(h, h_off)
    assert torch.equal(back.view(torch.int32), back_off.contiguous().view(torch.int32))


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19", "D3Q27"])
@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT", "RLBM"])
def test_shifted_step_is_rounded_fp32_step(engine, dev, fmt, lat, op):
    nx, ny, nz = (64, 12, 1) if lat == "D2Q9" else (32, 6, 5)
    f = torch.from_numpy(U.random_state(lat, nx, ny, nz, np.float32, seed=6)).to(dev)
    h0 = torch.empty(f.shape, dtype=torch.int16, device=dev)
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f, h0, nx, ny, nz, 1.0))
    f0 = torch.empty_like(f)
    engine.check(engine.decode_shifted_async(lat, fmt, "float", h0, f0, nx, ny, nz, 1.0))
    f1 = torch.empty_like(f)
    engine.check(engine.launch_step_gpu(lat, "float", op, f0, f1, nx, ny, nz, 1 / 0.6))
    want = torch.empty_like(h0)
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f1, want, nx, ny, nz, 1.0))
    h1 = torch.empty_like(h0)
    engine.check(engine.step_shifted_async(lat, fmt, op, h0, h1, nx, ny, nz, 1 / 0.6, 1.0))
    got_f, want_f = torch.empty_like(f), torch.empty_like(f)
    engine.check(engine.decode_shifted_async(lat, fmt, "float", h1, got_f, nx, ny, nz, 1.0))
    engine.check(engine.decode_shifted_async(lat, fmt, "float", want, want_f, nx, ny, nz, 1.0))
    torch.cuda.synchronize()
    w = _w(lat).to(dev).view(-1, 1)
    dv = (got_f.double() - want_f.double()).abs() / w
    step = ULP[fmt] * (want_f.double() / w - 1.0).abs() * 2 + 2 * ABS_FLOOR[fmt] + 2e-6
    assert bool((dv <= step).all()), float((dv - step).max())
    if _stochastic(fmt, lat, op):
        # each value one of the two 16-bit neighbours of the FP32 result, and
        # no bias: the signed error, in units of the local spacing, averages 0.
        # Checked where the spacing is 10x the FP32 paths' 2e-6 disagreement.
        exact = f1.double() / w - 1.0
        spacing = ULP[fmt] * torch.exp2(torch.floor(torch.log2(exact.abs().clamp_min(1e-30))))
        e = ((got_f.double() / w - 1.0 - exact) / spacing)[spacing >= 2e-5]
        assert e.numel() >= 500
        assert float(e.abs().max()) <= 1.2
        assert abs(float(e.mean())) <= 0.05, float(e.mean())
    else:
        assert float((h1 == want).double().mean()) >= 0.95


def _stochastic(fmt, lat, op):
    """The step rounds FP16 / BF16 stochastically wherever it collides on the
    deviations (BGK, TRT; MRT on D2Q9 / D3Q19)."""
    return fmt in ("f16s", "bf16s") and (op in ("BGK", "TRT") or (op == "MRT" and lat != "D3Q27"))


@pytest.mark.parametrize("nx", [512, 1024])
@pytest.mark.parametrize("fmt,op", [("f16s", "TRT"), ("q15s", "MRT")])
def test_shifted_step_wide_rows(engine, dev, nx, fmt, op):
    """Rows of 512 and 1024 cells: the row-staged D3Q19 kernel then holds 58 KB and
    117 KB of shared memory (more than the 48 KB default). One step is the
    rounded FP32 step to the bound above, and a second run gives the same bits."""
    lat, ny, nz = "D3Q19", 4, 3
    f = torch.from_numpy(U.random_state(lat, nx, ny, nz, np.float32, seed=12)).to(dev)
    h0 = torch.empty(f.shape, dtype=torch.int16, device=dev)
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f, h0, nx, ny, nz, 1.0))
    f0 = torch.empty_like(f)
    engine.check(engine.decode_shifted_async(lat, fmt, "float", h0, f0, nx, ny, nz, 1.0))
    f1 = torch.empty_like(f)
    engine.check(engine.launch_step_gpu(lat, "float", op, f0, f1, nx, ny, nz, 1 / 0.6))
    want_f = torch.empty_like(f)
    want = torch.empty_like(h0)
    engine.check(engine.encode_shifted_async(lat, fmt, "float", f1, want, nx, ny, nz, 1.0))
    engine.check(engine.decode_shifted_async(lat, fmt, "float", want, want_f, nx, ny, nz, 1.0))
    runs = []
    for _ in range(2):
        h1 = torch.full_like(h0, -1)
        engine.check(engine.step_shifted_async(lat, fmt, op, h0, h1, nx, ny, nz, 1 / 0.6, 1.0))
        runs.append(h1)
    assert engine.stage_timeouts(reset=True) == 0
    got_f = torch.empty_like(f)
    engine.check(engine.decode_shifted_async(lat, fmt, "float", runs[0], got_f, nx, ny, nz, 1.0))
    torch.cuda.synchronize()
    assert torch.equal(runs[0], runs[1])
    w = _w(lat).to(dev).view(-1, 1)
    dv = (got_f.double() - want_f.double()).abs().view(19, -1) / w
    step = ULP[fmt] * (want_f.double().view(19, -1) / w - 1.0).abs() * 2 + 2 * ABS_FLOOR[fmt] + 2e-6
    assert bool((dv <= step).all()), float((dv - step).max())


def test_shifted_rejects_unaligned_extent(engine, dev):
    h = torch.zeros((19, 4, 4, 30), dtype=torch.int16, device=dev)
    g = torch.empty_like(h)
    assert engine.step_shifted_async("D3Q19", "f16s", "TRT", h, g, 30, 4, 4, 1.5) == engine.cudaErrorInvalidValue


def _velocity(f, lat):
    c = torch.tensor(_CV[lat], dtype=f.dtype, device=f.device)
    rho = f.sum(0)
    u = torch.einsum("qd,q...->d...", c, f) / rho
    return rho, u


_CV = {"D3Q19": [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                 [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                 [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]]}


def tgv_noise_init(engine, dev, n, dtype):
    gen = torch.Generator(device=dev)
    gen.manual_seed(20261203)
    k = 2 * math.pi / n
    ax = torch.arange(n, device=dev, dtype=torch.float64) * k
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    u = torch.stack([0.05 * torch.sin(x) * torch.cos(y) * torch.cos(z),
                     -0.05 * torch.cos(x) * torch.sin(y) * torch.cos(z), torch.zeros_like(x)])
    u += 1e-3 * torch.randn(u.shape, generator=gen, device=dev, dtype=torch.float64)
    rho = torch.ones((n, n, n), device=dev, dtype=torch.float64)
    f = torch.empty((19, n, n, n), device=dev, dtype=dtype)
    real = "double" if dtype == torch.float64 else "float"
    engine.check(engine.init_equilibrium_async("D3Q19", real, rho.to(dtype), u.to(dtype).contiguous(), f, n, n, n))
    return f


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("op", ["TRT", "MRT"])
def test_shifted_2000_steps_vs_fp64(engine, dev, fmt, op):
    n, steps, tau = 256, 2000, 0.55
    f64 = tgv_noise_init(engine, dev, n, torch.float64)
    g64 = torch.empty_like(f64)
    f32 = f64.float()
    h = torch.empty(f32.shape, dtype=torch.int16, device=dev)
    engine.check(engine.encode_shifted_async("D3Q19", fmt, "float", f32, h, n, n, n, 1.0))
    del f32
    hg = torch.empty_like(h)
    for _ in range(steps):
        engine.check(engine.launch_step_gpu("D3Q19", "double", op, f64, g64, n, n, n, 1 / tau))
        f64, g64 = g64, f64
        engine.check(engine.step_shifted_async("D3Q19", fmt, op, h, hg, n, n, n, 1 / tau, 1.0))
        h, hg = hg, h
    del g64, hg
    fh = torch.empty((19, n, n, n), dtype=torch.float64, device=dev)
    engine.check(engine.decode_shifted_async("D3Q19", fmt, "double", h, fh, n, n, n, 1.0))
    torch.cuda.synchronize()
    _, u_ref = _velocity(f64, "D3Q19")
    _, u_h = _velocity(fh, "D3Q19")
    err = float(torch.linalg.vector_norm(u_h - u_ref) / torch.linalg.vector_norm(u_ref))
    print(f"{fmt} {op} velocity rel-L2 after {steps} steps: {err:.3e}")
    assert err <= BARS[(fmt, op)]


_SW = {"D2Q5": [1 / 3] + [1 / 6] * 4, "D3Q7": [1 / 4] + [1 / 8] * 6}


@pytest.mark.parametrize("fmt", ["f16s", "q15s"])
@pytest.mark.parametrize("fl", ["D2Q9", "D3Q19"])
@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT"])
def test_shifted_coupled_step_is_rounded_fp32_step(engine, dev, fmt, fl, op):
    """The 16-bit fluid + A + B -> C step against encode(FP32 coupled step(decode)):
    fluid and scalar values within one 16-bit step (+2e-6) of each other, at
    least 95 % of the codes equal."""
    sl = "D2Q5" if fl == "D2Q9" else "D3Q7"
    nx, ny, nz = (64, 12, 1) if fl == "D2Q9" else (32, 6, 5)
    f = torch.from_numpy(U.random_state(fl, nx, ny, nz, np.float32, seed=8)).to(dev)
    a = torch.from_numpy(U.random_scalar(sl, nx, ny, nz, np.float32, seed=9)).to(dev)
    b = torch.from_numpy(U.random_scalar(sl, nx, ny, nz, np.float32, seed=10)).to(dev)
    c0, k = 0.5, 0.3
    codes, exact = [], []
    for lat, t, ref in ((fl, f, 1.0), (sl, a, c0), (sl, b, c0)):
        h = torch.empty(t.shape, dtype=torch.int16, device=dev)
        engine.check(engine.encode_shifted_async(lat, fmt, "float", t, h, nx, ny, nz, ref))
        back = torch.empty_like(t)
        engine.check(engine.decode_shifted_async(lat, fmt, "float", h, back, nx, ny, nz, ref))
        codes.append(h)
        exact.append(back)
    nxt32 = [torch.empty_like(t) for t in exact]
    engine.check(engine.fluid_reaction_ab_async(fl, "float", op, exact[0], nxt32[0], exact[1], nxt32[1], exact[2],
                                                nxt32[2], nx, ny, nz, 1 / 0.6, 1 / 0.8, k))
    nxt16 = [torch.empty_like(h) for h in codes]
    engine.check(engine.fluid_reaction_ab_shifted_async(fl, fmt, op, codes[0], nxt16[0], codes[1], nxt16[1],
                                                        codes[2], nxt16[2], nx, ny, nz, 1 / 0.6, 1 / 0.8, k,
                                                        1.0, c0))
    for lat, t32, h16, ref in ((fl, nxt32[0], nxt16[0], 1.0), (sl, nxt32[1], nxt16[1], c0), (sl, nxt32[2], nxt16[2], c0)):
        want = torch.empty_like(h16)
        engine.check(engine.encode_shifted_async(lat, fmt, "float", t32, want, nx, ny, nz, ref))
        got_f, want_f = torch.empty_like(t32), torch.empty_like(t32)
        engine.check(engine.decode_shifted_async(lat, fmt, "float", h16, got_f, nx, ny, nz, ref))
        engine.check(engine.decode_shifted_async(lat, fmt, "float", want, want_f, nx, ny, nz, ref))
        torch.cuda.synchronize()
        w = (_w(lat) if lat == fl else torch.tensor(_SW[lat], dtype=torch.float64)).to(dev).view(-1, 1)
        dv = (got_f.double() - want_f.double()).abs() / w
        step = ULP[fmt] * (want_f.double() / w - ref).abs() * 2 + 2 * ABS_FLOOR[fmt] + 2e-6
        assert bool((dv <= step).all()), (lat, float((dv - step).max()))
        assert float((h16 == want).double().mean()) >= 0.95, lat

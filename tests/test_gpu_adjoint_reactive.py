"""GPU: the reactive-mixing adjoint (lbm_reactive_gradient_async) against
central finite differences of its own forward run, in FP64.

The coupled step is the fused fluid + A + B -> C launch (bit-identical to the
reference's two-launch sequence). Checked, for the mean-product objective
<C> = <A0> - <A> and the segregation intensity I_s, with BGK and TRT fluids:
dJ/dk, dJ/dtau, dJ/dtau_c and <dJ/dA0, d>, <dJ/dB0, d>, <dJ/du0, d> along seeded unit
directions, relative error <= 1e-6 plus the rounding noise of the
differences, 1e-13 |J| / h (central differences at h = 1e-3 and 5e-4 combined
by one Richardson step, error O(h^4)) (step count not a multiple of the
checkpoint interval, so a partial last segment is covered). J itself is
checked against a forward-only run through the public launchers. The FP32
gradient follows the FP64 one to the stated tolerances.
"""
import math

import pytest
import torch

import lbcube as E

pytestmark = pytest.mark.gpu

TAU, TAU_C, K = 0.8, 0.7, 0.6


def fields(fl, shape, dev, dtype, seed):
    """Smooth seeded u0 (amplitude 0.03), rho0 = 1, and A0, B0 in (0.1, 0.9)."""
    g = torch.Generator().manual_seed(seed)
    D = len(shape) if fl != "D2Q9" else 2
    axes = [torch.arange(n, dtype=torch.float64) * (2 * math.pi / n) for n in shape]
    grids = torch.meshgrid(*axes, indexing="ij")  # z, y, x (or y, x)
    def smooth():
        v = torch.zeros(shape, dtype=torch.float64)
        for _ in range(3):
            ks = torch.randint(0, 3, (len(shape),), generator=g).tolist()
            ph = float(torch.rand(1, generator=g)) * 2 * math.pi
            v += torch.cos(sum(k * x for k, x in zip(ks, grids)) + ph)
        return v / v.abs().max()
    u = torch.stack([0.03 * smooth() for _ in range(D)])
    a = 0.5 + 0.4 * smooth()
    b = 0.5 + 0.4 * smooth()
    rho = torch.ones(shape, dtype=torch.float64)
    return [t.to(device=dev, dtype=dtype).contiguous() for t in (rho, u, a, b)]


def gradient(fl, real, op, obj, rho, u, a, b, dims, steps, interval, tau=TAU, tau_c=TAU_C, k=K):
    nx, ny, nz = dims
    nb = E.reactive_gradient_workspace_bytes(fl, real, nx, ny, nz, steps, interval)
    ws = torch.empty(nb, dtype=torch.uint8, device=a.device)
    res = torch.zeros(4, dtype=torch.float64, device=a.device)
    ga, gb, gu = torch.empty_like(a), torch.empty_like(b), torch.empty_like(u)
    E.check(E.reactive_gradient_async(fl, real, op, obj, rho, u, a, b, nx, ny, nz, tau, tau_c, k, steps,
                                      interval, ws, nb, res, ga, gb, gu))
    torch.cuda.synchronize()
    gradient.last_u = gu
    return res.cpu().tolist(), ga, gb


def forward_objective(fl, real, op, obj, rho, u, a, b, dims, steps):
    """J from a forward-only run through the public launchers."""
    nx, ny, nz = dims
    sl = "D2Q5" if fl == "D2Q9" else "D3Q7"
    fq, sq = {"D2Q9": 9, "D3Q19": 19, "D3Q27": 27}[fl], (5 if fl == "D2Q9" else 7)
    shp = a.shape
    f = torch.empty((fq, *shp), dtype=a.dtype, device=a.device)
    sa, sb = torch.empty((sq, *shp), dtype=a.dtype, device=a.device), torch.empty((sq, *shp), dtype=a.dtype,
                                                                                   device=a.device)
    E.check(E.init_equilibrium_async(fl, real, rho, u, f, nx, ny, nz))
    E.check(E.init_equilibrium_async(sl, real, a, u, sa, nx, ny, nz))
    E.check(E.init_equilibrium_async(sl, real, b, u, sb, nx, ny, nz))
    f2, sa2, sb2 = torch.empty_like(f), torch.empty_like(sa), torch.empty_like(sb)
    for _ in range(steps):
        E.check(E.fluid_reaction_ab_async(fl, real, op, f, f2, sa, sa2, sb, sb2, nx, ny, nz, 1 / TAU,
                                          1 / TAU_C, K))
        f, f2, sa, sa2, sb, sb2 = f2, f, sa2, sa, sb2, sb
    if obj == "mean_product":
        return float(a.double().mean() - sa.double().sum(0).mean())
    part = torch.empty(E.stats_partials_bytes(fl, nx, ny, nz), dtype=torch.uint8, device=a.device)
    out = torch.empty(8, dtype=torch.float64, device=a.device)
    E.check(E.reactive_stats_async(sl, real, sa, sb, nx, ny, nz, K, part, part.numel(), out))
    return float(out[5])


CASES = [("D3Q19", (16, 12, 10)), ("D2Q9", (32, 24, 1))]


@pytest.mark.parametrize("fl,dims", CASES)
@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT"])
@pytest.mark.parametrize("obj", ["mean_product", "segregation"])
def test_reactive_gradient_central_differences_fp64(fl, dims, op, obj):
    dev = torch.device("cuda:0")
    nx, ny, nz = dims
    shape = (nz, ny, nx) if fl != "D2Q9" else (ny, nx)
    steps, interval = 23, 5
    rho, u, a, b = fields(fl, shape, dev, torch.float64, seed=11)
    (J, dk, dtau, dtc), ga, gb = gradient(fl, "double", op, obj, rho, u, a, b, dims, steps, interval)
    gu = gradient.last_u
    Jf = forward_objective(fl, "double", op, obj, rho, u, a, b, dims, steps)
    assert abs(J - Jf) <= 1e-12 * abs(Jf), (J, Jf)

    def Jat(**kw):
        kw2 = dict(tau=TAU, tau_c=TAU_C, k=K)
        aa, bb, uu = kw.pop("a", a), kw.pop("b", b), kw.pop("u", u)
        kw2.update(kw)
        return gradient(fl, "double", op, obj, rho, uu, aa, bb, dims, steps, interval, **kw2)[0][0]

    def richardson(J_of, h):
        """Central difference with one Richardson step (error O(h^4))."""
        d1 = (J_of(h) - J_of(-h)) / (2 * h)
        d2 = (J_of(h / 2) - J_of(-h / 2)) / h
        return (4 * d2 - d1) / 3

    def close(fd, ad, h):
        # 1e-6 relative, plus the rounding noise of a difference of two forward
        # runs: each J carries ~1e-13 |J| of accumulated FP64 rounding (tens of
        # roundings per population per step over all cells and steps)
        return abs(fd - ad) <= 1e-6 * max(abs(fd), abs(ad)) + 1e-13 * abs(J) / h

    h = 1e-3
    for name, x0, ad in (("k", K, dk), ("tau", TAU, dtau), ("tau_c", TAU_C, dtc)):
        fd = richardson(lambda e: Jat(**{name: x0 + e}), h)
        assert close(fd, ad, h / 2), (name, fd, ad)
    gen = torch.Generator().manual_seed(99)
    for field, grad in (("a", ga), ("b", gb), ("u", gu)):
        for _ in range(4 if field != "u" else 3):
            d = torch.randn(grad.shape, generator=gen, dtype=torch.float64).to(dev)
            d /= torch.linalg.vector_norm(d)
            base = {"a": a, "b": b, "u": u}[field]
            fd = richardson(lambda e: Jat(**{field: base + e * d}), h)
            ad = float((grad * d).sum())
            assert close(fd, ad, h / 2), (field, fd, ad)


def test_reactive_gradient_fp32_follows_fp64():
    dev = torch.device("cuda:0")
    dims, steps, interval = (32, 32, 32), 200, 50
    rho, u, a, b = fields("D3Q19", (32, 32, 32), dev, torch.float64, seed=5)
    r64, ga64, _ = gradient("D3Q19", "double", "TRT", "mean_product", rho, u, a, b, dims, steps, interval)
    r32, ga32, _ = gradient("D3Q19", "float", "TRT", "mean_product", rho.float(), u.float(), a.float(),
                            b.float(), dims, steps, interval)
    for q in range(4):
        assert abs(r32[q] - r64[q]) <= 2e-3 * abs(r64[q]) + 1e-9, (q, r32[q], r64[q])
    err = float(torch.linalg.vector_norm(ga32.double() - ga64) / torch.linalg.vector_norm(ga64))
    assert err <= 1e-3, err


@pytest.mark.parametrize("fmt", ["f16s", "q15s"])
def test_reactive_gradient_16bit_states_follow_fp32(fmt):
    """Forward in 16-bit shifted storage (fluid by 1, scalars by 0.5), adjoint in
    FP32 about the decoded states: J and the gradients follow the all-FP32 ones
    (bars: J 2e-3 relative, dJ/dk, dJ/dtau, dJ/dtau_c 3e-2, dJ/dA0 rel-L2 3e-2)."""
    dev = torch.device("cuda:0")
    dims, steps, interval = (32, 32, 32), 200, 50
    rho, u, a, b = fields("D3Q19", (32, 32, 32), dev, torch.float32, seed=5)
    r32, ga32, _ = gradient("D3Q19", "float", "TRT", "mean_product", rho, u, a, b, dims, steps, interval)
    nx, ny, nz = dims
    nb = E.reactive_gradient_workspace_bytes("D3Q19", "float", nx, ny, nz, steps, interval, storage=fmt)
    ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    res = torch.zeros(4, dtype=torch.float64, device=dev)
    ga = torch.empty_like(a)
    E.check(E.reactive_gradient_async("D3Q19", "float", "TRT", "mean_product", rho, u, a, b, nx, ny, nz, TAU, TAU_C,
                                      K, steps, interval, ws, nb, res, ga, storage=fmt, c0=0.5))
    torch.cuda.synchronize()
    r16 = res.tolist()
    assert abs(r16[0] - r32[0]) <= 2e-3 * abs(r32[0]), (r16[0], r32[0])
    for q in (1, 2, 3):
        assert abs(r16[q] - r32[q]) <= 3e-2 * abs(r32[q]) + 1e-9, (q, r16[q], r32[q])
    err = float(torch.linalg.vector_norm(ga.double() - ga32.double()) / torch.linalg.vector_norm(ga32.double()))
    assert err <= 3e-2, err

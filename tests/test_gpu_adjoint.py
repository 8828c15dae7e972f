"""GPU: the checkpointed discrete adjoint against central finite differences.

* FP64, D3Q19 BGK, TRT and MRT, 20^3: <grad J, d> along 16 seeded unit directions
  d of the initial velocity field and dJ/dtau match central differences of
  forward-only runs to relative 1e-6 (the bar the engine is held to is 1e-4);
  the step count is not a multiple of the checkpoint interval, so a partial
  last segment is covered;
* the FP32 gradient at 32^3 over 400 steps matches the FP64 one to rel-L2 1e-3;
* torch.autograd through the harness wrapper gives the same gradient.
"""
import math

import pytest
import torch

import lbcube as E
from lbm_autograd import KineticEnergy, run_gradient

pytestmark = pytest.mark.gpu

C19 = torch.tensor([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                    [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                    [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]], dtype=torch.float64)


def smooth_field(n, seed, amp, dev, dtype=torch.float64):
    """Seeded smooth random velocity field (a few low Fourier modes)."""
    g = torch.Generator().manual_seed(seed)
    k = 2 * math.pi / n
    ax = torch.arange(n, dtype=torch.float64) * k
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    u = torch.zeros((3, n, n, n), dtype=torch.float64)
    for d in range(3):
        for _ in range(4):
            kx, ky, kz = (torch.randint(0, 3, (3,), generator=g)).tolist()
            ph = float(torch.rand(1, generator=g)) * 2 * math.pi
            u[d] += torch.cos(kx * x + ky * y + kz * z + ph)
    u *= amp / u.abs().max()
    return u.to(device=dev, dtype=dtype).contiguous()


def forward_ke(u0, tau, steps, collision):
    """J from a forward-only run through the public step launcher (FP64 sums)."""
    nz, ny, nx = u0.shape[1:]
    real = "double" if u0.dtype == torch.float64 else "float"
    rho = torch.ones(u0.shape[1:], dtype=u0.dtype, device=u0.device)
    f = torch.empty((19, nz, ny, nx), dtype=u0.dtype, device=u0.device)
    E.check(E.init_equilibrium_async("D3Q19", real, rho, u0.contiguous(), f, nx, ny, nz))
    g = torch.empty_like(f)
    for _ in range(steps):
        E.check(E.launch_step_gpu("D3Q19", real, collision, f, g, nx, ny, nz, 1.0 / tau))
        f, g = g, f
    f = f.double()
    r = f.sum(0)
    j = torch.einsum("qd,q...->d...", C19.to(f.device), f)
    return float((0.5 * (j * j).sum(0) / r).sum())


@pytest.mark.parametrize("collision", ["BGK", "TRT", "MRT"])
def test_gradient_matches_central_differences_fp64(collision):
    dev = torch.device("cuda:0")
    n, steps, interval, tau = 20, 47, 10, 0.56
    u0 = smooth_field(n, 4, 0.03, dev)
    J, dtau, grad = run_gradient(u0, tau, steps, interval, collision)
    assert abs(J - forward_ke(u0, tau, steps, collision)) <= 1e-12 * abs(J)
    gen = torch.Generator().manual_seed(1234)
    eps = 1e-4
    worst = 0.0
    for _ in range(16):
        d = torch.randn(u0.shape, generator=gen, dtype=torch.float64).to(dev)
        d /= torch.linalg.vector_norm(d)
        fd = (forward_ke(u0 + eps * d, tau, steps, collision) -
              forward_ke(u0 - eps * d, tau, steps, collision)) / (2 * eps)
        ad = float((grad * d).sum())
        worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-30))
    assert worst <= 1e-6, worst
    et = 1e-6
    fd_tau = (forward_ke(u0, tau + et, steps, collision) - forward_ke(u0, tau - et, steps, collision)) / (2 * et)
    assert abs(fd_tau - dtau) <= 1e-6 * abs(fd_tau), (fd_tau, dtau)


def test_fp32_gradient_matches_fp64():
    dev = torch.device("cuda:0")
    n, steps, interval, tau = 32, 400, 100, 0.56
    u64 = smooth_field(n, 7, 0.03, dev)
    J64, d64, g64 = run_gradient(u64, tau, steps, interval, "BGK")
    J32, d32, g32 = run_gradient(u64.float(), tau, steps, interval, "BGK")
    assert abs(J32 - J64) <= 1e-5 * abs(J64)
    assert abs(d32 - d64) <= 1e-3 * abs(d64)
    err = float(torch.linalg.vector_norm(g32.double() - g64) / torch.linalg.vector_norm(g64))
    assert err <= 1e-3, err


def test_autograd_wrapper():
    dev = torch.device("cuda:0")
    u0 = smooth_field(16, 9, 0.02, dev).requires_grad_(True)
    tau = torch.tensor(0.6, dtype=torch.float64, requires_grad=True)
    J = KineticEnergy.apply(u0, tau, 30, 8, "TRT")
    J.backward()
    _, dtau, grad = run_gradient(u0.detach(), 0.6, 30, 8, "TRT")
    assert torch.equal(u0.grad, grad)
    assert float(tau.grad) == dtau


def test_d2q9_mrt_gradient_fp64():
    """D2Q9 MRT (the reference's rates 1.63, 1.14, 1.92, omega): KE gradient
    against central differences through the public 2-D launchers."""
    dev = torch.device("cuda:0")
    n, steps, interval, tau = 24, 31, 8, 0.6
    g = torch.Generator().manual_seed(77)
    k = 2 * math.pi / n
    ax = torch.arange(n, dtype=torch.float64) * k
    y, x = torch.meshgrid(ax, ax, indexing="ij")
    u0 = torch.stack([0.03 * torch.sin(x + 0.3) * torch.cos(2 * y), -0.02 * torch.cos(x) * torch.sin(y + 1.0)])
    u0 = (u0 + 0.005 * torch.randn(u0.shape, generator=g, dtype=torch.float64)).to(dev).contiguous()
    rho = torch.ones((n, n), dtype=torch.float64, device=dev)
    C9 = torch.tensor([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]],
                      dtype=torch.float64, device=dev)

    def ke(u, t):
        f = torch.empty((9, n, n), dtype=torch.float64, device=dev)
        E.check(E.init_equilibrium_async("D2Q9", "double", rho, u.contiguous(), f, n, n, 1))
        h = torch.empty_like(f)
        for _ in range(steps):
            E.check(E.launch_step_gpu("D2Q9", "double", "MRT", f, h, n, n, 1, 1.0 / t))
            f, h = h, f
        r = f.sum(0)
        j = torch.einsum("qd,q...->d...", C9, f)
        return float((0.5 * (j * j).sum(0) / r).sum())

    nb = E.ke_gradient_workspace_bytes("D2Q9", "double", n, n, 1, steps, interval)
    ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    grad = torch.empty_like(u0)
    E.check(E.ke_gradient_async("D2Q9", "double", "MRT", rho, u0, n, n, 1, tau, steps, interval, ws, nb, out,
                                grad))
    torch.cuda.synchronize()
    J, dtau = out.tolist()
    assert abs(J - ke(u0, tau)) <= 1e-12 * abs(J)
    for _ in range(6):
        d = torch.randn(u0.shape, generator=g, dtype=torch.float64).to(dev)
        d /= torch.linalg.vector_norm(d)
        fd = (ke(u0 + 1e-4 * d, tau) - ke(u0 - 1e-4 * d, tau)) / 2e-4
        ad = float((grad * d).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
    fd_tau = (ke(u0, tau + 1e-6) - ke(u0, tau - 1e-6)) / 2e-6
    assert abs(fd_tau - dtau) <= 1e-6 * abs(fd_tau) + 1e-13 * abs(J) / 1e-6, (fd_tau, dtau)

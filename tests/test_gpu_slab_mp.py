"""GPU: the z-slab decomposition with its ranks in separate processes.

Two processes form a gloo process group and each steps its slab of one
periodic box on cuda:0 with the engine's kernels (lbm_step_slab_async, and
lbm_fluid_reaction_slab_async for the coupled fluid + A + B -> C step);
HostExchange moves the face buffers between them through host memory, so no
kernel ever waits on the other rank. The assembled slabs must be bit-identical
to the whole box stepped in this process, and the reactive statistics
all-reduced over the two ranks must equal the whole box's to 1e-12; the
reactive gradient run as two slabs (slab.ReactiveSlabGradient.run) must give
the whole box's initial-state gradients bit for bit and its four scalars to
1e-10. (This
runs on one GPU; across GPUs the same host code moves the faces with NCCL,
slab.DistributedExchange.)
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import _util as U
import lbcube as E

pytestmark = pytest.mark.gpu

WORLD = 2
DIMS = (16, 6, 8)
STEPS = 6
OMEGA, OMEGA_C, K = 1 / 0.6, 1 / 0.8, 0.3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _states(lat, dt):
    nx, ny, nz = DIMS
    f = U.random_state(lat, nx, ny, nz, dt, seed=41)
    a = U.random_scalar("D3Q7", nx, ny, nz, dt, seed=42)
    b = U.random_scalar("D3Q7", nx, ny, nz, dt, seed=43)
    return f, a, b


def _worker(rank, port, case, q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (os.path.join(root, "lb-cube_b200"), os.path.join(root, "oracle"), os.path.dirname(__file__)):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import slab

    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=WORLD,
                                timeout=datetime.timedelta(seconds=60))
        dev = torch.device("cuda:0")
        torch.cuda.set_device(dev)
        lat, dn, op, overlap = case
        dt = np.float32 if dn == "float" else np.float64
        nx, ny, nz = DIMS
        f, a, b = _states(lat, dt)
        q_f = E.Q_OF[lat]
        ex = slab.HostExchange(dist)
        if op.startswith("adjoint-"):  # the reactive gradient: (result, dJ/dA0, dJ/dB0, dJ/du0)
            from test_gpu_adjoint_reactive import fields

            _, cop, obj = op.split("-", 2)
            rho, u, a0, b0 = fields(lat, (nz, ny, nx), dev, torch.float32 if dn == "float" else torch.float64, 91)
            g = slab.ReactiveSlabGradient(torch, lat, dn, cop, obj, nx, ny, nz, 0.8, 0.7, 0.6, 7, 3, rank, WORLD,
                                          dev)
            sl = slice(g.z0, g.z0 + g.nz)
            res = g.run(rho[sl].contiguous(), u[:, sl].contiguous(), a0[sl].contiguous(), b0[sl].contiguous(),
                        ex, dist)
            torch.cuda.synchronize()
            stats = res[0].cpu().numpy()
            out = [t.cpu().numpy() for t in res[1:]]
        elif op.startswith("coupled-"):
            d = slab.ReactiveSlabDomain(torch, lat, dn, op[8:], nx, ny, nz, OMEGA, OMEGA_C, K, rank, WORLD, dev)

            def mine(x, qq):
                return torch.from_numpy(np.ascontiguousarray(x.reshape(qq, nz, ny, nx)[:, d.z0:d.z0 + d.nz])).to(dev)

            cur = (mine(f, q_f), mine(a, 7), mine(b, 7))
            nxt = tuple(torch.empty_like(t) for t in cur)
            d.pack(cur)
            ex.exchange(d)
            for s in range(STEPS):
                d.compute(cur, nxt, stats=s == STEPS - 1)
                ex.exchange(d)
                cur, nxt = nxt, cur
            stats = d.statistics(dist).cpu().numpy()
            out = [t.cpu().numpy() for t in cur]
        else:
            d = slab.SlabDomain(torch, lat, dn, op, nx, ny, nz, OMEGA, rank, WORLD, dev)
            cur = torch.from_numpy(np.ascontiguousarray(f.reshape(q_f, nz, ny, nx)[:, d.z0:d.z0 + d.nz])).to(dev)
            nxt = torch.empty_like(cur)
            if overlap:  # SlabDomain.step: exchange on a second stream, overlapped with the interior planes
                d.prime(cur, ex)
                for _ in range(STEPS):
                    d.step(cur, nxt, ex)
                    cur, nxt = nxt, cur
                d.finish()
            else:
                d.pack(cur)
                ex.exchange(d)
                for _ in range(STEPS):
                    d.compute(cur, nxt)
                    ex.exchange(d)
                    cur, nxt = nxt, cur
            stats = None
            out = [cur.cpu().numpy()]
        torch.cuda.synchronize()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, out, stats, ""))
    except Exception as e:  # reported to the parent
        q.put((rank, None, None, repr(e)))


def _run(case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, case, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        res = sorted((q.get(timeout=300) for _ in range(WORLD)), key=lambda r: r[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for rank, _, _, err in res:
        assert not err, f"rank {rank}: {err}"
    return res


@pytest.mark.parametrize("case", [("D3Q19", "float", "TRT", False), ("D3Q19", "float", "TRT", True),
                                  ("D3Q27", "double", "TRT", False)])
def test_fluid_slabs_in_two_processes(engine, dev, case):
    lat, dn, op, _ = case
    nx, ny, nz = DIMS
    f, _, _ = _states(lat, np.float32 if dn == "float" else np.float64)
    a = torch.from_numpy(f).to(dev)
    b = torch.empty_like(a)
    for _ in range(STEPS):
        E.check(E.step_async(lat, dn, op, a, b, nx, ny, nz, OMEGA))
        a, b = b, a
    want = a.cpu().numpy()
    res = _run(case)
    q = E.Q_OF[lat]
    got = np.concatenate([r[1][0] for r in res], axis=1).reshape(q, -1)
    assert U.same_bits(got, want)


@pytest.mark.parametrize("lat,dn,op", [("D3Q19", "float", "TRT"), ("D3Q19", "double", "BGK")])
def test_coupled_slabs_in_two_processes(engine, dev, lat, dn, op):
    nx, ny, nz = DIMS
    f, a, b = _states(lat, np.float32 if dn == "float" else np.float64)
    cur = [torch.from_numpy(x).to(dev) for x in (f, a, b)]
    nxt = [torch.empty_like(x) for x in cur]
    pb = E.stats_partials_bytes(lat, nx, ny, nz)
    part = torch.empty(pb // 8, dtype=torch.float64, device=dev)
    want_stats = torch.empty(8, dtype=torch.float64, device=dev)
    for s in range(STEPS):
        last = s == STEPS - 1
        E.check(E.fluid_reaction_ab_async(lat, dn, op, cur[0], nxt[0], cur[1], nxt[1], cur[2], nxt[2], nx, ny, nz,
                                          OMEGA, OMEGA_C, K, part if last else None, pb if last else 0))
        cur, nxt = nxt, cur
    E.check(E.reactive_stats_finalize_async(lat, dn, nx, ny, nz, K, part, pb, want_stats))
    res = _run((lat, dn, f"coupled-{op}", False))
    for idx, qq in enumerate((E.Q_OF[lat], 7, 7)):
        got = np.concatenate([r[1][idx] for r in res], axis=1).reshape(qq, -1)
        assert U.same_bits(got, cur[idx].cpu().numpy().reshape(qq, -1)), ("fluid", "A", "B")[idx]
    w = want_stats.cpu().numpy()
    for rank, _, stats, _ in res:
        assert np.all(np.abs(stats - w) <= 1e-12 * np.maximum(np.abs(w), 1e-300)), (rank, stats, w)


@pytest.mark.parametrize("lat,dn,op", [("D3Q19", "double", "TRT"), ("D3Q27", "float", "BGK")])
def test_reactive_gradient_slabs_in_two_processes(engine, dev, lat, dn, op):
    from test_gpu_slab_adjoint import whole_box
    from test_gpu_adjoint_reactive import fields

    nx, ny, nz = DIMS
    rho, u, a0, b0 = fields(lat, (nz, ny, nx), dev, torch.float32 if dn == "float" else torch.float64, 91)
    want = whole_box(lat, dn, op, "mean_product", rho, u, a0, b0, DIMS, 7, 3)
    res = _run((lat, dn, f"adjoint-{op}-mean_product", False))
    for rank, _, result, _ in res:
        assert np.all(np.abs(result - want[0]) <= 1e-10 * np.abs(want[0])), (rank, result, want[0])
    for idx, axis in ((0, 0), (1, 0), (2, 1)):
        got = np.concatenate([r[1][idx] for r in res], axis=axis)
        assert U.same_bits(got, want[1 + idx]), ("dJ/dA0", "dJ/dB0", "dJ/du0")[idx]

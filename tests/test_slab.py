"""CPU: the z-slab decomposition's host side with gloo ranks (world size 2 and
3). The face exchange delivers each neighbour's send buffers into the right
halo buffers (also through host staging, alternating face buffers of two
element types), and a streaming step assembled from slabs (a numpy restatement
of the slab kernel's pull: halo_lo for c_z = +1 at plane 0, halo_hi for c_z = -1
at the top plane) equals the periodic streaming of the whole box."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

C19 = [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
       [1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
       [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]]
NX, NY, NZ = 6, 5, 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pack(f, send_lo, send_hi):
    up = [i for i, c in enumerate(C19) if c[2] > 0]
    dn = [i for i, c in enumerate(C19) if c[2] < 0]
    send_hi[:] = np.stack([f[i, -1] for i in up]).reshape(-1)
    send_lo[:] = np.stack([f[i, 0] for i in dn]).reshape(-1)


def _slab_stream(f, halo_lo, halo_hi):
    """Pull streaming of one slab with face halos: out_i(x) = f_i(x - c_i)."""
    q, nz, ny, nx = f.shape
    up = [i for i, c in enumerate(C19) if c[2] > 0]
    dn = [i for i, c in enumerate(C19) if c[2] < 0]
    hl = halo_lo.reshape(len(up), ny, nx)
    hh = halo_hi.reshape(len(dn), ny, nx)
    out = np.empty_like(f)
    for i, (cx, cy, cz) in enumerate(C19):
        ext = np.concatenate([hl[up.index(i)][None] if cz > 0 else f[i, -1:], f[i],
                              hh[dn.index(i)][None] if cz < 0 else f[i, :1]], axis=0)
        src = ext[1 - cz: 1 - cz + nz]
        out[i] = np.roll(np.roll(src, cy, axis=1), cx, axis=2)
    return out


def _worker(rank, world, port, q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "lb-cube_b200"))
    import slab

    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        d = slab.SlabDomain(torch, "D3Q19", "double", "BGK", NX, NY, NZ, 1.0, rank, world, "cpu")
        ex = slab.DistributedExchange(dist)
        # 1. pure exchange: rank-tagged patterns
        n = d.send_lo.numel()
        d.send_lo.copy_(torch.arange(n, dtype=torch.float64) + 1000 * rank + 1)
        d.send_hi.copy_(torch.arange(n, dtype=torch.float64) + 1000 * rank + 500)
        ex.exchange(d)
        lower, upper = (rank - 1) % world, (rank + 1) % world
        ok1 = (torch.equal(d.halo_lo, torch.arange(n, dtype=torch.float64) + 1000 * lower + 500) and
               torch.equal(d.halo_hi, torch.arange(n, dtype=torch.float64) + 1000 * upper + 1))
        # 16-bit codes (face buffers of a slab on shifted storage), bit patterns
        # that are NaN or subnormal as float16 included
        saved = (d.halo_lo, d.halo_hi, d.send_lo, d.send_hi)
        d.halo_lo, d.halo_hi, d.send_lo, d.send_hi = (torch.zeros(n, dtype=torch.int16) for _ in range(4))
        code = lambda r, side: ((torch.arange(n) * 7919 + 977 * r + 31 * side) % 65536 - 32768).to(torch.int16)
        d.send_lo.copy_(code(rank, 0))
        d.send_hi.copy_(code(rank, 1))
        ex.exchange(d)
        ok1 = ok1 and torch.equal(d.halo_lo, code(lower, 1)) and torch.equal(d.halo_hi, code(upper, 0))
        d.halo_lo, d.halo_hi, d.send_lo, d.send_hi = saved
        # 2. one streaming step assembled from slabs vs the whole box
        rng = np.random.default_rng(5)
        full = rng.random((19, NZ, NY, NX))
        mine = full[:, d.z0:d.z0 + d.nz].copy()
        lo, hi = d.send_lo.numpy(), d.send_hi.numpy()
        _pack(mine, lo, hi)
        ex.exchange(d)
        got = _slab_stream(mine, d.halo_lo.numpy(), d.halo_hi.numpy())
        want = np.stack([np.roll(full[i], shift=(c[2], c[1], c[0]), axis=(0, 1, 2)) for i, c in enumerate(C19)])
        ok2 = np.array_equal(got, want[:, d.z0:d.z0 + d.nz])
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, bool(ok1), bool(ok2), ""))
    except Exception as e:  # reported to the parent
        q.put((rank, False, False, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_slab_exchange_and_streaming_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for rank, ok1, ok2, err in sorted(res):
        assert not err, err
        assert ok1, f"rank {rank}: halos do not hold the neighbours' send buffers"
        assert ok2, f"rank {rank}: slab streaming differs from the periodic box"


def _host_worker(rank, world, port, q):
    """HostExchange alternating two kinds of face buffer (16-bit codes and FP64,
    as the slab reactive gradient does): each exchange must deliver the
    neighbours' buffers of the kind in use."""
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "lb-cube_b200"))
    import slab

    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        d = slab.SlabDomain(torch, "D3Q19", "double", "BGK", NX, NY, NZ, 1.0, rank, world, "cpu")
        n = d.send_lo.numel()
        kinds = {"codes": tuple(torch.zeros(n, dtype=torch.int16) for _ in range(4)),
                 "real": (d.halo_lo, d.halo_hi, d.send_lo, d.send_hi)}
        ex = slab.HostExchange(dist)
        lower, upper = (rank - 1) % world, (rank + 1) % world
        ok = True
        for step, kind in enumerate(["codes", "real", "codes", "real"]):
            d.halo_lo, d.halo_hi, d.send_lo, d.send_hi = kinds[kind]
            dt = d.send_lo.dtype
            tag = lambda r, side: (torch.arange(n) % 97 + 100 * r + 10 * side + step).to(dt)
            d.send_lo.copy_(tag(rank, 0))
            d.send_hi.copy_(tag(rank, 1))
            ex.exchange(d)
            ok = ok and torch.equal(d.halo_lo, tag(lower, 1)) and torch.equal(d.halo_hi, tag(upper, 0))
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, bool(ok), ""))
    except Exception as e:  # reported to the parent
        q.put((rank, False, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_host_exchange_two_face_kinds_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_host_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for rank, ok, err in sorted(res):
        assert not err, err
        assert ok, f"rank {rank}: a halo does not hold its neighbour's send buffer of the same kind"


def test_slab_domain_rejects_bad_splits():
    import slab

    with pytest.raises(ValueError):
        slab.SlabDomain(torch, "D3Q19", "float", "TRT", 8, 8, 10, 1.0, 0, 3, "cpu")
    with pytest.raises(ValueError):
        slab.SlabDomain(torch, "D2Q9", "float", "TRT", 8, 8, 1, 1.0, 0, 1, "cpu")

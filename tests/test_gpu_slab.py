"""GPU: the z-slab decomposition on one device. W ranks are emulated in one
process (LocalExchange copies the face buffers between slabs, standing in for
the point-to-point transfers); stepping the slabs is bit-identical to
stepping the whole periodic box with lbm_step_async, for W = 1..4 including
one-plane slabs. The single-rank path of SlabDomain.step (exchange on a second
stream, overlapped with the interior planes) is bit-identical too."""
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

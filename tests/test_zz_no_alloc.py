"""GPU: the allocation-free statistics entry point.

Some callers cannot allocate device memory: a plugin or FFI binding inside an
application that owns every device allocation hands this library only its
scalar fields, so it cannot provide the partial-sum scratch that
lbm_reactive_stats_async takes. lbm_reactive_stats_noalloc_async keeps that
scratch in a fixed array inside the library. Called through the C ABI, it must
give the same diagnostics as the scratch-taking entry point (within the 1e-12
relative tolerance of the statistics tests) on two calls in a row, accept the
largest domain its array holds and reject a larger one. This file is
collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import _util as U
import lbcube as E

pytestmark = pytest.mark.gpu

_vp, _sz = C.c_void_p, C.c_size_t


def _noalloc():
    fn = E.load().lbm_reactive_stats_noalloc_async
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_double, _vp, _vp]
    return fn


@pytest.mark.parametrize("lat,real,shape", [("D3Q7", "float", (131, 40, 24)),
                                            ("D2Q5", "double", (300, 77, 1))])
def test_noalloc_stats_match_scratch_entry(lat, real, shape):
    dev = torch.device("cuda:0")
    nx, ny, nz = shape
    dt = np.float32 if real == "float" else np.float64
    a = torch.from_numpy(U.random_scalar(lat, nx, ny, nz, dt, seed=81)).to(dev)
    b = torch.from_numpy(U.random_scalar(lat, nx, ny, nz, dt, seed=82)).to(dev)
    fluid = "D2Q9" if lat == "D2Q5" else "D3Q19"
    nbytes = E.stats_partials_bytes(fluid, nx, ny, nz)
    part = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
    want = torch.empty(8, dtype=torch.float64, device=dev)
    E.check(E.reactive_stats_async(lat, real, a, b, nx, ny, nz, 0.02, part, nbytes, want))
    fn = _noalloc()
    for call in range(2):
        got = torch.full((8,), float("nan"), dtype=torch.float64, device=dev)
        rc = fn(E.LATTICES[lat], E.REALS[real], a.data_ptr(), b.data_ptr(), nx, ny, nz, 0.02,
                 got.data_ptr(), None)
        assert rc == 0, f"call {call}: cudaError_t {rc}"
        torch.cuda.synchronize()
        for name, g, w in zip(E.STATS_FIELDS, got.cpu().tolist(), want.cpu().tolist()):
            assert abs(g - w) <= 1e-12 * max(abs(w), 1e-6), f"call {call}: {name}"


def _fields(lat, nx, ny, nz, seed):
    """Two scalar fields of the declared extent in separate device buffers, so
    that no overlap check can reject the call."""
    dev = torch.device("cuda:0")
    q = E.Q_OF[lat]
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    a = torch.rand((q, nz, ny, nx), generator=gen, device=dev) * 0.2
    b = torch.rand((q, nz, ny, nx), generator=gen, device=dev) * 0.2
    return a, b


def test_noalloc_accepts_the_largest_domain_its_array_holds():
    # ceil(256 / 128) * 256 * 256 = 131072 row segments: exactly the array's capacity
    assert E.stats_partials_bytes("D3Q19", 256, 256, 256) == 131072 * 5 * 8
    a, b = _fields("D3Q7", 256, 256, 256, seed=83)
    nbytes = E.stats_partials_bytes("D3Q19", 256, 256, 256)
    part = torch.empty(nbytes // 8, dtype=torch.float64, device=a.device)
    want = torch.empty(8, dtype=torch.float64, device=a.device)
    E.check(E.reactive_stats_async("D3Q7", "float", a, b, 256, 256, 256, 0.02, part, nbytes, want))
    got = torch.full((8,), float("nan"), dtype=torch.float64, device=a.device)
    rc = _noalloc()(E.LATTICES["D3Q7"], E.REALS["float"], a.data_ptr(), b.data_ptr(), 256, 256, 256, 0.02,
                    got.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    for name, g, w in zip(E.STATS_FIELDS, got.cpu().tolist(), want.cpu().tolist()):
        assert abs(g - w) <= 1e-12 * max(abs(w), 1e-6), name


def test_noalloc_rejects_domains_beyond_its_array():
    # ceil(129 / 128) * 256 * 257 = 131584 row segments > 131072. Real, disjoint
    # fields of the declared size: the scratch-taking entry accepts them, so the
    # only reason left to reject the call is the array's capacity.
    nx, ny, nz = 129, 256, 257
    a, b = _fields("D3Q7", nx, ny, nz, seed=84)
    nbytes = E.stats_partials_bytes("D3Q19", nx, ny, nz)
    assert nbytes == 131584 * 5 * 8
    part = torch.empty(nbytes // 8, dtype=torch.float64, device=a.device)
    out = torch.empty(8, dtype=torch.float64, device=a.device)
    E.check(E.reactive_stats_async("D3Q7", "float", a, b, nx, ny, nz, 0.02, part, nbytes, out))
    rc = _noalloc()(E.LATTICES["D3Q7"], E.REALS["float"], a.data_ptr(), b.data_ptr(), nx, ny, nz, 0.02,
                    out.data_ptr(), None)
    assert rc == E.cudaErrorInvalidValue

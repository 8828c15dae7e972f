"""GPU: the allocation-free statistics entry point.

Some callers cannot allocate device memory: a plugin or FFI binding inside an
application that owns every device allocation hands this library only its
scalar fields, so it cannot provide the partial-sum scratch that
lbm_reactive_stats_async takes. lbm_reactive_stats_noalloc_async keeps that
scratch in a fixed array inside the library. Called through the C ABI, it must
give the same diagnostics as the scratch-taking entry point (within the 1e-12
relative tolerance of the statistics tests) on two calls in a row, and reject a
domain larger than its array. This file is collected last on purpose.
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


def test_noalloc_rejects_domains_beyond_its_array():
    dev = torch.device("cuda:0")
    out = torch.empty(8, dtype=torch.float64, device=dev)
    fn = _noalloc()
    # ceil(129 / 128) * 256 * 257 = 131584 row segments > 131072; the call is
    # rejected before any kernel runs, so the (never read) field addresses can be fake.
    rc = fn(E.LATTICES["D3Q7"], E.REALS["float"], 0x10000000, 0x90000000, 129, 256, 257, 0.02,
            out.data_ptr(), None)
    assert rc == E.cudaErrorInvalidValue

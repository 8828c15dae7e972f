"""CPU: the engine library loads, exports every symbol its C header declares,
and its launchers reject bad arguments with the reference's error codes before
touching the GPU (src/lattice_cuda.cu:488-503). Fake, never-dereferenced
addresses stand in for device buffers: every case below returns before any
CUDA call is made."""
import ctypes as C

import pytest

import lbcube as E

# Fake device addresses (never dereferenced: validation fails first).
A0, A1, A2, A3, A4 = 0x10000000, 0x20000000, 0x30000000, 0x40000000, 0x50000000


@pytest.fixture(scope="module")
def lib():
    import os

    if not os.path.exists(E.LIB_PATH):
        import build

        build.build()
    return E.load()


def test_exports_every_declared_symbol(lib):
    declared = E.declared_symbols()
    assert len(declared) >= 44
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_reference_launcher_set_is_complete():
    """24 step + 6 scalar + 6 reaction instantiations (src/lattice_cuda.cu:756-1029)."""
    declared = set(E.declared_symbols())
    steps = [s for s in declared if s.startswith("lbm_launch_step_gpu_")]
    scal = [s for s in declared if s.startswith("lbm_launch_scalar_step_gpu_")]
    reac = [s for s in declared if s.startswith("lbm_launch_reaction_ab_gpu_")]
    assert (len(steps), len(scal), len(reac)) == (24, 6, 6)


@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19", "D3Q27"])
@pytest.mark.parametrize("real", ["float", "double"])
@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT", "RLBM"])
def test_step_validation_order(lib, lat, real, op):
    f = lambda *a, **k: E.launch_step_gpu(lat, real, op, *a, **k)  # noqa: E731
    # null pointer first, even with a zero block and zero extents
    assert f(None, A1, 0, 0, 0, 1.0, block=(0, 0, 0)) == E.cudaErrorInvalidDevicePointer
    assert f(A0, None, 8, 8, 8, 1.0) == E.cudaErrorInvalidDevicePointer
    # zero block dimension before extents
    assert f(A0, A1, 0, 8, 8, 1.0, block=(16, 0, 1)) == E.cudaErrorInvalidConfiguration
    assert f(A0, A1, 8, 8, 8, 1.0, block=(16, 8, 0)) == E.cudaErrorInvalidConfiguration
    # zero extents
    assert f(A0, A1, 0, 8, 8, 1.0) == E.cudaErrorInvalidValue
    assert f(A0, A1, 8, 0, 8, 1.0) == E.cudaErrorInvalidValue
    if lat != "D2Q9":
        assert f(A0, A1, 8, 8, 0, 1.0) == E.cudaErrorInvalidValue
    # overlapping read/write buffers (engine check)
    assert f(A0, A0, 8, 8, 8, 1.0) == E.cudaErrorInvalidValue
    assert f(A0, A0 + 64, 8, 8, 8, 1.0) == E.cudaErrorInvalidValue
    # more than 2^31 - 1 cells (engine limit)
    if lat != "D2Q9":
        assert f(A0, A0 + (1 << 44), 2048, 2048, 1024, 1.0) == E.cudaErrorInvalidValue


@pytest.mark.parametrize("fl", ["D2Q9", "D3Q19", "D3Q27"])
@pytest.mark.parametrize("real", ["float", "double"])
def test_scalar_and_reaction_validation(lib, fl, real):
    s = E.launch_scalar_step_gpu
    assert s(fl, real, A0, A1, None, 8, 8, 8, 1.2) == E.cudaErrorInvalidDevicePointer
    assert s(fl, real, A0, A1, A2, 8, 8, 8, 1.2, block=(0, 8, 1)) == E.cudaErrorInvalidConfiguration
    assert s(fl, real, A0, A1, A2, 0, 8, 8, 1.2) == E.cudaErrorInvalidValue
    assert s(fl, real, A0, A0, A2, 8, 8, 8, 1.2) == E.cudaErrorInvalidValue
    # LatticeMemory overload: mismatched scalar / fluid extents (src/lattice_cuda.cu:731-735)
    assert E.launch_scalar_step_gpu_mem(fl, real, (8, 8, 8), (8, 8, 4), A0, A1, A2, 1.2) == \
        E.cudaErrorInvalidValue
    r = E.launch_reaction_AB_gpu
    assert r(fl, real, A0, A1, A2, A3, None, 8, 8, 8, 1.2, 0.01) == E.cudaErrorInvalidDevicePointer
    assert r(fl, real, A0, A1, A2, A3, A4, 8, 8, 8, 1.2, 0.01, block=(1, 1, 0)) == \
        E.cudaErrorInvalidConfiguration
    assert r(fl, real, A0, A1, A2, A3, A4, 8, 0, 8, 1.2, 0.01) == E.cudaErrorInvalidValue
    # next_a aliasing current_b
    assert r(fl, real, A0, A2, A2, A3, A4, 8, 8, 8, 1.2, 0.01) == E.cudaErrorInvalidValue


def test_2d_block_z_checked_before_forcing(lib):
    """For 2D lattices the reference checks block.z == 0 before forcing it to 1
    (src/lattice_cuda.cu:492-499)."""
    assert E.launch_step_gpu("D2Q9", "float", "BGK", A0, A1, 8, 8, 1, 1.0, block=(16, 8, 0)) == \
        E.cudaErrorInvalidConfiguration


def test_extension_enum_validation(lib):
    assert E.load().lbm_step_async(7, 0, 0, A0, A1, 8, 8, 8, 1.0, None) == E.cudaErrorInvalidValue
    assert E.load().lbm_step_async(1, 5, 0, A0, A1, 8, 8, 8, 1.0, None) == E.cudaErrorInvalidValue
    assert E.load().lbm_step_async(1, 0, 9, A0, A1, 8, 8, 8, 1.0, None) == E.cudaErrorInvalidValue
    # the fused fluid + reaction launch has no RLBM variant
    assert E.fluid_reaction_ab_async("D3Q19", "float", "RLBM", A0, A1, A2, A3, A4, A4 + (1 << 30),
                                     8, 8, 8, 1.6, 1.2, 0.01) == E.cudaErrorInvalidValue
    assert E.stats_partials_bytes("D3Q19", 256, 256, 256) == 2 * 256 * 256 * 5 * 8
    assert E.stats_partials_bytes("D2Q9", 1024, 1024, 7) == 8 * 1024 * 5 * 8
    # a too-small partials buffer is rejected
    assert E.reactive_stats_async("D3Q7", "float", A0, A1, 256, 256, 256, 0.1, A2, 16, A3) == \
        E.cudaErrorInvalidValue


def test_diagnostics_validation(lib):
    assert E.diagnostics_partials_bytes("D3Q19", 256, 256, 256) == 2 * 256 * 256 * 4 * 8
    assert E.diagnostics_partials_bytes("D2Q9", 1024, 1024, 7) == 8 * 1024 * 4 * 8
    assert E.diagnostics_partials_bytes("D3Q19", 0, 4, 4) == 0
    need = E.diagnostics_partials_bytes("D3Q19", 8, 8, 8)
    # null populations, partials or output
    assert E.fluid_diagnostics_async("D3Q19", "float", None, 8, 8, 8, A1, need, A2) == \
        E.cudaErrorInvalidDevicePointer
    assert E.fluid_diagnostics_async("D3Q19", "float", A0, 8, 8, 8, None, need, A2) == \
        E.cudaErrorInvalidDevicePointer
    assert E.step_diagnostics_async("D3Q19", "float", "TRT", A0, A1, 8, 8, 8, 1.6, A2, need, None) == \
        E.cudaErrorInvalidDevicePointer
    # zero extent, too-small scratch, scratch overlapping the populations, bad enums
    assert E.fluid_diagnostics_async("D3Q19", "float", A0, 8, 0, 8, A1, need, A2) == E.cudaErrorInvalidValue
    assert E.fluid_diagnostics_async("D3Q19", "float", A0, 8, 8, 8, A1, need - 8, A2) == E.cudaErrorInvalidValue
    assert E.fluid_diagnostics_async("D3Q19", "float", A0, 8, 8, 8, A0 + 64, need, A2) == \
        E.cudaErrorInvalidValue
    assert E.step_diagnostics_async("D3Q19", "double", "BGK", A0, A1, 8, 8, 8, 1.6, A2, need, A1 + 8) == \
        E.cudaErrorInvalidValue
    assert E.fluid_diagnostics_async("D2Q5", "float", A0, 8, 8, 1, A1, need, A2) == E.cudaErrorInvalidValue
    assert E.load().lbm_step_diagnostics_async(1, 0, 9, A0, A1, 8, 8, 8, 1.6, 1.0, A2, need, A3, None) == \
        E.cudaErrorInvalidValue


def test_oracle_diagnostics_semantics():
    """The oracle's FP64-accumulated diagnostics: sums and max of the per-cell
    terms, NaN speeds skipped by the max but counted, the crash flag."""
    import numpy as np

    import _util as U
    import oracle as O

    f = U.random_state("D3Q19", 6, 5, 4, np.float64, seed=3)
    d = O.fluid_diagnostics64(f, "D3Q19", 6, 5, 4, speed_limit=1.0)
    rho, u = O.macro_fields(f, "D3Q19", 6, 5, 4)
    s2 = (u * u).sum(0)
    assert d[0] == pytest.approx(rho.sum(), rel=1e-14)
    assert d[1] == pytest.approx((0.5 * rho * s2).sum(), rel=1e-12)
    assert d[2] == np.sqrt(s2).max() and d[3] == 0 and d[4] == 0
    ref = O.fluid_diagnostics(f, "D3Q19", 6, 5, 4)
    assert d[2] == ref[2]
    assert O.fluid_diagnostics64(f, "D3Q19", 6, 5, 4, speed_limit=0.5 * d[2])[4] == 1
    g = f.copy()
    g[3, 7] = np.nan  # one cell with a NaN population
    dn = O.fluid_diagnostics64(g, "D3Q19", 6, 5, 4, speed_limit=1.0)
    assert np.isnan(dn[0]) and dn[3] == 1 and dn[4] == 1
    assert dn[2] == np.sqrt(np.delete(s2, 7)).max()


def test_reactive_gradient_validation(lib):
    nb = E.reactive_gradient_workspace_bytes("D3Q19", "float", 16, 12, 10, 20, 4)
    cells = 16 * 12 * 10
    up = lambda b: (b + 255) // 256 * 256  # noqa: E731
    state = up(19 * cells * 4) + 2 * up(7 * cells * 4)
    assert nb >= (6 + 4 + 2) * state  # 6 checkpoints, one segment of 4, two adjoint states
    assert E.reactive_gradient_workspace_bytes("D2Q5", "float", 16, 12, 1, 20, 4) == 0
    assert E.reactive_gradient_workspace_bytes("D3Q19", "float", 16, 12, 10, 20, 1) == 0
    args = dict(rho0=A0, u0=A1, a0=A2, b0=A3, nx=16, ny=12, nz=10, tau=0.8, tau_c=0.7, k_react=0.1,
                steps=20, interval=4, workspace=A4, workspace_bytes=nb, result=A4 + (1 << 30),
                grad_a0=A4 + (2 << 30))

    def call(**kw):
        a = dict(args)
        a.update(kw)
        return E.reactive_gradient_async(a.pop("fl", "D3Q19"), a.pop("real", "float"), a.pop("op", "TRT"),
                                         a.pop("obj", "mean_product"), **a)

    assert call(a0=None) == E.cudaErrorInvalidDevicePointer
    assert call(grad_a0=None) == E.cudaErrorInvalidDevicePointer
    assert call(nz=0) == E.cudaErrorInvalidValue
    assert call(op="RLBM") == E.cudaErrorInvalidValue
    assert call(fl="D3Q27", op="MRT") == E.cudaErrorInvalidValue  # MRT adjoint: D2Q9 and D3Q19 only
    assert call(tau=0.5) == E.cudaErrorInvalidValue
    assert call(tau_c=0.4) == E.cudaErrorInvalidValue
    assert call(workspace_bytes=nb - 1) == E.cudaErrorInvalidValue
    assert call(steps=0) == E.cudaErrorInvalidValue
    assert E.load().lbm_reactive_gradient_async(1, 0, 0, 0.5, 1, 7, A0, A1, A2, A3, 16, 12, 10, 0.8, 0.7, 0.1,
                                                20, 4, A4, nb, A4 + 8, A4 + 16, None, None, None) == \
        E.cudaErrorInvalidValue
    # 16-bit stored states: FP32 only, and a known format
    nb16 = E.reactive_gradient_workspace_bytes("D3Q19", "float", 16, 12, 10, 20, 4, storage="f16s")
    assert 0 < nb16 < nb
    assert E.reactive_gradient_workspace_bytes("D3Q19", "double", 16, 12, 10, 20, 4, storage="f16s") == 0
    assert call(real="double", storage="q15s") == E.cudaErrorInvalidValue
    assert E.load().lbm_reactive_gradient_async(1, 0, 9, 0.5, 1, 0, A0, A1, A2, A3, 16, 12, 10, 0.8, 0.7, 0.1,
                                                20, 4, A4, nb, A4 + 8, A4 + 16, None, None, None) == \
        E.cudaErrorInvalidValue


def test_copy_buffers_validation(lib):
    """lbm_copy_buffers_async (face copies of slabs sharing a device) rejects
    bad lists before it touches the device: more than 64 pairs, a null
    pointer, a destination overlapping a source or another destination."""
    arr = C.c_void_p * 65
    src, dst = arr(*[A0 + i * 4096 for i in range(65)]), arr(*[A4 + i * 4096 for i in range(65)])
    assert lib.lbm_copy_buffers_async(65, src, dst, 1024, None) == E.cudaErrorInvalidValue
    assert lib.lbm_copy_buffers_async(-1, src, dst, 1024, None) == E.cudaErrorInvalidValue
    assert lib.lbm_copy_buffers_async(2, None, dst, 1024, None) == E.cudaErrorInvalidDevicePointer
    two = C.c_void_p * 2
    assert lib.lbm_copy_buffers_async(2, two(A0, None), two(A4, A4 + 4096), 1024, None) == \
        E.cudaErrorInvalidDevicePointer
    # a destination inside a source, and two destinations that overlap
    assert lib.lbm_copy_buffers_async(2, two(A0, A0 + 4096), two(A0 + 512, A4), 1024, None) == \
        E.cudaErrorInvalidValue
    assert lib.lbm_copy_buffers_async(2, two(A0, A0 + 4096), two(A4, A4 + 512), 1024, None) == \
        E.cudaErrorInvalidValue
    assert lib.lbm_copy_buffers_async(0, two(A0, A0), two(A4, A4), 1024, None) == 0  # nothing to copy

"""Python front end of the B200 lattice Boltzmann engine (ctypes over the C ABI).

The launchers mirror LB-Cube's CUDA launcher API (include/lattice_cuda.cuh:
179-319): same names, same argument meaning (device buffers in the unpadded
[Q, Z, Y, X] layout, element extents, relaxation frequencies), and the same
``cudaError_t`` return codes, including the reference's validation order. Any
object with ``data_ptr()`` (a torch CUDA tensor) or a plain integer address can
be passed as a buffer; ``None`` is the null pointer.

The engine library (``liblbcube_b200.so`` next to this file, or the file the
environment variable ``LBCUBE_LIB`` names) must have been built
(``python lb-cube_b200/build.py``); loading it without it raises, there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# LBCUBE_LIB selects another build of the library (e.g. of an earlier commit, for A/B timing)
LIB_PATH = os.environ.get("LBCUBE_LIB") or os.path.join(HERE, "liblbcube_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "lbcube_b200.h")

LATTICES = {"D2Q9": 0, "D3Q19": 1, "D3Q27": 2, "D2Q5": 3, "D3Q7": 4}
Q_OF = {"D2Q9": 9, "D3Q19": 19, "D3Q27": 27, "D2Q5": 5, "D3Q7": 7}
D_OF = {"D2Q9": 2, "D3Q19": 3, "D3Q27": 3, "D2Q5": 2, "D3Q7": 3}
SCALAR_OF = {"D2Q9": "D2Q5", "D3Q19": "D3Q7", "D3Q27": "D3Q7"}
COLLISIONS = {"BGK": 0, "TRT": 1, "MRT": 2, "RLBM": 3}
REALS = {"float": 0, "double": 1}
FORMATS = {"f16s": 2, "bf16s": 3, "e3m12s": 4, "q15s": 5}  # shifted 16-bit population storage

# cudaError_t values returned by the launchers
cudaSuccess = 0
cudaErrorInvalidValue = 1
cudaErrorInvalidConfiguration = 9
cudaErrorInvalidDevicePointer = 17

STATS_FIELDS = ("mean_A", "mean_B", "var_A", "var_B", "covariance", "segregation_intensity",
                "true_reaction_rate", "mixed_reaction_rate")

_lib = None


class LbmCudaError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} failed with cudaError_t {code}")
        self.code = code


def library_path() -> str:
    return LIB_PATH


def load() -> C.CDLL:
    """The engine library, loaded once. Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"engine library {LIB_PATH} is missing: build it with "
                "`python lb-cube_b200/build.py` (there is no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_sz, _vp, _u = C.c_size_t, C.c_void_p, C.c_uint


def _declare(lib):
    for lat in ("d2q9", "d3q19", "d3q27"):
        for real, ct in (("float", C.c_float), ("double", C.c_double)):
            for op in ("bgk", "trt", "mrt", "rlbm"):
                fn = getattr(lib, f"lbm_launch_step_gpu_{lat}_{real}_{op}")
                fn.restype = C.c_int
                fn.argtypes = [_vp, _vp, _sz, _sz, _sz, ct, _u, _u, _u]
    for fl, sl in (("d2q9", "d2q5"), ("d3q19", "d3q7"), ("d3q27", "d3q7")):
        for real, ct in (("float", C.c_float), ("double", C.c_double)):
            fn = getattr(lib, f"lbm_launch_scalar_step_gpu_{fl}_{sl}_{real}")
            fn.restype = C.c_int
            fn.argtypes = [_vp, _vp, _vp, _sz, _sz, _sz, ct, ct, _u, _u, _u]
            fn = getattr(lib, f"lbm_launch_reaction_ab_gpu_{fl}_{sl}_{real}")
            fn.restype = C.c_int
            fn.argtypes = [_vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, ct, ct, _u, _u, _u]
    d = C.c_double
    sig = {
        "lbm_step_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, d, _vp],
        "lbm_scalar_step_async": [C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, d, d, _vp],
        "lbm_reaction_ab_async": [C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, d, d, _vp],
        "lbm_fluid_reaction_ab_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                        _sz, _sz, _sz, d, d, d, _vp, _sz, _vp],
        "lbm_reactive_stats_async": [C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, d, _vp, _sz, _vp, _vp],
        "lbm_reactive_stats_finalize_async": [C.c_int, C.c_int, _sz, _sz, _sz, d, _vp, _sz, _vp, _vp],
        "lbm_init_equilibrium_async": [C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, _vp],
        "lbm_step_shifted_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_float,
                                   C.c_float, _vp],
        "lbm_encode_shifted_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_float, _vp],
        "lbm_decode_shifted_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_float, _vp],
        "lbm_ke_gradient_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, d, C.c_int, C.c_int,
                                  _vp, _sz, _vp, _vp, _vp],
        "lbm_adjoint_step_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, d, _vp, _vp],
        "lbm_reactive_gradient_async": [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, _vp, _vp, _vp,
                                        _vp, _sz, _sz, _sz, d, d, d, C.c_int, C.c_int, _vp, _sz, _vp, _vp,
                                        _vp, _vp, _vp],
        "lbm_fluid_reaction_ab_shifted_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _sz,
                                                _sz, _sz, d, d, d, C.c_float, C.c_float, _vp, _sz, _vp],
        "lbm_step_slab_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, d, _vp, _vp, _vp, _vp, _sz,
                                _sz, _vp],
        "lbm_slab_pack_async": [C.c_int, C.c_int, _vp, _sz, _sz, _sz, _vp, _vp, _vp],
        "lbm_step_slab_shifted_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_float,
                                        C.c_float, _vp, _vp, _vp, _vp, _sz, _sz, _vp],
        "lbm_slab_pack_shifted_async": [C.c_int, _vp, _sz, _sz, _sz, _vp, _vp, _vp],
        "lbm_fluid_reaction_slab_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _sz,
                                          _sz, d, d, d, _vp, _vp, _vp, _vp, _sz, _sz, _vp, _sz, _vp],
        "lbm_fluid_reaction_slab_pack_async": [C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, _vp, _vp, _vp],
        "lbm_reactive_stats_sums_async": [C.c_int, _sz, _sz, _sz, _vp, _sz, _vp, _vp],
        "lbm_reactive_slab_pack_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, _vp, _vp, _vp],
        "lbm_reactive_slab_forward_async": [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _vp, _vp, _vp, _vp,
                                            _vp, _vp, _vp, _sz, _sz, _sz, d, d, d, _vp, _vp, _vp, _vp, _vp],
        "lbm_reactive_slab_adjoint_step_async": [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _vp, _vp, _vp,
                                                 _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz,
                                                 _sz, _sz, d, d, d, _vp, _sz, _vp],
        "lbm_reactive_slab_adjoint_unpack_async": [C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz,
                                                   _vp],
        "lbm_reactive_slab_seed_async": [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _vp, _vp, _vp, _vp, _vp,
                                         _vp, _vp, _sz, _sz, _sz, d, _vp, _sz, _vp],
        "lbm_reactive_slab_init_gradients_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                   _sz, _sz, _sz, d, _vp, _vp, _vp, _vp],
        "lbm_reactive_slab_sums_async": [C.c_int, _sz, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _vp],
        "lbm_reactive_slab_result_async": [C.c_int, C.c_int, _vp, _vp, d, d, _vp, _vp],
        "lbm_reactive_stats_append_async": [C.c_int, C.c_int, _sz, _sz, _sz, d, _vp, _sz, _vp, _sz, _vp, _vp],
        "lbm_reactive_stats_from_sums_async": [C.c_int, _vp, d, d, _vp, _vp],
        "lbm_macro_fields_async": [C.c_int, C.c_int, _vp, _sz, _sz, _sz, _vp, _vp, _vp, _vp],
        "lbm_write_vtk_legacy": [C.c_char_p, C.c_int, _sz, _sz, _sz, _sz, C.c_int, _vp, _vp, _vp],
        "lbm_write_populations": [C.c_char_p, C.c_int, C.c_int, _sz, _sz, _sz, _sz, _vp],
        "lbm_read_populations": [C.c_char_p, C.c_int, C.c_int, _sz, _sz, _sz, C.POINTER(C.c_size_t), _vp],
        "lbm_fluid_diagnostics_async": [C.c_int, C.c_int, _vp, _sz, _sz, _sz, d, _vp, _sz, _vp, _vp],
        "lbm_step_diagnostics_async": [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, d, d, _vp, _sz,
                                       _vp, _vp],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = args
    lib.lbm_stats_partials_bytes.restype = C.c_size_t
    lib.lbm_stats_partials_bytes.argtypes = [C.c_int, _sz, _sz, _sz]
    lib.lbm_slab_face_elems.restype = C.c_size_t
    lib.lbm_slab_face_elems.argtypes = [C.c_int, _sz, _sz]
    lib.lbm_fluid_reaction_slab_face_elems.restype = C.c_size_t
    lib.lbm_fluid_reaction_slab_face_elems.argtypes = [C.c_int, _sz, _sz]
    lib.lbm_reactive_gradient_workspace_bytes.restype = C.c_size_t
    lib.lbm_reactive_gradient_workspace_bytes.argtypes = [C.c_int, C.c_int, C.c_int, _sz, _sz, _sz, C.c_int,
                                                          C.c_int]
    lib.lbm_diagnostics_partials_bytes.restype = C.c_size_t
    lib.lbm_diagnostics_partials_bytes.argtypes = [C.c_int, _sz, _sz, _sz]
    lib.lbm_ke_gradient_workspace_bytes.restype = C.c_size_t
    lib.lbm_ke_gradient_workspace_bytes.argtypes = [C.c_int, C.c_int, _sz, _sz, _sz, C.c_int, C.c_int]
    lib.lbm_copy_buffers_async.restype = C.c_int
    lib.lbm_copy_buffers_async.argtypes = [C.c_int, C.POINTER(_vp), C.POINTER(_vp), _sz, _vp]
    for name in ("lbm_reactive_slab_slots_bytes", "lbm_reactive_slab_objective_bytes"):
        getattr(lib, name).restype = C.c_size_t
        getattr(lib, name).argtypes = [C.c_int, _sz, _sz, _sz]
    lib.lbm_stage_timeouts.restype = C.c_uint
    lib.lbm_stage_timeouts.argtypes = [C.c_int]


def copy_buffers_async(src, dst, nbytes, stream=None) -> int:
    """Copies device buffers src[i] -> dst[i] (nbytes each, at most 64 pairs) in one launch."""
    n = len(src)
    arr = (C.c_void_p * max(n, 1))
    return load().lbm_copy_buffers_async(n, arr(*[_ptr(b) for b in src]), arr(*[_ptr(b) for b in dst]),
                                         int(nbytes), _stream(stream))


def _ptr(buf):
    if buf is None:
        return None
    if isinstance(buf, int):
        return buf
    return buf.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def real_name(dtype) -> str:
    s = str(dtype)
    if "float32" in s or s == "float":
        return "float"
    if "float64" in s or s == "double":
        return "double"
    raise ValueError(f"unsupported precision {dtype}")


def check(code: int, what: str = "launch") -> None:
    if code != cudaSuccess:
        raise LbmCudaError(what, code)


# --------------------------------------------------------------------------
# Reference-named launchers (return the cudaError_t code, like the reference)
# --------------------------------------------------------------------------
def launch_step_gpu(lattice, real, collision, current_populations, next_populations, x_extent,
                    y_extent, z_extent, omega, block=(16, 8, 1)) -> int:
    """lbm::launch_step_gpu<Lattice, Real, CT> (include/lattice_cuda.cuh:179-190)."""
    fn = getattr(load(), f"lbm_launch_step_gpu_{lattice.lower()}_{real_name(real)}_{collision.lower()}")
    return fn(_ptr(current_populations), _ptr(next_populations), x_extent, y_extent, z_extent,
              omega, *block)


def launch_step_gpu_mem(lattice, real, collision, mem_extents, current_populations,
                        next_populations, omega, block=(16, 8, 1)) -> int:
    """The LatticeMemory overload (include/lattice_cuda.cuh:310-319): extents from a memory object."""
    nx, ny, nz = mem_extents
    return launch_step_gpu(lattice, real, collision, current_populations, next_populations, nx, ny,
                           nz, omega, block)


def launch_scalar_step_gpu(fluid_lattice, real, current_scalar, next_scalar, current_fluid,
                           x_extent, y_extent, z_extent, omega_c, source_term=0.0,
                           block=(16, 8, 1)) -> int:
    """lbm::launch_scalar_step_gpu<FL, SL, Real> (include/lattice_cuda.cuh:209-222)."""
    sl = SCALAR_OF[fluid_lattice].lower()
    fn = getattr(load(), f"lbm_launch_scalar_step_gpu_{fluid_lattice.lower()}_{sl}_{real_name(real)}")
    return fn(_ptr(current_scalar), _ptr(next_scalar), _ptr(current_fluid), x_extent, y_extent,
              z_extent, omega_c, source_term, *block)


def launch_scalar_step_gpu_mem(fluid_lattice, real, scalar_extents, fluid_extents, current_scalar,
                               next_scalar, current_fluid, omega_c, source_term=0.0,
                               block=(16, 8, 1)) -> int:
    """The LatticeMemory overload (include/lattice_cuda.cuh:243-255, src/lattice_cuda.cu:716-747):
    mismatched scalar/fluid extents return cudaErrorInvalidValue."""
    if tuple(scalar_extents) != tuple(fluid_extents):
        return cudaErrorInvalidValue
    nx, ny, nz = scalar_extents
    return launch_scalar_step_gpu(fluid_lattice, real, current_scalar, next_scalar, current_fluid,
                                  nx, ny, nz, omega_c, source_term, block)


def launch_reaction_AB_gpu(fluid_lattice, real, current_a, next_a, current_b, next_b,
                           current_fluid, x_extent, y_extent, z_extent, omega_c, k_react,
                           block=(16, 8, 1)) -> int:
    """lbm::launch_reaction_AB_gpu<FL, SL, Real> (include/lattice_cuda.cuh:276-291)."""
    sl = SCALAR_OF[fluid_lattice].lower()
    fn = getattr(load(), f"lbm_launch_reaction_ab_gpu_{fluid_lattice.lower()}_{sl}_{real_name(real)}")
    return fn(_ptr(current_a), _ptr(next_a), _ptr(current_b), _ptr(next_b), _ptr(current_fluid),
              x_extent, y_extent, z_extent, omega_c, k_react, *block)


# --------------------------------------------------------------------------
# Stream-ordered extensions
# --------------------------------------------------------------------------
def step_async(lattice, real, collision, cur, nxt, nx, ny, nz, omega, stream=None) -> int:
    return load().lbm_step_async(LATTICES[lattice], REALS[real_name(real)], COLLISIONS[collision],
                                 _ptr(cur), _ptr(nxt), nx, ny, nz, float(omega), _stream(stream))


def scalar_step_async(fluid_lattice, real, cur_s, nxt_s, cur_f, nx, ny, nz, omega_c, source=0.0,
                      stream=None) -> int:
    return load().lbm_scalar_step_async(LATTICES[fluid_lattice], REALS[real_name(real)], _ptr(cur_s),
                                        _ptr(nxt_s), _ptr(cur_f), nx, ny, nz, float(omega_c),
                                        float(source), _stream(stream))


def reaction_ab_async(fluid_lattice, real, cur_a, nxt_a, cur_b, nxt_b, cur_f, nx, ny, nz, omega_c,
                      k_react, stream=None) -> int:
    return load().lbm_reaction_ab_async(LATTICES[fluid_lattice], REALS[real_name(real)], _ptr(cur_a),
                                        _ptr(nxt_a), _ptr(cur_b), _ptr(nxt_b), _ptr(cur_f), nx, ny,
                                        nz, float(omega_c), float(k_react), _stream(stream))


def stats_partials_bytes(fluid_lattice, nx, ny, nz) -> int:
    return load().lbm_stats_partials_bytes(LATTICES[fluid_lattice], nx, ny, nz)


def fluid_reaction_ab_async(fluid_lattice, real, collision, cur_f, nxt_f, cur_a, nxt_a, cur_b, nxt_b,
                            nx, ny, nz, omega, omega_c, k_react, partials=None, partials_bytes=0,
                            stream=None) -> int:
    return load().lbm_fluid_reaction_ab_async(
        LATTICES[fluid_lattice], REALS[real_name(real)], COLLISIONS[collision], _ptr(cur_f),
        _ptr(nxt_f), _ptr(cur_a), _ptr(nxt_a), _ptr(cur_b), _ptr(nxt_b), nx, ny, nz, float(omega),
        float(omega_c), float(k_react), _ptr(partials), int(partials_bytes), _stream(stream))


def fluid_reaction_ab_shifted_async(fluid_lattice, fmt, collision, cur_f, nxt_f, cur_a, nxt_a, cur_b,
                                    nxt_b, nx, ny, nz, omega, omega_c, k_react, rho0=1.0, c0=0.5,
                                    partials=None, partials_bytes=0, stream=None) -> int:
    """The coupled fluid + A + B -> C step on shifted 16-bit populations."""
    return load().lbm_fluid_reaction_ab_shifted_async(
        LATTICES[fluid_lattice], FORMATS[fmt], COLLISIONS[collision], _ptr(cur_f), _ptr(nxt_f), _ptr(cur_a),
        _ptr(nxt_a), _ptr(cur_b), _ptr(nxt_b), nx, ny, nz, float(omega), float(omega_c), float(k_react),
        float(rho0), float(c0), _ptr(partials), int(partials_bytes), _stream(stream))


def reactive_stats_async(scalar_lattice, real, a, b, nx, ny, nz, k_react, partials, partials_bytes,
                         diagnostics, stream=None) -> int:
    return load().lbm_reactive_stats_async(LATTICES[scalar_lattice], REALS[real_name(real)], _ptr(a),
                                           _ptr(b), nx, ny, nz, float(k_react), _ptr(partials),
                                           int(partials_bytes), _ptr(diagnostics), _stream(stream))


def reactive_stats_append_async(fluid_lattice, real, nx, ny, nz, k_react, partials, partials_bytes, table,
                                table_rows, row_counter, stream=None) -> int:
    return load().lbm_reactive_stats_append_async(LATTICES[fluid_lattice], REALS[real_name(real)], nx, ny, nz,
                                                  float(k_react), _ptr(partials), int(partials_bytes),
                                                  _ptr(table), int(table_rows), _ptr(row_counter),
                                                  _stream(stream))


def reactive_stats_finalize_async(fluid_lattice, real, nx, ny, nz, k_react, partials, partials_bytes,
                                  diagnostics, stream=None) -> int:
    return load().lbm_reactive_stats_finalize_async(LATTICES[fluid_lattice], REALS[real_name(real)],
                                                    nx, ny, nz,
                                                    float(k_react), _ptr(partials),
                                                    int(partials_bytes), _ptr(diagnostics),
                                                    _stream(stream))


def init_equilibrium_async(lattice, real, rho, u, populations, nx, ny, nz, stream=None) -> int:
    return load().lbm_init_equilibrium_async(LATTICES[lattice], REALS[real_name(real)], _ptr(rho),
                                             _ptr(u), _ptr(populations), nx, ny, nz, _stream(stream))


def step_shifted_async(lattice, fmt, collision, cur, nxt, nx, ny, nz, omega, rho0=1.0,
                       stream=None) -> int:
    """One collide-stream step on shifted 16-bit populations (fmt in FORMATS)."""
    return load().lbm_step_shifted_async(LATTICES[lattice], FORMATS[fmt], COLLISIONS[collision],
                                         _ptr(cur), _ptr(nxt), nx, ny, nz, float(omega),
                                         float(rho0), _stream(stream))



def stage_timeouts(reset: bool = False) -> int:
    """Blocks of the row-staged 16-bit step that gave up waiting for a row copy
    (0 in a healthy run); `reset` clears the count."""
    return int(load().lbm_stage_timeouts(1 if reset else 0))

def encode_shifted_async(lattice, fmt, real, populations, shifted, nx, ny, nz, rho0=1.0,
                         stream=None) -> int:
    return load().lbm_encode_shifted_async(LATTICES[lattice], FORMATS[fmt], REALS[real_name(real)],
                                           _ptr(populations), _ptr(shifted), nx, ny, nz,
                                           float(rho0), _stream(stream))


def decode_shifted_async(lattice, fmt, real, shifted, populations, nx, ny, nz, rho0=1.0,
                         stream=None) -> int:
    return load().lbm_decode_shifted_async(LATTICES[lattice], FORMATS[fmt], REALS[real_name(real)],
                                           _ptr(shifted), _ptr(populations), nx, ny, nz,
                                           float(rho0), _stream(stream))


def ke_gradient_workspace_bytes(lattice, real, nx, ny, nz, steps, interval) -> int:
    return load().lbm_ke_gradient_workspace_bytes(LATTICES[lattice], REALS[real_name(real)], nx, ny,
                                                  nz, int(steps), int(interval))


def ke_gradient_async(lattice, real, collision, rho0, u0, nx, ny, nz, tau, steps, interval,
                      workspace, workspace_bytes, out2, grad_u0, stream=None) -> int:
    """Checkpointed adjoint of J = sum 0.5 rho |u|^2 after `steps` steps from
    f_eq(rho0, u0): out2 = [J, dJ/dtau] (device FP64), grad_u0 = dJ/du0."""
    return load().lbm_ke_gradient_async(LATTICES[lattice], REALS[real_name(real)], COLLISIONS[collision],
                                        _ptr(rho0), _ptr(u0), nx, ny, nz, float(tau), int(steps),
                                        int(interval), _ptr(workspace), int(workspace_bytes),
                                        _ptr(out2), _ptr(grad_u0), _stream(stream))


def adjoint_step_async(lattice, real, collision, populations, lambda_next, lam, nx, ny, nz, tau,
                       dtau_slots=None, stream=None) -> int:
    return load().lbm_adjoint_step_async(LATTICES[lattice], REALS[real_name(real)], COLLISIONS[collision],
                                         _ptr(populations), _ptr(lambda_next), _ptr(lam), nx, ny, nz,
                                         float(tau), _ptr(dtau_slots), _stream(stream))


OBJECTIVES = {"mean_product": 0, "segregation": 1}


def _storage(storage):
    return 0 if storage in (None, "native") else FORMATS[storage]


def reactive_gradient_workspace_bytes(fluid_lattice, real, nx, ny, nz, steps, interval, storage=None) -> int:
    return load().lbm_reactive_gradient_workspace_bytes(LATTICES[fluid_lattice], REALS[real_name(real)],
                                                        _storage(storage), nx, ny, nz, int(steps), int(interval))


def reactive_gradient_async(fluid_lattice, real, collision, objective, rho0, u0, a0, b0, nx, ny, nz,
                            tau, tau_c, k_react, steps, interval, workspace, workspace_bytes, result,
                            grad_a0, grad_b0=None, grad_u0=None, storage=None, c0=0.5, stream=None) -> int:
    """Checkpointed adjoint of the coupled fluid + A + B -> C run: result
    (device FP64[4]) = J, dJ/dk, dJ/dtau, dJ/dtau_c; grad_a0 (grad_b0,
    grad_u0) = dJ/da0 (dJ/db0, dJ/du0). objective in OBJECTIVES; storage None
    (states in `real`) or a 16-bit format of FORMATS (scalars shifted by c0)."""
    return load().lbm_reactive_gradient_async(
        LATTICES[fluid_lattice], REALS[real_name(real)], _storage(storage), float(c0), COLLISIONS[collision],
        OBJECTIVES[objective],
        _ptr(rho0), _ptr(u0), _ptr(a0), _ptr(b0), nx, ny, nz, float(tau), float(tau_c), float(k_react),
        int(steps), int(interval), _ptr(workspace), int(workspace_bytes), _ptr(result), _ptr(grad_a0),
        _ptr(grad_b0), _ptr(grad_u0), _stream(stream))


def macro_fields_async(lattice, real, populations, nx, ny, nz, density, velocity=None, speed=None,
                       stream=None) -> int:
    """Density (concentration for scalars), velocity [D, ...] and |u| on the
    device, in the population precision."""
    return load().lbm_macro_fields_async(LATTICES[lattice], REALS[real_name(real)], _ptr(populations), nx,
                                         ny, nz, _ptr(density), _ptr(velocity), _ptr(speed), _stream(stream))


def _host(a):
    """Host address of a contiguous numpy array or CPU tensor."""
    if hasattr(a, "ctypes"):
        assert a.flags.c_contiguous
        return a.ctypes.data
    assert not a.is_cuda and a.is_contiguous()
    return a.data_ptr()


def write_vtk_legacy(path, dims, nx, ny, nz, step, real, density, velocity, speed) -> int:
    """The reference's legacy ASCII VTK file from host macroscopic fields."""
    return load().lbm_write_vtk_legacy(os.fsencode(path), int(dims), nx, ny, nz, int(step),
                                       REALS[real_name(real)], _host(density), _host(velocity), _host(speed))


def write_populations(path, lattice, real, nx, ny, nz, step, populations) -> int:
    return load().lbm_write_populations(os.fsencode(path), LATTICES[lattice], REALS[real_name(real)], nx, ny,
                                        nz, int(step), _host(populations))


def read_populations(path, lattice, real, nx, ny, nz, out):
    """Fills host array ``out``; returns (code, stored time step)."""
    st = C.c_size_t(0)
    rc = load().lbm_read_populations(os.fsencode(path), LATTICES[lattice], REALS[real_name(real)], nx, ny,
                                     nz, C.byref(st), _host(out))
    return rc, st.value


IO_ERRORS = {"bad_argument": 1, "open_failed": 2, "write_failed": 3, "bad_file": 4, "mismatch": 5}


def diagnostics_partials_bytes(lattice, nx, ny, nz) -> int:
    return load().lbm_diagnostics_partials_bytes(LATTICES[lattice], nx, ny, nz)


def fluid_diagnostics_async(lattice, real, populations, nx, ny, nz, partials, partials_bytes,
                            diagnostics, speed_limit=math.inf, stream=None) -> int:
    """diagnostics (device FP64[5]) = total mass, total kinetic energy, max |u|,
    non-finite cells, blow-up flag (non-finite |u| or max |u| > speed_limit)."""
    return load().lbm_fluid_diagnostics_async(LATTICES[lattice], REALS[real_name(real)],
                                              _ptr(populations), nx, ny, nz, float(speed_limit),
                                              _ptr(partials), int(partials_bytes),
                                              _ptr(diagnostics), _stream(stream))


def step_diagnostics_async(lattice, real, collision, cur, nxt, nx, ny, nz, omega, partials,
                           partials_bytes, diagnostics, speed_limit=math.inf, stream=None) -> int:
    """One collide-stream step plus the diagnostics of the state it writes."""
    return load().lbm_step_diagnostics_async(LATTICES[lattice], REALS[real_name(real)],
                                             COLLISIONS[collision], _ptr(cur), _ptr(nxt), nx, ny, nz,
                                             float(omega), float(speed_limit), _ptr(partials),
                                             int(partials_bytes), _ptr(diagnostics), _stream(stream))


def declared_symbols(header: str = HEADER):
    """Names of every function the C ABI header declares."""
    import re
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^(?:int|size_t)\s+(lbm_\w+)\s*\(", text, flags=re.M)))

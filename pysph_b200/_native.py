"""ctypes binding of libsphb.so (include/sphb.h).

The structures below mirror the C ABI field by field; tests/test_abi.py
checks their sizes and offsets against the header compiled by gcc.  Loading
fails loudly when the library is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsphb.so")

MAX_ARRAYS = 4
FP64, FP32C = 0, 1
BIN_MOVE_INITIAL, BIN_BOX = 1, 2

OK = 0
ERRORS = {-1: "bad argument", -2: "workspace too small", -3: "CUDA launch failed",
          -4: "unsupported configuration"}

ST_GRID_OVERFLOW = 1 << 0
ST_NONFINITE_POS = 1 << 1
ST_OUT_OF_GRID = 1 << 2
ST_NONFINITE_RHO = 1 << 3
ST_NONFINITE_ACC = 1 << 4
ST_BAD_INDEX = 1 << 5
ST_NBR_CAPACITY = 1 << 6
ST_STAGE_TIMEOUT = 1 << 7
BIN_IF_NEEDED = 4
BIN_STEP_BEGIN = 8     # the first bin of a step runs the step prologue too
DENSITY_LIST_IF_VALID = 4
DENSITY_LISTS_ONLY = 8
STATUS_NAMES = {
    ST_GRID_OVERFLOW: "cell grid larger than cell_capacity",
    ST_NONFINITE_POS: "non-finite particle position",
    ST_OUT_OF_GRID: "particle outside its scene grid",
    ST_NONFINITE_RHO: "non-finite density or pressure",
    ST_NONFINITE_ACC: "non-finite acceleration",
    ST_BAD_INDEX: "index failed a bounds check",
    ST_NBR_CAPACITY: "neighbour list output too small",
    ST_STAGE_TIMEOUT: "shared-memory staging of a tiled pass timed out",
}

# engine field ids of sphb_exchange
FIELDS = {"x": 0, "y": 1, "z": 2, "u": 3, "v": 4, "w": 5,
          "_x0": 6, "_y0": 7, "_z0": 8, "_u0": 9, "_v0": 10, "_w0": 11,
          "m": 12, "h": 13, "rho": 14, "p": 15, "cs": 16,
          "_a_u_1": 17, "_a_v_1": 18, "_a_w_1": 19, "dt_fac": 20,
          # continuity scheme: the integrated density, its stage-initial copy
          # and its rate (_a_rho_1, scatter only)
          "rho_state": 21, "_rho0": 22, "_a_rho_1": 23,
          # XSPHCorrection velocity (scatter only)
          "_xsph_u": 24, "_xsph_v": 25, "_xsph_w": 26}

i32, u32, f64, vp = ctypes.c_int32, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p
u64, i64 = ctypes.c_uint64, ctypes.c_int64


class Config(ctypes.Structure):
    _fields_ = [("dim", i32), ("precision", i32), ("num_scenes", i32),
                ("num_arrays", i32), ("stencil", i32), ("lanes", i32),
                ("pair_block", i32), ("num_particles", i32),
                ("cell_capacity", i32), ("list_batch", i32),
                ("rho_src", u32 * MAX_ARRAYS), ("mom_src", u32 * MAX_ARRAYS),
                ("tait_on", u32), ("step_on", u32),
                ("rate_src", u32 * MAX_ARRAYS), ("xsph_src", u32 * MAX_ARRAYS),
                ("kernel", i32), ("pair_mode", i32)]

# smoothing kernels (KernelBase.get_type ids) and their support radii
KERNEL_CUBIC, KERNEL_QUINTIC, KERNEL_WENDLAND = 1, 3, 4
KERNEL_RADIUS = {KERNEL_CUBIC: 2.0, KERNEL_QUINTIC: 3.0, KERNEL_WENDLAND: 2.0}


class Scene(ctypes.Structure):
    _fields_ = [("cell_size", f64), ("radius_scale", f64), ("h_min", f64),
                ("c0", f64), ("rho0", f64), ("gamma", f64), ("B", f64),
                ("alpha", f64), ("beta", f64), ("eta", f64), ("g", f64 * 3),
                ("cfl", f64), ("dt_initial", f64), ("static_lo", f64 * 3),
                ("static_hi", f64 * 3), ("use_cfl", i32), ("uniform_h", i32),
                ("skin_max", f64), ("xsph_eps", f64),
                ("variable_h", i32), ("hks", i32)]


class SceneState(ctypes.Structure):
    _fields_ = [("lo", i32 * 3), ("n", i32 * 3), ("cell_base", i32),
                ("ncells", i32), ("box", u64 * 6), ("dt", f64), ("t", f64),
                ("count", i64), ("max_dtfac", u64), ("max_acc2", u64), ("max_disp2", u64)]


class Tile(ctypes.Structure):
    _fields_ = [("seg", i32), ("begin", i32), ("end", i32), ("pad0", i32)]


BUFFER_FIELDS = ("x", "y", "z", "u", "v", "w", "x0", "y0", "z0", "u0", "v0",
                 "w0", "m", "h", "idx", "tag", "rho", "rho0",
                 "kx", "ky", "kz", "ku", "kv", "kw", "krho")


ABI_VERSION = 2


class Buffers(ctypes.Structure):
    _fields_ = [(n, vp) for n in BUFFER_FIELDS]


FIELD_NAMES = ("rho", "p", "cs", "au", "av", "aw", "dt_fac", "geo", "mass",
               "vel", "thermo", "cell", "nbr", "nbr_cnt", "anchor", "drho", "xu", "xv", "xw",
               "geo_next", "vel_next")
FORCE_USE_LIST = 16
# cfg.pair_mode: neighbour lists (0) or shared-memory tiles (1)
PAIRS_LISTS, PAIRS_TILED = 0, 1
FORCE_NO_MAXIMA = 32


def FORCE_STAGE(kind: int) -> int:
    """sphb_momentum mode bits of the fused integrator stage `kind`."""
    return (kind + 1) << 8

DENSITY_EOS = 1
DENSITY_USE_LIST = 2


class Fields(ctypes.Structure):
    _fields_ = [(n, vp) for n in FIELD_NAMES] + [("list_cap", i32), ("pad0", i32)]


WORK_NAMES = ("count", "start", "key", "slot", "perm", "bsum", "meta",
              "status", "pairs")


class Work(ctypes.Structure):
    _fields_ = [(n, vp) for n in WORK_NAMES]


class EngineDesc(ctypes.Structure):
    _fields_ = [("cfg", Config), ("seg_offset", vp), ("scene", vp),
                ("sstate", vp), ("tiles", vp), ("pair_tiles", vp),
                ("num_tiles", i32), ("num_pair_tiles", i32),
                ("buf", Buffers * 2), ("f", Fields), ("work", Work)]


_lib = None


def lib():
    """Load libsphb.so; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m pysph_b200.build` "
            "(the CUDA engine has no fallback)")
    L = ctypes.CDLL(LIB_PATH)
    E = ctypes.POINTER(EngineDesc)
    sig = {
        "sphb_abi_version": (i32, []),
        "sphb_last_cuda_error": (ctypes.c_char_p, []),
        "sphb_make_tiles": (i32, [vp, i32, i32, vp, ctypes.POINTER(i32)]),
        "sphb_workspace_layout": (i32, [ctypes.POINTER(Config),
                                        ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_size_t)]),
        "sphb_box_init": (i32, [E, i32, vp]),
        "sphb_bin": (i32, [E, i32, i32, vp]),
        "sphb_neighbors": (i32, [E, i32, u32, u32, vp, vp, vp, i64, vp]),
        "sphb_cell_coords": (i32, [E, i32, vp, vp]),
        "sphb_density": (i32, [E, i32, u32, i32, vp]),
        "sphb_tait": (i32, [E, i32, u32, vp]),
        "sphb_momentum": (i32, [E, i32, u32, i32, i32, vp]),
        "sphb_pc_stage": (i32, [E, i32, i32, vp]),
        "sphb_step_begin": (i32, [E, vp]),
        "sphb_exchange": (i32, [E, i32, i32, i32, i32, vp, vp, vp]),
        "sphb_exchange_many": (i32, [E, i32, i32, i32, i32, vp, vp, vp, vp]),
        "sphb_exchange_tag": (i32, [E, i32, i32, i32, vp, vp, vp]),
        "sphb_init_index": (i32, [E, i32, vp]),
        "sphb_set_dt": (i32, [E, f64, vp]),
        "sphb_refresh": (i32, [E, i32, vp]),
        "sphb_permute": (i32, [E, i32, i32, i32, vp, vp, vp, vp]),
        "sphb_force_vjp": (i32, [E, i32, u32, vp, vp, vp, vp, vp, vp, vp]),
        "sphb_eos_vjp": (i32, [E, i32, vp, vp, vp, vp]),
        "sphb_density_vjp": (i32, [E, i32, u32, vp, vp, vp]),
        "sphb_neighbor_counts_static": (i32, [i32, i32, vp, vp, vp, vp, f64, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.sphb_abi_version() != ABI_VERSION:
        raise RuntimeError("libsphb.so ABI version mismatch")
    _lib = L
    return L


EXPORTED = ("sphb_abi_version", "sphb_last_cuda_error", "sphb_make_tiles",
            "sphb_workspace_layout", "sphb_box_init", "sphb_bin",
            "sphb_neighbors", "sphb_cell_coords", "sphb_density", "sphb_tait",
            "sphb_momentum", "sphb_pc_stage", "sphb_step_begin",
            "sphb_exchange", "sphb_exchange_many", "sphb_exchange_tag", "sphb_init_index",
            "sphb_set_dt", "sphb_refresh", "sphb_permute", "sphb_force_vjp", "sphb_eos_vjp",
            "sphb_density_vjp", "sphb_neighbor_counts_static")

STATIC_MAX_PARTICLES = 1 << 18
EXCHANGE_MAX = 8


def check(rc: int, what: str):
    if rc != OK:
        msg = ERRORS.get(rc, f"error {rc}")
        if rc == -3:
            msg += ": " + lib().sphb_last_cuda_error().decode()
        raise RuntimeError(f"{what} failed: {msg}")


def status_message(bits: int) -> str:
    return ", ".join(v for k, v in STATUS_NAMES.items() if bits & k)

"""ctypes binding of libfoilb200.so (declarations in include/foilb200.h).

The library is the only compute path: importing a solver or operator without the built
shared object, or calling one without a CUDA device, raises immediately. There is no
CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import numpy as np

LIB_NAME = "libfoilb200.so"
# the in-tree build; FOILB200_LIBRARY names another build of the same library (same ABI)
LIB_PATH = Path(os.environ.get("FOILB200_LIBRARY") or (Path(__file__).resolve().parent / LIB_NAME))

FB_OK = 0
FB_ERR_INVALID_ARGUMENT = 1
FB_ERR_CUDA = 2
FB_ERR_OUT_OF_MEMORY = 3
FB_ERR_NOT_INITIALIZED = 4
FB_ERR_NUMERICAL = 5
FB_ERR_DEVICE_TIMEOUT = 6
FB_ERR_BUDGET = 7

FLOAT32, FLOAT64 = 0, 1
PRESSURE_REFERENCE, PRESSURE_MIXED = 0, 1
ROW_TRANSFORM_AUTO, ROW_TRANSFORM_FFT, ROW_TRANSFORM_TENSOR = 0, 1, 2
ADVECT_SEMI_LAGRANGIAN, ADVECT_MACCORMACK, ADVECT_SKEW_RK2 = 0, 1, 2
IC_FREESTREAM, IC_TAYLOR_GREEN, IC_POISEUILLE = 0, 1, 2

REASONS = {
    0: "none",
    1: "excessive_velocity",
    2: "stability_limit",
    3: "nonfinite_state",
    4: "convergence_failure",
    5: "projection_failure",
    6: "postcondition_failure",
    7: "time_contract_failure",
}
STAGES = {
    0: "postcondition",
    1: "advection",
    2: "viscosity",
    3: "projection",
    4: "boundary",
    5: "postcondition",
    6: "canonical-import",
    7: "time-mapping",
}
TRACE_TAGS = {
    0: "start", 1: "init/faces->cells/mask", 2: "advection", 3: "maccormack", 4: "jacobi", 5: "faces+guard",
    6: "boundaries", 7: "rhs", 8: "cg update+row DST", 9: "cg column solve", 10: "cg row DST", 11: "cg p/Ap",
    12: "defect correction", 13: "true residual", 14: "gradient", 15: "final checks", 16: "viscosity scale",
    17: "mixed init", 18: "mean removal", 19: "face transport", 20: "cg update", 21: "cg row DST 1 (tensor cores)",
    22: "cg row DST 2 (tensor cores)", 63: "end",
}
DIAGNOSTIC_NAMES = (
    "kinetic_energy",
    "enstrophy",
    "divergence_l2",
    "divergence_linf",
    "solid_leakage",
    "wake_width",
    "recirculation_area",
)


class ScenarioDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("x0", ctypes.c_double),
        ("x1", ctypes.c_double),
        ("y0", ctypes.c_double),
        ("y1", ctypes.c_double),
        ("periodic_x", ctypes.c_int32),
        ("periodic_y", ctypes.c_int32),
        ("channel_walls", ctypes.c_int32),
        ("freestream_x", ctypes.c_double),
        ("freestream_y", ctypes.c_double),
        ("naca", ctypes.c_char * 4),
        ("chord", ctypes.c_double),
        ("pivot_x", ctypes.c_double),
        ("pivot_y", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("pressure_scheme", ctypes.c_int32),
        ("advection", ctypes.c_int32),
        ("initial_condition", ctypes.c_int32),
        ("reference_speed", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("pressure_tolerance", ctypes.c_double),
        ("pressure_max_iterations", ctypes.c_int32),
        ("pressure_fixed_iterations", ctypes.c_int32),
        ("mixed_inner_rtol", ctypes.c_double),
        ("divergence_limit", ctypes.c_double),
        ("leakage_limit", ctypes.c_double),
        ("passive_scalar", ctypes.c_int32),
        ("face_advection", ctypes.c_int32),
        ("row_transform", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 5),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("reason", ctypes.c_int32),
        ("stage", ctypes.c_int32),
        ("substeps", ctypes.c_int32),
        ("stability_retries", ctypes.c_int32),
        ("pressure_iterations", ctypes.c_int32),
        ("pressure_outer_iterations", ctypes.c_int32),
        ("pressure_converged", ctypes.c_int32),
        ("viscosity_iterations", ctypes.c_int32),
        ("viscosity_converged", ctypes.c_int32),
        ("total_pressure_iterations", ctypes.c_int32),
        ("reserved_i", ctypes.c_int32 * 5),
        ("max_speed", ctypes.c_double),
        ("wall_speed", ctypes.c_double),
        ("accepted_measure", ctypes.c_double),
        ("advective_rate", ctypes.c_double),
        ("boundary_sweep", ctypes.c_double),
        ("pressure_relative_residual", ctypes.c_double),
        ("viscosity_final_residual", ctypes.c_double),
        ("divergence_linf", ctypes.c_double),
        ("solid_leakage", ctypes.c_double),
        ("required_substeps", ctypes.c_double),
        ("evidence", ctypes.c_double * 6),
        ("device_ms", ctypes.c_double),
        ("kernel_launches", ctypes.c_int32),
        ("reserved_j", ctypes.c_int32 * 3),
    ]

    @property
    def reason_name(self) -> str:
        return REASONS.get(self.reason, "none")

    @property
    def stage_name(self) -> str:
        return STAGES.get(self.stage, "postcondition")


_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_U8P = ctypes.POINTER(ctypes.c_uint8)
_I32 = ctypes.c_int32
_SIG = {
    "fb_abi_version": (_I32, []),
    "fb_abi_struct_sizes": (_I32, [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "fb_last_error": (ctypes.c_char_p, []),
    "fb_device_count": (_I32, [ctypes.POINTER(_I32)]),
    "fb_ctx_create": (_I32, [_I32, ctypes.c_uint64, ctypes.POINTER(_P)]),
    "fb_ctx_destroy": (_I32, [_P]),
    "fb_ctx_bytes_in_use": (_I32, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "fb_host_alloc": (_I32, [ctypes.c_uint64, ctypes.POINTER(_P)]),
    "fb_host_free": (_I32, [_P]),
    "fb_solver_create": (_I32, [_P, ctypes.POINTER(ScenarioDesc), ctypes.POINTER(_P)]),
    "fb_solver_destroy": (_I32, [_P]),
    "fb_solver_bytes": (_I32, [ctypes.POINTER(ScenarioDesc), ctypes.POINTER(ctypes.c_uint64)]),
    "fb_initialize": (_I32, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.POINTER(Report)]),
    "fb_restart": (_I32, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                          ctypes.POINTER(Report)]),
    "fb_set_viscosity": (_I32, [_P, ctypes.c_double]),
    "fb_update_options": (_I32, [_P, ctypes.POINTER(ScenarioDesc)]),
    "fb_advance": (_I32, [_P, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                          ctypes.POINTER(Report)]),
    "fb_export_velocity": (_I32, [_P, _P, ctypes.c_size_t, _I32]),
    "fb_export_faces": (_I32, [_P, _P, ctypes.c_size_t, _P, ctypes.c_size_t]),
    "fb_export_state": (_I32, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int64)]),
    "fb_export_pressure": (_I32, [_P, _DP, ctypes.c_size_t]),
    "fb_export_mask": (_I32, [_P, _U8P, ctypes.c_size_t]),
    "fb_export_scalar": (_I32, [_P, _P, ctypes.c_size_t]),
    "fb_import_scalar": (_I32, [_P, _P, ctypes.c_size_t]),
    "fb_import_velocity": (_I32, [_P, _P, ctypes.c_size_t, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.POINTER(Report)]),
    "fb_sample_velocity": (_I32, [_P, _DP, ctypes.c_int64, _DP]),
    "fb_diagnostics": (_I32, [_P, _DP, _I32]),
    "fb_get_pose": (_I32, [_P, _DP, _DP, _DP]),
    "fb_trace_enable": (_I32, [_P, _I32]),
    "fb_trace_read": (_I32, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "fb_debug_barrier_timeout": (_I32, [_P, _I32, ctypes.c_uint64]),
    "fb_autotune": (_I32, [_P, ctypes.c_double, _I32, _DP, _I32]),
    "fb_set_launch_shape": (_I32, [_P, _I32, _I32]),
    "fb_get_launch_shape": (_I32, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I32), _DP]),
    "fb_compute_mask": (_I32, [_P, ctypes.POINTER(ScenarioDesc), ctypes.c_double, _U8P, ctypes.c_size_t]),
    "fb_naca_signed_distance": (_I32, [_P, ctypes.c_char_p, ctypes.c_double, ctypes.c_double, ctypes.c_double, _DP,
                                       ctypes.c_int64, ctypes.c_double, _DP]),
    "fb_op_advect_velocity": (_I32, [_P, ctypes.POINTER(ScenarioDesc), _P, _P, ctypes.c_double, _I32]),
    "fb_op_implicit_diffuse": (_I32, [_P, ctypes.POINTER(ScenarioDesc), _P, _P, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, _I32, ctypes.POINTER(Report)]),
    "fb_op_solve_masked_poisson": (_I32, [_P, ctypes.POINTER(ScenarioDesc), _DP, _U8P, _DP, ctypes.POINTER(Report)]),
    "fb_op_project_faces": (_I32, [_P, ctypes.POINTER(ScenarioDesc), _P, _P, _U8P, ctypes.c_double, ctypes.c_double,
                                   ctypes.POINTER(Report)]),
    "fb_forces": (_I32, [_P, _DP, _I32]),
    "fb_batch_create": (_I32, [_P, ctypes.POINTER(_P), _I32, ctypes.POINTER(_P)]),
    "fb_batch_destroy": (_I32, [_P]),
    "fb_batch_ctas": (_I32, [_P, ctypes.POINTER(_I32), _I32]),
    "fb_batch_advance": (_I32, [_P, _DP, _DP, _DP, _DP, ctypes.POINTER(Report), ctypes.POINTER(_I32)]),
    "fb_op_implicit_diffuse_noalloc": (_I32, [_I32, ctypes.POINTER(ScenarioDesc), _P, _P, _P, _P, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_double, _I32, _P, ctypes.POINTER(Report)]),
}
EXPORTED_SYMBOLS = tuple(_SIG)

_lib = None
_lock = threading.Lock()
_contexts: dict[int, "Context"] = {}


class NativeError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[fb status {code}] {message}")
        self.code = code
        self.code = code


def load_library(path: str | os.PathLike | None = None):
    """Load libfoilb200.so (built in-tree by ``foilbench_b200.build``) and bind prototypes."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        target = Path(path) if path is not None else LIB_PATH
        if not target.exists():
            raise ImportError(
                f"{target} is missing: build the CUDA library with `python -m foilbench_b200.build` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(target))
        for name, (restype, argtypes) in _SIG.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        if lib.fb_abi_version() != 1:
            raise ImportError("libfoilb200.so ABI version mismatch")
        db, rb = ctypes.c_uint64(0), ctypes.c_uint64(0)
        lib.fb_abi_struct_sizes(ctypes.byref(db), ctypes.byref(rb))
        if db.value != ctypes.sizeof(ScenarioDesc) or rb.value != ctypes.sizeof(Report):
            raise ImportError(f"struct layout mismatch: desc {db.value} vs {ctypes.sizeof(ScenarioDesc)}, "
                              f"report {rb.value} vs {ctypes.sizeof(Report)}")
        if path is None:
            _lib = lib
        return lib


def lib():
    return load_library()


def check(code: int, what: str = "") -> None:
    if code != FB_OK:
        msg = lib().fb_last_error().decode("utf-8", "replace")
        raise NativeError(code, f"{what}: {msg}" if what else msg)


def device_count() -> int:
    n = ctypes.c_int32(0)
    code = lib().fb_device_count(ctypes.byref(n))
    return int(n.value) if code == FB_OK else 0


class Context:
    """One CUDA device and an HBM budget (bytes, 0 = unlimited)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        if device_count() <= 0:
            raise RuntimeError("no CUDA device is visible: the Stable Fluids step runs only on the GPU")
        handle = ctypes.c_void_p()
        check(lib().fb_ctx_create(int(device), int(hbm_budget), ctypes.byref(handle)), "fb_ctx_create")
        self.handle = handle
        self.device = device

    def bytes_in_use(self) -> int:
        n = ctypes.c_uint64(0)
        check(lib().fb_ctx_bytes_in_use(self.handle, ctypes.byref(n)))
        return int(n.value)

    def close(self) -> None:
        if self.handle:
            lib().fb_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


def default_context(device: int = 0) -> Context:
    with _lock:
        ctx = _contexts.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _contexts[device] = ctx
    return ctx


class _HostBlock:
    """One page-locked block of the library's host pool, returned to the pool when the last
    array viewing it is gone."""

    __slots__ = ("addr", "free", "__weakref__")

    def __init__(self, addr: int, free):
        self.addr = addr
        self.free = free

    def __del__(self):
        try:
            self.free(ctypes.c_void_p(self.addr))
        except Exception:  # interpreter shutdown
            pass


def host_array(shape, dtype) -> np.ndarray:
    """An uninitialised array in page-locked host memory from the library's pool (ordinary
    memory when the pool is full or no GPU is present): device-to-host copies into it need no
    staging and touch no fresh pages. It behaves as any numpy array; its block goes back to
    the pool with it."""
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    if nbytes == 0:
        return np.empty(shape, dtype=dt)
    p = ctypes.c_void_p()
    library = lib()
    if library.fb_host_alloc(nbytes, ctypes.byref(p)) != FB_OK:
        return np.empty(shape, dtype=dt)
    block = _HostBlock(p.value, library.fb_host_free)
    raw = (ctypes.c_char * nbytes).from_address(p.value)
    raw._block = block  # the ctypes view keeps the block alive; numpy keeps the view as its base
    return np.frombuffer(raw, dtype=dt).reshape(shape)


def ptr(array: np.ndarray):
    return ctypes.c_void_p(array.ctypes.data)


def dptr(array: np.ndarray):
    return array.ctypes.data_as(_DP)


def u8ptr(array: np.ndarray):
    return array.ctypes.data_as(_U8P)

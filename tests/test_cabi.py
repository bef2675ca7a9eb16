"""The C-ABI library loads, exports every symbol include/foilb200.h declares, and its
struct layouts match the ctypes binding. No device compute runs here."""

import ctypes
import re
from pathlib import Path

import pytest

from foilbench_b200 import _native as N

HEADER = Path(__file__).resolve().parents[1] / "include" / "foilb200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not N.LIB_PATH.exists():
        from foilbench_b200.build import build

        build()
    return N.load_library()


def test_header_declares_the_lifecycle_and_operator_entry_points():
    names = declared_functions()
    for must in ("fb_ctx_create", "fb_solver_create", "fb_initialize", "fb_restart", "fb_advance",
                 "fb_export_velocity", "fb_import_velocity", "fb_sample_velocity", "fb_diagnostics",
                 "fb_compute_mask", "fb_op_solve_masked_poisson", "fb_op_project_faces"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) == set(N.EXPORTED_SYMBOLS)


def test_abi_version_and_struct_layouts(lib):
    assert lib.fb_abi_version() == 1
    db, rb = ctypes.c_uint64(0), ctypes.c_uint64(0)
    assert lib.fb_abi_struct_sizes(ctypes.byref(db), ctypes.byref(rb)) == 0
    assert db.value == ctypes.sizeof(N.ScenarioDesc)
    assert rb.value == ctypes.sizeof(N.Report)


def test_solver_bytes_is_host_arithmetic(lib):
    from foilbench_b200.models import ControlKeyframe, DomainSpec, FoilSpec, Scenario
    from foilbench_b200.solver import scenario_desc

    sc = Scenario(1, "b", DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (2048, 1024)), 5000.0, (1.0, 0.0),
                  FoilSpec("2412", 1.0, (0.0, 0.0)), (ControlKeyframe(0.0, 15.0),), 1.0, 0.001, "float32", 0,
                  {"pressure_tolerance": 1e-6})
    d = scenario_desc(sc, "semi-lagrangian")
    n = ctypes.c_uint64(0)
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(n)) == 0
    cells = 2048 * 1024
    assert 40 * cells < n.value < 200 * cells
    # the tensor-core row transform's table and operand (AUTO picks the tensor cores here)
    d.row_transform = N.ROW_TRANSFORM_TENSOR
    tc = ctypes.c_uint64(0)
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(tc)) == 0
    assert tc.value == n.value
    d.row_transform = N.ROW_TRANSFORM_FFT
    fft = ctypes.c_uint64(0)
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(fft)) == 0
    kh = 1024
    assert tc.value - fft.value >= 2 * (2 * kh * kh * 4)
    d.row_transform = N.ROW_TRANSFORM_TENSOR
    d.pressure_scheme = N.PRESSURE_REFERENCE
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(n)) == N.FB_ERR_INVALID_ARGUMENT
    assert b"tensor-core row transform" in lib.fb_last_error()
    d.pressure_scheme = N.PRESSURE_MIXED
    d.row_transform = 3
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(n)) == N.FB_ERR_INVALID_ARGUMENT
    d.row_transform = N.ROW_TRANSFORM_AUTO
    # FP64 rows over 4096 columns: the split convolution's three filter slices and spectrum
    # scratch (2 x 8192 complex doubles for each of up to 256 CTAs) are part of the footprint
    d.pressure_scheme = N.PRESSURE_REFERENCE
    d.nx, d.ny = 4096, 16
    below = ctypes.c_uint64(0)
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(below)) == 0
    d.nx = 4100
    split = ctypes.c_uint64(0)
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(split)) == 0
    assert split.value - below.value >= 256 * 2 * 8192 * 16
    d.pressure_scheme = N.PRESSURE_MIXED
    d.nx = 2
    assert lib.fb_solver_bytes(ctypes.byref(d), ctypes.byref(n)) == N.FB_ERR_INVALID_ARGUMENT
    assert b"four cells" in lib.fb_last_error()

"""The allocation-free viscosity entry point against the allocating one.

fb_op_implicit_diffuse_noalloc serves callers that cannot let the library allocate device
memory: a simulation or viewer loop that owns every device byte through its own pool and
forbids driver allocations while it runs. The test gives it device buffers that it allocates
itself, through torch, calls it twice in a row on different fields through the C ABI, and
compares each result and its iteration count with fb_op_implicit_diffuse on the same input
(tolerance 1e-12 absolute in float64, 2e-6 in float32, as in the other viscosity parity
tests). It also checks that the caller's current device is left as it was, and that the
size limit sits exactly where the header states it: the largest grid of a row width is
accepted, one more row is rejected with a clear error.

The file sorts last so that a run stopping at the first failure has run every other test.
"""

import ctypes

import numpy as np
import pytest

from foilbench_b200 import _native as N
from foilbench_b200 import grid_ops as G
from foilbench_b200.models import DomainSpec

pytestmark = pytest.mark.gpu


def _field(ny, nx, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    vel = np.stack((0.9 + 0.3 * np.sin(0.21 * xx + 0.13 * yy), 0.2 * np.cos(0.17 * xx - 0.3 * yy)), axis=-1)
    return vel + 0.02 * rng.normal(size=vel.shape)


def _noalloc(dom, vel, nu, dt, tol, precision):
    import torch

    dtype = torch.float64 if precision == "float64" else torch.float32
    vx = torch.tensor(np.ascontiguousarray(vel[:, :, 0]), dtype=dtype, device="cuda")
    vy = torch.tensor(np.ascontiguousarray(vel[:, :, 1]), dtype=dtype, device="cuda")
    ox = torch.empty_like(vx)
    oy = torch.empty_like(vy)
    d = G._desc(dom, precision)
    rep = N.Report()
    torch.cuda.synchronize()
    code = N.lib().fb_op_implicit_diffuse_noalloc(0, ctypes.byref(d), ctypes.c_void_p(vx.data_ptr()),
                                                  ctypes.c_void_p(vy.data_ptr()), ctypes.c_void_p(ox.data_ptr()),
                                                  ctypes.c_void_p(oy.data_ptr()), nu, dt, tol, 640, None,
                                                  ctypes.byref(rep))
    N.check(code, "fb_op_implicit_diffuse_noalloc")
    out = np.stack((ox.cpu().numpy(), oy.cpu().numpy()), axis=-1)
    return out, rep


@pytest.mark.parametrize("precision,periodic", [("float64", ()), ("float64", ("x", "y")), ("float32", ())])
def test_noalloc_viscosity_matches_allocating_entry_point_twice(precision, periodic):
    dom = DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (96, 40), periodic)
    atol = 1e-12 if precision == "float64" else 2e-6
    # a stop tolerance each precision can reach (float32 Jacobi stalls near 1e-7)
    tol = 1e-9 if precision == "float64" else 1e-5
    dtype = np.float64 if precision == "float64" else np.float32
    for call, (seed, nu, dt) in enumerate(((3, 0.01, 0.02), (4, 0.05, 0.01))):
        vel = _field(dom.ny, dom.nx, seed).astype(dtype)
        ref, rrep = G.implicit_diffuse(vel, nu, dt, dom, tol, 640)
        got, grep = _noalloc(dom, vel, nu, dt, tol, precision)
        assert grep.viscosity_converged == 1 and rrep.converged, call
        assert grep.viscosity_iterations == rrep.iterations, call
        np.testing.assert_allclose(got, ref, rtol=0, atol=atol)


# The limit stated in include/foilb200.h: four planes rounded up to 256 bytes beside a
# 393,728-byte header inside 64 MiB.
MAX_CELLS = {"float64": 2_084_832, "float32": 4_169_664}


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_noalloc_limit_is_exact(precision):
    import torch

    nx = 2048
    ny = MAX_CELLS[precision] // nx
    dom = DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (nx, ny))
    vel = _field(ny, nx, 5).astype(np.float64 if precision == "float64" else np.float32)
    before = torch.cuda.current_device()
    got, grep = _noalloc(dom, vel, 0.001, 0.002, 1e-5, precision)
    assert torch.cuda.current_device() == before
    assert grep.viscosity_converged == 1 and grep.status == 0
    ref, rrep = G.implicit_diffuse(vel, 0.001, 0.002, dom, 1e-5, 640)
    assert grep.viscosity_iterations == rrep.iterations
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 if precision == "float64" else 2e-6)
    # one row more no longer fits (rejected before any device work)
    big = DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (nx, ny + 1))
    d = G._desc(big, precision)
    dummy = ctypes.c_void_p(1)
    code = N.lib().fb_op_implicit_diffuse_noalloc(0, ctypes.byref(d), dummy, dummy, dummy, dummy, 0.01, 0.01, 1e-9,
                                                  10, None, None)
    assert code == N.FB_ERR_INVALID_ARGUMENT
    assert f"at most {MAX_CELLS[precision]} cells".encode() in N.lib().fb_last_error()


def test_noalloc_rejects_grids_beyond_its_scratch():
    dom = DomainSpec(2, ((0.0, 1.0), (0.0, 1.0)), (4096, 4096))
    d = G._desc(dom, "float64")
    dummy = ctypes.c_void_p(1)
    code = N.lib().fb_op_implicit_diffuse_noalloc(0, ctypes.byref(d), dummy, dummy, dummy, dummy, 0.01, 0.01, 1e-9,
                                                  10, None, None)
    assert code == N.FB_ERR_INVALID_ARGUMENT
    assert b"scratch" in N.lib().fb_last_error()

"""Batched Stable Fluids: many solvers advance together, one persistent launch per substep round.

Each member is an initialized :class:`~foilbench_b200.solver.StableFluidsSolver`; a batch
advance gives every member exactly the result of its own ``advance`` (same substep plan,
retries, postconditions and rollback), but runs all members' substeps in one shared launch in
which each member owns a group of CTAs in proportion to its expected work (``fb_batch_*`` in
``include/foilb200.h``). The reference advances one solver at a time
(``PY/benchmark/runner.py:240-273``); batching is how many small grids keep all SMs busy.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _native as N
from .models import ControlState, NumericalFailure, StepReport
from .solver import StableFluidsSolver, _failure_from_report


class StableFluidsBatch:
    """A fixed set of solvers on one device advanced in batched launches."""

    def __init__(self, solvers: Sequence[StableFluidsSolver]):
        if not solvers:
            raise ValueError("a batch needs at least one solver")
        ctxs = {id(s._context()) for s in solvers}
        if len(ctxs) != 1:
            raise ValueError("batch members must share one device context")
        natives = [s._require()[1] for s in solvers]
        self._solvers = list(solvers)
        self._ctx = solvers[0]._context()
        handles = (ctypes.c_void_p * len(natives))(*[n.handle.value for n in natives])
        h = ctypes.c_void_p()
        N.check(N.lib().fb_batch_create(self._ctx.handle, handles, len(natives), ctypes.byref(h)), "fb_batch_create")
        self._handle = h

    def __len__(self) -> int:
        return len(self._solvers)

    @property
    def solvers(self) -> list[StableFluidsSolver]:
        return list(self._solvers)

    def ctas(self) -> list[int]:
        """CTAs each member had in the latest batched launch (0 when it did not run)."""
        out = (ctypes.c_int32 * len(self._solvers))()
        N.check(N.lib().fb_batch_ctas(self._handle, out, len(self._solvers)), "fb_batch_ctas")
        return [int(v) for v in out]

    def advance(self, controls: Sequence[ControlState], target_dts: Sequence[float]
                ) -> list[StepReport | NumericalFailure]:
        """Advance member i by target_dts[i] toward controls[i].

        Returns, per member, its StepReport, or the NumericalFailure it would have raised
        (that member's state is then unchanged). Invalid arguments raise before any member
        changes."""
        n = len(self._solvers)
        if len(controls) != n or len(target_dts) != n:
            raise ValueError("one control and one target_dt per member")
        prepared = [s._prepare_advance(c, dt) for s, c, dt in zip(self._solvers, controls, target_dts)]
        times = np.array([c.time for c in controls], dtype=np.float64)
        angles = np.array([c.angle_degrees for c in controls], dtype=np.float64)
        omegas = np.array([c.angular_velocity_degrees for c in controls], dtype=np.float64)
        dts = np.array(list(target_dts), dtype=np.float64)
        reps = (N.Report * n)()
        status = (ctypes.c_int32 * n)()
        code = N.lib().fb_batch_advance(self._handle, N.dptr(times), N.dptr(angles), N.dptr(omegas), N.dptr(dts),
                                        reps, status)
        if code not in (N.FB_OK, N.FB_ERR_NUMERICAL):
            N.check(code, "fb_batch_advance")
        out: list[StepReport | NumericalFailure] = []
        for i, (s, (_, start_angle)) in enumerate(zip(self._solvers, prepared)):
            if status[i] == N.FB_OK:
                out.append(s._commit_advance(controls[i], float(target_dts[i]), reps[i], start_angle))
            elif status[i] == N.FB_ERR_NUMERICAL:
                out.append(_failure_from_report(reps[i], "Stable Fluids batch member failed"))
            else:
                raise N.NativeError(f"fb_batch_advance member {i}: status {status[i]}")
        return out

    def close(self) -> None:
        if self._handle:
            N.lib().fb_batch_destroy(self._handle)
            self._handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

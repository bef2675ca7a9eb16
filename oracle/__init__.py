"""CPU oracle for the FoilBench Stable Fluids time step.

TEST INFRASTRUCTURE ONLY. This package is a plain numpy restatement of the
reference Python solver (``implementations/python/src/foilbench_py``) and of the
two third-party algorithms it calls (scipy 1.18.0 ``scipy.sparse.linalg.cg`` and
``scipy.fft.dstn/idstn`` type 1, ``norm="ortho"``). It exists to check the CUDA
product path: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` may import it. The product path (``foilbench_b200``) never
imports, calls or falls back to anything here.

Parity pin: the restatement is checked against fixtures produced by running the
reference itself (``tests/golden/make_golden.py``), see ``tests/test_oracle_golden.py``.
"""

from oracle.stable_fluids import (  # noqa: F401
    Grid,
    OracleFailure,
    OracleSolver,
    advect_velocity,
    cell_centers,
    cell_to_faces,
    dst1_ortho,
    faces_to_cell,
    implicit_diffuse,
    naca_mask,
    naca_signed_distance,
    naca_surfaces,
    native_divergence_linf,
    pcg,
    project_faces,
    solid_face_leakage,
    solve_masked_poisson,
)

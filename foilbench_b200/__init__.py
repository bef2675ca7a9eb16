"""B200-native drop-in for the FoilBench Stable Fluids solver step.

The numerical work runs in ``libfoilb200.so`` (hand-written sm_100a CUDA behind a
C ABI, see ``include/foilb200.h``); this package is the host side: the reference's
model types, scenario and canonical-state I/O, and the ``StableFluidsSolver`` that
implements the reference ``FlowSolver`` lifecycle on top of the library.
"""

__version__ = "0.1.0"

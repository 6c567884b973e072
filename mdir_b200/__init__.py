"""mdir_b200: a B200-native short-range nonbonded + PME path with MDIR's
(vv137/mdir) interface for that path.

The kernels live in libmdrt_nb.so (C ABI: include/mdrt_nb.h); this package
holds the host-side mirror of MDIR's Python interface for the path:
`compile`, `Simulation`, `FrameEvaluator` and `mdir_b200.torch`."""

from . import systems  # noqa: F401
from .api import (CompileError, Electrostatics, Ensemble, EnsembleKind, Execution, InitialState,  # noqa: F401
                  InputError, Integrator, Precision, Program, Schedule, Simulation, SimulationError,
                  System, Target, Truncation, UnsupportedError, compile)
from .frames import FrameEnergies, FrameEvaluator  # noqa: F401
from .term import COULOMB, NonbondedTerm, exclusion_rows  # noqa: F401

"""mdir_b200: a B200-native short-range nonbonded + PME path with MDIR's
(vv137/mdir) interface for that path.

The kernels live in libmdrt_nb.so (C ABI: include/mdrt_nb.h); this package
holds the host-side mirror of MDIR's Python interface for the path."""

from .term import COULOMB, NonbondedTerm, exclusion_rows  # noqa: F401
from . import systems  # noqa: F401

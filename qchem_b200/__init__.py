"""qchem_b200: B200-native McMurchie-Davidson ERIs and direct J/K Fock builds for qchem's molecular
Hartree-Fock path.  The compute lives in libqchem_b200.so (include/qchem_b200.h); this package holds the
basis/workload helpers and the ctypes front end (api.py)."""
from . import basis, workloads  # noqa: F401
from .api import Engine, OrbitalHFIBS, QcgError, lib, library_path  # noqa: F401

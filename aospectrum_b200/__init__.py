"""B200-native CISS band engine with the AOSpectrum Band-path interfaces.

Host side (this package) mirrors the reference's Band path API: operator
bundles, k paths, CISS settings, ``BandCalculation``, checkpoints and the
``aospectrum band`` command.  All numerics of the hot path run on the GPU
in libaospectrum_b200.so (C ABI in include/aospectrum_b200.h).
"""

from .bundle import load_bundle, write_bundle
from .ciss import CissResult, CissSettings, EngineSettings, ShiftedResult
from .data import (
    AtomicStructure,
    ElectronicFilling,
    EnergyInterval,
    LocalizedOperatorBlocks,
    LocalizedOperatorBundle,
    OrbitalBasisLayout,
)
from .errors import AOSpectrumError, InputError, SolverError
from .kpath import KPath, read_kpath
from .sparse import SparsePair

__version__ = "1.0.0rc2+b200"

__all__ = [
    "AOSpectrumError", "AtomicStructure", "CissResult", "CissSettings", "ElectronicFilling",
    "EnergyInterval", "EngineSettings", "InputError", "KPath", "LocalizedOperatorBlocks",
    "LocalizedOperatorBundle", "OrbitalBasisLayout", "ShiftedResult", "SolverError",
    "SparsePair", "load_bundle", "read_kpath", "write_bundle",
]

"""B200 time-step library for the Orsay-Trento TDDFT 4He solver with a
Bohmian test-particle impurity: host-side Python mirror of the C ABI in
include/he4_tddft.h (the CUDA library is libhe4b200.so next to this file)."""
from . import abi, fno, parareal, workloads  # noqa: F401
from .host import He4Batch, He4Error, He4Step, load_library, params_default  # noqa: F401

"""grim_b200: B200-native implicit GRMHD/EMHD timestep (drop-in for
AFD-Illinois/grim's timeStepper::timeStep).

The compute path is libgrim_b200.so (CUDA, sm_100a) behind the C ABI in
include/grim_b200.h; this package holds the ctypes binding and the Python
mirror of the reference's timeStepperPy / gridPy interface.  The shared
library is loaded on first use and its absence is an error: there is no CPU
fallback.
"""
from . import config  # noqa: F401

__all__ = ["config"]

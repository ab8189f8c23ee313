"""B200-native photon-packet transport and ionization balance.

A from-scratch CUDA (sm_100a) implementation of the plain photoionization
method of ParallelCMacIonize: Monte Carlo photon packets traced cell by cell
through subgrids staged in shared memory, and the FP64 ionization balance.
The CUDA library (libcmacionize_b200.so) is the product; this package is its
host-side mirror.  Importing the package does not touch the GPU; creating a
TransportEngine loads the library and fails loudly when it was not built.
"""
from .engine import (PARSEC, PHOTON_DTYPE, TRAVEL_DIRECTIONS, CMIError, GridSpec,
                     TransportEngine, TravelDirection, blocked_to_cube, cube_to_blocked)
from .params import ParameterError, Parameters

__all__ = [
    "TransportEngine", "GridSpec", "CMIError", "PHOTON_DTYPE", "TravelDirection",
    "TRAVEL_DIRECTIONS", "PARSEC", "blocked_to_cube", "cube_to_blocked", "Parameters",
    "ParameterError",
]

"""cl2qcd_b200 -- B200-native (sm_100a) twisted-mass Wilson even-odd inverter hot path.

The compute path is the CUDA library ``libc2q_b200.so`` behind the C ABI of
``include/cl2qcd_b200.h``; ``host`` mirrors the reference's lattice,
fermion-matrix and solver call surface on top of it.
"""
from . import _lib
from .host import *  # noqa: F401,F403
from .host import (AdditionalParameters, Gaugefield, Lattice, SolverDidNotSolve, SolverParameters, SolverStuck,
                   Spinorfield_eo, System)

__all__ = ["System", "Lattice", "Gaugefield", "Spinorfield_eo", "AdditionalParameters", "SolverParameters",
           "SolverStuck", "SolverDidNotSolve"]

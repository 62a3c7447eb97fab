"""Seeded synthetic states for the oracle-side tests: the same generators the product's
workload module provides (lattice-boltzmann-method_b200/workloads.py), re-exported so
tests can build identical inputs for the reference library, the C oracle and the GPU."""
import os
import sys

_PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lattice-boltzmann-method_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from workloads import *  # noqa: E402,F401,F403
from workloads import MIXTURE_SC, SEED  # noqa: E402,F401

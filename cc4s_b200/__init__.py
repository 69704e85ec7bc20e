"""B200-native CoupledCluster step (cc4s methods Ccsd, Ccd, Drccd) and the
steps that consume its amplitudes: perturbative triples and the finite-size
correction.

The compute path is the CUDA library ``libcc4s_b200.so`` behind the C ABI of
``include/cc4s_cc.h``; this package is its host-side mirror of the
reference's operator surface.  Importing it does not load the library;
constructing a solver does, and fails if the library is missing.
"""
from .coupled_cluster import (CoupledCluster, CoupledClusterError,  # noqa: F401
                             FiniteSizeCorrection, PerturbativeTriples, Solver)
from .flops import reference_flops  # noqa: F401

"""CPU oracle for the cc4s ``CoupledCluster`` step (methods ``Ccsd`` and ``Ccd``).

TEST INFRASTRUCTURE ONLY.  Nothing in this package is part of the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and only as the checker.  The product path is the
CUDA library under ``cc4s_b200/`` and fails loudly when that library is
missing; it never falls back to this code.

What it is: a numpy (FP64 / complex128) restatement, term by term and in the
reference's order, of

* ``CoupledCluster::run`` / ``getEnergy`` / ``residuumToAmplitudes`` /
  ``calculateEnergyDifferences``  (src/main/algorithms/CoupledCluster.cxx:56-317)
* ``Ccsd<Real>::getResiduum``     (src/main/algorithms/coupledcluster/Ccsd.cxx:77-378)
* ``Ccsd<Complex>::getResiduum``  (src/main/algorithms/coupledcluster/Ccsd.cxx:382-633)
* ``CcsdReference::getResiduum``  (src/main/algorithms/coupledcluster/CcsdReference.cxx:35-240)
* ``DiisMixer`` / ``LinearMixer`` (src/main/mixers/DiisMixer.cxx:28-146,
  src/main/mixers/LinearMixer.cxx:27-70)
* MP2 (src/main/algorithms/SecondOrderPerturbationTheory.cxx:53-149)
* the transition structure factor S(G)
  (src/main/algorithms/FiniteSizeCorrection.cxx:50-133)
* the input chain DefineHolesAndParticles / SliceOperator /
  VertexCoulombIntegrals (src/main/algorithms/*.cxx) and the
  uniform-electron-gas vertex generator (src/main/algorithms/UegVertexGenerator.cxx:27-297).

How it is pinned: the reference cannot be built here (MPI and the Cyclops
Tensor Framework are absent), so the oracle is pinned against the
reference's own expected output of its UEG regression test
(test/tests/ueg/rs1.0-7occ-26virt/correct.out.yaml): the vertex of that test is
regenerated with the restated UEG generator and the restated complex CCSD must
reproduce the reference's correlation, direct, exchange and second-order
energies to the test harness' 1e-7 Eh (test/testis.py:264-292).  The real
path is cross-checked against the independent textbook formulation
(CcsdReference) and MP2.

Layout convention: numpy arrays carry the reference's logical index order
(T1[a,i], T2[a,b,i,j], Gamma[G,p,q]); the reference's column-major memory
layout (first index fastest) is ``np.asfortranarray`` of these arrays.
"""

"""CPU oracle for the plane-wave H|psi> and block-Davidson path (test infrastructure).

This package is the CHECKER, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import it.
It restates, in numpy/scipy, the reference's CPU algorithm for this path:

* ``hpsi``     -- ``SerialPlanewaveHamiltonianApplicator::apply_hamiltonian_batch``
                  (``hamiltonian_applicator/serial.hpp:264-700``), non-Gamma branch;
* ``davidson`` -- ``PlanewaveDavidsonDiagonalizer::solve`` (``davidson.hpp:324-841``)
                  with ``SerialPlanewaveSubspaceManager`` (``subspace_manager/serial.hpp``)
                  and ``SerialSubspaceDiagonalizer`` (``subspace/serial.hpp:18-151``),
                  calling the same LAPACK routines (zpotrf, ztrsm, zhegv) the
                  reference calls, from scipy's bundled OpenBLAS.

The FFT is numpy/scipy pocketfft, not FFTW 3.3.10 as the reference pins.
Pinning: the oracle is checked against the reference's own known-answer tests
for this path (FFT round trip and Parseval, ``test_fft_grid.cpp:13-83``; the
subspace eigensolver KATs and the 48x48 generalized problem,
``test_subspace_diagonalizer.cpp:11-166``); the reference's tests hold no
golden H|psi> or Davidson vectors for these synthetic cells.
"""

"""CPU oracle for the SIMP minimum-compliance / GMG-PCG path.

TEST INFRASTRUCTURE ONLY.  This package is a plain numpy/scipy restatement of the
reference's (ahnobari/EDGE-TO) FP64 algorithm for the structured Q4 / hex8 SIMP loop.
It exists to check the CUDA product path, never to stand in for it: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may import
it, and the product package ``edge_to_b200`` never does.

Pinning: every function here is checked (tests/test_oracle_golden.py) against golden
fixtures in tests/golden/ that were produced by running the reference's own CPU code
(tests/golden/make_golden.py).  The reference ships no tests or fixtures of its own, so
these generated vectors are the pin.

Modules
  elements  element stiffness (Q4 plane stress, hex8) by 2x2(x2) Gauss quadrature
  grid      structured node / element numbering of the reference
  ops       K(E) with BCs, diagonal, dk, density filter and its transpose,
            restriction / prolongation, Galerkin coarse operators
  mg        the multigrid-preconditioned CG solver
  topopt    the SIMP loop with the OC bisection update
"""

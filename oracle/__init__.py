"""CPU oracle for the Tet4/Tet10 Total-Lagrangian NeoHookean assembly path.

TEST INFRASTRUCTURE ONLY.  This package restates, in numpy, the reference
algorithm of pSierra (tanadul-s/psierra) for the path the CUDA library replaces:
element kinematics and NeoHookean stress/tangent, per-element f_int and k_tan,
and the COO->CSR / ``np.add.at`` global assembly.  Each function cites the
reference file:line it follows.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and only as the checker or as the timed CPU
baseline.  The product path (``psierra_b200``) never calls into it and fails
loudly if its CUDA library is missing.

Pinning: the restatement is checked against golden vectors produced by running
the reference itself (``tests/golden/make_golden.py`` imports the reference and
writes ``tests/golden/*.npz``); see ``tests/test_oracle_golden.py``.
"""

"""CPU oracle for the two-site DMRG hot path -- TEST INFRASTRUCTURE ONLY.

Plain numpy restatements of the reference's algorithms (each function cites the
reference file:line it follows), pinned against outputs of the reference itself
(``oracle/_ref``, built from the reference sources by ``oracle/Makefile``; the
fixtures in ``tests/golden`` are generated from it by
``tests/golden/make_golden.py``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The product path
(``symmetry-adapted-dmrg-library_b200``) never calls it.
"""

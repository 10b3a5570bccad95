"""Oracle for the R-matrix hot path -- TEST INFRASTRUCTURE, not product code.

A CPU restatement of HPRMAT's FP64 "Type 1" path (mesh, C(E) assembly, LAPACK ZGESV,
R extraction, collision matrix) and of its boundary functions (COULFG/JWKB/WHIT).
It is pinned against the golden outputs shipped with the reference (Descouvemont's
Ex1/Ex2/Ex4 collision matrices) by ``tests/test_oracle_golden.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py``
may import it; the product (``hprmat_b200``) never does.
"""

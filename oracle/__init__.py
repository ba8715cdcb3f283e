"""ORACLE — test infrastructure only (CPU restatement of ForceConstants.jl).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker.  The product library
(``forceconstants.jl_b200``) never imports, links or calls anything here.
"""

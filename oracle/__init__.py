"""CPU oracle for the tree-approach deduplicator: TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference arm import
this package.  It is the checker, never the product: the GPU library never calls it.
"""

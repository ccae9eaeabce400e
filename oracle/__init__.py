"""ORACLE — CPU restatement of the reference's algorithm, used only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference arm as the
checker.  Nothing in the product (sympack_b200/) imports this package."""

"""CPU oracle for the batched contraction generator.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this package; only `tests/`,
`__graft_entry__.smoke()` and `bench.py` (its CPU-baseline legs) use it, and only as the
checker or the timed CPU reference. Parity is pinned by golden vectors produced by the
reference's own generated OpenMP kernels (`tests/golden/make_golden.py`).
"""

"""CPU oracle for the phaser multislice hot path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (`phaser_b200`) imports this package.  It is used by
`tests/` as the parity reference, by `__graft_entry__.smoke()` to check one
small GPU invocation, and by `bench.py` for its CPU-baseline leg (the timed
numpy implementation of the same algorithm, reported beside the GPU number).

`phaser_np` restates the reference's numpy algorithms (LSQ-ML, ePIE, the
gradient-engine model, cutouts, propagators, groupings) with each function
citing the reference file:line it follows.  The restatement is pinned against
fixtures produced by running the reference itself (see
`tests/golden/make_golden.py`).
"""

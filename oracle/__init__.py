"""Oracle: CPU restatement of cuGAL's FUGAL alignment path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
directory; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` use it, and only as the checker (or as the timed CPU baseline),
never as the thing measured on the GPU.

Parity pins: ``tests/test_oracle_golden.py`` checks every function here against
golden vectors produced by running the reference's own Python implementation
(``tests/golden/make_golden.py``), and against networkx / scipy known answers.
"""

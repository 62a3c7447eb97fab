"""CPU checkers for the D3Q27 hot path (test infrastructure, never the product).

* ``oracle.refsc``  -- ctypes view of ``_ref/libref_sc.so``, the reference's own
  single-component sources compiled here (see ``oracle/Makefile``).
* ``oracle.sc``     -- ctypes view of ``liboracle.so``, the plain-C restatement.
* ``oracle.cases``  -- seeded synthetic initial states (Taylor-Green vortex, ...).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
this package.
"""

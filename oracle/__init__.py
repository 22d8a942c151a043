"""TEST INFRASTRUCTURE ONLY: CPU oracles for the vertical-line-locus path.

* ``oracle.refpy``    -- ctypes access to the reference SETSM implementation,
                         compiled from its own sources into
                         ``oracle/_ref/libsetsm_ref.so`` (see oracle/Makefile).
* ``oracle.oraclepy`` -- ctypes access to the C restatement in
                         ``oracle/vll_oracle.c`` (``oracle/liboracle_vll.so``).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker / baseline -- never as the product.
"""

"""Oracle for the Slater-Jastrow walker path -- TEST INFRASTRUCTURE ONLY.

* ``qmc_oracle.c``: C restatement of the reference algorithm (the port).
* ``ref_shim.cpp`` + ``Makefile``: the reference QMcBeaver CPU code compiled
  from its own sources into ``_ref/`` (where the reference tree exists).
* ``evaluators.py``: ctypes front ends with one interface for both.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may use this package, and only as the checker.
"""

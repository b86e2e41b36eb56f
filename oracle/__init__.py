"""CPU oracle for the 2-D shallow-water finite-volume step.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
directory: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, and there only as the checker (or as the timed CPU
baseline), never as the code path being measured or shipped.

Contents
--------
``swe_numpy``  A dtype-parametric NumPy restatement of the reference solver
               (``src/hybrid_flood/numpy_solver/shallow_water_2d.py`` and the
               per-side boundary codes of
               ``src/hybrid_flood/jax_solver/boundary_conditions.py``), plus an
               FP64 mass ledger.  At float32 with all-reflective boundaries it
               reproduces the reference bit-for-bit (pinned by
               ``tests/golden``, generated from the unmodified reference).
``swe_oracle.c`` The same algorithm in plain C (float and double, OpenMP over
               rows), used for sizes the NumPy restatement is too slow for and
               as the timed CPU baseline ("port").  ``cport`` wraps it with
               ctypes.
"""

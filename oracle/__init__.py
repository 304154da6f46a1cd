"""Oracle package -- TEST INFRASTRUCTURE ONLY.

CPU restatements of paintop's Poisson / screened-Poisson solver used to check
the CUDA library. Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this package; the product path never does.
"""

"""CPU FP64 oracle for the kernel-PC CI hot path.

TEST INFRASTRUCTURE ONLY.  This package restates the reference's algorithm
(wyjistest/fastkpc and legacy kpcalg) in numpy so the test-suite can check
the CUDA library against it.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` may import it; the shipped library never
does, and it has no code path that falls back to it.

Modules: ``rng`` (R-compatible MT19937 permutation streams), ``tprs`` (mgcv
thin-plate / additive design), ``gcv`` (magic-style GCV selection and
residuals), ``stats`` (dCov / HSIC statistics and p-values), ``skeleton``
(pcalg-stable level replay).
"""

"""CPU oracle for the DOGPUP forward/sensitivity path -- TEST INFRASTRUCTURE ONLY.

This package is a float64 NumPy/SciPy restatement of the reference
formulation.  Only the test-suite, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import it, and only to check or to time
against; the product path (``dogpup_b200``) never calls it and has no CPU
fallback.

Every function cites the reference file:line it restates (paths relative to
the DOGPUP project root).

Pinning status:
  * The three reference CUDA kernels (``smv_CUDA.cu``, ``FSAImv_CUDA.cu``,
    ``FSAIP_CUDA.cu``) compile from their own sources with a stub ``mex.h``
    (recipe: ``oracle/Makefile``, output ``oracle/_ref/``); the GPU tests run
    them on identical inputs and check this oracle's ``smv``/``fsai_apply``/
    ``fsai_factor`` and the product kernels against their outputs.
  * The MATLAB parts (assembly, FSAI pattern, BiCGSTAB driver, transforms,
    Jacobian, ``tik_inv``) cannot run here (no MATLAB); the reference ships
    no golden vectors or tests.  These parts are **parity unpinned** by
    reference outputs and are anchored instead on mathematical identities
    (P1 mass/stiffness identities, FSAI defining identities, a sparse-direct
    complex128 solve, Parseval/round-trip identities, finite differences).
"""

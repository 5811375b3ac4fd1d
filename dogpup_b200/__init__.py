"""dogpup_b200: the DOGPUP forward/sensitivity path on NVIDIA B200 (sm_100a).

Device FEM assembly, FSAI-preconditioned BiCGSTAB over every source x
harmonic (FP64, or complex-FP32 with FP64 iterative refinement), detector
read-out, Fourier-series transforms, the adjoint absorption Jacobian and the
LM normal-equation step -- all in hand-written CUDA behind the C ABI of
``include/dogpup_b200.h``.  The compute modules (``api``, ``dmesh``, ...)
load ``libdogpup_b200.so`` on import and raise if it has not been built
(``python -m dogpup_b200.build``); there is no CPU fallback.
"""


def __getattr__(name):
    if name in ("DgpError", "lib"):
        from . import _lib
        return getattr(_lib, name)
    raise AttributeError(name)

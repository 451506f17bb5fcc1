"""menodax_b200: ensemble ODE integration (Tsit5, Rodas5P) on one NVIDIA B200.

The drop-in for the ``modax`` package: ``menodax_b200.tsit5.solve`` and
``menodax_b200.rodas5P.solve`` take a tuple-form right-hand side
``ode_fn(y, t, p)``, trace it once on the host, and run hand-written sm_100a
kernels compiled with NVRTC through the C ABI in ``include/menodax.h``.
"""

from menodax_b200 import rodas5P, tsit5  # noqa: F401

__all__ = ["tsit5", "rodas5P"]

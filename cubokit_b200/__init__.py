"""cubokit_b200: CuboPtycho's gradient-descent ptychography on NVIDIA B200 (sm_100a).

The engine is ``libcuboptycho.so`` (CUDA kernels behind the C ABI of ``include/cubo_ptycho.h``); this package is its
Python binding and the host-side mirror of CuboPtycho's API: ``SingleslicePtychography`` (FP32, split-BF16 and FP64
forms, position correction), ``PtychographyPreparation.amplitudes``, ``PtychographyProbe.build``,
``MixedstatePtychography`` and ``MultislicePtychography`` (FP64), device-resident ``Plan`` and graph-replayed
``Batch`` objects, and ``sharded.reconstruct`` (one reconstruction over several GPUs).
"""
from .ptycho import (Batch, CancellationError, Context, DeviceError, MixedstatePtychography,
                     MultislicePtychography, Plan,
                     PtychographyAmplitudes, PtychographyError,
                     PtychographyPositionCorrection, PtychographyPreparation, PtychographyProbe, Result,
                     SingleslicePtychography, UnsupportedError, context, electron_wavelength)

__all__ = ["Batch", "CancellationError", "Context", "DeviceError", "MixedstatePtychography", "MultislicePtychography", "Plan", "PtychographyAmplitudes", "PtychographyError",
           "PtychographyPositionCorrection", "PtychographyPreparation", "PtychographyProbe", "Result", "SingleslicePtychography", "UnsupportedError", "context",
           "electron_wavelength"]
from . import sharded  # noqa: E402  one reconstruction over several GPUs

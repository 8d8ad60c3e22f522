"""B200-native estimation-based SpGEMM (C = A·B, CSR, FP64) behind a C ABI.

The product is the CUDA library ``libocean.so`` (hand-written sm_100a kernels,
C ABI in ``include/ocean.h``); this package holds its ctypes binding, the
seeded matrix generators and the ``.hicsr`` reader/writer.
"""
from .ocean import DeviceCSR, HostCSR, OceanError, SpGEMM, lib  # noqa: F401

__all__ = ["SpGEMM", "HostCSR", "DeviceCSR", "OceanError", "lib"]

"""mspai_b200: B200-native MSPAI preconditioner setup (sparse approximate inverse).

The setup solves, for every column k, min ||C(I_k,J_k) m_k - B(I_k,k)||_2 in
hand-written sm_100a CUDA kernels behind a C ABI (include/mspai_b200.h).
"""
from .api import (DeviceCSC, Handle, Options, assemble_probing, block_pattern, measure_fma_peak,
                  mspai, pattern_power2, pattern_powers, read_mm,
                  start_pattern,
                  write_mm)
from ._lib import MspaiError

__all__ = ["pattern_power2", "pattern_powers", "DeviceCSC", "Handle", "Options", "MspaiError", "assemble_probing", "mspai",
           "read_mm", "start_pattern", "write_mm"]

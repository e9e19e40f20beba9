"""B200-native Gamma-SMC pairwise TMRCA scan.

Drop-in for ``gamma_smc_cu.infer`` / ``infer_blockwise`` and the
``_core.FlowContext`` they drive; the device work runs in hand-written sm_100a
kernels in ``lib/libgsmc_b200.so`` (C ABI in ``include/gsmc_b200.h``).
"""
from . import _core
from ._core import (FlowContext, bitpack, cuda_mem_info, gamma_smc_flow_fb, get_device,
                    get_device_count, set_device, unpack)
from .infer import infer, infer_blockwise

__all__ = [
    "FlowContext",
    "bitpack",
    "unpack",
    "cuda_mem_info",
    "gamma_smc_flow_fb",
    "get_device",
    "get_device_count",
    "set_device",
    "infer",
    "infer_blockwise",
]
__version__ = "0.1.0"

"""mcpet -- B200 (sm_100a) photon-transport path of MCGPU-PET.

Thin Python binding over the C ABI in include/mcpet.h (libmcpet.so).  The
compute runs in the CUDA kernels of the library; there is no CPU path.
"""
from ._abi import (ALGORITHM_AUTO, ALGORITHM_EVENTS, ALGORITHM_HISTORIES, LANES_BALANCED, LANES_REFERENCE,
                   MAX_MATERIALS, McpetError, EXPORTED, LIB_PATH, lib)
from .scene import (PSF_DTYPE, BatchGraph, RunOptions, RunResult, Scene, autotune, device_tallies_for,
                    probe_compton, probe_detector, probe_rayleigh, probe_rng, probe_source, read_config)

__all__ = [
    "ALGORITHM_AUTO", "ALGORITHM_EVENTS", "ALGORITHM_HISTORIES", "LANES_BALANCED", "LANES_REFERENCE", "MAX_MATERIALS", "McpetError", "EXPORTED", "LIB_PATH", "lib", "PSF_DTYPE",
    "BatchGraph", "RunOptions", "RunResult", "Scene", "autotune", "device_tallies_for", "probe_compton", "probe_detector", "probe_rayleigh", "probe_rng",
    "probe_source", "read_config",
]


def version() -> str:
    return lib().mcpet_version().decode()

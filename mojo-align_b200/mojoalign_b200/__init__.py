"""B200-native seed-and-extend path of the mojo-align linear bisulfite mapper.

The compute path is libmojoalign_b200.so (CUDA, sm_100a), loaded through
ctypes by `_lib`; importing this package fails when the library is missing.
"""
from ._lib import MojoAlignError
from .mapper import GpuContext, GpuIndex, MapResult, build_index, map_batch, map_batch_device, probe_index
from .params import BENCH_PARAMS, FmParams

__all__ = ["MojoAlignError", "GpuContext", "GpuIndex", "MapResult", "build_index", "map_batch",
           "map_batch_device", "probe_index", "FmParams", "BENCH_PARAMS"]

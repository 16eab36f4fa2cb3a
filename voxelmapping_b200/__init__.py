"""B200-native voxel-hashing TSDF mapping (fuse / raycast / mesh).

The compute path is libvmap_b200.so (CUDA, sm_100a) behind the C ABI in
include/vmap_c.h; this package holds its ctypes binding, the Python mirror of
the reference's VoxelMapping class and the synthetic-scene generator.
"""
from ._lib import VmapError, lib  # noqa: F401
from .vmapping import HostPipeline, MapBatch, VoxelMapping, snapshot_header  # noqa: F401

__all__ = ["VoxelMapping", "MapBatch", "HostPipeline", "snapshot_header", "VmapError", "lib"]

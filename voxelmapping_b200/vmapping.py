"""Python mirror of the reference's ``vmap::VoxelMapping`` class.

Same methods, argument meaning and ownership as include/vmapping.h:10-27 of
xingruiyang/VoxelMapping (whose Python bindings live in an external project),
implemented over the C ABI of libvmap_b200.so. Device images are torch CUDA
tensors (torch is only the device-memory and stream plumbing); host images are
numpy arrays.

    vm = VoxelMapping(640, 480, K)
    vm.CreateMap(numEntries=1 << 21, numVoxels=1 << 20, voxelSize=0.005)
    vm.FuseDepth(depth_cuda, camToWorld)           # float metres (h, w)
    vmap = vm.RenderScene(None, camToWorld)        # (h, w, 4) camera-frame vertices
    n, verts, norms = vm.Polygonize()              # reference: int + two float* (9 per triangle)

Differences from the reference, by design: errors raise VmapError instead of
exit(0); FuseDepthAndImage is implemented (a stub in the reference,
vmapping.cpp:167-170); misses in the vertex map are NaN in all four lanes.
"""
import ctypes as C

import numpy as np

from . import _lib as L


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class VoxelMapping:
    def __init__(self, w, h, K, voxel_format="f32", with_color=True, max_weight=0, truncation=0.0,
                 raycast_mode=0, num_buckets=0):
        self.width, self.height = int(w), int(h)
        self.K = np.asarray(K, dtype=np.float64).reshape(3, 3)
        self.voxel_format = L.FORMAT_NAMES[voxel_format] if isinstance(voxel_format, str) else int(voxel_format)
        self.with_color = bool(with_color)
        self.max_weight = int(max_weight)
        self.truncation = float(truncation)
        self.raycast_mode = int(raycast_mode)
        self.num_buckets = int(num_buckets)
        self._map = None
        self._mem = None
        self._lib = L.lib()

    # -- lifetime ------------------------------------------------------------
    def _config(self, numEntries, numVoxels, voxelSize):
        return L.Config(self.width, self.height, float(self.K[0, 0]), float(self.K[1, 1]), float(self.K[0, 2]),
                        float(self.K[1, 2]), int(numEntries), int(numVoxels), float(voxelSize), self.num_buckets,
                        self.truncation, self.voxel_format, self.max_weight, int(self.with_color), self.raycast_mode)

    def CreateMap(self, numEntries, numVoxels, voxelSize):
        """vmapping.cpp:57-75: allocate and reset the map."""
        self.release()
        cfg = self._config(numEntries, numVoxels, voxelSize)
        h = C.c_void_p()
        L.check(self._lib.vmap_create(C.byref(cfg), C.byref(h)), "vmap_create")
        self._map = h
        self.config = self.get_config()

    def required_bytes(self, numEntries, numVoxels, voxelSize):
        """Device bytes CreateMapIn needs for this map (vmap_required_bytes)."""
        n = C.c_uint64()
        L.check(self._lib.vmap_required_bytes(C.byref(self._config(numEntries, numVoxels, voxelSize)), C.byref(n)),
                "vmap_required_bytes")
        return n.value

    def CreateMapIn(self, numEntries, numVoxels, voxelSize, memory):
        """CreateMap inside `memory`, a CUDA uint8 tensor of at least
        required_bytes() (vmap_create_in; the reset is asynchronous on the
        current stream). The map keeps a reference to the tensor until
        release(), which the caller calls only once the map's work is done."""
        self.release()
        cfg = self._config(numEntries, numVoxels, voxelSize)
        h = C.c_void_p()
        L.check(self._lib.vmap_create_in(C.byref(cfg), C.c_void_p(memory.data_ptr()),
                                         memory.numel() * memory.element_size(), _stream(), C.byref(h)),
                "vmap_create_in")
        self._map = h
        self._mem = memory
        self.config = self.get_config()

    def release(self):
        if self._map is not None:
            L.check(self._lib.vmap_destroy(self._map), "vmap_destroy")
            self._map = None
        self._mem = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def reset(self):
        L.check(self._lib.vmap_reset(self._need(), _stream()), "vmap_reset")

    def _need(self):
        if self._map is None:
            raise L.VmapError(1, "map not created (call CreateMap first)")
        return self._map

    def get_launch_config(self):
        """Grid of every stage in CTAs per SM (vmap_get_launch_config)."""
        c = L.LaunchConfig()
        L.check(self._lib.vmap_get_launch_config(self._need(), C.byref(c)), "vmap_get_launch_config")
        return {k: getattr(c, k) for k, _ in c._fields_}

    def set_launch_config(self, **kw):
        """Sets some stages' grids (keys of get_launch_config; 0 = default)."""
        cur = self.get_launch_config()
        cur.update(kw)
        L.check(self._lib.vmap_set_launch_config(self._need(), C.byref(L.LaunchConfig(**cur))),
                "vmap_set_launch_config")

    def get_config(self):
        cfg = L.Config()
        L.check(self._lib.vmap_get_config(self._need(), C.byref(cfg)), "vmap_get_config")
        return {k: getattr(cfg, k) for k, _ in cfg._fields_}

    # -- fusion --------------------------------------------------------------
    def FuseDepth(self, depth, camToWorld, depth_scale=0.001):
        """Fuse a device depth image: float32 metres or uint16 (x depth_scale)."""
        import torch
        assert depth.is_cuda and depth.shape[-2:] == (self.height, self.width)
        dt = L.DEPTH_U16 if depth.dtype in (torch.uint16, torch.int16) else L.DEPTH_F32
        if dt == L.DEPTH_F32:
            assert depth.dtype == torch.float32
        L.check(self._lib.vmap_fuse_depth(self._need(), _ptr(depth), dt, depth.stride(0) * depth.element_size(),
                                          depth_scale, L.pose_arg(camToWorld), _stream()), "vmap_fuse_depth")

    def FuseDepthAndImage(self, rgb, depth, camToWorld, depth_scale=0.001):
        """Fuse depth + uint8x3 colour. numpy inputs take the host-buffer path
        (the reference signature takes cv::Mat), torch CUDA tensors the device path."""
        m = self._need()
        if isinstance(depth, np.ndarray):
            depth = np.ascontiguousarray(depth)
            rgb_p = None
            if rgb is not None:
                rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
                rgb_p = rgb.ctypes.data_as(C.c_void_p)
            dt = L.DEPTH_U16 if depth.dtype == np.uint16 else L.DEPTH_F32
            if dt == L.DEPTH_F32:
                depth = depth.astype(np.float32, copy=False)
            L.check(self._lib.vmap_fuse_host(m, depth.ctypes.data_as(C.c_void_p), dt, depth_scale, rgb_p,
                                             L.pose_arg(camToWorld), _stream()), "vmap_fuse_host")
            import torch
            torch.cuda.current_stream().synchronize()  # host buffers may be pageable and reused
            return
        import torch
        dt = L.DEPTH_U16 if depth.dtype in (torch.uint16, torch.int16) else L.DEPTH_F32
        L.check(self._lib.vmap_fuse_depth_rgb(m, _ptr(depth), dt, depth.stride(0) * depth.element_size(),
                                              depth_scale, _ptr(rgb), rgb.stride(0), L.pose_arg(camToWorld),
                                              _stream()), "vmap_fuse_depth_rgb")

    def CheckVisibleBlocks(self, camToWorld):
        L.check(self._lib.vmap_check_visible_blocks(self._need(), L.pose_arg(camToWorld), _stream()))
        return self.stats()["visible_blocks"]

    # -- raycast -------------------------------------------------------------
    def RenderScene(self, vmap, camToWorld, nmap=None):
        """Raycast the map at camToWorld into vmap ((h, w, 4) float32 CUDA,
        allocated when None); nmap receives normals when given. Returns vmap."""
        import torch
        if vmap is None:
            vmap = torch.empty((self.height, self.width, 4), dtype=torch.float32, device="cuda")
        L.check(self._lib.vmap_render_scene(self._need(), L.pose_arg(camToWorld), _ptr(vmap), vmap.stride(0) * 4,
                                            _ptr(nmap) if nmap is not None else None,
                                            nmap.stride(0) * 4 if nmap is not None else 0, _stream()),
                "vmap_render_scene")
        return vmap

    # -- meshing -------------------------------------------------------------
    def Polygonize(self):
        """Returns (num_triangles, verts, norms): (n, 9) float32 arrays copied
        from the library-owned host buffers (reference: int + float*&)."""
        vp, np_ = C.POINTER(C.c_float)(), C.POINTER(C.c_float)()
        n = C.c_uint32()
        L.check(self._lib.vmap_polygonize_host(self._need(), C.byref(vp), C.byref(np_), C.byref(n), _stream()),
                "vmap_polygonize_host")
        k = n.value
        if k == 0:
            return 0, np.zeros((0, 9), np.float32), np.zeros((0, 9), np.float32)
        verts = np.ctypeslib.as_array(vp, shape=(k, 9)).copy()
        norms = np.ctypeslib.as_array(np_, shape=(k, 9)).copy()
        return k, verts, norms

    def GetSurfacePoints(self):
        """Triangle centroids, (n, 3) float32 (vmapping.cpp:134-147)."""
        import torch
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        L.check(self._lib.vmap_polygonize(self._need(), None, None, 0, _ptr(cnt), _stream()))
        k = int(cnt.item())
        if k == 0:
            return np.zeros((0, 3), np.float32)
        verts = torch.empty((k, 9), dtype=torch.float32, device="cuda")
        L.check(self._lib.vmap_polygonize(self._map, _ptr(verts), None, k, _ptr(cnt), _stream()))
        pts = torch.empty((k, 3), dtype=torch.float32, device="cuda")
        L.check(self._lib.vmap_surface_points(_ptr(verts), k, _ptr(pts), _stream()))
        return pts.cpu().numpy()

    # -- inspection ----------------------------------------------------------
    def stats(self):
        s = L.Stats()
        L.check(self._lib.vmap_get_stats(self._need(), _stream(), C.byref(s)), "vmap_get_stats")
        return s.as_dict()

    def clear_errors(self):
        L.check(self._lib.vmap_clear_errors(self._need(), _stream()))

    def export_blocks_static(self, first, count):
        """vmap_export_blocks_static: at most 256 blocks, no allocation."""
        coords = np.zeros((count, 3), np.int32)
        tsdf = np.zeros((count, 512), np.float32)
        weight = np.zeros((count, 512), np.float32)
        got = C.c_uint32()
        L.check(self._lib.vmap_export_blocks_static(self._need(), first, count, coords.ctypes.data, tsdf.ctypes.data,
                                                    weight.ctypes.data, None, C.byref(got), _stream()))
        k = got.value
        return {"coords": coords[:k], "tsdf": tsdf[:k], "weight": weight[:k]}

    def snapshot_bytes(self):
        """Size of vmap_snapshot_save's output for the map as it is now."""
        n = C.c_uint64()
        L.check(self._lib.vmap_snapshot_save(self._need(), None, 0, C.byref(n), _stream()), "vmap_snapshot_save")
        return n.value

    def save_snapshot(self, out=None):
        """vmap_snapshot_save into `out` (a uint8 numpy array or a torch uint8
        tensor, host, pinned or CUDA, of at least snapshot_bytes()), or into a
        new numpy array. Returns the filled prefix."""
        n = self.snapshot_bytes()
        if out is None:
            out = np.empty(n, np.uint8)
        ptr = out.ctypes.data if isinstance(out, np.ndarray) else out.data_ptr()
        cap = out.nbytes if isinstance(out, np.ndarray) else out.numel() * out.element_size()
        got = C.c_uint64()
        L.check(self._lib.vmap_snapshot_save(self._need(), C.c_void_p(ptr), cap, C.byref(got), _stream()),
                "vmap_snapshot_save")
        return out[:got.value]

    def load_snapshot(self, snap):
        """vmap_snapshot_load from a uint8 numpy array or torch tensor."""
        ptr = snap.ctypes.data if isinstance(snap, np.ndarray) else snap.data_ptr()
        nbytes = snap.nbytes if isinstance(snap, np.ndarray) else snap.numel() * snap.element_size()
        L.check(self._lib.vmap_snapshot_load(self._need(), C.c_void_p(ptr), nbytes, _stream()), "vmap_snapshot_load")

    def export_blocks(self, with_rgb=None):
        """Allocated blocks in pool order: coords (n, 3) int32, tsdf / weight
        (n, 512) float32 (voxel x + 8y + 64z), rgb (n, 512, 3) uint8 or None."""
        n = self.stats()["allocated_blocks"]
        with_rgb = self.with_color if with_rgb is None else with_rgb
        coords = np.zeros((n, 3), np.int32)
        tsdf = np.zeros((n, 512), np.float32)
        weight = np.zeros((n, 512), np.float32)
        rgb = np.zeros((n, 512, 3), np.uint8) if with_rgb else None
        got = C.c_uint32()
        cp = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
        L.check(self._lib.vmap_export_blocks(self._map, cp(coords), cp(tsdf), cp(weight), cp(rgb), n,
                                             C.byref(got), _stream()), "vmap_export_blocks")
        return {"coords": coords, "tsdf": tsdf, "weight": weight, "rgb": rgb}


def snapshot_header(snap):
    """Fields of the vmap_snapshot_header at the start of a snapshot image (a
    uint8 numpy array, bytes, or a torch uint8 tensor on any device): format,
    colour, block count and bytes, voxel size, truncation, weight cap, sticky
    error flags and the key / pool offsets. Raises ValueError on an image
    that is too short or does not start with the snapshot magic."""
    size = C.sizeof(L.SnapshotHeader)
    if isinstance(snap, (bytes, bytearray, memoryview)):
        raw = bytes(snap[:size])
    elif isinstance(snap, np.ndarray):
        raw = snap.reshape(-1).view(np.uint8)[:size].tobytes()
    else:
        raw = snap.reshape(-1)[:size].cpu().numpy().tobytes()
    if len(raw) < size:
        raise ValueError("a snapshot image holds at least %d bytes, got %d" % (size, len(raw)))
    h = L.SnapshotHeader.from_buffer_copy(raw)
    if h.magic != b"VMAPSNAP":
        raise ValueError("not a snapshot image (magic %r)" % h.magic)
    return {k: getattr(h, k) for k, _ in L.SnapshotHeader._fields_ if k != "magic"}


class HostPipeline:
    """Frames from host memory through vmap_frame_host_async: copies of
    neighbouring frames overlap each other's kernels.

        pipe = HostPipeline(vm)
        for depth, rgb, pose in frames:         # numpy arrays
            vmap, nmap = pipe.submit(depth, rgb, pose)
        pipe.wait()                              # every result is now in vmap / nmap

    Inputs are copied into pinned buffers (so the caller may reuse its
    arrays at once); each frame's results land in fresh pinned buffers,
    returned as numpy arrays that hold them, complete after `wait()`."""

    def __init__(self, vm, depth_scale=0.001, normals=True):
        import torch
        self.vm, self.scale, self.normals = vm, depth_scale, normals
        self._torch = torch
        self._keep = []

    def submit(self, depth, rgb=None, pose=None, render=True):
        torch = self._torch
        vm = self.vm
        d = torch.from_numpy(np.ascontiguousarray(depth)).pin_memory()
        c = torch.from_numpy(np.ascontiguousarray(rgb)).pin_memory() if rgb is not None else None
        f = L.HostFrame()
        f.depth_host = d.data_ptr()
        f.depth_type = L.DEPTH_F32 if d.dtype == torch.float32 else L.DEPTH_U16
        f.depth_scale = self.scale
        f.rgb_host = c.data_ptr() if c is not None else None
        f.pose[:] = [float(x) for x in np.asarray(pose, np.float64).reshape(16)]
        out = None
        if render:
            v = torch.empty((vm.height, vm.width, 4), dtype=torch.float32).pin_memory()
            n = torch.empty_like(v).pin_memory() if self.normals else None
            f.vmap_host = v.data_ptr()
            f.nmap_host = n.data_ptr() if n is not None else None
            out = (v.numpy(), n.numpy() if n is not None else None)
        self._keep.append((d, c, out))
        L.check(vm._lib.vmap_frame_host_async(vm._need(), C.byref(f), _stream()), "vmap_frame_host_async")
        return out

    def wait(self):
        """Orders the current stream after every copy so far and synchronises it."""
        L.check(self.vm._lib.vmap_host_wait(self.vm._need(), _stream()), "vmap_host_wait")
        self._torch.cuda.current_stream().synchronize()
        self._keep = []  # the returned arrays keep their own buffers alive


class MapBatch:
    """Fuse + raycast many VoxelMapping maps per step (vmap_batch_*).

    step(depths, rgbs, poses, vmaps, nmaps) fuses depths[i] (and rgbs[i]) into
    maps[i] at poses[i] and raycasts maps[i] at the same pose into vmaps[i]
    (and nmaps[i]). By default every stage is one launch over all maps;
    set_launch_config(batch_schedule=2) runs the whole step as one persistent
    launch instead (same results). Either is replayed as a CUDA graph from the
    third step on (non-default streams)."""

    def __init__(self, maps):
        self.maps = list(maps)
        self._lib = L.lib()
        arr = (C.c_void_p * len(self.maps))(*[m._need().value for m in self.maps])
        h = C.c_void_p()
        L.check(self._lib.vmap_batch_create(arr, len(self.maps), C.byref(h)), "vmap_batch_create")
        self._h = h
        self._frames = (L.BatchFrame * len(self.maps))()

    def get_launch_config(self):
        c = L.LaunchConfig()
        L.check(self._lib.vmap_batch_get_launch_config(self._h, C.byref(c)), "vmap_batch_get_launch_config")
        return {k: getattr(c, k) for k, _ in c._fields_}

    def set_launch_config(self, **kw):
        """Sets some stages' grids; the batch records its graphs again."""
        cur = self.get_launch_config()
        cur.update(kw)
        L.check(self._lib.vmap_batch_set_launch_config(self._h, C.byref(L.LaunchConfig(**cur))),
                "vmap_batch_set_launch_config")

    def release(self):
        if getattr(self, "_h", None) is not None:
            L.check(self._lib.vmap_batch_destroy(self._h), "vmap_batch_destroy")
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def step(self, depths, rgbs, poses, vmaps, nmaps=None, depth_scale=0.001, stream=None):
        """One fuse + render step over every map of the batch. ``depths[i]`` None
        skips map i's fusion and ``vmaps[i]`` None its render (a fuse-only or
        render-only request); both None leave the map idle."""
        s = self._fill(depths, rgbs, poses, vmaps, nmaps, depth_scale, stream)
        L.check(self._lib.vmap_batch_step(self._h, self._frames, s), "vmap_batch_step")

    def stall_probe(self, depths, rgbs, poses, vmaps, nmaps=None, stall_ms=200, depth_scale=0.001, stream=None):
        """vmap_batch_stall_probe: the step as one persistent launch that cannot
        proceed, so its bounded wait runs out after stall_ms."""
        s = self._fill(depths, rgbs, poses, vmaps, nmaps, depth_scale, stream)
        L.check(self._lib.vmap_batch_stall_probe(self._h, self._frames, int(stall_ms), s), "vmap_batch_stall_probe")

    def _fill(self, depths, rgbs, poses, vmaps, nmaps, depth_scale, stream):
        import torch
        for i, m in enumerate(self.maps):
            f = self._frames[i]
            d = depths[i]
            f.depth_dev = d.data_ptr() if d is not None else None
            f.depth_type = L.DEPTH_U16 if d is not None and d.dtype in (torch.uint16, torch.int16) else L.DEPTH_F32
            f.depth_pitch = d.stride(0) * d.element_size() if d is not None else 0
            f.depth_scale = depth_scale
            c = rgbs[i] if rgbs is not None else None
            f.rgb_dev = c.data_ptr() if c is not None else None
            f.rgb_pitch = c.stride(0) * c.element_size() if c is not None else 0
            p = np.asarray(poses[i], np.float64).reshape(16)
            for k in range(16):
                f.pose[k] = p[k]
            v = vmaps[i]
            f.vmap_dev = v.data_ptr() if v is not None else None
            f.vmap_pitch = v.stride(0) * 4 if v is not None else 0
            n = nmaps[i] if nmaps is not None else None
            f.nmap_dev = n.data_ptr() if n is not None else None
            f.nmap_pitch = n.stride(0) * 4 if n is not None else 0
        return C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)

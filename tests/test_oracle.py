"""Known-answer tests of the CPU oracle (no GPU): a fronto-parallel wall at a
known depth has a closed-form TSDF and surface, so fusion, ray marching and
marching cubes can be checked against geometry, in both the FP32
reference-arithmetic mode and the FP64 mode; plus the reference's validity
rules (depth range, NaN), weight cap and colour blend (depth_fusion.cu:148-196,
328-380; map_struct.h:9-10)."""
import numpy as np
import pytest

from oracle import oracle as O

W, H, F = 64, 48, 50.0
K = np.array([[F, 0, (W - 1) / 2], [0, F, (H - 1) / 2], [0, 0, 1]])
VS = 0.008
MU = np.float32(VS) * np.float32(4)
D = 1.0
POSE = np.eye(4)


def wall(depth=D):
    return np.full((H, W), depth, np.float32)


@pytest.mark.parametrize("precision", [O.FP32, O.FP64])
def test_wall_tsdf_matches_projective_distance(precision):
    om = O.OracleMap(W, H, K, 4096, VS, precision=precision, storage="f32", with_color=False)
    res = om.fuse(wall(), None, POSE)
    assert res["visible"] > 0 and res["failed"] == 0
    e = om.export()
    assert len(e["coords"]) > 0
    # voxel corner points (block * 8 + local) * vs, local index x + 8y + 64z
    loc = np.arange(512)
    lx, ly, lz = loc % 8, (loc // 8) % 8, loc // 64
    z = (e["coords"][:, 2:3] * 8 + lz[None, :]) * VS
    w = e["weight"]
    assert set(np.unique(w)) <= {0.0, 1.0}
    obs = w > 0
    want = np.minimum(1.0, (D - z) / MU)
    assert np.abs(e["tsdf"][obs] - want[obs]).max() < 1e-5
    # observed exactly where the voxel projects into the image and lies at most mu behind the wall
    assert (z[obs] <= D + MU + 1e-6).all()
    assert np.isclose(w[(np.abs(z - D) < 0.5 * float(MU))].mean(), 1.0, atol=0.2)


@pytest.mark.parametrize("precision", [O.FP32, O.FP64])
def test_wall_raycast_and_mesh_lie_on_the_wall(precision):
    om = O.OracleMap(W, H, K, 4096, VS, precision=precision, storage="f32", with_color=False)
    for _ in range(2):
        om.fuse(wall(), None, POSE)
    v = om.raycast(POSE)
    hit = np.isfinite(v[..., 0])
    assert hit[4:-4, 4:-4].mean() > 0.95
    assert np.abs(v[hit][:, 2] - D).max() < 1e-3  # a linear field: trilinear + refinement land on it
    assert (v[hit][:, 3] == 1.0).all()
    n, verts, norms = om.polygonize()
    assert n > 100
    zs = verts.reshape(-1, 3)[:, 2]
    assert np.abs(zs - D).max() < 1e-4
    nz = norms.reshape(-1, 3)[:, 2]
    assert (np.abs(np.abs(nz) - 1.0) < 1e-3).mean() > 0.95  # facing the camera


def test_depth_validity_rules():
    for depth in (0.0, 0.05, 5.5, np.nan):
        om = O.OracleMap(W, H, K, 4096, VS, storage="f32", with_color=False)
        res = om.fuse(wall(depth), None, POSE)
        assert om.num_blocks() == 0 and res["visible"] == 0, depth
    om = O.OracleMap(W, H, K, 4096, VS, storage="f32", with_color=False)
    om.fuse(wall(4.9), None, POSE)
    assert om.num_blocks() > 0


def test_weight_cap_and_colour_blend():
    om = O.OracleMap(W, H, K, 4096, VS, storage="f32", max_weight=3, with_color=True)
    c1 = np.full((H, W, 3), (100, 40, 250), np.uint8)
    c2 = np.full((H, W, 3), (200, 90, 10), np.uint8)
    om.fuse(wall(), c1, POSE)
    e1 = om.export()
    obs1 = e1["weight"] > 0
    assert (e1["rgb"][obs1] == (100, 40, 250)).all()  # first observation copies the colour
    om.fuse(wall(), c2, POSE)
    e2 = om.export()
    obs2 = e2["weight"] > 0
    want = np.floor(0.7 * np.array([100, 40, 250]) + 0.3 * np.array([200, 90, 10]) + 1e-4).astype(np.uint8)
    seen_twice = e2["weight"] == 2
    assert seen_twice.any() and (e2["rgb"][seen_twice] == want).all()
    for _ in range(4):
        om.fuse(wall(), c2, POSE)
    assert om.export()["weight"].max() == 3


def test_fp32_and_fp64_modes_agree_on_a_room_frame():
    from voxelmapping_b200 import synth
    wl = synth.WORKLOADS["room_small"]
    d, _, pose = synth.Scene(wl).render(0, noisy=False, dropout=0.0)
    dm = synth.depth_to_metres(d)
    maps = [O.OracleMap(wl.width, wl.height, wl.K, 1 << 16, wl.voxel_size, precision=p, storage="f32")
            for p in (O.FP32, O.FP64)]
    for om in maps:
        om.fuse(dm, None, pose)
    k32, k64 = (set(map(tuple, om.export()["coords"])) for om in maps)
    # a sample on a block boundary can round into either neighbour (0.4 % of
    # blocks on this noise-free frame)
    assert len(k32 ^ k64) <= 1e-2 * len(k32)
    v32, v64 = (om.raycast(pose) for om in maps)
    both = np.isfinite(v32[..., 0]) & np.isfinite(v64[..., 0])
    assert both.mean() > 0.5
    assert (np.abs(v32[..., 2][both] - v64[..., 2][both]) <= 1e-3).mean() >= 0.995


def sphere_depth(center, radius):
    """Depth image of a sphere seen from the origin along +z (NaN where missed)."""
    u, v = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    d = np.stack([(u - K[0, 2]) / F, (v - K[1, 2]) / F, np.ones_like(u)], -1)  # ray with z = 1
    c = np.asarray(center, np.float64)
    a = (d * d).sum(-1)
    b = (d * c).sum(-1)
    disc = b * b - a * ((c * c).sum() - radius * radius)
    t = (b - np.sqrt(np.maximum(disc, 0))) / a  # depth = t (z component of the ray is 1)
    return np.where(disc > 0, t, np.nan).astype(np.float32)


@pytest.mark.parametrize("precision", [O.FP32, O.FP64])
def test_sphere_raycast_lands_on_the_surface(precision):
    center, radius = (0.05, -0.03, 1.2), 0.35
    depth = sphere_depth(center, radius)
    om = O.OracleMap(W, H, K, 8192, VS, precision=precision, storage="f32", with_color=False)
    om.fuse(np.nan_to_num(depth, nan=0.0), None, POSE)
    v = om.raycast(POSE)
    hit = np.isfinite(v[..., 0])
    inside = np.isfinite(depth)
    core = inside & (np.abs(depth - depth[inside].min()) < 0.15)  # away from the grazing rim
    assert hit[core].mean() > 0.98
    pts = v[hit & core][:, :3].astype(np.float64)
    r = np.linalg.norm(pts - np.array(center), axis=-1)
    assert np.abs(r - radius).max() < 2e-3  # within a quarter voxel of the analytic surface


def test_normals_of_a_planar_vertex_map():
    # vertices of the plane z = 1 + 0.5 x: the normal is (-0.5, 0, 1) normalised, up to sign
    u, v = np.meshgrid(np.arange(W, dtype=np.float32), np.arange(H, dtype=np.float32))
    x = (u - 31.5) / 50.0
    y = (v - 23.5) / 50.0
    z = 1.0 + 0.5 * x
    vm = np.stack([x, y, z, np.ones_like(x)], -1).astype(np.float32)
    nm = O.compute_normal(vm)
    want = np.array([-0.5, 0.0, 1.0]) / np.linalg.norm([-0.5, 0.0, 1.0])
    interior = nm[1:-1, 1:-1, :3].reshape(-1, 3)
    assert np.abs(np.abs(interior @ want) - 1.0).max() < 1e-5
    assert np.isnan(nm[-1]).all() and np.isnan(nm[:, -1]).all()  # last row and column are undefined


def restated_blocks(depth, t, R):
    """Block set of the reference's allocation (depth_fusion.cu:32-59) for a
    camera with identity rotation at translation t, restated in numpy in the
    arithmetic type R: band ends floored to voxels, the segment between them
    sampled at ceil(2 |dir|) points by repeated addition, each sample
    truncated toward zero (cast<int>) and then mapped voxel -> block."""
    vs, tdh = R(np.float32(VS)), R(np.float32(VS) * np.float32(4)) * R(0.5)
    ifx, ify = R(1.0 / np.float64(np.float32(F))), R(1.0 / np.float64(np.float32(F)))
    cx, cy = R(np.float32(K[0, 2])), R(np.float32(K[1, 2]))
    y, x = np.mgrid[0:H, 0:W]
    d = depth.astype(R).ravel()
    dn = np.maximum(d - tdh, R(0.1))
    df = np.maximum(d + tdh, R(0.1))
    ends = []
    for z in (dn, df):
        u = np.stack([ifx * (x.ravel().astype(R) - cx) * z, ify * (y.ravel().astype(R) - cy) * z, z], 1).astype(R)
        w = (np.asarray(t, np.float64).astype(R)[None, :] + u).astype(R)
        ends.append(np.floor(w / vs).astype(np.int64))
    pn, pf = ends
    dirv = (pf - pn).astype(R)
    n = np.ceil(2.0 * np.sqrt((dirv.astype(np.float64) ** 2).sum(1))).astype(np.int64)
    with np.errstate(divide="ignore", invalid="ignore"):
        step = (dirv / (n - 1).astype(R)[:, None]).astype(R)
    pos = pn.astype(R)
    out = set()
    for k in range(int(n.max())):
        live = n > k
        v = np.trunc(pos[live]).astype(np.int64)
        q = np.where(v < 0, v - 7, v)
        b = np.where(q < 0, -((-q) // 8), q // 8)
        out |= set(map(tuple, b))
        pos = (pos + step).astype(R)
    return out


@pytest.mark.parametrize("precision", [O.FP32, O.FP64])
def test_negative_octant_allocation_follows_the_reference_rule(precision):
    # a wall seen from a camera in the negative octant: the reference truncates
    # band samples toward zero (cast<int>) where fusion floors
    # (map_struct.h:111-180), and whether the band's last sample, reached by
    # repeated addition, lands just above a negative integer decides whether a
    # second layer of blocks is touched; the oracle must follow that rule in
    # either arithmetic type
    R = np.float32 if precision == O.FP32 else np.float64
    sb = np.array([-25, -20, -38], np.int64)
    pose = np.eye(4)
    pose[:3, 3] = sb * 8 * VS
    depth = np.full((H, W), 1.003, np.float32)  # surface and band ends off the voxel boundaries
    maps = []
    for p in (POSE, pose):
        om = O.OracleMap(W, H, K, 4096, VS, precision=precision, storage="f32", with_color=False)
        om.fuse(depth, None, p)
        maps.append(om)
    k0 = set(map(tuple, maps[0].export()["coords"].astype(np.int64)))
    k1 = set(map(tuple, maps[1].export()["coords"].astype(np.int64)))
    assert k0 == restated_blocks(depth, (0, 0, 0), R)
    want = restated_blocks(depth, pose[:3, 3], R)
    assert all(min(b) < 0 for b in k1)
    assert k1 == want  # FP32: 342 blocks in one layer; FP64: 598, the last samples reach z = -22
    # fusion and ray marching floor, so the surface itself is where it was
    v0, v1 = maps[0].raycast(POSE), maps[1].raycast(pose)
    both = np.isfinite(v0[..., 0]) & np.isfinite(v1[..., 0])
    assert both[4:-4, 4:-4].mean() > 0.95
    assert np.abs(v1[..., 2][both] - 1.003).max() < 1e-3
    assert np.abs(v1[..., 2][both] - v0[..., 2][both]).max() < 1e-3


def test_full_pool_keeps_its_blocks_and_counts_refusals():
    full = O.OracleMap(W, H, K, 4096, VS, storage="f32", with_color=False)
    need = full.fuse(wall(), None, POSE)["new"]
    om = O.OracleMap(W, H, K, 50, VS, storage="f32", with_color=False)
    res = om.fuse(wall(), None, POSE)
    assert need > 50 and res["new"] == 50 and res["failed"] > 0 and om.num_blocks() == 50
    kept = set(map(tuple, om.export()["coords"]))
    assert kept <= set(map(tuple, full.export()["coords"]))
    e = om.export()
    assert (e["weight"] > 0).any(axis=1).all()  # the blocks it kept are fused
    res2 = om.fuse(wall(), None, POSE)
    assert res2["new"] == 0 and res2["failed"] > 0 and set(map(tuple, om.export()["coords"])) == kept


@pytest.mark.parametrize("storage", ["ref", "i16", "f16"])
def test_wall_tsdf_quantised_like_the_storage_format(storage):
    om = O.OracleMap(W, H, K, 4096, VS, storage=storage, with_color=False)
    om.fuse(wall(), None, POSE)
    e = om.export()
    loc = np.arange(512)
    z = (e["coords"][:, 2:3] * 8 + (loc // 64)[None, :]) * VS
    obs = e["weight"] > 0
    want = np.minimum(1.0, (D - z) / MU)[obs]
    got = e["tsdf"][obs]
    if storage == "f16":
        # IEEE half, round to nearest even
        assert np.array_equal(got, want.astype(np.float16).astype(np.float64))
    else:
        # int16 x 32767, truncated toward zero (packFloat, map_struct.h:72-80)
        codes = np.round(got * 32767)
        assert np.abs(got * 32767 - codes).max() < 1e-3
        assert np.array_equal(codes, np.trunc(want * 32767))


def test_sixteen_bit_weights_cap_above_255():
    om = O.OracleMap(W, H, K, 4096, VS, storage="i16", max_weight=260, with_color=False)
    for _ in range(262):
        om.fuse(wall(), None, POSE)
    w = om.export()["weight"]
    assert w.max() == 260 and set(np.unique(w)) <= {0.0, 260.0}


@pytest.mark.parametrize("precision", [O.FP32, O.FP64])
def test_sphere_mesh_lies_on_the_surface_with_outward_normals(precision):
    center, radius = np.array([0.05, -0.03, 1.2]), 0.35
    om = O.OracleMap(W, H, K, 8192, VS, precision=precision, storage="f32", with_color=False)
    om.fuse(np.nan_to_num(sphere_depth(center, radius), nan=0.0), None, POSE)
    n, verts, norms = om.polygonize()
    assert n > 1000
    p = verts.reshape(-1, 3).astype(np.float64)
    r = np.linalg.norm(p - center, axis=1)
    radial = (p - center) / r[:, None]
    facing = (radial * -p / np.linalg.norm(p, axis=1)[:, None]).sum(1) > 0.9  # the cap facing the camera
    assert facing.mean() > 0.05
    # one 64x48 frame: a pixel covers 2.5 voxels at 1 m and each voxel takes its nearest pixel's depth
    assert np.abs(r[facing] - radius).max() < 0.5 * VS
    assert np.abs(r - radius).max() < 1.5 * VS  # grazing rim included
    # face normals point out of the surface, into the observed free space (TSDF > 0)
    assert ((norms.reshape(-1, 3) * radial).sum(1) > 0).all()

/*
 * Precision-generic body of the CPU oracle (test infrastructure only).
 * Included twice by vmap_oracle.c:
 *   R = float,  SFX = _f, FMA = fmaf   -> reference FP32 arithmetic
 *   R = double, SFX = _d, FMA = fma    -> FP64 accuracy oracle
 * Every function cites the reference code it restates.
 */
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

typedef struct { R m[3][4]; } FN(xform_t); /* 3x4 affine, row-major */

static void FN(make_xform)(const double p[16], FN(xform_t) * t)
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) t->m[r][c] = (R)p[4 * r + c];
}

/* Eigen 3.3 Transform<.,3,Affine> * Vector3 (map_struct.h:201,212): the 4x4
 * matrix times (v, 1), each row's redux in halves, (c0 + c1) + (c2 + c3) with
 * c3 = m_i3 * 1; nvcc contracts the first product of each half. Pinned by the
 * arithmetic probe of the reference's own build (oracle/ref_harness.cu). */
static inline void FN(xform_pt)(const FN(xform_t) * t, const R v[3], R out[3])
{
    for (int i = 0; i < 3; ++i)
        out[i] = FMA(t->m[i][0], v[0], t->m[i][1] * v[1]) + FMA(t->m[i][2], v[2], t->m[i][3]);
}

/* unproject (map_struct.h:189-194): (ifx*(x-cx))*z, (ify*(y-cy))*z, z */
static inline void FN(unproject)(int x, int y, R z, R ifx, R ify, R cx, R cy, R out[3])
{
    out[0] = ifx * ((R)x - cx) * z;
    out[1] = ify * ((R)y - cy) * z;
    out[2] = z;
}

/* Eigen squaredNorm(): v0^2 + (v1^2 + v2^2) with contraction. */
static inline R FN(sqnorm)(const R v[3]) { return FMA(v[0], v[0], FMA(v[1], v[1], v[2] * v[2])); }

/* Eigen normalized(): v / sqrt(|v|^2) when |v|^2 > 0, else v unchanged.
 * Inside normalized() nvcc contracts the squared norm as v0^2 + (v2^2 + v1^2)
 * (pinned by the arithmetic probe of the reference's own build). */
static inline void FN(normalize)(R v[3])
{
    R s = FMA(v[0], v[0], FMA(v[2], v[2], v[1] * v[1]));
    if (s > 0) {
        R n = SQRT(s);
        v[0] = v[0] / n;
        v[1] = v[1] / n;
        v[2] = v[2] / n;
    }
}

/* Eigen cross(): a1*b2 - a2*b1 ... contracted as fma(a1, b2, -(a2*b1)). */
static inline void FN(cross)(const R a[3], const R b[3], R out[3])
{
    out[0] = FMA(a[1], b[2], -(a[2] * b[1]));
    out[1] = FMA(a[2], b[0], -(a[0] * b[2]));
    out[2] = FMA(a[0], b[1], -(a[1] * b[0]));
}

/* checkVertexVisible / checkBlockVisible (map_struct.h:204-244). */
static int FN(block_visible)(const int32_t bp[3], const FN(xform_t) * tinv, R vs, int cols, int rows,
                             R fx, R fy, R cx, R cy)
{
    const R scale = vs * (R)8;
    for (int c = 0; c < 8; ++c) {
        R w[3] = {(R)(bp[0] + (c & 1)) * scale, (R)(bp[1] + ((c >> 1) & 1)) * scale,
                  (R)(bp[2] + ((c >> 2) & 1)) * scale};
        R p[3];
        FN(xform_pt)(tinv, w, p);
        R px = fx * p[0] / p[2] + cx;
        R py = fy * p[1] / p[2] + cy;
        if (!(px < 0 || py < 0 || px > (R)(cols - 1) || py > (R)(rows - 1) || p[2] < (R)ORC_MIN_DEPTH ||
              p[2] > (R)ORC_MAX_DEPTH))
            return 1;
    }
    return 0;
}

/* ---- voxel storage access ------------------------------------------------ */
static inline R FN(load_tsdf)(const orc_map* m, size_t i)
{
#if ORC_IS_FP64
    return m->tsdf64[i];
#else
    int32_t c = m->tsdf_code[i];
    switch (m->cfg.storage) {
    case ORC_STORE_F32: { float f; memcpy(&f, &c, 4); return f; }
    case ORC_STORE_F16: return half_to_float((uint16_t)c);
    default: return (float)c / 32767.0f; /* unpackFloat, map_struct.h:72-75 */
    }
#endif
}

static inline void FN(store_tsdf)(orc_map* m, size_t i, R v)
{
#if ORC_IS_FP64
    m->tsdf64[i] = v;
#else
    switch (m->cfg.storage) {
    case ORC_STORE_F32: { int32_t c; memcpy(&c, &v, 4); m->tsdf_code[i] = c; break; }
    case ORC_STORE_F16: m->tsdf_code[i] = float_to_half(v); break;
    default: m->tsdf_code[i] = (int16_t)f2i_rz(v * 32767.0f); /* packFloat, map_struct.h:77-80 */
    }
#endif
}

static inline R FN(load_w)(const orc_map* m, size_t i)
{
#if ORC_IS_FP64
    return m->wt64[i];
#else
    return m->wt32[i];
#endif
}

static inline void FN(store_w)(orc_map* m, size_t i, R v)
{
#if ORC_IS_FP64
    m->wt64[i] = v;
#else
    m->wt32[i] = v;
#endif
}

/* ---- allocation: CreateBlockLineTracingFunctor (depth_fusion.cu:32-59) ---- */
typedef struct { int32_t* b; int n, cap; } FN(blist_t);

static void FN(blist_push)(FN(blist_t) * l, const int32_t b[3])
{
    if (l->n == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 256;
        l->b = (int32_t*)realloc(l->b, sizeof(int32_t) * 3 * (size_t)l->cap);
    }
    memcpy(l->b + 3 * (size_t)l->n, b, 12);
    l->n++;
}

static int FN(allocate)(orc_map* m, const float* depth, const double pose[16], int* n_failed_out)
{
    const orc_config* c = &m->cfg;
    const int W = c->width, H = c->height;
    FN(xform_t) T;
    FN(make_xform)(pose, &T);
    const R vs = (R)c->voxel_size;
    const R tdh = (R)c->truncation * (R)0.5;
    const R ifx = (R)(1.0 / (double)c->fx), ify = (R)(1.0 / (double)c->fy);
    const R cx = (R)c->cx, cy = (R)c->cy;
    const R dmin = (R)ORC_MIN_DEPTH, dmax = (R)ORC_MAX_DEPTH;

    FN(blist_t)* rows = (FN(blist_t)*)calloc((size_t)H, sizeof(FN(blist_t)));
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const R d = (R)depth[(size_t)y * W + x];
            if (d != d || d < dmin || d > dmax) continue;
            R dn = d - tdh, df = d + tdh;
            dn = dn > dmin ? dn : dmin; /* max(depthMin, .) */
            df = df > dmin ? df : dmin;
            if (dn >= df) continue;
            R u[3], w[3];
            int32_t pn[3], pf[3];
            FN(unproject)(x, y, dn, ifx, ify, cx, cy, u);
            FN(xform_pt)(&T, u, w);
            for (int i = 0; i < 3; ++i) pn[i] = R2I_RZ(FLOOR(w[i] / vs)); /* worldPtToVoxelPos */
            FN(unproject)(x, y, df, ifx, ify, cx, cy, u);
            FN(xform_pt)(&T, u, w);
            for (int i = 0; i < 3; ++i) pf[i] = R2I_RZ(FLOOR(w[i] / vs));
            /* end points outside +-2^23 voxels (+-2^20 blocks): the product
             * cannot key such blocks and skips the pixel; so does the oracle */
            int out_of_range = 0;
            for (int i = 0; i < 3; ++i)
                out_of_range |= pn[i] < -(1 << 23) || pn[i] >= (1 << 23) || pf[i] < -(1 << 23) || pf[i] >= (1 << 23);
            if (out_of_range) continue;
            R dir[3] = {(R)(pf[0] - pn[0]), (R)(pf[1] - pn[1]), (R)(pf[2] - pn[2])};
            const R len = SQRT(FN(sqnorm)(dir));
            const int nsteps = (int)ceil(2.0 * (double)len);
            for (int i = 0; i < 3; ++i) dir[i] = dir[i] / (R)(nsteps - 1);
            R p[3] = {(R)pn[0], (R)pn[1], (R)pn[2]};
            int32_t last[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
            for (int s = 0; s < nsteps; ++s) {
                int32_t b[3];
                for (int i = 0; i < 3; ++i) b[i] = voxel_to_block(R2I_RZ(p[i])); /* cast<int>: truncation */
                if (b[0] != last[0] || b[1] != last[1] || b[2] != last[2]) {
                    FN(blist_push)(&rows[y], b);
                    memcpy(last, b, 12);
                }
                for (int i = 0; i < 3; ++i) p[i] = p[i] + dir[i];
            }
        }
    }
    int n_new = 0, n_failed = 0;
    for (int y = 0; y < H; ++y) {
        for (int k = 0; k < rows[y].n; ++k) {
            int r = orc_insert(m, rows[y].b + 3 * (size_t)k);
            if (r == 1) n_new++;
            else if (r < 0) n_failed++;
        }
    }
    /* unique blocks the frame's band samples touched (its A) */
    uint8_t* seen = (uint8_t*)calloc(m->nblk > 0 ? (size_t)m->nblk : 1, 1);
    int touched = 0;
    for (int y = 0; y < H; ++y) {
        for (int k = 0; k < rows[y].n; ++k) {
            const int bi = orc_find(m, rows[y].b + 3 * (size_t)k);
            if (bi >= 0 && !seen[bi]) {
                seen[bi] = 1;
                touched++;
            }
        }
        free(rows[y].b);
    }
    free(seen);
    free(rows);
    m->last_alloc_blocks = touched;
    if (n_failed_out) *n_failed_out = n_failed;
    return n_new;
}

/* ---- fusion: CheckEntryVisibilityFunctor + DepthFusionFunctor /
 *      ImageFusionFunctor (depth_fusion.cu:82-196, 328-380) ------------------ */
static int FN(integrate)(orc_map* m, const float* depth, const uint8_t* rgb, const double pose[16])
{
    const orc_config* c = &m->cfg;
    const int W = c->width, H = c->height;
    double invd[16];
    orc_pose_inverse(pose, invd);
    FN(xform_t) Ti;
    FN(make_xform)(invd, &Ti);
    const R vs = (R)c->voxel_size, mu = (R)c->truncation;
    const R fx = (R)c->fx, fy = (R)c->fy, cx = (R)c->cx, cy = (R)c->cy;
    const R dmin = (R)ORC_MIN_DEPTH, dmax = (R)ORC_MAX_DEPTH;
    const R wmax = (R)c->max_weight;
    const int nb = m->nblk;
    int nvis = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : nvis)
    for (int b = 0; b < nb; ++b) {
        const int32_t* bp = m->coords + 3 * (size_t)b;
        if (!FN(block_visible)(bp, &Ti, vs, W, H, fx, fy, cx, cy)) continue;
        nvis++;
        for (int z = 0; z < 8; ++z)
            for (int y = 0; y < 8; ++y)
                for (int x = 0; x < 8; ++x) {
                    R wp[3] = {(R)(bp[0] * 8 + x) * vs, (R)(bp[1] * 8 + y) * vs, (R)(bp[2] * 8 + z) * vs};
                    R p[3];
                    FN(xform_pt)(&Ti, wp, p);
                    /* __float2int_rd(fx*p0/p2 + cx + 0.5): the double 0.5 add
                     * rounds back to float, i.e. a float add. */
                    const int u = R2I_RD(fx * p[0] / p[2] + cx + (R)0.5);
                    const int v = R2I_RD(fy * p[1] / p[2] + cy + (R)0.5);
                    if (u < 0 || v < 0 || u > W - 1 || v > H - 1) continue;
                    const R d = (R)depth[(size_t)v * W + u];
                    if (d != d || d > dmax || d < dmin) continue;
                    R sdf = d - p[2];
                    if (sdf < -mu) continue;
                    sdf = sdf / mu;
                    sdf = sdf < (R)1 ? sdf : (R)1; /* fmin(1, .) */
                    const size_t vi = (size_t)b * 512 + (size_t)(z * 64 + y * 8 + x);
                    const R ow = FN(load_w)(m, vi);
                    if (ow == 0) {
                        FN(store_tsdf)(m, vi, sdf);
                        FN(store_w)(m, vi, (R)1);
                        if (rgb && m->rgb)
                            memcpy(m->rgb + 3 * vi, rgb + 3 * ((size_t)v * W + u), 3);
                    } else {
                        const R os = FN(load_tsdf)(m, vi);
                        FN(store_tsdf)(m, vi, FMA(os, ow, sdf) / (ow + (R)1));
                        const R nw = ow + (R)1;
                        FN(store_w)(m, vi, nw < wmax ? nw : wmax);
                        if (rgb && m->rgb) {
                            uint8_t* o = m->rgb + 3 * vi;
                            const uint8_t* n = rgb + 3 * ((size_t)v * W + u);
                            for (int k = 0; k < 3; ++k) /* (0.7*old + 0.3*new).cast<uchar> */
                                o[k] = (uint8_t)R2I_RZ(FMA((R)0.7f, (R)o[k], (R)0.3f * (R)n[k]));
                        }
                    }
                }
    }
    return nvis;
}

/* ---- raycast: MapRenderingDelegate (ray_tracing.cu:272-400) --------------- */
/* lookup cache of one ray (or cube); `touched`, when set, marks every
 * allocated block a lookup finds (the unique blocks any ray sampled) */
typedef struct { int32_t key[3]; int32_t blk; uint8_t* touched; } FN(cache_t);

static inline R FN(read_sdf)(const orc_map* m, FN(cache_t) * cache, const R p[3], int* valid)
{
    int32_t v[3], b[3];
    for (int i = 0; i < 3; ++i) {
        v[i] = R2I_RZ(FLOOR(p[i]));
        b[i] = voxel_to_block(v[i]);
    }
    if (b[0] != cache->key[0] || b[1] != cache->key[1] || b[2] != cache->key[2]) {
        memcpy(cache->key, b, 12);
        cache->blk = orc_find(m, b);
        if (cache->touched && cache->blk >= 0) cache->touched[cache->blk] = 1;
    }
    if (cache->blk >= 0) {
        const size_t vi = (size_t)cache->blk * 512 + (size_t)voxel_local_idx(v);
        if (FN(load_w)(m, vi) != 0) {
            *valid = 1;
            return FN(load_tsdf)(m, vi);
        }
    }
    *valid = 0;
    return (R)1;
}

static R FN(read_sdf_interp)(const orc_map* m, FN(cache_t) * cache, const R p[3], int* valid)
{
    const R fx = p[0] - FLOOR(p[0]), fy = p[1] - FLOOR(p[1]), fz = p[2] - FLOOR(p[2]);
    R s[8];
    int ok = 1, v;
    for (int c = 0; c < 8; ++c) {
        /* corner order of read_sdf_interped: x fastest, then y, then z */
        R q[3] = {p[0] + (R)(c & 1), p[1] + (R)((c >> 1) & 1), p[2] + (R)((c >> 2) & 1)};
        s[c] = FN(read_sdf)(m, cache, q, &v);
        ok &= v;
    }
    const R r0 = FMA((R)1 - fx, s[0], fx * s[1]);
    const R r1 = FMA((R)1 - fx, s[2], fx * s[3]);
    const R r2 = FMA((R)1 - fy, r0, fy * r1);
    const R r4 = FMA((R)1 - fx, s[4], fx * s[5]);
    const R r5 = FMA((R)1 - fx, s[6], fx * s[7]);
    const R r3 = FMA((R)1 - fy, r4, fy * r5);
    *valid = ok;
    return FMA((R)1 - fz, r2, fz * r3);
}

static int FN(raycast)(const orc_map* m, const double pose[16], float* vmap, uint8_t* touched)
{
    const orc_config* c = &m->cfg;
    const int W = c->width, H = c->height;
    double invd[16];
    orc_pose_inverse(pose, invd);
    FN(xform_t) T, Ti;
    FN(make_xform)(pose, &T);
    FN(make_xform)(invd, &Ti);
    const R ifx = (R)(1.0 / (double)c->fx), ify = (R)(1.0 / (double)c->fy);
    const R cx = (R)c->cx, cy = (R)c->cy;
    const R vsinv = (R)(1.0 / (double)c->voxel_size);
    const R rts = (R)c->truncation / (R)c->voxel_size; /* raytraceStep */
    int hits = 0;
#pragma omp parallel for schedule(dynamic, 2) reduction(+ : hits)
    for (int y = 0; y < H; ++y) {
        FN(cache_t) cache = {{INT32_MIN, INT32_MIN, INT32_MIN}, -1, touched};
        for (int x = 0; x < W; ++x) {
            float* out = vmap + 4 * ((size_t)y * W + x);
            out[0] = out[1] = out[2] = out[3] = NAN;
            R pt[3], bs[3], be[3], dir[3];
            FN(unproject)(x, y, (R)ORC_MIN_DEPTH, ifx, ify, cx, cy, pt);
            R dist_s = SQRT(FN(sqnorm)(pt)) * vsinv;
            FN(xform_pt)(&T, pt, bs);
            for (int i = 0; i < 3; ++i) bs[i] = bs[i] * vsinv;
            FN(unproject)(x, y, (R)ORC_MAX_DEPTH, ifx, ify, cx, cy, pt);
            const R dist_e = SQRT(FN(sqnorm)(pt)) * vsinv;
            FN(xform_pt)(&T, pt, be);
            for (int i = 0; i < 3; ++i) be[i] = be[i] * vsinv;
            for (int i = 0; i < 3; ++i) dir[i] = be[i] - bs[i];
            FN(normalize)(dir);
            R r[3] = {bs[0], bs[1], bs[2]};
            R sdf = (R)1, step;
            int valid = 0, found = 0;
            while (dist_s < dist_e) {
                sdf = FN(read_sdf)(m, &cache, r, &valid);
                if (sdf <= (R)0.5f && sdf >= (R)-0.5f) sdf = FN(read_sdf_interp)(m, &cache, r, &valid);
                if (sdf <= (R)0) break;
                if (valid) {
                    step = sdf * rts;
                    step = step > (R)1 ? step : (R)1;
                } else
                    step = (R)1;
                for (int i = 0; i < 3; ++i) r[i] = FMA(step, dir[i], r[i]);
                dist_s += step;
            }
            if (sdf <= (R)0) {
                step = sdf * rts;
                for (int i = 0; i < 3; ++i) r[i] = FMA(step, dir[i], r[i]);
                sdf = FN(read_sdf_interp)(m, &cache, r, &valid);
                step = sdf * rts;
                for (int i = 0; i < 3; ++i) r[i] = FMA(step, dir[i], r[i]);
                found = valid;
            }
            if (found) {
                R q[3] = {r[0] / vsinv, r[1] / vsinv, r[2] / vsinv}, o[3];
                FN(xform_pt)(&Ti, q, o);
                out[0] = (float)o[0];
                out[1] = (float)o[1];
                out[2] = (float)o[2];
                out[3] = 1.0f;
                hits++;
            }
        }
    }
    return hits;
}

/* ---- marching cubes: BuildVertexArray (marching_cubes.cu:52-242) ---------- */
static inline R FN(mc_interp)(R v1, R v2)
{
    /* interpolateLinear: thresholds are the double literal 1e-6 */
    if (fabs((double)((R)0 - v1)) < 1e-6) return (R)0;
    if (fabs((double)((R)0 - v2)) < 1e-6) return (R)1;
    if (fabs((double)(v1 - v2)) < 1e-6) return (R)0;
    return ((R)0 - v1) / (v2 - v1);
}

/* Returns the cube index (0 when the cube is skipped), fills verts[12][3]. */
static int FN(mc_cube)(const orc_map* m, FN(cache_t) * cache, const int32_t vp[3], R verts[12][3])
{
    static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                     {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    static const int edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                    {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    R s[8];
    for (int k = 0; k < 8; ++k) {
        R q[3] = {(R)(vp[0] + corner[k][0]), (R)(vp[1] + corner[k][1]), (R)(vp[2] + corner[k][2])};
        int valid;
        s[k] = FN(read_sdf)(m, cache, q, &valid);
        if (!valid) return 0;
    }
    int ci = 0;
    for (int k = 0; k < 8; ++k)
        if (s[k] < 0) ci |= 1 << k;
    if (ci == 0 || ci == 255) return 0;
    const R base[3] = {(R)vp[0], (R)vp[1], (R)vp[2]};
    for (int e = 0; e < 12; ++e) {
        const int a = edge[e][0], b = edge[e][1];
        if (((ci >> a) & 1) == ((ci >> b) & 1)) continue;
        const R t = FN(mc_interp)(s[a], s[b]);
        /* make_vertex: the moving axis gets val (or 1 - val when the edge runs
         * from the high corner to the low one), the others the corner offset */
        for (int i = 0; i < 3; ++i) {
            const int ca = corner[a][i], cb = corner[b][i];
            R off;
            if (ca == cb) off = (R)ca;
            else off = ca == 0 ? t : (R)1 - t;
            verts[e][i] = base[i] + off;
        }
    }
    return ci;
}

static long FN(polygonize)(const orc_map* m, float* verts, float* norms, long max_tris)
{
    const int nb = m->nblk;
    const R vs = (R)m->cfg.voxel_size;
    long* cnt = (long*)calloc((size_t)nb + 1, sizeof(long));
#pragma omp parallel for schedule(dynamic, 16)
    for (int b = 0; b < nb; ++b) {
        FN(cache_t) cache = {{INT32_MIN, INT32_MIN, INT32_MIN}, -1, NULL};
        R vv[12][3];
        long n = 0;
        const int32_t* bp = m->coords + 3 * (size_t)b;
        for (int z = 0; z < 8; ++z)
            for (int y = 0; y < 8; ++y)
                for (int x = 0; x < 8; ++x) {
                    int32_t vp[3] = {bp[0] * 8 + x, bp[1] * 8 + y, bp[2] * 8 + z};
                    int ci = FN(mc_cube)(m, &cache, vp, vv);
                    if (ci) n += g_tri_count[ci];
                }
        cnt[b + 1] = n;
    }
    for (int b = 0; b < nb; ++b) cnt[b + 1] += cnt[b];
    const long total = cnt[nb];
    if (verts || norms) {
#pragma omp parallel for schedule(dynamic, 16)
        for (int b = 0; b < nb; ++b) {
            if (cnt[b] >= max_tris) continue;
            FN(cache_t) cache = {{INT32_MIN, INT32_MIN, INT32_MIN}, -1, NULL};
            R vv[12][3];
            long t = cnt[b];
            const int32_t* bp = m->coords + 3 * (size_t)b;
            for (int z = 0; z < 8; ++z)
                for (int y = 0; y < 8; ++y)
                    for (int x = 0; x < 8; ++x) {
                        int32_t vp[3] = {bp[0] * 8 + x, bp[1] * 8 + y, bp[2] * 8 + z};
                        int ci = FN(mc_cube)(m, &cache, vp, vv);
                        if (!ci) continue;
                        for (int k = 0; g_tri_table[ci][k] != -1; k += 3, ++t) {
                            if (t >= max_tris) continue;
                            R tri[3][3];
                            for (int i = 0; i < 3; ++i) { /* reversed winding */
                                tri[2][i] = vv[g_tri_table[ci][k]][i] * vs;
                                tri[1][i] = vv[g_tri_table[ci][k + 1]][i] * vs;
                                tri[0][i] = vv[g_tri_table[ci][k + 2]][i] * vs;
                            }
                            R e1[3], e2[3], n[3];
                            for (int i = 0; i < 3; ++i) {
                                e1[i] = tri[1][i] - tri[0][i];
                                e2[i] = tri[2][i] - tri[0][i];
                            }
                            FN(cross)(e1, e2, n);
                            FN(normalize)(n);
                            for (int j = 0; j < 3; ++j)
                                for (int i = 0; i < 3; ++i) {
                                    if (verts) verts[9 * t + 3 * j + i] = (float)tri[j][i];
                                    if (norms) norms[9 * t + 3 * j + i] = (float)n[i];
                                }
                        }
                    }
        }
    }
    free(cnt);
    return total;
}

#undef FN
#undef CAT
#undef CAT_

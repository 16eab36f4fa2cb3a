/*
 * CPU oracle (test infrastructure only; see vmap_oracle.h for scope and the
 * reference lines each part restates). Build: oracle/Makefile.
 */
#include "vmap_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Reference constants: include/map_struct.h:6-10, src/vmapping.cpp:59,
 * src/depth_fusion.cu:193, src/ray_tracing.cu:7. */
#define ORC_MIN_DEPTH 0.1f
#define ORC_MAX_DEPTH 5.f
#define ORC_HASH_P0 73856093
#define ORC_HASH_P1 19349669
#define ORC_HASH_P2 83492791

static int g_tri_table[256][16];
static int g_tri_count[256];
static int g_tables_set = 0;

struct orc_map {
    orc_config cfg;
    int nblk, cap;
    int32_t* coords;     /* 3 per block */
    int32_t* tsdf_code;  /* FP32 mode: stored code per voxel */
    float* wt32;         /* FP32 mode: weight per voxel */
    double* tsdf64;      /* FP64 mode */
    double* wt64;
    uint8_t* rgb;        /* 3 per voxel, optional */
    /* block-coordinate hash map: open addressing, linear probing */
    int32_t* hkeys;      /* 3 per slot */
    int32_t* hvals;      /* block index or -1 */
    size_t hcap, hcount;
    int last_raycast_blocks; /* unique allocated blocks the last raycast read */
    int last_alloc_blocks;   /* unique blocks the last frame's allocation touched */
};

/* ---- GPU-semantics conversions (cvt.rzi / cvt.rmi saturate, NaN -> 0) ---- */
static inline int f2i_rz(double x)
{
    if (x != x) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return (int)x;
}
#define R2I_RZ(x) f2i_rz((double)(x))
#define R2I_RD(x) f2i_rz(floor((double)(x)))

/* IEEE binary16 conversions, round-to-nearest-even (as __float2half_rn). */
static float half_to_float(uint16_t h)
{
    uint32_t s = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1f, f = h & 0x3ff, u;
    if (e == 0) {
        if (f == 0) u = s;
        else { /* subnormal */
            float v = ldexpf((float)f, -24);
            memcpy(&u, &v, 4);
            u |= s;
        }
    } else if (e == 31) u = s | 0x7f800000u | (f << 13);
    else u = s | ((e + 112) << 23) | (f << 13);
    float out;
    memcpy(&out, &u, 4);
    return out;
}

static int32_t float_to_half(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    uint32_t s = (u >> 16) & 0x8000, e = (u >> 23) & 0xff, f = u & 0x7fffff;
    if (e == 0xff) return (int32_t)(s | 0x7c00 | (f ? 0x200 : 0));
    int ee = (int)e - 127 + 15;
    if (ee >= 31) return (int32_t)(s | 0x7c00);
    if (ee <= 0) { /* subnormal or zero */
        if (ee < -10) return (int32_t)s;
        uint32_t m = f | 0x800000;
        int shift = 14 - ee;
        uint32_t hm = m >> shift, rem = m & ((1u << shift) - 1), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (hm & 1))) hm++;
        return (int32_t)(s | hm);
    }
    uint32_t hm = f >> 13, rem = f & 0x1fff;
    uint32_t out = s | ((uint32_t)ee << 10) | hm;
    if (rem > 0x1000 || (rem == 0x1000 && (hm & 1))) out++;
    return (int32_t)out;
}

/* voxelPosToBlockPos (map_struct.h:131-141): subtract 7 if negative, then /8 */
static inline int32_t voxel_to_block(int32_t v) { return (v < 0 ? v - 7 : v) / 8; }
/* voxelPosToLocalIdx (map_struct.h:148-180): ((v % 8) + 8) % 8, z*64 + y*8 + x */
static inline int voxel_local_idx(const int32_t v[3])
{
    int l[3];
    for (int i = 0; i < 3; ++i) {
        l[i] = v[i] % 8;
        if (l[i] < 0) l[i] += 8;
    }
    return l[2] * 64 + l[1] * 8 + l[0];
}

/* hash (map_struct.h:104-109): int32 wrap-around products, C remainder. */
int orc_hash(int x, int y, int z, int n_buckets)
{
    int32_t r = (int32_t)(((uint32_t)x * (uint32_t)ORC_HASH_P0) ^ ((uint32_t)y * (uint32_t)ORC_HASH_P1) ^
                          ((uint32_t)z * (uint32_t)ORC_HASH_P2));
    r %= n_buckets;
    return r < 0 ? r + n_buckets : r;
}

/* ---- block-coordinate hash map (oracle bookkeeping, not the GPU layout) --- */
static size_t hslot(const int32_t b[3], size_t cap)
{
    uint64_t h = (uint64_t)(uint32_t)b[0] * 0x9E3779B97F4A7C15ull;
    h ^= (uint64_t)(uint32_t)b[1] * 0xC2B2AE3D27D4EB4Full;
    h ^= (uint64_t)(uint32_t)b[2] * 0x165667B19E3779F9ull;
    h ^= h >> 29;
    return (size_t)(h & (cap - 1));
}

static void hgrow(orc_map* m)
{
    size_t ncap = m->hcap ? m->hcap * 2 : 1 << 16;
    int32_t* nk = (int32_t*)malloc(sizeof(int32_t) * 3 * ncap);
    int32_t* nv = (int32_t*)malloc(sizeof(int32_t) * ncap);
    for (size_t i = 0; i < ncap; ++i) nv[i] = -2; /* -2 = empty slot */
    for (size_t i = 0; i < m->hcap; ++i) {
        if (m->hvals[i] == -2) continue;
        size_t s = hslot(m->hkeys + 3 * i, ncap);
        while (nv[s] != -2) s = (s + 1) & (ncap - 1);
        memcpy(nk + 3 * s, m->hkeys + 3 * i, 12);
        nv[s] = m->hvals[i];
    }
    free(m->hkeys);
    free(m->hvals);
    m->hkeys = nk;
    m->hvals = nv;
    m->hcap = ncap;
}

static int orc_find(const orc_map* m, const int32_t b[3])
{
    if (!m->hcap) return -1;
    size_t s = hslot(b, m->hcap);
    while (m->hvals[s] != -2) {
        const int32_t* k = m->hkeys + 3 * s;
        if (k[0] == b[0] && k[1] == b[1] && k[2] == b[2]) return m->hvals[s];
        s = (s + 1) & (m->hcap - 1);
    }
    return -1;
}

static void grow_pool(orc_map* m)
{
    int ncap = m->cap ? m->cap * 2 : 1024;
    if (ncap > m->cfg.num_blocks) ncap = m->cfg.num_blocks;
    size_t nv = (size_t)ncap * 512, ov = (size_t)m->cap * 512;
    m->coords = (int32_t*)realloc(m->coords, sizeof(int32_t) * 3 * (size_t)ncap);
    if (m->cfg.precision == ORC_FP64) {
        m->tsdf64 = (double*)realloc(m->tsdf64, sizeof(double) * nv);
        m->wt64 = (double*)realloc(m->wt64, sizeof(double) * nv);
        memset(m->tsdf64 + ov, 0, sizeof(double) * (nv - ov));
        memset(m->wt64 + ov, 0, sizeof(double) * (nv - ov));
    } else {
        m->tsdf_code = (int32_t*)realloc(m->tsdf_code, sizeof(int32_t) * nv);
        m->wt32 = (float*)realloc(m->wt32, sizeof(float) * nv);
        memset(m->tsdf_code + ov, 0, sizeof(int32_t) * (nv - ov));
        memset(m->wt32 + ov, 0, sizeof(float) * (nv - ov));
    }
    if (m->cfg.with_color) {
        m->rgb = (uint8_t*)realloc(m->rgb, 3 * nv);
        memset(m->rgb + 3 * ov, 0, 3 * (nv - ov));
    }
    m->cap = ncap;
}

/* createBlock (map_struct.h:304-354) without its lock skips: 1 = new block,
 * 0 = already present, -1 = pool exhausted (AllocateHashEntry fails). */
static int orc_insert(orc_map* m, const int32_t b[3])
{
    if (orc_find(m, b) >= 0) return 0;
    if (m->nblk >= m->cfg.num_blocks) return -1;
    if (2 * (m->hcount + 1) > m->hcap) hgrow(m);
    if (m->nblk == m->cap) grow_pool(m);
    size_t s = hslot(b, m->hcap);
    while (m->hvals[s] != -2) s = (s + 1) & (m->hcap - 1);
    memcpy(m->hkeys + 3 * s, b, 12);
    m->hvals[s] = m->nblk;
    m->hcount++;
    memcpy(m->coords + 3 * (size_t)m->nblk, b, 12);
    return (m->nblk++, 1);
}

/* Affine inverse of a row-major camera-to-world pose, in double:
 * inv(A) = adj(A) / det(A), t' = -inv(A) t. */
void orc_pose_inverse(const double p[16], double o[16])
{
    const double a = p[0], b = p[1], c = p[2], d = p[4], e = p[5], f = p[6], g = p[8], h = p[9], i = p[10];
    const double A = e * i - f * h, B = f * g - d * i, C = d * h - e * g;
    const double det = a * A + b * B + c * C;
    const double r = 1.0 / det;
    o[0] = A * r;
    o[1] = (c * h - b * i) * r;
    o[2] = (b * f - c * e) * r;
    o[4] = B * r;
    o[5] = (a * i - c * g) * r;
    o[6] = (c * d - a * f) * r;
    o[8] = C * r;
    o[9] = (b * g - a * h) * r;
    o[10] = (a * e - b * d) * r;
    for (int k = 0; k < 3; ++k)
        o[4 * k + 3] = -(o[4 * k] * p[3] + o[4 * k + 1] * p[7] + o[4 * k + 2] * p[11]);
    o[12] = o[13] = o[14] = 0.0;
    o[15] = 1.0;
}

/* ---- precision-generic bodies -------------------------------------------- */
#define R float
#define SFX _f
#define FMA fmaf
#define SQRT sqrtf
#define FLOOR floorf
#define ORC_IS_FP64 0
#include "oracle_impl.h"
#undef R
#undef SFX
#undef FMA
#undef SQRT
#undef FLOOR
#undef ORC_IS_FP64

#define R double
#define SFX _d
#define FMA fma
#define SQRT sqrt
#define FLOOR floor
#define ORC_IS_FP64 1
#include "oracle_impl.h"
#undef R
#undef SFX
#undef FMA
#undef SQRT
#undef FLOOR
#undef ORC_IS_FP64

/* ---- public API ---------------------------------------------------------- */
void orc_set_mc_tables(const int* t)
{
    for (int c = 0; c < 256; ++c) {
        int n = 0;
        for (int k = 0; k < 16; ++k) {
            g_tri_table[c][k] = t[16 * c + k];
            if (t[16 * c + k] != -1 && n == k) n = k + 1;
        }
        g_tri_count[c] = n / 3;
    }
    g_tables_set = 1;
}

orc_map* orc_create(const orc_config* cfg)
{
    if (!cfg || cfg->width <= 0 || cfg->height <= 0 || cfg->num_blocks <= 0 || cfg->voxel_size <= 0)
        return NULL;
    orc_map* m = (orc_map*)calloc(1, sizeof(orc_map));
    m->cfg = *cfg;
    return m;
}

void orc_reset(orc_map* m)
{
    free(m->coords);
    free(m->tsdf_code);
    free(m->wt32);
    free(m->tsdf64);
    free(m->wt64);
    free(m->rgb);
    free(m->hkeys);
    free(m->hvals);
    orc_config c = m->cfg;
    memset(m, 0, sizeof(*m));
    m->cfg = c;
}

int orc_last_raycast_blocks(const orc_map* m) { return m->last_raycast_blocks; }
int orc_last_alloc_blocks(const orc_map* m) { return m->last_alloc_blocks; }

void orc_destroy(orc_map* m)
{
    if (!m) return;
    orc_reset(m);
    free(m);
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}

int orc_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_allocate(orc_map* m, const float* depth, const double pose[16], int* n_failed)
{
    return m->cfg.precision == ORC_FP64 ? allocate_d(m, depth, pose, n_failed)
                                        : allocate_f(m, depth, pose, n_failed);
}

int orc_fuse(orc_map* m, const float* depth, const uint8_t* rgb, const double pose[16], int* n_new,
             int* n_failed)
{
    int nn = orc_allocate(m, depth, pose, n_failed);
    if (n_new) *n_new = nn;
    return m->cfg.precision == ORC_FP64 ? integrate_d(m, depth, rgb, pose) : integrate_f(m, depth, rgb, pose);
}

int orc_raycast(orc_map* m, const double pose[16], float* vmap)
{
    uint8_t* touched = (uint8_t*)calloc(m->nblk > 0 ? (size_t)m->nblk : 1, 1);
    const int hits = m->cfg.precision == ORC_FP64 ? raycast_d(m, pose, vmap, touched) : raycast_f(m, pose, vmap, touched);
    int u = 0;
    for (int b = 0; b < m->nblk; ++b) u += touched[b];
    free(touched);
    m->last_raycast_blocks = u;
    return hits;
}

long orc_polygonize(orc_map* m, float* verts, float* norms, long max_tris)
{
    if (!g_tables_set) return -1;
    return m->cfg.precision == ORC_FP64 ? polygonize_d(m, verts, norms, max_tris)
                                        : polygonize_f(m, verts, norms, max_tris);
}

/* computeNormalKernel (image_proc.cu:74-93), FP32. Pixels the reference leaves
 * unwritten (last row / column) and pixels with a NaN neighbour are NaN. */
void orc_compute_normal(const float* vm, int W, int H, float* nm)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float* o = nm + 4 * ((size_t)y * W + x);
            o[0] = o[1] = o[2] = o[3] = NAN;
            if (x >= W - 1 || y >= H - 1) continue;
            const int x10 = x - 1 > 0 ? x - 1 : 0, x01 = x + 1;
            const int y10 = y - 1 > 0 ? y - 1 : 0, y01 = y + 1;
            const float* v00 = vm + 4 * ((size_t)y * W + x10);
            const float* v01 = vm + 4 * ((size_t)y * W + x01);
            const float* v10 = vm + 4 * ((size_t)y10 * W + x);
            const float* v11 = vm + 4 * ((size_t)y01 * W + x);
            if (isnan(v00[0]) || isnan(v01[0]) || isnan(v10[0]) || isnan(v11[0])) continue;
            float a[3], b[3], n[3];
            for (int i = 0; i < 3; ++i) {
                a[i] = v01[i] - v00[i];
                b[i] = v11[i] - v10[i];
            }
            cross_f(a, b, n);
            normalize_f(n);
            o[0] = n[0];
            o[1] = n[1];
            o[2] = n[2];
            o[3] = 1.0f;
        }
}

/* renderPoint / renderSceneKernel (image_proc.cu:8-61): Phong, light at
 * (5,5,5), Ka 0.3, Kd 0.5, Ks 0.2, exponent 20, unit material colour. */
void orc_render_phong(const float* vm, const float* nm, int W, int H, uint8_t* rgba)
{
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            const float* p = vm + 4 * i;
            const float* n = nm + 4 * i;
            float col[3] = {4.f / 255.f, 2.f / 255.f, 2.f / 255.f};
            if (!isnan(p[0])) {
                float L[3] = {5.f - p[0], 5.f - p[1], 5.f - p[2]};
                float V[3] = {0.f - p[0], 0.f - p[1], 0.f - p[2]};
                normalize_f(L);
                normalize_f(V);
                const float nl = fmaf(n[0], L[0], fmaf(n[1], L[1], n[2] * L[2]));
                float Rv[3];
                for (int k = 0; k < 3; ++k) Rv[k] = fmaf(2.f * n[k], nl, -L[k]);
                normalize_f(Rv);
                const float rv = fmaf(Rv[0], V[0], fmaf(Rv[1], V[1], Rv[2] * V[2]));
                /* Ax*Ka*Dx + Lx*Kd*Dx*max(0,n.L) + Lx*Ks*Sx*pow(max(0,R.V), 20) with
                 * unit colours; both adds take a product, so both contract */
                const float I = fmaf(0.2f, powf(fmaxf(0.f, rv), 20.f), fmaf(0.5f, fmaxf(0.f, nl), 0.3f));
                col[0] = col[1] = col[2] = I;
            }
            for (int k = 0; k < 3; ++k) {
                float c = col[k] != col[k] ? 0.f : (col[k] < 0.f ? 0.f : (col[k] > 1.f ? 1.f : col[k]));
                rgba[4 * i + k] = (uint8_t)(c * 255.f);
            }
            rgba[4 * i + 3] = 255;
        }
}

/* compute_surface_point_kernel (marching_cubes.cu:314-328): (a + b + c) / 3 */
void orc_surface_points(const float* v, long n, float* pts)
{
#pragma omp parallel for schedule(static)
    for (long t = 0; t < n; ++t)
        for (int i = 0; i < 3; ++i) pts[3 * t + i] = (v[9 * t + i] + v[9 * t + 3 + i] + v[9 * t + 6 + i]) / 3.0f;
}

int orc_num_blocks(const orc_map* m) { return m->nblk; }

void orc_export(const orc_map* m, int32_t* coords, double* tsdf, double* weight, uint8_t* rgb)
{
    const size_t nv = (size_t)m->nblk * 512;
    if (coords) memcpy(coords, m->coords, sizeof(int32_t) * 3 * (size_t)m->nblk);
    for (size_t i = 0; i < nv; ++i) {
        if (m->cfg.precision == ORC_FP64) {
            if (tsdf) tsdf[i] = m->tsdf64[i];
            if (weight) weight[i] = m->wt64[i];
        } else {
            if (tsdf) tsdf[i] = load_tsdf_f(m, i);
            if (weight) weight[i] = m->wt32[i];
        }
    }
    if (rgb && m->rgb) memcpy(rgb, m->rgb, 3 * nv);
}

void orc_constants(int out[9])
{
    out[0] = 8;
    out[1] = (int)lround(ORC_MIN_DEPTH * 1000.0);
    out[2] = (int)lround(ORC_MAX_DEPTH * 1000.0);
    out[3] = 4;
    out[4] = 255;
    out[5] = ORC_HASH_P0;
    out[6] = ORC_HASH_P1;
    out[7] = ORC_HASH_P2;
    out[8] = 8;
}

/* The expression shapes of the reference's arithmetic probe
 * (oracle/ref_harness.cu, probe_kernel), evaluated with this oracle's FP32
 * helpers; a GPU test requires both to agree bit for bit. in: 20 floats per
 * item, out: 4 floats per item (unused lanes NaN). */
void orc_probe(int which, const float* in, int n, float* out)
{
    for (int k = 0; k < n; ++k) {
        const float* a = in + 20 * (size_t)k;
        float* o = out + 4 * (size_t)k;
        o[0] = o[1] = o[2] = o[3] = NAN;
        xform_t_f T;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) T.m[r][c] = a[4 * r + c];
        switch (which) {
        case 0: xform_pt_f(&T, a + 12, o); break;
        case 1: {
            float u[3];
            unproject_f((int)a[12], (int)a[13], a[14], a[15], a[16], a[17], a[18], u);
            xform_pt_f(&T, u, o);
            break;
        }
        case 2:
            o[0] = a[3] * a[0] / a[2] + a[5];
            o[1] = a[4] * a[1] / a[2] + a[6];
            break;
        case 3: o[0] = sqnorm_f(a); break;
        case 4: o[0] = sqrtf(sqnorm_f(a)); break;
        case 5: o[0] = a[0], o[1] = a[1], o[2] = a[2]; normalize_f(o); break;
        case 6: cross_f(a, a + 3, o); break;
        case 7: o[0] = fmaf(a[0], a[3], fmaf(a[1], a[4], a[2] * a[5])); break;
        case 8: o[0] = fmaf(1.0f - a[0], a[1], a[0] * a[2]); break;
        case 9: {
            const float w = (float)(unsigned char)a[1];
            o[0] = fmaf(a[0], w, a[2]) / (w + 1.0f);
            break;
        }
        case 10:
            for (int i = 0; i < 3; ++i) o[i] = (float)(uint8_t)f2i_rz((double)fmaf(0.7f, a[i], 0.3f * a[3 + i]));
            break;
        case 11:
            for (int i = 0; i < 3; ++i) o[i] = fmaf(a[3], a[4 + i], a[i]);
            break;
        case 12: {
            float p[4] = {a[0], a[1], a[2], 1.f}, nn[4] = {a[3], a[4], a[5], 1.f};
            uint8_t px[4];
            orc_render_phong(p, nn, 1, 1, px);
            for (int i = 0; i < 4; ++i) o[i] = (float)px[i];
            break;
        }
        case 13: o[0] = mc_interp_f(a[0], a[1]); break;
        default: break;
        }
    }
}


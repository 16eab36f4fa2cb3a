// Synthetic RGB-D scenes: an axis-aligned box room seen from inside plus
// seeded spheres, rendered exactly (ray-primitive intersection in FP64) into
// uint16 millimetre depth with an axial noise model and random dropouts, and
// per-object uint8 colour. Camera trajectories: a circle looking at the room
// centre and a figure-8 looking at a target that circles the room.
//
// Counter-based random numbers (splitmix64 of seed/frame/pixel) make every
// frame independent of thread count and order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "vmap_synth.h"

namespace {

inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline double u01(uint64_t h) { return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

struct Rng {
    uint64_t s;
    double next() { return u01(s = mix64(s)); }
};

inline void norm3(double v[3])
{
    double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (n > 0) {
        v[0] /= n;
        v[1] /= n;
        v[2] /= n;
    }
}

inline void cross3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

struct vmap_scene {
    vmap_scene_desc desc;
    double sphere[VMAP_SYNTH_MAX_SPHERES][4];  // cx, cy, cz, r
    uint8_t colour[6 + VMAP_SYNTH_MAX_SPHERES][3];
};

extern "C" {

int vmap_synth_scene_create(const vmap_scene_desc* d, vmap_scene** out)
{
    if (!d || !out || d->n_spheres < 0 || d->n_spheres > VMAP_SYNTH_MAX_SPHERES || d->size[0] <= 0 ||
        d->size[1] <= 0 || d->size[2] <= 0)
        return -1;
    vmap_scene* s = new vmap_scene();
    s->desc = *d;
    Rng rng{d->seed * 0x2545F4914F6CDD1Dull + 1};
    for (int k = 0; k < 6 + VMAP_SYNTH_MAX_SPHERES; ++k)
        for (int c = 0; c < 3; ++c) s->colour[k][c] = (uint8_t)(40 + (int)(rng.next() * 200.0));
    const double hx = d->size[0] * 0.5, hy = d->size[1] * 0.5, hz = d->size[2];
    const double rscale = std::fmin(1.0, std::fmin(d->size[0], d->size[1]) / 4.0);
    const double cam_r = d->cam_radius, cam_h = d->cam_height;
    for (int k = 0; k < d->n_spheres; ++k) {
        double c[3], r = 0;
        for (int attempt = 0; attempt < 1000; ++attempt) {
            r = (0.1 + 0.4 * rng.next()) * rscale;
            c[0] = -hx + r + (2 * hx - 2 * r) * rng.next();
            c[1] = -hy + r + (2 * hy - 2 * r) * rng.next();
            c[2] = r + (hz - 2 * r) * rng.next();
            // keep clear of the camera path: a horizontal ring/figure-8 of
            // half-width cam_r at height cam_h (0.25 m margin)
            const double rad = std::sqrt(c[0] * c[0] + c[1] * c[1]);
            const double dz = std::fabs(c[2] - cam_h);
            if (dz > r + 0.25 || rad > cam_r + r + 0.25) break;
        }
        s->sphere[k][0] = c[0];
        s->sphere[k][1] = c[1];
        s->sphere[k][2] = c[2];
        s->sphere[k][3] = r;
    }
    *out = s;
    return 0;
}

void vmap_synth_scene_destroy(vmap_scene* s) { delete s; }

int vmap_synth_scene_spheres(const vmap_scene* s, double* out)
{
    for (int k = 0; k < s->desc.n_spheres; ++k)
        for (int i = 0; i < 4; ++i) out[4 * k + i] = s->sphere[k][i];
    return s->desc.n_spheres;
}

// Camera-to-world pose (row-major 4x4, OpenCV camera axes: x right, y down,
// z forward) at `pos` looking at `target`, world z up.
static void look_at(const double pos[3], const double target[3], double* T)
{
    double f[3] = {target[0] - pos[0], target[1] - pos[1], target[2] - pos[2]};
    norm3(f);
    const double up[3] = {0, 0, 1};
    double r[3], dn[3];
    cross3(f, up, r);
    norm3(r);
    cross3(f, r, dn);
    for (int i = 0; i < 3; ++i) {
        T[4 * i + 0] = r[i];
        T[4 * i + 1] = dn[i];
        T[4 * i + 2] = f[i];
        T[4 * i + 3] = pos[i];
    }
    T[12] = T[13] = T[14] = 0;
    T[15] = 1;
}

int vmap_synth_trajectory(int kind, int n, double radius, double height, double* poses)
{
    if (n <= 0 || !poses) return -1;
    const double two_pi = 6.283185307179586;
    for (int i = 0; i < n; ++i) {
        const double t = two_pi * (double)i / (double)n;
        double pos[3], tgt[3];
        if (kind == VMAP_TRAJ_CIRCLE) {
            pos[0] = radius * std::cos(t);
            pos[1] = radius * std::sin(t);
            pos[2] = height;
            tgt[0] = 0;
            tgt[1] = 0;
            tgt[2] = height;
        } else {
            // figure-8 (lemniscate of Gerono) with a slow vertical bob; the
            // camera looks at a target on a 1.5x wider circle, so the whole
            // room is swept once per lap
            pos[0] = radius * std::sin(t);
            pos[1] = radius * std::sin(t) * std::cos(t);
            pos[2] = height + 0.1 * radius * std::sin(3 * t);
            tgt[0] = 1.5 * radius * std::cos(t);
            tgt[1] = 1.5 * radius * std::sin(t);
            tgt[2] = height - 0.2 * radius;
        }
        look_at(pos, tgt, poses + 16 * (size_t)i);
    }
    return n;
}

int vmap_synth_render(const vmap_scene* s, const double* pose, int w, int h, double fx, double fy, double cx,
                      double cy, uint64_t frame_seed, int noisy, double dropout, uint16_t* depth_mm,
                      uint8_t* rgb, float* depth_true)
{
    if (!s || !pose || w <= 0 || h <= 0) return -1;
    const double lo[3] = {-s->desc.size[0] * 0.5, -s->desc.size[1] * 0.5, 0.0};
    const double hi[3] = {s->desc.size[0] * 0.5, s->desc.size[1] * 0.5, s->desc.size[2]};
    const double o[3] = {pose[3], pose[7], pose[11]};
    const int ns = s->desc.n_spheres;
#pragma omp parallel for schedule(static)
    for (int v = 0; v < h; ++v) {
        for (int u = 0; u < w; ++u) {
            const size_t idx = (size_t)v * w + u;
            const double dc[3] = {(u - cx) / fx, (v - cy) / fy, 1.0};
            double dw[3];
            for (int i = 0; i < 3; ++i) dw[i] = pose[4 * i] * dc[0] + pose[4 * i + 1] * dc[1] + pose[4 * i + 2] * dc[2];
            // exit of the room box (camera inside): nearest positive plane hit
            double t = 1e30;
            int obj = -1;
            for (int i = 0; i < 3; ++i) {
                if (dw[i] > 1e-12) {
                    const double ti = (hi[i] - o[i]) / dw[i];
                    if (ti < t) t = ti, obj = 2 * i + 1;
                } else if (dw[i] < -1e-12) {
                    const double ti = (lo[i] - o[i]) / dw[i];
                    if (ti < t) t = ti, obj = 2 * i;
                }
            }
            for (int k = 0; k < ns; ++k) {
                const double* sp = s->sphere[k];
                const double oc[3] = {o[0] - sp[0], o[1] - sp[1], o[2] - sp[2]};
                const double a = dw[0] * dw[0] + dw[1] * dw[1] + dw[2] * dw[2];
                const double b = oc[0] * dw[0] + oc[1] * dw[1] + oc[2] * dw[2];
                const double c = oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2] - sp[3] * sp[3];
                const double disc = b * b - a * c;
                if (disc < 0) continue;
                const double sq = std::sqrt(disc);
                double tk = (-b - sq) / a;
                if (tk <= 1e-9) tk = (-b + sq) / a;
                if (tk > 1e-9 && tk < t) t = tk, obj = 6 + k;
            }
            // dc has unit z, so the ray parameter is the camera-frame depth
            double z = (obj >= 0 && t < 1e29) ? t : 0.0;
            if (depth_true) depth_true[idx] = (float)z;
            const uint64_t hsh = mix64(mix64(s->desc.seed ^ (frame_seed * 0xD6E8FEB86659FD93ull)) ^ (uint64_t)idx);
            double zn = z;
            if (noisy && z > 0) {
                const double u1 = u01(mix64(hsh ^ 1)), u2 = u01(mix64(hsh ^ 2));
                const double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
                const double sigma = 0.0012 + 0.0019 * (z - 0.4) * (z - 0.4);
                zn = z + g * sigma;
            }
            if (dropout > 0 && u01(mix64(hsh ^ 3)) < dropout) zn = 0.0;
            long mm = std::lround(zn * 1000.0);
            if (mm < 0) mm = 0;
            if (mm > 65535) mm = 65535;
            if (depth_mm) depth_mm[idx] = (uint16_t)mm;
            if (rgb) {
                for (int c = 0; c < 3; ++c) rgb[3 * idx + c] = obj >= 0 ? s->colour[obj][c] : 0;
            }
        }
    }
    return 0;
}

}  // extern "C"

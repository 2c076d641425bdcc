// pf_common.cuh -- device math shared by the Power Foam render kernels.
//
// Every expression is written in the order the reference writes it and the
// library is compiled with -fmad=false, -prec-div=true, -prec-sqrt=true: the
// kernels evaluate the same IEEE float32 operations as a literal reading of
// the reference's Warp source (powerfoam/camera.py, rendering_math.py,
// texture.py, rasterize.py, raytrace.py).  Small spheres seen from afar put
// the ray/sphere discriminant in heavy cancellation, so any change of rounding
// (an FMA, a reciprocal instead of a divide) moves composited colours by
// ~1e-3; keeping the operation sequence is what makes results reproducible.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include "../../include/pfoam.h"

#define PF_HD __host__ __device__ __forceinline__
#define PF_D __device__ __forceinline__

namespace pf {

struct v3 {
    float x, y, z;
};

PF_HD v3 mk(float x, float y, float z) { return v3{x, y, z}; }
PF_HD v3 operator+(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
PF_HD v3 operator-(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
PF_HD v3 operator-(v3 a) { return mk(-a.x, -a.y, -a.z); }
PF_HD v3 operator*(float s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
PF_HD v3 operator/(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
PF_HD float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PF_HD v3 cross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
PF_HD float length(v3 a) { return sqrtf(dot(a, a)); }
PF_HD v3 normalize(v3 a) {
    float l = length(a);
    if (l > 0.0f) return a / l;
    return mk(0.f, 0.f, 0.f);
}
// Warp's min/max: ternary forms (NaN in the first operand yields the second).
PF_HD float fmin_t(float a, float b) { return a < b ? a : b; }
PF_HD float fmax_t(float a, float b) { return a > b ? a : b; }
PF_HD int imin(int a, int b) { return a < b ? a : b; }
PF_HD int imax(int a, int b) { return a > b ? a : b; }

// float -> int32 as cvt.rzi.s32.f32: truncation, saturation, NaN -> 0.
PF_D int sat_f2i(float x) { return __float2int_rz(x); }

struct Cam {
    v3 eye, right, up;
    int W, H;
};

PF_HD Cam load_cam(const pf_camera& c) {
    Cam k;
    k.eye = mk(c.eye[0], c.eye[1], c.eye[2]);
    k.right = mk(c.right[0], c.right[1], c.right[2]);
    k.up = mk(c.up[0], c.up[1], c.up[2]);
    k.W = c.width;
    k.H = c.height;
    return k;
}

// camera.py:19-24 get_ray_dir (+ normalisation at every call site)
PF_D v3 ray_dir(const Cam& c, int pix_i, int pix_j) {
    float i = (float)pix_i, j = (float)pix_j;
    v3 forward = normalize(cross(c.up, c.right));
    float x = 2.0f * j / ((float)c.W - 1.0f) - 1.0f;
    float y = 1.0f - 2.0f * i / ((float)c.H - 1.0f);
    v3 d = (x * c.right + y * c.up) + forward;
    return d / length(d);
}

// rendering_math.py:4-23
PF_D bool ray_sphere(v3 eye, v3 dir, v3 c, float r, float& tn, float& tf) {
    v3 oc = eye - c;
    float qb = 2.0f * dot(oc, dir);
    float qc = dot(oc, oc) - r * r;
    float disc = qb * qb - 4.0f * qc;
    if (disc < 0.0f) {
        tn = 0.f;
        tf = 0.f;
        return false;
    }
    float s = sqrtf(disc);
    float t_far = (-qb + s) / 2.0f;
    float t_near = (-qb - s) / 2.0f;
    if (t_near < 0.0f && t_far < 0.0f) {
        tn = 0.f;
        tf = 0.f;
        return false;
    }
    tn = t_near < 0.0f ? 0.0f : t_near;
    tf = t_far;
    return true;
}

// rendering_math.py:26-59
PF_D void ray_sphere_bwd(v3 eye, v3 dir, v3 c, float r, v3& dn_dc, v3& df_dc, float& dn_dr, float& df_dr) {
    v3 oc = eye - c;
    float qa = dot(dir, dir);
    float qb = 2.0f * dot(oc, dir);
    float qc = dot(oc, oc) - r * r;
    float disc = qb * qb - 4.0f * qa * qc;
    dn_dc = mk(0.f, 0.f, 0.f);
    df_dc = mk(0.f, 0.f, 0.f);
    dn_dr = 0.f;
    df_dr = 0.f;
    if (disc < 0.0f) return;
    float s = sqrtf(disc);
    float t_far = (-qb + s) / (2.0f * qa);
    float t_near = (-qb - s) / (2.0f * qa);
    if (t_near < 0.0f && t_far < 0.0f) return;
    v3 g = ((2.0f * qa) * oc - qb * dir) / (qa * s);
    if (t_near < 0.0f) {
        df_dc = dir / qa + g;
        df_dr = 2.0f * r / s;
    } else {
        dn_dc = dir / qa - g;
        dn_dr = -2.0f * r / s;
        df_dc = dir / qa + g;
        df_dr = 2.0f * r / s;
    }
}

// A power face of cell i against neighbour j (rendering_math.py:62-82 with
// adj_center = center + (c_j - c_i as stored)): n = adj_center - center and
// num = face_offset - dot(eye, n) do not depend on the ray direction.
struct Face {
    v3 n;
    float num;
};

PF_D Face make_face(v3 eye, v3 center, float cc, float rr, v3 adj_center, float adj_radius) {
    Face f;
    f.n = adj_center - center;
    float face_offset = 0.5f * (dot(adj_center, adj_center) - cc + rr - adj_radius * adj_radius);
    f.num = face_offset - dot(eye, f.n);
    return f;
}

// rendering_math.py:85-98: precomputed (diff, pm_diff) encoding
PF_D Face make_face_pm(v3 eye, v3 diff, float pm_diff) {
    Face f;
    f.n = diff;
    f.num = pm_diff - dot(eye, diff);
    return f;
}

// rendering_math.py:101-125
PF_D void ray_pface_bwd(v3 eye, v3 dir, v3 center, float radius, v3 adj_center, float adj_radius, v3& dc,
                        float& dr, v3& dac, float& dar) {
    v3 face_n = adj_center - center;
    float face_offset = 0.5f * (dot(adj_center, adj_center) - dot(center, center) + radius * radius -
                                adj_radius * adj_radius);
    float num = face_offset - dot(eye, face_n);
    float dp = dot(dir, face_n);
    v3 q = ((num * dir) / dp) / dp;
    dc = (-center + eye) / dp + q;
    dac = (adj_center - eye) / dp - q;
    dr = radius / dp;
    dar = -adj_radius / dp;
}

// rendering_math.py:128-135
PF_D float ray_plane(v3 eye, v3 dir, v3 p, v3 n, float h, float& dp) {
    dp = dot(n, dir);
    return (dot(p - eye, n) + h) / dp;
}

// rendering_math.py:138-147
PF_D void ray_plane_bwd(v3 eye, v3 dir, v3 p, v3 n, float h, v3& dtdp, v3& dtdn, float& dtdh) {
    float dp = dot(n, dir);
    dtdp = n / (dp + 1e-6f);
    dtdh = 1.0f / (dp + 1e-6f);
    dtdn = (p - eye) / (dp + 1e-6f) - ((dot(p - eye, n) + h) * dir) / (dp * dp + 1e-6f);
}

constexpr float kTemp = 10.0f;  // texture.py:6
constexpr int kMaxSites = 8;    // texture.py:7
constexpr int kNoCell = 0x7FFFFFFF;

// Texel data of one primitive, as the kernels stage it.
struct Texels {
    v3 site[kMaxSites];
    v3 rgb[kMaxSites];
    float h[kMaxSites];
};

struct PlaneRes {
    float _t_surf, _dp, height, _wsum, t_surf, dp, wsum;
    v3 rgb;
};

// texture.py:10-72 plane_intersection_fwd (hit == true path).  LOCAL selects
// the rasterize.py:62-137 variant, which multiplies by a precomputed 1/r^2.
template <bool LOCAL>
PF_D PlaneRes plane_fwd(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const Texels& tx, int S) {
    PlaneRes r;
    float _dp;
    float _t_surf = ray_plane(o, d, po, pn, 0.0f, _dp);
    float _tq = _dp >= 0.0f ? t_near : fmax_t(t_near, _t_surf);
    v3 _pt = o + _tq * d;
    float rr = radius * radius;
    float inv_r2 = 1.0f / rr;
    float hsum = 0.f, _wsum = 0.f;
#pragma unroll
    for (int i = 0; i < kMaxSites; i++) {
        if (i < S) {
            v3 df = _pt - tx.site[i];
            float dist_sq = LOCAL ? dot(df, df) * inv_r2 : dot(df, df) / rr;
            float w = expf(-kTemp * dist_sq);
            hsum += w * tx.h[i];
            _wsum += w;
        }
    }
    _wsum = fmax_t(_wsum, 1e-20f);
    float height = hsum / _wsum;
    float dp;
    float t_surf = ray_plane(o, d, po, pn, height, dp);
    float tq = dp >= 0.0f ? t_near : fmax_t(t_near, t_surf);
    v3 pt = o + tq * d;
    v3 rgb_sum = mk(0.f, 0.f, 0.f);
    float wsum = 0.f;
#pragma unroll
    for (int i = 0; i < kMaxSites; i++) {
        if (i < S) {
            v3 df = pt - tx.site[i];
            float dist_sq = LOCAL ? dot(df, df) * inv_r2 : dot(df, df) / rr;
            float w = expf(-kTemp * dist_sq);
            rgb_sum = rgb_sum + w * tx.rgb[i];
            wsum += w;
        }
    }
    wsum = fmax_t(wsum, 1e-20f);
    r._t_surf = _t_surf;
    r._dp = _dp;
    r.height = height;
    r._wsum = _wsum;
    r.t_surf = t_surf;
    r.dp = dp;
    r.rgb = rgb_sum / wsum;
    r.wsum = wsum;
    return r;
}

// ---------------------------------------------------------------------------
// warp helpers
PF_D unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

PF_D float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

PF_D float h2f(uint16_t h) { return __half2float(__ushort_as_half(h)); }

}  // namespace pf

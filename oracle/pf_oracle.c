/*
 * pf_oracle.c -- CPU restatement of the Power Foam rendering hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (powerfoam_b200/) links,
 * loads or calls this file; it is the checker that the CUDA kernels are
 * compared against, and the timed CPU baseline of bench.py.
 *
 * Parity status: pinned against golden vectors produced by executing the
 * reference's own Warp kernel source (powerfoam/rasterize.py, raytrace.py,
 * texture.py, rendering_math.py, camera.py) under a numpy restatement of the
 * Warp 1.10 runtime (tests/golden/warp_shim.py).  The reference cannot run
 * on a GPU here (warp-lang is not installable offline), so the Warp runtime
 * semantics themselves (float32 arithmetic without contraction, C integer
 * division, saturating float->int conversion, bit-cast in wp.cast, RNE
 * float16) are restated, not executed.
 *
 * Arithmetic convention: every expression is evaluated literally in the order
 * the reference writes it, in IEEE single precision (or double for the _f64
 * build used by finite-difference checks), with no FMA contraction
 * (-ffp-contract=off).  min/max are the ternary forms a<b?a:b / a>b?a:b.
 *
 * Built twice by oracle/Makefile: once with real=float (symbols *_f32) and
 * once with real=double (symbols *_f64).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef PF_F64
typedef double real;
#define r_sqrt sqrt
#define r_exp exp
#define r_log log
#define r_floor floor
#define r_ceil ceil
#define r_fabs fabs
#define FN(n) n##_f64
#else
typedef float real;
#define r_sqrt sqrtf
#define r_exp expf
#define r_log logf
#define r_floor floorf
#define r_ceil ceilf
#define r_fabs fabsf
#define FN(n) n##_f32
#endif

#define K(x) ((real)(x)) /* a Warp float literal: Python double rounded to float32 */

/* image-space outputs are float32 in the f32 build and float64 in the f64
 * build (finite-difference checks need the extra digits) */
typedef real out_t;

/* ------------------------------------------------------------------------ */
/* status codes (shared meaning with include/pfoam.h)                        */
#define ORC_OK 0
#define ORC_ERR_OVERFLOW 1
#define ORC_ERR_STEP_CAP 2
#define ORC_ERR_ARGS 3

/* ------------------------------------------------------------------------ */
/* vec3 helpers: Warp vec_t semantics (per-component ops, dot summed in      */
/* index order, normalize = a/length(a) if length > 0).                      */
typedef struct { real x, y, z; } v3;

static inline v3 mk(real x, real y, real z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline v3 smul(real s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline v3 vdivs(v3 a, real s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline real dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline real length(v3 a) { return r_sqrt(dot(a, a)); }
static inline v3 normalize(v3 a) {
    real l = length(a);
    if (l > K(0.0)) return vdivs(a, l);
    return mk(0, 0, 0);
}
static inline real rmin(real a, real b) { return a < b ? a : b; }
static inline real rmax(real a, real b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline v3 ld3(const float *p) { return mk((real)p[0], (real)p[1], (real)p[2]); }

/* float -> int32 as the GPU converts it (cvt.rzi.s32.f32): truncate toward
 * zero, saturate to the int32 range, NaN -> 0. */
static inline int sat_f2i(real x) {
    if (x != x) return 0;
    if (x >= (real)2147483647.0) return INT_MAX;
    if (x <= (real)-2147483648.0) return INT_MIN;
    return (int)x;
}

/* IEEE binary16 round-to-nearest-even, as __float2half_rn / wp.float16. */
uint16_t FN(orc_f2h)(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xffu;
    uint32_t man = x & 0x7fffffu;
    if (exp == 0xffu) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u | (man >> 13) : 0));
    int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000u;
        int shift = 14 - e;
        uint32_t h = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (h & 1u))) h++;
        return (uint16_t)(sign | h);
    }
    uint32_t h = ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return (uint16_t)(sign | h);
}

float FN(orc_h2f)(uint16_t h) {
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t x;
    if (exp == 0) {
        if (man == 0) {
            x = sign;
        } else {
            int e = -1;
            do { man <<= 1; e++; } while (!(man & 0x400u));
            man &= 0x3ffu;
            x = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 31) {
        x = sign | 0x7f800000u | (man << 13);
    } else {
        x = sign | ((exp + 127 - 15) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &x, 4);
    return f;
}

/* ------------------------------------------------------------------------ */
/* camera (powerfoam/camera.py:8-24)                                         */
typedef struct {
    float eye[3], right[3], up[3];
    int32_t width, height;
} orc_camera;

typedef struct { v3 eye, right, up; int W, H; } cam_t;

static cam_t cam_load(const orc_camera *c) {
    cam_t k;
    k.eye = ld3(c->eye); k.right = ld3(c->right); k.up = ld3(c->up);
    k.W = c->width; k.H = c->height;
    return k;
}

/* camera.py:19-24 get_ray_dir */
static v3 get_ray_dir(const cam_t *c, real i, real j) {
    v3 forward = normalize(cross(c->up, c->right));
    real x = K(2.0) * j / ((real)c->W - K(1.0)) - K(1.0);
    real y = K(1.0) - K(2.0) * i / ((real)c->H - K(1.0));
    return vadd(vadd(smul(x, c->right), smul(y, c->up)), forward);
}

/* camera.py:79-128 proj_sphere_to_obb */
static void proj_sphere_to_obb(const cam_t *cam, v3 center, real radius, real out[6]) {
    v3 C = vsub(center, cam->eye);
    real C2 = dot(C, C);
    real R = radius;
    real R2 = R * R;
    v3 X = cam->right, Y = cam->up;
    v3 Z = normalize(cross(Y, X));
    real cx = dot(C, X), cy = dot(C, Y), cz = dot(C, Z);
    /* x ** 2.0 is the correctly rounded square */
    real a = cx * cx - (C2 - R2) * dot(X, X);
    real b = cy * cy - (C2 - R2) * dot(Y, Y);
    real f = cz * cz - (C2 - R2) * dot(Z, Z);
    real c = K(2.0) * cx * cy;
    real d = K(2.0) * cx * cz;
    real e = K(2.0) * cy * cz;
    real denom = K(4.0) * a * b - c * c;
    if (r_fabs(denom) < K(1e-8)) {
        out[0] = 0; out[1] = 0; out[2] = 0; out[3] = 0; out[4] = K(1.0); out[5] = 0;
        return;
    }
    real uc = (c * e - K(2.0) * b * d) / denom;
    real vc = (c * d - K(2.0) * a * e) / denom;
    real F0 = a * uc * uc + b * vc * vc + c * uc * vc + d * uc + e * vc + f;
    real term_sqrt = r_sqrt((a - b) * (a - b) + c * c);
    real l1 = (a + b + term_sqrt) / K(2.0);
    real l2 = (a + b - term_sqrt) / K(2.0);
    real r1 = r_sqrt(-F0 / l1);
    real r2 = r_sqrt(-F0 / l2);
    real vx = K(0.5) * c;
    real vy = l1 - a;
    real norm = r_sqrt(vx * vx + vy * vy);
    if (norm < K(1e-6)) {
        vx = K(1.0); vy = K(0.0);
    } else {
        vx = vx / norm; vy = vy / norm;
    }
    out[0] = uc; out[1] = vc; out[2] = r1; out[3] = r2; out[4] = vx; out[5] = vy;
}

/* camera.py:131-178 verify_tile_obb_intersection */
static int verify_tile_obb(int tile_i, int tile_j, const cam_t *cam, int TW, const real o[6]) {
    real uc = o[0], vc = o[1], r1 = o[2], r2 = o[3], vx = o[4], vy = o[5];
    real u_min = K(2.0) * (real)(tile_j * TW) / (real)(cam->W - 1) - K(1.0);
    real u_max = K(2.0) * (real)((tile_j + 1) * TW) / (real)(cam->W - 1) - K(1.0);
    real v_max = K(1.0) - K(2.0) * (real)(tile_i * TW) / (real)(cam->H - 1);
    real v_min = K(1.0) - K(2.0) * (real)((tile_i + 1) * TW) / (real)(cam->H - 1);
    real u_center = (u_min + u_max) * K(0.5);
    real v_center = (v_min + v_max) * K(0.5);
    real eu = (u_max - u_min) * K(0.5);
    real ev = (v_max - v_min) * K(0.5);
    real du = u_center - uc;
    real dv = v_center - vc;
    real p1 = du * vx + dv * vy;
    real t1 = eu * r_fabs(vx) + ev * r_fabs(vy);
    if (r_fabs(p1) > r1 + t1) return 0;
    real p2 = du * -vy + dv * vx;
    real t2 = eu * r_fabs(-vy) + ev * r_fabs(vx);
    if (r_fabs(p2) > r2 + t2) return 0;
    return 1;
}

/* rasterize.py:140-200 / 293-363: the per-primitive tile walk shared by the
 * count and write kernels.  Calls emit(tile_idx) for each tile that passes
 * the SAT test, in tile_i-major, tile_j-minor order.  Returns 0 if culled. */
typedef void (*emit_fn)(void *ctx, int tile_idx);

static int prim_tiles(const cam_t *cam, int TW, v3 center, real radius, emit_fn emit, void *ctx) {
    int tiles_h = 1 + (cam->H - 1) / TW;
    v3 v = vsub(center, cam->eye);
    v3 forward = cross(cam->up, cam->right);
    if (length(v) < K(4.0) * radius || dot(v, forward) < K(0.1)) return 0;
    real o[6];
    proj_sphere_to_obb(cam, center, radius, o);
    real uc = o[0], vc = o[1], r1 = o[2], r2 = o[3], vx = o[4], vy = o[5];
    real extent_u = r_fabs(vx * r1) + r_fabs(vy * r2);
    real extent_v = r_fabs(vy * r1) + r_fabs(vx * r2);
    real u_min = uc - extent_u, u_max = uc + extent_u;
    real v_min = vc - extent_v, v_max = vc + extent_v;
    real j_min_f = (u_min + K(1.0)) * K(0.5) * (real)(cam->W - 1);
    real j_max_f = (u_max + K(1.0)) * K(0.5) * (real)(cam->W - 1);
    real i_min_f = (K(1.0) - v_max) * K(0.5) * (real)(cam->H - 1);
    real i_max_f = (K(1.0) - v_min) * K(0.5) * (real)(cam->H - 1);
    int i_min = imax(sat_f2i(r_floor(i_min_f)), 0);
    int i_max = imin(sat_f2i(r_ceil(i_max_f)), cam->H - 1);
    int j_min = imax(sat_f2i(r_floor(j_min_f)), 0);
    int j_max = imin(sat_f2i(r_ceil(j_max_f)), cam->W - 1);
    /* Warp integer floordiv on the GPU is C division (truncation) */
    int ti0 = i_min / TW, ti1 = i_max / TW, tj0 = j_min / TW, tj1 = j_max / TW;
    for (int ti = ti0; ti <= ti1; ti++)
        for (int tj = tj0; tj <= tj1; tj++) {
            if (!verify_tile_obb(ti, tj, cam, TW, o)) continue;
            emit(ctx, ti + tj * tiles_h);
        }
    return 1;
}

static void count_emit(void *ctx, int tile) { (void)tile; (*(int64_t *)ctx)++; }

typedef struct {
    int64_t *pos;
    int64_t cap;
    int64_t *keys;
    int32_t *prims;
    int32_t prim;
    uint32_t depth_bits;
} write_ctx;

static void write_emit(void *vctx, int tile) {
    write_ctx *w = (write_ctx *)vctx;
    int64_t p = *w->pos;
    if (p < w->cap) {
        w->keys[p] = ((int64_t)tile << 32) | (int64_t)w->depth_bits;
        w->prims[p] = w->prim;
    }
    *w->pos = p + 1;
}

typedef struct { int64_t key; int64_t ord; int32_t prim; } pair_t;
static int pair_cmp(const void *a, const void *b) {
    const pair_t *x = (const pair_t *)a, *y = (const pair_t *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->ord < y->ord ? -1 : (x->ord > y->ord);
}

/*
 * Binning: rasterize.py:1681-1768 (count -> cumsum -> write -> argsort).
 * Emission is in primitive order (the reference's atomic order is
 * nondeterministic); the sort is stable, so equal keys keep ascending
 * primitive index.  Writes the sorted keys and primitive ids (up to cap),
 * per-tile offsets (T+1, int64) and the per-primitive tile counts.
 * *n_pairs receives the total; returns ORC_ERR_OVERFLOW if it exceeds cap.
 */
int FN(orc_bin)(const orc_camera *camera, const float *spheres, int64_t N, int TW,
                int64_t cap, int64_t *keys_out, int32_t *prims_out, int64_t *tile_offsets,
                int32_t *prim_counts, int64_t *n_pairs) {
    if (TW <= 0) return ORC_ERR_ARGS;
    cam_t cam = cam_load(camera);
    int tiles_h = 1 + (cam.H - 1) / TW, tiles_w = 1 + (cam.W - 1) / TW;
    int64_t T = (int64_t)tiles_h * tiles_w;
    int64_t total = 0;
    for (int64_t p = 0; p < N; p++) {
        int64_t c = 0;
        const float *s = spheres + 4 * p;
        prim_tiles(&cam, TW, ld3(s), (real)s[3], count_emit, &c);
        if (prim_counts) prim_counts[p] = (int32_t)c;
        total += c;
    }
    *n_pairs = total;
    pair_t *pairs = (pair_t *)malloc(sizeof(pair_t) * (size_t)(total > 0 ? total : 1));
    int64_t *tk = (int64_t *)malloc(sizeof(int64_t) * (size_t)(total > 0 ? total : 1));
    int32_t *tp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
    int64_t pos = 0;
    for (int64_t p = 0; p < N; p++) {
        const float *s = spheres + 4 * p;
        v3 c = ld3(s);
        real r = (real)s[3];
        v3 v = vsub(c, cam.eye);
        float pd = (float)(dot(v, v) - r * r);
        write_ctx w;
        w.pos = &pos; w.cap = total; w.keys = tk; w.prims = tp; w.prim = (int32_t)p;
        memcpy(&w.depth_bits, &pd, 4);
        prim_tiles(&cam, TW, c, r, write_emit, &w);
    }
    for (int64_t k = 0; k < total; k++) {
        pairs[k].key = tk[k]; pairs[k].ord = k; pairs[k].prim = tp[k];
    }
    qsort(pairs, (size_t)total, sizeof(pair_t), pair_cmp);
    for (int64_t t = 0; t <= T; t++) tile_offsets[t] = 0;
    for (int64_t k = 0; k < total; k++) {
        int64_t t = pairs[k].key >> 32;
        tile_offsets[t + 1]++;
        if (k < cap) { keys_out[k] = pairs[k].key; prims_out[k] = pairs[k].prim; }
    }
    for (int64_t t = 0; t < T; t++) tile_offsets[t + 1] += tile_offsets[t];
    free(pairs); free(tk); free(tp);
    return total > cap ? ORC_ERR_OVERFLOW : ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Generic-camera binning (rasterize.py:202-291, 365-569, 1518-1585): a     */
/* hierarchy of ray cones over the ray map, leaves of 2x2 pixels, each level */
/* merging 2x2 children up to one root; a primitive descends from the root  */
/* into every child cone its sphere meets (camera.py:28-44) and is emitted   */
/* into the tiles of the tile level.                                          */

#define ORC_LEAF 2
#define ORC_MAX_LEVELS 32

typedef struct {
    int n_levels, tile_level;
    int off[ORC_MAX_LEVELS], dh[ORC_MAX_LEVELS], dw[ORC_MAX_LEVELS];
    int64_t total;
} cone_dims;

static int cone_layout(int H, int W, int TW, cone_dims *cd) {
    int dh = (H + ORC_LEAF - 1) / ORC_LEAF, dw = (W + ORC_LEAF - 1) / ORC_LEAF;
    cd->n_levels = 0;
    cd->total = 0;
    for (;;) {
        if (cd->n_levels == ORC_MAX_LEVELS) return ORC_ERR_ARGS;
        cd->off[cd->n_levels] = (int)cd->total;
        cd->dh[cd->n_levels] = dh;
        cd->dw[cd->n_levels] = dw;
        cd->n_levels++;
        cd->total += (int64_t)dh * dw;
        if (dh == 1 && dw == 1) break;
        dh = (dh + 1) / 2;
        dw = (dw + 1) / 2;
    }
    cd->tile_level = 0;
    for (int sz = ORC_LEAF; sz < TW; sz *= 2) cd->tile_level++;
    return ORC_OK;
}

/* compute_leaf_cones_kernel (rasterize.py:473-515) and merge_cones_kernel
 * (:517-569); cones (total, 4): axis, cos of the half angle (2: empty). */
static void build_cones(const cam_t *cam, const float *ray_maps, const cone_dims *cd, real *cones) {
    const int lw = cd->dw[0];
    const int64_t n_leaf = (int64_t)cd->dh[0] * lw;
    for (int64_t t = 0; t < n_leaf; t++) {
        int a = (int)(t / lw), b = (int)(t % lw);
        v3 axis_sum = mk(0, 0, 0), rays[4];
        int valid = 0;
        for (int di = 0; di < ORC_LEAF; di++)
            for (int dj = 0; dj < ORC_LEAF; dj++) {
                int pi = imin(a * ORC_LEAF + di, cam->H - 1), pj = imin(b * ORC_LEAF + dj, cam->W - 1);
                v3 ray = ld3(ray_maps + 6 * ((int64_t)pi * cam->W + pj) + 3);
                real len = length(ray);
                if (len > K(1.0e-6)) {
                    v3 rn = vdivs(ray, len);
                    rays[valid++] = rn;
                    axis_sum = vadd(axis_sum, rn);
                }
            }
        real *c = cones + 4 * t;
        if (valid == 0) { c[0] = c[1] = c[2] = 0; c[3] = K(2.0); continue; }
        v3 axis = normalize(axis_sum);
        real ch = K(1.0);
        for (int i = 0; i < valid; i++) ch = rmin(ch, dot(axis, rays[i]));
        c[0] = axis.x; c[1] = axis.y; c[2] = axis.z; c[3] = ch;
    }
    for (int l = 1; l < cd->n_levels; l++) {
        const int pdw = cd->dw[l], cdh = cd->dh[l - 1], cdw = cd->dw[l - 1];
        const int64_t n = (int64_t)cd->dh[l] * pdw;
        for (int64_t t = 0; t < n; t++) {
            int a = (int)(t / pdw), b = (int)(t % pdw);
            v3 axis_sum = mk(0, 0, 0), axes[4];
            real chs[4];
            int valid = 0;
            for (int di = 0; di < 2; di++)
                for (int dj = 0; dj < 2; dj++) {
                    int ca = 2 * a + di, cb = 2 * b + dj;
                    if (ca < cdh && cb < cdw) {
                        const real *cc = cones + 4 * ((int64_t)cd->off[l - 1] + (int64_t)ca * cdw + cb);
                        if (cc[3] <= K(1.0)) {
                            axes[valid] = mk(cc[0], cc[1], cc[2]);
                            chs[valid] = cc[3];
                            axis_sum = vadd(axis_sum, axes[valid]);
                            valid++;
                        }
                    }
                }
            real *c = cones + 4 * ((int64_t)cd->off[l] + t);
            if (valid == 0) { c[0] = c[1] = c[2] = 0; c[3] = K(2.0); continue; }
            v3 axis = normalize(axis_sum);
            real ch = K(1.0);
            for (int i = 0; i < valid; i++) {
                real dv = dot(axis, axes[i]);
                real sin_angle = r_sqrt(rmax(K(1.0) - dv * dv, K(0.0)));
                real sin_child = r_sqrt(rmax(K(1.0) - chs[i] * chs[i], K(0.0)));
                real extent = dv * chs[i] - sin_angle * sin_child;
                ch = rmin(ch, extent);
            }
            c[0] = axis.x; c[1] = axis.y; c[2] = axis.z; c[3] = ch;
        }
    }
}

/* camera.py:28-44 */
static int sphere_cone(v3 center, real radius, v3 eye, v3 axis, real cos_half) {
    v3 v = vsub(center, eye);
    real dist = length(v);
    real cos_alpha = dot(v, axis) / dist;
    real sin_half = r_sqrt(K(1.0) - cos_half * cos_half);
    real sin_beta = radius / dist;
    real cos_beta = r_sqrt(K(1.0) - sin_beta * sin_beta);
    real threshold = cos_half * cos_beta - sin_half * sin_beta;
    return cos_alpha > threshold;
}

/* count / write_visible_generic_kernel traversal (rasterize.py:202-291,
 * 365-464): emits every tile-level cone the sphere reaches. */
static int prim_tiles_generic(const cam_t *cam, const cone_dims *cd, const real *cones, int TW, v3 center,
                              real radius, emit_fn emit, void *ctx) {
    int tiles_h = 1 + (cam->H - 1) / TW;
    v3 v = vsub(center, cam->eye);
    v3 forward = cross(cam->up, cam->right);
    if (length(v) < K(4.0) * radius || dot(v, forward) < K(0.1)) return 0;
    int st_l[4 * ORC_MAX_LEVELS], st_a[4 * ORC_MAX_LEVELS], st_b[4 * ORC_MAX_LEVELS];
    int n = 1;
    st_l[0] = cd->n_levels - 1; st_a[0] = 0; st_b[0] = 0;
    while (n > 0) {
        n--;
        int level = st_l[n], a = st_a[n], b = st_b[n];
        const real *c = cones + 4 * ((int64_t)cd->off[level] + (int64_t)a * cd->dw[level] + b);
        if (c[3] > K(1.0)) continue;
        if (!sphere_cone(center, radius, cam->eye, mk(c[0], c[1], c[2]), c[3])) continue;
        if (level == cd->tile_level) {
            emit(ctx, a + b * tiles_h);
            continue;
        }
        int cl = level - 1;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++) {
                int ca = 2 * a + di, cb = 2 * b + dj;
                if (ca < cd->dh[cl] && cb < cd->dw[cl]) {
                    st_l[n] = cl; st_a[n] = ca; st_b[n] = cb;
                    n++;
                }
            }
    }
    return 1;
}

/* Binning with a generic camera; as orc_bin otherwise.  cones_out (total x
 * 4, optional) receives the cone hierarchy; *n_cones its node count. */
int FN(orc_bin_generic)(const orc_camera *camera, const float *ray_maps, const float *spheres, int64_t N, int TW,
                        int64_t cap, int64_t *keys_out, int32_t *prims_out, int64_t *tile_offsets,
                        int32_t *prim_counts, int64_t *n_pairs, out_t *cones_out, int64_t *n_cones) {
    if (TW <= 0 || !ray_maps) return ORC_ERR_ARGS;
    cam_t cam = cam_load(camera);
    cone_dims cd;
    if (cone_layout(cam.H, cam.W, TW, &cd) != ORC_OK) return ORC_ERR_ARGS;
    if (n_cones) *n_cones = cd.total;
    real *cones = (real *)malloc(sizeof(real) * 4 * (size_t)cd.total);
    build_cones(&cam, ray_maps, &cd, cones);
    if (cones_out)
        for (int64_t k = 0; k < 4 * cd.total; k++) cones_out[k] = (out_t)cones[k];
    int tiles_h = 1 + (cam.H - 1) / TW, tiles_w = 1 + (cam.W - 1) / TW;
    int64_t T = (int64_t)tiles_h * tiles_w;
    int64_t total = 0;
    for (int64_t p = 0; p < N; p++) {
        int64_t c = 0;
        const float *s = spheres + 4 * p;
        prim_tiles_generic(&cam, &cd, cones, TW, ld3(s), (real)s[3], count_emit, &c);
        if (prim_counts) prim_counts[p] = (int32_t)c;
        total += c;
    }
    *n_pairs = total;
    pair_t *pairs = (pair_t *)malloc(sizeof(pair_t) * (size_t)(total > 0 ? total : 1));
    int64_t *tk = (int64_t *)malloc(sizeof(int64_t) * (size_t)(total > 0 ? total : 1));
    int32_t *tp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
    int64_t pos = 0;
    for (int64_t p = 0; p < N; p++) {
        const float *s = spheres + 4 * p;
        v3 c = ld3(s);
        real r = (real)s[3];
        v3 v = vsub(c, cam.eye);
        float pd = (float)(dot(v, v) - r * r);
        write_ctx w;
        w.pos = &pos; w.cap = total; w.keys = tk; w.prims = tp; w.prim = (int32_t)p;
        memcpy(&w.depth_bits, &pd, 4);
        prim_tiles_generic(&cam, &cd, cones, TW, c, r, write_emit, &w);
    }
    for (int64_t k = 0; k < total; k++) {
        pairs[k].key = tk[k]; pairs[k].ord = k; pairs[k].prim = tp[k];
    }
    qsort(pairs, (size_t)total, sizeof(pair_t), pair_cmp);
    for (int64_t t = 0; t <= T; t++) tile_offsets[t] = 0;
    for (int64_t k = 0; k < total; k++) {
        int64_t t = pairs[k].key >> 32;
        tile_offsets[t + 1]++;
        if (k < cap) { keys_out[k] = pairs[k].key; prims_out[k] = pairs[k].prim; }
    }
    for (int64_t t = 0; t < T; t++) tile_offsets[t + 1] += tile_offsets[t];
    free(pairs); free(tk); free(tp); free(cones);
    return total > cap ? ORC_ERR_OVERFLOW : ORC_OK;
}

/* rasterize.py:580-606 prefetch_adjacency_kernel: (half(c_j - c_i), half(r_j)) */
void FN(orc_prefetch_adjacency)(const float *spheres, const int32_t *adj, const int32_t *adj_off,
                                int64_t N, uint16_t *adj_diff) {
    for (int64_t p = 0; p < N; p++) {
        const float *s = spheres + 4 * p;
        for (int32_t e = adj_off[p]; e < adj_off[p + 1]; e++) {
            const float *t = spheres + 4 * (int64_t)adj[e];
            adj_diff[4 * (int64_t)e + 0] = FN(orc_f2h)(t[0] - s[0]);
            adj_diff[4 * (int64_t)e + 1] = FN(orc_f2h)(t[1] - s[1]);
            adj_diff[4 * (int64_t)e + 2] = FN(orc_f2h)(t[2] - s[2]);
            adj_diff[4 * (int64_t)e + 3] = FN(orc_f2h)(t[3]);
        }
    }
}

/* benchmark.py:297-302: (half(c_j - c_i), half(pm_j - pm_i)), pm = (|c|^2 - r^2)/2
 * computed as 0.5 * (norm(c) ** 2 - r ** 2) in float32. */
void FN(orc_power_adjacency_diff)(const float *points, const float *radii, const int32_t *adj,
                                  const int32_t *adj_off, int64_t N, uint16_t *adj_diff) {
    for (int64_t p = 0; p < N; p++) {
        const float *c = points + 3 * p;
        float n = sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        float pm_i = 0.5f * (n * n - radii[p] * radii[p]);
        for (int32_t e = adj_off[p]; e < adj_off[p + 1]; e++) {
            int64_t q = adj[e];
            const float *d = points + 3 * q;
            float m = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            float pm_j = 0.5f * (m * m - radii[q] * radii[q]);
            adj_diff[4 * (int64_t)e + 0] = FN(orc_f2h)(d[0] - c[0]);
            adj_diff[4 * (int64_t)e + 1] = FN(orc_f2h)(d[1] - c[1]);
            adj_diff[4 * (int64_t)e + 2] = FN(orc_f2h)(d[2] - c[2]);
            adj_diff[4 * (int64_t)e + 3] = FN(orc_f2h)(pm_j - pm_i);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* rendering_math.py                                                         */

/* rendering_math.py:4-23 */
static int ray_sphere(v3 eye, v3 dir, v3 c, real r, real *tn, real *tf) {
    v3 oc = vsub(eye, c);
    real qb = K(2.0) * dot(oc, dir);
    real qc = dot(oc, oc) - r * r;
    real disc = qb * qb - K(4.0) * qc;
    if (disc < 0) { *tn = 0; *tf = 0; return 0; }
    real t_far = (-qb + r_sqrt(disc)) / K(2.0);
    real t_near = (-qb - r_sqrt(disc)) / K(2.0);
    if (t_near < K(0.0) && t_far < K(0.0)) { *tn = 0; *tf = 0; return 0; }
    if (t_near < K(0.0)) { *tn = 0; *tf = t_far; return 1; }
    *tn = t_near; *tf = t_far;
    return 1;
}

/* rendering_math.py:26-59 */
static void ray_sphere_bwd(v3 eye, v3 dir, v3 c, real r, v3 *dn_dc, v3 *df_dc, real *dn_dr, real *df_dr) {
    v3 oc = vsub(eye, c);
    real qa = dot(dir, dir);
    real qb = K(2.0) * dot(oc, dir);
    real qc = dot(oc, oc) - r * r;
    real disc = qb * qb - K(4.0) * qa * qc;
    *dn_dc = mk(0, 0, 0); *df_dc = mk(0, 0, 0); *dn_dr = 0; *df_dr = 0;
    if (disc < 0) return;
    real t_far = (-qb + r_sqrt(disc)) / (K(2.0) * qa);
    real t_near = (-qb - r_sqrt(disc)) / (K(2.0) * qa);
    if (t_near < K(0.0) && t_far < K(0.0)) return;
    v3 g = vdivs(vsub(smul(K(2.0) * qa, oc), smul(qb, dir)), qa * r_sqrt(disc));
    if (t_near < K(0.0)) {
        *df_dc = vadd(vdivs(dir, qa), g);
        *df_dr = K(2.0) * r / r_sqrt(disc);
    } else {
        *dn_dc = vsub(vdivs(dir, qa), g);
        *dn_dr = K(-2.0) * r / r_sqrt(disc);
        *df_dc = vadd(vdivs(dir, qa), g);
        *df_dr = K(2.0) * r / r_sqrt(disc);
    }
}

/* rendering_math.py:62-82 */
static real ray_pface(v3 eye, v3 dir, v3 center, real radius, v3 adj_center, real adj_radius, real *dp_out) {
    v3 face_n = vsub(adj_center, center);
    real face_offset = K(0.5) * (dot(adj_center, adj_center) - dot(center, center) + radius * radius -
                                 adj_radius * adj_radius);
    real dp = dot(dir, face_n);
    *dp_out = dp;
    return (face_offset - dot(eye, face_n)) / dp;
}

/* rendering_math.py:85-98 */
static real ray_pface_diff(v3 eye, v3 dir, v3 diff, real pm_diff, real *dp_out) {
    real dp = dot(dir, diff);
    *dp_out = dp;
    return (pm_diff - dot(eye, diff)) / dp;
}

/* rendering_math.py:101-125 */
static void ray_pface_bwd(v3 eye, v3 dir, v3 center, real radius, v3 adj_center, real adj_radius,
                          v3 *dc, real *dr, v3 *dac, real *dar) {
    v3 face_n = vsub(adj_center, center);
    real face_offset = K(0.5) * (dot(adj_center, adj_center) - dot(center, center) + radius * radius -
                                 adj_radius * adj_radius);
    real num = face_offset - dot(eye, face_n);
    real dp = dot(dir, face_n);
    v3 q = vdivs(vdivs(smul(num, dir), dp), dp);
    *dc = vadd(vdivs(vadd(vneg(center), eye), dp), q);
    *dac = vsub(vdivs(vsub(adj_center, eye), dp), q);
    *dr = radius / dp;
    *dar = -adj_radius / dp;
}

/* rendering_math.py:128-135 */
static real ray_plane(v3 eye, v3 dir, v3 p, v3 n, real h, real *dp_out) {
    real dp = dot(n, dir);
    *dp_out = dp;
    return (dot(vsub(p, eye), n) + h) / dp;
}

/* rendering_math.py:138-147 */
static void ray_plane_bwd(v3 eye, v3 dir, v3 p, v3 n, real h, v3 *dtdp, v3 *dtdn, real *dtdh) {
    real dp = dot(n, dir);
    *dtdp = vdivs(n, dp + K(1e-6));
    *dtdh = K(1.0) / (dp + K(1e-6));
    *dtdn = vsub(vdivs(vsub(p, eye), dp + K(1e-6)),
                 vdivs(smul(dot(vsub(p, eye), n) + h, dir), dp * dp + K(1e-6)));
}

/* ------------------------------------------------------------------------ */
/* texture.py                                                                */
#define TEMP K(10.0)

typedef struct {
    real _t_surf, _dp, height, _wsum, t_surf, dp, wsum;
    v3 rgb;
} plane_res;

/* texture.py:10-72 plane_intersection_fwd; sites (S,3), values (S,4) rgb+h */
static plane_res plane_fwd(v3 o, v3 d, real t_near, v3 po, v3 pn, real radius, int hit,
                           const float *sites, const float *values, int S) {
    plane_res r;
    memset(&r, 0, sizeof(r));
    if (!hit) return r;
    real _dp;
    real _t_surf = ray_plane(o, d, po, pn, K(0.0), &_dp);
    real _tq = _dp >= K(0.0) ? t_near : rmax(t_near, _t_surf);
    v3 _pt = vadd(o, smul(_tq, d));
    real hsum = 0, _wsum = 0;
    for (int i = 0; i < S; i++) {
        v3 site = ld3(sites + 3 * i);
        v3 df = vsub(_pt, site);
        real dist_sq = dot(df, df) / (radius * radius);
        real w = r_exp(-TEMP * dist_sq);
        hsum += w * (real)values[4 * i + 3];
        _wsum += w;
    }
    _wsum = rmax(_wsum, K(1e-20));
    real height = hsum / _wsum;
    real dp;
    real t_surf = ray_plane(o, d, po, pn, height, &dp);
    real tq = dp >= K(0.0) ? t_near : rmax(t_near, t_surf);
    v3 pt = vadd(o, smul(tq, d));
    v3 rgb_sum = mk(0, 0, 0);
    real wsum = 0;
    for (int i = 0; i < S; i++) {
        v3 site = ld3(sites + 3 * i);
        v3 df = vsub(pt, site);
        real dist_sq = dot(df, df) / (radius * radius);
        real w = r_exp(-TEMP * dist_sq);
        rgb_sum = vadd(rgb_sum, smul(w, ld3(values + 4 * i)));
        wsum += w;
    }
    wsum = rmax(wsum, K(1e-20));
    r._t_surf = _t_surf; r._dp = _dp; r.height = height; r._wsum = _wsum;
    r.t_surf = t_surf; r.dp = dp; r.rgb = vdivs(rgb_sum, wsum); r.wsum = wsum;
    return r;
}

/* rasterize.py:62-137 (== raytrace.py:42-113) plane_intersection_fwd_local:
 * sites/rgbs/heights as separate arrays (S,3),(S,3),(S); 1/r^2 precomputed. */
static plane_res plane_fwd_local(v3 o, v3 d, real t_near, v3 po, v3 pn, real radius,
                                 const float *sites, const float *rgbs, const float *heights, int S) {
    plane_res r;
    real _dp;
    real _t_surf = ray_plane(o, d, po, pn, K(0.0), &_dp);
    real _tq = _dp >= K(0.0) ? t_near : rmax(t_near, _t_surf);
    v3 _pt = vadd(o, smul(_tq, d));
    real inv_r2 = K(1.0) / (radius * radius);
    real hsum = 0, _wsum = 0;
    for (int i = 0; i < S; i++) {
        v3 df = vsub(_pt, ld3(sites + 3 * i));
        real dist_sq = dot(df, df) * inv_r2;
        real w = r_exp(-TEMP * dist_sq);
        hsum += w * (real)heights[i];
        _wsum += w;
    }
    _wsum = rmax(_wsum, K(1e-20));
    real height = hsum / _wsum;
    real dp;
    real t_surf = ray_plane(o, d, po, pn, height, &dp);
    real tq = dp >= K(0.0) ? t_near : rmax(t_near, t_surf);
    v3 pt = vadd(o, smul(tq, d));
    v3 rgb_sum = mk(0, 0, 0);
    real wsum = 0;
    for (int i = 0; i < S; i++) {
        v3 df = vsub(pt, ld3(sites + 3 * i));
        real dist_sq = dot(df, df) * inv_r2;
        real w = r_exp(-TEMP * dist_sq);
        rgb_sum = vadd(rgb_sum, smul(w, ld3(rgbs + 3 * i)));
        wsum += w;
    }
    wsum = rmax(wsum, K(1e-20));
    r._t_surf = _t_surf; r._dp = _dp; r.height = height; r._wsum = _wsum;
    r.t_surf = t_surf; r.dp = dp; r.rgb = vdivs(rgb_sum, wsum); r.wsum = wsum;
    return r;
}

#ifdef _OPENMP
#define ATOMIC_ADD(dst, v) do { real _v = (v); _Pragma("omp atomic") (dst) += (__typeof__(dst))_v; } while (0)
#else
#define ATOMIC_ADD(dst, v) ((dst) += (__typeof__(dst))(v))
#endif

/* texture.py:74-186 plane_intersection_bwd.  Gradient accumulators are the
 * primitive's rows of the texel grads (S,3), (S,3), (S). */
static void plane_bwd(v3 o, v3 d, real _t_near, v3 po, v3 pn, real radius, int hit,
                      const float *sites, const float *values, real _dp, real _t_surf, real height_in,
                      real _weight_sum, real dp, real t_surf, v3 rgb_in, real weight_sum, v3 dLdrgb_in,
                      real dLdt_surf_in, int S, float *sites_g, float *rgb_g, float *height_g,
                      v3 *dLdpo_out, v3 *dLdpn_out, real *dLd_t_near_out) {
    v3 dLdpo = mk(0, 0, 0), dLdpn = mk(0, 0, 0);
    real dLdheight_in = 0;
    *dLdpo_out = dLdpo; *dLdpn_out = dLdpn; *dLd_t_near_out = 0;
    if (!hit) return;
    real tq = dp >= K(0.0) ? _t_near : rmax(_t_near, t_surf);
    v3 pt = vadd(o, smul(tq, d));
    v3 dLdpt = mk(0, 0, 0);
    real grad_dp_in = dot(dLdrgb_in, rgb_in);
    for (int i = 0; i < S; i++) {
        v3 site = ld3(sites + 3 * i);
        v3 df = vsub(pt, site);
        real dist_sq = dot(df, df) / (radius * radius);
        real w = r_exp(-TEMP * dist_sq);
        if (w / weight_sum < K(1e-3)) continue;
        v3 dwds = vdivs(smul(K(2.0) * TEMP * w, vsub(pt, site)), radius * radius);
        v3 rgb_grad = vdivs(smul(w, dLdrgb_in), weight_sum);
        ATOMIC_ADD(rgb_g[3 * i + 0], rgb_grad.x);
        ATOMIC_ADD(rgb_g[3 * i + 1], rgb_grad.y);
        ATOMIC_ADD(rgb_g[3 * i + 2], rgb_grad.z);
        real grad_dp = dot(dLdrgb_in, ld3(values + 4 * i));
        v3 site_grad = vdivs(smul(grad_dp - grad_dp_in, dwds), weight_sum);
        ATOMIC_ADD(sites_g[3 * i + 0], site_grad.x);
        ATOMIC_ADD(sites_g[3 * i + 1], site_grad.y);
        ATOMIC_ADD(sites_g[3 * i + 2], site_grad.z);
        dLdpt = vadd(dLdpt, vneg(site_grad));
    }
    real dLdt_query = dot(dLdpt, d);
    real dLd_t_near = (dp >= K(0.0) || _t_near >= t_surf) ? dLdt_query : K(0.0);
    real dLdt_surf = (dp < K(0.0) && _t_near < t_surf) ? dLdt_query : K(0.0);
    dLdt_surf += dLdt_surf_in;
    if (r_fabs(dLdt_surf) > K(0.0)) {
        v3 a, b;
        real c;
        ray_plane_bwd(o, d, po, pn, height_in, &a, &b, &c);
        dLdpo = vadd(dLdpo, smul(dLdt_surf, a));
        dLdpn = vadd(dLdpn, smul(dLdt_surf, b));
        dLdheight_in += c * dLdt_surf;
    }
    real _tq = _dp >= K(0.0) ? _t_near : rmax(_t_near, _t_surf);
    v3 _pt = vadd(o, smul(_tq, d));
    v3 dLd_pt = mk(0, 0, 0);
    real _grad_dp_in = dLdheight_in * height_in;
    for (int i = 0; i < S; i++) {
        v3 site = ld3(sites + 3 * i);
        v3 df = vsub(_pt, site);
        real dist_sq = dot(df, df) / (radius * radius);
        real w = r_exp(-TEMP * dist_sq);
        if (w / weight_sum < K(1e-3)) continue;
        v3 dwds = vdivs(smul(K(2.0) * TEMP * w, vsub(_pt, site)), radius * radius);
        real height_grad = w * dLdheight_in / _weight_sum;
        ATOMIC_ADD(height_g[i], height_grad);
        real _grad_dp = dLdheight_in * (real)values[4 * i + 3];
        v3 site_grad = vdivs(smul(_grad_dp - _grad_dp_in, dwds), _weight_sum);
        ATOMIC_ADD(sites_g[3 * i + 0], site_grad.x);
        ATOMIC_ADD(sites_g[3 * i + 1], site_grad.y);
        ATOMIC_ADD(sites_g[3 * i + 2], site_grad.z);
        dLd_pt = vadd(dLd_pt, vneg(site_grad));
    }
    real dLd_t_query = dot(dLd_pt, d);
    dLd_t_near += (dp >= K(0.0) || _t_near >= _t_surf) ? dLd_t_query : K(0.0);
    real dLd_t_surf = (dp < K(0.0) && _t_near < _t_surf) ? dLd_t_query : K(0.0);
    if (r_fabs(dLd_t_surf) > K(0.0)) {
        v3 a, b;
        real c;
        ray_plane_bwd(o, d, po, pn, K(0.0), &a, &b, &c);
        dLdpo = vadd(dLdpo, smul(dLd_t_surf, a));
        dLdpn = vadd(dLdpn, smul(dLd_t_surf, b));
    }
    *dLdpo_out = dLdpo; *dLdpn_out = dLdpn; *dLd_t_near_out = dLd_t_near;
}

/* Neighbour e of a primitive as the face clip sees it: centre + half(c_j - c_i)
 * and half(r_j) from the prefetched encoding (rasterize.py:1054-1058); with
 * adj_diff == NULL the exact neighbour sphere (used by finite-difference
 * checks, where the float16 quantisation would make the image piecewise
 * constant in the primitive positions). */
static void nbr_sphere(const float *spheres, const int32_t *adj, const uint16_t *adj_diff, int32_t e, v3 center,
                       v3 *ac, real *ar) {
    if (adj_diff) {
        const uint16_t *h = adj_diff + 4 * (int64_t)e;
        *ac = vadd(center, mk((real)FN(orc_h2f)(h[0]), (real)FN(orc_h2f)(h[1]), (real)FN(orc_h2f)(h[2])));
        *ar = (real)FN(orc_h2f)(h[3]);
    } else {
        const float *t = spheres + 4 * (int64_t)adj[e];
        *ac = ld3(t);
        *ar = (real)t[3];
    }
}

/* ------------------------------------------------------------------------ */
/* Rasterizer forward (rasterize.py:892-1146 forward_kernel, host side      */
/* rasterize.py:1587-1856).  One tile = one Warp block of TW*TW threads; the */
/* block-wide tile_max / tile_sum are emulated by running the lanes of a     */
/* tile in lockstep.  Outputs must be pre-initialised by the caller exactly  */
/* as the reference does (zeros; quantile depths -1).                        */

typedef struct {
    v3 o, d;
    int oob, pi, pj;
    real log_t, nd, err;
    v3 rgb, normal;
    int qi;
    real q;
    v3 gt;
    int hit;
    real tn, tf;
} fwd_lane;

/* The ray of lane l: the pinhole ray from the eye, or with ray_maps (H,W,6)
 * (the generic camera, rasterize.py:940-954) the pixel's own origin and its
 * direction divided by its length. */
static void lane_setup(const cam_t *cam, const float *ray_maps, int TW, int tiles_h, int64_t tile, int l, v3 *o,
                       v3 *d, int *oob, int *pi, int *pj) {
    int ti = (int)(tile % tiles_h), tj = (int)(tile / tiles_h);
    int i_in = l % TW, j_in = l / TW;
    int pix_i = ti * TW + i_in, pix_j = tj * TW + j_in;
    *oob = pix_i >= cam->H || pix_j >= cam->W;
    pix_i = imin(pix_i, cam->H - 1);
    pix_j = imin(pix_j, cam->W - 1);
    if (ray_maps) {
        const float *m = ray_maps + 6 * ((int64_t)pix_i * cam->W + pix_j);
        *o = ld3(m);
        v3 rd = ld3(m + 3);
        *d = vdivs(rd, length(rd));
    } else {
        v3 rd = get_ray_dir(cam, (real)pix_i, (real)pix_j);
        *d = vdivs(rd, length(rd));
        *o = cam->eye;
    }
    *pi = pix_i; *pj = pix_j;
}

static int FN(raster_forward)(const orc_camera *camera, const float *ray_maps, int TW, int64_t N,
                              const float *spheres, const float *nsigmas, const float *sites, const float *rgbh,
                              int S, const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                              const int64_t *tile_offsets, const int32_t *tile_prims, const float *depth_q, int Q,
                              const float *ray_gt, float thr, int return_point_err, out_t *color, out_t *log_t_out,
                              out_t *nd_out, out_t *normal_out, out_t *qdepth_out, out_t *err_out, out_t *contrib,
                              out_t *point_err, int32_t *early_stop) {
    (void)N; (void)adj;
    cam_t cam = cam_load(camera);
    int tiles_h = 1 + (cam.H - 1) / TW, tiles_w = 1 + (cam.W - 1) / TW;
    int64_t T = (int64_t)tiles_h * tiles_w;
    int TS = TW * TW;
    real HW = (real)(cam.H * cam.W);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t tile = 0; tile < T; tile++) {
        fwd_lane *L = (fwd_lane *)calloc((size_t)TS, sizeof(fwd_lane));
        for (int l = 0; l < TS; l++) {
            fwd_lane *a = &L[l];
            lane_setup(&cam, ray_maps, TW, tiles_h, tile, l, &a->o, &a->d, &a->oob, &a->pi, &a->pj);
            a->log_t = 0; a->nd = 0; a->rgb = mk(0, 0, 0); a->normal = mk(0, 0, 0);
            int64_t px = (int64_t)a->pi * cam.W + a->pj;
            if (depth_q) { a->qi = 0; a->q = (real)depth_q[px * Q + 0]; } else { a->qi = 0; a->q = 0; }
            a->err = 0;
            if (return_point_err || err_out) a->gt = ld3(ray_gt + 3 * px);
        }
        int nq = depth_q ? Q : 0;
        int64_t start = tile_offsets[tile], end = tile_offsets[tile + 1];
        int32_t total = (int32_t)(end - start);
        int stopped = 0;
        for (int32_t k = 0; k < total; k++) {
            int32_t prim = tile_prims[start + k];
            int all_below = 1;
            for (int l = 0; l < TS; l++)
                if (!(r_exp(L[l].log_t) < (real)thr)) all_below = 0;
            if (all_below) { early_stop[tile] = k; stopped = 1; break; }
            const float *sp = spheres + 4 * (int64_t)prim;
            const float *ns = nsigmas + 4 * (int64_t)prim;
            v3 center = ld3(sp);
            real radius = (real)sp[3];
            v3 pn = ld3(ns);
            real sigma = (real)ns[3];
            int any = 0;
            for (int l = 0; l < TS; l++) {
                L[l].hit = ray_sphere(L[l].o, L[l].d, center, radius, &L[l].tn, &L[l].tf);
                any += L[l].hit;
            }
            if (any == 0) continue;
            int32_t a0 = adj_off[prim], a1 = adj_off[prim + 1];
            const float *ps = sites + (int64_t)prim * S * 3;
            const float *pv = rgbh + (int64_t)prim * S * 4;
            for (int l = 0; l < TS; l++) {
                fwd_lane *a = &L[l];
                real tn = a->tn, tf = a->tf;
                if (a->hit) {
                    for (int32_t e = a0; e < a1; e++) {
                        v3 ac;
                        real ar;
                        nbr_sphere(spheres, adj, adj_diff, e, center, &ac, &ar);
                        real dp;
                        real t_face = ray_pface(a->o, a->d, center, radius, ac, ar, &dp);
                        tf = dp >= K(0.0) ? rmin(t_face, tf) : tf;
                        tn = dp < K(0.0) ? rmax(t_face, tn) : tn;
                    }
                }
                plane_res pr = plane_fwd(a->o, a->d, tn, center, pn, radius, !a->oob && a->hit, ps, pv, S);
                tf = pr.dp >= K(0.0) ? rmin(pr.t_surf, tf) : tf;
                tn = pr.dp < K(0.0) ? rmax(pr.t_surf, tn) : tn;
                real dt = tf - tn;
                if (a->hit && dt > K(0.0)) {
                    real dlt = -sigma * dt;
                    real alpha = K(1.0) - r_exp(dlt);
                    real trans = r_exp(a->log_t);
                    if (err_out) {
                        v3 de = vsub(pr.rgb, a->gt);
                        a->err += dot(de, de) * alpha * trans;
                    }
                    a->rgb = vadd(a->rgb, smul(trans, smul(alpha, pr.rgb)));
                    a->log_t += dlt;
                    ATOMIC_ADD(contrib[prim], alpha * trans / HW);
                    if (return_point_err) {
                        v3 df = vsub(pr.rgb, a->gt);
                        real l1 = r_fabs(df.x) + r_fabs(df.y) + r_fabs(df.z);
                        ATOMIC_ADD(point_err[prim], alpha * trans * l1 / HW);
                    }
                    real ndv = dot(pn, a->d);
                    if (ndv > 0) a->nd += ndv * ndv * alpha * trans;
                    a->normal = vadd(a->normal, smul(alpha * trans, pn));
                    real next_trans = r_exp(a->log_t);
                    int64_t px = (int64_t)a->pi * cam.W + a->pj;
                    while (a->qi < nq && next_trans < a->q) {
                        real qd = tn + r_log(trans / a->q) / sigma;
                        qdepth_out[px * Q + a->qi] = (out_t)qd;
                        a->qi += 1;
                        if (a->qi < nq) a->q = (real)depth_q[px * Q + a->qi];
                    }
                }
            }
        }
        if (!stopped) early_stop[tile] = total;
        for (int l = 0; l < TS; l++) {
            fwd_lane *a = &L[l];
            if (a->oob) continue;
            int64_t px = (int64_t)a->pi * cam.W + a->pj;
            color[3 * px + 0] = (out_t)a->rgb.x;
            color[3 * px + 1] = (out_t)a->rgb.y;
            color[3 * px + 2] = (out_t)a->rgb.z;
            log_t_out[px] = (out_t)a->log_t;
            nd_out[px] = (out_t)a->nd;
            normal_out[3 * px + 0] = (out_t)a->normal.x;
            normal_out[3 * px + 1] = (out_t)a->normal.y;
            normal_out[3 * px + 2] = (out_t)a->normal.z;
            if (err_out) {
                v3 de = vsub(mk(0, 0, 0), a->gt);
                err_out[px] = (out_t)(a->err + dot(de, de) * r_exp(a->log_t));
            }
        }
        free(L);
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
int FN(orc_raster_forward)(const orc_camera *camera, int TW, int64_t N, const float *spheres,
                           const float *nsigmas, const float *sites, const float *rgbh, int S,
                           const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                           const int64_t *tile_offsets, const int32_t *tile_prims, const float *depth_q,
                           int Q, const float *ray_gt, float thr, int return_point_err, out_t *color,
                           out_t *log_t_out, out_t *nd_out, out_t *normal_out, out_t *qdepth_out,
                           out_t *err_out, out_t *contrib, out_t *point_err, int32_t *early_stop) {
    return FN(raster_forward)(camera, NULL, TW, N, spheres, nsigmas, sites, rgbh, S, adj, adj_off, adj_diff,
                              tile_offsets, tile_prims, depth_q, Q, ray_gt, thr, return_point_err, color, log_t_out,
                              nd_out, normal_out, qdepth_out, err_out, contrib, point_err, early_stop);
}

/* The same with a generic camera: per-pixel rays from ray_maps (H,W,6). */
int FN(orc_raster_forward_generic)(const orc_camera *camera, const float *ray_maps, int TW, int64_t N,
                                   const float *spheres, const float *nsigmas, const float *sites, const float *rgbh,
                                   int S, const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                                   const int64_t *tile_offsets, const int32_t *tile_prims, const float *depth_q,
                                   int Q, const float *ray_gt, float thr, int return_point_err, out_t *color,
                                   out_t *log_t_out, out_t *nd_out, out_t *normal_out, out_t *qdepth_out,
                                   out_t *err_out, out_t *contrib, out_t *point_err, int32_t *early_stop) {
    return FN(raster_forward)(camera, ray_maps, TW, N, spheres, nsigmas, sites, rgbh, S, adj, adj_off, adj_diff,
                              tile_offsets, tile_prims, depth_q, Q, ray_gt, thr, return_point_err, color, log_t_out,
                              nd_out, normal_out, qdepth_out, err_out, contrib, point_err, early_stop);
}

/* ------------------------------------------------------------------------ */
/* Rasterizer backward (rasterize.py:1150-1514 backward_kernel; host side   */
/* rasterize.py:1861-1980).  log_t_grad is dL/dlog_t = -dL/dopacity*exp(log_t)*/
/* (computed by the caller as the reference's host code does).  Gradient    */
/* outputs must be zeroed by the caller; non-finite entries are zeroed here  */
/* at the end, as rasterize.py:1954-1958 does.                               */

typedef struct {
    v3 o, d;
    int oob, pi, pj;
    real log_t, dLdlog_t;
    v3 g_rgb, g_n;
    real g_nd;
    int qi;
    real q;
    int hit;
    real tn, tf;
} bwd_lane;

static void zero_nonfinite(float *a, int64_t n) {
    for (int64_t i = 0; i < n; i++)
        if (!isfinite(a[i])) a[i] = 0.0f;
}

static int FN(raster_backward)(const orc_camera *camera, const float *ray_maps, int TW, int64_t N,
                               const float *spheres, const float *nsigmas, const float *sites, const float *rgbh,
                               int S, const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                               const int64_t *tile_offsets, const int32_t *tile_prims, const int32_t *early_stop,
                               const float *depth_q, int Q, const float *log_t_in, const float *color_grad,
                               const float *log_t_grad, const float *nd_grad, const float *normal_grad,
                               const float *qdepth_grad, const float *contrib_grad, float *spheres_g,
                               float *nsigmas_g, float *sites_g, float *rgb_g, float *height_g) {
    cam_t cam = cam_load(camera);
    int tiles_h = 1 + (cam.H - 1) / TW, tiles_w = 1 + (cam.W - 1) / TW;
    int64_t T = (int64_t)tiles_h * tiles_w;
    int TS = TW * TW;
    real HW = (real)(cam.H * cam.W);
    v3 bkgd = mk(0, 0, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t tile = 0; tile < T; tile++) {
        bwd_lane *L = (bwd_lane *)calloc((size_t)TS, sizeof(bwd_lane));
        for (int l = 0; l < TS; l++) {
            bwd_lane *a = &L[l];
            lane_setup(&cam, ray_maps, TW, tiles_h, tile, l, &a->o, &a->d, &a->oob, &a->pi, &a->pj);
            int64_t px = (int64_t)a->pi * cam.W + a->pj;
            a->log_t = (real)log_t_in[px];
            if (depth_q) { a->qi = Q - 1; a->q = (real)depth_q[px * Q + Q - 1]; } else { a->qi = -1; a->q = K(1.0); }
            a->g_rgb = ld3(color_grad + 3 * px);
            real g_logt = (real)log_t_grad[px];
            a->g_nd = (real)nd_grad[px];
            a->g_n = ld3(normal_grad + 3 * px);
            real dLdtrans = dot(a->g_rgb, bkgd);
            a->dLdlog_t = dLdtrans * r_exp(a->log_t);
            a->dLdlog_t += g_logt;
        }
        int64_t start = tile_offsets[tile];
        int32_t es = early_stop[tile];
        for (int32_t k = es - 1; k >= 0; k--) {
            int32_t prim = tile_prims[start + k];
            const float *sp = spheres + 4 * (int64_t)prim;
            const float *ns = nsigmas + 4 * (int64_t)prim;
            v3 center = ld3(sp);
            real radius = (real)sp[3];
            v3 pn = ld3(ns);
            real sigma = (real)ns[3];
            int any = 0;
            for (int l = 0; l < TS; l++) {
                L[l].hit = ray_sphere(L[l].o, L[l].d, center, radius, &L[l].tn, &L[l].tf);
                any += L[l].hit;
            }
            if (any == 0) continue;
            int32_t a0 = adj_off[prim], a1 = adj_off[prim + 1];
            int n_adj = a1 - a0;
            const float *ps = sites + (int64_t)prim * S * 3;
            const float *pv = rgbh + (int64_t)prim * S * 4;
            float *gs = sites_g + (int64_t)prim * S * 3;
            float *gr = rgb_g + (int64_t)prim * S * 3;
            float *gh = height_g + (int64_t)prim * S;
            for (int l = 0; l < TS; l++) {
                bwd_lane *a = &L[l];
                int hit = a->hit;
                real t_near = a->tn, t_far = a->tf;
                int t_near_id = t_near < K(1e-8) ? -2 : -1;
                int t_far_id = t_far < K(1e-8) ? -2 : -1;
                if (hit) {
                    for (int32_t e = a0; e < a1; e++) {
                        v3 ac;
                        real ar;
                        nbr_sphere(spheres, adj, adj_diff, e, center, &ac, &ar);
                        real dp;
                        real t_face = ray_pface(a->o, a->d, center, radius, ac, ar, &dp);
                        int adj_idx = e - a0;
                        t_far_id = (dp >= K(0.0) && t_face < t_far) ? adj_idx : t_far_id;
                        t_far = dp >= K(0.0) ? rmin(t_face, t_far) : t_far;
                        t_near_id = (dp < K(0.0) && t_face > t_near) ? adj_idx : t_near_id;
                        t_near = dp < K(0.0) ? rmax(t_face, t_near) : t_near;
                    }
                }
                real _t_near = t_near;
                int _t_near_id = t_near_id, _t_far_id = t_far_id;
                plane_res pr = plane_fwd(a->o, a->d, t_near, center, pn, radius, !a->oob && hit, ps, pv, S);
                t_far_id = (pr.dp >= K(0.0) && pr.t_surf < t_far) ? n_adj : t_far_id;
                t_far = pr.dp >= K(0.0) ? rmin(pr.t_surf, t_far) : t_far;
                t_near_id = (pr.dp < K(0.0) && pr.t_surf > t_near) ? n_adj : t_near_id;
                t_near = pr.dp < K(0.0) ? rmax(pr.t_surf, t_near) : t_near;
                real dt = t_far - t_near;
                real dLdt_near = 0, dLdt_far = 0, dLdradius = 0, dLdsigma = 0;
                v3 dLdcenter = mk(0, 0, 0), dLdnormal = mk(0, 0, 0), dLdcolor = mk(0, 0, 0);
                int contributes = !a->oob && hit && dt > K(0.0);
                if (contributes) {
                    int64_t px = (int64_t)a->pi * cam.W + a->pj;
                    real delta_log_t = -sigma * dt;
                    a->log_t -= delta_log_t;
                    real alpha = K(1.0) - r_exp(delta_log_t);
                    real trans = r_exp(a->log_t);
                    real ndv = dot(pn, a->d);
                    real dLdlog_t_i = a->dLdlog_t;
                    real dLddelta_log_t = a->dLdlog_t;
                    real cg = (real)contrib_grad[prim];
                    real dLdalpha = dot(a->g_rgb, pr.rgb) * trans;
                    if (ndv > 0) dLdalpha += a->g_nd * ndv * trans;
                    dLdalpha += cg * trans / HW;
                    dLdalpha += dot(a->g_n, pn) * trans;
                    real dLdtrans = dot(a->g_rgb, pr.rgb) * alpha;
                    if (ndv > 0) dLdtrans += a->g_nd * ndv * alpha;
                    dLdtrans += cg * alpha / HW;
                    dLdtrans += dot(a->g_n, pn) * alpha;
                    dLdcolor = vadd(dLdcolor, smul(alpha, smul(trans, a->g_rgb)));
                    dLdlog_t_i += dLdtrans * r_exp(a->log_t);
                    dLddelta_log_t += -dLdalpha * r_exp(delta_log_t);
                    dLdsigma += dLddelta_log_t * -dt;
                    dLdt_near += dLddelta_log_t * sigma;
                    dLdt_far += dLddelta_log_t * -sigma;
                    while (a->qi >= 0 && trans > a->q) {
                        real dq = (real)qdepth_grad[px * Q + a->qi];
                        dLdsigma += -dq * r_log(trans / a->q) / (sigma * sigma + K(1e-6));
                        dLdt_near += dq;
                        dLdlog_t_i += dq / (sigma + K(1e-6));
                        a->qi -= 1;
                        if (a->qi >= 0) a->q = (real)depth_q[px * Q + a->qi];
                    }
                    dLdnormal = vadd(dLdnormal, smul(alpha * trans, a->g_n));
                    if (ndv > 0) dLdnormal = vadd(dLdnormal, smul(a->g_nd * alpha * trans, a->d));
                    a->dLdlog_t = dLdlog_t_i;
                }
                real dLdt_surf;
                if (t_near_id == n_adj) dLdt_surf = dLdt_near;
                else if (t_far_id == n_adj) dLdt_surf = dLdt_far;
                else dLdt_surf = K(0.0);
                v3 _dc, _dn;
                real dLd_t_near;
                plane_bwd(a->o, a->d, _t_near, center, pn, radius, contributes, ps, pv, pr._dp, pr._t_surf,
                          pr.height, pr._wsum, pr.dp, pr.t_surf, pr.rgb, pr.wsum, dLdcolor, dLdt_surf, S, gs,
                          gr, gh, &_dc, &_dn, &dLd_t_near);
                dLdcenter = vadd(dLdcenter, _dc);
                dLdnormal = vadd(dLdnormal, _dn);
                if (t_near_id != n_adj) dLd_t_near += dLdt_near;
                if (contributes) {
                    for (int i = 0; i < 2; i++) {
                        int t_id = i == 0 ? _t_near_id : _t_far_id;
                        real dLdt = i == 0 ? dLd_t_near : dLdt_far;
                        if (t_id == -1) {
                            v3 ndc, fdc;
                            real ndr, fdr;
                            ray_sphere_bwd(a->o, a->d, center, radius, &ndc, &fdc, &ndr, &fdr);
                            if (i == 0) {
                                dLdcenter = vadd(dLdcenter, smul(dLdt, ndc));
                                dLdradius += dLdt * ndr;
                            } else {
                                dLdcenter = vadd(dLdcenter, smul(dLdt, fdc));
                                dLdradius += dLdt * fdr;
                            }
                        } else if (t_id >= 0 && t_id < n_adj) {
                            int32_t adjacent = adj[a0 + t_id];
                            const float *as = spheres + 4 * (int64_t)adjacent;
                            v3 dc, dac;
                            real dr, dar;
                            ray_pface_bwd(a->o, a->d, center, radius, ld3(as), (real)as[3], &dc, &dr, &dac, &dar);
                            dLdcenter = vadd(dLdcenter, smul(dLdt, dc));
                            dLdradius += dLdt * dr;
                            v3 g = smul(dLdt, dac);
                            ATOMIC_ADD(spheres_g[4 * (int64_t)adjacent + 0], g.x);
                            ATOMIC_ADD(spheres_g[4 * (int64_t)adjacent + 1], g.y);
                            ATOMIC_ADD(spheres_g[4 * (int64_t)adjacent + 2], g.z);
                            ATOMIC_ADD(spheres_g[4 * (int64_t)adjacent + 3], dLdt * dar);
                        }
                    }
                    ATOMIC_ADD(spheres_g[4 * (int64_t)prim + 0], dLdcenter.x);
                    ATOMIC_ADD(spheres_g[4 * (int64_t)prim + 1], dLdcenter.y);
                    ATOMIC_ADD(spheres_g[4 * (int64_t)prim + 2], dLdcenter.z);
                    ATOMIC_ADD(spheres_g[4 * (int64_t)prim + 3], dLdradius);
                    ATOMIC_ADD(nsigmas_g[4 * (int64_t)prim + 0], dLdnormal.x);
                    ATOMIC_ADD(nsigmas_g[4 * (int64_t)prim + 1], dLdnormal.y);
                    ATOMIC_ADD(nsigmas_g[4 * (int64_t)prim + 2], dLdnormal.z);
                    ATOMIC_ADD(nsigmas_g[4 * (int64_t)prim + 3], dLdsigma);
                }
            }
        }
        free(L);
    }
    zero_nonfinite(spheres_g, 4 * N);
    zero_nonfinite(nsigmas_g, 4 * N);
    zero_nonfinite(sites_g, 3 * N * S);
    zero_nonfinite(rgb_g, 3 * N * S);
    zero_nonfinite(height_g, N * S);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Rasterizer benchmark path (rasterize.py:614-734 benchmark_kernel): per-   */
/* thread early-out, (dc, dpm)-encoded neighbour faces with break, local     */
/* plane with separate sites/rgb/height arrays (which hold float32 values,   */
/* already rounded to float16 by the caller for attr_dtype "half").          */
int FN(orc_raster_backward)(const orc_camera *camera, int TW, int64_t N, const float *spheres,
                            const float *nsigmas, const float *sites, const float *rgbh, int S,
                            const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                            const int64_t *tile_offsets, const int32_t *tile_prims,
                            const int32_t *early_stop, const float *depth_q, int Q,
                            const float *log_t_in, const float *color_grad, const float *log_t_grad,
                            const float *nd_grad, const float *normal_grad, const float *qdepth_grad,
                            const float *contrib_grad, float *spheres_g, float *nsigmas_g, float *sites_g,
                            float *rgb_g, float *height_g) {
    return FN(raster_backward)(camera, NULL, TW, N, spheres, nsigmas, sites, rgbh, S, adj, adj_off, adj_diff,
                               tile_offsets, tile_prims, early_stop, depth_q, Q, log_t_in, color_grad, log_t_grad,
                               nd_grad, normal_grad, qdepth_grad, contrib_grad, spheres_g, nsigmas_g, sites_g,
                               rgb_g, height_g);
}

/* The same with a generic camera: per-pixel rays from ray_maps (H,W,6). */
int FN(orc_raster_backward_generic)(const orc_camera *camera, const float *ray_maps, int TW, int64_t N,
                                    const float *spheres, const float *nsigmas, const float *sites,
                                    const float *rgbh, int S, const int32_t *adj, const int32_t *adj_off,
                                    const uint16_t *adj_diff, const int64_t *tile_offsets,
                                    const int32_t *tile_prims, const int32_t *early_stop, const float *depth_q,
                                    int Q, const float *log_t_in, const float *color_grad, const float *log_t_grad,
                                    const float *nd_grad, const float *normal_grad, const float *qdepth_grad,
                                    const float *contrib_grad, float *spheres_g, float *nsigmas_g, float *sites_g,
                                    float *rgb_g, float *height_g) {
    return FN(raster_backward)(camera, ray_maps, TW, N, spheres, nsigmas, sites, rgbh, S, adj, adj_off, adj_diff,
                               tile_offsets, tile_prims, early_stop, depth_q, Q, log_t_in, color_grad, log_t_grad,
                               nd_grad, normal_grad, qdepth_grad, contrib_grad, spheres_g, nsigmas_g, sites_g,
                               rgb_g, height_g);
}

int FN(orc_raster_benchmark)(const orc_camera *camera, int TW, const float *spheres, const float *nsigmas,
                             const float *sites, const float *rgbs, const float *heights, int S,
                             const int32_t *adj_off, const uint16_t *adj_diff, const int64_t *tile_offsets,
                             const int32_t *tile_prims, float thr, float *color) {
    cam_t cam = cam_load(camera);
    int tiles_h = 1 + (cam.H - 1) / TW, tiles_w = 1 + (cam.W - 1) / TW;
    int64_t T = (int64_t)tiles_h * tiles_w;
    int TS = TW * TW;
    v3 o = cam.eye;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t tile = 0; tile < T; tile++) {
        for (int l = 0; l < TS; l++) {
            v3 d;
            int oob, pi, pj;
            v3 o_unused;
            lane_setup(&cam, NULL, TW, tiles_h, tile, l, &o_unused, &d, &oob, &pi, &pj);
            v3 rgb = mk(0, 0, 0);
            real log_t = 0;
            int64_t start = tile_offsets[tile], end = tile_offsets[tile + 1];
            int32_t total = (int32_t)(end - start);
            for (int32_t k = 0; k < total; k++) {
                int32_t prim = tile_prims[start + k];
                real trans = r_exp(log_t);
                if (trans < (real)thr) break;
                const float *sp = spheres + 4 * (int64_t)prim;
                const float *ns = nsigmas + 4 * (int64_t)prim;
                v3 center = ld3(sp);
                real radius = (real)sp[3];
                v3 pn = ld3(ns);
                real sigma = (real)ns[3];
                real tn, tf;
                int hit = ray_sphere(o, d, center, radius, &tn, &tf);
                if (!hit) continue;
                for (int32_t e = adj_off[prim]; e < adj_off[prim + 1]; e++) {
                    const uint16_t *h = adj_diff + 4 * (int64_t)e;
                    v3 diff = mk((real)FN(orc_h2f)(h[0]), (real)FN(orc_h2f)(h[1]), (real)FN(orc_h2f)(h[2]));
                    real pm = (real)FN(orc_h2f)(h[3]);
                    real dp;
                    real t_face = ray_pface_diff(o, d, diff, pm, &dp);
                    tf = dp >= K(0.0) ? rmin(t_face, tf) : tf;
                    tn = dp < K(0.0) ? rmax(t_face, tn) : tn;
                    if (tn > tf) break;
                }
                if (tn > tf) continue;
                plane_res pr = plane_fwd_local(o, d, tn, center, pn, radius, sites + (int64_t)prim * S * 3,
                                               rgbs + (int64_t)prim * S * 3, heights + (int64_t)prim * S, S);
                tf = pr.dp >= K(0.0) ? rmin(pr.t_surf, tf) : tf;
                tn = pr.dp < K(0.0) ? rmax(pr.t_surf, tn) : tn;
                real dt = tf - tn;
                if (hit && dt > K(0.0)) {
                    real dlt = -sigma * dt;
                    real alpha = K(1.0) - r_exp(dlt);
                    trans = r_exp(log_t);
                    rgb = vadd(rgb, smul(trans, smul(alpha, pr.rgb)));
                    log_t += dlt;
                }
            }
            if (!oob) {
                int64_t px = (int64_t)pi * cam.W + pj;
                color[3 * px + 0] = (float)rgb.x;
                color[3 * px + 1] = (float)rgb.y;
                color[3 * px + 2] = (float)rgb.z;
            }
        }
    }
    return ORC_OK;
}

/* rasterize.py:738-888 visualization_kernel (viewer path, headless). */
int FN(orc_raster_visualize)(const orc_camera *camera, int TW, const float *spheres, const float *nsigmas,
                             const float *sites, const float *rgbs, const float *heights, int S,
                             const int32_t *adj_off, const uint16_t *adj_diff, const int64_t *tile_offsets,
                             const int32_t *tile_prims, float thr, int max_intersections, float depth_quantile,
                             const float *bkgd, float *color, float *depth, float *normal, float *alpha_out,
                             int32_t *intersections) {
    cam_t cam = cam_load(camera);
    int tiles_h = 1 + (cam.H - 1) / TW, tiles_w = 1 + (cam.W - 1) / TW;
    int64_t T = (int64_t)tiles_h * tiles_w;
    int TS = TW * TW;
    v3 o = cam.eye;
    v3 bk = ld3(bkgd);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t tile = 0; tile < T; tile++) {
        for (int l = 0; l < TS; l++) {
            v3 d;
            int oob, pi, pj;
            v3 o_unused;
            lane_setup(&cam, NULL, TW, tiles_h, tile, l, &o_unused, &d, &oob, &pi, &pj);
            v3 rgb = mk(0, 0, 0), nacc = mk(0, 0, 0);
            real dq_out = 0;
            int dq_found = 0;
            real log_t = 0;
            int32_t n_hit = 0;
            int64_t start = tile_offsets[tile], end = tile_offsets[tile + 1];
            int32_t total = (int32_t)(end - start);
            for (int32_t k = 0; k < total; k++) {
                n_hit += 1;
                if (k >= max_intersections) break;
                int32_t prim = tile_prims[start + k];
                real trans = r_exp(log_t);
                if (trans < (real)thr) break;
                const float *sp = spheres + 4 * (int64_t)prim;
                const float *ns = nsigmas + 4 * (int64_t)prim;
                v3 center = ld3(sp);
                real radius = (real)sp[3];
                v3 pn = ld3(ns);
                real sigma = (real)ns[3];
                real tn, tf;
                int hit = ray_sphere(o, d, center, radius, &tn, &tf);
                if (!hit) continue;
                for (int32_t e = adj_off[prim]; e < adj_off[prim + 1]; e++) {
                    const uint16_t *h = adj_diff + 4 * (int64_t)e;
                    v3 ac = vadd(center, mk((real)FN(orc_h2f)(h[0]), (real)FN(orc_h2f)(h[1]),
                                            (real)FN(orc_h2f)(h[2])));
                    real ar = (real)FN(orc_h2f)(h[3]);
                    real dp;
                    real t_face = ray_pface(o, d, center, radius, ac, ar, &dp);
                    tf = dp >= K(0.0) ? rmin(t_face, tf) : tf;
                    tn = dp < K(0.0) ? rmax(t_face, tn) : tn;
                    if (tn > tf) break;
                }
                if (tn > tf) continue;
                plane_res pr = plane_fwd_local(o, d, tn, center, pn, radius, sites + (int64_t)prim * S * 3,
                                               rgbs + (int64_t)prim * S * 3, heights + (int64_t)prim * S, S);
                tf = pr.dp >= K(0.0) ? rmin(pr.t_surf, tf) : tf;
                tn = pr.dp < K(0.0) ? rmax(pr.t_surf, tn) : tn;
                real dt = tf - tn;
                if (hit && dt > K(0.0)) {
                    real dlt = -sigma * dt;
                    real alpha = K(1.0) - r_exp(dlt);
                    trans = r_exp(log_t);
                    rgb = vadd(rgb, smul(trans, smul(alpha, pr.rgb)));
                    nacc = vadd(nacc, smul(trans, smul(alpha, pn)));
                    log_t += dlt;
                    if (!dq_found) {
                        real next_trans = r_exp(log_t);
                        if (next_trans < (real)depth_quantile) {
                            dq_out = tn + r_log(trans / (real)depth_quantile) / sigma;
                            dq_found = 1;
                        }
                    }
                }
            }
            if (!oob) {
                int64_t px = (int64_t)pi * cam.W + pj;
                real ray_trans = r_exp(log_t);
                real ray_alpha = K(1.0) - ray_trans;
                rgb = vadd(rgb, smul(ray_trans, bk));
                color[3 * px + 0] = (float)rgb.x;
                color[3 * px + 1] = (float)rgb.y;
                color[3 * px + 2] = (float)rgb.z;
                depth[px] = (float)dq_out;
                normal[3 * px + 0] = (float)nacc.x;
                normal[3 * px + 1] = (float)nacc.y;
                normal[3 * px + 2] = (float)nacc.z;
                alpha_out[px] = (float)ray_alpha;
                intersections[px] = n_hit;
            }
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Ray tracer (raytrace.py:115-241 benchmark_kernel).                        */
/* Extensions over the reference kernel, none of which changes the colour:   */
/*  - per-ray start cells (start_cells may be NULL: every ray starts at     */
/*    start_idx, as the reference does);                                     */
/*  - a step cap (the reference loops without bound); hitting it sets the   */
/*    ray's status to ORC_ERR_STEP_CAP;                                      */
/*  - the cycle guard (cycle_closed): the next cell is a function of the    */
/*    current one (raytrace.py:183-199), so a ray that returns to a cell    */
/*    with no hit since (sphere hit, tn <= tf, sigma >= 1e-3) repeats those */
/*    cells forever with an unchanged transmittance -- the reference never  */
/*    returns from such a ray.  The walk keeps the cell of step 0, 1, 2, 4, */
/*    ... (Brent's power-of-two saves) and ends when it comes back to it    */
/*    with no hit since; rays the reference finishes never meet the guard;  */
/*  - depth (first crossing of T < depth_quantile, visualization_kernel's   */
/*    formula), normal (sum alpha*T*n, forward_kernel's formula), final      */
/*    log transmittance, and the visited-cell log (every cell whose sphere  */
/*    the walk reads, in order).                                             */
/* depth_seg/depth_sigma record which step produced the depth and that       */
/* cell's sigma (-1 / 0 when the ray never crosses the quantile); they are   */
/* the only state the backward needs besides the forward outputs.            */
#define NO_CELL 0x7FFFFFFF

static int cycle_closed(int32_t *saved, int *hit_since, int32_t prim, int steps) {
    if (prim == *saved && !*hit_since) return 1;
    if ((steps & (steps - 1)) == 0) {
        *saved = prim;
        *hit_since = 0;
    }
    return 0;
}

/* (c_j - c_i, pm_j - pm_i) of neighbour e: from the float16 encoding of
 * benchmark.py:296-302, or exactly from the spheres when adj_diff == NULL
 * (finite-difference checks) */
static void nbr_pm(const float *spheres, const int32_t *adj, const uint16_t *adj_diff, int32_t prim, int32_t e,
                   v3 *diff, real *pm) {
    if (adj_diff) {
        const uint16_t *h = adj_diff + 4 * (int64_t)e;
        *diff = mk((real)FN(orc_h2f)(h[0]), (real)FN(orc_h2f)(h[1]), (real)FN(orc_h2f)(h[2]));
        *pm = (real)FN(orc_h2f)(h[3]);
    } else {
        const float *si = spheres + 4 * (int64_t)prim, *sj = spheres + 4 * (int64_t)adj[e];
        v3 ci = ld3(si), cj = ld3(sj);
        real ri = (real)si[3], rj = (real)sj[3];
        *diff = vsub(cj, ci);
        *pm = K(0.5) * (dot(cj, cj) - rj * rj) - K(0.5) * (dot(ci, ci) - ri * ri);
    }
}

/* The walk of orc_trace_forward.  With label outputs it also records, per
 * ray, the first cell after whose compositing the transmittance is below
 * label_thr: the t at which the ray enters that cell (label_t), the cell
 * (label_cell) and the number of cells walked before it (label_step); -1 in
 * all three when the transmittance never falls below label_thr. */
static int FN(trace_walk)(const orc_camera *camera, const float *spheres, const float *nsigmas,
                          const float *sites, const float *rgbs, const float *heights, int S,
                          const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                          int32_t start_idx, const int32_t *start_cells, float thr, int max_steps,
                          float depth_quantile, out_t *color, out_t *log_t_out, out_t *depth, out_t *normal,
                          int32_t *depth_seg, out_t *depth_sigma, int32_t *visit_log, int visit_cap,
                          int32_t *visit_count, int32_t *status, float label_thr, out_t *label_t,
                          int32_t *label_cell, int32_t *label_step, const int64_t *pixels, int64_t n_pixels) {
    cam_t cam = cam_load(camera);
    const int64_t HW = (int64_t)cam.H * cam.W;
    int64_t P = pixels ? n_pixels : HW;
    v3 o = cam.eye;
    int worst = ORC_OK;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : worst)
    for (int64_t px = 0; px < P; px++) {
        /* px indexes the outputs; ray is the camera pixel traced (a subset of
         * the pixels when a list is given) */
        const int64_t ray = pixels ? pixels[px] : px;
        if (ray < 0 || ray >= HW) {
            if (status) status[px] = ORC_ERR_ARGS;
            if (ORC_ERR_ARGS > worst) worst = ORC_ERR_ARGS;
            continue;
        }
        int pi = (int)(ray / cam.W), pj = (int)(ray % cam.W);
        v3 rd = get_ray_dir(&cam, (real)pi, (real)pj);
        v3 d = vdivs(rd, length(rd));
        v3 rgb = mk(0, 0, 0), nacc = mk(0, 0, 0);
        real log_t = 0;
        int32_t prim = start_cells ? start_cells[ray] : start_idx;
        real pt_near = 0;
        int steps = 0, st = ORC_OK, seg = 0;
        int32_t dseg = -1;
        real dout = 0, dsig = 0;
        real lab_t = -1;
        int32_t lab_cell = -1, lab_step = -1;
        int32_t cg_saved = -1;
        int cg_hit = 0;
        for (;;) {
            real trans = r_exp(log_t);
            if (trans < (real)thr || prim == NO_CELL) break;
            if (steps >= max_steps) { st = ORC_ERR_STEP_CAP; break; }
            if (cycle_closed(&cg_saved, &cg_hit, prim, steps)) break;
            if (visit_log && steps < visit_cap) visit_log[px * visit_cap + steps] = prim;
            const real cell_entry = pt_near;
            const int32_t cell = prim;
            steps++;
            const float *sp = spheres + 4 * (int64_t)prim;
            v3 center = ld3(sp);
            real radius = (real)sp[3];
            real tn, tf;
            int hit = ray_sphere(o, d, center, radius, &tn, &tf);
            v3 v = vsub(center, o);
            if (length(v) < K(4.0) * radius) hit = 0;
            int32_t next = NO_CELL;
            real pt_far = K(1e10);
            for (int32_t e = adj_off[prim]; e < adj_off[prim + 1]; e++) {
                v3 diff;
                real pm;
                nbr_pm(spheres, adj, adj_diff, prim, e, &diff, &pm);
                real dp;
                real t_face = ray_pface_diff(o, d, diff, pm, &dp);
                if (dp >= K(0.0) && t_face < pt_far) { next = adj[e]; pt_far = t_face; }
                tf = dp >= K(0.0) ? rmin(t_face, tf) : tf;
                tn = dp < K(0.0) ? rmax(t_face, tn) : tn;
            }
            const float *ns = nsigmas + 4 * (int64_t)prim;
            v3 pn = ld3(ns);
            real sigma = (real)ns[3];
            if (!hit || tn > tf || sigma < K(1e-3)) {
                prim = next;
                pt_near = rmax(pt_near, pt_far);
                continue;
            }
            cg_hit = 1;
            plane_res pr = plane_fwd_local(o, d, tn, center, pn, radius, sites + (int64_t)prim * S * 3,
                                           rgbs + (int64_t)prim * S * 3, heights + (int64_t)prim * S, S);
            tf = pr.dp >= K(0.0) ? rmin(pr.t_surf, tf) : tf;
            tn = pr.dp < K(0.0) ? rmax(pr.t_surf, tn) : tn;
            prim = next;
            pt_near = rmax(pt_near, pt_far);
            real dt = tf - tn;
            if (hit && dt > K(0.0)) {
                real dlt = -sigma * dt;
                real alpha = K(1.0) - r_exp(dlt);
                rgb = vadd(rgb, smul(trans, smul(alpha, pr.rgb)));
                nacc = vadd(nacc, smul(alpha * trans, pn));
                log_t += dlt;
                if (dseg < 0 && r_exp(log_t) < (real)depth_quantile) {
                    dout = tn + r_log(trans / (real)depth_quantile) / sigma;
                    dseg = seg;
                    dsig = sigma;
                }
                if (lab_cell < 0 && r_exp(log_t) < (real)label_thr) {
                    lab_t = cell_entry;
                    lab_cell = cell;
                    lab_step = steps - 1;
                }
                seg++;
            }
        }
        if (label_t) label_t[px] = (out_t)lab_t;
        if (label_cell) label_cell[px] = lab_cell;
        if (label_step) label_step[px] = lab_step;
        color[3 * px + 0] = (out_t)rgb.x;
        color[3 * px + 1] = (out_t)rgb.y;
        color[3 * px + 2] = (out_t)rgb.z;
        if (log_t_out) log_t_out[px] = (out_t)log_t;
        if (depth) depth[px] = (out_t)dout;
        if (normal) {
            normal[3 * px + 0] = (out_t)nacc.x;
            normal[3 * px + 1] = (out_t)nacc.y;
            normal[3 * px + 2] = (out_t)nacc.z;
        }
        if (depth_seg) depth_seg[px] = dseg;
        if (depth_sigma) depth_sigma[px] = (out_t)dsig;
        if (visit_count) visit_count[px] = steps;
        if (status) status[px] = st;
        if (st > worst) worst = st;
    }
    return worst;
}

int FN(orc_trace_forward)(const orc_camera *camera, const float *spheres, const float *nsigmas,
                          const float *sites, const float *rgbs, const float *heights, int S,
                          const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                          int32_t start_idx, const int32_t *start_cells, float thr, int max_steps,
                          float depth_quantile, out_t *color, out_t *log_t_out, out_t *depth, out_t *normal,
                          int32_t *depth_seg, out_t *depth_sigma, int32_t *visit_log, int visit_cap,
                          int32_t *visit_count, int32_t *status) {
    return FN(trace_walk)(camera, spheres, nsigmas, sites, rgbs, heights, S, adj, adj_off, adj_diff, start_idx,
                          start_cells, thr, max_steps, depth_quantile, color, log_t_out, depth, normal, depth_seg,
                          depth_sigma, visit_log, visit_cap, visit_count, status, 0.0f, NULL, NULL, NULL, NULL, 0);
}

/* orc_trace_forward on a list of camera pixels (row-major indices): output
 * i (and visit_log row i) belongs to pixel pixels[i]; start_cells, when
 * given, is still indexed by camera pixel.  Test infrastructure for
 * comparing walks of sampled rays of a large frame. */
int FN(orc_trace_forward_pixels)(const orc_camera *camera, const float *spheres, const float *nsigmas,
                                 const float *sites, const float *rgbs, const float *heights, int S,
                                 const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                                 int32_t start_idx, const int32_t *start_cells, float thr, int max_steps,
                                 float depth_quantile, const int64_t *pixels, int64_t n_pixels, out_t *color,
                                 out_t *log_t_out, out_t *depth, out_t *normal, int32_t *depth_seg,
                                 out_t *depth_sigma, int32_t *visit_log, int visit_cap, int32_t *visit_count,
                                 int32_t *status) {
    if (!pixels || n_pixels < 0) return ORC_ERR_ARGS;
    return FN(trace_walk)(camera, spheres, nsigmas, sites, rgbs, heights, S, adj, adj_off, adj_diff, start_idx,
                          start_cells, thr, max_steps, depth_quantile, color, log_t_out, depth, normal, depth_seg,
                          depth_sigma, visit_log, visit_cap, visit_count, status, 0.0f, NULL, NULL, NULL, pixels,
                          n_pixels);
}

/* Training labels of the ray-proposal network (no counterpart in the
 * reference): the walk of orc_trace_forward with the label outputs of
 * trace_walk; colour is written too (the image the labels belong to). */
int FN(orc_trace_labels)(const orc_camera *camera, const float *spheres, const float *nsigmas,
                         const float *sites, const float *rgbs, const float *heights, int S,
                         const int32_t *adj, const int32_t *adj_off, const uint16_t *adj_diff,
                         int32_t start_idx, const int32_t *start_cells, float thr, int max_steps,
                         float label_thr, out_t *color, out_t *label_t, int32_t *label_cell, int32_t *label_step,
                         int32_t *visit_count, int32_t *status) {
    return FN(trace_walk)(camera, spheres, nsigmas, sites, rgbs, heights, S, adj, adj_off, adj_diff, start_idx,
                          start_cells, thr, max_steps, 0.5f, color, NULL, NULL, NULL, NULL, NULL, NULL, 0,
                          visit_count, status, label_thr, label_t, label_cell, label_step, NULL, 0);
}

/* start cell of benchmark.py:320-324: argmin_i |p_i - eye|^2 - r_i^2 with the
 * norm taken first (torch.linalg.norm), first index on ties. */
int32_t FN(orc_start_cell)(const float *points, const float *radii, int64_t N, const float *eye) {
    int32_t best = 0;
    float bv = 0;
    for (int64_t i = 0; i < N; i++) {
        float dx = points[3 * i] - eye[0], dy = points[3 * i + 1] - eye[1], dz = points[3 * i + 2] - eye[2];
        float n = sqrtf(dx * dx + dy * dy + dz * dz);
        float v = n * n - radii[i] * radii[i];
        if (i == 0 || v < bv) { bv = v; best = (int32_t)i; }
    }
    return best;
}

/* ------------------------------------------------------------------------ */
/* Texel colour pre-step used by the synthetic scenes: real spherical        */
/* harmonics of degree 3 (16 coefficients per channel, the constants of      */
/* powerfoam/sh_utils.py:4-50) evaluated at normalize(p - eye), plus 0.5,    */
/* clamped at 0, broadcast to the S texel sites.  sh is (N,16,3).           */
static void FN(sh_basis)(v3 dir, real b[16]) {
    const real C0 = K(0.28209479177387814), C1 = K(0.4886025119029199);
    const real C2[5] = {K(1.0925484305920792), K(-1.0925484305920792), K(0.31539156525252005),
                        K(-1.0925484305920792), K(0.5462742152960396)};
    const real C3[7] = {K(-0.5900435899266435), K(2.890611442640554), K(-0.4570457994644658),
                        K(0.3731763325901154), K(-0.4570457994644658), K(1.445305721320277),
                        K(-0.5900435899266435)};
    real x = dir.x, y = dir.y, z = dir.z;
    real xx = x * x, yy = y * y, zz = z * z;
    b[0] = C0;
    b[1] = -C1 * y; b[2] = C1 * z; b[3] = -C1 * x;
    b[4] = C2[0] * (x * y); b[5] = C2[1] * (y * z); b[6] = C2[2] * (K(2.0) * zz - xx - yy);
    b[7] = C2[3] * (x * z); b[8] = C2[4] * (xx - yy);
    b[9] = C3[0] * y * (K(3.0) * xx - yy); b[10] = C3[1] * (x * y) * z;
    b[11] = C3[2] * y * (K(4.0) * zz - xx - yy); b[12] = C3[3] * z * (K(2.0) * zz - K(3.0) * xx - K(3.0) * yy);
    b[13] = C3[4] * x * (K(4.0) * zz - xx - yy); b[14] = C3[5] * z * (xx - yy);
    b[15] = C3[6] * x * (xx - K(3.0) * yy);
}

static real FN(sh_raw)(const real b[16], const float *c, int ch) {
    real acc = 0;
    for (int k = 0; k < 16; k++) acc += b[k] * (real)c[k * 3 + ch];
    return acc + K(0.5);
}

void FN(orc_sh_texel_rgb)(const float *points, const float *sh, int64_t N, int S, const float *eye,
                          float *texel_rgb) {
    for (int64_t p = 0; p < N; p++) {
        real b[16];
        FN(sh_basis)(normalize(vsub(ld3(points + 3 * p), ld3(eye))), b);
        for (int c = 0; c < 3; c++) {
            real acc = FN(sh_raw)(b, sh + p * 48, c);
            acc = acc > K(0.0) ? acc : K(0.0);
            for (int s = 0; s < S; s++) texel_rgb[(p * S + s) * 3 + c] = (float)acc;
        }
    }
}

/* Adjoint of orc_sh_texel_rgb with respect to the coefficients, ADDED into
 * grad_sh (N,16,3): the colour is broadcast to the S sites (its gradient is
 * the sum over sites) and the clamp passes it where the pre-clamp value is
 * positive.  No gradient reaches the points through the view direction. */
void FN(orc_sh_texel_rgb_backward)(const float *points, const float *sh, int64_t N, int S, const float *eye,
                                   const float *grad_texel_rgb, float *grad_sh) {
    for (int64_t p = 0; p < N; p++) {
        real b[16];
        FN(sh_basis)(normalize(vsub(ld3(points + 3 * p), ld3(eye))), b);
        for (int c = 0; c < 3; c++) {
            if (!(FN(sh_raw)(b, sh + p * 48, c) > K(0.0))) continue;
            real g = 0;
            for (int s = 0; s < S; s++) g += (real)grad_texel_rgb[(p * S + s) * 3 + c];
            for (int k = 0; k < 16; k++) grad_sh[p * 48 + k * 3 + c] += (float)(b[k] * g);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Interpenetration penalty (powerfoam/geometry.py:88-117): for sphere i,    */
/* areas_i = sum over its list, in list order from 0, of (s - d)^2 for the    */
/* entries with d < s, where d = |c_i - c_j| and s = r_i + r_j.  pow(x, 2.0)  */
/* is taken as x * x.                                                         */
void FN(orc_interpenetration)(const float *spheres, const int32_t *adj, const int32_t *adj_off, int64_t N,
                              out_t *areas) {
    for (int64_t i = 0; i < N; i++) {
        v3 c = ld3(spheres + 4 * i);
        real r = (real)spheres[4 * i + 3];
        real acc = K(0.0);
        for (int32_t e = adj_off[i]; e < adj_off[i + 1]; e++) {
            const float *q = spheres + 4 * (int64_t)adj[e];
            real d = length(vsub(c, ld3(q)));
            real s = r + (real)q[3];
            if (d < s) {
                real x = s - d;
                acc += x * x;
            }
        }
        areas[i] = acc;
    }
}

/* Adjoint of orc_interpenetration as Warp's generated adjoint of the same  */
/* kernel computes it (InterpenetrationFunction.backward, geometry.py:158-  */
/* 189): the list is replayed in reverse; per overlapping entry              */
/* g = (2 (s - d)) dL/dareas_i reaches r_i and r_j; when d > 0 the centre    */
/* share a = (v / d) (-g), v = c_i - c_j, is added to c_i and subtracted     */
/* from c_j (length's adjoint is zero at d = 0).  The neighbour's share is   */
/* added at once, the own share once after the list.  grad_spheres (N,4) is  */
/* added into.                                                               */
void FN(orc_interpenetration_backward)(const float *spheres, const int32_t *adj, const int32_t *adj_off, int64_t N,
                                       const float *grad_areas, out_t *grad_spheres) {
    for (int64_t i = 0; i < N; i++) {
        v3 c = ld3(spheres + 4 * i);
        real r = (real)spheres[4 * i + 3];
        real ga = (real)grad_areas[i];
        v3 gc = mk(K(0.0), K(0.0), K(0.0));
        real gr = K(0.0);
        for (int32_t e = adj_off[i + 1] - 1; e >= adj_off[i]; e--) {
            int64_t j = adj[e];
            const float *q = spheres + 4 * j;
            v3 v = vsub(c, ld3(q));
            real d = length(v);
            real s = r + (real)q[3];
            if (!(d < s)) continue;
            real g = (K(2.0) * (s - d)) * ga;
            gr += g;
            grad_spheres[4 * j + 3] += g;
            if (d > K(0.0)) {
                v3 a = mk((v.x / d) * -g, (v.y / d) * -g, (v.z / d) * -g);
                gc = vadd(gc, a);
                grad_spheres[4 * j + 0] -= a.x;
                grad_spheres[4 * j + 1] -= a.y;
                grad_spheres[4 * j + 2] -= a.z;
            }
        }
        grad_spheres[4 * i + 0] += gc.x;
        grad_spheres[4 * i + 1] += gc.y;
        grad_spheres[4 * i + 2] += gc.z;
        grad_spheres[4 * i + 3] += gr;
    }
}

/* ------------------------------------------------------------------------ */
/* Spherical-Voronoi texel colour (powerfoam/color_fn.py:54-184), float32    */
/* attributes: sites / values (dof, N, 3), temps (dof, N).                   */
void FN(orc_sv_forward)(const float *points, const float *origin, const float *forward, float cutoff,
                        const float *sites, const float *values, const float *temps, int64_t N, int dof,
                        out_t *value_out, out_t *wsum_out) {
    v3 o = ld3(origin), fw = ld3(forward);
    for (int64_t t = 0; t < N; t++) {
        v3 dir = normalize(vsub(ld3(points + 3 * t), o));
        if (dot(dir, fw) < (real)cutoff) {
            value_out[3 * t] = value_out[3 * t + 1] = value_out[3 * t + 2] = K(0.5);
            wsum_out[t] = 0;
            continue;
        }
        real ws = K(0.0);
        v3 vs = mk(0, 0, 0);
        for (int i = 0; i < dof; i++) {
            int64_t e = (int64_t)i * N + t;
            v3 axis = ld3(sites + 3 * e), val = ld3(values + 3 * e);
            real temp = (real)temps[e];
            real dist = length(vsub(dir, axis));
            real w = r_exp(-temp * dist);
            ws += w;
            vs = vadd(vs, smul(w, val));
        }
        wsum_out[t] = (out_t)ws;
        v3 v = vadd(vdivs(vs, ws), mk(K(0.5), K(0.5), K(0.5)));
        value_out[3 * t] = (out_t)rmax(v.x, K(0.0));
        value_out[3 * t + 1] = (out_t)rmax(v.y, K(0.0));
        value_out[3 * t + 2] = (out_t)rmax(v.z, K(0.0));
    }
}

/* the adjoint (color_fn.py:105-182); gradients written where the site's
 * normalised weight is >= 1e-3, left untouched elsewhere */
void FN(orc_sv_backward)(const float *points, const float *origin, const float *forward, float cutoff,
                         const float *sites, const float *values, const float *temps, const float *wsum_in,
                         const float *value_in, const float *grad_value, int64_t N, int dof, out_t *g_sites,
                         out_t *g_values, out_t *g_temps) {
    v3 o = ld3(origin), fw = ld3(forward);
    for (int64_t t = 0; t < N; t++) {
        v3 dir = normalize(vsub(ld3(points + 3 * t), o));
        if (dot(dir, fw) < (real)cutoff) continue;
        real ws = (real)wsum_in[t];
        v3 value = ld3(value_in + 3 * t), g = ld3(grad_value + 3 * t);
        if (value.x <= K(0.0)) g.x = 0;
        if (value.y <= K(0.0)) g.y = 0;
        if (value.z <= K(0.0)) g.z = 0;
        value = vsub(value, mk(K(0.5), K(0.5), K(0.5)));
        real dp_out = dot(g, value);
        for (int i = 0; i < dof; i++) {
            int64_t e = (int64_t)i * N + t;
            v3 axis = ld3(sites + 3 * e), val = ld3(values + 3 * e);
            real temp = (real)temps[e];
            real dist = length(vsub(dir, axis));
            real w = r_exp(-temp * dist);
            if (w / ws < K(1e-3)) continue;
            v3 dval = vdivs(smul(w, g), ws);
            g_values[3 * e] = (out_t)dval.x; g_values[3 * e + 1] = (out_t)dval.y; g_values[3 * e + 2] = (out_t)dval.z;
            v3 dwds = vdivs(smul(temp * w, vsub(dir, axis)), dist);
            real dwdt = -dist * w;
            real dp = dot(g, val);
            v3 daxis = vdivs(smul(dp - dp_out, dwds), ws);
            g_sites[3 * e] = (out_t)daxis.x; g_sites[3 * e + 1] = (out_t)daxis.y; g_sites[3 * e + 2] = (out_t)daxis.z;
            g_temps[e] = (out_t)(dwdt * (dp - dp_out) / ws);
        }
    }
}

int FN(orc_num_threads)(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Ray-tracer adjoint.  The reference tracer (raytrace.py:115-241) has no   */
/* backward; this is the exact derivative of orc_trace_forward's colour,    */
/* log transmittance, depth and normal outputs with respect to every        */
/* primitive attribute.  Per ray the walk is repeated front to back; with   */
/* the forward's final colour C and normal N,                               */
/*   dL/d delta_k = gC.(C - C_<=k - c_k T_k+1) + gN.(N - N_<=k - n_k T_k+1)  */
/*                  + gL + [k < m] gD / sigma_m        (delta = -sigma dt)   */
/* where m is the segment that produced the depth.  dL/dt_near and          */
/* dL/dt_far go to the one surface that bounds each end of the segment      */
/* (sphere, power face or texture plane).  Face derivatives use the exact   */
/* spheres (the walk itself uses the float16 encoding, as the forward).     */
/* The texture plane's derivative includes every dependency of the local    */
/* variant (sites, colours, heights, plane origin and normal, the query     */
/* depth and the radius through 1/r^2).  Gradients accumulate into the     */
/* zeroed outputs (float atomics).                                          */

typedef struct {
    int hit;         /* contributes */
    int pre_hit;     /* sphere hit, tn <= tf, sigma >= 1e-3 (before the texture plane) */
    real tn, tf, dt; /* final segment */
    int tn_id, tf_id, pre_tn_id, pre_tf_id; /* -2 none, -1 sphere, k face, n_adj plane */
    real pre_tn;     /* t_near before the plane (query depth of the texture) */
    plane_res pr;
    int32_t next;
    real sigma;
    v3 center, pn;
    real radius;
} trace_seg;

/* one step of the walk at cell `prim`; mirrors orc_trace_forward */
static void trace_step(v3 o, v3 d, const float *spheres, const float *nsigmas, const float *sites, const float *rgbs,
                       const float *heights, int S, const int32_t *adj, const int32_t *adj_off,
                       const uint16_t *adj_diff, int32_t prim, trace_seg *sg) {
    const float *sp = spheres + 4 * (int64_t)prim;
    v3 center = ld3(sp);
    real radius = (real)sp[3];
    real tn, tf;
    int hit = ray_sphere(o, d, center, radius, &tn, &tf);
    v3 v = vsub(center, o);
    if (length(v) < K(4.0) * radius) hit = 0;
    int tn_id = tn < K(1e-8) ? -2 : -1, tf_id = tf < K(1e-8) ? -2 : -1;
    int32_t next = NO_CELL;
    real pt_far = K(1e10);
    int32_t a0 = adj_off[prim], a1 = adj_off[prim + 1];
    for (int32_t e = a0; e < a1; e++) {
        v3 diff;
        real pm;
        nbr_pm(spheres, adj, adj_diff, prim, e, &diff, &pm);
        real dp;
        real t_face = ray_pface_diff(o, d, diff, pm, &dp);
        if (dp >= K(0.0) && t_face < pt_far) { next = adj[e]; pt_far = t_face; }
        if (dp >= K(0.0) && t_face < tf) tf_id = e - a0;
        tf = dp >= K(0.0) ? rmin(t_face, tf) : tf;
        if (dp < K(0.0) && t_face > tn) tn_id = e - a0;
        tn = dp < K(0.0) ? rmax(t_face, tn) : tn;
    }
    const float *ns = nsigmas + 4 * (int64_t)prim;
    v3 pn = ld3(ns);
    real sigma = (real)ns[3];
    sg->next = next;
    sg->sigma = sigma;
    sg->center = center;
    sg->pn = pn;
    sg->radius = radius;
    sg->hit = 0;
    sg->pre_hit = 0;
    if (!hit || tn > tf || sigma < K(1e-3)) return;
    sg->pre_hit = 1;
    sg->pre_tn = tn;
    sg->pre_tn_id = tn_id;
    sg->pre_tf_id = tf_id;
    plane_res pr = plane_fwd_local(o, d, tn, center, pn, radius, sites + (int64_t)prim * S * 3,
                                   rgbs + (int64_t)prim * S * 3, heights + (int64_t)prim * S, S);
    int n_adj = a1 - a0;
    if (pr.dp >= K(0.0) && pr.t_surf < tf) tf_id = n_adj;
    tf = pr.dp >= K(0.0) ? rmin(pr.t_surf, tf) : tf;
    if (pr.dp < K(0.0) && pr.t_surf > tn) tn_id = n_adj;
    tn = pr.dp < K(0.0) ? rmax(pr.t_surf, tn) : tn;
    sg->pr = pr;
    sg->tn = tn;
    sg->tf = tf;
    sg->tn_id = tn_id;
    sg->tf_id = tf_id;
    sg->dt = tf - tn;
    sg->hit = sg->dt > K(0.0);
}

static void add3(float *g, v3 v) {
    ATOMIC_ADD(g[0], v.x);
    ATOMIC_ADD(g[1], v.y);
    ATOMIC_ADD(g[2], v.z);
}

/* derivative of the local texture plane (rasterize.py:62-137 / raytrace.py:
 * 42-113) for upstream dL/drgb and dL/dt_surf; returns dL/d(pre-plane
 * t_near) and accumulates into the primitive's gradients */
static real plane_local_bwd(v3 o, v3 d, real tn, v3 po, v3 pn, real radius, const float *sites, const float *rgbs,
                            const float *heights, int S, const plane_res *pr, v3 g_rgb, real g_tsurf, v3 *g_po,
                            v3 *g_pn, real *g_radius, float *gs, float *gr, float *gh) {
    real inv_r2 = K(1.0) / (radius * radius);
    real g_inv_r2 = 0, g_tn = 0;
    /* colour pass at pt */
    real tq = pr->dp >= K(0.0) ? tn : rmax(tn, pr->t_surf);
    v3 pt = vadd(o, smul(tq, d));
    real V = pr->wsum; /* already clamped */
    int vclamp = !(pr->wsum > K(1e-20)) ? 0 : 1;
    v3 g_pt = mk(0, 0, 0);
    for (int i = 0; i < S; i++) {
        v3 s = ld3(sites + 3 * i);
        v3 df = vsub(pt, s);
        real q2 = dot(df, df);
        real vi = r_exp(-TEMP * q2 * inv_r2);
        v3 ci = ld3(rgbs + 3 * i);
        v3 gci = smul(vi / V, g_rgb);
        ATOMIC_ADD(gr[3 * i + 0], gci.x);
        ATOMIC_ADD(gr[3 * i + 1], gci.y);
        ATOMIC_ADD(gr[3 * i + 2], gci.z);
        real g_vi = vclamp ? dot(vsub(ci, pr->rgb), g_rgb) / V : dot(ci, g_rgb) / V;
        /* dv/dpt = v (-2 T inv_r2) (pt - s) */
        v3 dvdpt = smul(vi * (-K(2.0) * TEMP * inv_r2), df);
        g_pt = vadd(g_pt, smul(g_vi, dvdpt));
        v3 gsi = smul(-g_vi, dvdpt);
        ATOMIC_ADD(gs[3 * i + 0], gsi.x);
        ATOMIC_ADD(gs[3 * i + 1], gsi.y);
        ATOMIC_ADD(gs[3 * i + 2], gsi.z);
        g_inv_r2 += g_vi * vi * (-TEMP * q2);
    }
    real g_tq = dot(g_pt, d);
    real g_tsurf_all = g_tsurf;
    if (pr->dp >= K(0.0) || tn > pr->t_surf) g_tn += g_tq;
    else g_tsurf_all += g_tq;
    /* t_surf = (dot(po - o, pn) + height) / dp */
    real g_height = 0;
    if (g_tsurf_all != K(0.0)) {
        real k = g_tsurf_all / pr->dp;
        *g_po = vadd(*g_po, smul(k, pn));
        *g_pn = vadd(*g_pn, smul(k, vsub(vsub(po, o), smul(pr->t_surf, d))));
        g_height = k;
    }
    /* height pass at _pt */
    real _tq = pr->_dp >= K(0.0) ? tn : rmax(tn, pr->_t_surf);
    v3 _pt = vadd(o, smul(_tq, d));
    real W = pr->_wsum;
    int wclamp = pr->_wsum > K(1e-20);
    v3 g__pt = mk(0, 0, 0);
    if (g_height != K(0.0)) {
        for (int i = 0; i < S; i++) {
            v3 s = ld3(sites + 3 * i);
            v3 df = vsub(_pt, s);
            real q2 = dot(df, df);
            real wi = r_exp(-TEMP * q2 * inv_r2);
            real hi = (real)heights[i];
            ATOMIC_ADD(gh[i], wi / W * g_height);
            real g_wi = wclamp ? (hi - pr->height) / W * g_height : hi / W * g_height;
            v3 dwdpt = smul(wi * (-K(2.0) * TEMP * inv_r2), df);
            g__pt = vadd(g__pt, smul(g_wi, dwdpt));
            v3 gsi = smul(-g_wi, dwdpt);
            ATOMIC_ADD(gs[3 * i + 0], gsi.x);
            ATOMIC_ADD(gs[3 * i + 1], gsi.y);
            ATOMIC_ADD(gs[3 * i + 2], gsi.z);
            g_inv_r2 += g_wi * wi * (-TEMP * q2);
        }
    }
    real g__tq = dot(g__pt, d);
    if (g__tq != K(0.0)) {
        if (pr->_dp >= K(0.0) || tn > pr->_t_surf) {
            g_tn += g__tq;
        } else {
            real k = g__tq / pr->_dp;
            *g_po = vadd(*g_po, smul(k, pn));
            *g_pn = vadd(*g_pn, smul(k, vsub(vsub(po, o), smul(pr->_t_surf, d))));
        }
    }
    *g_radius += g_inv_r2 * (-K(2.0) / (radius * radius * radius));
    return g_tn;
}

/* d t / d (centre, radius) of the near (sign -1) or far (+1) sphere root:
 * t = (-qb -+ s)/2, qb = 2 oc.d, s = sqrt(qb^2 - 4 (|oc|^2 - r^2)), oc = o - c */
static void sphere_root_grad(v3 o, v3 d, v3 c, real r, int far, v3 *dc, real *dr) {
    v3 oc = vsub(o, c);
    real qb = K(2.0) * dot(oc, d);
    real qc = dot(oc, oc) - r * r;
    real s = r_sqrt(qb * qb - K(4.0) * qc);
    /* d disc / dc = -4 qb d + 8 oc */
    v3 ddisc = vadd(smul(-K(4.0) * qb, d), smul(K(8.0), oc));
    v3 ds = smul(K(1.0) / (K(2.0) * s), ddisc);
    real sg = far ? K(1.0) : K(-1.0);
    *dc = vadd(d, smul(sg * K(0.5), ds));
    *dr = sg * K(2.0) * r / s;
}

/* d t / d (c_i, r_i, c_j, r_j) of the power face between i and j */
static void face_grad(v3 o, v3 d, v3 ci, real ri, v3 cj, real rj, v3 *dci, real *dri, v3 *dcj, real *drj) {
    v3 n = vsub(cj, ci);
    real num = K(0.5) * (dot(cj, cj) - rj * rj - dot(ci, ci) + ri * ri) - dot(o, n);
    real den = dot(d, n);
    real t = num / den;
    *dci = smul(K(1.0) / den, vadd(vsub(o, ci), smul(t, d)));
    *dcj = smul(K(1.0) / den, vsub(vsub(cj, o), smul(t, d)));
    *dri = ri / den;
    *drj = -rj / den;
}

int FN(orc_trace_backward)(const orc_camera *camera, const float *spheres, const float *nsigmas, const float *sites,
                           const float *rgbs, const float *heights, int S, const int32_t *adj, const int32_t *adj_off,
                           const uint16_t *adj_diff, int32_t start_idx, const int32_t *start_cells, float thr,
                           int max_steps, float depth_quantile, const out_t *color, const out_t *normal,
                           const int32_t *depth_seg, const out_t *depth_sigma, const float *g_color,
                           const float *g_log_t, const float *g_depth, const float *g_normal, float *g_spheres,
                           float *g_nsigmas, float *g_sites, float *g_rgb, float *g_height) {
    cam_t cam = cam_load(camera);
    int64_t P = (int64_t)cam.H * cam.W;
    v3 o = cam.eye;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t px = 0; px < P; px++) {
        int pi = (int)(px / cam.W), pj = (int)(px % cam.W);
        v3 rd = get_ray_dir(&cam, (real)pi, (real)pj);
        v3 d = vdivs(rd, length(rd));
        v3 gC = g_color ? ld3(g_color + 3 * px) : mk(0, 0, 0);
        v3 gN = g_normal ? ld3(g_normal + 3 * px) : mk(0, 0, 0);
        real gL = g_log_t ? (real)g_log_t[px] : 0;
        real gD = g_depth ? (real)g_depth[px] : 0;
        int m = depth_seg ? depth_seg[px] : -1;
        real sig_m = depth_sigma ? (real)depth_sigma[px] : 1;
        v3 Cf = mk((real)color[3 * px], (real)color[3 * px + 1], (real)color[3 * px + 2]);
        v3 Nf = normal ? mk((real)normal[3 * px], (real)normal[3 * px + 1], (real)normal[3 * px + 2]) : mk(0, 0, 0);
        v3 Cacc = mk(0, 0, 0), Nacc = mk(0, 0, 0);
        real log_t = 0;
        int32_t prim = start_cells ? start_cells[px] : start_idx;
        int steps = 0, seg = 0;
        int32_t cg_saved = -1;
        int cg_hit = 0;
        for (;;) {
            real trans = r_exp(log_t);
            if (trans < (real)thr || prim == NO_CELL || steps >= max_steps) break;
            if (cycle_closed(&cg_saved, &cg_hit, prim, steps)) break;
            steps++;
            trace_seg sg;
            trace_step(o, d, spheres, nsigmas, sites, rgbs, heights, S, adj, adj_off, adj_diff, prim, &sg);
            int32_t cur = prim;
            prim = sg.next;
            if (sg.pre_hit) cg_hit = 1;
            if (!sg.hit) continue;
            real sigma = sg.sigma, dt = sg.dt;
            real dlt = -sigma * dt;
            real e = r_exp(dlt);
            real alpha = K(1.0) - e;
            v3 c = sg.pr.rgb;
            Cacc = vadd(Cacc, smul(trans, smul(alpha, c)));
            Nacc = vadd(Nacc, smul(alpha * trans, sg.pn));
            real trans_next = trans * e;
            real g_delta = dot(gC, vsub(vsub(Cf, Cacc), smul(trans_next, c))) +
                           dot(gN, vsub(vsub(Nf, Nacc), smul(trans_next, sg.pn))) + gL;
            if (m >= 0 && seg < m) g_delta += gD / sig_m;
            real g_sigma = -dt * g_delta;
            real g_tf = -sigma * g_delta, g_tn = sigma * g_delta;
            if (seg == m) {
                g_tn += gD;
                g_sigma += -gD * r_log(trans / (real)depth_quantile) / (sigma * sigma);
            }
            v3 g_c = smul(alpha * trans, gC);
            v3 g_pn = smul(alpha * trans, gN);
            v3 g_po = mk(0, 0, 0);
            real g_r = 0;
            int n_adj = adj_off[cur + 1] - adj_off[cur];
            /* the plane bounds at most one end */
            real g_tsurf = 0;
            if (sg.tn_id == n_adj) { g_tsurf += g_tn; g_tn = 0; }
            if (sg.tf_id == n_adj) { g_tsurf += g_tf; g_tf = 0; }
            real g_pre_tn = plane_local_bwd(o, d, sg.pre_tn, sg.center, sg.pn, sg.radius,
                                            sites + (int64_t)cur * S * 3, rgbs + (int64_t)cur * S * 3,
                                            heights + (int64_t)cur * S, S, &sg.pr, g_c, g_tsurf, &g_po, &g_pn, &g_r,
                                            g_sites + (int64_t)cur * S * 3, g_rgb + (int64_t)cur * S * 3,
                                            g_height + (int64_t)cur * S);
            if (sg.tn_id != n_adj) g_tn += g_pre_tn;
            else g_pre_tn = g_pre_tn; /* query depth is the pre-plane t_near */
            real g_ends[2] = {sg.tn_id == n_adj ? g_pre_tn : g_tn, g_tf};
            int ids[2] = {sg.tn_id == n_adj ? sg.pre_tn_id : sg.tn_id, sg.tf_id};
            v3 g_center = g_po;
            for (int i = 0; i < 2; i++) {
                real gt = g_ends[i];
                int id = ids[i];
                if (gt == K(0.0)) continue;
                if (id == -1) {
                    v3 dc;
                    real dr;
                    sphere_root_grad(o, d, sg.center, sg.radius, i == 1, &dc, &dr);
                    g_center = vadd(g_center, smul(gt, dc));
                    g_r += gt * dr;
                } else if (id >= 0 && id < n_adj) {
                    int32_t nb = adj[adj_off[cur] + id];
                    const float *ns = spheres + 4 * (int64_t)nb;
                    v3 dci, dcj;
                    real dri, drj;
                    face_grad(o, d, sg.center, sg.radius, ld3(ns), (real)ns[3], &dci, &dri, &dcj, &drj);
                    g_center = vadd(g_center, smul(gt, dci));
                    g_r += gt * dri;
                    add3(g_spheres + 4 * (int64_t)nb, smul(gt, dcj));
                    ATOMIC_ADD(g_spheres[4 * (int64_t)nb + 3], gt * drj);
                }
            }
            add3(g_spheres + 4 * (int64_t)cur, g_center);
            ATOMIC_ADD(g_spheres[4 * (int64_t)cur + 3], g_r);
            add3(g_nsigmas + 4 * (int64_t)cur, g_pn);
            ATOMIC_ADD(g_nsigmas[4 * (int64_t)cur + 3], g_sigma);
            log_t += dlt;
            seg++;
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Čech adjacency (powerfoam/bvh.py:7-69 predicate, build_cech_complex       */
/* bvh.py:96-123): j is a neighbour of i (j != i) when the AABBs of the two   */
/* balls overlap (the BVH query) and |c_i - c_j| < r_i + r_j, with c and r    */
/* recomputed from the AABB as the reference's bvh_query does.  Lists are     */
/* ascending.  Candidates come from a uniform grid of cell edge >= 2 max r,   */
/* so every overlapping pair lies in adjacent cells; the grid only prunes, it  */
/* never decides.  Two calls: adjacency NULL -> counts only (offsets filled,  */
/* *n_edges set); then with adjacency of *n_edges entries.                   */
#ifndef PF_F64
typedef struct { float lo[3], hi[3], c[3], r; } cech_ball;

static cech_ball cech_make(const float *pts, const float *radii, int64_t i) {
    cech_ball b;
    float r = radii[i];
    for (int k = 0; k < 3; k++) {
        float p = pts[3 * i + k];
        b.lo[k] = p - r;
        b.hi[k] = p + r;
    }
    for (int k = 0; k < 3; k++) b.c[k] = 0.5f * (b.lo[k] + b.hi[k]);
    b.r = 0.5f * (b.hi[0] - b.lo[0]);
    return b;
}

static int cech_overlap(const cech_ball *a, const cech_ball *b) {
    for (int k = 0; k < 3; k++)
        if (!(a->lo[k] <= b->hi[k] && a->hi[k] >= b->lo[k])) return 0;
    float dx = a->c[0] - b->c[0], dy = a->c[1] - b->c[1], dz = a->c[2] - b->c[2];
    float d = sqrtf((dx * dx + dy * dy) + dz * dz);
    return d < a->r + b->r;
}

static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

int orc_cech_adjacency_f32(const float *pts, const float *radii, int64_t N, int32_t *offsets, int32_t *adjacency,
                           int64_t *n_edges) {
    if (N <= 0) {
        offsets[0] = 0;
        *n_edges = 0;
        return ORC_OK;
    }
    float lo[3] = {pts[0], pts[1], pts[2]}, hi[3] = {pts[0], pts[1], pts[2]}, rmax = 0.0f;
    for (int64_t i = 0; i < N; i++) {
        for (int k = 0; k < 3; k++) {
            float v = pts[3 * i + k];
            lo[k] = v < lo[k] ? v : lo[k];
            hi[k] = v > hi[k] ? v : hi[k];
        }
        rmax = radii[i] > rmax ? radii[i] : rmax;
    }
    double h = 2.0 * (double)rmax * 1.0001 + 1e-12;
    int n[3];
    for (;;) {
        int ok = 1;
        for (int k = 0; k < 3; k++) {
            double c = floor(((double)hi[k] - (double)lo[k]) / h) + 1.0;
            n[k] = c > 1024.0 ? 1025 : (int)c;
            if (n[k] > 1024) ok = 0;
        }
        if (ok && (int64_t)n[0] * n[1] * n[2] <= (int64_t)1 << 26) break;
        h *= 1.5;
    }
    int64_t ncell = (int64_t)n[0] * n[1] * n[2];
    int64_t *cell_of = (int64_t *)malloc(sizeof(int64_t) * N);
    int64_t *start = (int64_t *)calloc(ncell + 1, sizeof(int64_t));
    int64_t *sorted = (int64_t *)malloc(sizeof(int64_t) * N);
    if (!cell_of || !start || !sorted) {
        free(cell_of);
        free(start);
        free(sorted);
        return ORC_ERR_ARGS;
    }
    for (int64_t i = 0; i < N; i++) {
        int64_t cc[3];
        for (int k = 0; k < 3; k++) {
            int64_t c = (int64_t)floor(((double)pts[3 * i + k] - (double)lo[k]) / h);
            cc[k] = c < 0 ? 0 : (c >= n[k] ? n[k] - 1 : c);
        }
        cell_of[i] = (cc[2] * n[1] + cc[1]) * n[0] + cc[0];
        start[cell_of[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) start[c + 1] += start[c];
    {
        int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (ncell + 1));
        memcpy(fill, start, sizeof(int64_t) * (ncell + 1));
        for (int64_t i = 0; i < N; i++) sorted[fill[cell_of[i]]++] = i;
        free(fill);
    }
    int32_t *counts = adjacency ? NULL : offsets; /* pass 1 counts into offsets[1..N] */
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : bad)
    for (int64_t i = 0; i < N; i++) {
        cech_ball bi = cech_make(pts, radii, i);
        int64_t ci = cell_of[i];
        int64_t cx = ci % n[0], cy = (ci / n[0]) % n[1], cz = ci / ((int64_t)n[0] * n[1]);
        int64_t pos = adjacency ? offsets[i] : 0;
        int32_t cnt = 0;
        for (int64_t z = cz - 1; z <= cz + 1; z++) {
            if (z < 0 || z >= n[2]) continue;
            for (int64_t y = cy - 1; y <= cy + 1; y++) {
                if (y < 0 || y >= n[1]) continue;
                for (int64_t x = cx - 1; x <= cx + 1; x++) {
                    if (x < 0 || x >= n[0]) continue;
                    int64_t c = (z * n[1] + y) * n[0] + x;
                    for (int64_t s = start[c]; s < start[c + 1]; s++) {
                        int64_t j = sorted[s];
                        if (j == i) continue;
                        cech_ball bj = cech_make(pts, radii, j);
                        if (cech_overlap(&bi, &bj)) {
                            if (adjacency) adjacency[pos + cnt] = (int32_t)j;
                            cnt++;
                        }
                    }
                }
            }
        }
        if (adjacency) {
            if (cnt != offsets[i + 1] - offsets[i]) bad = 1;
            qsort(adjacency + pos, (size_t)cnt, sizeof(int32_t), cmp_i32);
        } else {
            counts[i + 1] = cnt;
        }
    }
    if (!adjacency) {
        offsets[0] = 0;
        int64_t total = 0;
        for (int64_t i = 0; i < N; i++) {
            total += offsets[i + 1];
            offsets[i + 1] = (int32_t)total;
        }
        *n_edges = total;
    } else {
        *n_edges = offsets[N];
    }
    free(cell_of);
    free(start);
    free(sorted);
    return bad ? ORC_ERR_ARGS : ORC_OK;
}
#endif

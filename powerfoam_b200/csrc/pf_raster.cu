// pf_raster.cu -- tile compositing forward / adjoint, benchmark and viewer
// variants, neighbour encodings.
//
// Work decomposition (forward and adjoint): a tile of TW x TW pixels is owned
// by G = TW*TW/64 warps; every lane owns two pixels of the tile.  The
// reference's block-wide tile_max (early termination) and tile_sum (any hit)
// become one warp vote for TW = 8 and one __syncthreads_and/or for TW = 16,
// 32.  Each warp stages the tile's primitive records (sphere, normal+sigma)
// 32 at a time in shared memory, turns the neighbours of the current
// primitive into face planes (n, num) cooperatively (one neighbour per lane)
// and stages the primitive's texel records once per primitive.  Per-primitive
// gradients of the adjoint are summed over the warp's 64 pixels with a
// reduce-scatter (62 shuffles) before one atomic per value, instead of one
// atomic per pixel and value.
#include <algorithm>

#include "pf_common.cuh"
#include "pf_raster_common.cuh"
#include "pf_api.h"

namespace pf {

// ---------------------------------------------------------------------------
// benchmark / viewer variants: per-pixel early-out, no tile collectives
// (rasterize.py:614-734 and :738-888); one thread per pixel, 64 per tile.
template <typename A>
PF_D float ldA(const A* p, int64_t i);
template <>
PF_D float ldA<float>(const float* p, int64_t i) { return __ldg(p + i); }
template <>
PF_D float ldA<__half>(const __half* p, int64_t i) { return __half2float(p[i]); }

template <typename A>
PF_D PlaneRes plane_fwd_local_g(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const A* sites, const A* rgbs,
                                const A* heights, int S) {
    PlaneRes r;
    float _dp;
    float _t_surf = ray_plane(o, d, po, pn, 0.0f, _dp);
    float _tq = _dp >= 0.0f ? t_near : fmax_t(t_near, _t_surf);
    v3 _pt = o + _tq * d;
    float inv_r2 = 1.0f / (radius * radius);
    float hsum = 0.f, _wsum = 0.f;
    for (int i = 0; i < S; i++) {
        v3 df = _pt - mk(ldA(sites, 3 * i), ldA(sites, 3 * i + 1), ldA(sites, 3 * i + 2));
        float dist_sq = dot(df, df) * inv_r2;
        float w = expf(-kTemp * dist_sq);
        hsum += w * ldA(heights, i);
        _wsum += w;
    }
    _wsum = fmax_t(_wsum, 1e-20f);
    float height = hsum / _wsum;
    float dp;
    float t_surf = ray_plane(o, d, po, pn, height, dp);
    float tq = dp >= 0.0f ? t_near : fmax_t(t_near, t_surf);
    v3 pt = o + tq * d;
    v3 rgb_sum = mk(0.f, 0.f, 0.f);
    float wsum = 0.f;
    for (int i = 0; i < S; i++) {
        v3 df = pt - mk(ldA(sites, 3 * i), ldA(sites, 3 * i + 1), ldA(sites, 3 * i + 2));
        float dist_sq = dot(df, df) * inv_r2;
        float w = expf(-kTemp * dist_sq);
        rgb_sum = rgb_sum + w * mk(ldA(rgbs, 3 * i), ldA(rgbs, 3 * i + 1), ldA(rgbs, 3 * i + 2));
        wsum += w;
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

template <typename A>
PF_D void load_nsig(const void* nsig, int64_t p, v3& n, float& sigma) {
    const A* q = (const A*)nsig + 4 * p;
    n = mk(ldA(q, 0), ldA(q, 1), ldA(q, 2));
    sigma = ldA(q, 3);
}

// VIS = false: benchmark_kernel; VIS = true: visualization_kernel
template <typename A, bool VIS>
__global__ void __launch_bounds__(256)
raster_pixel_kernel(RasterParams P, const void* nsig, const A* sites, const A* rgbs, const A* heights,
                    int max_inter, float depth_q, v3 bkgd, float* __restrict__ color, float* __restrict__ depth,
                    float* __restrict__ normal, float* __restrict__ alpha_out, int32_t* __restrict__ inter_out) {
    const int TS = P.TW * P.TW;
    int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t tile = tid / TS;
    if (tile >= P.T) return;
    int idx = (int)(tid % TS);
    PixGeom g = pixel_geom(P, tile, idx);
    const v3 o = P.cam.eye;
    const v3 d = g.d;
    v3 rgb = mk(0.f, 0.f, 0.f), nacc = mk(0.f, 0.f, 0.f);
    float dq_out = 0.f;
    bool dq_found = false;
    float log_t = 0.f;
    int n_hit = 0;
    const int64_t start = P.tile_off[tile];
    const int total = (int)(P.tile_off[tile + 1] - start);
    for (int k = 0; k < total; k++) {
        if (VIS) {
            n_hit += 1;
            if (k >= max_inter) break;
        }
        const int32_t prim = __ldg(&P.tile_prims[start + k]);
        float trans = expf(log_t);
        if (trans < P.thr) break;
        const float4 s4 = __ldg(&P.spheres[prim]);
        const v3 center = mk(s4.x, s4.y, s4.z);
        const float radius = s4.w;
        float tn, tf;
        bool hit = ray_sphere(o, d, center, radius, tn, tf);
        if (!hit) continue;
        const int32_t a0 = __ldg(&P.adj_off[prim]), a1 = __ldg(&P.adj_off[prim + 1]);
        const float cc = dot(center, center), rr = radius * radius;
        for (int32_t e = a0; e < a1; e++) {
            uint2 raw = __ldg(&P.adj_diff[e]);
            v3 diff = mk(h2f((uint16_t)(raw.x & 0xffffu)), h2f((uint16_t)(raw.x >> 16)), h2f((uint16_t)(raw.y & 0xffffu)));
            float w4 = h2f((uint16_t)(raw.y >> 16));
            Face f = VIS ? make_face(o, center, cc, rr, center + diff, w4) : make_face_pm(o, diff, w4);
            float dp = dot(d, f.n);
            float t_face = f.num / dp;
            tf = dp >= 0.0f ? fmin_t(t_face, tf) : tf;
            tn = dp < 0.0f ? fmax_t(t_face, tn) : tn;
            if (tn > tf) break;
        }
        if (tn > tf) continue;
        v3 pn;
        float sigma;
        load_nsig<A>(nsig, prim, pn, sigma);
        int64_t b3 = (int64_t)prim * P.S * 3;
        PlaneRes pr = plane_fwd_local_g<A>(o, d, tn, center, pn, radius, sites + b3, rgbs + b3,
                                           heights + (int64_t)prim * P.S, P.S);
        tf = pr.dp >= 0.0f ? fmin_t(pr.t_surf, tf) : tf;
        tn = pr.dp < 0.0f ? fmax_t(pr.t_surf, tn) : tn;
        float dt = tf - tn;
        if (dt > 0.0f) {
            float dlt = -sigma * dt;
            float alpha = 1.0f - expf(dlt);
            trans = expf(log_t);
            rgb = rgb + trans * (alpha * pr.rgb);
            if (VIS) nacc = nacc + trans * (alpha * pn);
            log_t += dlt;
            if (VIS && !dq_found) {
                float next_trans = expf(log_t);
                if (next_trans < depth_q) {
                    dq_out = tn + logf(trans / depth_q) / sigma;
                    dq_found = true;
                }
            }
        }
    }
    if (g.oob) return;
    int64_t p = g.px;
    if (VIS) {
        float ray_trans = expf(log_t);
        float ray_alpha = 1.0f - ray_trans;
        rgb = rgb + ray_trans * bkgd;
        depth[p] = dq_out;
        normal[3 * p] = nacc.x;
        normal[3 * p + 1] = nacc.y;
        normal[3 * p + 2] = nacc.z;
        alpha_out[p] = ray_alpha;
        inter_out[p] = n_hit;
    }
    color[3 * p] = rgb.x;
    color[3 * p + 1] = rgb.y;
    color[3 * p + 2] = rgb.z;
}

// ---------------------------------------------------------------------------
// neighbour encodings
__global__ void prefetch_adjacency_kernel(const float4* __restrict__ spheres, const int32_t* __restrict__ adj,
                                          const int32_t* __restrict__ adj_off, int64_t N, uint2* __restrict__ out) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    float4 s = spheres[p];
    for (int32_t e = adj_off[p]; e < adj_off[p + 1]; e++) {
        float4 t = __ldg(&spheres[adj[e]]);
        uint32_t h0 = __half_as_ushort(__float2half_rn(t.x - s.x));
        uint32_t h1 = __half_as_ushort(__float2half_rn(t.y - s.y));
        uint32_t h2 = __half_as_ushort(__float2half_rn(t.z - s.z));
        uint32_t h3 = __half_as_ushort(__float2half_rn(t.w));
        out[e] = make_uint2(h0 | (h1 << 16), h2 | (h3 << 16));
    }
}

// benchmark.py:296-302; pm = 0.5 * (norm(p) ** 2 - r ** 2), norm as sqrt of
// the sum of squares in index order
__global__ void power_diff_kernel(const float* __restrict__ pts, const float* __restrict__ radii,
                                  const int32_t* __restrict__ adj, const int32_t* __restrict__ adj_off, int64_t N,
                                  uint2* __restrict__ out) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    v3 c = mk(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]);
    float n = sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
    float pm_i = 0.5f * (n * n - radii[p] * radii[p]);
    for (int32_t e = adj_off[p]; e < adj_off[p + 1]; e++) {
        int64_t q = adj[e];
        v3 cq = mk(pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]);
        float m = sqrtf(cq.x * cq.x + cq.y * cq.y + cq.z * cq.z);
        float pm_j = 0.5f * (m * m - radii[q] * radii[q]);
        uint32_t h0 = __half_as_ushort(__float2half_rn(cq.x - c.x));
        uint32_t h1 = __half_as_ushort(__float2half_rn(cq.y - c.y));
        uint32_t h2 = __half_as_ushort(__float2half_rn(cq.z - c.z));
        uint32_t h3 = __half_as_ushort(__float2half_rn(pm_j - pm_i));
        out[e] = make_uint2(h0 | (h1 << 16), h2 | (h3 << 16));
    }
}

}  // namespace pf

using namespace pf;

template <bool VIS>
static int launch_pixel(const pf_raster_inputs* in, int max_inter, float depth_q, v3 bkgd, float* color,
                        float* depth, float* normal, float* alpha, int32_t* inter, cudaStream_t st) {
    RasterParams P;
    const char* why = "";
    if (!fill_params(in, P, false, &why)) return pf_fail(PF_ERR_ARGS, why);
    int64_t threads = P.T * P.TW * P.TW;
    if (threads == 0) return PF_OK;
    unsigned grid = (unsigned)((threads + 255) / 256);
    if (in->attr_half) {
        raster_pixel_kernel<__half, VIS><<<grid, 256, 0, st>>>(P, in->nsigmas, (const __half*)in->texel_sites,
                                                               (const __half*)in->texel_rgb,
                                                               (const __half*)in->texel_height, max_inter, depth_q,
                                                               bkgd, color, depth, normal, alpha, inter);
    } else {
        raster_pixel_kernel<float, VIS><<<grid, 256, 0, st>>>(P, in->nsigmas, (const float*)in->texel_sites,
                                                              (const float*)in->texel_rgb,
                                                              (const float*)in->texel_height, max_inter, depth_q, bkgd,
                                                              color, depth, normal, alpha, inter);
    }
    return pf_check_launch(VIS ? "pf_raster_visualize" : "pf_raster_benchmark");
}

extern "C" int pf_raster_benchmark(const pf_raster_inputs* in, float* color, void* stream) {
    if (!color) return pf_fail(PF_ERR_ARGS, "pf_raster_benchmark: missing output");
    return launch_pixel<false>(in, 0, 0.f, mk(0.f, 0.f, 0.f), color, nullptr, nullptr, nullptr, nullptr,
                               (cudaStream_t)stream);
}

extern "C" int pf_raster_visualize(const pf_raster_inputs* in, int32_t max_intersections, float depth_quantile,
                                   float bkgd_r, float bkgd_g, float bkgd_b, float* color, float* depth, float* normal,
                                   float* alpha, int32_t* intersections, void* stream) {
    if (!color || !depth || !normal || !alpha || !intersections)
        return pf_fail(PF_ERR_ARGS, "pf_raster_visualize: missing output");
    return launch_pixel<true>(in, max_intersections, depth_quantile, mk(bkgd_r, bkgd_g, bkgd_b), color, depth, normal,
                              alpha, intersections, (cudaStream_t)stream);
}

extern "C" int pf_adjacency_prefetch(const float* spheres, const int32_t* adjacency, const int32_t* adjacency_offsets,
                                     int64_t n_prims, uint16_t* adjacency_diff, void* stream) {
    if (n_prims < 0 || (n_prims > 0 && (!spheres || !adjacency_offsets)))
        return pf_fail(PF_ERR_ARGS, "pf_adjacency_prefetch: bad arguments");
    if (n_prims == 0) return PF_OK;
    prefetch_adjacency_kernel<<<(unsigned)((n_prims + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const float4*)spheres, adjacency, adjacency_offsets, n_prims, (uint2*)adjacency_diff);
    return pf_check_launch("pf_adjacency_prefetch");
}

extern "C" int pf_adjacency_power_diff(const float* points, const float* radii, const int32_t* adjacency,
                                       const int32_t* adjacency_offsets, int64_t n_prims, uint16_t* adjacency_diff,
                                       void* stream) {
    if (n_prims < 0 || (n_prims > 0 && (!points || !radii || !adjacency_offsets)))
        return pf_fail(PF_ERR_ARGS, "pf_adjacency_power_diff: bad arguments");
    if (n_prims == 0) return PF_OK;
    power_diff_kernel<<<(unsigned)((n_prims + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        points, radii, adjacency, adjacency_offsets, n_prims, (uint2*)adjacency_diff);
    return pf_check_launch("pf_adjacency_power_diff");
}

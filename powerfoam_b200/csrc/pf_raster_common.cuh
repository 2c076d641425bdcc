// pf_raster_common.cuh -- parameters, pixel mapping and per-warp staging
// shared by the rasterizer kernels.
#pragma once
#include "pf_common.cuh"

namespace pf {

constexpr int kWarpsPerBlock8 = 4;  // TW = 8: four tiles per 128-thread block

struct RasterParams {
    Cam cam;
    int TW, S, Q;
    int64_t N, T;
    int tiles_h;
    const float4* spheres;
    const float4* nsigmas;
    const float* sites;   // (N,S,3)
    const float* rgb;     // (N,S,3)
    const float* height;  // (N,S)
    const int32_t* adj;
    const int32_t* adj_off;
    const uint2* adj_diff;  // (E) 4 x f16
    const int64_t* tile_off;
    const int32_t* tile_prims;
    const float* dq;   // (H,W,Q)
    const float* gt;   // (H,W,3)
    float thr;
    const int32_t* tile_order;  // processing order of the tiles (NULL: 0..T-1)
    int* queue;                 // work-queue counter (NULL: one group per tile)
    const float* ray_maps;      // (H,W,6) per-pixel origin, direction (generic camera) or NULL
    float4* seg;                // segment records, seg_stride float4 each, or NULL
    uint32_t* seg_mask;         // hit masks (pairs x TW^2 / 32)
    int32_t* seg_off;           // first record of each (pair, warp), -1: none (pairs x TW^2 / 32)
    unsigned long long* seg_count;  // records reserved
    int64_t seg_pairs;          // pairs the mask and offset arrays hold
    int64_t seg_cap;            // records the buffer holds
    int seg_stride;             // 4: the records hold the plane results (float4 1..3), 1: intervals only
};

// texture-plane result in float4 1..3 of a 64-byte record (the interval is
// float4 0): a pixel with a non-empty interval moves two whole 32-byte
// sectors, one with an empty interval the first only
PF_D void store_plane(float4* slot, const PlaneRes& r) {
    slot[1] = make_float4(r.rgb.x, r.rgb.y, r.rgb.z, r.height);
    slot[2] = make_float4(r.wsum, r._wsum, r.t_surf, r.dp);
    slot[3] = make_float4(r._t_surf, r._dp, 0.f, 0.f);
}
// Segment-record loads: through the read-only path when the records were
// written by an earlier launch, through L2 (ld.global.cg) when the forward
// that wrote them runs in the same launch (the read-only path is only valid
// for data that no thread writes during the launch).
// Bring `bytes` at `p` into L2 ahead of use (cp.async.bulk.prefetch, no
// registers written); skipped unless both are 16-byte multiples.
PF_D void prefetch_l2_bulk(const void* p, uint32_t bytes) {
    if (bytes != 0u && (((uintptr_t)p | bytes) & 15u) == 0)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <bool COH, class T>
PF_D T seg_load(const T* p) {
    if constexpr (COH) return __ldcg(p);
    else return __ldg(p);
}

template <bool COH = false>
PF_D PlaneRes load_plane(const float4* slot) {
    const float4 a = seg_load<COH>(slot + 1), b = seg_load<COH>(slot + 2), c = seg_load<COH>(slot + 3);
    PlaneRes r;
    r.rgb = mk(a.x, a.y, a.z);
    r.height = a.w;
    r.wsum = b.x;
    r._wsum = b.y;
    r.t_surf = b.z;
    r.dp = b.w;
    r._t_surf = c.x;
    r._dp = c.y;
    return r;
}

// segment record ids: the surfaces bounding a segment (-2 behind the eye, -1
// the sphere, else the face's place in the adjacency list), 16 bits each
PF_D float pack_seg_ids(int tn_id, int tf_id) {
    return __uint_as_float(((uint32_t)(tn_id + 2) & 0xffffu) | ((uint32_t)(tf_id + 2) << 16));
}
PF_D void unpack_seg_ids(float v, int& tn_id, int& tf_id) {
    const uint32_t u = __float_as_uint(v);
    tn_id = (int)(u & 0xffffu) - 2;
    tf_id = (int)(u >> 16) - 2;
}

// ---------------------------------------------------------------------------
// group collectives: G == 1 -> warp vote; G > 1 -> block barrier with reduction
template <int G>
PF_D bool group_all(bool p) {
    if constexpr (G == 1) return __all_sync(0xffffffffu, p);
    else return __syncthreads_and(p) != 0;
}
template <int G>
PF_D bool group_any(bool p) {
    if constexpr (G == 1) return __any_sync(0xffffffffu, p);
    else return __syncthreads_or(p) != 0;
}

struct PixGeom {
    v3 d;
    int64_t px;  // pixel index, valid when !oob
    bool oob;
};

PF_D PixGeom pixel_geom(const RasterParams& P, int64_t tile, int idx) {
    PixGeom g;
    int ti = (int)(tile % P.tiles_h), tj = (int)(tile / P.tiles_h);
    int i_in = idx % P.TW, j_in = idx / P.TW;
    int pi = ti * P.TW + i_in, pj = tj * P.TW + j_in;
    g.oob = pi >= P.cam.H || pj >= P.cam.W;
    pi = imin(pi, P.cam.H - 1);
    pj = imin(pj, P.cam.W - 1);
    g.d = ray_dir(P.cam, pi, pj);
    g.px = (int64_t)pi * P.cam.W + pj;
    return g;
}

// A generic camera's ray (rasterize.py:944-954): the pixel's own origin and
// its direction divided by its length.
PF_D void pixel_ray_map(const RasterParams& P, PixGeom& g, v3& o) {
    const float* m = P.ray_maps + 6 * g.px;
    o = mk(m[0], m[1], m[2]);
    const v3 rd = mk(m[3], m[4], m[5]);
    g.d = rd / length(rd);
}

// Per-warp shared staging area.
struct WarpStage {
    float4 sph[32];
    float4 nsg[32];
    int32_t pid[32];
    float4 face[32];
    float ts[3 * kMaxSites];
    float tr[3 * kMaxSites];
    float th[kMaxSites];
};

PF_D void stage_prims(WarpStage& ws, const RasterParams& P, int64_t start, int k0, int total, int lane) {
    int k = k0 + lane;
    if (k >= 0 && k < total) {
        int32_t p = P.tile_prims[start + k];
        ws.pid[lane] = p;
        ws.sph[lane] = __ldg(&P.spheres[p]);
        ws.nsg[lane] = __ldg(&P.nsigmas[p]);
    }
    __syncwarp();
}

// Asynchronous global -> shared copies (cp.async, 4 or 16 bytes, aligned to
// their size); cp_async_wait_all waits for this thread's copies only.
PF_D void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
PF_D void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
PF_D void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// stage_texels without waiting: the copies land after cp_async_wait_all and
// a __syncwarp
PF_D void stage_texels_async(WarpStage& ws, const RasterParams& P, int32_t prim, int lane) {
    const int S = P.S;
    int64_t b3 = (int64_t)prim * S * 3;
    if (lane < 3 * S) {
        cp_async4(&ws.ts[lane], &P.sites[b3 + lane]);
        cp_async4(&ws.tr[lane], &P.rgb[b3 + lane]);
    }
    if (lane < S) cp_async4(&ws.th[lane], &P.height[(int64_t)prim * S + lane]);
}

PF_D void stage_texels(WarpStage& ws, const RasterParams& P, int32_t prim, int lane) {
    const int S = P.S;
    int64_t b3 = (int64_t)prim * S * 3;
    if (lane < 3 * S) {
        ws.ts[lane] = __ldg(&P.sites[b3 + lane]);
        ws.tr[lane] = __ldg(&P.rgb[b3 + lane]);
    }
    if (lane < S) ws.th[lane] = __ldg(&P.height[(int64_t)prim * S + lane]);
    __syncwarp();
}

// faces e0..e0+31 of the current primitive -> ws.face (n.xyz, num)
PF_D void stage_faces(WarpStage& ws, const RasterParams& P, int32_t a0, int e0, int n_adj, v3 eye, v3 center,
                      float cc, float rr, int lane) {
    int e = e0 + lane;
    if (e < n_adj) {
        uint2 raw = __ldg(&P.adj_diff[a0 + e]);
        v3 diff = mk(h2f((uint16_t)(raw.x & 0xffffu)), h2f((uint16_t)(raw.x >> 16)), h2f((uint16_t)(raw.y & 0xffffu)));
        float ar = h2f((uint16_t)(raw.y >> 16));
        Face f = make_face(eye, center, cc, rr, center + diff, ar);
        ws.face[lane] = make_float4(f.n.x, f.n.y, f.n.z, f.num);
    }
    __syncwarp();
}

// texel records of one primitive, from the warp's shared staging area or
// straight from global memory (read-only path)
struct SmemTexels {
    const WarpStage& ws;
    PF_D v3 site(int i) const { return mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]); }
    PF_D v3 rgb(int i) const { return mk(ws.tr[3 * i], ws.tr[3 * i + 1], ws.tr[3 * i + 2]); }
    PF_D float height(int i) const { return ws.th[i]; }
};

struct GlobalTexels {
    const float* s;  // (S,3) of the primitive
    const float* c;  // (S,3)
    const float* h;  // (S)
    PF_D v3 site(int i) const { return mk(__ldg(s + 3 * i), __ldg(s + 3 * i + 1), __ldg(s + 3 * i + 2)); }
    PF_D v3 rgb(int i) const { return mk(__ldg(c + 3 * i), __ldg(c + 3 * i + 1), __ldg(c + 3 * i + 2)); }
    PF_D float height(int i) const { return __ldg(h + i); }
};

PF_D GlobalTexels global_texels(const RasterParams& P, int32_t prim) {
    const int64_t b3 = (int64_t)prim * P.S * 3;
    return GlobalTexels{P.sites + b3, P.rgb + b3, P.height + (int64_t)prim * P.S};
}

// texture.py:10-72 (hit path); one copy of the arithmetic for every texel
// source.  Texels read from global memory unroll the site loops by 2 so two
// sites' loads are in flight together (the sums keep their order).
template <typename TX>
struct TexUnroll {
    static constexpr int value = 1;
};
template <>
struct TexUnroll<GlobalTexels> {
    static constexpr int value = 2;
};

template <typename TX>
PF_D PlaneRes plane_fwd_tex(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const TX& tx, int S) {
    PlaneRes r;
    float _dp;
    float _t_surf = ray_plane(o, d, po, pn, 0.0f, _dp);
    float _tq = _dp >= 0.0f ? t_near : fmax_t(t_near, _t_surf);
    v3 _pt = o + _tq * d;
    float rr = radius * radius;
    float hsum = 0.f, _wsum = 0.f;
#pragma unroll TexUnroll<TX>::value
    for (int i = 0; i < S; i++) {
        v3 df = _pt - tx.site(i);
        float dist_sq = dot(df, df) / rr;
        float w = expf(-kTemp * dist_sq);
        hsum += w * tx.height(i);
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
#pragma unroll TexUnroll<TX>::value
    for (int i = 0; i < S; i++) {
        v3 df = pt - tx.site(i);
        float dist_sq = dot(df, df) / rr;
        float w = expf(-kTemp * dist_sq);
        rgb_sum = rgb_sum + w * tx.rgb(i);
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

PF_D PlaneRes plane_fwd_smem(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const WarpStage& ws, int S) {
    return plane_fwd_tex(o, d, t_near, po, pn, radius, SmemTexels{ws}, S);
}


inline bool fill_params(const pf_raster_inputs* in, RasterParams& P, bool need_f32, const char** why) {
    if (!in) {
        *why = "null inputs";
        return false;
    }
    if (in->cam.width < 2 || in->cam.height < 2) {
        *why = "image must be at least 2x2";
        return false;
    }
    if (in->n_sites < 0 || in->n_sites > kMaxSites) {
        *why = "n_sites must be in [0, 8]";
        return false;
    }
    if (in->tile_width <= 0) {
        *why = "tile_width must be positive";
        return false;
    }
    if (need_f32 && in->attr_half) {
        *why = "forward/backward take float32 attributes";
        return false;
    }
    if (in->n_quantiles < 0 || (in->n_quantiles > 0 && !in->depth_quantiles)) {
        *why = "bad quantiles";
        return false;
    }
    if (in->n_prims > 0 && (!in->spheres || !in->nsigmas || !in->adjacency_offsets || !in->texel_sites ||
                            !in->texel_rgb || !in->texel_height)) {
        *why = "missing primitive arrays";
        return false;
    }
    if (!in->tile_offsets || !in->tile_prims) {
        *why = "missing tile lists";
        return false;
    }
    P.cam = load_cam(in->cam);
    P.TW = in->tile_width;
    P.S = in->n_sites;
    P.Q = in->n_quantiles;
    P.N = in->n_prims;
    P.tiles_h = 1 + (in->cam.height - 1) / P.TW;
    int tiles_w = 1 + (in->cam.width - 1) / P.TW;
    P.T = (int64_t)P.tiles_h * tiles_w;
    P.spheres = (const float4*)in->spheres;
    P.nsigmas = (const float4*)in->nsigmas;
    P.sites = (const float*)in->texel_sites;
    P.rgb = (const float*)in->texel_rgb;
    P.height = (const float*)in->texel_height;
    P.adj = in->adjacency;
    P.adj_off = in->adjacency_offsets;
    P.adj_diff = (const uint2*)in->adjacency_diff;
    P.tile_off = in->tile_offsets;
    P.tile_prims = in->tile_prims;
    P.dq = in->depth_quantiles;
    P.gt = in->ray_gt;
    P.thr = in->transmittance_threshold;
    P.tile_order = in->tile_order;
    P.seg = (float4*)in->segments;
    P.seg_mask = in->segment_masks;
    P.seg_off = in->segment_offsets;
    P.seg_count = (unsigned long long*)in->segment_count;
    P.seg_pairs = in->segments ? in->segment_pairs : 0;
    P.seg_cap = in->segments ? in->segment_capacity : 0;
    P.seg_stride = in->segment_planes ? 4 : 1;
    if (in->segments && (!in->segment_masks || !in->segment_offsets || !in->segment_count ||
                         ((uintptr_t)in->segments % 16) != 0 || in->segment_pairs < 0 ||
                         in->segment_capacity < 0 || in->segment_capacity >= ((int64_t)1 << 31) ||
                         (in->tile_width != 8 && in->tile_width != 16))) {
        *why = "segments need segment_masks, segment_offsets, segment_count, 16-byte alignment, "
               "0 <= segment_capacity < 2^31 and tile width 8 or 16";
        return false;
    }
    P.queue = (int*)in->scratch;
    P.ray_maps = in->ray_maps;
    return true;
}


}  // namespace pf

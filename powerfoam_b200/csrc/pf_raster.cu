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
#include "pf_api.h"

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
};

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

// texture.py:10-72 with texel data in shared memory (hit path)
PF_D PlaneRes plane_fwd_smem(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const WarpStage& ws, int S) {
    PlaneRes r;
    float _dp;
    float _t_surf = ray_plane(o, d, po, pn, 0.0f, _dp);
    float _tq = _dp >= 0.0f ? t_near : fmax_t(t_near, _t_surf);
    v3 _pt = o + _tq * d;
    float rr = radius * radius;
    float hsum = 0.f, _wsum = 0.f;
#pragma unroll
    for (int i = 0; i < kMaxSites; i++) {
        if (i < S) {
            v3 df = _pt - mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]);
            float dist_sq = dot(df, df) / rr;
            float w = expf(-kTemp * dist_sq);
            hsum += w * ws.th[i];
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
            v3 df = pt - mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]);
            float dist_sq = dot(df, df) / rr;
            float w = expf(-kTemp * dist_sq);
            rgb_sum = rgb_sum + w * mk(ws.tr[3 * i], ws.tr[3 * i + 1], ws.tr[3 * i + 2]);
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
// forward (rasterize.py:892-1146)
struct FwdPix {
    PixGeom g;
    float log_t, trans, nd, err;
    v3 rgb, nrm, gt;
    int qi;
    float q;
    bool hit;
    float tn, tf;
};

template <int TW>
__global__ void __launch_bounds__(TW == 32 ? 512 : 128)
raster_fwd_kernel(RasterParams P, int rpe, float* __restrict__ color, float* __restrict__ log_t_out,
                  float* __restrict__ nd_out, float* __restrict__ normal_out, float* __restrict__ qd_out,
                  float* __restrict__ err_out, float* __restrict__ contrib, float* __restrict__ point_err,
                  int32_t* __restrict__ early_stop, int32_t* __restrict__ tile_contrib_pairs) {
    constexpr int G = TW * TW / 64;
    constexpr int WPB = G == 1 ? kWarpsPerBlock8 : G;
    __shared__ WarpStage stage[WPB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t tile = G == 1 ? (int64_t)blockIdx.x * WPB + warp : (int64_t)blockIdx.x;
    if (tile >= P.T) return;  // G == 1 only: whole warps
    const int wig = G == 1 ? 0 : warp;  // warp index within the tile's group
    WarpStage& ws = stage[warp];
    const v3 o = P.cam.eye;
    const float HW = (float)(P.cam.H * P.cam.W);
    FwdPix px[2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        int idx = wig * 32 + lane + s * (TW * TW / 2);
        px[s].g = pixel_geom(P, tile, idx);
        px[s].log_t = 0.f;
        px[s].trans = 1.0f;
        px[s].nd = 0.f;
        px[s].err = 0.f;
        px[s].rgb = mk(0.f, 0.f, 0.f);
        px[s].nrm = mk(0.f, 0.f, 0.f);
        px[s].qi = 0;
        px[s].q = 0.f;
        if (!px[s].g.oob) {
            if (P.Q > 0) {
                px[s].q = P.dq[px[s].g.px * P.Q];
                for (int q = 0; q < P.Q; q++) qd_out[px[s].g.px * P.Q + q] = -1.0f;
            }
            if (rpe || err_out) px[s].gt = mk(P.gt[3 * px[s].g.px], P.gt[3 * px[s].g.px + 1], P.gt[3 * px[s].g.px + 2]);
        }
    }
    const int64_t start = P.tile_off[tile];
    const int total = (int)(P.tile_off[tile + 1] - start);
    int es = total;
    int n_contrib_pairs = 0;
    bool stopped = false;
    for (int k0 = 0; k0 < total && !stopped; k0 += 32) {
        stage_prims(ws, P, start, k0, total, lane);
        const int kn = min(32, total - k0);
        for (int kk = 0; kk < kn; kk++) {
            bool below = (px[0].g.oob ? false : px[0].trans < P.thr) && (px[1].g.oob ? false : px[1].trans < P.thr);
            if (group_all<G>(below)) {
                es = k0 + kk;
                stopped = true;
                break;
            }
            float4 s4 = ws.sph[kk];
            float4 n4 = ws.nsg[kk];
            const v3 center = mk(s4.x, s4.y, s4.z);
            const float radius = s4.w;
#pragma unroll
            for (int s = 0; s < 2; s++)
                px[s].hit = px[s].g.oob ? false : ray_sphere(o, px[s].g.d, center, radius, px[s].tn, px[s].tf);
            if (!group_any<G>(px[0].hit || px[1].hit)) continue;
            const int32_t prim = ws.pid[kk];
            const v3 pn = mk(n4.x, n4.y, n4.z);
            const float sigma = n4.w;
            const int32_t a0 = __ldg(&P.adj_off[prim]);
            const int n_adj = __ldg(&P.adj_off[prim + 1]) - a0;
            const float cc = dot(center, center), rr = radius * radius;
            for (int e0 = 0; e0 < n_adj; e0 += 32) {
                stage_faces(ws, P, a0, e0, n_adj, o, center, cc, rr, lane);
                const int en = min(32, n_adj - e0);
                for (int q = 0; q < en; q++) {
                    float4 f = ws.face[q];
                    v3 fn = mk(f.x, f.y, f.z);
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        if (px[s].hit) {
                            float dp = dot(px[s].g.d, fn);
                            float t_face = f.w / dp;
                            px[s].tf = dp >= 0.0f ? fmin_t(t_face, px[s].tf) : px[s].tf;
                            px[s].tn = dp < 0.0f ? fmax_t(t_face, px[s].tn) : px[s].tn;
                        }
                    }
                }
                __syncwarp();
            }
            stage_texels(ws, P, prim, lane);
            float c_acc = 0.f, e_acc = 0.f;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                FwdPix& a = px[s];
                if (!a.hit) continue;
                PlaneRes pr = plane_fwd_smem(o, a.g.d, a.tn, center, pn, radius, ws, P.S);
                float tf = pr.dp >= 0.0f ? fmin_t(pr.t_surf, a.tf) : a.tf;
                float tn = pr.dp < 0.0f ? fmax_t(pr.t_surf, a.tn) : a.tn;
                float dt = tf - tn;
                if (dt > 0.0f) {
                    float dlt = -sigma * dt;
                    float alpha = 1.0f - expf(dlt);
                    float trans = a.trans;
                    if (err_out) {
                        v3 de = pr.rgb - a.gt;
                        a.err += dot(de, de) * alpha * trans;
                    }
                    a.rgb = a.rgb + trans * (alpha * pr.rgb);
                    a.log_t += dlt;
                    c_acc += alpha * trans / HW;
                    if (rpe) {
                        v3 df = pr.rgb - a.gt;
                        float l1 = fabsf(df.x) + fabsf(df.y) + fabsf(df.z);
                        e_acc += alpha * trans * l1 / HW;
                    }
                    float ndv = dot(pn, a.g.d);
                    if (ndv > 0.0f) a.nd += ndv * ndv * alpha * trans;
                    a.nrm = a.nrm + (alpha * trans) * pn;
                    float next_trans = expf(a.log_t);
                    while (a.qi < P.Q && next_trans < a.q) {
                        float qd = tn + logf(trans / a.q) / sigma;
                        qd_out[a.g.px * P.Q + a.qi] = qd;
                        a.qi += 1;
                        if (a.qi < P.Q) a.q = P.dq[a.g.px * P.Q + a.qi];
                    }
                    a.trans = next_trans;
                }
            }
            // one atomic per primitive per warp for contrib / point_err
            if (__any_sync(0xffffffffu, c_acc != 0.f || e_acc != 0.f)) {
                n_contrib_pairs++;
                float cs = warp_sum(c_acc);
                float esum = rpe ? warp_sum(e_acc) : 0.f;
                if (lane == 0) {
                    atomicAdd(&contrib[prim], cs);
                    if (rpe) atomicAdd(&point_err[prim], esum);
                }
            }
            __syncwarp();
        }
        __syncwarp();
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const FwdPix& a = px[s];
        if (a.g.oob) continue;
        int64_t p = a.g.px;
        color[3 * p] = a.rgb.x;
        color[3 * p + 1] = a.rgb.y;
        color[3 * p + 2] = a.rgb.z;
        log_t_out[p] = a.log_t;
        nd_out[p] = a.nd;
        normal_out[3 * p] = a.nrm.x;
        normal_out[3 * p + 1] = a.nrm.y;
        normal_out[3 * p + 2] = a.nrm.z;
        if (err_out) {
            // background is black (rasterize.py:59)
            v3 de = mk(0.f, 0.f, 0.f) - a.gt;
            err_out[p] = a.err + dot(de, de) * expf(a.log_t);
        }
    }
    if (lane == 0 && wig == 0) early_stop[tile] = es;
    if (tile_contrib_pairs && lane == 0) atomicAdd(&tile_contrib_pairs[tile], n_contrib_pairs);
}

// ---------------------------------------------------------------------------
// adjoint (rasterize.py:1150-1514 + texture.py:74-186)
struct BwdPix {
    PixGeom g;
    float log_t, dLdlog_t, g_nd;
    v3 g_rgb, g_n;
    int qi;
    float q;
    bool hit;
    float tn, tf;
    int tn_id, tf_id;
};

// Accumulators of one primitive's gradient over a lane's pixels, in the
// order of the reduce-scatter: [0,3) centre, 3 radius, [4,7) normal, 7 sigma,
// [8,32) sites, [32,56) rgb, [56,64) height.
struct GradAcc {
    float v[64];
};

PF_D void plane_bwd_acc(v3 o, v3 d, float _t_near, v3 po, v3 pn, float radius, const WarpStage& ws, int S,
                        const PlaneRes& pr, v3 dLdrgb_in, float dLdt_surf_in, GradAcc& acc, v3& dLdpo_out,
                        v3& dLdpn_out, float& dLd_t_near_out) {
    v3 dLdpo = mk(0.f, 0.f, 0.f), dLdpn = mk(0.f, 0.f, 0.f);
    float dLdheight_in = 0.f;
    const float height_in = pr.height, weight_sum = pr.wsum, _weight_sum = pr._wsum;
    const float rr = radius * radius;
    float tq = pr.dp >= 0.0f ? _t_near : fmax_t(_t_near, pr.t_surf);
    v3 pt = o + tq * d;
    v3 dLdpt = mk(0.f, 0.f, 0.f);
    float grad_dp_in = dot(dLdrgb_in, pr.rgb);
#pragma unroll
    for (int i = 0; i < kMaxSites; i++) {
        if (i < S) {
            v3 site = mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]);
            v3 df = pt - site;
            float dist_sq = dot(df, df) / rr;
            float w = expf(-kTemp * dist_sq);
            if (!(w / weight_sum < 1e-3f)) {
                v3 dwds = ((2.0f * kTemp * w) * (pt - site)) / rr;
                v3 rgb_grad = (w * dLdrgb_in) / weight_sum;
                acc.v[32 + 3 * i] += rgb_grad.x;
                acc.v[33 + 3 * i] += rgb_grad.y;
                acc.v[34 + 3 * i] += rgb_grad.z;
                float grad_dp = dot(dLdrgb_in, mk(ws.tr[3 * i], ws.tr[3 * i + 1], ws.tr[3 * i + 2]));
                v3 site_grad = ((grad_dp - grad_dp_in) * dwds) / weight_sum;
                acc.v[8 + 3 * i] += site_grad.x;
                acc.v[9 + 3 * i] += site_grad.y;
                acc.v[10 + 3 * i] += site_grad.z;
                dLdpt = dLdpt + (-site_grad);
            }
        }
    }
    float dLdt_query = dot(dLdpt, d);
    float dLd_t_near = (pr.dp >= 0.0f || _t_near >= pr.t_surf) ? dLdt_query : 0.0f;
    float dLdt_surf = (pr.dp < 0.0f && _t_near < pr.t_surf) ? dLdt_query : 0.0f;
    dLdt_surf += dLdt_surf_in;
    if (fabsf(dLdt_surf) > 0.0f) {
        v3 a, b;
        float c;
        ray_plane_bwd(o, d, po, pn, height_in, a, b, c);
        dLdpo = dLdpo + dLdt_surf * a;
        dLdpn = dLdpn + dLdt_surf * b;
        dLdheight_in += c * dLdt_surf;
    }
    float _tq = pr._dp >= 0.0f ? _t_near : fmax_t(_t_near, pr._t_surf);
    v3 _pt = o + _tq * d;
    v3 dLd_pt = mk(0.f, 0.f, 0.f);
    float _grad_dp_in = dLdheight_in * height_in;
#pragma unroll
    for (int i = 0; i < kMaxSites; i++) {
        if (i < S) {
            v3 site = mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]);
            v3 df = _pt - site;
            float dist_sq = dot(df, df) / rr;
            float w = expf(-kTemp * dist_sq);
            if (!(w / weight_sum < 1e-3f)) {
                v3 dwds = ((2.0f * kTemp * w) * (_pt - site)) / rr;
                acc.v[56 + i] += w * dLdheight_in / _weight_sum;
                float _grad_dp = dLdheight_in * ws.th[i];
                v3 site_grad = ((_grad_dp - _grad_dp_in) * dwds) / _weight_sum;
                acc.v[8 + 3 * i] += site_grad.x;
                acc.v[9 + 3 * i] += site_grad.y;
                acc.v[10 + 3 * i] += site_grad.z;
                dLd_pt = dLd_pt + (-site_grad);
            }
        }
    }
    float dLd_t_query = dot(dLd_pt, d);
    dLd_t_near += (pr.dp >= 0.0f || _t_near >= pr._t_surf) ? dLd_t_query : 0.0f;
    float dLd_t_surf = (pr.dp < 0.0f && _t_near < pr._t_surf) ? dLd_t_query : 0.0f;
    if (fabsf(dLd_t_surf) > 0.0f) {
        v3 a, b;
        float c;
        ray_plane_bwd(o, d, po, pn, 0.0f, a, b, c);
        dLdpo = dLdpo + dLd_t_surf * a;
        dLdpn = dLdpn + dLd_t_surf * b;
    }
    dLdpo_out = dLdpo;
    dLdpn_out = dLdpn;
    dLd_t_near_out = dLd_t_near;
}

struct GradOut {
    float* points;   // (N,3)
    float* radii;    // (N)
    float* normals;  // (N,3)
    float* density;  // (N)
    float* sites;    // (N,S,3)
    float* rgb;      // (N,S,3)
    float* height;   // (N,S)
};

PF_D float* grad_slot(const GradOut& go, int S, int64_t prim, int j) {
    if (j < 3) return go.points + 3 * prim + j;
    if (j == 3) return go.radii + prim;
    if (j < 7) return go.normals + 3 * prim + (j - 4);
    if (j == 7) return go.density + prim;
    if (j < 32) {
        int r = j - 8;
        return (r < 3 * S) ? go.sites + prim * S * 3 + r : nullptr;
    }
    if (j < 56) {
        int r = j - 32;
        return (r < 3 * S) ? go.rgb + prim * S * 3 + r : nullptr;
    }
    int r = j - 56;
    return (r < S) ? go.height + prim * S + r : nullptr;
}

// reduce-scatter of 64 values over the warp: lane l ends with the sums of
// values 2l and 2l+1, then adds them to the gradient arrays.
PF_D void flush_grads(GradAcc& acc, const GradOut& go, int S, int64_t prim, int lane) {
#pragma unroll
    for (int step = 0; step < 5; step++) {
        const int off = 16 >> step;
        const int half = 32 >> step;
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int i = 0; i < half; i++) {
            float send = upper ? acc.v[i] : acc.v[i + half];
            float keep = upper ? acc.v[i + half] : acc.v[i];
            acc.v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        float val = acc.v[h];
        if (val != 0.0f) {
            float* dst = grad_slot(go, S, prim, 2 * lane + h);
            if (dst) atomicAdd(dst, val);
        }
    }
}

template <int TW>
__global__ void __launch_bounds__(TW == 32 ? 512 : 128)
raster_bwd_kernel(RasterParams P, const int32_t* __restrict__ early_stop, const float* __restrict__ log_t_in,
                  const float* __restrict__ g_color, const float* __restrict__ g_opacity,
                  const float* __restrict__ g_nd, const float* __restrict__ g_normal, const float* __restrict__ g_qd,
                  const float* __restrict__ g_contrib, GradOut go) {
    constexpr int G = TW * TW / 64;
    constexpr int WPB = G == 1 ? kWarpsPerBlock8 : G;
    __shared__ WarpStage stage[WPB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t tile = G == 1 ? (int64_t)blockIdx.x * WPB + warp : (int64_t)blockIdx.x;
    if (tile >= P.T) return;
    const int wig = G == 1 ? 0 : warp;
    WarpStage& ws = stage[warp];
    const v3 o = P.cam.eye;
    const float HW = (float)(P.cam.H * P.cam.W);
    const v3 bkgd = mk(0.f, 0.f, 0.f);
    BwdPix px[2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        int idx = wig * 32 + lane + s * (TW * TW / 2);
        BwdPix& a = px[s];
        a.g = pixel_geom(P, tile, idx);
        int64_t p = a.g.px;
        a.log_t = log_t_in[p];
        if (P.Q > 0) {
            a.qi = P.Q - 1;
            a.q = P.dq[p * P.Q + P.Q - 1];
        } else {
            a.qi = -1;
            a.q = 1.0f;
        }
        a.g_rgb = mk(g_color[3 * p], g_color[3 * p + 1], g_color[3 * p + 2]);
        // rasterize.py:1905: grad_log_t = -grad_opacity * exp(log_t)
        float g_logt = -g_opacity[p] * expf(a.log_t);
        a.g_nd = g_nd ? g_nd[p] : 0.f;
        a.g_n = g_normal ? mk(g_normal[3 * p], g_normal[3 * p + 1], g_normal[3 * p + 2]) : mk(0.f, 0.f, 0.f);
        float dLdtrans = dot(a.g_rgb, bkgd);
        a.dLdlog_t = dLdtrans * expf(a.log_t);
        a.dLdlog_t += g_logt;
    }
    const int64_t start = P.tile_off[tile];
    const int es = early_stop[tile];
    for (int k1 = es - 1; k1 >= 0; k1 -= 32) {
        const int k0 = k1 - 31;  // batch [k0, k1], may start below 0
        stage_prims(ws, P, start, k0, es, lane);
        for (int k = k1; k >= 0 && k >= k0; k--) {
            const int kk = k - k0;
            float4 s4 = ws.sph[kk];
            float4 n4 = ws.nsg[kk];
            const v3 center = mk(s4.x, s4.y, s4.z);
            const float radius = s4.w;
#pragma unroll
            for (int s = 0; s < 2; s++)
                px[s].hit = px[s].g.oob ? false : ray_sphere(o, px[s].g.d, center, radius, px[s].tn, px[s].tf);
            if (!group_any<G>(px[0].hit || px[1].hit)) continue;
            const int32_t prim = ws.pid[kk];
            const v3 pn = mk(n4.x, n4.y, n4.z);
            const float sigma = n4.w;
            const int32_t a0 = __ldg(&P.adj_off[prim]);
            const int n_adj = __ldg(&P.adj_off[prim + 1]) - a0;
            const float cc = dot(center, center), rr = radius * radius;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                px[s].tn_id = px[s].tn < 1e-8f ? -2 : -1;
                px[s].tf_id = px[s].tf < 1e-8f ? -2 : -1;
            }
            for (int e0 = 0; e0 < n_adj; e0 += 32) {
                stage_faces(ws, P, a0, e0, n_adj, o, center, cc, rr, lane);
                const int en = min(32, n_adj - e0);
                for (int q = 0; q < en; q++) {
                    float4 f = ws.face[q];
                    v3 fn = mk(f.x, f.y, f.z);
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        BwdPix& a = px[s];
                        if (a.hit) {
                            float dp = dot(a.g.d, fn);
                            float t_face = f.w / dp;
                            int adj_idx = e0 + q;
                            a.tf_id = (dp >= 0.0f && t_face < a.tf) ? adj_idx : a.tf_id;
                            a.tf = dp >= 0.0f ? fmin_t(t_face, a.tf) : a.tf;
                            a.tn_id = (dp < 0.0f && t_face > a.tn) ? adj_idx : a.tn_id;
                            a.tn = dp < 0.0f ? fmax_t(t_face, a.tn) : a.tn;
                        }
                    }
                }
                __syncwarp();
            }
            stage_texels(ws, P, prim, lane);
            const float cg = g_contrib ? __ldg(&g_contrib[prim]) : 0.f;
            GradAcc acc;
#pragma unroll
            for (int j = 0; j < 64; j++) acc.v[j] = 0.f;
            bool any_contrib = false;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                BwdPix& a = px[s];
                if (!a.hit) continue;  // oob pixels never hit here
                const v3 d = a.g.d;
                float t_near = a.tn, t_far = a.tf;
                int t_near_id = a.tn_id, t_far_id = a.tf_id;
                const float _t_near = t_near;
                const int _t_near_id = t_near_id, _t_far_id = t_far_id;
                PlaneRes pr = plane_fwd_smem(o, d, t_near, center, pn, radius, ws, P.S);
                t_far_id = (pr.dp >= 0.0f && pr.t_surf < t_far) ? n_adj : t_far_id;
                t_far = pr.dp >= 0.0f ? fmin_t(pr.t_surf, t_far) : t_far;
                t_near_id = (pr.dp < 0.0f && pr.t_surf > t_near) ? n_adj : t_near_id;
                t_near = pr.dp < 0.0f ? fmax_t(pr.t_surf, t_near) : t_near;
                const float dt = t_far - t_near;
                const bool contributes = dt > 0.0f;
                if (!contributes) continue;  // plane_bwd with hit=false returns zeros
                any_contrib = true;
                float dLdt_near = 0.f, dLdt_far = 0.f, dLdradius = 0.f, dLdsigma = 0.f;
                v3 dLdcenter = mk(0.f, 0.f, 0.f), dLdnormal = mk(0.f, 0.f, 0.f), dLdcolor = mk(0.f, 0.f, 0.f);
                {
                    float delta_log_t = -sigma * dt;
                    a.log_t -= delta_log_t;
                    float alpha = 1.0f - expf(delta_log_t);
                    float trans = expf(a.log_t);
                    float ndv = dot(pn, d);
                    float dLdlog_t_i = a.dLdlog_t;
                    float dLddelta_log_t = a.dLdlog_t;
                    float dLdalpha = dot(a.g_rgb, pr.rgb) * trans;
                    if (ndv > 0.0f) dLdalpha += a.g_nd * ndv * trans;
                    dLdalpha += cg * trans / HW;
                    dLdalpha += dot(a.g_n, pn) * trans;
                    float dLdtrans = dot(a.g_rgb, pr.rgb) * alpha;
                    if (ndv > 0.0f) dLdtrans += a.g_nd * ndv * alpha;
                    dLdtrans += cg * alpha / HW;
                    dLdtrans += dot(a.g_n, pn) * alpha;
                    dLdcolor = dLdcolor + alpha * (trans * a.g_rgb);
                    dLdlog_t_i += dLdtrans * expf(a.log_t);
                    dLddelta_log_t += -dLdalpha * expf(delta_log_t);
                    dLdsigma += dLddelta_log_t * -dt;
                    dLdt_near += dLddelta_log_t * sigma;
                    dLdt_far += dLddelta_log_t * -sigma;
                    while (a.qi >= 0 && trans > a.q) {
                        float dq = g_qd ? g_qd[a.g.px * P.Q + a.qi] : 0.f;
                        dLdsigma += -dq * logf(trans / a.q) / (sigma * sigma + 1e-6f);
                        dLdt_near += dq;
                        dLdlog_t_i += dq / (sigma + 1e-6f);
                        a.qi -= 1;
                        if (a.qi >= 0) a.q = P.dq[a.g.px * P.Q + a.qi];
                    }
                    dLdnormal = dLdnormal + (alpha * trans) * a.g_n;
                    if (ndv > 0.0f) dLdnormal = dLdnormal + (a.g_nd * alpha * trans) * d;
                    a.dLdlog_t = dLdlog_t_i;
                }
                float dLdt_surf;
                if (t_near_id == n_adj) dLdt_surf = dLdt_near;
                else if (t_far_id == n_adj) dLdt_surf = dLdt_far;
                else dLdt_surf = 0.0f;
                v3 _dc, _dn;
                float dLd_t_near;
                plane_bwd_acc(o, d, _t_near, center, pn, radius, ws, P.S, pr, dLdcolor, dLdt_surf, acc, _dc, _dn,
                              dLd_t_near);
                dLdcenter = dLdcenter + _dc;
                dLdnormal = dLdnormal + _dn;
                if (t_near_id != n_adj) dLd_t_near += dLdt_near;
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    const int t_id = i == 0 ? _t_near_id : _t_far_id;
                    const float dLdt = i == 0 ? dLd_t_near : dLdt_far;
                    if (t_id == -1) {
                        v3 ndc, fdc;
                        float ndr, fdr;
                        ray_sphere_bwd(o, d, center, radius, ndc, fdc, ndr, fdr);
                        if (i == 0) {
                            dLdcenter = dLdcenter + dLdt * ndc;
                            dLdradius += dLdt * ndr;
                        } else {
                            dLdcenter = dLdcenter + dLdt * fdc;
                            dLdradius += dLdt * fdr;
                        }
                    } else if (t_id >= 0 && t_id < n_adj) {
                        const int32_t adjacent = __ldg(&P.adj[a0 + t_id]);
                        const float4 as = __ldg(&P.spheres[adjacent]);
                        v3 dc, dac;
                        float dr, dar;
                        ray_pface_bwd(o, d, center, radius, mk(as.x, as.y, as.z), as.w, dc, dr, dac, dar);
                        dLdcenter = dLdcenter + dLdt * dc;
                        dLdradius += dLdt * dr;
                        v3 gac = dLdt * dac;
                        atomicAdd(&go.points[3 * (int64_t)adjacent], gac.x);
                        atomicAdd(&go.points[3 * (int64_t)adjacent + 1], gac.y);
                        atomicAdd(&go.points[3 * (int64_t)adjacent + 2], gac.z);
                        atomicAdd(&go.radii[adjacent], dLdt * dar);
                    }
                }
                acc.v[0] += dLdcenter.x;
                acc.v[1] += dLdcenter.y;
                acc.v[2] += dLdcenter.z;
                acc.v[3] += dLdradius;
                acc.v[4] += dLdnormal.x;
                acc.v[5] += dLdnormal.y;
                acc.v[6] += dLdnormal.z;
                acc.v[7] += dLdsigma;
            }
            if (__any_sync(0xffffffffu, any_contrib)) flush_grads(acc, go, P.S, prim, lane);
        }
        __syncwarp();
    }
}

__global__ void zero_nonfinite_kernel(float* __restrict__ a, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        float v = a[i];
        if (!isfinite(v)) a[i] = 0.0f;
    }
}

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

static bool fill_params(const pf_raster_inputs* in, RasterParams& P, bool need_f32, const char** why) {
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
    return true;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_raster_forward(const pf_raster_inputs* in, int32_t return_point_err, float* color, float* log_t,
                                 float* normal_distance, float* normal, float* quantile_depths, float* err,
                                 float* contrib, float* point_err, int32_t* early_stop, int32_t* tile_contrib_pairs,
                                 void* stream) {
    RasterParams P;
    const char* why = "";
    if (!fill_params(in, P, true, &why)) return pf_fail(PF_ERR_ARGS, why);
    if (return_point_err && (!in->ray_gt || !point_err))
        return pf_fail(PF_ERR_ARGS, "Ground truth rays must be provided to return point error");
    if (err && !in->ray_gt)
        return pf_fail(PF_ERR_ARGS, "Ground truth rays must be provided for surface loss accumulation");
    if (!color || !log_t || !normal_distance || !normal || !contrib || !early_stop || (P.Q > 0 && !quantile_depths))
        return pf_fail(PF_ERR_ARGS, "pf_raster_forward: missing output");
    if (P.TW != 8 && P.TW != 16 && P.TW != 32) return pf_fail(PF_ERR_ARGS, "tile_width must be 8, 16 or 32");
    cudaStream_t st = (cudaStream_t)stream;
    if (P.N > 0) cudaMemsetAsync(contrib, 0, sizeof(float) * (size_t)P.N, st);
    if (return_point_err && P.N > 0) cudaMemsetAsync(point_err, 0, sizeof(float) * (size_t)P.N, st);
    if (tile_contrib_pairs && P.T > 0) cudaMemsetAsync(tile_contrib_pairs, 0, sizeof(int32_t) * (size_t)P.T, st);
    if (P.T == 0) return PF_OK;
    if (P.TW == 8) {
        unsigned grid = (unsigned)((P.T + kWarpsPerBlock8 - 1) / kWarpsPerBlock8);
        raster_fwd_kernel<8><<<grid, 32 * kWarpsPerBlock8, 0, st>>>(P, return_point_err, color, log_t, normal_distance,
                                                                   normal, quantile_depths, err, contrib, point_err,
                                                                   early_stop, tile_contrib_pairs);
    } else if (P.TW == 16) {
        raster_fwd_kernel<16><<<(unsigned)P.T, 128, 0, st>>>(P, return_point_err, color, log_t, normal_distance, normal,
                                                             quantile_depths, err, contrib, point_err, early_stop,
                                                             tile_contrib_pairs);
    } else {
        raster_fwd_kernel<32><<<(unsigned)P.T, 512, 0, st>>>(P, return_point_err, color, log_t, normal_distance, normal,
                                                             quantile_depths, err, contrib, point_err, early_stop,
                                                             tile_contrib_pairs);
    }
    return pf_check_launch("pf_raster_forward");
}

extern "C" int pf_raster_backward(const pf_raster_inputs* in, const int32_t* early_stop, const float* log_t,
                                  const float* grad_color, const float* grad_opacity,
                                  const float* grad_normal_distance, const float* grad_normal,
                                  const float* grad_quantile_depths, const float* grad_contrib, float* grad_points,
                                  float* grad_radii, float* grad_normals, float* grad_density, float* grad_texel_sites,
                                  float* grad_texel_rgb, float* grad_texel_height, void* stream) {
    RasterParams P;
    const char* why = "";
    if (!fill_params(in, P, true, &why)) return pf_fail(PF_ERR_ARGS, why);
    if (!early_stop || !log_t || !grad_color || !grad_opacity || !grad_points || !grad_radii || !grad_normals ||
        !grad_density || !grad_texel_sites || !grad_texel_rgb || !grad_texel_height)
        return pf_fail(PF_ERR_ARGS, "pf_raster_backward: missing argument");
    if (P.TW != 8 && P.TW != 16 && P.TW != 32) return pf_fail(PF_ERR_ARGS, "tile_width must be 8, 16 or 32");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t N = (size_t)P.N, S = (size_t)P.S;
    float* outs[7] = {grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites, grad_texel_rgb,
                      grad_texel_height};
    size_t lens[7] = {3 * N, N, 3 * N, N, 3 * N * S, 3 * N * S, N * S};
    for (int i = 0; i < 7; i++)
        if (lens[i]) cudaMemsetAsync(outs[i], 0, sizeof(float) * lens[i], st);
    GradOut go{grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites, grad_texel_rgb, grad_texel_height};
    const float* gq = P.Q > 0 ? grad_quantile_depths : nullptr;
    if (P.T > 0) {
        if (P.TW == 8) {
            unsigned grid = (unsigned)((P.T + kWarpsPerBlock8 - 1) / kWarpsPerBlock8);
            raster_bwd_kernel<8><<<grid, 32 * kWarpsPerBlock8, 0, st>>>(P, early_stop, log_t, grad_color, grad_opacity,
                                                                       grad_normal_distance, grad_normal, gq,
                                                                       grad_contrib, go);
        } else if (P.TW == 16) {
            raster_bwd_kernel<16><<<(unsigned)P.T, 128, 0, st>>>(P, early_stop, log_t, grad_color, grad_opacity,
                                                                 grad_normal_distance, grad_normal, gq, grad_contrib,
                                                                 go);
        } else {
            raster_bwd_kernel<32><<<(unsigned)P.T, 512, 0, st>>>(P, early_stop, log_t, grad_color, grad_opacity,
                                                                 grad_normal_distance, grad_normal, gq, grad_contrib,
                                                                 go);
        }
    }
    for (int i = 0; i < 7; i++)
        if (lens[i]) {
            int64_t n = (int64_t)lens[i];
            unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
            zero_nonfinite_kernel<<<grid, 256, 0, st>>>(outs[i], n);
        }
    return pf_check_launch("pf_raster_backward");
}

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

// pf_composite.cuh -- tile-level forward and adjoint of the compositing,
// shared by the per-view kernels (pf_composite.cu) and the batched multi-view
// kernel (pf_batch.cu).  See pf_composite.cu for the design.
#pragma once
#include <algorithm>

#include "pf_api.h"
#include "pf_common.cuh"
#include "pf_raster_common.cuh"

namespace pf {


constexpr int kAccRows = 64;
constexpr int kFaceSlots = 16;
static_assert(kFaceSlots <= 32, "one neighbour slot per lane");

// Group layout per tile width: TW = 8 and 16 use one pixel per lane (G = 2
// and 8 warps per tile), TW = 32 two pixels per lane (G = 16).
template <int TW>
struct Layout {
    static constexpr int PPL = TW == 32 ? 2 : 1;
    static constexpr int G = TW * TW / (32 * PPL);
    static constexpr int THREADS = 32 * G;
    // resident blocks per SM the adjoint is compiled for (register budget)
    static constexpr int BWD_MIN_BLOCKS = TW == 8 ? 10 : 1;
    // the forward's: 14 blocks hold it to 72 registers (the record-writing
    // variant would otherwise take 80, 12 blocks: 5.73 against 5.55 ms at
    // 1M primitives, 1080p)
    static constexpr int FWD_MIN_BLOCKS = TW == 8 ? 14 : 1;
};

// Early termination across the warps of a tile (forward).  The reference
// stops a tile before primitive k when every pixel's transmittance is below
// the threshold (tile_max).  Transmittance never increases, so each warp
// records the first k at which all of ITS pixels are below (below_at) and the
// last k it has voted on (prog).  A warp that is not all-below knows the tile
// cannot stop at k and goes on without waiting; a warp that is all-below at k
// waits until every other warp has either recorded below_at <= k (stop) or
// voted on k while not below (go on).  The warp furthest behind never waits,
// so the protocol always progresses; the wait is nevertheless bounded by a
// clock limit, after which the kernel reports PF_ERR_CUDA in the status word
// and carries on compositing.
struct StopState {
    int below_at[32];
    int prog[32];
};

constexpr long long kWaitLimitCycles = 20000000000ll;  // ~10 s

template <int G>
PF_D void stop_reset(StopState& ss, int wig, int lane) {
    if (G > 1 && lane == 0) {
        ss.below_at[wig] = 0x7fffffff;
        ss.prog[wig] = -1;
    }
}

// returns true when the tile stops before primitive k
template <int G>
PF_D bool stop_vote(StopState& ss, int wig, int lane, int k, bool below, int* status) {
    const bool mine = __all_sync(0xffffffffu, below);
    if constexpr (G == 1) return mine;
    int stop = 0;
    if (lane == 0) {
        volatile int* vb = ss.below_at;
        volatile int* vp = ss.prog;
        if (mine && vb[wig] == 0x7fffffff) vb[wig] = k;
        __threadfence_block();
        vp[wig] = k;
        if (mine) {
            stop = 1;
            const long long t0 = clock64();
            for (int v = 0; v < G && stop; v++) {
                if (v == wig) continue;
                for (;;) {
                    if (vb[v] <= k) break;  // v below at k
                    if (vp[v] >= k) {
                        __threadfence_block();
                        if (vb[v] > k) stop = 0;  // v voted at k, not below
                        break;
                    }
                    if (clock64() - t0 > kWaitLimitCycles) {
                        if (status) atomicMax(status, PF_ERR_CUDA);
                        stop = 0;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
    }
    return __shfl_sync(0xffffffffu, stop, 0) != 0;
}

// next tile of this group; -1 when the queue is exhausted
template <int G>
PF_D int64_t next_tile(const RasterParams& P, int64_t& static_next, int lane, StopState* ss) {
    int64_t t;
    if (P.queue) {
        if constexpr (G == 1) {
            int v = 0;
            if (lane == 0) v = atomicAdd(P.queue, 1);
            t = __shfl_sync(0xffffffffu, v, 0);
        } else {
            __shared__ int s_t;
            __syncthreads();
            if (ss) stop_reset<G>(*ss, threadIdx.x >> 5, lane);
            if (threadIdx.x == 0) s_t = atomicAdd(P.queue, 1);
            __syncthreads();
            t = s_t;
        }
    } else {
        if constexpr (G > 1) {
            __syncthreads();
            if (ss) stop_reset<G>(*ss, threadIdx.x >> 5, lane);
            __syncthreads();
        }
        t = static_next;
        static_next = P.T;  // one tile per group without a queue
    }
    if (t >= P.T) return -1;
    return P.tile_order ? (int64_t)P.tile_order[t] : t;
}

// A face can change the running interval only if its exact crossing
// q = num / dp lies before t_far (dp >= 0) or after t_near (dp < 0); rounding
// is monotone, so rn(q) < t_far implies q < t_far.  With dp != 0 both tests
// read t * dp - num >= 0, and fma gives that value's exact sign in one
// rounding, so the (costly) IEEE division runs only for faces that may clip;
// dp == +-0 and NaNs always take the division.  Skipped faces would leave
// t_near, t_far and their ids unchanged, so the result is bit-identical.
PF_D bool face_may_clip(float dp, float num, float tn, float tf) {
    float tref = dp >= 0.0f ? tf : tn;
    float r = fmaf(tref, dp, -num);
    return !(r < 0.0f) || dp == 0.0f;
}

// ---------------------------------------------------------------------------
// forward
struct FwdPix {
    PixGeom g;
    v3 o;  // ray origin (generic cameras)
    float log_t, trans, nd, err;
    v3 rgb, nrm, gt;
    int qi;
    float q;
    bool hit;
    float tn, tf;
};

PF_D void swap_pix(FwdPix& a, FwdPix& b) {
    FwdPix t = a;
    a = b;
    b = t;
}

// The origin of pixel x's ray: the eye, or with a generic camera its own.
template <bool GEN, typename X>
PF_D v3 ray_org(const X& x, v3 eye) {
    if constexpr (GEN)
        return x.o;
    else
        return eye;
}

// Face numerator for pixel x.  The staged value is face_offset - eye . n for
// a pinhole camera; a generic camera stages face_offset alone (eye = 0) and
// subtracts its own origin here, as rendering_math.py:71-80 does per ray.
template <bool GEN, typename X>
PF_D float face_num(const float4& f, v3 fn, const X& x) {
    if constexpr (GEN)
        return f.w - dot(x.o, fn);
    else
        return f.w;
}

struct FwdOut {
    float* color;
    float* log_t;
    float* nd;
    float* normal;
    float* qd;
    float* err;
    float* contrib;
    float* point_err;
    int32_t* early_stop;
    int32_t* tile_contrib_pairs;
    int rpe;
    int* status;
};

template <int G, int PPL, bool GEN = false>
PF_D void fwd_tile(const RasterParams& P, const FwdOut& out, int64_t tile, int wig, int lane, WarpStage& ws,
                   StopState& ss) {
    const int TS = P.TW * P.TW;
    const v3 o = P.cam.eye;
    const float HW = (float)(P.cam.H * P.cam.W);
    const bool want_gt = out.rpe || out.err;
    FwdPix a, b;
    b.g.oob = true;
    b.hit = false;
    b.trans = 1.0f;
#pragma unroll 1
    for (int s = 0; s < PPL; s++) {
        FwdPix& x = a;
        int idx = wig * 32 + lane + s * (TS / 2);
        x.g = pixel_geom(P, tile, idx);
        if constexpr (GEN) pixel_ray_map(P, x.g, x.o);
        x.log_t = 0.f;
        x.trans = 1.0f;
        x.nd = 0.f;
        x.err = 0.f;
        x.rgb = mk(0.f, 0.f, 0.f);
        x.nrm = mk(0.f, 0.f, 0.f);
        x.gt = mk(0.f, 0.f, 0.f);
        x.qi = 0;
        x.q = 0.f;
        x.hit = false;
        x.tn = 0.f;
        x.tf = 0.f;
        if (!x.g.oob) {
            if (P.Q > 0) {
                x.q = P.dq[x.g.px * P.Q];
                for (int q = 0; q < P.Q; q++) out.qd[x.g.px * P.Q + q] = -1.0f;
            }
            if (want_gt) x.gt = mk(P.gt[3 * x.g.px], P.gt[3 * x.g.px + 1], P.gt[3 * x.g.px + 2]);
        }
        if (PPL == 2) swap_pix(a, b);
    }
    // a = pixel idx, b = pixel idx + TS/2
    const int64_t start = P.tile_off[tile];
    const int total = (int)(P.tile_off[tile + 1] - start);
    int es = total;
    int n_contrib_pairs = 0;
    bool stopped = false;
    for (int k0 = 0; k0 < total && !stopped; k0 += 32) {
        stage_prims(ws, P, start, k0, total, lane);
        const int kn = min(32, total - k0);
        for (int kk = 0; kk < kn; kk++) {
            // an out-of-image pixel blocks the stop (rasterize.py:984-990: its
            // transmittance stays 1); a lane without a second pixel does not
            const bool below = (a.g.oob ? false : a.trans < P.thr) &&
                               (PPL == 1 ? true : (b.g.oob ? false : b.trans < P.thr));
            if (stop_vote<G>(ss, wig, lane, k0 + kk, below, out.status)) {
                es = k0 + kk;
                stopped = true;
                break;
            }
            const float4 s4 = ws.sph[kk];
            const v3 center = mk(s4.x, s4.y, s4.z);
            const float radius = s4.w;
            a.hit = a.g.oob ? false : ray_sphere(ray_org<GEN>(a, o), a.g.d, center, radius, a.tn, a.tf);
            if (PPL == 2) b.hit = b.g.oob ? false : ray_sphere(ray_org<GEN>(b, o), b.g.d, center, radius, b.tn, b.tf);
            // The reference skips a primitive no pixel of the tile hits (tile_sum);
            // the skip changes no output, so each warp decides for its own pixels.
            if (!__any_sync(0xffffffffu, a.hit || b.hit)) continue;
            const int32_t prim = ws.pid[kk];
            const float4 n4 = ws.nsg[kk];
            const v3 pn = mk(n4.x, n4.y, n4.z);
            const float sigma = n4.w;
            const int32_t a0 = __ldg(&P.adj_off[prim]);
            const int n_adj = __ldg(&P.adj_off[prim + 1]) - a0;
            const float cc = dot(center, center), rr = radius * radius;
            for (int e0 = 0; e0 < n_adj; e0 += 32) {
                stage_faces(ws, P, a0, e0, n_adj, GEN ? mk(0.f, 0.f, 0.f) : o, center, cc, rr, lane);
                const int en = min(32, n_adj - e0);
#pragma unroll 2
                for (int q = 0; q < en; q++) {
                    const float4 f = ws.face[q];
                    const v3 fn = mk(f.x, f.y, f.z);
                    if (a.hit) {
                        float dp = dot(a.g.d, fn);
                        const float num = face_num<GEN>(f, fn, a);
                        if (face_may_clip(dp, num, a.tn, a.tf)) {
                            float t_face = num / dp;
                            a.tf = dp >= 0.0f ? fmin_t(t_face, a.tf) : a.tf;
                            a.tn = dp < 0.0f ? fmax_t(t_face, a.tn) : a.tn;
                        }
                    }
                    if (PPL == 2 && b.hit) {
                        float dp = dot(b.g.d, fn);
                        const float num = face_num<GEN>(f, fn, b);
                        if (face_may_clip(dp, num, b.tn, b.tf)) {
                            float t_face = num / dp;
                            b.tf = dp >= 0.0f ? fmin_t(t_face, b.tf) : b.tf;
                            b.tn = dp < 0.0f ? fmax_t(t_face, b.tn) : b.tn;
                        }
                    }
                }
                __syncwarp();
            }
            stage_texels(ws, P, prim, lane);
            float c_acc = 0.f, e_acc = 0.f;
#pragma unroll 1
            for (int s = 0; s < PPL; s++) {
                if (a.hit) {
                    PlaneRes pr = plane_fwd_smem(ray_org<GEN>(a, o), a.g.d, a.tn, center, pn, radius, ws, P.S);
                    float tf = pr.dp >= 0.0f ? fmin_t(pr.t_surf, a.tf) : a.tf;
                    float tn = pr.dp < 0.0f ? fmax_t(pr.t_surf, a.tn) : a.tn;
                    float dt = tf - tn;
                    if (dt > 0.0f) {
                        float dlt = -sigma * dt;
                        float alpha = 1.0f - expf(dlt);
                        float trans = a.trans;
                        if (out.err) {
                            v3 de = pr.rgb - a.gt;
                            a.err += dot(de, de) * alpha * trans;
                        }
                        a.rgb = a.rgb + trans * (alpha * pr.rgb);
                        a.log_t += dlt;
                        c_acc += alpha * trans / HW;
                        if (out.rpe) {
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
                            out.qd[a.g.px * P.Q + a.qi] = qd;
                            a.qi += 1;
                            if (a.qi < P.Q) a.q = P.dq[a.g.px * P.Q + a.qi];
                        }
                        a.trans = next_trans;
                    }
                }
                if (PPL == 2) swap_pix(a, b);
            }
            // one atomic per primitive per warp for contrib / point_err
            if (__any_sync(0xffffffffu, c_acc != 0.f || e_acc != 0.f)) {
                n_contrib_pairs++;
                float cs = warp_sum(c_acc);
                float esum = out.rpe ? warp_sum(e_acc) : 0.f;
                if (lane == 0) {
                    atomicAdd(&out.contrib[prim], cs);
                    if (out.rpe) atomicAdd(&out.point_err[prim], esum);
                }
            }
        }
        __syncwarp();
    }
#pragma unroll 1
    for (int s = 0; s < PPL; s++) {
        if (!a.g.oob) {
            int64_t p = a.g.px;
            out.color[3 * p] = a.rgb.x;
            out.color[3 * p + 1] = a.rgb.y;
            out.color[3 * p + 2] = a.rgb.z;
            out.log_t[p] = a.log_t;
            out.nd[p] = a.nd;
            out.normal[3 * p] = a.nrm.x;
            out.normal[3 * p + 1] = a.nrm.y;
            out.normal[3 * p + 2] = a.nrm.z;
            if (out.err) {
                // background is black (rasterize.py:59)
                v3 de = mk(0.f, 0.f, 0.f) - a.gt;
                out.err[p] = a.err + dot(de, de) * expf(a.log_t);
            }
        }
        if (PPL == 2) swap_pix(a, b);
    }
    if (lane == 0 && wig == 0) out.early_stop[tile] = es;
    if (out.tile_contrib_pairs && lane == 0) atomicAdd(&out.tile_contrib_pairs[tile], n_contrib_pairs);
}

// ---------------------------------------------------------------------------
// Forward with (primitive, pixel) hit pairs packed onto the lanes (one pixel
// per lane layouts).  Per batch of 32 staged primitives every lane tests its
// pixel against all of them (hit masks by ballot); the pairs that hit, in
// primitive order, are dealt 32 per round to the lanes, which clip the segment
// by the primitive's faces and evaluate the texture (the costly part, now on
// every lane instead of the ~45 % whose pixel a primitive covers) and leave
// (dt, rgb, t_near) in a two-round ring; after each round every lane
// composites, in primitive order, the pairs of its own pixel for the
// primitives completed so far, with the early-termination vote before each
// primitive exactly as the one-primitive-at-a-time loop.  Each pair is
// evaluated with the same functions on the same operands, so the images are
// bit-identical to fwd_tile's.  Face planes of a sub-batch of primitives
// (<= kFaceCap faces) are staged once; a primitive with more faces than that
// builds them from global memory per pair.
constexpr int kFaceCap = 256;

struct FwdCStage {
    float4 sph[32];     // staged primitives (as WarpStage)
    float4 nsg[32];
    int32_t pid[32];
    float4 face[kFaceCap];
    float4 rec[64];     // per pair: dt, rgb
    float rec_tn[64];   // per pair: segment start (quantile depths)
    float4 dir[32];     // ray direction of each lane's pixel
    uint32_t mask[32];  // hit mask of each staged primitive
    int32_t off[32];    // its first segment record (REC), -1: none
    int pair_off[33];
    int face_off[33];
};

PF_D int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// position of the n-th (0-based) set bit of m (n < popc(m))
PF_D int nth_set_bit(uint32_t m, int n) {
    int pos = 0;
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
        const uint32_t low = m & ((1u << w) - 1u);
        const int c = __popc(low);
        if (n >= c) {
            n -= c;
            m >>= w;
            pos += w;
        } else {
            m = low;
        }
    }
    return pos;
}

// largest j in [0, n) with off[j] <= x (off non-decreasing, off[0] = 0)
PF_D int seg_search(const int* off, int n, int x) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// GEN: per-pixel rays of a generic camera; `org` (32 per warp, shared) then
// holds the pixels' ray origins, and faces are staged with the ray-independent
// face_offset, each pair subtracting its own origin's dot product.
// REC: also write each hit pair's segment record (the sphere interval after
// the power faces and the ids of its bounding surfaces) and each primitive's
// hit mask, which the adjoint reads instead of clipping again (P.seg).
template <int G, bool GEN = false, bool REC = false>
PF_D void fwd_tile_c(const RasterParams& P, const FwdOut& out, int64_t tile, int wig, int lane, FwdCStage& cs,
                     StopState& ss, float4* org = nullptr) {
    const v3 o = P.cam.eye;
    const float HW = (float)(P.cam.H * P.cam.W);
    const bool want_gt = out.rpe || out.err;
    FwdPix a;
    a.g = pixel_geom(P, tile, wig * 32 + lane);
    if constexpr (GEN) pixel_ray_map(P, a.g, a.o);
    a.log_t = 0.f;
    a.trans = 1.0f;
    a.nd = 0.f;
    a.err = 0.f;
    a.rgb = mk(0.f, 0.f, 0.f);
    a.nrm = mk(0.f, 0.f, 0.f);
    a.gt = mk(0.f, 0.f, 0.f);
    a.qi = 0;
    a.q = 0.f;
    if (!a.g.oob) {
        if (P.Q > 0) {
            a.q = P.dq[a.g.px * P.Q];
            for (int q = 0; q < P.Q; q++) out.qd[a.g.px * P.Q + q] = -1.0f;
        }
        if (want_gt) a.gt = mk(P.gt[3 * a.g.px], P.gt[3 * a.g.px + 1], P.gt[3 * a.g.px + 2]);
    }
    cs.dir[lane] = make_float4(a.g.d.x, a.g.d.y, a.g.d.z, 0.f);
    if constexpr (GEN) org[lane] = make_float4(a.o.x, a.o.y, a.o.z, 0.f);
    const uint32_t lt_mask = (1u << lane) - 1u;
    const int64_t start = P.tile_off[tile];
    const int total = (int)(P.tile_off[tile + 1] - start);
    int es = total;
    int n_contrib_pairs = 0;
    bool stopped = false;
    for (int k0 = 0; k0 < total && !stopped; k0 += 32) {
        {
            const int k = k0 + lane;
            if (k < total) {
                const int32_t p = P.tile_prims[start + k];
                cs.pid[lane] = p;
                cs.sph[lane] = __ldg(&P.spheres[p]);
                cs.nsg[lane] = __ldg(&P.nsigmas[p]);
            }
            __syncwarp();
        }
        const int kn = min(32, total - k0);
        for (int kk = 0; kk < kn; kk++) {
            const float4 s4 = cs.sph[kk];
            float tn, tf;
            const bool hit = a.g.oob ? false : ray_sphere(ray_org<GEN>(a, o), a.g.d, mk(s4.x, s4.y, s4.z), s4.w, tn, tf);
            const uint32_t m = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) cs.mask[kk] = m;
        }
        __syncwarp();
        if (REC) {
            // one reservation per 32 primitives: the warp's hit pixels of primitive kk get the
            // records off[kk] + (their rank among its hit pixels)
            const int hits = lane < kn ? __popc(cs.mask[lane]) : 0;
            const int incl = warp_incl_scan(hits, lane);
            const int all = __shfl_sync(0xffffffffu, incl, 31);
            long long base = -1;
            if (lane == 0 && all > 0) {
                const unsigned long long b = atomicAdd(P.seg_count, (unsigned long long)all);
                base = (b + (unsigned long long)all <= (unsigned long long)P.seg_cap) ? (long long)b : -1;
            }
            base = __shfl_sync(0xffffffffu, base, 0);
            if (lane < kn) {
                const int32_t off = base >= 0 ? (int32_t)(base + incl - hits) : -1;
                cs.off[lane] = off;
                const int64_t pi = start + k0 + lane;
                if (pi < P.seg_pairs) {
                    P.seg_mask[pi * G + wig] = cs.mask[lane];
                    P.seg_off[pi * G + wig] = off;
                }
            }
            __syncwarp();
        }
        int kb = 0;
        while (kb < kn && !stopped) {
            // sub-batch [kb, kb + nsub): primitives whose faces fit the staging area
            const int kl = kb + lane;
            int deg = 0;
            if (kl < kn && cs.mask[kl] != 0u) {
                const int32_t pr = cs.pid[kl];
                deg = __ldg(&P.adj_off[pr + 1]) - __ldg(&P.adj_off[pr]);
            }
            const int incl = warp_incl_scan(deg, lane);
            const uint32_t fits = __ballot_sync(0xffffffffu, kl < kn && incl <= kFaceCap);
            const int cnt = __popc(fits);  // a prefix of the lanes
            const bool big = cnt == 0;     // the first primitive alone exceeds the staging area
            const int nsub = big ? 1 : cnt;
            const int np = (lane < nsub) ? __popc(cs.mask[kl]) : 0;
            const int pincl = warp_incl_scan(np, lane);
            if (lane < nsub) {
                cs.face_off[lane] = big ? 0 : incl - deg;
                cs.pair_off[lane] = pincl - np;
            }
            if (lane == nsub - 1) {
                cs.face_off[nsub] = big ? 0 : incl;
                cs.pair_off[nsub] = pincl;
            }
            __syncwarp();
            const int n_faces = cs.face_off[nsub];
            const int n_pairs = cs.pair_off[nsub];
            for (int i = lane; i < n_faces; i += 32) {
                const int j = seg_search(cs.face_off, nsub, i);
                const int kk = kb + j;
                const int32_t pr = cs.pid[kk];
                const float4 s4 = cs.sph[kk];
                const v3 center = mk(s4.x, s4.y, s4.z);
                const int32_t a0 = __ldg(&P.adj_off[pr]);
                const uint2 raw = __ldg(&P.adj_diff[a0 + (i - cs.face_off[j])]);
                const v3 diff = mk(h2f((uint16_t)(raw.x & 0xffffu)), h2f((uint16_t)(raw.x >> 16)),
                                   h2f((uint16_t)(raw.y & 0xffffu)));
                const Face f = make_face(GEN ? mk(0.f, 0.f, 0.f) : o, center, dot(center, center), s4.w * s4.w,
                                         center + diff, h2f((uint16_t)(raw.y >> 16)));
                cs.face[i] = make_float4(f.n.x, f.n.y, f.n.z, f.num);
            }
            __syncwarp();
            int next = 0;  // next primitive of the sub-batch to composite
            for (int base = 0; next < nsub; base += 32) {
                const int j = base + lane;
                if (j < n_pairs) {
                    const int r = seg_search(cs.pair_off, nsub, j);
                    const int kk = kb + r;
                    const int p = nth_set_bit(cs.mask[kk], j - cs.pair_off[r]);
                    const float4 d4 = cs.dir[p];
                    const v3 d = mk(d4.x, d4.y, d4.z);
                    v3 po = o;  // the pair's ray origin
                    if constexpr (GEN) po = mk(org[p].x, org[p].y, org[p].z);
                    const float4 s4 = cs.sph[kk];
                    const v3 center = mk(s4.x, s4.y, s4.z);
                    const float radius = s4.w;
                    const int32_t prim = cs.pid[kk];
                    float tn, tf;
                    ray_sphere(po, d, center, radius, tn, tf);
                    int tn_id = tn < 1e-8f ? -2 : -1, tf_id = tf < 1e-8f ? -2 : -1;  // REC (as the adjoint)
                    if (!big) {
                        const int f0 = cs.face_off[r], f1 = cs.face_off[r + 1];
#pragma unroll 2
                        for (int q = f0; q < f1; q++) {
                            const float4 f = cs.face[q];
                            const v3 fn = mk(f.x, f.y, f.z);
                            const float dp = dot(d, fn);
                            const float num = GEN ? f.w - dot(po, fn) : f.w;
                            if (face_may_clip(dp, num, tn, tf)) {
                                const float t_face = num / dp;
                                if (REC) {
                                    tf_id = (dp >= 0.0f && t_face < tf) ? q - f0 : tf_id;
                                    tn_id = (dp < 0.0f && t_face > tn) ? q - f0 : tn_id;
                                }
                                tf = dp >= 0.0f ? fmin_t(t_face, tf) : tf;
                                tn = dp < 0.0f ? fmax_t(t_face, tn) : tn;
                            }
                        }
                    } else {
                        const int32_t a0 = __ldg(&P.adj_off[prim]);
                        const int32_t a1 = __ldg(&P.adj_off[prim + 1]);
                        const float cc = dot(center, center), rr = radius * radius;
                        for (int32_t e = a0; e < a1; e++) {
                            const uint2 raw = __ldg(&P.adj_diff[e]);
                            const v3 diff = mk(h2f((uint16_t)(raw.x & 0xffffu)), h2f((uint16_t)(raw.x >> 16)),
                                               h2f((uint16_t)(raw.y & 0xffffu)));
                            const Face f = make_face(po, center, cc, rr, center + diff, h2f((uint16_t)(raw.y >> 16)));
                            const float dp = dot(d, f.n);
                            if (face_may_clip(dp, f.num, tn, tf)) {
                                const float t_face = f.num / dp;
                                if (REC) {
                                    tf_id = (dp >= 0.0f && t_face < tf) ? e - a0 : tf_id;
                                    tn_id = (dp < 0.0f && t_face > tn) ? e - a0 : tn_id;
                                }
                                tf = dp >= 0.0f ? fmin_t(t_face, tf) : tf;
                                tn = dp < 0.0f ? fmax_t(t_face, tn) : tn;
                            }
                        }
                    }
                    int64_t rec = -1;  // REC: this pair's record
                    if (REC && cs.off[kk] >= 0) {
                        rec = (int64_t)cs.off[kk] + __popc(cs.mask[kk] & ((1u << p) - 1u));
                        P.seg[rec * P.seg_stride] = make_float4(tn, tf, pack_seg_ids(tn_id, tf_id), 0.f);
                    }
                    if (tn < tf) {  // else the plane, which only shrinks [tn, tf], leaves dt <= 0 (or NaN)
                        const float4 n4 = cs.nsg[kk];
                        const PlaneRes pr = plane_fwd_tex(po, d, tn, center, mk(n4.x, n4.y, n4.z), radius,
                                                          global_texels(P, prim), P.S);
                        if (REC && P.seg_stride == 4 && rec >= 0) store_plane(P.seg + rec * 4, pr);
                        const float tf2 = pr.dp >= 0.0f ? fmin_t(pr.t_surf, tf) : tf;
                        const float tn2 = pr.dp < 0.0f ? fmax_t(pr.t_surf, tn) : tn;
                        cs.rec[j & 63] = make_float4(tf2 - tn2, pr.rgb.x, pr.rgb.y, pr.rgb.z);
                        cs.rec_tn[j & 63] = tn2;
                    } else {
                        cs.rec[j & 63] = make_float4(-1.0f, 0.f, 0.f, 0.f);
                        cs.rec_tn[j & 63] = tn;
                    }
                }
                __syncwarp();
                const int done = min(base + 32, n_pairs);
                while (next < nsub && cs.pair_off[next + 1] <= done) {
                    const int kk = kb + next;
                    const bool below = a.g.oob ? false : a.trans < P.thr;
                    if (stop_vote<G>(ss, wig, lane, k0 + kk, below, out.status)) {
                        es = k0 + kk;
                        stopped = true;
                        break;
                    }
                    const uint32_t m = cs.mask[kk];
                    float c_acc = 0.f, e_acc = 0.f;
                    if ((m >> lane) & 1u) {
                        const int slot = (cs.pair_off[next] + __popc(m & lt_mask)) & 63;
                        const float4 rc = cs.rec[slot];
                        const float dt = rc.x;
                        if (dt > 0.0f) {
                            const v3 prgb = mk(rc.y, rc.z, rc.w);
                            const float tn = cs.rec_tn[slot];
                            const float4 n4 = cs.nsg[kk];
                            const v3 pn = mk(n4.x, n4.y, n4.z);
                            const float sigma = n4.w;
                            float dlt = -sigma * dt;
                            float alpha = 1.0f - expf(dlt);
                            float trans = a.trans;
                            if (out.err) {
                                v3 de = prgb - a.gt;
                                a.err += dot(de, de) * alpha * trans;
                            }
                            a.rgb = a.rgb + trans * (alpha * prgb);
                            a.log_t += dlt;
                            c_acc += alpha * trans / HW;
                            if (out.rpe) {
                                v3 df = prgb - a.gt;
                                float l1 = fabsf(df.x) + fabsf(df.y) + fabsf(df.z);
                                e_acc += alpha * trans * l1 / HW;
                            }
                            float ndv = dot(pn, a.g.d);
                            if (ndv > 0.0f) a.nd += ndv * ndv * alpha * trans;
                            a.nrm = a.nrm + (alpha * trans) * pn;
                            float next_trans = expf(a.log_t);
                            while (a.qi < P.Q && next_trans < a.q) {
                                float qd = tn + logf(trans / a.q) / sigma;
                                out.qd[a.g.px * P.Q + a.qi] = qd;
                                a.qi += 1;
                                if (a.qi < P.Q) a.q = P.dq[a.g.px * P.Q + a.qi];
                            }
                            a.trans = next_trans;
                        }
                    }
                    if (__any_sync(0xffffffffu, c_acc != 0.f || e_acc != 0.f)) {
                        n_contrib_pairs++;
                        float csum = warp_sum(c_acc);
                        float esum = out.rpe ? warp_sum(e_acc) : 0.f;
                        if (lane == 0) {
                            atomicAdd(&out.contrib[cs.pid[kk]], csum);
                            if (out.rpe) atomicAdd(&out.point_err[cs.pid[kk]], esum);
                        }
                    }
                    next++;
                }
                if (stopped) break;
            }
            __syncwarp();
            kb += nsub;
        }
        __syncwarp();
    }
    if (!a.g.oob) {
        const int64_t p = a.g.px;
        out.color[3 * p] = a.rgb.x;
        out.color[3 * p + 1] = a.rgb.y;
        out.color[3 * p + 2] = a.rgb.z;
        out.log_t[p] = a.log_t;
        out.nd[p] = a.nd;
        out.normal[3 * p] = a.nrm.x;
        out.normal[3 * p + 1] = a.nrm.y;
        out.normal[3 * p + 2] = a.nrm.z;
        if (out.err) {
            v3 de = mk(0.f, 0.f, 0.f) - a.gt;
            out.err[p] = a.err + dot(de, de) * expf(a.log_t);
        }
    }
    if (lane == 0 && wig == 0) out.early_stop[tile] = es;
    if (out.tile_contrib_pairs && lane == 0) atomicAdd(&out.tile_contrib_pairs[tile], n_contrib_pairs);
}

// ---------------------------------------------------------------------------
// adjoint
struct BwdPix {
    PixGeom g;
    v3 o;  // ray origin (generic cameras)
    float log_t, dLdlog_t, g_nd;
    v3 g_rgb, g_n;
    int qi;
    float q;
    bool hit;
    float tn, tf;
    int tn_id, tf_id;
};

PF_D void swap_pix(BwdPix& a, BwdPix& b) {
    BwdPix t = a;
    a = b;
    b = t;
}

struct __align__(16) BwdStage {
    float acc[kAccRows][32];     // per-lane gradient columns of the current primitive (rows 16-byte aligned)
    float4 face_acc[kFaceSlots]; // neighbour sphere gradients per neighbour slot
    float4 nbr_sph[kFaceSlots];  // exact neighbour spheres (face adjoint)
    int32_t nbr_id[kFaceSlots];
};

struct GradOut {
    float* points;   // (N,3)
    float* radii;    // (N)
    float* normals;  // (N,3)
    float* density;  // (N)
    float* sites;    // (N,S,3)
    float* rgb;      // (N,S,3)
    float* height;   // (N,S)
};

// row j of the gradient table -> destination in the gradient arrays
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

// Derivative-only arithmetic of the adjoint.  Gradients are compared at a
// relative tolerance (they are sums over pixels and primitives, and the
// reference accumulates them with atomics in arbitrary order), so the
// divisions that only scale derivative values use one reciprocal each.
// Every DECISION of the adjoint (which surface bounds a segment, whether a
// texel site passes w / sum(w) >= 1e-3, the sphere-root sign tests) is still
// taken on the exact operations of the reference.

// rendering_math.py:26-59
PF_D void ray_sphere_bwd_d(v3 eye, v3 dir, v3 c, float r, v3& dn_dc, v3& df_dc, float& dn_dr, float& df_dr) {
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
    float inv_qa = 1.0f / qa, inv_s = 1.0f / s;
    v3 g = (inv_qa * inv_s) * ((2.0f * qa) * oc - qb * dir);
    v3 dq = inv_qa * dir;
    df_dc = dq + g;
    df_dr = 2.0f * r * inv_s;
    if (t_near >= 0.0f) {
        dn_dc = dq - g;
        dn_dr = -df_dr;
    }
}

// rendering_math.py:101-125
PF_D void ray_pface_bwd_d(v3 eye, v3 dir, v3 center, float radius, v3 adj_center, float adj_radius, v3& dc,
                          float& dr, v3& dac, float& dar) {
    v3 face_n = adj_center - center;
    float face_offset = 0.5f * (dot(adj_center, adj_center) - dot(center, center) + radius * radius -
                                adj_radius * adj_radius);
    float num = face_offset - dot(eye, face_n);
    float inv_dp = 1.0f / dot(dir, face_n);
    v3 q = (num * inv_dp * inv_dp) * dir;
    dc = inv_dp * (eye - center) + q;
    dac = inv_dp * (adj_center - eye) - q;
    dr = radius * inv_dp;
    dar = -adj_radius * inv_dp;
}

// rendering_math.py:138-147
PF_D void ray_plane_bwd_d(v3 eye, v3 dir, v3 p, v3 n, float h, v3& dtdp, v3& dtdn, float& dtdh) {
    float dp = dot(n, dir);
    float i1 = 1.0f / (dp + 1e-6f);
    float i2 = 1.0f / (dp * dp + 1e-6f);
    dtdp = i1 * n;
    dtdh = i1;
    dtdn = i1 * (p - eye) - ((dot(p - eye, n) + h) * i2) * dir;
}

// texture.py:74-186, accumulating into this lane's column of bs.acc
// ASSIGN: the gradient table's rows are still zero for this lane (one pixel
// per lane: the first pass writes each colour and site row at most once), so
// they are stored instead of read, added and stored.
template <bool ASSIGN = false>
PF_D void plane_bwd_acc(v3 o, v3 d, float _t_near, v3 po, v3 pn, float radius, const WarpStage& ws, int S,
                        const PlaneRes& pr, v3 dLdrgb_in, float dLdt_surf_in, BwdStage& bs, int lane, v3& dLdpo_out,
                        v3& dLdpn_out, float& dLd_t_near_out) {
    v3 dLdpo = mk(0.f, 0.f, 0.f), dLdpn = mk(0.f, 0.f, 0.f);
    float dLdheight_in = 0.f;
    const float height_in = pr.height, weight_sum = pr.wsum, _weight_sum = pr._wsum;
    const float rr = radius * radius;
    const float inv_rr = 1.0f / rr, inv_ws = 1.0f / weight_sum, inv__ws = 1.0f / _weight_sum;
    float tq = pr.dp >= 0.0f ? _t_near : fmax_t(_t_near, pr.t_surf);
    v3 pt = o + tq * d;
    v3 dLdpt = mk(0.f, 0.f, 0.f);
    float grad_dp_in = dot(dLdrgb_in, pr.rgb);
    const v3 rgb_scale = inv_ws * dLdrgb_in;
#pragma unroll 1
    for (int i = 0; i < S; i++) {
        v3 site = mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]);
        v3 df = pt - site;
        float w = expf(-kTemp * (dot(df, df) / rr));  // texture.py:116-117 (as the forward)
        if (!(w / weight_sum < 1e-3f)) {
            v3 dwds = ((2.0f * kTemp * w) * inv_rr) * df;
            v3 rgb_grad = w * rgb_scale;
            float grad_dp = dot(dLdrgb_in, mk(ws.tr[3 * i], ws.tr[3 * i + 1], ws.tr[3 * i + 2]));
            v3 site_grad = ((grad_dp - grad_dp_in) * inv_ws) * dwds;
            if constexpr (ASSIGN) {
                bs.acc[32 + 3 * i][lane] = rgb_grad.x;
                bs.acc[33 + 3 * i][lane] = rgb_grad.y;
                bs.acc[34 + 3 * i][lane] = rgb_grad.z;
                bs.acc[8 + 3 * i][lane] = site_grad.x;
                bs.acc[9 + 3 * i][lane] = site_grad.y;
                bs.acc[10 + 3 * i][lane] = site_grad.z;
            } else {
                bs.acc[32 + 3 * i][lane] += rgb_grad.x;
                bs.acc[33 + 3 * i][lane] += rgb_grad.y;
                bs.acc[34 + 3 * i][lane] += rgb_grad.z;
                bs.acc[8 + 3 * i][lane] += site_grad.x;
                bs.acc[9 + 3 * i][lane] += site_grad.y;
                bs.acc[10 + 3 * i][lane] += site_grad.z;
            }
            dLdpt = dLdpt - site_grad;
        }
    }
    float dLdt_query = dot(dLdpt, d);
    float dLd_t_near = (pr.dp >= 0.0f || _t_near >= pr.t_surf) ? dLdt_query : 0.0f;
    float dLdt_surf = (pr.dp < 0.0f && _t_near < pr.t_surf) ? dLdt_query : 0.0f;
    dLdt_surf += dLdt_surf_in;
    if (fabsf(dLdt_surf) > 0.0f) {
        v3 ga, gb;
        float gc;
        ray_plane_bwd_d(o, d, po, pn, height_in, ga, gb, gc);
        dLdpo = dLdpo + dLdt_surf * ga;
        dLdpn = dLdpn + dLdt_surf * gb;
        dLdheight_in += gc * dLdt_surf;
    }
    float _tq = pr._dp >= 0.0f ? _t_near : fmax_t(_t_near, pr._t_surf);
    v3 _pt = o + _tq * d;
    v3 dLd_pt = mk(0.f, 0.f, 0.f);
    float _grad_dp_in = dLdheight_in * height_in;
    if (dLdheight_in != 0.0f) {  // every term of this pass is proportional to dLdheight_in
#pragma unroll 1
        for (int i = 0; i < S; i++) {
            v3 site = mk(ws.ts[3 * i], ws.ts[3 * i + 1], ws.ts[3 * i + 2]);
            v3 df = _pt - site;
            float w = expf(-kTemp * (dot(df, df) / rr));  // texture.py:156-157
            if (!(w / weight_sum < 1e-3f)) {
                v3 dwds = ((2.0f * kTemp * w) * inv_rr) * df;
                bs.acc[56 + i][lane] += w * dLdheight_in * inv__ws;
                float _grad_dp = dLdheight_in * ws.th[i];
                v3 site_grad = ((_grad_dp - _grad_dp_in) * inv__ws) * dwds;
                bs.acc[8 + 3 * i][lane] += site_grad.x;
                bs.acc[9 + 3 * i][lane] += site_grad.y;
                bs.acc[10 + 3 * i][lane] += site_grad.z;
                dLd_pt = dLd_pt - site_grad;
            }
        }
    }
    float dLd_t_query = dot(dLd_pt, d);
    dLd_t_near += (pr.dp >= 0.0f || _t_near >= pr._t_surf) ? dLd_t_query : 0.0f;
    float dLd_t_surf = (pr.dp < 0.0f && _t_near < pr._t_surf) ? dLd_t_query : 0.0f;
    if (fabsf(dLd_t_surf) > 0.0f) {
        v3 ga, gb;
        float gc;
        ray_plane_bwd_d(o, d, po, pn, 0.0f, ga, gb, gc);
        dLdpo = dLdpo + dLd_t_surf * ga;
        dLdpn = dLdpn + dLd_t_surf * gb;
    }
    dLdpo_out = dLdpo;
    dLdpn_out = dLdpn;
    dLd_t_near_out = dLd_t_near;
}

struct BwdIn {
    const int32_t* early_stop;
    const float* log_t;
    const float* g_color;
    const float* g_opacity;
    const float* g_nd;
    const float* g_normal;
    const float* g_qd;
    const float* g_contrib;
};

// REC >= 1: the hit masks and the clipped sphere intervals come from the
// forward's segment records (P.seg), so the sphere tests and the face
// clipping are not repeated; REC == 2: the texture-plane results too
// (P.seg_stride == 4).  One pixel per lane only.
// FB: some (pair, warp) may have no records (the forward found the buffer
// full) and is clipped here; without FB every hit has its record, and the
// masks, record offsets and neighbour ranges of the 32 staged primitives are
// staged with them (in the stage's face area, which the clipping alone uses).
// COH: the records were written earlier in the same launch (a fused
// forward + adjoint), so they are read through L2, not the read-only path.
template <int G, int PPL, bool GEN = false, int REC = 0, bool FB = true, bool COH = false>
PF_D void bwd_tile(const RasterParams& P, const BwdIn& in, const GradOut& go, int64_t tile, int wig, int lane,
                   WarpStage& ws, BwdStage& bs) {
    static_assert(!REC || PPL == 1, "segment records are written by the pair-compacted forward");
    // without FB the face area (128 words) holds the staged batch's hit masks, record offsets and
    // neighbour ranges instead
    uint32_t* const st_mask = reinterpret_cast<uint32_t*>(ws.face);
    int32_t* const st_off = reinterpret_cast<int32_t*>(ws.face) + 32;
    int32_t* const st_a0 = reinterpret_cast<int32_t*>(ws.face) + 64;
    int32_t* const st_nadj = reinterpret_cast<int32_t*>(ws.face) + 96;
    static_assert(sizeof(WarpStage::face) >= 128 * sizeof(int32_t), "staging area");
    const int TS = P.TW * P.TW;
    const v3 o = P.cam.eye;
    const float HW = (float)(P.cam.H * P.cam.W);
    const v3 bkgd = mk(0.f, 0.f, 0.f);
    BwdPix a, b;
    b.g.oob = true;
    b.hit = false;
#pragma unroll 1
    for (int s = 0; s < PPL; s++) {
        int idx = wig * 32 + lane + s * (TS / 2);
        a.g = pixel_geom(P, tile, idx);
        if constexpr (GEN) pixel_ray_map(P, a.g, a.o);
        int64_t p = a.g.px;
        a.log_t = in.log_t[p];
        if (P.Q > 0) {
            a.qi = P.Q - 1;
            a.q = P.dq[p * P.Q + P.Q - 1];
        } else {
            a.qi = -1;
            a.q = 1.0f;
        }
        a.g_rgb = mk(in.g_color[3 * p], in.g_color[3 * p + 1], in.g_color[3 * p + 2]);
        // rasterize.py:1905: grad_log_t = -grad_opacity * exp(log_t)
        float g_logt = in.g_opacity ? -in.g_opacity[p] * expf(a.log_t) : 0.f;
        a.g_nd = in.g_nd ? in.g_nd[p] : 0.f;
        a.g_n = in.g_normal ? mk(in.g_normal[3 * p], in.g_normal[3 * p + 1], in.g_normal[3 * p + 2])
                            : mk(0.f, 0.f, 0.f);
        float dLdtrans = dot(a.g_rgb, bkgd);
        a.dLdlog_t = dLdtrans * expf(a.log_t);
        a.dLdlog_t += g_logt;
        a.hit = false;
        a.tn = a.tf = 0.f;
        a.tn_id = a.tf_id = -2;
        if (PPL == 2) swap_pix(a, b);
    }
    const int64_t start = P.tile_off[tile];
    const int es = in.early_stop[tile];
    for (int k1 = es - 1; k1 >= 0; k1 -= 32) {
        const int k0 = k1 - 31;  // batch [k0, k1]; may start below 0
        stage_prims(ws, P, start, k0, es, lane);
        if constexpr (REC && !FB) {
            const int kl = k0 + lane;
            uint32_t m = 0u;
            int32_t off = -1;
            if (kl >= 0 && kl < es && start + kl < P.seg_pairs) {
                m = seg_load<COH>(&P.seg_mask[(start + kl) * G + wig]);
                off = seg_load<COH>(&P.seg_off[(start + kl) * G + wig]);
            }
            st_mask[lane] = m;
            st_off[lane] = off;
            // the records of a (pair, warp) are one contiguous run, most of them still in DRAM:
            // fetched into L2 for the whole batch now (staging them one batch ahead, or the
            // texels too, measured slower)
            if (m != 0u) {
                prefetch_l2_bulk(P.seg + (int64_t)off * P.seg_stride,
                                 (uint32_t)__popc(m) * (uint32_t)P.seg_stride * 16u);
                // the primitive's neighbour range, so that a live primitive's neighbour staging
                // below waits on two dependent loads instead of three
                const int32_t pr = ws.pid[lane];
                const int32_t q0 = __ldg(&P.adj_off[pr]);
                st_a0[lane] = q0;
                st_nadj[lane] = __ldg(&P.adj_off[pr + 1]) - q0;
            }
            __syncwarp();
        }
        for (int k = k1; k >= 0 && k >= k0; k--) {
            const int kk = k - k0;
            const float4 s4 = ws.sph[kk];
            const v3 center = mk(s4.x, s4.y, s4.z);
            const float radius = s4.w;
            int64_t rec = -1;  // REC: this lane's record
            bool clip = !REC;  // warp-uniform: clip and evaluate the plane here
            int32_t nb_pre = 0;  // REC without FB: this lane's neighbour slot id
            if constexpr (REC) {
                uint32_t m = 0u;
                int32_t off = -1;
                if constexpr (FB) {
                    const int64_t pi = start + k;
                    if (pi < P.seg_pairs) {
                        m = seg_load<COH>(&P.seg_mask[pi * G + wig]);
                        off = seg_load<COH>(&P.seg_off[pi * G + wig]);
                    }
                } else {
                    m = st_mask[kk];
                    off = st_off[kk];
                }
                if (m == 0u) continue;  // no output changes (see forward)
                if constexpr (!FB) {  // the first neighbour slots' ids, loaded while the record loads
                    if (lane < min(st_nadj[kk], kFaceSlots)) nb_pre = __ldg(&P.adj[st_a0[kk] + lane]);
                }
                if (!FB || off >= 0) {
                    a.hit = (m >> lane) & 1u;
                    if (a.hit) {
                        rec = (int64_t)off + __popc(m & ((1u << lane) - 1u));
                        const float4 r = seg_load<COH>(&P.seg[rec * P.seg_stride]);
                        a.tn = r.x;
                        a.tf = r.y;
                        unpack_seg_ids(r.z, a.tn_id, a.tf_id);
                    }
                } else if constexpr (FB) {  // the forward found the record buffer full: as without records
                    clip = true;
                    a.hit = a.g.oob ? false : ray_sphere(ray_org<GEN>(a, o), a.g.d, center, radius, a.tn, a.tf);
                }
            } else {
                a.hit = a.g.oob ? false : ray_sphere(ray_org<GEN>(a, o), a.g.d, center, radius, a.tn, a.tf);
                if (PPL == 2)
                    b.hit = b.g.oob ? false : ray_sphere(ray_org<GEN>(b, o), b.g.d, center, radius, b.tn, b.tf);
                if (!__any_sync(0xffffffffu, a.hit || b.hit)) continue;  // no output changes (see forward)
            }
            const int32_t prim = ws.pid[kk];
            const float4 n4 = ws.nsg[kk];
            const v3 pn = mk(n4.x, n4.y, n4.z);
            const float sigma = n4.w;
            int32_t a0;
            int n_adj;
            if constexpr (REC && !FB) {
                a0 = st_a0[kk];
                n_adj = st_nadj[kk];
            } else {
                a0 = __ldg(&P.adj_off[prim]);
                n_adj = __ldg(&P.adj_off[prim + 1]) - a0;
            }
            const float cc = dot(center, center), rr = radius * radius;
            if (clip) {
            a.tn_id = a.tn < 1e-8f ? -2 : -1;
            a.tf_id = a.tf < 1e-8f ? -2 : -1;
            b.tn_id = b.tn < 1e-8f ? -2 : -1;
            b.tf_id = b.tf < 1e-8f ? -2 : -1;
            for (int e0 = 0; e0 < n_adj; e0 += 32) {
                stage_faces(ws, P, a0, e0, n_adj, GEN ? mk(0.f, 0.f, 0.f) : o, center, cc, rr, lane);
                const int en = min(32, n_adj - e0);
#pragma unroll 2
                for (int q = 0; q < en; q++) {
                    const float4 f = ws.face[q];
                    const v3 fn = mk(f.x, f.y, f.z);
                    const int adj_idx = e0 + q;
                    if (a.hit) {
                        float dp = dot(a.g.d, fn);
                        const float num = face_num<GEN>(f, fn, a);
                        if (face_may_clip(dp, num, a.tn, a.tf)) {
                            float t_face = num / dp;
                            a.tf_id = (dp >= 0.0f && t_face < a.tf) ? adj_idx : a.tf_id;
                            a.tf = dp >= 0.0f ? fmin_t(t_face, a.tf) : a.tf;
                            a.tn_id = (dp < 0.0f && t_face > a.tn) ? adj_idx : a.tn_id;
                            a.tn = dp < 0.0f ? fmax_t(t_face, a.tn) : a.tn;
                        }
                    }
                    if (PPL == 2 && b.hit) {
                        float dp = dot(b.g.d, fn);
                        const float num = face_num<GEN>(f, fn, b);
                        if (face_may_clip(dp, num, b.tn, b.tf)) {
                            float t_face = num / dp;
                            b.tf_id = (dp >= 0.0f && t_face < b.tf) ? adj_idx : b.tf_id;
                            b.tf = dp >= 0.0f ? fmin_t(t_face, b.tf) : b.tf;
                            b.tn_id = (dp < 0.0f && t_face > b.tn) ? adj_idx : b.tn_id;
                            b.tn = dp < 0.0f ? fmax_t(t_face, b.tn) : b.tn;
                        }
                    }
                }
                __syncwarp();
            }
            }  // clip
            // The texture plane only shrinks [tn, tf] (and a NaN end never
            // gives dt > 0), so a lane whose faces left tn >= tf adds nothing:
            // with no such lane left the primitive is done (28 % of the hit
            // primitives at 1M primitives, 1080p).
            if (!__any_sync(0xffffffffu, (a.hit && a.tn < a.tf) || (PPL == 2 && b.hit && b.tn < b.tf))) continue;
            // the record's plane part, loaded now so that it arrives during the staging below
            PlaneRes pr_pre;
            if constexpr (REC == 2 && !FB) {
                if (a.hit && a.tn < a.tf) pr_pre = load_plane<COH>(P.seg + rec * 4);
            }
            // the texels and the neighbour slots used by the face adjoint, copied
            // asynchronously so that the texels' latency hides under the neighbour
            // ids' and spheres' (read across lanes after the barrier)
            stage_texels_async(ws, P, prim, lane);
            for (int e = lane; e < min(n_adj, kFaceSlots); e += 32) {
                int32_t nb;
                if constexpr (REC && !FB) nb = nb_pre;  // e == lane (kFaceSlots <= 32)
                else nb = __ldg(&P.adj[a0 + e]);
                bs.nbr_id[e] = nb;
                cp_async16(&bs.nbr_sph[e], &P.spheres[nb]);
                bs.face_acc[e] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            cp_async_wait_all();
            __syncwarp();
            const float cg = in.g_contrib ? __ldg(&in.g_contrib[prim]) : 0.f;
            bool any_contrib = false;
            float g_c0 = 0.f, g_c1 = 0.f, g_c2 = 0.f, g_r = 0.f, g_n0 = 0.f, g_n1 = 0.f, g_n2 = 0.f, g_s = 0.f;
#pragma unroll 1
            for (int s = 0; s < PPL; s++) {
                BwdPix& x = a;
                if (x.hit && x.tn < x.tf) {  // oob pixels never hit here; tn >= tf adds nothing (above)
                    const v3 d = x.g.d;
                    float t_near = x.tn, t_far = x.tf;
                    int t_near_id = x.tn_id, t_far_id = x.tf_id;
                    const float _t_near = t_near;
                    const int _t_near_id = t_near_id, _t_far_id = t_far_id;
                    const v3 xo = ray_org<GEN>(x, o);
                    PlaneRes pr;
                    if (REC == 2 && !FB)
                        pr = pr_pre;
                    else if (REC == 2 && !clip)
                        pr = load_plane<COH>(P.seg + rec * 4);
                    else
                        pr = plane_fwd_smem(xo, d, t_near, center, pn, radius, ws, P.S);
                    t_far_id = (pr.dp >= 0.0f && pr.t_surf < t_far) ? n_adj : t_far_id;
                    t_far = pr.dp >= 0.0f ? fmin_t(pr.t_surf, t_far) : t_far;
                    t_near_id = (pr.dp < 0.0f && pr.t_surf > t_near) ? n_adj : t_near_id;
                    t_near = pr.dp < 0.0f ? fmax_t(pr.t_surf, t_near) : t_near;
                    const float dt = t_far - t_near;
                    if (dt > 0.0f) {  // else plane_bwd(hit=false) and no routing: nothing to add
                        any_contrib = true;
                        float dLdt_near = 0.f, dLdt_far = 0.f, dLdradius = 0.f, dLdsigma = 0.f;
                        v3 dLdcenter = mk(0.f, 0.f, 0.f), dLdnormal = mk(0.f, 0.f, 0.f),
                           dLdcolor = mk(0.f, 0.f, 0.f);
                        {
                            float delta_log_t = -sigma * dt;
                            x.log_t -= delta_log_t;
                            float alpha = 1.0f - expf(delta_log_t);
                            float trans = expf(x.log_t);
                            float ndv = dot(pn, d);
                            float dLdlog_t_i = x.dLdlog_t;
                            float dLddelta_log_t = x.dLdlog_t;
                            float dLdalpha = dot(x.g_rgb, pr.rgb) * trans;
                            if (ndv > 0.0f) dLdalpha += x.g_nd * ndv * trans;
                            dLdalpha += cg * trans / HW;
                            dLdalpha += dot(x.g_n, pn) * trans;
                            float dLdtrans = dot(x.g_rgb, pr.rgb) * alpha;
                            if (ndv > 0.0f) dLdtrans += x.g_nd * ndv * alpha;
                            dLdtrans += cg * alpha / HW;
                            dLdtrans += dot(x.g_n, pn) * alpha;
                            dLdcolor = dLdcolor + alpha * (trans * x.g_rgb);
                            dLdlog_t_i += dLdtrans * expf(x.log_t);
                            dLddelta_log_t += -dLdalpha * expf(delta_log_t);
                            dLdsigma += dLddelta_log_t * -dt;
                            dLdt_near += dLddelta_log_t * sigma;
                            dLdt_far += dLddelta_log_t * -sigma;
                            while (x.qi >= 0 && trans > x.q) {
                                float dq = in.g_qd ? in.g_qd[x.g.px * P.Q + x.qi] : 0.f;
                                dLdsigma += -dq * logf(trans / x.q) / (sigma * sigma + 1e-6f);
                                dLdt_near += dq;
                                dLdlog_t_i += dq / (sigma + 1e-6f);
                                x.qi -= 1;
                                if (x.qi >= 0) x.q = P.dq[x.g.px * P.Q + x.qi];
                            }
                            dLdnormal = dLdnormal + (alpha * trans) * x.g_n;
                            if (ndv > 0.0f) dLdnormal = dLdnormal + (x.g_nd * alpha * trans) * d;
                            x.dLdlog_t = dLdlog_t_i;
                        }
                        float dLdt_surf;
                        if (t_near_id == n_adj) dLdt_surf = dLdt_near;
                        else if (t_far_id == n_adj) dLdt_surf = dLdt_far;
                        else dLdt_surf = 0.0f;
                        v3 _dc, _dn;
                        float dLd_t_near;
                        plane_bwd_acc<PPL == 1>(xo, d, _t_near, center, pn, radius, ws, P.S, pr, dLdcolor, dLdt_surf, bs, lane,
                                      _dc, _dn, dLd_t_near);
                        dLdcenter = dLdcenter + _dc;
                        dLdnormal = dLdnormal + _dn;
                        if (t_near_id != n_adj) dLd_t_near += dLdt_near;
#pragma unroll 1
                        for (int i = 0; i < 2; i++) {
                            const int t_id = i == 0 ? _t_near_id : _t_far_id;
                            const float dLdt = i == 0 ? dLd_t_near : dLdt_far;
                            if (t_id == -1) {
                                v3 ndc, fdc;
                                float ndr, fdr;
                                ray_sphere_bwd_d(xo, d, center, radius, ndc, fdc, ndr, fdr);
                                dLdcenter = dLdcenter + dLdt * (i == 0 ? ndc : fdc);
                                dLdradius += dLdt * (i == 0 ? ndr : fdr);
                            } else if (t_id >= 0 && t_id < n_adj) {
                                int32_t adjacent;
                                float4 as;
                                if (t_id < kFaceSlots) {
                                    adjacent = bs.nbr_id[t_id];
                                    as = bs.nbr_sph[t_id];
                                } else {
                                    adjacent = __ldg(&P.adj[a0 + t_id]);
                                    as = __ldg(&P.spheres[adjacent]);
                                }
                                v3 dc, dac;
                                float dr, dar;
                                ray_pface_bwd_d(xo, d, center, radius, mk(as.x, as.y, as.z), as.w, dc, dr, dac, dar);
                                dLdcenter = dLdcenter + dLdt * dc;
                                dLdradius += dLdt * dr;
                                v3 gac = dLdt * dac;
                                float gar = dLdt * dar;
                                if (t_id < kFaceSlots) {
                                    atomicAdd(&bs.face_acc[t_id].x, gac.x);
                                    atomicAdd(&bs.face_acc[t_id].y, gac.y);
                                    atomicAdd(&bs.face_acc[t_id].z, gac.z);
                                    atomicAdd(&bs.face_acc[t_id].w, gar);
                                } else {
                                    atomicAdd(&go.points[3 * (int64_t)adjacent], gac.x);
                                    atomicAdd(&go.points[3 * (int64_t)adjacent + 1], gac.y);
                                    atomicAdd(&go.points[3 * (int64_t)adjacent + 2], gac.z);
                                    atomicAdd(&go.radii[adjacent], gar);
                                }
                            }
                        }
                        g_c0 += dLdcenter.x;
                        g_c1 += dLdcenter.y;
                        g_c2 += dLdcenter.z;
                        g_r += dLdradius;
                        g_n0 += dLdnormal.x;
                        g_n1 += dLdnormal.y;
                        g_n2 += dLdnormal.z;
                        g_s += dLdsigma;
                    }
                }
                if (PPL == 2) swap_pix(a, b);
            }
            if (__any_sync(0xffffffffu, any_contrib)) {
                bs.acc[0][lane] = g_c0;  // rows 0-7 are written once per primitive (zero before)
                bs.acc[1][lane] = g_c1;
                bs.acc[2][lane] = g_c2;
                bs.acc[3][lane] = g_r;
                bs.acc[4][lane] = g_n0;
                bs.acc[5][lane] = g_n1;
                bs.acc[6][lane] = g_n2;
                bs.acc[7][lane] = g_s;
                __syncwarp();
                // sum rows 2l, 2l+1 over the 32 columns, four at a time (128-bit
                // accesses rotated by lane: each 8-lane phase hits distinct banks),
                // zero them
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = 2 * lane + h;
                    float4* r4 = reinterpret_cast<float4*>(bs.acc[row]);
                    float sum = 0.f;
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const int cc = (c + lane) & 7;
                        const float4 v = r4[cc];
                        sum += v.x;
                        sum += v.y;
                        sum += v.z;
                        sum += v.w;
                        r4[cc] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                    if (sum != 0.0f) {
                        float* dst = grad_slot(go, P.S, prim, row);
                        if (dst) atomicAdd(dst, sum);
                    }
                }
                for (int e = lane; e < min(n_adj, kFaceSlots); e += 32) {
                    float4 f = bs.face_acc[e];
                    if (f.x != 0.f || f.y != 0.f || f.z != 0.f || f.w != 0.f) {
                        int64_t nb = bs.nbr_id[e];
                        atomicAdd(&go.points[3 * nb], f.x);
                        atomicAdd(&go.points[3 * nb + 1], f.y);
                        atomicAdd(&go.points[3 * nb + 2], f.z);
                        atomicAdd(&go.radii[nb], f.w);
                    }
                }
            }
            __syncwarp();
        }
        __syncwarp();
    }
}


}  // namespace pf

// pf_trace.cu -- cell-walk ray tracer (powerfoam/raytrace.py:115-241),
// start-cell search (benchmark.py:320-324) and the SH texel colour pre-step.
//
// One thread per ray, threads laid out tile by tile (8 x 8 rays per two warps)
// as the reference launches them, so neighbouring lanes walk neighbouring
// cells.  The walk is bounded by max_steps; a ray that reaches the cap stops
// and raises PF_ERR_STEP_CAP in the status word instead of looping forever.
#include <algorithm>
#include <type_traits>

#include "pf_common.cuh"
#include "pf_api.h"

namespace pf {

struct TraceParams {
    Cam cam;
    int S;
    int64_t N;
    const float4* spheres;
    const void* nsig;
    const void* sites;
    const void* rgb;
    const void* height;
    const int32_t* adj;
    const int32_t* adj_off;
    const uint2* adj_diff;
    bool tex4;  // f32 texels, S % 4 == 0, 16-byte aligned rows: texels read as float4 groups
    int32_t start_idx;
    const int32_t* start_cells;
    float thr;
    int max_steps;
    float depth_q;
};

template <typename A>
PF_D float ldT(const A* p, int64_t i);
template <>
PF_D float ldT<float>(const float* p, int64_t i) { return __ldg(p + i); }
template <>
PF_D float ldT<__half>(const __half* p, int64_t i) { return __half2float(p[i]); }

// rasterize.py:62-137 / raytrace.py:42-113 plane_intersection_fwd_local
template <typename A>
PF_D PlaneRes plane_local(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const A* sites, const A* rgbs,
                          const A* heights, int S) {
    PlaneRes r;
    float _dp;
    float _t_surf = ray_plane(o, d, po, pn, 0.0f, _dp);
    float _tq = _dp >= 0.0f ? t_near : fmax_t(t_near, _t_surf);
    v3 _pt = o + _tq * d;
    float inv_r2 = 1.0f / (radius * radius);
    float hsum = 0.f, _wsum = 0.f;
    for (int i = 0; i < S; i++) {
        v3 df = _pt - mk(ldT(sites, 3 * i), ldT(sites, 3 * i + 1), ldT(sites, 3 * i + 2));
        float dist_sq = dot(df, df) * inv_r2;
        float w = expf(-kTemp * dist_sq);
        hsum += w * ldT(heights, i);
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
        v3 df = pt - mk(ldT(sites, 3 * i), ldT(sites, 3 * i + 1), ldT(sites, 3 * i + 2));
        float dist_sq = dot(df, df) * inv_r2;
        float w = expf(-kTemp * dist_sq);
        rgb_sum = rgb_sum + w * mk(ldT(rgbs, 3 * i), ldT(rgbs, 3 * i + 1), ldT(rgbs, 3 * i + 2));
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

PF_D float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// plane_local for f32 texels with S % 4 == 0 and 16-byte aligned rows: the
// same arithmetic in the same order, texels fetched four sites at a time.
PF_D PlaneRes plane_local4(v3 o, v3 d, float t_near, v3 po, v3 pn, float radius, const float* sites,
                           const float* rgbs, const float* heights, int S) {
    PlaneRes r;
    float _dp;
    float _t_surf = ray_plane(o, d, po, pn, 0.0f, _dp);
    float _tq = _dp >= 0.0f ? t_near : fmax_t(t_near, _t_surf);
    v3 _pt = o + _tq * d;
    float inv_r2 = 1.0f / (radius * radius);
    float hsum = 0.f, _wsum = 0.f;
    for (int g = 0; g < S; g += 4) {
        const float4 a = ldg4(sites + 3 * g), b = ldg4(sites + 3 * g + 4), c = ldg4(sites + 3 * g + 8);
        const float4 h = ldg4(heights + g);
        const float sx[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
        const float hh[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            v3 df = _pt - mk(sx[3 * u], sx[3 * u + 1], sx[3 * u + 2]);
            float dist_sq = dot(df, df) * inv_r2;
            float w = expf(-kTemp * dist_sq);
            hsum += w * hh[u];
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
    for (int g = 0; g < S; g += 4) {
        const float4 a = ldg4(sites + 3 * g), b = ldg4(sites + 3 * g + 4), c = ldg4(sites + 3 * g + 8);
        const float4 e = ldg4(rgbs + 3 * g), f = ldg4(rgbs + 3 * g + 4), k = ldg4(rgbs + 3 * g + 8);
        const float sx[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
        const float cx[12] = {e.x, e.y, e.z, e.w, f.x, f.y, f.z, f.w, k.x, k.y, k.z, k.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            v3 df = pt - mk(sx[3 * u], sx[3 * u + 1], sx[3 * u + 2]);
            float dist_sq = dot(df, df) * inv_r2;
            float w = expf(-kTemp * dist_sq);
            rgb_sum = rgb_sum + w * mk(cx[3 * u], cx[3 * u + 1], cx[3 * u + 2]);
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

// thread -> pixel in the reference's 8 x 8 tile order
PF_D bool trace_pixel(const Cam& cam, int64_t tid, int& pi, int& pj) {
    int tiles_h = 1 + (cam.H - 1) / 8;
    int64_t tile = tid / 64;
    int l = (int)(tid % 64);
    int ti = (int)(tile % tiles_h), tj = (int)(tile / tiles_h);
    pi = ti * 8 + l % 8;
    pj = tj * 8 + l / 8;
    return pi < cam.H && pj < cam.W;
}

// Segment records of the adjoint (see pf_trace_backward): one per segment
// of a ray (a walked cell with dt > 0), written by the recording forward or
// by the adjoint's own walk.
struct SegRec {
    int32_t cell;
    float tn, tf;
    uint32_t ids;  // tn_id in the low, tf_id in the high 16 bits (|id| < 2^15)
    float trans;
    v3 C, N;
    int32_t seg;
};

PF_D uint32_t pack_ids(int tn_id, int tf_id) { return ((uint32_t)tn_id & 0xffffu) | ((uint32_t)tf_id << 16); }

struct SegWs {
    int64_t n;       // ray slots
    int kb;          // recorded segments per ray
    int32_t* count;  // [n] recorded segments
    float4* rec;     // [kb][n][3]
    int32_t* n_over; // overflow rays
    int32_t* over;   // [n] their slots
    float4* state;   // [n][3] their walk state
};

PF_D void store_rec(float4* p, const SegRec& r) {
    p[0] = make_float4(__int_as_float(r.cell), r.tn, r.tf, __uint_as_float(r.ids));
    p[1] = make_float4(r.trans, r.C.x, r.C.y, r.C.z);
    p[2] = make_float4(r.N.x, r.N.y, r.N.z, __int_as_float(r.seg));
}

// Labels of the ray-proposal network (no counterpart in the reference): the
// first cell after whose compositing the transmittance is below `thr`, the t
// at which the ray enters it and the number of cells walked before it.
struct LabelOut {
    float thr;
    float* t;
    int32_t* cell;
    int32_t* step;
};

// A walk's next cell is a function of its current cell alone (the exit face
// with the smallest t among those the ray leaves through, raytrace.py:183-199),
// so a ray that comes back to a cell repeats the same cells forever.  If none
// of them was a hit (sphere hit, non-empty interval, density >= 1e-3) its
// transmittance never changes and the reference's loop (raytrace.py:162-241)
// never ends: the float16 face planes of neighbouring cells need not agree, so
// a ray running almost along a face can bounce between two cells.  The guard
// keeps the cell of step 0, 1, 2, 4, 8, ... (Brent's power-of-two saves) and
// ends the walk when it returns to that cell with no hit since, as if the ray
// had left the foam.  A ray the reference finishes never returns to a cell
// without a hit in between, so its result is unchanged.  Every walk (forward,
// labels, recording, the adjoint's walk and resume) applies the same guard at
// the same place: after the end tests, before the step.
struct CycleGuard {
    int32_t saved = -1;
    bool hit = false;
};

PF_D bool cycle_closed(CycleGuard& g, int32_t prim, int steps) {
    if (prim == g.saved && !g.hit) return true;
    if ((steps & (steps - 1)) == 0) {
        g.saved = prim;
        g.hit = false;
    }
    return false;
}

// REC: also write the adjoint's segment records (W): up to W.kb per ray, the
// walk state of a ray with more left on W's overflow list for the adjoint's
// resume launch -- the records pf_trace_backward's own walk would write, so
// the adjoint can start at its segment launch.
template <typename A, bool LABELS = false, bool REC = false>
__global__ void __launch_bounds__(128)
trace_fwd_kernel(TraceParams P, int64_t nthreads, float* __restrict__ color, float* __restrict__ log_t_out,
                 float* __restrict__ depth, float* __restrict__ normal, int32_t* __restrict__ depth_seg,
                 float* __restrict__ depth_sigma, int32_t* __restrict__ visit_log, int visit_cap,
                 int32_t* __restrict__ visit_count, int32_t* __restrict__ status, LabelOut lab = LabelOut{},
                 SegWs W = SegWs{}) {
    int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nthreads) return;
    int pi, pj;
    if (!trace_pixel(P.cam, tid, pi, pj)) {
        if (REC) W.count[tid] = 0;
        return;
    }
    const int64_t px = (int64_t)pi * P.cam.W + pj;
    const v3 o = P.cam.eye;
    const v3 d = ray_dir(P.cam, pi, pj);
    const A* nsig = (const A*)P.nsig;
    v3 rgb = mk(0.f, 0.f, 0.f), nacc = mk(0.f, 0.f, 0.f);
    float log_t = 0.f;
    int32_t prim = P.start_cells ? P.start_cells[px] : P.start_idx;
    float pt_near = 0.f;
    int steps = 0, seg = 0, st = PF_OK;
    int32_t dseg = -1;
    float dout = 0.f, dsig = 0.f;
    float lab_t = -1.0f;
    int32_t lab_cell = -1, lab_step = -1;
    int nrec = 0;  // REC: segments recorded
    CycleGuard cg;
    for (;;) {
        float trans = expf(log_t);
        if (trans < P.thr || prim == kNoCell) break;
        if (steps >= P.max_steps) {
            st = PF_ERR_STEP_CAP;
            break;
        }
        if (prim < 0 || prim >= P.N) {
            st = PF_ERR_ARGS;
            break;
        }
        if (REC && nrec == W.kb) {  // the rest of this ray's segments go to the resume launch
            const int32_t k = atomicAdd(W.n_over, 1);
            W.over[k] = (int32_t)tid;
            W.state[3 * (int64_t)k] = make_float4(__int_as_float(prim), __int_as_float(steps), log_t,
                                                   __int_as_float(seg));
            W.state[3 * (int64_t)k + 1] = make_float4(rgb.x, rgb.y, rgb.z, nacc.x);
            W.state[3 * (int64_t)k + 2] = make_float4(nacc.y, nacc.z, __int_as_float(cg.saved),
                                                       __int_as_float((int)cg.hit));
            nrec = W.kb + 1;  // saved once; the walk goes on unrecorded
        }
        if (cycle_closed(cg, prim, steps)) break;
        if (visit_log && steps < visit_cap) visit_log[px * visit_cap + steps] = prim;
        const float cell_entry = pt_near;
        const int32_t cell = prim;
        steps++;
        const float4 s4 = __ldg(&P.spheres[prim]);
        const v3 center = mk(s4.x, s4.y, s4.z);
        const float radius = s4.w;
        float tn, tf;
        bool hit = ray_sphere(o, d, center, radius, tn, tf);
        v3 v = center - o;
        if (length(v) < 4.0f * radius) hit = false;
        int32_t next = kNoCell;
        float pt_far = 1e10f;
        int tn_id = 0, tf_id = 0;  // REC: surfaces bounding the segment (as walk_step)
        if (REC) {
            tn_id = tn < 1e-8f ? -2 : -1;
            tf_id = tf < 1e-8f ? -2 : -1;
        }
        const int32_t a0 = __ldg(&P.adj_off[prim]), a1 = __ldg(&P.adj_off[prim + 1]);
        for (int32_t e = a0; e < a1; e++) {
            uint2 raw = __ldg(&P.adj_diff[e]);
            v3 diff = mk(h2f((uint16_t)(raw.x & 0xffffu)), h2f((uint16_t)(raw.x >> 16)), h2f((uint16_t)(raw.y & 0xffffu)));
            Face f = make_face_pm(o, diff, h2f((uint16_t)(raw.y >> 16)));
            float dp = dot(d, f.n);
            float t_face = f.num / dp;
            if (dp >= 0.0f && t_face < pt_far) {
                next = __ldg(&P.adj[e]);
                pt_far = t_face;
            }
            if (REC) {
                if (dp >= 0.0f && t_face < tf) tf_id = e - a0;
                if (dp < 0.0f && t_face > tn) tn_id = e - a0;
            }
            tf = dp >= 0.0f ? fmin_t(t_face, tf) : tf;
            tn = dp < 0.0f ? fmax_t(t_face, tn) : tn;
        }
        const float pre_tn = tn, pre_tf = tf;
        v3 pn = mk(ldT(nsig, 4 * (int64_t)prim), ldT(nsig, 4 * (int64_t)prim + 1), ldT(nsig, 4 * (int64_t)prim + 2));
        float sigma = ldT(nsig, 4 * (int64_t)prim + 3);
        if (!hit || tn > tf || sigma < 1e-3f) {
            prim = next;
            pt_near = fmax_t(pt_near, pt_far);
            continue;
        }
        cg.hit = true;
        int64_t b3 = (int64_t)prim * P.S * 3;
        PlaneRes pr;
        if constexpr (std::is_same<A, float>::value) {
            if (P.tex4)
                pr = plane_local4(o, d, tn, center, pn, radius, (const float*)P.sites + b3, (const float*)P.rgb + b3,
                                  (const float*)P.height + (int64_t)prim * P.S, P.S);
            else
                pr = plane_local<A>(o, d, tn, center, pn, radius, (const A*)P.sites + b3, (const A*)P.rgb + b3,
                                    (const A*)P.height + (int64_t)prim * P.S, P.S);
        } else {
            pr = plane_local<A>(o, d, tn, center, pn, radius, (const A*)P.sites + b3, (const A*)P.rgb + b3,
                                (const A*)P.height + (int64_t)prim * P.S, P.S);
        }
        tf = pr.dp >= 0.0f ? fmin_t(pr.t_surf, tf) : tf;
        tn = pr.dp < 0.0f ? fmax_t(pr.t_surf, tn) : tn;
        prim = next;
        pt_near = fmax_t(pt_near, pt_far);
        float dt = tf - tn;
        if (dt > 0.0f) {
            float dlt = -sigma * dt;
            float alpha = 1.0f - expf(dlt);
            rgb = rgb + trans * (alpha * pr.rgb);
            nacc = nacc + (alpha * trans) * pn;
            log_t += dlt;
            if (dseg < 0 && expf(log_t) < P.depth_q) {
                dout = tn + logf(trans / P.depth_q) / sigma;
                dseg = seg;
                dsig = sigma;
            }
            if (LABELS && lab_cell < 0 && expf(log_t) < lab.thr) {
                lab_t = cell_entry;
                lab_cell = cell;
                lab_step = steps - 1;
            }
            if (REC && nrec < W.kb) {
                SegRec r;
                r.cell = cell;
                r.tn = pre_tn;
                r.tf = pre_tf;
                r.ids = pack_ids(tn_id, tf_id);
                r.trans = trans;
                r.C = rgb;
                r.N = nacc;
                r.seg = seg;
                store_rec(W.rec + 3 * ((int64_t)nrec * W.n + tid), r);
                nrec++;
            }
            seg++;
        }
    }
    if (REC) W.count[tid] = nrec > W.kb ? W.kb : nrec;
    if (LABELS) {
        lab.t[px] = lab_t;
        lab.cell[px] = lab_cell;
        lab.step[px] = lab_step;
    }
    color[3 * px] = rgb.x;
    color[3 * px + 1] = rgb.y;
    color[3 * px + 2] = rgb.z;
    if (log_t_out) log_t_out[px] = log_t;
    if (depth) depth[px] = dout;
    if (normal) {
        normal[3 * px] = nacc.x;
        normal[3 * px + 1] = nacc.y;
        normal[3 * px + 2] = nacc.z;
    }
    if (depth_seg) depth_seg[px] = dseg;
    if (depth_sigma) depth_sigma[px] = dsig;
    if (visit_count) visit_count[px] = steps;
    if (visit_log)
        for (int k = steps; k < visit_cap; k++) visit_log[px * visit_cap + k] = -1;
    if (st != PF_OK && status) atomicMax(status, st);
}

// ---------------------------------------------------------------------------
// Adjoint of the walk (no counterpart in the reference, whose tracer is
// forward-only).  Per ray the walk is repeated front to back; with the
// forward's final colour C and normal N,
//   dL/d delta_k = gC.(C - C_<=k - c_k T_k+1) + gN.(N - N_<=k - n_k T_k+1)
//                  + gL + [k < m] gD / sigma_m          (delta = -sigma dt)
// where m is the segment that produced the depth.  dL/dt_near and dL/dt_far
// go to the one surface bounding each end (sphere, power face, texture
// plane); face derivatives use the exact spheres; the texture plane's
// derivative covers sites, colours, heights, plane origin and normal, the
// query depth and the radius (through 1/r^2).

// One step of the walk without the texture plane: the cell's sphere and power
// faces bound the segment [tn, tf] (ids: -1 sphere, -2 behind the eye, else
// the face index), `next` is the cell across the nearest exit face.  `hit`
// is false for a cell the ray misses, an empty interval or density < 1e-3.
struct WalkStep {
    bool hit;
    float tn, tf, sigma;
    int tn_id, tf_id;
    int32_t next;
};

PF_D WalkStep walk_step(const TraceParams& P, v3 o, v3 d, int32_t prim) {
    WalkStep w;
    const float4 s4 = __ldg(&P.spheres[prim]);
    const v3 center = mk(s4.x, s4.y, s4.z);
    const float radius = s4.w;
    float tn, tf;
    bool hit = ray_sphere(o, d, center, radius, tn, tf);
    v3 v = center - o;
    if (length(v) < 4.0f * radius) hit = false;
    int tn_id = tn < 1e-8f ? -2 : -1, tf_id = tf < 1e-8f ? -2 : -1;
    int32_t next = kNoCell;
    float pt_far = 1e10f;
    const int32_t a0 = __ldg(&P.adj_off[prim]), a1 = __ldg(&P.adj_off[prim + 1]);
    for (int32_t e = a0; e < a1; e++) {
        uint2 raw = __ldg(&P.adj_diff[e]);
        v3 diff = mk(h2f((uint16_t)(raw.x & 0xffffu)), h2f((uint16_t)(raw.x >> 16)), h2f((uint16_t)(raw.y & 0xffffu)));
        Face f = make_face_pm(o, diff, h2f((uint16_t)(raw.y >> 16)));
        float dp = dot(d, f.n);
        float t_face = f.num / dp;
        if (dp >= 0.0f && t_face < pt_far) {
            next = __ldg(&P.adj[e]);
            pt_far = t_face;
        }
        if (dp >= 0.0f && t_face < tf) tf_id = e - a0;
        tf = dp >= 0.0f ? fmin_t(t_face, tf) : tf;
        if (dp < 0.0f && t_face > tn) tn_id = e - a0;
        tn = dp < 0.0f ? fmax_t(t_face, tn) : tn;
    }
    w.sigma = __ldg((const float*)P.nsig + 4 * (int64_t)prim + 3);
    w.next = next;
    w.tn = tn;
    w.tf = tf;
    w.tn_id = tn_id;
    w.tf_id = tf_id;
    w.hit = hit && !(tn > tf) && !(w.sigma < 1e-3f);
    return w;
}

struct TraceGrads {
    float* points;
    float* radii;
    float* normals;
    float* density;
    float* sites;
    float* rgb;
    float* height;
    bool vec4;  // S % 4 == 0 and the texel gradient arrays 16-byte aligned: float4 atomics
};

PF_D void atomic_add3(float* g, v3 v) {
    atomicAdd(g, v.x);
    atomicAdd(g + 1, v.y);
    atomicAdd(g + 2, v.z);
}

// derivative of the local texture plane; returns dL/d(pre-plane t_near)
PF_D float plane_local_bwd(v3 o, v3 d, float tn, v3 po, v3 pn, float radius, const float* sites, const float* rgbs,
                           const float* heights, int S, const PlaneRes& pr, v3 g_rgb, float g_tsurf, v3& g_po, v3& g_pn,
                           float& g_radius, float* gs, float* gr, float* gh) {
    const float inv_r2 = 1.0f / (radius * radius);
    float g_inv_r2 = 0.f, g_tn = 0.f;
    const float tq = pr.dp >= 0.0f ? tn : fmax_t(tn, pr.t_surf);
    const v3 pt = o + tq * d;
    const float V = pr.wsum, inv_V = 1.0f / pr.wsum;
    const bool v_open = pr.wsum > 1e-20f;
    v3 g_pt = mk(0.f, 0.f, 0.f);
    for (int i = 0; i < S; i++) {
        v3 s = mk(sites[3 * i], sites[3 * i + 1], sites[3 * i + 2]);
        v3 df = pt - s;
        float q2 = dot(df, df);
        float vi = expf(-kTemp * q2 * inv_r2);
        v3 ci = mk(rgbs[3 * i], rgbs[3 * i + 1], rgbs[3 * i + 2]);
        atomic_add3(gr + 3 * i, (vi * inv_V) * g_rgb);
        float g_vi = (v_open ? dot(ci - pr.rgb, g_rgb) : dot(ci, g_rgb)) * inv_V;
        v3 dvdpt = (vi * (-2.0f * kTemp * inv_r2)) * df;
        g_pt = g_pt + g_vi * dvdpt;
        atomic_add3(gs + 3 * i, (-g_vi) * dvdpt);
        g_inv_r2 += g_vi * vi * (-kTemp * q2);
    }
    (void)V;
    float g_tq = dot(g_pt, d);
    float g_ts = g_tsurf;
    if (pr.dp >= 0.0f || tn > pr.t_surf) g_tn += g_tq;
    else g_ts += g_tq;
    float g_height = 0.f;
    if (g_ts != 0.0f) {
        float k = g_ts / pr.dp;
        g_po = g_po + k * pn;
        g_pn = g_pn + k * ((po - o) - pr.t_surf * d);
        g_height = k;
    }
    if (g_height != 0.0f) {
        const float _tq = pr._dp >= 0.0f ? tn : fmax_t(tn, pr._t_surf);
        const v3 _pt = o + _tq * d;
        const float inv_W = 1.0f / pr._wsum;
        const bool w_open = pr._wsum > 1e-20f;
        v3 g__pt = mk(0.f, 0.f, 0.f);
        for (int i = 0; i < S; i++) {
            v3 s = mk(sites[3 * i], sites[3 * i + 1], sites[3 * i + 2]);
            v3 df = _pt - s;
            float q2 = dot(df, df);
            float wi = expf(-kTemp * q2 * inv_r2);
            float hi = heights[i];
            atomicAdd(gh + i, wi * inv_W * g_height);
            float g_wi = (w_open ? (hi - pr.height) : hi) * inv_W * g_height;
            v3 dwdpt = (wi * (-2.0f * kTemp * inv_r2)) * df;
            g__pt = g__pt + g_wi * dwdpt;
            atomic_add3(gs + 3 * i, (-g_wi) * dwdpt);
            g_inv_r2 += g_wi * wi * (-kTemp * q2);
        }
        float g__tq = dot(g__pt, d);
        if (g__tq != 0.0f) {
            if (pr._dp >= 0.0f || tn > pr._t_surf) {
                g_tn += g__tq;
            } else {
                float k = g__tq / pr._dp;
                g_po = g_po + k * pn;
                g_pn = g_pn + k * ((po - o) - pr._t_surf * d);
            }
        }
    }
    g_radius += g_inv_r2 * (-2.0f / (radius * radius * radius));
    return g_tn;
}

PF_D void red4(float* p, const float* v) { atomicAdd((float4*)p, make_float4(v[0], v[1], v[2], v[3])); }

// plane_local_bwd for S a multiple of 4 with 16-byte aligned texel and
// gradient rows: texels are read and their gradients leave as float4 groups
// of four sites, and a site's colour and height terms are summed before its
// atomic (the colour terms are recomputed when the height term is live, i.e.
// when the plane bounds the segment or holds the colour query point).  Every
// other value is computed in plane_local_bwd's order.
PF_D float plane_local_bwd4(v3 o, v3 d, float tn, v3 po, v3 pn, float radius, const float* sites, const float* rgbs,
                            const float* heights, int S, const PlaneRes& pr, v3 g_rgb, float g_tsurf, v3& g_po,
                            v3& g_pn, float& g_radius, float* gs, float* gr, float* gh) {
    const float inv_r2 = 1.0f / (radius * radius);
    float g_inv_r2 = 0.f, g_tn = 0.f;
    const float tq = pr.dp >= 0.0f ? tn : fmax_t(tn, pr.t_surf);
    const v3 pt = o + tq * d;
    const float inv_V = 1.0f / pr.wsum;
    const bool v_open = pr.wsum > 1e-20f;
    const bool on_plane = !(pr.dp >= 0.0f || tn > pr.t_surf);
    const bool height_live = g_tsurf != 0.0f || on_plane;
    v3 g_pt = mk(0.f, 0.f, 0.f);
    for (int g = 0; g < S; g += 4) {
        float rg[12], sg[12];
        const float4 a0 = ldg4(sites + 3 * g), a1 = ldg4(sites + 3 * g + 4), a2 = ldg4(sites + 3 * g + 8);
        const float4 c0 = ldg4(rgbs + 3 * g), c1 = ldg4(rgbs + 3 * g + 4), c2 = ldg4(rgbs + 3 * g + 8);
        const float sx[12] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w};
        const float cx[12] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            v3 s = mk(sx[3 * u], sx[3 * u + 1], sx[3 * u + 2]);
            v3 df = pt - s;
            float q2 = dot(df, df);
            float vi = expf(-kTemp * q2 * inv_r2);
            v3 ci = mk(cx[3 * u], cx[3 * u + 1], cx[3 * u + 2]);
            const v3 a = (vi * inv_V) * g_rgb;
            rg[3 * u] = a.x;
            rg[3 * u + 1] = a.y;
            rg[3 * u + 2] = a.z;
            float g_vi = (v_open ? dot(ci - pr.rgb, g_rgb) : dot(ci, g_rgb)) * inv_V;
            v3 dvdpt = (vi * (-2.0f * kTemp * inv_r2)) * df;
            g_pt = g_pt + g_vi * dvdpt;
            const v3 b = (-g_vi) * dvdpt;
            sg[3 * u] = b.x;
            sg[3 * u + 1] = b.y;
            sg[3 * u + 2] = b.z;
            g_inv_r2 += g_vi * vi * (-kTemp * q2);
        }
        red4(gr + 3 * g, rg);
        red4(gr + 3 * g + 4, rg + 4);
        red4(gr + 3 * g + 8, rg + 8);
        if (!height_live) {
            red4(gs + 3 * g, sg);
            red4(gs + 3 * g + 4, sg + 4);
            red4(gs + 3 * g + 8, sg + 8);
        }
    }
    float g_tq = dot(g_pt, d);
    float g_ts = g_tsurf;
    if (!on_plane) g_tn += g_tq;
    else g_ts += g_tq;
    float g_height = 0.f;
    if (g_ts != 0.0f) {
        float k = g_ts / pr.dp;
        g_po = g_po + k * pn;
        g_pn = g_pn + k * ((po - o) - pr.t_surf * d);
        g_height = k;
    }
    if (height_live) {
        const float _tq = pr._dp >= 0.0f ? tn : fmax_t(tn, pr._t_surf);
        const v3 _pt = o + _tq * d;
        const float inv_W = 1.0f / pr._wsum;
        const bool w_open = pr._wsum > 1e-20f;
        const bool h_on = g_height != 0.0f;
        v3 g__pt = mk(0.f, 0.f, 0.f);
        for (int g = 0; g < S; g += 4) {
            float sg[12], hg[4];
            const float4 a0 = ldg4(sites + 3 * g), a1 = ldg4(sites + 3 * g + 4), a2 = ldg4(sites + 3 * g + 8);
            const float4 c0 = ldg4(rgbs + 3 * g), c1 = ldg4(rgbs + 3 * g + 4), c2 = ldg4(rgbs + 3 * g + 8);
            const float4 h4 = ldg4(heights + g);
            const float sx[12] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w};
            const float cx[12] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w};
            const float hx[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
            for (int u = 0; u < 4; u++) {
                v3 s = mk(sx[3 * u], sx[3 * u + 1], sx[3 * u + 2]);
                v3 df = pt - s;
                float q2 = dot(df, df);
                float vi = expf(-kTemp * q2 * inv_r2);
                v3 ci = mk(cx[3 * u], cx[3 * u + 1], cx[3 * u + 2]);
                float g_vi = (v_open ? dot(ci - pr.rgb, g_rgb) : dot(ci, g_rgb)) * inv_V;
                v3 b = (-g_vi) * ((vi * (-2.0f * kTemp * inv_r2)) * df);
                hg[u] = 0.f;
                if (h_on) {
                    v3 dfw = _pt - s;
                    float q2w = dot(dfw, dfw);
                    float wi = expf(-kTemp * q2w * inv_r2);
                    float hi = hx[u];
                    hg[u] = wi * inv_W * g_height;
                    float g_wi = (w_open ? (hi - pr.height) : hi) * inv_W * g_height;
                    v3 dwdpt = (wi * (-2.0f * kTemp * inv_r2)) * dfw;
                    g__pt = g__pt + g_wi * dwdpt;
                    b = b + (-g_wi) * dwdpt;
                    g_inv_r2 += g_wi * wi * (-kTemp * q2w);
                }
                sg[3 * u] = b.x;
                sg[3 * u + 1] = b.y;
                sg[3 * u + 2] = b.z;
            }
            red4(gs + 3 * g, sg);
            red4(gs + 3 * g + 4, sg + 4);
            red4(gs + 3 * g + 8, sg + 8);
            if (h_on) red4(gh + g, hg);
        }
        float g__tq = dot(g__pt, d);
        if (g__tq != 0.0f) {
            if (pr._dp >= 0.0f || tn > pr._t_surf) {
                g_tn += g__tq;
            } else {
                float k = g__tq / pr._dp;
                g_po = g_po + k * pn;
                g_pn = g_pn + k * ((po - o) - pr._t_surf * d);
            }
        }
    }
    g_radius += g_inv_r2 * (-2.0f / (radius * radius * radius));
    return g_tn;
}

// A segment of the walk: the cell, the interval its sphere and faces bound
// before the texture plane (ids as in WalkStep), the transmittance before
// it, the colour and normal accumulated up to and including it, and its
// index among the ray's segments.

// Per-pixel inputs of the adjoint: the forward's colour / normal / depth
// segment and the loss gradients (any may be null where the reference's
// interface allows it).
struct TraceAdjIn {
    const float* color;
    const float* normal;
    const int32_t* depth_seg;
    const float* depth_sigma;
    const float* g_color;
    const float* g_log_t;
    const float* g_depth;
    const float* g_normal;
};

// Gradients of one segment into every primitive attribute it depends on.
// `pr` is the texture plane of the segment's cell at the pre-plane t_near.
PF_D void segment_adjoint(const TraceParams& P, const TraceAdjIn& A, const TraceGrads& G, v3 o, v3 d, int64_t px,
                          const SegRec& r, const PlaneRes& pr) {
    const int32_t cur = r.cell;
    const float4 s4 = __ldg(&P.spheres[cur]);
    const v3 center = mk(s4.x, s4.y, s4.z);
    const float radius = s4.w;
    const float* ns = (const float*)P.nsig + 4 * (int64_t)cur;
    const v3 pn = mk(__ldg(ns), __ldg(ns + 1), __ldg(ns + 2));
    const float sigma = __ldg(ns + 3);
    const int32_t a0 = __ldg(&P.adj_off[cur]);
    const int n_adj = __ldg(&P.adj_off[cur + 1]) - a0;
    const int pre_tn_id = (int)(int16_t)(r.ids & 0xffffu);
    int tn_id = pre_tn_id, tf_id = (int)r.ids >> 16;
    float tn = r.tn, tf = r.tf;
    if (pr.dp >= 0.0f && pr.t_surf < tf) tf_id = n_adj;
    tf = pr.dp >= 0.0f ? fmin_t(pr.t_surf, tf) : tf;
    if (pr.dp < 0.0f && pr.t_surf > tn) tn_id = n_adj;
    tn = pr.dp < 0.0f ? fmax_t(pr.t_surf, tn) : tn;
    const float dt = tf - tn;
    const float trans = r.trans;
    const v3 gC = A.g_color ? mk(A.g_color[3 * px], A.g_color[3 * px + 1], A.g_color[3 * px + 2]) : mk(0.f, 0.f, 0.f);
    const v3 gN =
        A.g_normal ? mk(A.g_normal[3 * px], A.g_normal[3 * px + 1], A.g_normal[3 * px + 2]) : mk(0.f, 0.f, 0.f);
    const float gL = A.g_log_t ? A.g_log_t[px] : 0.f;
    const float gD = A.g_depth ? A.g_depth[px] : 0.f;
    const int m = A.depth_seg ? A.depth_seg[px] : -1;
    const float sig_m = A.depth_sigma ? A.depth_sigma[px] : 1.f;
    const v3 Cf = mk(A.color[3 * px], A.color[3 * px + 1], A.color[3 * px + 2]);
    const v3 Nf = A.normal ? mk(A.normal[3 * px], A.normal[3 * px + 1], A.normal[3 * px + 2]) : mk(0.f, 0.f, 0.f);
    const float dlt = -sigma * dt;
    const float e = expf(dlt);
    const float alpha = 1.0f - e;
    const v3 c = pr.rgb;
    const float trans_next = trans * e;
    float g_delta = dot(gC, (Cf - r.C) - trans_next * c) + dot(gN, (Nf - r.N) - trans_next * pn) + gL;
    if (m >= 0 && r.seg < m) g_delta += gD / sig_m;
    float g_sigma = -dt * g_delta;
    float g_tf = -sigma * g_delta, g_tn = sigma * g_delta;
    if (r.seg == m) {
        g_tn += gD;
        g_sigma += -gD * logf(trans / P.depth_q) / (sigma * sigma);
    }
    const v3 g_c = (alpha * trans) * gC;
    v3 g_pn = (alpha * trans) * gN;
    v3 g_po = mk(0.f, 0.f, 0.f);
    float g_r = 0.f;
    float g_ts = 0.f;
    if (tn_id == n_adj) {
        g_ts += g_tn;
        g_tn = 0.f;
    }
    if (tf_id == n_adj) {
        g_ts += g_tf;
        g_tf = 0.f;
    }
    const int64_t b3 = (int64_t)cur * P.S * 3;
    const float* ts = (const float*)P.sites + b3;
    const float* tr = (const float*)P.rgb + b3;
    const float* th = (const float*)P.height + (int64_t)cur * P.S;
    float g_pre_tn =
        G.vec4 && P.tex4 ? plane_local_bwd4(o, d, r.tn, center, pn, radius, ts, tr, th, P.S, pr, g_c, g_ts, g_po, g_pn, g_r,
                                  G.sites + b3, G.rgb + b3, G.height + (int64_t)cur * P.S)
               : plane_local_bwd(o, d, r.tn, center, pn, radius, ts, tr, th, P.S, pr, g_c, g_ts, g_po, g_pn, g_r,
                                 G.sites + b3, G.rgb + b3, G.height + (int64_t)cur * P.S);
    if (tn_id != n_adj) g_tn += g_pre_tn;
    const float g_ends[2] = {tn_id == n_adj ? g_pre_tn : g_tn, g_tf};
    const int end_ids[2] = {tn_id == n_adj ? pre_tn_id : tn_id, tf_id};
    v3 g_center = g_po;
    for (int i = 0; i < 2; i++) {
        const float gt = g_ends[i];
        const int id = end_ids[i];
        if (gt == 0.0f) continue;
        if (id == -1) {
            // t = (-qb -+ s)/2, qb = 2 oc.d, s = sqrt(qb^2 - 4(|oc|^2 - r^2)), oc = o - c
            v3 oc = o - center;
            float qb = 2.0f * dot(oc, d);
            float qc = dot(oc, oc) - radius * radius;
            float s = sqrtf(qb * qb - 4.0f * qc);
            v3 ds = (1.0f / (2.0f * s)) * ((-4.0f * qb) * d + 8.0f * oc);
            float sgn = i == 1 ? 1.0f : -1.0f;
            g_center = g_center + gt * (d + (sgn * 0.5f) * ds);
            g_r += gt * (sgn * 2.0f * radius / s);
        } else if (id >= 0 && id < n_adj) {
            const int32_t nb = __ldg(&P.adj[a0 + id]);
            const float4 sj = __ldg(&P.spheres[nb]);
            const v3 cj = mk(sj.x, sj.y, sj.z), ci = center;
            v3 n = cj - ci;
            float num = 0.5f * (dot(cj, cj) - sj.w * sj.w - dot(ci, ci) + radius * radius) - dot(o, n);
            float inv_den = 1.0f / dot(d, n);
            float t = num * inv_den;
            g_center = g_center + (gt * inv_den) * ((o - ci) + t * d);
            g_r += gt * radius * inv_den;
            atomic_add3(G.points + 3 * (int64_t)nb, (gt * inv_den) * ((cj - o) - t * d));
            atomicAdd(G.radii + nb, -gt * sj.w * inv_den);
        }
    }
    atomic_add3(G.points + 3 * (int64_t)cur, g_center);
    atomicAdd(G.radii + cur, g_r);
    atomic_add3(G.normals + 3 * (int64_t)cur, g_pn);
    atomicAdd(G.density + cur, g_sigma);
}

PF_D PlaneRes cell_plane(const TraceParams& P, v3 o, v3 d, int32_t cell, float t_near) {
    const float4 s4 = __ldg(&P.spheres[cell]);
    const float* ns = (const float*)P.nsig + 4 * (int64_t)cell;
    const int64_t b3 = (int64_t)cell * P.S * 3;
    const v3 c = mk(s4.x, s4.y, s4.z), pn = mk(__ldg(ns), __ldg(ns + 1), __ldg(ns + 2));
    const float* ts = (const float*)P.sites + b3;
    const float* tr = (const float*)P.rgb + b3;
    const float* th = (const float*)P.height + (int64_t)cell * P.S;
    return P.tex4 ? plane_local4(o, d, t_near, c, pn, s4.w, ts, tr, th, P.S)
                  : plane_local<float>(o, d, t_near, c, pn, s4.w, ts, tr, th, P.S);
}

// The adjoint runs in three launches over the rays of the trace (thread
// index = pixel slot in the 8 x 8 tile order):
//  1. trace_bwd_walk_kernel repeats the walk of the forward (the same float
//     sequence for transmittance, colour and normal) and records up to
//     `kb` segments per ray in the workspace; a ray with more stops there
//     and leaves its walk state (cell, steps, log T, segment index,
//     accumulated colour / normal) on an overflow list.
//  2. trace_bwd_segment_kernel: the recorded segments, every lane of a warp
//     on one segment index at a time, texture plane recomputed, gradients
//     by atomics.
//  3. trace_bwd_resume_kernel finishes the overflow rays from their saved
//     state (empty list: every warp returns at once).
// Launches 1 and 2 carry no per-ray loop around the gradient work, so the
// walk runs at the forward's register count and occupancy and the gradient
// work on full warps (only about one walked cell in five is a segment).
PF_D SegRec load_rec(const float4* p) {
    const float4 a = p[0], b = p[1], c = p[2];
    SegRec r;
    r.cell = __float_as_int(a.x);
    r.tn = a.y;
    r.tf = a.z;
    r.ids = __float_as_uint(a.w);
    r.trans = b.x;
    r.C = mk(b.y, b.z, b.w);
    r.N = mk(c.x, c.y, c.z);
    r.seg = __float_as_int(c.w);
    return r;
}

__global__ void __launch_bounds__(128)
trace_bwd_walk_kernel(TraceParams P, SegWs W) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= W.n) return;
    int pi, pj;
    if (!trace_pixel(P.cam, tid, pi, pj)) {
        W.count[tid] = 0;
        return;
    }
    const int64_t px = (int64_t)pi * P.cam.W + pj;
    const v3 o = P.cam.eye;
    const v3 d = ray_dir(P.cam, pi, pj);
    v3 Cacc = mk(0.f, 0.f, 0.f), Nacc = mk(0.f, 0.f, 0.f);
    float log_t = 0.f;
    int32_t prim = P.start_cells ? P.start_cells[px] : P.start_idx;
    int steps = 0, seg = 0, nrec = 0;
    CycleGuard cg;
    for (;;) {
        const float trans = expf(log_t);
        if (trans < P.thr || prim == kNoCell || steps >= P.max_steps || prim < 0 || prim >= P.N) break;
        if (nrec == W.kb) {  // the rest of this ray goes to the resume launch
            const int32_t k = atomicAdd(W.n_over, 1);
            W.over[k] = (int32_t)tid;
            W.state[3 * (int64_t)k] = make_float4(__int_as_float(prim), __int_as_float(steps), log_t,
                                                   __int_as_float(seg));
            W.state[3 * (int64_t)k + 1] = make_float4(Cacc.x, Cacc.y, Cacc.z, Nacc.x);
            W.state[3 * (int64_t)k + 2] = make_float4(Nacc.y, Nacc.z, __int_as_float(cg.saved),
                                                       __int_as_float((int)cg.hit));
            break;
        }
        if (cycle_closed(cg, prim, steps)) break;
        steps++;
        const WalkStep ws = walk_step(P, o, d, prim);
        const int32_t cur = prim;
        prim = ws.next;
        if (!ws.hit) continue;
        cg.hit = true;
        const PlaneRes pr = cell_plane(P, o, d, cur, ws.tn);
        const float tf = pr.dp >= 0.0f ? fmin_t(pr.t_surf, ws.tf) : ws.tf;
        const float tn = pr.dp < 0.0f ? fmax_t(pr.t_surf, ws.tn) : ws.tn;
        const float dt = tf - tn;
        if (!(dt > 0.0f)) continue;
        const float* ns = (const float*)P.nsig + 4 * (int64_t)cur;
        const v3 pn = mk(__ldg(ns), __ldg(ns + 1), __ldg(ns + 2));
        const float dlt = -ws.sigma * dt;
        const float alpha = 1.0f - expf(dlt);
        Cacc = Cacc + trans * (alpha * pr.rgb);
        Nacc = Nacc + (alpha * trans) * pn;
        SegRec r;
        r.cell = cur;
        r.tn = ws.tn;
        r.tf = ws.tf;
        r.ids = pack_ids(ws.tn_id, ws.tf_id);
        r.trans = trans;
        r.C = Cacc;
        r.N = Nacc;
        r.seg = seg;
        store_rec(W.rec + 3 * ((int64_t)nrec * W.n + tid), r);
        nrec++;
        log_t += dlt;
        seg++;
    }
    W.count[tid] = nrec;
}

// Grid y = kSegStride: the thread of ray slot `tid` takes its segments
// blockIdx.y, blockIdx.y + kSegStride, ... below its count, so the lanes of
// a warp work on one segment index at a time (as with one block per index)
// without a block launched for every index up to kb.
constexpr int kSegStride = 8;

// 6 resident blocks (80 registers, some spilled): the launch waits mostly on its
// record and texel loads, and 4 blocks at 125 registers left too few warps to hide
// them (trace1m: 7.19 -> 7.14 ms per step; 8 blocks at 64 registers: 7.48 ms)
__global__ void __launch_bounds__(128, 6)
trace_bwd_segment_kernel(TraceParams P, SegWs W, TraceAdjIn A, TraceGrads G) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= W.n) return;
    const int count = W.count[tid];
    if ((int)blockIdx.y >= count) return;
    int pi, pj;
    trace_pixel(P.cam, tid, pi, pj);
    const int64_t px = (int64_t)pi * P.cam.W + pj;
    const v3 o = P.cam.eye;
    const v3 d = ray_dir(P.cam, pi, pj);
    for (int k = blockIdx.y; k < count; k += gridDim.y) {
        const SegRec r = load_rec(W.rec + 3 * ((int64_t)k * W.n + tid));
        segment_adjoint(P, A, G, o, d, px, r, cell_plane(P, o, d, r.cell, r.tn));
    }
}

// Resume launch: each warp takes 32 overflow rays and runs them in rounds.
// Walk: every live lane steps its ray until it holds kTrQueue hit cells
// (sphere and faces give a non-empty interval) or the ray ends.  Texture
// planes: the warp's queued hits, compacted, over all 32 lanes.  Prefix:
// each lane folds its own hits in walk order into the transmittance and
// the accumulated colour / normal, dropping hits after the transmittance
// fell below the threshold.  Gradients: the compacted segments over all
// lanes.
constexpr int kTrQueue = 3;    // queued hits per lane and round
constexpr int kTrItem = 23;    // words per queued hit (odd: conflict-free strides)
constexpr int kTrWarps = 4;    // warps per 128-thread block
// queued hit words
enum : int {
    kQCell = 0, kQTn = 1, kQTf = 2, kQIds = 3, kQSigma = 4,
    kQPr = 5,       // PlaneRes: _t_surf _dp height _wsum t_surf dp wsum rgb.x rgb.y rgb.z (5..14)
    kQTrans = 15, kQC = 16, kQN = 19, kQSeg = 22
};

PF_D void q_store_pr(float* q, const PlaneRes& r) {
    q[kQPr] = r._t_surf;
    q[kQPr + 1] = r._dp;
    q[kQPr + 2] = r.height;
    q[kQPr + 3] = r._wsum;
    q[kQPr + 4] = r.t_surf;
    q[kQPr + 5] = r.dp;
    q[kQPr + 6] = r.wsum;
    q[kQPr + 7] = r.rgb.x;
    q[kQPr + 8] = r.rgb.y;
    q[kQPr + 9] = r.rgb.z;
}

PF_D PlaneRes q_load_pr(const float* q) {
    PlaneRes r;
    r._t_surf = q[kQPr];
    r._dp = q[kQPr + 1];
    r.height = q[kQPr + 2];
    r._wsum = q[kQPr + 3];
    r.t_surf = q[kQPr + 4];
    r.dp = q[kQPr + 5];
    r.wsum = q[kQPr + 6];
    r.rgb = mk(q[kQPr + 7], q[kQPr + 8], q[kQPr + 9]);
    return r;
}

PF_D int warp_incl_scan(int v, int lane) {
    for (int s = 1; s < 32; s <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, s);
        if (lane >= s) v += t;
    }
    return v;
}

constexpr size_t trace_resume_smem() {
    return sizeof(float) * kTrWarps * 32 * (kTrQueue * kTrItem + 4) + sizeof(int) * kTrWarps * 32 * kTrQueue;
}

__global__ void __launch_bounds__(128)
trace_bwd_resume_kernel(TraceParams P, SegWs W, TraceAdjIn A, TraceGrads G) {
    extern __shared__ float tr_smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t first = ((int64_t)blockIdx.x * kTrWarps + w) * 32;  // warp-uniform
    const int n_over = *W.n_over;
    if (first >= n_over) return;
    float* Q = tr_smem + (size_t)w * 32 * kTrQueue * kTrItem;                      // queued hits
    float* R = tr_smem + (size_t)kTrWarps * 32 * kTrQueue * kTrItem + w * 32 * 4;   // per lane: d, px
    int* I = (int*)(tr_smem + (size_t)kTrWarps * 32 * (kTrQueue * kTrItem + 4)) + w * 32 * kTrQueue;
    const int64_t pos = first + lane;
    bool alive = pos < n_over;
    int pi = 0, pj = 0;
    v3 Cacc = mk(0.f, 0.f, 0.f), Nacc = mk(0.f, 0.f, 0.f);
    float log_t = 0.f;
    int32_t prim = kNoCell;
    int steps = 0, seg = 0;
    CycleGuard cg;
    if (alive) {
        trace_pixel(P.cam, W.over[pos], pi, pj);
        const float4 a = W.state[3 * pos], b = W.state[3 * pos + 1], c = W.state[3 * pos + 2];
        prim = __float_as_int(a.x);
        steps = __float_as_int(a.y);
        log_t = a.z;
        seg = __float_as_int(a.w);
        Cacc = mk(b.x, b.y, b.z);
        Nacc = mk(b.w, c.x, c.y);
        cg.saved = __float_as_int(c.z);
        cg.hit = __float_as_int(c.w) != 0;
    }
    const int64_t px = (int64_t)pi * P.cam.W + pj;
    const v3 o = P.cam.eye;
    const v3 d = ray_dir(P.cam, pi, pj);
    R[lane * 4] = d.x;
    R[lane * 4 + 1] = d.y;
    R[lane * 4 + 2] = d.z;
    R[lane * 4 + 3] = __int_as_float((int)px);
    for (;;) {
        // walk until kTrQueue hits are queued or the ray ends
        int cnt = 0;
        while (alive && cnt < kTrQueue) {
            if (expf(log_t) < P.thr || prim == kNoCell || steps >= P.max_steps || prim < 0 || prim >= P.N ||
                cycle_closed(cg, prim, steps)) {
                alive = false;
                break;
            }
            steps++;
            const WalkStep ws = walk_step(P, o, d, prim);
            if (ws.hit) {
                cg.hit = true;
                float* q = Q + (lane * kTrQueue + cnt) * kTrItem;
                q[kQCell] = __int_as_float(prim);
                q[kQTn] = ws.tn;
                q[kQTf] = ws.tf;
                q[kQIds] = __uint_as_float(pack_ids(ws.tn_id, ws.tf_id));
                q[kQSigma] = ws.sigma;
                cnt++;
            }
            prim = ws.next;
        }
        const int incl = warp_incl_scan(cnt, lane);
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        if (total == 0) break;  // a live lane leaves the walk only with a full queue
        for (int k = 0; k < cnt; k++) I[incl - cnt + k] = lane * kTrQueue + k;
        __syncwarp();
        // texture planes of the queued hits, all lanes
        for (int j = lane; j < total; j += 32) {
            const int slot = I[j];
            float* q = Q + slot * kTrItem;
            const float* rr = R + (slot / kTrQueue) * 4;
            q_store_pr(q, cell_plane(P, o, mk(rr[0], rr[1], rr[2]), __float_as_int(q[kQCell]), q[kQTn]));
        }
        __syncwarp();
        // transmittance and accumulated colour / normal, per ray in walk order
        bool opaque = false;  // queued hits past the transmittance threshold are dropped
        for (int k = 0; k < cnt; k++) {
            float* q = Q + (lane * kTrQueue + k) * kTrItem;
            q[kQSeg] = __int_as_float(-1);
            const float trans = expf(log_t);
            if (opaque || trans < P.thr) {
                opaque = true;
                alive = false;
                continue;
            }
            float tn = q[kQTn], tf = q[kQTf];
            const float t_surf = q[kQPr + 4], dp = q[kQPr + 5];
            tf = dp >= 0.0f ? fmin_t(t_surf, tf) : tf;
            tn = dp < 0.0f ? fmax_t(t_surf, tn) : tn;
            const float dt = tf - tn;
            if (!(dt > 0.0f)) continue;
            const int32_t cell = __float_as_int(q[kQCell]);
            const float* ns = (const float*)P.nsig + 4 * (int64_t)cell;
            const v3 pn = mk(__ldg(ns), __ldg(ns + 1), __ldg(ns + 2));
            const float dlt = -q[kQSigma] * dt;
            const float alpha = 1.0f - expf(dlt);
            Cacc = Cacc + trans * (alpha * mk(q[kQPr + 7], q[kQPr + 8], q[kQPr + 9]));
            Nacc = Nacc + (alpha * trans) * pn;
            q[kQTrans] = trans;
            q[kQC] = Cacc.x;
            q[kQC + 1] = Cacc.y;
            q[kQC + 2] = Cacc.z;
            q[kQN] = Nacc.x;
            q[kQN + 1] = Nacc.y;
            q[kQN + 2] = Nacc.z;
            q[kQSeg] = __int_as_float(seg);
            log_t += dlt;
            seg++;
        }
        __syncwarp();
        // gradients of the queued segments, all lanes
        for (int j = lane; j < total; j += 32) {
            const int slot = I[j];
            const float* q = Q + slot * kTrItem;
            SegRec r;
            r.seg = __float_as_int(q[kQSeg]);
            if (r.seg < 0) continue;
            const float* rr = R + (slot / kTrQueue) * 4;
            r.cell = __float_as_int(q[kQCell]);
            r.tn = q[kQTn];
            r.tf = q[kQTf];
            r.ids = __float_as_uint(q[kQIds]);
            r.trans = q[kQTrans];
            r.C = mk(q[kQC], q[kQC + 1], q[kQC + 2]);
            r.N = mk(q[kQN], q[kQN + 1], q[kQN + 2]);
            segment_adjoint(P, A, G, o, mk(rr[0], rr[1], rr[2]), (int64_t)__float_as_int(rr[3]), r, q_load_pr(q));
        }
        __syncwarp();
    }
}

__global__ void trace_zero_nonfinite_kernel(float* __restrict__ a, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float v = a[i];
        if (!isfinite(v)) a[i] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// start cell: argmin_i (|p_i - eye|)^2 - r_i^2, first index on ties.  The
// float is mapped to an order-preserving uint32 and packed above the index,
// so one 64-bit atomicMin per block finds the first minimum.
PF_D uint32_t orderable(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void start_cell_kernel(const float* __restrict__ pts, const float* __restrict__ radii, int64_t N, v3 eye,
                                  unsigned long long* __restrict__ best) {
    __shared__ unsigned long long sb;
    if (threadIdx.x == 0) sb = ~0ull;
    __syncthreads();
    unsigned long long mine = ~0ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        float dx = pts[3 * i] - eye.x, dy = pts[3 * i + 1] - eye.y, dz = pts[3 * i + 2] - eye.z;
        float n = sqrtf(dx * dx + dy * dy + dz * dz);
        float v = n * n - radii[i] * radii[i];
        unsigned long long key = ((unsigned long long)orderable(v) << 32) | (unsigned long long)(uint32_t)i;
        mine = key < mine ? key : mine;
    }
    atomicMin(&sb, mine);
    __syncthreads();
    if (threadIdx.x == 0) atomicMin(best, sb);
}

__global__ void start_cell_finish_kernel(const unsigned long long* __restrict__ best, int32_t* __restrict__ out) {
    *out = (int32_t)(*best & 0xffffffffull);
}

// ---------------------------------------------------------------------------
// degree-3 real SH colour pre-step (constants of powerfoam/sh_utils.py:4-50)
PF_D void sh_basis(v3 dir, float b[16]) {
    const float C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
    const float C2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f, -1.0925484305920792f,
                         0.5462742152960396f};
    const float C3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f, 0.3731763325901154f,
                         -0.4570457994644658f, 1.445305721320277f, -0.5900435899266435f};
    float x = dir.x, y = dir.y, z = dir.z;
    float xx = x * x, yy = y * y, zz = z * z;
    b[0] = C0;
    b[1] = -C1 * y;
    b[2] = C1 * z;
    b[3] = -C1 * x;
    b[4] = C2[0] * (x * y);
    b[5] = C2[1] * (y * z);
    b[6] = C2[2] * (2.0f * zz - xx - yy);
    b[7] = C2[3] * (x * z);
    b[8] = C2[4] * (xx - yy);
    b[9] = C3[0] * y * (3.0f * xx - yy);
    b[10] = C3[1] * (x * y) * z;
    b[11] = C3[2] * y * (4.0f * zz - xx - yy);
    b[12] = C3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    b[13] = C3[4] * x * (4.0f * zz - xx - yy);
    b[14] = C3[5] * z * (xx - yy);
    b[15] = C3[6] * x * (xx - 3.0f * yy);
}

// pre-clamp colour of one channel: sum_k b_k sh[k][ch] + 0.5
PF_D float sh_raw(const float b[16], const float* c, int ch) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) acc += b[k] * c[k * 3 + ch];
    return acc + 0.5f;
}

// vec: sh and out 16-byte aligned and S % 4 == 0 -- the 48 coefficients are
// read as 12 float4 and the S x 3 broadcast colours written as float4 (the
// same sums in the same order either way)
__global__ void sh_texel_rgb_kernel(const float* __restrict__ pts, const float* __restrict__ sh, int64_t N, int S,
                                    v3 eye, float* __restrict__ out, bool vec) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    float b[16];
    sh_basis(normalize(mk(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]) - eye), b);
    float c[48];
    if (vec) {
        const float4* c4 = reinterpret_cast<const float4*>(sh + p * 48);
#pragma unroll
        for (int i = 0; i < 12; i++) {
            const float4 v = __ldg(c4 + i);
            c[4 * i] = v.x;
            c[4 * i + 1] = v.y;
            c[4 * i + 2] = v.z;
            c[4 * i + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 48; i++) c[i] = __ldg(sh + p * 48 + i);
    }
    float rgb[3];
#pragma unroll
    for (int ch = 0; ch < 3; ch++) {
        const float acc = sh_raw(b, c, ch);
        rgb[ch] = acc > 0.0f ? acc : 0.0f;
    }
    if (vec) {
        float4* o4 = reinterpret_cast<float4*>(out + p * S * 3);
        for (int q = 0; q < 3 * S / 4; q++) {
            const int e = 4 * q;  // element e of the row is channel e % 3
            o4[q] = make_float4(rgb[e % 3], rgb[(e + 1) % 3], rgb[(e + 2) % 3], rgb[(e + 3) % 3]);
        }
    } else {
        for (int s = 0; s < S; s++)
            for (int ch = 0; ch < 3; ch++) out[(p * S + s) * 3 + ch] = rgb[ch];
    }
}

// adjoint with respect to the coefficients: the colour is broadcast to the S
// sites, so its gradient is the sum over sites; the clamp passes it where the
// pre-clamp value is positive.  Accumulates into grad_sh.
__global__ void sh_texel_rgb_bwd_kernel(const float* __restrict__ pts, const float* __restrict__ sh, int64_t N,
                                        int S, v3 eye, const float* __restrict__ g_rgb, float* __restrict__ g_sh) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    float b[16];
    sh_basis(normalize(mk(pts[3 * p], pts[3 * p + 1], pts[3 * p + 2]) - eye), b);
    const float* c = sh + p * 48;
    for (int ch = 0; ch < 3; ch++) {
        if (!(sh_raw(b, c, ch) > 0.0f)) continue;
        float g = 0.f;
        for (int s = 0; s < S; s++) g += g_rgb[(p * S + s) * 3 + ch];
#pragma unroll
        for (int k = 0; k < 16; k++) g_sh[p * 48 + k * 3 + ch] += b[k] * g;
    }
}

}  // namespace pf

using namespace pf;

extern "C" int pf_trace_forward(const pf_trace_inputs* in, float* color, float* log_t, float* depth, float* normal,
                                int32_t* depth_seg, float* depth_sigma, int32_t* visit_log, int32_t visit_cap,
                                int32_t* visit_count, int32_t* status, void* stream) {
    if (!in || !color) return pf_fail(PF_ERR_ARGS, "pf_trace_forward: missing argument");
    if (in->cam.width < 2 || in->cam.height < 2) return pf_fail(PF_ERR_ARGS, "image must be at least 2x2");
    if (in->n_sites < 0 || in->n_sites > kMaxSites) return pf_fail(PF_ERR_ARGS, "n_sites must be in [0, 8]");
    if (in->max_steps <= 0) return pf_fail(PF_ERR_ARGS, "max_steps must be positive");
    if (visit_log && visit_cap <= 0) return pf_fail(PF_ERR_ARGS, "visit_cap must be positive with a visit log");
    if (in->n_prims <= 0) return pf_fail(PF_ERR_ARGS, "pf_trace_forward: no primitives");
    if (!in->start_cells && (in->start_idx < 0 || in->start_idx >= in->n_prims) && in->start_idx != kNoCell)
        return pf_fail(PF_ERR_ARGS, "start_idx out of range");
    TraceParams P;
    P.cam = load_cam(in->cam);
    P.S = in->n_sites;
    P.N = in->n_prims;
    P.spheres = (const float4*)in->spheres;
    P.nsig = in->nsigmas;
    P.sites = in->texel_sites;
    P.rgb = in->texel_rgb;
    P.height = in->texel_height;
    P.adj = in->adjacency;
    P.adj_off = in->adjacency_offsets;
    P.adj_diff = (const uint2*)in->adjacency_diff;
    P.tex4 = !in->attr_half && in->n_sites % 4 == 0 && ((uintptr_t)in->texel_sites % 16) == 0 &&
             ((uintptr_t)in->texel_rgb % 16) == 0 && ((uintptr_t)in->texel_height % 16) == 0;
    P.start_idx = in->start_idx;
    P.start_cells = in->start_cells;
    P.thr = in->transmittance_threshold;
    P.max_steps = in->max_steps;
    P.depth_q = in->depth_quantile;
    int64_t tiles = (int64_t)(1 + (in->cam.height - 1) / 8) * (1 + (in->cam.width - 1) / 8);
    int64_t n = tiles * 64;
    unsigned grid = (unsigned)((n + 127) / 128);
    cudaStream_t st = (cudaStream_t)stream;
    if (in->attr_half)
        trace_fwd_kernel<__half><<<grid, 128, 0, st>>>(P, n, color, log_t, depth, normal, depth_seg, depth_sigma,
                                                       visit_log, visit_cap, visit_count, status);
    else
        trace_fwd_kernel<float><<<grid, 128, 0, st>>>(P, n, color, log_t, depth, normal, depth_seg, depth_sigma,
                                                      visit_log, visit_cap, visit_count, status);
    return pf_check_launch("pf_trace_forward");
}

static bool fill_trace(const pf_trace_inputs* in, TraceParams& P, const char** why);

extern "C" int pf_trace_labels(const pf_trace_inputs* in, float label_threshold, float* color, float* label_t,
                               int32_t* label_cell, int32_t* label_step, int32_t* visit_count, int32_t* status,
                               void* stream) {
    TraceParams P;
    const char* why = "";
    if (!fill_trace(in, P, &why)) return pf_fail(PF_ERR_ARGS, why);
    if (in->attr_half) return pf_fail(PF_ERR_ARGS, "pf_trace_labels: attributes must be f32");
    if (!color || !label_t || !label_cell || !label_step)
        return pf_fail(PF_ERR_ARGS, "pf_trace_labels: missing output");
    const int64_t tiles = (int64_t)(1 + (P.cam.H - 1) / 8) * (1 + (P.cam.W - 1) / 8);
    const int64_t n = tiles * 64;
    const unsigned grid = (unsigned)((n + 127) / 128);
    LabelOut lab{label_threshold, label_t, label_cell, label_step};
    trace_fwd_kernel<float, true><<<grid, 128, 0, (cudaStream_t)stream>>>(
        P, n, color, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, visit_count, status, lab);
    return pf_check_launch("pf_trace_labels");
}

static bool fill_trace(const pf_trace_inputs* in, TraceParams& P, const char** why) {
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
    if (in->max_steps <= 0) {
        *why = "max_steps must be positive";
        return false;
    }
    if (in->n_prims <= 0) {
        *why = "no primitives";
        return false;
    }
    if (!in->start_cells && (in->start_idx < 0 || in->start_idx >= in->n_prims) && in->start_idx != kNoCell) {
        *why = "start_idx out of range";
        return false;
    }
    P.cam = load_cam(in->cam);
    P.S = in->n_sites;
    P.N = in->n_prims;
    P.spheres = (const float4*)in->spheres;
    P.nsig = in->nsigmas;
    P.sites = in->texel_sites;
    P.rgb = in->texel_rgb;
    P.height = in->texel_height;
    P.adj = in->adjacency;
    P.adj_off = in->adjacency_offsets;
    P.adj_diff = (const uint2*)in->adjacency_diff;
    P.tex4 = !in->attr_half && in->n_sites % 4 == 0 && ((uintptr_t)in->texel_sites % 16) == 0 &&
             ((uintptr_t)in->texel_rgb % 16) == 0 && ((uintptr_t)in->texel_height % 16) == 0;
    P.start_idx = in->start_idx;
    P.start_cells = in->start_cells;
    P.thr = in->transmittance_threshold;
    P.max_steps = in->max_steps;
    P.depth_q = in->depth_quantile;
    return true;
}

// Workspace of the adjoint for `kb` recorded segments per ray: counts,
// records (48 B per segment slot), overflow list and states.
static size_t seg_ws_layout(int64_t n, int kb, size_t off[5]) {
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t o = 0;
    off[0] = o;  o = up(o + sizeof(int32_t) * n);                 // count
    off[1] = o;  o = up(o + sizeof(float4) * 3 * n * (size_t)kb); // records
    off[2] = o;  o = up(o + sizeof(int32_t));                     // n_over
    off[3] = o;  o = up(o + sizeof(int32_t) * n);                 // over
    off[4] = o;  o = up(o + sizeof(float4) * 3 * n);              // state
    return o;
}

static int64_t trace_slots(const pf_trace_inputs* in) {
    return (int64_t)(1 + (in->cam.height - 1) / 8) * (1 + (in->cam.width - 1) / 8) * 64;
}

extern "C" int pf_trace_backward_workspace_size(const pf_trace_inputs* in, int32_t segments_per_ray, size_t* bytes) {
    if (!in || !bytes || segments_per_ray < 0 || segments_per_ray > 65535 || in->cam.width <= 0 ||
        in->cam.height <= 0)
        return pf_fail(PF_ERR_ARGS, "pf_trace_backward_workspace_size: bad arguments");
    size_t off[5];
    *bytes = seg_ws_layout(trace_slots(in), segments_per_ray, off);
    return PF_OK;
}

static SegWs seg_ws(const pf_trace_inputs* in, int kb, void* workspace) {
    const int64_t n = trace_slots(in);
    size_t off[5];
    seg_ws_layout(n, kb, off);
    char* ws = (char*)workspace;
    return SegWs{n, kb, (int32_t*)(ws + off[0]), (float4*)(ws + off[1]), (int32_t*)(ws + off[2]),
                 (int32_t*)(ws + off[3]), (float4*)(ws + off[4])};
}

static int check_seg_ws(const pf_trace_inputs* in, int32_t segments_per_ray, const void* workspace,
                        size_t workspace_bytes, const char* who) {
    size_t need = 0;
    if (pf_trace_backward_workspace_size(in, segments_per_ray, &need) != PF_OK) return PF_ERR_ARGS;
    if (!workspace || workspace_bytes < need || ((uintptr_t)workspace & 255))
        return pf_fail(PF_ERR_ARGS, who);
    return PF_OK;
}

// walk = true: the adjoint's own recording walk first; false: the records of
// pf_trace_forward_record are in the workspace already
static int trace_backward_impl(const pf_trace_inputs* in, const float* color, const float* normal,
                               const int32_t* depth_seg, const float* depth_sigma, const float* grad_color,
                               const float* grad_log_t, const float* grad_depth, const float* grad_normal,
                               float* grad_points, float* grad_radii, float* grad_normals, float* grad_density,
                               float* grad_texel_sites, float* grad_texel_rgb, float* grad_texel_height,
                               int32_t segments_per_ray, void* workspace, size_t workspace_bytes, void* stream,
                               bool walk) {
    TraceParams P;
    const char* why = "";
    if (!fill_trace(in, P, &why)) return pf_fail(PF_ERR_ARGS, why);
    if (in->attr_half) return pf_fail(PF_ERR_ARGS, "Backward pass only supports float precision");
    if (!color || !grad_points || !grad_radii || !grad_normals || !grad_density || !grad_texel_sites ||
        !grad_texel_rgb || !grad_texel_height || (grad_depth && (!depth_seg || !depth_sigma)) ||
        (grad_normal && !normal))
        return pf_fail(PF_ERR_ARGS, "pf_trace_backward: missing argument");
    if (check_seg_ws(in, segments_per_ray, workspace, workspace_bytes,
                     "pf_trace_backward: workspace missing, too small or not 256-byte aligned") != PF_OK)
        return PF_ERR_ARGS;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t N = (size_t)P.N, S = (size_t)P.S;
    float* outs[7] = {grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites, grad_texel_rgb,
                      grad_texel_height};
    size_t lens[7] = {3 * N, N, 3 * N, N, 3 * N * S, 3 * N * S, N * S};
    for (int i = 0; i < 7; i++)
        if (lens[i]) cudaMemsetAsync(outs[i], 0, sizeof(float) * lens[i], st);
    const bool vec4 = (P.S % 4) == 0 && ((uintptr_t)grad_texel_sites % 16) == 0 &&
                      ((uintptr_t)grad_texel_rgb % 16) == 0 && ((uintptr_t)grad_texel_height % 16) == 0;
    TraceGrads G{grad_points,      grad_radii,     grad_normals,      grad_density,
                 grad_texel_sites, grad_texel_rgb, grad_texel_height, vec4};
    TraceAdjIn A{color, normal, depth_seg, depth_sigma, grad_color, grad_log_t, grad_depth, grad_normal};
    const SegWs W = seg_ws(in, segments_per_ray, workspace);
    const unsigned blocks = (unsigned)((W.n + 127) / 128);
    if (walk) {
        cudaMemsetAsync(W.n_over, 0, sizeof(int32_t), st);
        trace_bwd_walk_kernel<<<blocks, 128, 0, st>>>(P, W);
    }
    if (segments_per_ray > 0)
        trace_bwd_segment_kernel<<<dim3(blocks, std::min(segments_per_ray, kSegStride)), 128, 0, st>>>(P, W, A, G);
    static_assert(trace_resume_smem() <= 48 * 1024, "resume queue above the default shared-memory limit");
    trace_bwd_resume_kernel<<<blocks, 128, trace_resume_smem(), st>>>(P, W, A, G);
    for (int i = 0; i < 7; i++)
        if (lens[i]) {
            int64_t k = (int64_t)lens[i];
            trace_zero_nonfinite_kernel<<<(unsigned)std::min<int64_t>((k + 255) / 256, 148 * 16), 256, 0, st>>>(
                outs[i], k);
        }
    return pf_check_launch("pf_trace_backward");
}

extern "C" int pf_trace_backward(const pf_trace_inputs* in, const float* color, const float* normal,
                                 const int32_t* depth_seg, const float* depth_sigma, const float* grad_color,
                                 const float* grad_log_t, const float* grad_depth, const float* grad_normal,
                                 float* grad_points, float* grad_radii, float* grad_normals, float* grad_density,
                                 float* grad_texel_sites, float* grad_texel_rgb, float* grad_texel_height,
                                 int32_t segments_per_ray, void* workspace, size_t workspace_bytes, void* stream) {
    return trace_backward_impl(in, color, normal, depth_seg, depth_sigma, grad_color, grad_log_t, grad_depth,
                               grad_normal, grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites,
                               grad_texel_rgb, grad_texel_height, segments_per_ray, workspace, workspace_bytes,
                               stream, true);
}

extern "C" int pf_trace_backward_recorded(const pf_trace_inputs* in, const float* color, const float* normal,
                                          const int32_t* depth_seg, const float* depth_sigma,
                                          const float* grad_color, const float* grad_log_t, const float* grad_depth,
                                          const float* grad_normal, float* grad_points, float* grad_radii,
                                          float* grad_normals, float* grad_density, float* grad_texel_sites,
                                          float* grad_texel_rgb, float* grad_texel_height, int32_t segments_per_ray,
                                          const void* workspace, size_t workspace_bytes, void* stream) {
    return trace_backward_impl(in, color, normal, depth_seg, depth_sigma, grad_color, grad_log_t, grad_depth,
                               grad_normal, grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites,
                               grad_texel_rgb, grad_texel_height, segments_per_ray, const_cast<void*>(workspace),
                               workspace_bytes, stream, false);
}

extern "C" int pf_trace_forward_record(const pf_trace_inputs* in, float* color, float* log_t, float* depth,
                                       float* normal, int32_t* depth_seg, float* depth_sigma, int32_t* visit_count,
                                       int32_t* status, int32_t segments_per_ray, void* workspace,
                                       size_t workspace_bytes, void* stream) {
    TraceParams P;
    const char* why = "";
    if (!fill_trace(in, P, &why)) return pf_fail(PF_ERR_ARGS, why);
    if (in->attr_half) return pf_fail(PF_ERR_ARGS, "pf_trace_forward_record: attributes must be f32");
    if (!color) return pf_fail(PF_ERR_ARGS, "pf_trace_forward_record: missing argument");
    if (check_seg_ws(in, segments_per_ray, workspace, workspace_bytes,
                     "pf_trace_forward_record: workspace missing, too small or not 256-byte aligned") != PF_OK)
        return PF_ERR_ARGS;
    cudaStream_t st = (cudaStream_t)stream;
    const SegWs W = seg_ws(in, segments_per_ray, workspace);
    cudaMemsetAsync(W.n_over, 0, sizeof(int32_t), st);
    const unsigned grid = (unsigned)((W.n + 127) / 128);
    trace_fwd_kernel<float, false, true><<<grid, 128, 0, st>>>(P, W.n, color, log_t, depth, normal, depth_seg,
                                                              depth_sigma, nullptr, 0, visit_count, status,
                                                              LabelOut{}, W);
    return pf_check_launch("pf_trace_forward_record");
}

extern "C" int pf_start_cell_workspace_size(int64_t n_prims, size_t* bytes) {
    if (!bytes || n_prims < 0) return pf_fail(PF_ERR_ARGS, "pf_start_cell_workspace_size: bad arguments");
    *bytes = 256;
    return PF_OK;
}

extern "C" int pf_start_cell(const float* points, const float* radii, int64_t n_prims, const float* eye_host,
                             void* workspace, size_t workspace_bytes, int32_t* out_idx, void* stream) {
    if (n_prims <= 0 || !points || !radii || !eye_host || !out_idx || !workspace || workspace_bytes < 8)
        return pf_fail(PF_ERR_ARGS, "pf_start_cell: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long* best = (unsigned long long*)workspace;
    cudaMemsetAsync(best, 0xff, 8, st);
    unsigned grid = (unsigned)std::min<int64_t>((n_prims + 255) / 256, 148 * 8);
    start_cell_kernel<<<grid, 256, 0, st>>>(points, radii, n_prims, mk(eye_host[0], eye_host[1], eye_host[2]), best);
    start_cell_finish_kernel<<<1, 1, 0, st>>>(best, out_idx);
    return pf_check_launch("pf_start_cell");
}

extern "C" int pf_sh_texel_rgb(const float* points, const float* sh, int64_t n_prims, int32_t n_sites,
                               const float* eye_host, float* texel_rgb, void* stream) {
    if (n_prims < 0 || n_sites < 0 || !eye_host || (n_prims > 0 && (!points || !sh || !texel_rgb)))
        return pf_fail(PF_ERR_ARGS, "pf_sh_texel_rgb: bad arguments");
    if (n_prims == 0) return PF_OK;
    const bool vec = n_sites % 4 == 0 && ((uintptr_t)sh % 16) == 0 && ((uintptr_t)texel_rgb % 16) == 0;
    sh_texel_rgb_kernel<<<(unsigned)((n_prims + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        points, sh, n_prims, n_sites, mk(eye_host[0], eye_host[1], eye_host[2]), texel_rgb, vec);
    return pf_check_launch("pf_sh_texel_rgb");
}

extern "C" int pf_sh_texel_rgb_backward(const float* points, const float* sh, int64_t n_prims, int32_t n_sites,
                                        const float* eye_host, const float* grad_texel_rgb, float* grad_sh,
                                        void* stream) {
    if (n_prims < 0 || n_sites < 0 || !eye_host || (n_prims > 0 && (!points || !sh || !grad_texel_rgb || !grad_sh)))
        return pf_fail(PF_ERR_ARGS, "pf_sh_texel_rgb_backward: bad arguments");
    if (n_prims == 0) return PF_OK;
    sh_texel_rgb_bwd_kernel<<<(unsigned)((n_prims + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        points, sh, n_prims, n_sites, mk(eye_host[0], eye_host[1], eye_host[2]), grad_texel_rgb, grad_sh);
    return pf_check_launch("pf_sh_texel_rgb_backward");
}

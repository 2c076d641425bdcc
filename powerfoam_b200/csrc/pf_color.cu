// pf_color.cu -- spherical-Voronoi texel colour (forward and adjoint).
//
// Replaces spherical_voronoi_fwd_kernel / spherical_voronoi_bwd_kernel of
// SphericalVoronoi (powerfoam/color_fn.py:54-184, host side :186-315).  Per
// texel point p with view direction d = normalize(p - eye):
//     w_i = exp(-temp_i |d - axis_i|),  colour = max(sum w_i val_i / sum w_i + 0.5, 0)
// over its sv_dof sites, or 0.5 grey with weight sum 0 outside the camera
// cone (d . forward < fov_cos_cutoff).  The adjoint writes every site's
// gradients: zero for sites whose normalised weight is below 1e-3 and for
// points outside the cone (the reference leaves its zero-initialised outputs
// there), the derivatives elsewhere; the points receive none (the
// reference's point gradient is disabled).  Float32 arithmetic in the
// reference's order; attributes may be float32 or float16 (then read and
// written rounded as the reference's half kernels do).  One thread per
// point; the site arrays are (sv_dof, N, ...), so a warp reads contiguous
// 384-byte runs.  The kernels stream 28 bytes per site (f32) and are
// HBM-bound.

#include <cstdint>

#include <cuda_fp16.h>

#include "pf_api.h"
#include "pf_common.cuh"

namespace pf {

template <typename T>
PF_D float ld_attr(const T* p, int64_t i);
template <>
PF_D float ld_attr<float>(const float* p, int64_t i) {
    return p[i];
}
template <>
PF_D float ld_attr<__half>(const __half* p, int64_t i) {
    return __half2float(p[i]);
}
template <typename T>
PF_D void st_attr(T* p, int64_t i, float v);
template <>
PF_D void st_attr<float>(float* p, int64_t i, float v) {
    p[i] = v;
}
template <>
PF_D void st_attr<__half>(__half* p, int64_t i, float v) {
    p[i] = __float2half_rn(v);
}

struct SvArgs {
    v3 origin, forward;
    float cutoff;
    int64_t n;
    int dof;
};

// normalize(p - origin) and whether it lies inside the camera cone
PF_D bool sv_direction(const float* points, int64_t t, const SvArgs& a, v3& dir) {
    dir = normalize(mk(points[3 * t], points[3 * t + 1], points[3 * t + 2]) - a.origin);
    return !(dot(dir, a.forward) < a.cutoff);
}

template <typename T>
__global__ void sv_forward_kernel(const float* __restrict__ points, SvArgs a, const T* __restrict__ sites,
                                  const T* __restrict__ values, const T* __restrict__ temps, T* __restrict__ value_out,
                                  T* __restrict__ wsum_out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    v3 dir;
    if (!sv_direction(points, t, a, dir)) {
        for (int k = 0; k < 3; k++) st_attr(value_out, 3 * t + k, 0.5f);
        st_attr(wsum_out, t, 0.0f);
        return;
    }
    float ws = 0.0f;
    v3 vs = mk(0.f, 0.f, 0.f);
    for (int i = 0; i < a.dof; i++) {
        const int64_t e = (int64_t)i * a.n + t;
        const v3 axis = mk(ld_attr(sites, 3 * e), ld_attr(sites, 3 * e + 1), ld_attr(sites, 3 * e + 2));
        const v3 val = mk(ld_attr(values, 3 * e), ld_attr(values, 3 * e + 1), ld_attr(values, 3 * e + 2));
        const float temp = ld_attr(temps, e);
        const float dist = length(dir - axis);
        const float w = expf(-temp * dist);
        ws += w;
        vs = vs + w * val;
    }
    st_attr(wsum_out, t, ws);
    const v3 v = vs / ws + mk(0.5f, 0.5f, 0.5f);
    st_attr(value_out, 3 * t, fmax_t(v.x, 0.0f));
    st_attr(value_out, 3 * t + 1, fmax_t(v.y, 0.0f));
    st_attr(value_out, 3 * t + 2, fmax_t(v.z, 0.0f));
}

template <typename T>
__global__ void sv_backward_kernel(const float* __restrict__ points, SvArgs a, const T* __restrict__ sites,
                                   const T* __restrict__ values, const T* __restrict__ temps,
                                   const T* __restrict__ wsum_in, const T* __restrict__ value_in,
                                   const T* __restrict__ grad_value, T* __restrict__ g_sites, T* __restrict__ g_values,
                                   T* __restrict__ g_temps) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    v3 dir;
    if (!sv_direction(points, t, a, dir)) {  // no gradient outside the camera cone
        for (int i = 0; i < a.dof; i++) {
            const int64_t e = (int64_t)i * a.n + t;
            for (int k = 0; k < 3; k++) {
                st_attr(g_sites, 3 * e + k, 0.0f);
                st_attr(g_values, 3 * e + k, 0.0f);
            }
            st_attr(g_temps, e, 0.0f);
        }
        return;
    }
    const float ws = ld_attr(wsum_in, t);
    v3 value = mk(ld_attr(value_in, 3 * t), ld_attr(value_in, 3 * t + 1), ld_attr(value_in, 3 * t + 2));
    v3 g = mk(ld_attr(grad_value, 3 * t), ld_attr(grad_value, 3 * t + 1), ld_attr(grad_value, 3 * t + 2));
    if (value.x <= 0.0f) g.x = 0.0f;
    if (value.y <= 0.0f) g.y = 0.0f;
    if (value.z <= 0.0f) g.z = 0.0f;
    value = value - mk(0.5f, 0.5f, 0.5f);
    const float dp_out = dot(g, value);
    for (int i = 0; i < a.dof; i++) {
        const int64_t e = (int64_t)i * a.n + t;
        const v3 axis = mk(ld_attr(sites, 3 * e), ld_attr(sites, 3 * e + 1), ld_attr(sites, 3 * e + 2));
        const v3 val = mk(ld_attr(values, 3 * e), ld_attr(values, 3 * e + 1), ld_attr(values, 3 * e + 2));
        const float temp = ld_attr(temps, e);
        const float dist = length(dir - axis);
        const float w = expf(-temp * dist);
        if (w / ws < 1e-3f) {  // a negligible site: zero gradient
            for (int k = 0; k < 3; k++) {
                st_attr(g_sites, 3 * e + k, 0.0f);
                st_attr(g_values, 3 * e + k, 0.0f);
            }
            st_attr(g_temps, e, 0.0f);
            continue;
        }
        const v3 dval = (w * g) / ws;
        st_attr(g_values, 3 * e, dval.x);
        st_attr(g_values, 3 * e + 1, dval.y);
        st_attr(g_values, 3 * e + 2, dval.z);
        const v3 dwds = ((temp * w) * (dir - axis)) / dist;
        const float dwdt = -dist * w;
        const float dp = dot(g, val);
        const v3 daxis = ((dp - dp_out) * dwds) / ws;
        const float dtemp = (dwdt * (dp - dp_out)) / ws;
        st_attr(g_sites, 3 * e, daxis.x);
        st_attr(g_sites, 3 * e + 1, daxis.y);
        st_attr(g_sites, 3 * e + 2, daxis.z);
        st_attr(g_temps, e, dtemp);
    }
}

static bool sv_args(const float* origin, const float* forward, float cutoff, int64_t n, int32_t dof, SvArgs& a) {
    if (!origin || !forward || n < 0 || dof < 1) return false;
    a.origin = mk(origin[0], origin[1], origin[2]);
    a.forward = mk(forward[0], forward[1], forward[2]);
    a.cutoff = cutoff;
    a.n = n;
    a.dof = dof;
    return true;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_sv_forward(const float* points, const float* camera_origin, const float* camera_forward,
                             float fov_cos_cutoff, const void* att_sites, const void* att_values,
                             const void* att_temps, int64_t n_points, int32_t sv_dof, int32_t attr_half,
                             void* value_out, void* weights_sum_out, void* stream) {
    SvArgs a;
    if (!sv_args(camera_origin, camera_forward, fov_cos_cutoff, n_points, sv_dof, a) ||
        (n_points > 0 && (!points || !att_sites || !att_values || !att_temps || !value_out || !weights_sum_out)))
        return pf_fail(PF_ERR_ARGS, "pf_sv_forward: bad arguments");
    if (n_points == 0) return PF_OK;
    const unsigned g = (unsigned)((n_points + 255) / 256);
    cudaStream_t st = (cudaStream_t)stream;
    if (attr_half)
        sv_forward_kernel<__half><<<g, 256, 0, st>>>(points, a, (const __half*)att_sites, (const __half*)att_values,
                                                     (const __half*)att_temps, (__half*)value_out,
                                                     (__half*)weights_sum_out);
    else
        sv_forward_kernel<float><<<g, 256, 0, st>>>(points, a, (const float*)att_sites, (const float*)att_values,
                                                    (const float*)att_temps, (float*)value_out,
                                                    (float*)weights_sum_out);
    return pf_check_launch("pf_sv_forward");
}

extern "C" int pf_sv_backward(const float* points, const float* camera_origin, const float* camera_forward,
                              float fov_cos_cutoff, const void* att_sites, const void* att_values,
                              const void* att_temps, const void* weights_sum, const void* values,
                              const void* grad_values, int64_t n_points, int32_t sv_dof, int32_t attr_half,
                              void* grad_att_sites, void* grad_att_values, void* grad_att_temps, void* stream) {
    SvArgs a;
    if (!sv_args(camera_origin, camera_forward, fov_cos_cutoff, n_points, sv_dof, a) ||
        (n_points > 0 && (!points || !att_sites || !att_values || !att_temps || !weights_sum || !values ||
                          !grad_values || !grad_att_sites || !grad_att_values || !grad_att_temps)))
        return pf_fail(PF_ERR_ARGS, "pf_sv_backward: bad arguments");
    if (n_points == 0) return PF_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = (unsigned)((n_points + 255) / 256);
    if (attr_half)
        sv_backward_kernel<__half><<<g, 256, 0, st>>>(
            points, a, (const __half*)att_sites, (const __half*)att_values, (const __half*)att_temps,
            (const __half*)weights_sum, (const __half*)values, (const __half*)grad_values, (__half*)grad_att_sites,
            (__half*)grad_att_values, (__half*)grad_att_temps);
    else
        sv_backward_kernel<float><<<g, 256, 0, st>>>(
            points, a, (const float*)att_sites, (const float*)att_values, (const float*)att_temps,
            (const float*)weights_sum, (const float*)values, (const float*)grad_values, (float*)grad_att_sites,
            (float*)grad_att_values, (float*)grad_att_temps);
    return pf_check_launch("pf_sv_backward");
}

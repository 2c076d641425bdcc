// pf_composite.cu -- front-to-back compositing forward and its adjoint.
//
// forward: rasterize.py:892-1146 (forward_kernel) + the launch of :1795-1825
// adjoint: rasterize.py:1150-1514 (backward_kernel), texture.py:74-186
//          (plane_intersection_bwd), rendering_math.py:26-147, and the host
//          side of Rasterizer._backward (:1861-1980).
//
// Work decomposition.  A tile of TW x TW pixels belongs to a block of G warps
// (TW = 8: 2 warps, one pixel per lane; TW = 16: 8 warps, one pixel per lane;
// TW = 32: 16 warps, two pixels per lane).  Blocks are persistent: each takes
// the next tile from a work queue ordered by decreasing list length (longest
// first, so the last tiles are short), and the reference's block-wide
// tile_max / tile_sum become __syncthreads_and / __syncthreads_or.  A warp
// whose pixels miss the primitive skips it after the block vote.
//
// Per primitive a warp stages the sphere and normal+sigma records of 32
// primitives at a time, turns the primitive's neighbours into face planes
// (n, num) one per lane, and stages the texel records once.  There is ONE copy
// of the per-pixel code (with two pixels per lane their states are swapped in
// registers between the two passes) and the texel loops are rolled: the hot
// loops then fit the instruction caches.
//
// Adjoint accumulation.  Each lane adds its pixels' contributions to the
// primitive's 64 gradient values (centre, radius, normal, sigma, 8 x site,
// 8 x rgb, 8 x height) in its own column of a 64 x 32 shared-memory table;
// after the primitive the warp sums each row (lane l sums rows 2l, 2l+1,
// reading the row with a lane-rotated column order so the 32 lanes hit 32
// different banks) and issues one global atomic per non-zero value.
// Gradients of the neighbour spheres bounding a pixel's segment are first
// summed per neighbour slot in shared memory and flushed once per primitive.
#include <algorithm>

#include "pf_composite.cuh"

namespace pf {

// GEN: a generic camera (per-pixel rays from ray maps); REC: write the
// adjoint's segment records (the compacted layouts only)
template <int TW, bool GEN = false, bool REC = false>
__global__ void __launch_bounds__(Layout<TW>::THREADS, Layout<TW>::FWD_MIN_BLOCKS)
raster_fwd_kernel(RasterParams P, FwdOut out) {
    constexpr int G = Layout<TW>::G;
    constexpr bool COMPACT = Layout<TW>::PPL == 1;
    // the per-pixel layouts stage per warp here; the compacted one keeps its
    // staging in dynamic shared memory
    __shared__ WarpStage stage[COMPACT ? 1 : G];
    __shared__ StopState ss;
    extern __shared__ float4 fwd_dyn[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t static_next = (int64_t)blockIdx.x;
    for (;;) {
        int64_t tile = next_tile<G>(P, static_next, lane, &ss);
        if (tile < 0) break;
        if constexpr (COMPACT)
            // generic cameras keep the pixels' ray origins after the stages
            fwd_tile_c<G, GEN, REC>(P, out, tile, warp, lane, reinterpret_cast<FwdCStage*>(fwd_dyn)[warp], ss,
                               reinterpret_cast<float4*>(reinterpret_cast<FwdCStage*>(fwd_dyn) + G) + 32 * warp);
        else
            fwd_tile<G, Layout<TW>::PPL, GEN>(P, out, tile, warp, lane, stage[warp], ss);
    }
}

// dynamic shared memory of the forward: the pair-compaction stage per warp
template <int TW, bool GEN = false>
constexpr size_t fwd_dyn_bytes() {
    return Layout<TW>::PPL == 1 ? (sizeof(FwdCStage) + (GEN ? 32 * sizeof(float4) : 0)) * Layout<TW>::G : 0;
}


// REC > 0: launched twice, without and with FB; the launch that does not fit
// the forward's record count (all hits recorded, or some not) returns at once
template <int TW, bool GEN = false, int REC = 0, bool FB = true>
__global__ void __launch_bounds__(Layout<TW>::THREADS, Layout<TW>::BWD_MIN_BLOCKS)
raster_bwd_kernel(RasterParams P, BwdIn in, GradOut go) {
    if constexpr (REC > 0) {
        const bool full = *(volatile unsigned long long*)P.seg_count > (unsigned long long)P.seg_cap;
        if (full != FB) return;
    }
    constexpr int G = Layout<TW>::G;
    __shared__ WarpStage stage[G];
    extern __shared__ float4 dyn_smem[];
    BwdStage* bstage = reinterpret_cast<BwdStage*>(dyn_smem);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    BwdStage& bs = bstage[warp];
    for (int r = 0; r < kAccRows; r++) bs.acc[r][lane] = 0.f;
    __syncwarp();
    int64_t static_next = (int64_t)blockIdx.x;
    for (;;) {
        int64_t tile = next_tile<G>(P, static_next, lane, nullptr);
        if (tile < 0) break;
        bwd_tile<G, Layout<TW>::PPL, GEN, REC, FB>(P, in, go, tile, warp, lane, stage[warp], bs);
    }
}

// the gradient arrays of one adjoint, sanitised in one launch: array a covers
// elements [start[a], start[a + 1]) of the combined index range; arrays whose
// address is 16-byte aligned and whose length is a multiple of 4 go by float4
struct SanitizeList {
    float* ptr[7];
    int64_t start[8];  // in units of the array's access (float4 or float)
    bool vec[7];
};

__global__ void zero_nonfinite_list_kernel(SanitizeList L) {
    const int64_t total = L.start[7];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        int a = 0;
#pragma unroll
        for (int k = 1; k < 7; k++) a += i >= L.start[k] ? 1 : 0;
        const int64_t j = i - L.start[a];
        if (L.vec[a]) {
            float4* p = reinterpret_cast<float4*>(L.ptr[a]) + j;
            float4 v = *p;
            if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w)) {
                v.x = isfinite(v.x) ? v.x : 0.0f;
                v.y = isfinite(v.y) ? v.y : 0.0f;
                v.z = isfinite(v.z) ? v.z : 0.0f;
                v.w = isfinite(v.w) ? v.w : 0.0f;
                *p = v;
            }
        } else {
            float* p = L.ptr[a] + j;
            if (!isfinite(*p)) *p = 0.0f;
        }
    }
}

// grid: persistent when a queue is available, else one group per tile
template <int TW, typename K>
static unsigned composite_grid(const RasterParams& P, K kernel, size_t dyn_smem) {
    const int64_t groups = P.T;
    if (!P.queue) return (unsigned)groups;
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Layout<TW>::THREADS, dyn_smem);
    int64_t resident = (int64_t)sms * std::max(per_sm, 1);
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(groups, resident));
}

template <int TW, bool GEN, bool REC>
static int launch_fwd_t(const RasterParams& P, const FwdOut& out, cudaStream_t st) {
    const size_t dyn = fwd_dyn_bytes<TW, GEN>();
    if (dyn > 0) {
        cudaError_t e = cudaFuncSetAttribute(raster_fwd_kernel<TW, GEN, REC>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        if (e != cudaSuccess) return pf_fail(PF_ERR_CUDA, cudaGetErrorString(e));
    }
    unsigned grid = composite_grid<TW>(P, raster_fwd_kernel<TW, GEN, REC>, dyn);
    raster_fwd_kernel<TW, GEN, REC><<<grid, Layout<TW>::THREADS, dyn, st>>>(P, out);
    return PF_OK;
}

template <int TW, bool GEN>
static int launch_fwd_g(const RasterParams& P, const FwdOut& out, cudaStream_t st) {
    if constexpr (Layout<TW>::PPL == 1) {
        if (P.seg) return launch_fwd_t<TW, GEN, true>(P, out, st);
    }
    return launch_fwd_t<TW, GEN, false>(P, out, st);
}

template <int TW>
static int launch_fwd(const RasterParams& P, const FwdOut& out, cudaStream_t st) {
    return P.ray_maps ? launch_fwd_g<TW, true>(P, out, st) : launch_fwd_g<TW, false>(P, out, st);
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
    if (P.T == 0) return pf_check_launch("pf_raster_forward");
    if (P.queue) cudaMemsetAsync(P.queue, 0, 2 * sizeof(int), st);
    FwdOut out{color, log_t, normal_distance, normal, quantile_depths, err, contrib, point_err, early_stop,
               tile_contrib_pairs, return_point_err, P.queue ? P.queue + 1 : nullptr};
    int rc;
    if (P.TW == 8) rc = launch_fwd<8>(P, out, st);
    else if (P.TW == 16) rc = launch_fwd<16>(P, out, st);
    else rc = launch_fwd<32>(P, out, st);
    if (rc != PF_OK) return rc;
    return pf_check_launch("pf_raster_forward");
}

template <int TW, bool GEN, int REC, bool FB = true>
static void launch_bwd_t(const RasterParams& P, const BwdIn& bi, const GradOut& go, cudaStream_t st) {
    const size_t dyn = sizeof(BwdStage) * Layout<TW>::G;
    cudaFuncSetAttribute(raster_bwd_kernel<TW, GEN, REC, FB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    unsigned grid = composite_grid<TW>(P, raster_bwd_kernel<TW, GEN, REC, FB>, dyn);
    raster_bwd_kernel<TW, GEN, REC, FB><<<grid, Layout<TW>::THREADS, dyn, st>>>(P, bi, go);
}

// with records: the launch for a forward that recorded every hit, then the one
// for a forward that found the buffer full (each returns at once when the
// other applies)
template <int TW, bool GEN, int REC>
static void launch_bwd_rec(const RasterParams& P, const BwdIn& bi, const GradOut& go, cudaStream_t st) {
    launch_bwd_t<TW, GEN, REC, false>(P, bi, go, st);
    launch_bwd_t<TW, GEN, REC, true>(P, bi, go, st);
}

template <int TW, bool GEN>
static void launch_bwd_g(const RasterParams& P, const BwdIn& bi, const GradOut& go, cudaStream_t st) {
    if constexpr (Layout<TW>::PPL == 1) {
        if (P.seg && P.seg_stride == 4) {
            launch_bwd_rec<TW, GEN, 2>(P, bi, go, st);
            return;
        }
        if (P.seg) {
            launch_bwd_rec<TW, GEN, 1>(P, bi, go, st);
            return;
        }
    }
    launch_bwd_t<TW, GEN, 0>(P, bi, go, st);
}

template <int TW>
static void launch_bwd(const RasterParams& P, const BwdIn& bi, const GradOut& go, cudaStream_t st) {
    if (P.ray_maps)
        launch_bwd_g<TW, true>(P, bi, go, st);
    else
        launch_bwd_g<TW, false>(P, bi, go, st);
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
    BwdIn bi{early_stop, log_t, grad_color, grad_opacity, grad_normal_distance, grad_normal,
             P.Q > 0 ? grad_quantile_depths : nullptr, grad_contrib};
    if (P.T > 0) {
        if (P.queue) cudaMemsetAsync(P.queue, 0, sizeof(int), st);
        if (P.TW == 8) launch_bwd<8>(P, bi, go, st);
        else if (P.TW == 16) launch_bwd<16>(P, bi, go, st);
        else launch_bwd<32>(P, bi, go, st);
    }
    SanitizeList L;
    L.start[0] = 0;
    for (int i = 0; i < 7; i++) {
        L.ptr[i] = outs[i];
        L.vec[i] = lens[i] % 4 == 0 && ((uintptr_t)outs[i] % 16) == 0;
        L.start[i + 1] = L.start[i] + (int64_t)(L.vec[i] ? lens[i] / 4 : lens[i]);
    }
    if (L.start[7] > 0) {
        const unsigned grid = (unsigned)std::min<int64_t>((L.start[7] + 255) / 256, 148 * 16);
        zero_nonfinite_list_kernel<<<grid, 256, 0, st>>>(L);
    }
    return pf_check_launch("pf_raster_backward");
}

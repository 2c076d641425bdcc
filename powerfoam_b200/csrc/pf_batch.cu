// pf_batch.cu -- multi-view training step in one persistent launch.
//
// No counterpart in the reference, whose scene renders one view per
// Rasterizer.forward call (powerfoam/scene.py:314-353); per view the step is
// the forward of forward_kernel (rasterize.py:892-1146), the L2 loss
// sum((color - target)^2) and the adjoint of backward_kernel
// (rasterize.py:1150-1514), with the gradients of all views summed.
//
// Work items are (view, tile) pairs of every view, ordered either by
// decreasing list length over all views (longest first, so the last items
// are short) or view by view.  Resident blocks pop `chunk` consecutive items
// per atomic on a device counter.  For each item the block runs the tile's
// forward, forms dL/dcolor = 2 (color - target) for its own pixels (the L2
// gradient is pixel-local, so no other tile is needed), and runs the tile's
// adjoint straight away, while the tile's primitive list and records are
// still in L2.  The per-view parameters are kernel parameters (64 views at
// most) copied into shared memory when a block changes view.
#include <algorithm>
#include <mutex>

#include "pf_composite.cuh"
#include "pf_sort.cuh"

namespace pf {

constexpr int kMaxViews = PF_BATCH_MAX_VIEWS;

struct BatchView {
    Cam cam;
    int tiles_h;
    int64_t T;
    int64_t item_base;  // index of the view's first tile in the loss array
    const int64_t* tile_off;
    const int32_t* tile_prims;
    const float* rgb;
    const float* target;
    float* color;
    float* log_t;
    float* nd;
    float* normal;
    float* g_color;
    float* contrib;
    int32_t* early_stop;
    int32_t* tile_contrib_pairs;
    float* g_rgb;
    int64_t seg_pair_base;  // the view's first (pair) entry in the segment mask / offset arrays
    int64_t seg_pairs;      // its pairs there
    int32_t seg_group;      // the record group it renders in (0 without records)
};

struct BatchParams {
    RasterParams base;      // scene-wide fields; the per-view ones are set per item
    GradOut go;             // rgb is per view
    const uint32_t* items;  // (view << 24) | tile, in processing order
    int64_t n_items;
    int chunk;
    int* queue;
    int* status;
    float* tile_loss;
    int n_views;
    BatchView views[kMaxViews];
};

union BatchStage {
    FwdCStage fwd;
    BwdStage bwd;
};

struct BatchShared {
    RasterParams P;
    FwdOut out;
    BwdIn in;
    GradOut go;
    const float* target;
    float* g_color;
    float* tile_loss;  // view's slice
    float loss[16];
    int64_t next;
};

PF_D void load_view(const BatchParams& B, int v, BatchShared& sh) {
    const BatchView& V = B.views[v];
    sh.P = B.base;
    sh.P.cam = V.cam;
    sh.P.tiles_h = V.tiles_h;
    sh.P.T = V.T;
    sh.P.tile_off = V.tile_off;
    sh.P.tile_prims = V.tile_prims;
    sh.P.rgb = V.rgb;
    if (B.base.seg) {  // the view's slice of the segment masks and offsets
        const int64_t g = (int64_t)B.base.TW * B.base.TW / 32;
        sh.P.seg_mask = B.base.seg_mask + V.seg_pair_base * g;
        sh.P.seg_off = B.base.seg_off + V.seg_pair_base * g;
        sh.P.seg_pairs = V.seg_pairs;
    }
    sh.out = FwdOut{V.color, V.log_t, V.nd, V.normal, nullptr, nullptr, V.contrib, nullptr, V.early_stop,
                    V.tile_contrib_pairs, 0, B.status};
    sh.in = BwdIn{V.early_stop, V.log_t, V.g_color, nullptr, nullptr, nullptr, nullptr, nullptr};
    sh.go = B.go;
    sh.go.rgb = V.g_rgb;
    sh.target = V.target;
    sh.g_color = V.g_color;
    sh.tile_loss = B.tile_loss + V.item_base;
}

// Phases of one work item: the fused schedule runs the tile's forward, its L2
// gradient and its adjoint back to back in one launch; the split schedule runs
// one persistent launch of forwards (+ L2 gradients) over all items, then one
// of adjoints, each kernel at its own occupancy.
enum BatchPhase { kFused = 0, kFwdOnly = 1, kBwdOnly = 2 };

template <int TW, int PH>
struct BatchKernel {
    static constexpr int MIN_BLOCKS = PH == kFwdOnly ? 1 : Layout<TW>::BWD_MIN_BLOCKS;
    static constexpr size_t STAGE = PH == kFused    ? sizeof(BatchStage)
                                    : PH == kBwdOnly ? sizeof(BwdStage)
                                    : (Layout<TW>::PPL == 1 ? sizeof(FwdCStage) : 0);
};

// REC > 0: the forward writes segment records and the adjoint reads them (as
// pf_raster_forward / pf_raster_backward); the adjoint-only launch comes in
// the pair without / with FB, of which the one that does not apply returns
template <int TW, int PH, int REC = 0, bool FB = true>
__global__ void __launch_bounds__(Layout<TW>::THREADS, BatchKernel<TW, PH>::MIN_BLOCKS)
batch_step_kernel(const __grid_constant__ BatchParams B) {
    if constexpr (REC > 0 && PH == kBwdOnly) {
        const bool full = *(volatile unsigned long long*)B.base.seg_count > (unsigned long long)B.base.seg_cap;
        if (full != FB) return;
    }
    constexpr int G = Layout<TW>::G, PPL = Layout<TW>::PPL;
    constexpr int TS = TW * TW;
    constexpr bool FWD = PH != kBwdOnly, BWD = PH != kFwdOnly;
    __shared__ WarpStage stage[G];
    __shared__ StopState ss;
    __shared__ BatchShared sh;
    extern __shared__ float4 dyn_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // per-warp area: the forward's pair compaction stage (one-pixel-per-lane
    // layouts) and the adjoint's gradient table, in turn when fused
    BwdStage& bs = *reinterpret_cast<BwdStage*>(reinterpret_cast<char*>(dyn_smem) + warp * BatchKernel<TW, PH>::STAGE);
    FwdCStage& fs = *reinterpret_cast<FwdCStage*>(reinterpret_cast<char*>(dyn_smem) + warp * BatchKernel<TW, PH>::STAGE);
    int* queue = B.queue + (PH == kBwdOnly ? 1 : 0);
    if (PH == kBwdOnly) {
        for (int r = 0; r < kAccRows; r++) bs.acc[r][lane] = 0.f;
        __syncwarp();
    }
    stop_reset<G>(ss, warp, lane);
    int view = -1;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) sh.next = atomicAdd(queue, B.chunk);
        __syncthreads();
        const int64_t c0 = sh.next;
        if (c0 >= B.n_items) break;
        const int64_t c1 = std::min<int64_t>(c0 + B.chunk, B.n_items);
        for (int64_t it = c0; it < c1; it++) {
            if (it > c0) __syncthreads();  // previous item done with ss / sh
            const uint32_t code = B.items[it];
            const int v = (int)(code >> 24);
            const int64_t tile = (int64_t)(code & 0xffffffu);
            if (v != view) {
                if (threadIdx.x == 0) load_view(B, v, sh);
                __syncthreads();
                view = v;
            }
            if constexpr (FWD) {
                if constexpr (PPL == 1) fwd_tile_c<G, false, (REC > 0)>(sh.P, sh.out, tile, warp, lane, fs, ss);
                else fwd_tile<G, PPL>(sh.P, sh.out, tile, warp, lane, stage[warp], ss);
                // dL/dcolor of this thread's own pixels (written by it in the forward)
                float l = 0.f;
#pragma unroll 1
                for (int s = 0; s < PPL; s++) {
                    PixGeom g = pixel_geom(sh.P, tile, warp * 32 + lane + s * (TS / 2));
                    if (!g.oob) {
                        const int64_t p = g.px;
                        float d0 = sh.out.color[3 * p] - __ldg(&sh.target[3 * p]);
                        float d1 = sh.out.color[3 * p + 1] - __ldg(&sh.target[3 * p + 1]);
                        float d2 = sh.out.color[3 * p + 2] - __ldg(&sh.target[3 * p + 2]);
                        sh.g_color[3 * p] = 2.0f * d0;
                        sh.g_color[3 * p + 1] = 2.0f * d1;
                        sh.g_color[3 * p + 2] = 2.0f * d2;
                        l += d0 * d0 + d1 * d1 + d2 * d2;
                    }
                }
                l = warp_sum(l);
                if (lane == 0) sh.loss[warp] = l;
                __syncthreads();  // early_stop, log_t and g_color of the whole tile are written
                if (threadIdx.x == 0) {
                    float t = 0.f;
                    for (int w = 0; w < G; w++) t += sh.loss[w];
                    sh.tile_loss[tile] = t;
                }
                stop_reset<G>(ss, warp, lane);  // ready for the next tile's forward
            }
            if constexpr (BWD) {
                if constexpr (PH == kFused) {
                    for (int r = 0; r < kAccRows; r++) bs.acc[r][lane] = 0.f;  // the forward used this area
                    __syncwarp();
                }
                bwd_tile<G, PPL, false, (PPL == 1 ? REC : 0), FB, PH == kFused>(sh.P, sh.in, sh.go, tile, warp, lane,
                                                                                stage[warp], bs);
            }
        }
    }
}

__global__ void batch_keys_kernel(const __grid_constant__ BatchParams B, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ vals) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= B.n_items) return;
    int v = 0;
    while (v + 1 < B.n_views && B.views[v + 1].item_base <= g) v++;
    const int64_t t = g - B.views[v].item_base;
    const int64_t len = B.views[v].tile_off[t + 1] - B.views[v].tile_off[t];
    // record group (6 bits) above the list length (18 bits, longer lists tie): group-major,
    // longest first within a group
    if (keys)
        keys[g] = ((uint32_t)B.views[v].seg_group << 18) | (0x3ffffu - (uint32_t)std::min<int64_t>(len, 0x3ffff));
    vals[g] = ((uint32_t)v << 24) | (uint32_t)t;
}

__global__ void batch_zero_nonfinite_kernel(float* __restrict__ a, int64_t n) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        float x = a[i];
        if (!isfinite(x)) a[i] = 0.0f;
    }
}

struct BatchLayout {
    size_t k0, v0, k1, v1, items, rhist, rpart, queue, bytes;
};

inline BatchLayout batch_layout(int64_t n_items) {
    BatchLayout L;
    size_t off = 0;
    auto take = [&](size_t b) {
        size_t o = off;
        off += (b + 255) & ~(size_t)255;
        return o;
    };
    const size_t b4 = sizeof(uint32_t) * (size_t)std::max<int64_t>(n_items, 1);
    L.k0 = take(b4);
    L.v0 = take(b4);
    L.k1 = take(b4);
    L.v1 = take(b4);
    L.items = take(b4);
    const int64_t nb = radix_blocks(std::max<int64_t>(n_items, 1));
    L.rhist = take(sizeof(uint32_t) * (size_t)(256 * nb));
    L.rpart = take(sizeof(uint32_t) * (size_t)(scan_blocks(256 * nb) + 1));
    L.queue = take(sizeof(int) * 2 * kMaxViews);  // two work counters per record group
    L.bytes = off;
    return L;
}

template <int TW, int PH, int REC = 0, bool FB = true>
static int launch_phase(const BatchParams& B, cudaStream_t st) {
    const size_t dyn = BatchKernel<TW, PH>::STAGE * Layout<TW>::G;
    cudaError_t e = cudaFuncSetAttribute(batch_step_kernel<TW, PH, REC, FB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return pf_fail(PF_ERR_CUDA, cudaGetErrorString(e));
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_step_kernel<TW, PH, REC, FB>, Layout<TW>::THREADS,
                                                  dyn);
    if (per_sm < 1) return pf_fail(PF_ERR_CUDA, "pf_batch_render: kernel does not fit on an SM");
    const int64_t items_per_pop = std::max(B.chunk, 1);
    const int64_t pops = (B.n_items + items_per_pop - 1) / items_per_pop;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, pops));
    batch_step_kernel<TW, PH, REC, FB><<<grid, Layout<TW>::THREADS, dyn, st>>>(B);
    return PF_OK;
}

template <int TW, int REC>
static int launch_batch_rec(const BatchParams& B, bool split, cudaStream_t st) {
    if (!split) return launch_phase<TW, kFused, REC, true>(B, st);  // a tile's adjoint follows its forward
    int rc = launch_phase<TW, kFwdOnly, REC>(B, st);
    if (rc != PF_OK) return rc;
    if constexpr (REC > 0) {
        rc = launch_phase<TW, kBwdOnly, REC, false>(B, st);
        if (rc != PF_OK) return rc;
    }
    return launch_phase<TW, kBwdOnly, REC, true>(B, st);
}

template <int TW>
static int launch_batch(const BatchParams& B, bool split, cudaStream_t st) {
    if constexpr (Layout<TW>::PPL == 1) {
        if (B.base.seg && B.base.seg_stride == 4) return launch_batch_rec<TW, 2>(B, split, st);
        if (B.base.seg) return launch_batch_rec<TW, 1>(B, split, st);
    }
    return launch_batch_rec<TW, 0>(B, split, st);
}

static int batch_params(const pf_batch_scene* sc, const pf_batch_view* views, int32_t n_views, int32_t tile_width,
                        BatchParams& B, const char** why) {
    if (!sc || !views || n_views < 1 || n_views > kMaxViews) {
        *why = "pf_batch: need a scene and 1..64 views";
        return 0;
    }
    if (tile_width != 8 && tile_width != 16 && tile_width != 32) {
        *why = "pf_batch: tile_width must be 8, 16 or 32";
        return 0;
    }
    if (sc->n_sites < 0 || sc->n_sites > kMaxSites || sc->n_prims < 0) {
        *why = "pf_batch: bad scene sizes";
        return 0;
    }
    if (sc->n_prims > 0 && (!sc->spheres || !sc->nsigmas || !sc->texel_sites || !sc->texel_height ||
                            !sc->adjacency_offsets || !sc->adjacency_diff)) {
        *why = "pf_batch: missing scene arrays";
        return 0;
    }
    RasterParams& P = B.base;
    P = RasterParams{};
    P.TW = tile_width;
    P.S = sc->n_sites;
    P.Q = 0;
    P.N = sc->n_prims;
    P.spheres = (const float4*)sc->spheres;
    P.nsigmas = (const float4*)sc->nsigmas;
    P.sites = sc->texel_sites;
    P.height = sc->texel_height;
    P.adj = sc->adjacency;
    P.adj_off = sc->adjacency_offsets;
    P.adj_diff = (const uint2*)sc->adjacency_diff;
    P.dq = nullptr;
    P.gt = nullptr;
    P.thr = sc->transmittance_threshold;
    P.tile_order = nullptr;
    P.queue = nullptr;
    if (sc->segments) {
        if ((tile_width != 8 && tile_width != 16) || !sc->segment_masks || !sc->segment_offsets ||
            !sc->segment_count || ((uintptr_t)sc->segments % 16) != 0 || sc->segment_capacity < 0 ||
            sc->segment_capacity >= ((int64_t)1 << 31)) {
            *why = "pf_batch: segments need tile width 8 or 16, masks, offsets, a counter, 16-byte alignment and "
                   "0 <= segment_capacity < 2^31";
            return 0;
        }
        P.seg = (float4*)sc->segments;
        P.seg_mask = sc->segment_masks;
        P.seg_off = sc->segment_offsets;
        P.seg_count = (unsigned long long*)sc->segment_count;
        P.seg_cap = sc->segment_capacity;
        P.seg_stride = sc->segment_planes ? 4 : 1;
    }
    B.n_views = n_views;
    int64_t base = 0;
    for (int v = 0; v < n_views; v++) {
        const pf_batch_view& w = views[v];
        if (w.cam.width < 2 || w.cam.height < 2) {
            *why = "pf_batch: every image must be at least 2x2";
            return 0;
        }
        if (!w.tile_offsets || !w.tile_prims || !w.target || !w.color || !w.log_t || !w.normal_distance ||
            !w.normal || !w.grad_color || !w.contrib || !w.early_stop || !w.grad_texel_rgb ||
            (sc->n_prims > 0 && !w.texel_rgb)) {
            *why = "pf_batch: missing view array";
            return 0;
        }
        BatchView& V = B.views[v];
        V.cam = load_cam(w.cam);
        V.tiles_h = 1 + (w.cam.height - 1) / tile_width;
        const int64_t tiles_w = 1 + (w.cam.width - 1) / tile_width;
        V.T = (int64_t)V.tiles_h * tiles_w;
        if (V.T >= ((int64_t)1 << 24)) {
            *why = "pf_batch: more than 2^24 tiles in one view";
            return 0;
        }
        V.item_base = base;
        base += V.T;
        V.tile_off = w.tile_offsets;
        V.tile_prims = w.tile_prims;
        V.rgb = w.texel_rgb;
        V.target = w.target;
        V.color = w.color;
        V.log_t = w.log_t;
        V.nd = w.normal_distance;
        V.normal = w.normal;
        V.g_color = w.grad_color;
        V.contrib = w.contrib;
        V.early_stop = w.early_stop;
        V.tile_contrib_pairs = w.tile_contrib_pairs;
        V.g_rgb = w.grad_texel_rgb;
        V.seg_pair_base = w.segment_pair_base;
        V.seg_pairs = sc->segments ? w.segment_pairs : 0;
        V.seg_group = sc->segments ? w.segment_group : 0;
        if (sc->segments && (w.segment_pair_base < 0 || w.segment_pairs < 0)) {
            *why = "pf_batch: bad segment pair range";
            return 0;
        }
        const int32_t prev = v > 0 ? views[v - 1].segment_group : 0;
        if (sc->segments && (w.segment_group < prev || w.segment_group > prev + (v > 0 ? 1 : 0))) {
            *why = "pf_batch: segment groups must start at 0 and grow by 0 or 1 from one view to the next";
            return 0;
        }
    }
    B.n_items = base;
    return 1;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_batch_workspace_size(const pf_batch_view* views, int32_t n_views, int32_t tile_width,
                                       size_t* bytes) {
    if (!views || !bytes || n_views < 1 || n_views > kMaxViews || tile_width <= 0)
        return pf_fail(PF_ERR_ARGS, "pf_batch_workspace_size: bad arguments");
    int64_t n = 0;
    for (int v = 0; v < n_views; v++) {
        if (views[v].cam.width < 2 || views[v].cam.height < 2)
            return pf_fail(PF_ERR_ARGS, "pf_batch_workspace_size: every image must be at least 2x2");
        n += (int64_t)(1 + (views[v].cam.height - 1) / tile_width) * (1 + (views[v].cam.width - 1) / tile_width);
    }
    *bytes = batch_layout(n).bytes;
    return PF_OK;
}

extern "C" int pf_batch_render(const pf_batch_scene* scene, const pf_batch_view* views, int32_t n_views,
                               int32_t tile_width, int32_t chunk, int32_t order, int32_t split, void* workspace,
                               size_t workspace_bytes, float* tile_loss, float* grad_points, float* grad_radii,
                               float* grad_normals, float* grad_density, float* grad_texel_sites,
                               float* grad_texel_height, int32_t* status, void* stream) {
    static BatchParams B;  // ~12 KB: kept off the host stack; the launch copies it
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    const char* why = "";
    if (!batch_params(scene, views, n_views, tile_width, B, &why)) return pf_fail(PF_ERR_ARGS, why);
    if (chunk < 1 || chunk > 1024) return pf_fail(PF_ERR_ARGS, "pf_batch_render: chunk must be in [1, 1024]");
    if (order != PF_BATCH_ORDER_LONGEST && order != PF_BATCH_ORDER_VIEW)
        return pf_fail(PF_ERR_ARGS, "pf_batch_render: unknown order");
    if (!tile_loss || !status || !workspace || !grad_points || !grad_radii || !grad_normals || !grad_density ||
        !grad_texel_sites || !grad_texel_height)
        return pf_fail(PF_ERR_ARGS, "pf_batch_render: missing argument");
    const BatchLayout L = batch_layout(B.n_items);
    if (workspace_bytes < L.bytes) return pf_fail(PF_ERR_ARGS, "pf_batch_render: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    char* ws = (char*)workspace;
    const size_t N = (size_t)B.base.N, S = (size_t)B.base.S;
    float* outs[6] = {grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites, grad_texel_height};
    const size_t lens[6] = {3 * N, N, 3 * N, N, 3 * N * S, N * S};
    for (int i = 0; i < 6; i++)
        if (lens[i]) cudaMemsetAsync(outs[i], 0, sizeof(float) * lens[i], st);
    for (int v = 0; v < n_views; v++) {
        if (N) cudaMemsetAsync(views[v].grad_texel_rgb, 0, sizeof(float) * 3 * N * S, st);
        if (N) cudaMemsetAsync(views[v].contrib, 0, sizeof(float) * N, st);
        if (views[v].tile_contrib_pairs)
            cudaMemsetAsync(views[v].tile_contrib_pairs, 0, sizeof(int32_t) * (size_t)B.views[v].T, st);
    }
    B.go = GradOut{grad_points, grad_radii, grad_normals, grad_density, grad_texel_sites, nullptr, grad_texel_height};
    B.items = (const uint32_t*)(ws + L.items);
    B.chunk = chunk;
    B.queue = (int*)(ws + L.queue);
    B.status = (int*)status;
    B.tile_loss = tile_loss;
    // with segment records the views render in groups (non-decreasing segment_group), one
    // after the other, each with its own work counters and record counter, reusing the one
    // record buffer
    const int n_groups = B.base.seg ? B.views[n_views - 1].seg_group + 1 : 1;
    cudaMemsetAsync(B.queue, 0, 2 * sizeof(int) * (size_t)n_groups, st);
    if (B.base.seg) cudaMemsetAsync(B.base.seg_count, 0, sizeof(int64_t) * (size_t)n_groups, st);
    // work list
    uint32_t* k0 = (uint32_t*)(ws + L.k0);
    uint32_t* v0 = (uint32_t*)(ws + L.v0);
    uint32_t* k1 = (uint32_t*)(ws + L.k1);
    uint32_t* v1 = (uint32_t*)(ws + L.v1);
    uint32_t* items = (uint32_t*)(ws + L.items);
    const unsigned gk = (unsigned)((B.n_items + 255) / 256);
    if (order == PF_BATCH_ORDER_VIEW) {
        batch_keys_kernel<<<gk, 256, 0, st>>>(B, nullptr, items);
    } else {
        batch_keys_kernel<<<gk, 256, 0, st>>>(B, k0, v0);
        RadixScratch rs{(uint32_t*)(ws + L.rhist), (uint32_t*)(ws + L.rpart)};
        uint32_t* kf = radix_final_key_buffer(k0, k1, 24);
        radix_sort_pairs(k0, v0, k1, v1, kf, items, B.n_items, nullptr, 24, rs, st);
    }
    static BatchParams Bg;  // a group's launch parameters
    int rc = PF_OK;
    for (int g = 0, v = 0; g < n_groups && rc == PF_OK; g++) {
        // a group's items follow each other in both orders (group-major keys, or view order)
        int64_t first = -1, n = 0;
        for (; v < n_views && B.views[v].seg_group == g; v++) {
            if (first < 0) first = B.views[v].item_base;
            n += B.views[v].T;
        }
        if (n == 0) continue;
        const BatchParams* Bp = &B;
        if (n_groups > 1) {
            Bg = B;
            Bg.items = B.items + first;
            Bg.n_items = n;
            Bg.queue = B.queue + 2 * g;
            Bg.base.seg_count = B.base.seg_count + g;
            Bp = &Bg;
        }
        if (tile_width == 8) rc = launch_batch<8>(*Bp, split != 0, st);
        else if (tile_width == 16) rc = launch_batch<16>(*Bp, split != 0, st);
        else rc = launch_batch<32>(*Bp, split != 0, st);
    }
    if (rc != PF_OK) return rc;
    auto sanitize = [&](float* a, size_t n) {
        if (!n) return;
        unsigned grid = (unsigned)std::min<int64_t>(((int64_t)n + 255) / 256, 148 * 16);
        batch_zero_nonfinite_kernel<<<grid, 256, 0, st>>>(a, (int64_t)n);
    };
    for (int i = 0; i < 6; i++) sanitize(outs[i], lens[i]);
    for (int v = 0; v < n_views; v++) {
        bool seen = false;  // a shared rgb gradient array is sanitised once
        for (int u = 0; u < v && !seen; u++) seen = views[u].grad_texel_rgb == views[v].grad_texel_rgb;
        if (!seen) sanitize(views[v].grad_texel_rgb, 3 * N * S);
    }
    return pf_check_launch("pf_batch_render");
}

// Schedule tuner: every candidate (chunk, order, split) is run `warmup` times
// untimed and `iters` times between two CUDA events on `stream`; the host
// waits for each candidate's end event, so the call is not capturable.
extern "C" int pf_batch_autotune(const pf_batch_scene* scene, const pf_batch_view* views, int32_t n_views,
                                 int32_t tile_width, pf_batch_schedule* cands, int32_t n_cands, int32_t warmup,
                                 int32_t iters, void* workspace, size_t workspace_bytes, float* tile_loss,
                                 float* grad_points, float* grad_radii, float* grad_normals, float* grad_density,
                                 float* grad_texel_sites, float* grad_texel_height, int32_t* status, int32_t* best,
                                 void* stream) {
    if (!cands || n_cands < 1 || !best || warmup < 0 || iters < 1)
        return pf_fail(PF_ERR_ARGS, "pf_batch_autotune: need candidates, a best index, warmup >= 0, iters >= 1");
    cudaEvent_t ev[2];
    if (cudaEventCreate(&ev[0]) != cudaSuccess) return pf_fail(PF_ERR_CUDA, "pf_batch_autotune: event");
    if (cudaEventCreate(&ev[1]) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return pf_fail(PF_ERR_CUDA, "pf_batch_autotune: event");
    }
    cudaStream_t st = (cudaStream_t)stream;
    int rc = PF_OK;
    *best = -1;
    float best_ms = 0.f;
    for (int32_t c = 0; c < n_cands && rc == PF_OK; c++) {
        pf_batch_schedule& s = cands[c];
        auto run = [&]() {
            return pf_batch_render(scene, views, n_views, tile_width, s.chunk, s.order, s.split, workspace,
                                   workspace_bytes, tile_loss, grad_points, grad_radii, grad_normals, grad_density,
                                   grad_texel_sites, grad_texel_height, status, stream);
        };
        for (int32_t i = 0; i < warmup && rc == PF_OK; i++) rc = run();
        if (rc != PF_OK) break;
        cudaEventRecord(ev[0], st);
        for (int32_t i = 0; i < iters && rc == PF_OK; i++) rc = run();
        if (rc != PF_OK) break;
        cudaEventRecord(ev[1], st);
        if (cudaEventSynchronize(ev[1]) != cudaSuccess) {
            rc = pf_fail(PF_ERR_CUDA, "pf_batch_autotune: a timed run failed");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        s.ms = ms / (float)iters;
        if (*best < 0 || s.ms < best_ms) {
            *best = c;
            best_ms = s.ms;
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return rc;
}

// pf_mlp.cu -- ray-proposal network on the 5th-generation tensor cores.
//
// No counterpart in the reference.  The network maps a ray (origin / 3 and
// unit direction, 6 values) through a 6-frequency positional encoding (the
// raw values, sin and cos of 2^k pi x for k = 0..5: 78 features) and three
// hidden ReLU layers of width 64 to two outputs: the entry distance of the
// first significant cell (divided by kTScale) and a confidence logit.
//
// Every layer reads an 80-wide input whose column ones_col(l) holds the
// constant 1 (the bias is that column of the weight matrix) and whose other
// pad columns hold 0, so the layer is one GEMM  Z = X W^T  (X: 128 rays x 80,
// W: out x 80) with K = 80.  Weights are BF16, accumulation FP32 in tensor
// memory (TMEM).  One CTA of 128 threads owns one SM (its shared-memory
// footprint allows no second CTA) and walks tiles of 128 rays; thread r owns
// ray r, which is also TMEM lane r of every accumulator.
//
// Operand layout in shared memory (no swizzle): a matrix whose contiguous
// axis is "c" and other axis "r" (R rows) stores element (r, c) at byte
//   (c / 8) * (R * 16) + r * 16 + (c % 8) * 2,
// i.e. 16-byte pieces of 8 consecutive c, all rows of one 8-column chunk
// together.  Read with c as K this is the canonical K-major layout (stride
// between 8-row groups SBO = 128 B, between 8-column K chunks LBO = R * 16 B);
// read with c as M or N it is the canonical MN-major layout (SBO = R * 16 B
// between 8-element M/N groups, LBO = 128 B between 8-row K groups).  So an
// activation buffer (rays x features) is the K-major A operand of the next
// layer's forward GEMM and the MN-major B operand of the weight gradient
// dW = dZ^T H, and a weight image (out x in) is the K-major B operand of the
// forward GEMM and the MN-major B operand of the data gradient dH = dZ W.
//
// Training step per tile: forward (4 GEMMs), loss gradient in registers, then
// per layer dH = dZ W (M 128, N 80) and dW += dZ^T H (M 128 with rows >= out
// unused, N 80, K = the tile's 128 rays), the dW accumulators staying in
// TMEM across all tiles of the CTA and flushed once with float atomics.
// Adam (FP32 master weights) writes the next step's BF16 image.
//
// Every wait on the tensor core is bounded; on timeout the kernel records
// PF_ERR_CUDA, waits (bounded) for its last commit, frees its TMEM and exits.
#include <cuda_bf16.h>

#include <algorithm>

#include "pf_api.h"
#include "pf_common.cuh"

namespace pf {
namespace mlp {

constexpr int kRays = 128;
constexpr int kIn = 80;
constexpr int kLayers = 4;
constexpr float kTScale = 6.0f;
__host__ __device__ constexpr int layer_out(int l) { return l == 3 ? 16 : 64; }
__host__ __device__ constexpr int w_off(int l) { return l * 64 * kIn; }  // fp32 master, (out x 80) row-major
constexpr int kParams = 3 * 64 * kIn + 16 * kIn;                         // 16640
__host__ __device__ constexpr int img_off(int l) { return l * 64 * kIn * 2; }  // bytes in the BF16 image
constexpr int kImgBytes = 3 * 64 * kIn * 2 + 16 * kIn * 2;                    // 33280

// shared-memory map (bytes from a 1024-aligned base).  The MN-major A operand
// of dW (M = 128 over an out-wide buffer) reads 32 KB from its start: each dZ
// buffer is followed by at least that much shared memory.
constexpr int kSmW = 0;
constexpr int kSmDz4 = 33792;
constexpr int kSmDz3 = kSmDz4 + 4096;
constexpr int kSmDz2 = kSmDz3 + 16384;
constexpr int kSmDz1 = kSmDz2 + 16384;
constexpr int kSmX = kSmDz1 + 16384;
constexpr int kSmH1 = kSmX + 20480;
constexpr int kSmH2 = kSmH1 + 20480;
constexpr int kSmH3 = kSmH2 + 20480;
constexpr int kSmBar = kSmH3 + 20480;
constexpr int kSmEnd = kSmBar + 64;
constexpr int kSmBytes = kSmEnd + 1024;  // + alignment slack

// inference layout: no gradient buffers, the activations ping-pong between two
// buffers (layer 3 overwrites layer 1's output, which layer 2 has consumed),
// 96 KB so two blocks share an SM and one encodes while the other waits for
// the tensor core
constexpr int kFsX = 33792;
constexpr int kFsHa = kFsX + 20480;
constexpr int kFsHb = kFsHa + 20480;
constexpr int kFsBar = kFsHb + 20480;
constexpr int kFsEnd = kFsBar + 64;
constexpr int kFsBytes = kFsEnd + 1024;
constexpr uint32_t kFsTmCols = 128;  // layer outputs only

// TMEM columns: activations / data gradients, then the four dW accumulators
constexpr uint32_t kTmAcc = 0;
__host__ __device__ constexpr uint32_t tm_grad(int l) { return 128 + 80 * l; }
constexpr uint32_t kTmCols = 512;

constexpr long long kWaitIters = 1ll << 22;

// ---------------------------------------------------------------------------
// PTX wrappers
PF_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle (sm_100 format, version 1)
PF_D uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: BF16 x BF16 -> FP32, dense
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn_major, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

PF_D void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

PF_D void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

PF_D void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
PF_D void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
PF_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

PF_D void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

PF_D bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

PF_D bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitIters; i++)
        if (mbar_try(bar, parity)) return true;
    return false;
}

PF_D void tmem_alloc(uint32_t slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

PF_D void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's lane; the wait is tied to the
// registers so no use can be scheduled before it
PF_D void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

PF_D uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// 8 consecutive features (chunk c) of row r of an R-row operand buffer
PF_D void put_chunk(uint8_t* buf, int R, int r, int c, const float* v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(buf + c * (R * 16) + r * 16) = q;
}

// ---------------------------------------------------------------------------
// GEMM issue helpers (one elected thread)
//   forward:  Z = A B^T, A = rays x 80 (K-major), B = W (out x 80, K-major)
PF_D void issue_forward(uint32_t d, uint32_t a_buf, uint32_t w_img, int out) {
    const uint32_t id = idesc_bf16(128, out, 0, 0);
#pragma unroll 1
    for (int ks = 0; ks < kIn / 16; ks++) {
        uint64_t a = sdesc(a_buf + ks * 2 * (kRays * 16), kRays * 16, 128);
        uint64_t b = sdesc(w_img + ks * 2 * (out * 16), out * 16, 128);
        mma(d, a, b, id, ks > 0);
    }
}

//   data gradient: dH = dZ W, A = dZ (rays x out, K-major over out), B = W read
//   MN-major (N = 80 inputs, K = out)
PF_D void issue_dgrad(uint32_t d, uint32_t dz_buf, uint32_t w_img, int out) {
    const uint32_t id = idesc_bf16(128, kIn, 0, 1);
#pragma unroll 1
    for (int ks = 0; ks < out / 16; ks++) {
        uint64_t a = sdesc(dz_buf + ks * 2 * (kRays * 16), kRays * 16, 128);
        uint64_t b = sdesc(w_img + ks * 2 * 128, 128, out * 16);
        mma(d, a, b, id, ks > 0);
    }
}

//   weight gradient: dW (+)= dZ^T H, A = dZ^T read MN-major (M = 128 >= out,
//   K = rays), B = H^T read MN-major (N = 80, K = rays)
PF_D void issue_wgrad(uint32_t d, uint32_t dz_buf, uint32_t h_buf, bool accumulate) {
    const uint32_t id = idesc_bf16(128, kIn, 1, 1);
#pragma unroll 1
    for (int ks = 0; ks < kRays / 16; ks++) {
        uint64_t a = sdesc(dz_buf + ks * 2 * 128, 128, kRays * 16);
        uint64_t b = sdesc(h_buf + ks * 2 * 128, 128, kRays * 16);
        mma(d, a, b, id, (accumulate || ks > 0) ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------
// positional encoding of one ray into 80 features
PF_D void encode(const float u[6], float f[80]) {
#pragma unroll
    for (int i = 0; i < 6; i++) f[i] = u[i];
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const float s = (float)(1 << k);
#pragma unroll
        for (int i = 0; i < 6; i++) {
            float sv, cv;
            sincospif(s * u[i], &sv, &cv);
            f[6 + 12 * k + 2 * i] = sv;
            f[6 + 12 * k + 2 * i + 1] = cv;
        }
    }
    f[78] = 1.0f;
    f[79] = 0.0f;
}

struct Ctx {
    uint8_t* sm;
    uint32_t sbase;
    uint32_t tmem;
    uint32_t bar;
    uint32_t phase;
    int* status;
    bool ok;
    uint32_t cols;  // TMEM columns held
};

// commit, then every thread waits for the tensor core.  The outcome is made
// uniform over the block (a thread may see the completion just after another
// gave up); on failure the phase stays on the pending commit so the exit path
// can wait for it once more.
PF_D bool commit_wait(Ctx& c) {
    if (threadIdx.x == 0) mma_commit(c.bar);
    const bool done = mbar_wait(c.bar, c.phase);
    const bool all = __syncthreads_and(done) != 0;
    fence_after();
    if (all) {
        c.phase ^= 1u;
    } else {
        if (c.status && threadIdx.x == 0) atomicMax(c.status, PF_ERR_CUDA);
        c.ok = false;
    }
    return all;
}

// make this thread's shared-memory writes visible to the tensor core and
// order earlier TMEM reads before the next MMA
PF_D void publish() {
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
}

// 64 FP32 accumulator columns -> ReLU -> BF16 activation buffer (with the
// bias column); returns the ReLU mask
PF_D void relu_store(Ctx& c, uint32_t acc_col, uint8_t* buf, uint32_t mask[2]) {
    const int r = threadIdx.x;
    const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31) << 16;
    mask[0] = mask[1] = 0u;
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
        float v[16];
        tmem_ld16(c.tmem + lane_base + acc_col + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int j = 16 * q + i;
            const bool pos = v[i] > 0.0f;
            v[i] = pos ? v[i] : 0.0f;
            if (pos) mask[j >> 5] |= 1u << (j & 31);
        }
        put_chunk(buf, kRays, r, 2 * q, v);
        put_chunk(buf, kRays, r, 2 * q + 1, v + 8);
    }
    float e[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    put_chunk(buf, kRays, r, 8, e);
    e[0] = 0.f;
    put_chunk(buf, kRays, r, 9, e);
}

// 64 data-gradient columns masked by the ReLU -> BF16 dZ buffer
PF_D void dz_store(Ctx& c, uint8_t* buf, const uint32_t mask[2]) {
    const int r = threadIdx.x;
    const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31) << 16;
#pragma unroll 1
    for (int q = 0; q < 4; q++) {
        float v[16];
        tmem_ld16(c.tmem + lane_base + kTmAcc + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int j = 16 * q + i;
            if (!((mask[j >> 5] >> (j & 31)) & 1u)) v[i] = 0.0f;
        }
        put_chunk(buf, kRays, r, 2 * q, v);
        put_chunk(buf, kRays, r, 2 * q + 1, v + 8);
    }
}

PF_D void load_weights(uint8_t* sm, const uint8_t* __restrict__ img) {
    const uint4* src = reinterpret_cast<const uint4*>(img);
    uint4* dst = reinterpret_cast<uint4*>(sm + kSmW);
    for (int i = threadIdx.x; i < kImgBytes / 16; i += blockDim.x) dst[i] = __ldg(src + i);
}

// TMEM allocation by warp 0; every thread learns the base address
PF_D void setup(Ctx& c, uint8_t* sm, int* status, int bar_off = kSmBar, uint32_t cols = kTmCols) {
    c.sm = sm;
    c.sbase = smem_u32(sm);
    c.bar = c.sbase + bar_off;
    c.phase = 0;
    c.status = status;
    c.ok = true;
    c.cols = cols;
    uint32_t slot = c.sbase + bar_off + 16;
    if (threadIdx.x == 0) mbar_init(c.bar, 1);
    if (threadIdx.x < 32) tmem_alloc(slot, cols);
    fence_before();
    __syncthreads();
    fence_after();
    c.tmem = *reinterpret_cast<volatile uint32_t*>(sm + bar_off + 16);
}

PF_D void teardown(Ctx& c) {
    fence_before();
    __syncthreads();
    fence_after();
    if (threadIdx.x < 32) tmem_free(c.tmem, c.cols);
}

// forward of one tile whose encoded rays are in the X buffer; leaves H1..H3
// and the two outputs of this thread's ray in out[2]; masks for the adjoint.
// INF: the inference layout (H3 overwrites H1).
template <bool INF = false>
PF_D bool forward_tile(Ctx& c, float out[2], uint32_t m1[2], uint32_t m2[2], uint32_t m3[2]) {
    constexpr int X = INF ? kFsX : kSmX, H1 = INF ? kFsHa : kSmH1, H2 = INF ? kFsHb : kSmH2,
                  H3 = INF ? kFsHa : kSmH3;
    const uint32_t W = c.sbase + kSmW;
    publish();
    if (threadIdx.x == 0) issue_forward(c.tmem + kTmAcc, c.sbase + X, W + img_off(0), 64);
    if (!commit_wait(c)) return false;
    relu_store(c, kTmAcc, c.sm + H1, m1);
    publish();
    if (threadIdx.x == 0) issue_forward(c.tmem + kTmAcc, c.sbase + H1, W + img_off(1), 64);
    if (!commit_wait(c)) return false;
    relu_store(c, kTmAcc, c.sm + H2, m2);
    publish();
    if (threadIdx.x == 0) issue_forward(c.tmem + kTmAcc, c.sbase + H2, W + img_off(2), 64);
    if (!commit_wait(c)) return false;
    relu_store(c, kTmAcc, c.sm + H3, m3);
    publish();
    if (threadIdx.x == 0) issue_forward(c.tmem + kTmAcc, c.sbase + H3, W + img_off(3), 16);
    if (!commit_wait(c)) return false;
    float v[16];
    tmem_ld16(c.tmem + ((uint32_t)(threadIdx.x & ~31) << 16) + kTmAcc, v);
    out[0] = v[0];
    out[1] = v[1];
    return true;
}

PF_D void put_features(uint8_t* sm, const float f[80], int x_off = kSmX) {
#pragma unroll
    for (int ch = 0; ch < 10; ch++) put_chunk(sm + x_off, kRays, threadIdx.x, ch, f + 8 * ch);
}

PF_D float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

struct FwdArgs {
    const float* rays;  // (n, 6) origin, unit direction; or NULL with a camera
    Cam cam;
    int64_t n;
    const uint8_t* img;
    float* t_out;     // world units
    float* conf_out;  // sigmoid
    int* status;
};

__global__ void __launch_bounds__(128, 2) mlp_forward_kernel(FwdArgs A) {
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    Ctx c;
    load_weights(sm, A.img);
    setup(c, sm, A.status, kFsBar, kFsTmCols);
    const int64_t tiles = (A.n + kRays - 1) / kRays;
    for (int64_t t = blockIdx.x; t < tiles && c.ok; t += gridDim.x) {
        const int64_t i = t * kRays + threadIdx.x;
        const bool valid = i < A.n;
        float u[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 1.f};
        if (valid) {
            if (A.rays) {
                for (int k = 0; k < 6; k++) u[k] = A.rays[6 * i + k];
            } else {
                // pixel ray of the camera, as the tracer casts it (raytrace.py:140-146)
                const int pi = (int)(i / A.cam.W), pj = (int)(i % A.cam.W);
                const v3 d = ray_dir(A.cam, pi, pj);
                u[0] = A.cam.eye.x;
                u[1] = A.cam.eye.y;
                u[2] = A.cam.eye.z;
                u[3] = d.x;
                u[4] = d.y;
                u[5] = d.z;
            }
            u[0] *= (1.0f / 3.0f);
            u[1] *= (1.0f / 3.0f);
            u[2] *= (1.0f / 3.0f);
        }
        float f[80];
        encode(u, f);
        put_features(sm, f, kFsX);
        float out[2];
        uint32_t m1[2], m2[2], m3[2];
        if (!forward_tile<true>(c, out, m1, m2, m3)) break;
        if (valid) {
            A.t_out[i] = out[0] * kTScale;
            A.conf_out[i] = sigmoid(out[1]);
        }
    }
    if (!c.ok && threadIdx.x == 0) mbar_wait(c.bar, c.phase);  // the pending commit, before TMEM is freed
    teardown(c);
}

struct TrainArgs {
    const float* rays;  // (n_rays, 8): origin, unit direction, label t (< 0: no label), no-hit flag
    int64_t n_rays;
    int batch;
    const int* step;  // device step counter (sampling seed)
    uint32_t seed;
    const uint8_t* img;
    float* grad;  // (kParams) fp32, accumulated
    float* loss;  // [0] entry-distance loss, [1] confidence loss (sums over the batch)
    float w_over, margin;
    int* status;
};

PF_D uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(128, 1) mlp_train_kernel(TrainArgs A) {
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    Ctx c;
    load_weights(sm, A.img);
    setup(c, sm, A.status);
    const uint32_t W = c.sbase + kSmW;
    const int step = *A.step;
    const int tiles = (A.batch + kRays - 1) / kRays;
    const float inv_b = 1.0f / (float)A.batch;
    bool first = true;
    float lt = 0.f, lc = 0.f;
    const int r = threadIdx.x;
    const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31) << 16;
    for (int t = blockIdx.x; t < tiles && c.ok; t += gridDim.x) {
        const int bi = t * kRays + r;
        const bool valid = bi < A.batch;
        float u[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 1.f};
        float t_lab = -1.0f, nohit = 0.0f;
        if (valid) {
            const uint32_t h = mix32(mix32((uint32_t)bi * 2654435761u + A.seed) ^ (uint32_t)step * 0x9e3779b9u);
            const int64_t i = (int64_t)(h % (uint32_t)A.n_rays);
            for (int k = 0; k < 6; k++) u[k] = __ldg(&A.rays[8 * i + k]);
            t_lab = __ldg(&A.rays[8 * i + 6]);
            nohit = __ldg(&A.rays[8 * i + 7]);
            u[0] *= (1.0f / 3.0f);
            u[1] *= (1.0f / 3.0f);
            u[2] *= (1.0f / 3.0f);
        }
        float f[80];
        encode(u, f);
        put_features(sm, f);
        float out[2];
        uint32_t m1[2], m2[2], m3[2];
        if (!forward_tile(c, out, m1, m2, m3)) break;
        // loss gradient of this ray
        float g0 = 0.f, g1 = 0.f;
        if (valid) {
            // a flagged ray never reaches a significant cell: its label (where it leaves the
            // primitives' box) is the furthest useful seed, and any seed is safe
            const bool hit = t_lab >= 0.0f, flagged = nohit != 0.0f;
            if (hit) {
                const float e = out[0] - t_lab / kTScale;
                const float w = (e > 0.0f && !flagged) ? A.w_over : 1.0f;
                lt += w * e * e;
                g0 = 2.0f * w * e * inv_b;
            }
            const float safe = (hit && (flagged || out[0] * kTScale - A.margin <= t_lab)) ? 1.0f : 0.0f;
            const float p = sigmoid(out[1]);
            lc += -(safe * logf(fmaxf(p, 1e-12f)) + (1.0f - safe) * logf(fmaxf(1.0f - p, 1e-12f)));
            g1 = (p - safe) * inv_b;
        }
        {
            float g[16] = {g0, g1};
#pragma unroll
            for (int k = 2; k < 16; k++) g[k] = 0.f;
            put_chunk(c.sm + kSmDz4, kRays, r, 0, g);
            put_chunk(c.sm + kSmDz4, kRays, r, 1, g + 8);
        }
        // layer 4: dH3 = dZ4 W4, dW4 += dZ4^T H3
        publish();
        if (threadIdx.x == 0) {
            issue_dgrad(c.tmem + kTmAcc, c.sbase + kSmDz4, W + img_off(3), 16);
            issue_wgrad(c.tmem + tm_grad(3), c.sbase + kSmDz4, c.sbase + kSmH3, !first);
        }
        if (!commit_wait(c)) break;
        dz_store(c, c.sm + kSmDz3, m3);
        publish();
        if (threadIdx.x == 0) {
            issue_dgrad(c.tmem + kTmAcc, c.sbase + kSmDz3, W + img_off(2), 64);
            issue_wgrad(c.tmem + tm_grad(2), c.sbase + kSmDz3, c.sbase + kSmH2, !first);
        }
        if (!commit_wait(c)) break;
        dz_store(c, c.sm + kSmDz2, m2);
        publish();
        if (threadIdx.x == 0) {
            issue_dgrad(c.tmem + kTmAcc, c.sbase + kSmDz2, W + img_off(1), 64);
            issue_wgrad(c.tmem + tm_grad(1), c.sbase + kSmDz2, c.sbase + kSmH1, !first);
        }
        if (!commit_wait(c)) break;
        dz_store(c, c.sm + kSmDz1, m1);
        publish();
        if (threadIdx.x == 0) issue_wgrad(c.tmem + tm_grad(0), c.sbase + kSmDz1, c.sbase + kSmX, !first);
        if (!commit_wait(c)) break;
        first = false;
    }
    if (c.ok && !first) {
        // flush the weight gradients: lane r holds output row r of every layer
#pragma unroll 1
        for (int l = 0; l < kLayers; l++) {
#pragma unroll 1
            for (int q = 0; q < kIn / 16; q++) {
                float v[16];
                tmem_ld16(c.tmem + lane_base + tm_grad(l) + 16 * q, v);
                if (r < layer_out(l))
                    for (int i = 0; i < 16; i++)
                        if (v[i] != 0.0f) atomicAdd(&A.grad[w_off(l) + r * kIn + 16 * q + i], v[i]);
            }
        }
    }
    if (c.ok && A.loss) {
        for (int o = 16; o > 0; o >>= 1) {
            lt += __shfl_xor_sync(0xffffffffu, lt, o);
            lc += __shfl_xor_sync(0xffffffffu, lc, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&A.loss[0], lt);
            atomicAdd(&A.loss[1], lc);
        }
    }
    if (!c.ok && threadIdx.x == 0) mbar_wait(c.bar, c.phase);
    teardown(c);
}

// Adam on the FP32 master weights; writes the BF16 shared-memory image and
// clears the gradient.  The last block to finish advances the step counter.
struct AdamArgs {
    float* w;
    float* m;
    float* v;
    float* grad;
    uint8_t* img;
    int* step;
    unsigned int* done;
    float lr, b1, b2, eps;
};

PF_D int param_layer(int i) { return i < 3 * 64 * kIn ? i / (64 * kIn) : 3; }

PF_D void image_put(uint8_t* img, int i, float w) {
    const int l = param_layer(i);
    const int j = i - w_off(l);
    const int o = j / kIn, k = j % kIn;
    const int out = layer_out(l);
    __nv_bfloat16 h = __float2bfloat16_rn(w);
    *reinterpret_cast<__nv_bfloat16*>(img + img_off(l) + (k / 8) * (out * 16) + o * 16 + (k % 8) * 2) = h;
}

__global__ void mlp_adam_kernel(AdamArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = *A.step + 1;
    if (i < kParams) {
        const float g = A.grad[i];
        const float m = A.b1 * A.m[i] + (1.0f - A.b1) * g;
        const float v = A.b2 * A.v[i] + (1.0f - A.b2) * g * g;
        A.m[i] = m;
        A.v[i] = v;
        const float mh = m / (1.0f - powf(A.b1, (float)t));
        const float vh = v / (1.0f - powf(A.b2, (float)t));
        const float w = A.w[i] - A.lr * mh / (sqrtf(vh) + A.eps);
        A.w[i] = w;
        A.grad[i] = 0.0f;
        image_put(A.img, i, w);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int prev = atomicAdd(A.done, 1u);
        if (prev == gridDim.x - 1) {
            *A.done = 0u;
            __threadfence();
            atomicAdd(A.step, 1);
        }
    }
}

__global__ void mlp_image_kernel(const float* __restrict__ w, uint8_t* __restrict__ img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kParams) image_put(img, i, w[i]);
}

// ---------------------------------------------------------------------------
// self-test of the three operand arrangements (one CTA): D = A B^T with
// A (128 x 128) and B (80 x 128) BF16 row-major in global memory, K = 128.
//   mode 0: A K-major, B K-major      (forward GEMMs)
//   mode 1: A K-major, B MN-major     (data-gradient GEMMs)
//   mode 2: A MN-major, B MN-major    (weight-gradient GEMMs)
__global__ void __launch_bounds__(128, 1)
mlp_selftest_kernel(const uint16_t* __restrict__ a, const uint16_t* __restrict__ b, int mode, float* __restrict__ d,
                    int* status) {
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    constexpr int kA = 0, kB = 32768, kBar = 32768 + 20480;
    const uint32_t sb = smem_u32(sm);
    const int r = threadIdx.x;
    // A (m, k): K-major (k/8)*2048 + m*16 + (k%8)*2; MN-major (m/8)*2048 + (k%8)*16 + (k/8)*128 + (m%8)*2
    for (int k = 0; k < 128; k++) {
        uint16_t v = a[r * 128 + k];
        int off = mode == 2 ? (r / 8) * 2048 + (k % 8) * 16 + (k / 8) * 128 + (r % 8) * 2
                            : (k / 8) * 2048 + r * 16 + (k % 8) * 2;
        *reinterpret_cast<uint16_t*>(sm + kA + off) = v;
    }
    if (r < 80) {
        for (int k = 0; k < 128; k++) {
            uint16_t v = b[r * 128 + k];
            int off = mode == 0 ? (k / 8) * (80 * 16) + r * 16 + (k % 8) * 2
                                : (r / 8) * 2048 + (k % 8) * 16 + (k / 8) * 128 + (r % 8) * 2;
            *reinterpret_cast<uint16_t*>(sm + kB + off) = v;
        }
    }
    Ctx c;
    c.sm = sm;
    c.sbase = sb;
    c.bar = sb + kBar;
    c.phase = 0;
    c.status = status;
    c.ok = true;
    if (threadIdx.x == 0) mbar_init(c.bar, 1);
    if (threadIdx.x < 32) tmem_alloc(sb + kBar + 16, 128);
    fence_before();
    __syncthreads();
    fence_after();
    c.tmem = *reinterpret_cast<volatile uint32_t*>(sm + kBar + 16);
    publish();
    if (threadIdx.x == 0) {
        const uint32_t id = idesc_bf16(128, 80, mode == 2, mode >= 1);
        for (int ks = 0; ks < 8; ks++) {
            uint64_t da, db;
            if (mode == 2) da = sdesc(sb + kA + ks * 256, 128, 2048);
            else da = sdesc(sb + kA + ks * 4096, 2048, 128);
            if (mode == 0) db = sdesc(sb + kB + ks * 2 * (80 * 16), 80 * 16, 128);
            else db = sdesc(sb + kB + ks * 256, 128, 2048);
            mma(c.tmem, da, db, id, ks > 0);
        }
    }
    if (commit_wait(c)) {
#pragma unroll 1
        for (int q = 0; q < 5; q++) {
            float v[16];
            tmem_ld16(c.tmem + ((uint32_t)(threadIdx.x & ~31) << 16) + 16 * q, v);
            for (int i = 0; i < 16; i++) d[r * 80 + 16 * q + i] = v[i];
        }
    } else if (threadIdx.x == 0) {
        mbar_wait(c.bar, c.phase);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (threadIdx.x < 32) tmem_free(c.tmem, 128);
}

static int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace mlp
}  // namespace pf

using namespace pf;
using namespace pf::mlp;

extern "C" int pf_mlp_param_count(void) { return kParams; }
extern "C" int pf_mlp_image_bytes(void) { return kImgBytes; }

extern "C" int pf_mlp_pack(const float* weights, uint8_t* image, void* stream) {
    if (!weights || !image) return pf_fail(PF_ERR_ARGS, "pf_mlp_pack: missing argument");
    mlp_image_kernel<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(weights, image);
    return pf_check_launch("pf_mlp_pack");
}

static int set_smem(const void* f, int bytes) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return pf_fail(PF_ERR_CUDA, cudaGetErrorString(e));
    return PF_OK;
}

extern "C" int pf_mlp_forward(const uint8_t* image, const float* rays, int64_t n_rays, const pf_camera* cam,
                              float* t_entry, float* confidence, int32_t* status, void* stream) {
    if (!image || !t_entry || !confidence || !status || n_rays < 0 || (!rays && !cam))
        return pf_fail(PF_ERR_ARGS, "pf_mlp_forward: missing argument");
    FwdArgs A;
    A.rays = rays;
    if (!rays) {
        if (cam->width < 2 || cam->height < 2) return pf_fail(PF_ERR_ARGS, "pf_mlp_forward: image must be >= 2x2");
        A.cam = load_cam(*cam);
        n_rays = (int64_t)cam->width * cam->height;
    } else {
        A.cam = Cam{};
    }
    A.n = n_rays;
    A.img = image;
    A.t_out = t_entry;
    A.conf_out = confidence;
    A.status = (int*)status;
    if (n_rays == 0) return PF_OK;
    int rc = set_smem((const void*)mlp_forward_kernel, kFsBytes);
    if (rc) return rc;
    const int64_t tiles = (n_rays + kRays - 1) / kRays;
    const unsigned grid = (unsigned)std::min<int64_t>(tiles, 2 * (int64_t)sm_count());
    mlp_forward_kernel<<<grid, 128, kFsBytes, (cudaStream_t)stream>>>(A);
    return pf_check_launch("pf_mlp_forward");
}

extern "C" int pf_mlp_train_step(const uint8_t* image, const float* rays, int64_t n_rays, int32_t batch,
                                 const int32_t* step, uint32_t seed, float overshoot_weight, float margin,
                                 float* grad, float* loss, int32_t* status, void* stream) {
    if (!image || !rays || n_rays <= 0 || n_rays >= ((int64_t)1 << 32) || batch <= 0 || !step || !grad || !status)
        return pf_fail(PF_ERR_ARGS, "pf_mlp_train_step: bad arguments");
    TrainArgs A;
    A.rays = rays;
    A.n_rays = n_rays;
    A.batch = batch;
    A.step = (const int*)step;
    A.seed = seed;
    A.img = image;
    A.grad = grad;
    A.loss = loss;
    A.w_over = overshoot_weight;
    A.margin = margin;
    A.status = (int*)status;
    int rc = set_smem((const void*)mlp_train_kernel, kSmBytes);
    if (rc) return rc;
    const int tiles = (batch + kRays - 1) / kRays;
    const unsigned grid = (unsigned)std::min(tiles, sm_count());
    mlp_train_kernel<<<grid, 128, kSmBytes, (cudaStream_t)stream>>>(A);
    return pf_check_launch("pf_mlp_train_step");
}

extern "C" int pf_mlp_adam(float* weights, float* m, float* v, float* grad, uint8_t* image, int32_t* step,
                           uint32_t* done, float lr, float beta1, float beta2, float eps, void* stream) {
    if (!weights || !m || !v || !grad || !image || !step || !done)
        return pf_fail(PF_ERR_ARGS, "pf_mlp_adam: missing argument");
    AdamArgs A{weights, m, v, grad, image, (int*)step, done, lr, beta1, beta2, eps};
    mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(A);
    return pf_check_launch("pf_mlp_adam");
}

extern "C" int pf_mlp_gemm_selftest(const uint16_t* a, const uint16_t* b, int32_t mode, float* d, int32_t* status,
                                    void* stream) {
    if (!a || !b || !d || !status || mode < 0 || mode > 2)
        return pf_fail(PF_ERR_ARGS, "pf_mlp_gemm_selftest: bad arguments");
    const int bytes = 32768 + 20480 + 64 + 1024;
    int rc = set_smem((const void*)mlp_selftest_kernel, bytes);
    if (rc) return rc;
    mlp_selftest_kernel<<<1, 128, bytes, (cudaStream_t)stream>>>(a, b, mode, d, (int*)status);
    return pf_check_launch("pf_mlp_gemm_selftest");
}

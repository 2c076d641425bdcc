// pf_sort.cuh -- device-wide exclusive scan and stable LSD radix sort.
//
// Both are written from the textbook three-phase formulation (per-block
// reduce / scan of block totals / per-block scan with carry-in; for the sort:
// per-block digit histogram / digit-major scan / stable per-block scatter).
// Item counts may live in device memory (`n_dev`), so a grid sized for an
// upper bound runs without a host round trip: blocks past the live count
// contribute empty histograms.  Stable ranking inside a block uses
// __match_any_sync: within a warp items are ranked in index order, warps are
// ranked in index order, blocks by the digit-major scan.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pf {

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;
constexpr int kScanItems = kScanThreads * kScanPerThread;  // 4096

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// exclusive block scan of one value per thread (blockDim.x == kScanThreads);
// `total` receives the block sum
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T& total) {
    __shared__ T warp_tot[kScanThreads / 32];
    __shared__ T s_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanThreads / 32 ? warp_tot[lane] : T(0);
        T wi = warp_incl_scan(w);
        if (lane < kScanThreads / 32) warp_tot[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) s_total = wi;
    }
    __syncthreads();
    T excl = inc - v + warp_tot[warp];
    total = s_total;
    __syncthreads();
    return excl;
}

template <typename Tin, typename Tout>
__global__ void scan_reduce_kernel(const Tin* __restrict__ in, int64_t n, Tout* __restrict__ partial) {
    int64_t base = (int64_t)blockIdx.x * kScanItems;
    Tout s = 0;
    for (int k = 0; k < kScanPerThread; k++) {
        int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += (Tout)in[i];
    }
    Tout tot;
    block_excl_scan<Tout>(s, tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// single block, exclusive scan of the block totals in place; writes the grand
// total to *total (if not null)
template <typename T>
__global__ void scan_partials_kernel(T* __restrict__ partial, int64_t nb, T* __restrict__ total) {
    T carry = 0;
    for (int64_t b0 = 0; b0 < nb; b0 += kScanThreads) {
        int64_t i = b0 + threadIdx.x;
        T v = i < nb ? partial[i] : T(0);
        T tot;
        T ex = block_excl_scan<T>(v, tot);
        if (i < nb) partial[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <typename Tin, typename Tout>
__global__ void scan_downsweep_kernel(const Tin* __restrict__ in, int64_t n, const Tout* __restrict__ partial,
                                      Tout* __restrict__ out) {
    __shared__ Tout buf[kScanItems];
    int64_t base = (int64_t)blockIdx.x * kScanItems;
    for (int k = 0; k < kScanPerThread; k++) {
        int j = k * kScanThreads + threadIdx.x;
        int64_t i = base + j;
        buf[j] = i < n ? (Tout)in[i] : Tout(0);
    }
    __syncthreads();
    Tout loc[kScanPerThread];
    Tout s = 0;
#pragma unroll
    for (int k = 0; k < kScanPerThread; k++) {
        loc[k] = s;
        s += buf[threadIdx.x * kScanPerThread + k];
    }
    Tout tot;
    Tout ex = block_excl_scan<Tout>(s, tot) + partial[blockIdx.x];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanPerThread; k++) buf[threadIdx.x * kScanPerThread + k] = ex + loc[k];
    __syncthreads();
    for (int k = 0; k < kScanPerThread; k++) {
        int j = k * kScanThreads + threadIdx.x;
        int64_t i = base + j;
        if (i < n) out[i] = buf[j];
    }
}

inline int64_t scan_blocks(int64_t n) { return (n + kScanItems - 1) / kScanItems; }

// Exclusive scan in -> out (n items, host-known); partial needs
// scan_blocks(n) elements; *total receives the sum (device).
template <typename Tin, typename Tout>
inline void exclusive_scan(const Tin* in, Tout* out, int64_t n, Tout* partial, Tout* total, cudaStream_t st) {
    int64_t nb = scan_blocks(n);
    if (nb == 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(Tout), st);
        return;
    }
    scan_reduce_kernel<Tin, Tout><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, partial);
    scan_partials_kernel<Tout><<<1, kScanThreads, 0, st>>>(partial, nb, total);
    scan_downsweep_kernel<Tin, Tout><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, partial, out);
}

// ---------------------------------------------------------------------------
// radix sort
constexpr int kRadixThreads = 256;
constexpr int kRadixPerThread = 16;
constexpr int kRadixItems = kRadixThreads * kRadixPerThread;  // 4096
constexpr int kRadixWarps = kRadixThreads / 32;

__device__ __forceinline__ int64_t live_count(int64_t n_host, const int64_t* n_dev, int64_t cap) {
    if (!n_dev) return n_host;
    int64_t n = *n_dev;
    return n < cap ? n : cap;
}

static __global__ void radix_hist_kernel(const uint32_t* __restrict__ keys, int64_t n_host, const int64_t* n_dev,
                                  int shift, uint32_t* __restrict__ hist, int nblocks) {
    __shared__ uint32_t bins[256];
    bins[threadIdx.x] = 0;
    __syncthreads();
    int64_t n = live_count(n_host, n_dev, n_host);
    int64_t base = (int64_t)blockIdx.x * kRadixItems;
    for (int k = 0; k < kRadixPerThread; k++) {
        int64_t i = base + (int64_t)k * kRadixThreads + threadIdx.x;
        if (i < n) atomicAdd(&bins[(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = bins[threadIdx.x];
}

static __global__ void radix_scatter_kernel(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                     uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n_host,
                                     const int64_t* n_dev, int shift, const uint32_t* __restrict__ offs,
                                     int nblocks) {
    __shared__ uint32_t cnt[kRadixWarps][256];
    __shared__ uint32_t gbase[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = 0; w < kRadixWarps; w++) cnt[w][threadIdx.x] = 0;
    gbase[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    __syncthreads();
    int64_t n = live_count(n_host, n_dev, n_host);
    int64_t base = (int64_t)blockIdx.x * kRadixItems + (int64_t)warp * (kRadixItems / kRadixWarps);
    if ((int64_t)blockIdx.x * kRadixItems >= n) return;
    uint32_t k_[kRadixPerThread], v_[kRadixPerThread], r_[kRadixPerThread];
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
#pragma unroll
    for (int r = 0; r < kRadixPerThread; r++) {
        int64_t i = base + r * 32 + lane;
        bool valid = i < n;
        uint32_t key = valid ? kin[i] : 0u;
        k_[r] = key;
        v_[r] = valid ? vin[i] : 0u;
        uint32_t d = valid ? ((key >> shift) & 0xffu) : 256u;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t before = valid ? cnt[warp][d] : 0u;
        __syncwarp();
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) cnt[warp][d] = before + __popc(peers);
        __syncwarp();
        r_[r] = before + __popc(peers & lt);
    }
    __syncthreads();
    {
        uint32_t s = 0;
        for (int w = 0; w < kRadixWarps; w++) {
            uint32_t t = cnt[w][threadIdx.x];
            cnt[w][threadIdx.x] = s;
            s += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRadixPerThread; r++) {
        int64_t i = base + r * 32 + lane;
        if (i < n) {
            uint32_t d = (k_[r] >> shift) & 0xffu;
            uint32_t pos = gbase[d] + cnt[warp][d] + r_[r];
            kout[pos] = k_[r];
            vout[pos] = v_[r];
        }
    }
}

struct RadixScratch {
    uint32_t* hist;     // 256 * blocks
    uint32_t* partial;  // scan_blocks(256 * blocks)
};

inline int64_t radix_blocks(int64_t cap) { return (cap + kRadixItems - 1) / kRadixItems; }
inline size_t radix_scratch_bytes(int64_t cap) {
    int64_t nb = radix_blocks(cap);
    return sizeof(uint32_t) * (size_t)(256 * nb + scan_blocks(256 * nb) + 1);
}

// Stable sort of (keys, vals) by bits [0, bits) of the keys.  Items start in
// (k0, v0); (k1, v1) is scratch; pass p reads buffer p and writes buffer p+1
// where the intermediate buffers alternate (k1,v1), (k0,v0), ... and the last
// pass writes (kf, vf).  The caller picks (kf, vf) distinct from the last
// intermediate.  n_dev (optional) caps the live count at run time; the grid
// is sized for cap.
inline int radix_passes(int bits) { return (bits + 7) / 8; }

inline void radix_sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, uint32_t* kf, uint32_t* vf,
                             int64_t cap, const int64_t* n_dev, int bits, RadixScratch scr, cudaStream_t st) {
    int passes = radix_passes(bits);
    int64_t nb = radix_blocks(cap);
    if (cap == 0) return;
    if (passes == 0) {
        if (kf != k0) cudaMemcpyAsync(kf, k0, sizeof(uint32_t) * cap, cudaMemcpyDeviceToDevice, st);
        if (vf != v0) cudaMemcpyAsync(vf, v0, sizeof(uint32_t) * cap, cudaMemcpyDeviceToDevice, st);
        return;
    }
    uint32_t *ki = k0, *vi = v0;
    for (int p = 0; p < passes; p++) {
        uint32_t *ko, *vo;
        if (p == passes - 1) {
            ko = kf;
            vo = vf;
        } else if (p % 2 == 0) {
            ko = k1;
            vo = v1;
        } else {
            ko = k0;
            vo = v0;
        }
        radix_hist_kernel<<<(unsigned)nb, kRadixThreads, 0, st>>>(ki, cap, n_dev, 8 * p, scr.hist, (int)nb);
        exclusive_scan<uint32_t, uint32_t>(scr.hist, scr.hist, 256 * nb, scr.partial, (uint32_t*)nullptr, st);
        radix_scatter_kernel<<<(unsigned)nb, kRadixThreads, 0, st>>>(ki, vi, ko, vo, cap, n_dev, 8 * p, scr.hist,
                                                                     (int)nb);
        ki = ko;
        vi = vo;
    }
}

// buffers (kf, vf) must not be the input of the last pass: with (k0, v0) as
// input, that input is (k0, v0) for odd pass counts > 1 ... use this helper
// to pick a legal key destination among k0 / k1.
inline uint32_t* radix_final_key_buffer(uint32_t* k0, uint32_t* k1, int bits) {
    int passes = radix_passes(bits);
    if (passes <= 1) return k1;
    // input of the last pass is k1 when passes-1 is odd, k0 when even
    return ((passes - 1) % 2 == 1) ? k0 : k1;
}

}  // namespace pf

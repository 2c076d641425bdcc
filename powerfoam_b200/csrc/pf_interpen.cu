// pf_interpen.cu -- interpenetration penalty of overlapping spheres and its
// adjoint.
//
// Replaces interpenetration_kernel and InterpenetrationFunction
// (powerfoam/geometry.py:88-189).  For sphere i with list
// adjacency[offsets[i] : offsets[i+1]]
//     areas_i = sum over the list of (s - d)^2 where d < s,
//     d = |c_i - c_j|, s = r_i + r_j,
// accumulated in list order from 0 (the reference's per-thread loop), with
// pow(x, 2) evaluated as the correctly rounded x * x.  The adjoint is the one
// Warp generates for that kernel: per overlapping entry g = (2 (s - d)) dL/dareas_i
// reaches r_i and r_j, and for d > 0 the centre share a = (v / d) (-g),
// v = c_i - c_j, is added to c_i and subtracted from c_j.
//
// Work split: a warp owns 32 consecutive spheres, whose lists form one
// contiguous range of the adjacency array.  The lanes walk that range 32
// entries at a time (coalesced index reads, balanced however uneven the
// degrees), each entry finds its row with a shuffle binary search over the 32
// row starts, and the per-entry terms pass through a per-warp shared buffer in
// which every lane then sums its own row in list order -- so the forward sum
// has the reference's order and is bit-identical to it.  The adjoint adds the
// neighbour's share with one float4 atomic per pair and the own share once per
// sphere.  The kernel is bound by the gather of neighbour spheres (16 B per
// pair, mostly L2 hits for Morton-ordered primitives) and the index stream
// (4 B per pair from HBM).

#include <cstdint>

#include "pf_api.h"
#include "pf_common.cuh"

namespace pf {

constexpr int kIpWarps = 8;             // warps per block
constexpr int kIpChunk = 128;           // entries a warp stages per round
constexpr int kIpPerLane = kIpChunk / 32;
constexpr unsigned kFull = 0xffffffffu;

template <bool BWD>
struct IpTerm {
    using T = float;
};
template <>
struct IpTerm<true> {
    using T = float4;
};

template <bool BWD>
__global__ void __launch_bounds__(kIpWarps * 32)
    interpen_kernel(const float4* __restrict__ spheres, const int32_t* __restrict__ adjacency,
                    const int32_t* __restrict__ offsets, int64_t n, int64_t n_edges,
                    const float* __restrict__ grad_areas,
                    float* __restrict__ areas, float4* __restrict__ grad_spheres, int32_t* __restrict__ status) {
    using T = typename IpTerm<BWD>::T;
    __shared__ T buf[kIpWarps][kIpChunk];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int64_t r0 = ((int64_t)blockIdx.x * kIpWarps + w) * 32;
    if (r0 >= n) return;  // uniform over the warp
    const int64_t i = r0 + lane;
    const bool valid = i < n;
    // lanes past the end hold empty rows at offsets[n]
    const int32_t lo = offsets[valid ? i : n];
    const int32_t hi = valid ? offsets[i + 1] : lo;
    // malformed offsets (decreasing, or outside [0, n_edges]) are clamped
    // and reported; no entry outside the adjacency array is read
    bool bad = valid && hi < lo;
    int32_t e_begin = __shfl_sync(kFull, lo, 0);
    int32_t e_end = __shfl_sync(kFull, hi, 31);
    if (e_begin < 0 || (int64_t)e_end > n_edges) {
        bad = true;
        e_begin = max(e_begin, 0);
        e_end = (int32_t)min((int64_t)e_end, n_edges);
    }
    const float4 me = valid ? spheres[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float ga = (BWD && valid) ? grad_areas[i] : 0.f;
    float acc = 0.f;
    float4 own = make_float4(0.f, 0.f, 0.f, 0.f);
    T* wb = buf[w];

    for (int32_t base = e_begin; base < e_end; base += kIpChunk) {
#pragma unroll
        for (int k = 0; k < kIpPerLane; ++k) {
            const int32_t e = base + k * 32 + lane;
            // row of entry e: the largest lane whose list starts at or before e
            // (empty rows share their start with the next row, which wins)
            int row = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int32_t lp = __shfl_sync(kFull, lo, row + step);
                if (lp <= e) row += step;
            }
            float4 ci;
            ci.x = __shfl_sync(kFull, me.x, row);
            ci.y = __shfl_sync(kFull, me.y, row);
            ci.z = __shfl_sync(kFull, me.z, row);
            ci.w = __shfl_sync(kFull, me.w, row);
            const float gi = BWD ? __shfl_sync(kFull, ga, row) : 0.f;
            T val;
            if constexpr (BWD)
                val = make_float4(0.f, 0.f, 0.f, 0.f);
            else
                val = 0.f;
            if (e < e_end) {
                const int32_t j = __ldg(adjacency + e);
                if ((uint64_t)(int64_t)j >= (uint64_t)n) {
                    bad = true;
                } else {
                    const float4 cj = __ldg(spheres + j);
                    const float vx = ci.x - cj.x, vy = ci.y - cj.y, vz = ci.z - cj.z;
                    const float d = sqrtf(vx * vx + vy * vy + vz * vz);
                    const float s = ci.w + cj.w;
                    if (d < s) {
                        const float x = s - d;
                        if constexpr (BWD) {
                            const float g = (2.f * x) * gi;
                            val.w = g;
                            if (d > 0.f) {
                                val.x = (vx / d) * -g;
                                val.y = (vy / d) * -g;
                                val.z = (vz / d) * -g;
                            }
                            atomicAdd(grad_spheres + j, make_float4(-val.x, -val.y, -val.z, g));
                        } else {
                            val = x * x;
                        }
                    }
                }
            }
            wb[k * 32 + lane] = val;
        }
        __syncwarp();
        const int32_t a = max(lo, base);
        const int32_t b = min(hi, base + kIpChunk);
        for (int32_t e = a; e < b; ++e) {
            if constexpr (BWD) {
                const float4 t = wb[e - base];
                own.x += t.x;
                own.y += t.y;
                own.z += t.z;
                own.w += t.w;
            } else {
                acc += wb[e - base];
            }
        }
        __syncwarp();
    }
    if (bad && status) atomicMax(status, PF_ERR_ARGS);
    if (!valid) return;
    if constexpr (BWD) {
        if (hi > lo) atomicAdd(grad_spheres + i, own);
    } else {
        areas[i] = acc;
    }
}

static bool interpen_args_ok(const float* spheres, const int32_t* adjacency, const int32_t* offsets,
                             int64_t n_prims, int64_t n_edges) {
    return n_prims >= 0 && n_prims < ((int64_t)1 << 31) && n_edges >= 0 && n_edges < ((int64_t)1 << 31) &&
           (n_prims == 0 || (spheres && offsets && ((uintptr_t)spheres & 15) == 0)) && (n_edges == 0 || adjacency);
}

static unsigned interpen_blocks(int64_t n) { return (unsigned)((n + 32 * kIpWarps - 1) / (32 * kIpWarps)); }

}  // namespace pf

using namespace pf;

extern "C" int pf_interpenetration(const float* spheres, const int32_t* adjacency, const int32_t* adjacency_offsets,
                                   int64_t n_prims, int64_t n_edges, float* areas, int32_t* status, void* stream) {
    if (!interpen_args_ok(spheres, adjacency, adjacency_offsets, n_prims, n_edges) || (n_prims > 0 && !areas))
        return pf_fail(PF_ERR_ARGS, "pf_interpenetration: bad arguments");
    if (n_prims == 0) return PF_OK;
    interpen_kernel<false><<<interpen_blocks(n_prims), 32 * kIpWarps, 0, (cudaStream_t)stream>>>(
        (const float4*)spheres, adjacency, adjacency_offsets, n_prims, n_edges, nullptr, areas, nullptr, status);
    return pf_check_launch("pf_interpenetration");
}

extern "C" int pf_interpenetration_backward(const float* spheres, const int32_t* adjacency,
                                            const int32_t* adjacency_offsets, int64_t n_prims, int64_t n_edges,
                                            const float* grad_areas, float* grad_spheres, int32_t* status,
                                            void* stream) {
    if (!interpen_args_ok(spheres, adjacency, adjacency_offsets, n_prims, n_edges) ||
        (n_prims > 0 && (!grad_areas || !grad_spheres || ((uintptr_t)grad_spheres & 15) != 0)))
        return pf_fail(PF_ERR_ARGS, "pf_interpenetration_backward: bad arguments");
    if (n_prims == 0) return PF_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(grad_spheres, 0, 16 * (size_t)n_prims, st) != cudaSuccess)
        return pf_check_launch("pf_interpenetration_backward");
    interpen_kernel<true><<<interpen_blocks(n_prims), 32 * kIpWarps, 0, st>>>(
        (const float4*)spheres, adjacency, adjacency_offsets, n_prims, n_edges, grad_areas, nullptr,
        (float4*)grad_spheres,
        status);
    return pf_check_launch("pf_interpenetration_backward");
}

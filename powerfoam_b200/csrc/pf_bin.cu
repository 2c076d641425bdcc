// pf_bin.cu -- tile binning: count -> depth sort -> scan -> emit -> tile sort.
//
// Replaces rasterize.py:1671-1768 (count_visible_pinhole_kernel :140-200,
// cumsum + .item(), write_visible_pinhole_kernel :293-363, argsort :1767).
// The reference sorts 64-bit (tile << 32 | depth bits) keys with an unstable
// argsort over pairs emitted in atomic order.  Here the order is fixed to
// (tile, depth bits, primitive index) and reached with two cheaper stable
// sorts: primitives are first sorted by their 32-bit depth key (N items, four
// 8-bit passes), the pairs are then emitted in that order and stably sorted by
// tile (ceil(log2 T) bits).  Nothing here waits on the host: the pair count
// stays on the device and a grid sized for the caller's capacity reads it.
#include <mutex>

#include "pf_common.cuh"
#include "pf_sort.cuh"
#include "pf_api.h"

namespace pf {

// camera.py:79-128 proj_sphere_to_obb
struct Obb {
    float uc, vc, r1, r2, vx, vy;
};

PF_D Obb proj_sphere_to_obb(const Cam& cam, v3 center, float radius) {
    v3 C = center - cam.eye;
    float C2 = dot(C, C);
    float R = radius;
    float R2 = R * R;
    v3 X = cam.right, Y = cam.up;
    v3 Z = normalize(cross(Y, X));
    float cx = dot(C, X), cy = dot(C, Y), cz = dot(C, Z);
    // x ** 2.0 taken as the correctly rounded square
    float a = cx * cx - (C2 - R2) * dot(X, X);
    float b = cy * cy - (C2 - R2) * dot(Y, Y);
    float f = cz * cz - (C2 - R2) * dot(Z, Z);
    float c = 2.0f * cx * cy;
    float d = 2.0f * cx * cz;
    float e = 2.0f * cy * cz;
    float denom = 4.0f * a * b - c * c;
    Obb o;
    if (fabsf(denom) < 1e-8f) {
        o.uc = 0.f; o.vc = 0.f; o.r1 = 0.f; o.r2 = 0.f; o.vx = 1.f; o.vy = 0.f;
        return o;
    }
    float uc = (c * e - 2.0f * b * d) / denom;
    float vc = (c * d - 2.0f * a * e) / denom;
    float F0 = a * uc * uc + b * vc * vc + c * uc * vc + d * uc + e * vc + f;
    float term_sqrt = sqrtf((a - b) * (a - b) + c * c);
    float l1 = (a + b + term_sqrt) / 2.0f;
    float l2 = (a + b - term_sqrt) / 2.0f;
    float r1 = sqrtf(-F0 / l1);
    float r2 = sqrtf(-F0 / l2);
    float vx = 0.5f * c;
    float vy = l1 - a;
    float norm = sqrtf(vx * vx + vy * vy);
    if (norm < 1e-6f) {
        vx = 1.0f;
        vy = 0.0f;
    } else {
        vx = vx / norm;
        vy = vy / norm;
    }
    o.uc = uc; o.vc = vc; o.r1 = r1; o.r2 = r2; o.vx = vx; o.vy = vy;
    return o;
}

// camera.py:131-178 verify_tile_obb_intersection
PF_D bool tile_obb(int tile_i, int tile_j, const Cam& cam, int TW, const Obb& o) {
    float u_min = 2.0f * (float)(tile_j * TW) / (float)(cam.W - 1) - 1.0f;
    float u_max = 2.0f * (float)((tile_j + 1) * TW) / (float)(cam.W - 1) - 1.0f;
    float v_max = 1.0f - 2.0f * (float)(tile_i * TW) / (float)(cam.H - 1);
    float v_min = 1.0f - 2.0f * (float)((tile_i + 1) * TW) / (float)(cam.H - 1);
    float u_center = (u_min + u_max) * 0.5f;
    float v_center = (v_min + v_max) * 0.5f;
    float eu = (u_max - u_min) * 0.5f;
    float ev = (v_max - v_min) * 0.5f;
    float du = u_center - o.uc;
    float dv = v_center - o.vc;
    float p1 = du * o.vx + dv * o.vy;
    float t1 = eu * fabsf(o.vx) + ev * fabsf(o.vy);
    if (fabsf(p1) > o.r1 + t1) return false;
    float p2 = du * -o.vy + dv * o.vx;
    float t2 = eu * fabsf(-o.vy) + ev * fabsf(o.vx);
    if (fabsf(p2) > o.r2 + t2) return false;
    return true;
}

// rasterize.py:150-200: cull, project, tile range.  Returns false if culled.
struct TileRange {
    int ti0, ti1, tj0, tj1;
    Obb o;
};

PF_D bool prim_tile_range(const Cam& cam, int TW, v3 center, float radius, TileRange& tr) {
    v3 v = center - cam.eye;
    v3 forward = cross(cam.up, cam.right);
    if (length(v) < 4.0f * radius || dot(v, forward) < 0.1f) return false;
    Obb o = proj_sphere_to_obb(cam, center, radius);
    float extent_u = fabsf(o.vx * o.r1) + fabsf(o.vy * o.r2);
    float extent_v = fabsf(o.vy * o.r1) + fabsf(o.vx * o.r2);
    float u_min = o.uc - extent_u, u_max = o.uc + extent_u;
    float v_min = o.vc - extent_v, v_max = o.vc + extent_v;
    float j_min_f = (u_min + 1.0f) * 0.5f * (float)(cam.W - 1);
    float j_max_f = (u_max + 1.0f) * 0.5f * (float)(cam.W - 1);
    float i_min_f = (1.0f - v_max) * 0.5f * (float)(cam.H - 1);
    float i_max_f = (1.0f - v_min) * 0.5f * (float)(cam.H - 1);
    int i_min = imax(sat_f2i(floorf(i_min_f)), 0);
    int i_max = imin(sat_f2i(ceilf(i_max_f)), cam.H - 1);
    int j_min = imax(sat_f2i(floorf(j_min_f)), 0);
    int j_max = imin(sat_f2i(ceilf(j_max_f)), cam.W - 1);
    // Warp's integer // is C division (truncation toward zero)
    tr.ti0 = i_min / TW;
    tr.ti1 = i_max / TW;
    tr.tj0 = j_min / TW;
    tr.tj1 = j_max / TW;
    tr.o = o;
    return true;
}

// ---------------------------------------------------------------------------
// Generic cameras (rasterize.py:202-291, 365-569, 1518-1585): a hierarchy of
// ray cones over the ray map -- leaves of 2x2 pixels, each level merging 2x2
// children, up to one root -- and a per-primitive descent into every child
// cone the sphere meets (camera.py:28-44); the cones of the tile level are
// the tiles.  Level sizes are host-known; the cones live in the workspace.
constexpr int kConeLeaf = 2;
constexpr int kConeMaxLevels = 24;
constexpr int kConeStack = 4 * kConeMaxLevels;

struct ConeTree {
    const float4* cones;
    int n_levels, tile_level;
    int off[kConeMaxLevels], dh[kConeMaxLevels], dw[kConeMaxLevels];
};

// level sizes of an H x W image and the level whose cones are TW x TW tiles;
// false if the image needs more levels or TW is not a power of two >= 2
static bool cone_layout(int H, int W, int TW, ConeTree& ct, int64_t* total) {
    if (TW < kConeLeaf || (TW & (TW - 1))) return false;
    int dh = (H + kConeLeaf - 1) / kConeLeaf, dw = (W + kConeLeaf - 1) / kConeLeaf;
    int64_t t = 0;
    ct.n_levels = 0;
    for (;;) {
        if (ct.n_levels == kConeMaxLevels) return false;
        ct.off[ct.n_levels] = (int)t;
        ct.dh[ct.n_levels] = dh;
        ct.dw[ct.n_levels] = dw;
        ct.n_levels++;
        t += (int64_t)dh * dw;
        if (dh == 1 && dw == 1) break;
        dh = (dh + 1) / 2;
        dw = (dw + 1) / 2;
    }
    ct.tile_level = 0;
    for (int sz = kConeLeaf; sz < TW; sz *= 2) ct.tile_level++;
    *total = t;
    return true;
}

// compute_leaf_cones_kernel (rasterize.py:473-515): axis = normalised sum of
// the unit rays of the 2x2 pixels, cos half angle = min dot (2: no ray)
__global__ void cone_leaf_kernel(const float* __restrict__ ray_maps, int H, int W, int leaf_w, int64_t n,
                                 float4* __restrict__ cones) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int a = (int)(t / leaf_w), b = (int)(t % leaf_w);
    v3 sum = mk(0.f, 0.f, 0.f), rays[4];
    int valid = 0;
    for (int di = 0; di < kConeLeaf; di++)
        for (int dj = 0; dj < kConeLeaf; dj++) {
            const int pi = imin(a * kConeLeaf + di, H - 1), pj = imin(b * kConeLeaf + dj, W - 1);
            const float* m = ray_maps + 6 * ((int64_t)pi * W + pj) + 3;
            const v3 ray = mk(m[0], m[1], m[2]);
            const float len = length(ray);
            if (len > 1.0e-6f) {
                const v3 rn = ray / len;
                rays[valid++] = rn;
                sum = sum + rn;
            }
        }
    if (valid == 0) {
        cones[t] = make_float4(0.f, 0.f, 0.f, 2.0f);
        return;
    }
    const v3 axis = normalize(sum);
    float ch = 1.0f;
    for (int i = 0; i < valid; i++) ch = fmin_t(ch, dot(axis, rays[i]));
    cones[t] = make_float4(axis.x, axis.y, axis.z, ch);
}

// merge_cones_kernel (rasterize.py:517-569)
__global__ void cone_merge_kernel(float4* __restrict__ cones, int parent_off, int child_off, int parent_w,
                                  int child_h, int child_w, int64_t n) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int a = (int)(t / parent_w), b = (int)(t % parent_w);
    v3 sum = mk(0.f, 0.f, 0.f), axes[4];
    float chs[4];
    int valid = 0;
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++) {
            const int ca = 2 * a + di, cb = 2 * b + dj;
            if (ca < child_h && cb < child_w) {
                const float4 c = cones[child_off + (int64_t)ca * child_w + cb];
                if (c.w <= 1.0f) {
                    axes[valid] = mk(c.x, c.y, c.z);
                    chs[valid] = c.w;
                    sum = sum + axes[valid];
                    valid++;
                }
            }
        }
    if (valid == 0) {
        cones[parent_off + t] = make_float4(0.f, 0.f, 0.f, 2.0f);
        return;
    }
    const v3 axis = normalize(sum);
    float ch = 1.0f;
    for (int i = 0; i < valid; i++) {
        const float dv = dot(axis, axes[i]);
        const float sin_angle = sqrtf(fmax_t(1.0f - dv * dv, 0.0f));
        const float sin_child = sqrtf(fmax_t(1.0f - chs[i] * chs[i], 0.0f));
        ch = fmin_t(ch, dv * chs[i] - sin_angle * sin_child);
    }
    cones[parent_off + t] = make_float4(axis.x, axis.y, axis.z, ch);
}

// camera.py:28-44
PF_D bool sphere_cone(v3 center, float radius, v3 eye, v3 axis, float cos_half) {
    const v3 v = center - eye;
    const float dist = length(v);
    const float cos_alpha = dot(v, axis) / dist;
    const float sin_half = sqrtf(1.0f - cos_half * cos_half);
    const float sin_beta = radius / dist;
    const float cos_beta = sqrtf(1.0f - sin_beta * sin_beta);
    const float threshold = cos_half * cos_beta - sin_half * sin_beta;
    return cos_alpha > threshold;
}

// the generic kernels' cull and descent (rasterize.py:214-291): calls
// emit(tile) for every tile-level cone the sphere reaches; false if culled
template <typename Emit>
PF_D bool cone_tiles(const Cam& cam, const ConeTree& ct, int tiles_h, v3 c, float r, Emit emit) {
    const v3 v = c - cam.eye;
    const v3 forward = cross(cam.up, cam.right);
    if (length(v) < 4.0f * r || dot(v, forward) < 0.1f) return false;
    int st_l[kConeStack], st_a[kConeStack], st_b[kConeStack];
    int n = 1;
    st_l[0] = ct.n_levels - 1;
    st_a[0] = 0;
    st_b[0] = 0;
    while (n > 0) {
        n--;
        const int level = st_l[n], a = st_a[n], b = st_b[n];
        const float4 cn = ct.cones[ct.off[level] + (int64_t)a * ct.dw[level] + b];
        if (cn.w > 1.0f) continue;
        if (!sphere_cone(c, r, cam.eye, mk(cn.x, cn.y, cn.z), cn.w)) continue;
        if (level == ct.tile_level) {
            emit(a + b * tiles_h);
            continue;
        }
        const int cl = level - 1;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++) {
                const int ca = 2 * a + di, cb = 2 * b + dj;
                if (ca < ct.dh[cl] && cb < ct.dw[cl]) {  // at most 1 + 3 (levels - 1) entries
                    st_l[n] = cl;
                    st_a[n] = ca;
                    st_b[n] = cb;
                    n++;
                }
            }
    }
    return true;
}

template <bool GEN>
__global__ void bin_count_kernel(pf_camera camera, int TW, const float4* __restrict__ spheres, int64_t N,
                                 int32_t* __restrict__ counts, uint32_t* __restrict__ depth_key,
                                 uint32_t* __restrict__ depth_by_prim, uint32_t* __restrict__ idx, ConeTree ct) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    Cam cam = load_cam(camera);
    float4 s = spheres[p];
    v3 c = mk(s.x, s.y, s.z);
    v3 v = c - cam.eye;
    float pow_dist = dot(v, v) - s.w * s.w;
    depth_key[p] = __float_as_uint(pow_dist);
    depth_by_prim[p] = __float_as_uint(pow_dist);
    idx[p] = (uint32_t)p;
    int n = 0;
    if constexpr (GEN) {
        cone_tiles(cam, ct, 1 + (cam.H - 1) / TW, c, s.w, [&](int) { n++; });
    } else {
        TileRange tr;
        if (prim_tile_range(cam, TW, c, s.w, tr)) {
            for (int ti = tr.ti0; ti <= tr.ti1; ti++)
                for (int tj = tr.tj0; tj <= tr.tj1; tj++)
                    if (tile_obb(ti, tj, cam, TW, tr.o)) n++;
        }
    }
    counts[p] = n;
}

__global__ void gather_counts_kernel(const uint32_t* __restrict__ order, const int32_t* __restrict__ counts,
                                     int64_t N, int32_t* __restrict__ sorted_counts) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < N) sorted_counts[k] = counts[order[k]];
}

template <bool GEN>
__global__ void bin_emit_kernel(pf_camera camera, int TW, const float4* __restrict__ spheres, int64_t N,
                                const uint32_t* __restrict__ order, const int32_t* __restrict__ sorted_counts,
                                const int64_t* __restrict__ offsets, const int64_t* __restrict__ total,
                                int64_t capacity, uint32_t* __restrict__ tile_key, uint32_t* __restrict__ pair_prim,
                                uint8_t* __restrict__ prim_visible, ConeTree ct) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    if (*total > capacity) return;
    if (sorted_counts[k] == 0) return;
    uint32_t p = order[k];
    if (prim_visible) prim_visible[p] = 1;
    Cam cam = load_cam(camera);
    int tiles_h = 1 + (cam.H - 1) / TW;
    float4 s = spheres[p];
    v3 c = mk(s.x, s.y, s.z);
    int64_t pos = offsets[k];
    if constexpr (GEN) {
        // the descent finds the same tiles as the counting pass did
        const int64_t end = pos + sorted_counts[k];
        cone_tiles(cam, ct, tiles_h, c, s.w, [&](int tile) {
            if (pos < end) {
                tile_key[pos] = (uint32_t)tile;
                pair_prim[pos] = p;
                pos++;
            }
        });
        return;
    }
    TileRange tr;
    if (!prim_tile_range(cam, TW, c, s.w, tr)) return;
    for (int ti = tr.ti0; ti <= tr.ti1; ti++)
        for (int tj = tr.tj0; tj <= tr.tj1; tj++)
            if (tile_obb(ti, tj, cam, TW, tr.o)) {
                tile_key[pos] = (uint32_t)(ti + tj * tiles_h);
                pair_prim[pos] = p;
                pos++;
            }
}

// tile_offsets[t] = first sorted position with tile >= t; also the optional
// 64-bit reference keys.  Grid over capacity; the live count is on device.
__global__ void tile_ranges_kernel(const uint32_t* __restrict__ tile_key, const int32_t* __restrict__ prims,
                                   const uint32_t* __restrict__ depth_key, const int64_t* __restrict__ total,
                                   int64_t capacity, int64_t T, int64_t* __restrict__ tile_offsets,
                                   int64_t* __restrict__ sort_keys, int32_t* __restrict__ status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t n = *total;
    if (n > capacity) {
        // overflow: empty every list, report
        for (int64_t t = i; t <= T; t += (int64_t)gridDim.x * blockDim.x) tile_offsets[t] = 0;
        if (i == 0) atomicMax(status, PF_ERR_OVERFLOW);
        return;
    }
    if (i > n) return;
    int64_t lo = (i == 0) ? 0 : (int64_t)tile_key[i - 1] + 1;
    int64_t hi = (i == n) ? T : (int64_t)tile_key[i];
    for (int64_t t = lo; t <= hi; t++) tile_offsets[t] = i;
    if (i < n && sort_keys) sort_keys[i] = ((int64_t)tile_key[i] << 32) | (int64_t)depth_key[prims[i]];
}

// keys for the tile processing order: longest lists first, ties by tile index
__global__ void tile_len_key_kernel(const int64_t* __restrict__ tile_offsets, int64_t T, uint32_t* __restrict__ key,
                                    uint32_t* __restrict__ idx) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    int64_t len = tile_offsets[t + 1] - tile_offsets[t];
    if (len > 0xFFFFFF) len = 0xFFFFFF;
    key[t] = 0xFFFFFFu - (uint32_t)len;
    idx[t] = (uint32_t)t;
}

__global__ void pack_prims_kernel(const float* __restrict__ points, const float* __restrict__ radii,
                                  const float* __restrict__ normals, const float* __restrict__ density, int64_t N,
                                  float4* __restrict__ spheres, float4* __restrict__ nsigmas,
                                  int32_t* __restrict__ status) {
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    bool finite = true;
    if (spheres) {
        float4 s = make_float4(points[3 * p], points[3 * p + 1], points[3 * p + 2], radii[p]);
        spheres[p] = s;
        finite = isfinite(s.x) && isfinite(s.y) && isfinite(s.z) && isfinite(s.w);
    }
    if (nsigmas) {
        float4 n = make_float4(normals[3 * p], normals[3 * p + 1], normals[3 * p + 2], density[p]);
        nsigmas[p] = n;
        finite = finite && isfinite(n.x) && isfinite(n.y) && isfinite(n.z) && isfinite(n.w);
    }
    if (status && !finite) atomicMax(status, PF_ERR_NONFINITE);
}

// ---------------------------------------------------------------------------
struct BinLayout {
    size_t counts, dprim, dkey0, idx0, dkey1, idx1, scounts, offsets, spart, pkey0, pprim0, pkey1, pprim1, tk0, tv0,
        tk1, tv1, rhist, rpart, total;
    size_t bytes;
};

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

static BinLayout bin_layout(int64_t N, int64_t cap, int64_t T) {
    BinLayout L;
    size_t o = 0;
    auto take = [&](size_t b) {
        size_t r = o;
        o = align_up(o + b);
        return r;
    };
    L.counts = take(4 * (size_t)N);
    L.dprim = take(4 * (size_t)N);
    L.dkey0 = take(4 * (size_t)N);
    L.idx0 = take(4 * (size_t)N);
    L.dkey1 = take(4 * (size_t)N);
    L.idx1 = take(4 * (size_t)N);
    L.scounts = take(4 * (size_t)N);
    L.offsets = take(8 * (size_t)N);
    L.spart = take(8 * (size_t)(scan_blocks(N) + 1));
    L.pkey0 = take(4 * (size_t)cap);
    L.pprim0 = take(4 * (size_t)cap);
    L.pkey1 = take(4 * (size_t)cap);
    L.pprim1 = take(4 * (size_t)cap);
    L.tk0 = take(4 * (size_t)T);
    L.tv0 = take(4 * (size_t)T);
    L.tk1 = take(4 * (size_t)T);
    L.tv1 = take(4 * (size_t)T);
    int64_t mx = cap > N ? cap : N;
    mx = mx > T ? mx : T;
    int64_t rb = radix_blocks(mx);
    L.rhist = take(4 * (size_t)(256 * rb));
    L.rpart = take(4 * (size_t)(scan_blocks(256 * rb) + 1));
    L.total = take(8);
    L.bytes = o;
    return L;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_bin_workspace_size(int64_t n_prims, int64_t pair_capacity, int64_t n_tiles, size_t* bytes) {
    if (n_prims < 0 || pair_capacity < 0 || pair_capacity >= (int64_t)1 << 31 || n_tiles < 0 || !bytes)
        return pf_fail(PF_ERR_ARGS, "pf_bin_workspace_size: bad arguments");
    *bytes = bin_layout(n_prims, pair_capacity, n_tiles).bytes;
    return PF_OK;
}

extern "C" int pf_pack_prims(const float* points, const float* radii, const float* normals, const float* density,
                             int64_t n_prims, float* spheres, float* nsigmas, int32_t* status, void* stream) {
    if (n_prims < 0) return pf_fail(PF_ERR_ARGS, "pf_pack_prims: n_prims < 0");
    if (n_prims == 0) return PF_OK;
    if ((spheres && (!points || !radii)) || (nsigmas && (!normals || !density)))
        return pf_fail(PF_ERR_ARGS, "pf_pack_prims: missing input");
    cudaStream_t st = (cudaStream_t)stream;
    pack_prims_kernel<<<(unsigned)((n_prims + 255) / 256), 256, 0, st>>>(points, radii, normals, density, n_prims,
                                                                        (float4*)spheres, (float4*)nsigmas, status);
    return pf_check_launch("pf_pack_prims");
}

// the pinhole binning (ct == NULL) or the generic one over a built cone tree
static int bin_impl(const pf_camera* cam, int32_t tile_width, const float* spheres, int64_t n_prims,
                    void* workspace, size_t workspace_bytes, int64_t pair_capacity, int64_t* tile_offsets,
                    int32_t* tile_prims, int64_t* sort_keys, uint8_t* prim_visible, int32_t* tile_order,
                    int64_t* n_pairs, int32_t* status, void* stream, const ConeTree* ct) {
    if (!cam || tile_width <= 0 || n_prims < 0 || pair_capacity < 0 || pair_capacity >= (int64_t)1 << 31 ||
        !tile_offsets || !n_pairs || !status || (n_prims > 0 && !spheres) || (pair_capacity > 0 && !tile_prims))
        return pf_fail(PF_ERR_ARGS, "pf_bin: bad arguments");
    if (cam->width < 2 || cam->height < 2) return pf_fail(PF_ERR_ARGS, "pf_bin: image must be at least 2x2");
    const int64_t T_ = (int64_t)(1 + (cam->height - 1) / tile_width) * (1 + (cam->width - 1) / tile_width);
    BinLayout L = bin_layout(n_prims, pair_capacity, T_);
    if (workspace_bytes < L.bytes || (!workspace && L.bytes)) return pf_fail(PF_ERR_ARGS, "pf_bin: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const ConeTree no_cones{};
    char* ws = (char*)workspace;
    int32_t* counts = (int32_t*)(ws + L.counts);
    uint32_t* dprim = (uint32_t*)(ws + L.dprim);
    uint32_t* dkey0 = (uint32_t*)(ws + L.dkey0);
    uint32_t* idx0 = (uint32_t*)(ws + L.idx0);
    uint32_t* dkey1 = (uint32_t*)(ws + L.dkey1);
    uint32_t* idx1 = (uint32_t*)(ws + L.idx1);
    int32_t* scounts = (int32_t*)(ws + L.scounts);
    int64_t* offsets = (int64_t*)(ws + L.offsets);
    int64_t* spart = (int64_t*)(ws + L.spart);
    uint32_t* pkey0 = (uint32_t*)(ws + L.pkey0);
    uint32_t* pprim0 = (uint32_t*)(ws + L.pprim0);
    uint32_t* pkey1 = (uint32_t*)(ws + L.pkey1);
    uint32_t* pprim1 = (uint32_t*)(ws + L.pprim1);
    RadixScratch rs{(uint32_t*)(ws + L.rhist), (uint32_t*)(ws + L.rpart)};
    const int TW = tile_width;
    const int64_t tiles_h = 1 + (cam->height - 1) / TW, tiles_w = 1 + (cam->width - 1) / TW;
    const int64_t T = tiles_h * tiles_w;
    if (prim_visible && n_prims) cudaMemsetAsync(prim_visible, 0, (size_t)n_prims, st);
    auto order = [&]() {
        if (!tile_order || T == 0) return;
        uint32_t *tk0 = (uint32_t*)(ws + L.tk0), *tv0 = (uint32_t*)(ws + L.tv0);
        uint32_t *tk1 = (uint32_t*)(ws + L.tk1), *tv1 = (uint32_t*)(ws + L.tv1);
        tile_len_key_kernel<<<(unsigned)((T + 255) / 256), 256, 0, st>>>(tile_offsets, T, tk0, tv0);
        uint32_t* kf = radix_final_key_buffer(tk0, tk1, 24);
        radix_sort_pairs(tk0, tv0, tk1, tv1, kf, (uint32_t*)tile_order, T, nullptr, 24, rs, st);
    };
    if (n_prims == 0) {
        cudaMemsetAsync(n_pairs, 0, 8, st);
        cudaMemsetAsync(tile_offsets, 0, 8 * (size_t)(T + 1), st);
        order();
        return pf_check_launch("pf_bin");
    }
    const unsigned gN = (unsigned)((n_prims + 255) / 256);
    if (ct)
        bin_count_kernel<true><<<gN, 256, 0, st>>>(*cam, TW, (const float4*)spheres, n_prims, counts, dkey0, dprim,
                                                   idx0, *ct);
    else
        bin_count_kernel<false><<<gN, 256, 0, st>>>(*cam, TW, (const float4*)spheres, n_prims, counts, dkey0, dprim,
                                                    idx0, no_cones);
    // stable sort of primitives by depth bits: 4 passes, result back in (dkey0, idx0)
    radix_sort_pairs(dkey0, idx0, dkey1, idx1, dkey0, idx0, n_prims, nullptr, 32, rs, st);
    gather_counts_kernel<<<gN, 256, 0, st>>>(idx0, counts, n_prims, scounts);
    exclusive_scan<int32_t, int64_t>(scounts, offsets, n_prims, spart, n_pairs, st);
    if (ct)
        bin_emit_kernel<true><<<gN, 256, 0, st>>>(*cam, TW, (const float4*)spheres, n_prims, idx0, scounts, offsets,
                                                  n_pairs, pair_capacity, pkey0, pprim0, prim_visible, *ct);
    else
        bin_emit_kernel<false><<<gN, 256, 0, st>>>(*cam, TW, (const float4*)spheres, n_prims, idx0, scounts, offsets,
                                                   n_pairs, pair_capacity, pkey0, pprim0, prim_visible, no_cones);
    // stable sort of the pairs by tile
    int bits = 0;
    while (((int64_t)1 << bits) < T) bits++;
    uint32_t* kf = radix_final_key_buffer(pkey0, pkey1, bits);
    radix_sort_pairs(pkey0, pprim0, pkey1, pprim1, kf, (uint32_t*)tile_prims, pair_capacity, n_pairs, bits, rs, st);
    int64_t nthreads = pair_capacity + 1;
    tile_ranges_kernel<<<(unsigned)((nthreads + 255) / 256), 256, 0, st>>>(kf, tile_prims, dprim, n_pairs,
                                                                           pair_capacity, T, tile_offsets,
                                                                           sort_keys, status);
    order();
    return pf_check_launch("pf_bin");
}

extern "C" int pf_bin(const pf_camera* cam, int32_t tile_width, const float* spheres, int64_t n_prims,
                      void* workspace, size_t workspace_bytes, int64_t pair_capacity, int64_t* tile_offsets,
                      int32_t* tile_prims, int64_t* sort_keys, uint8_t* prim_visible, int32_t* tile_order,
                      int64_t* n_pairs, int32_t* status, void* stream) {
    return bin_impl(cam, tile_width, spheres, n_prims, workspace, workspace_bytes, pair_capacity, tile_offsets,
                    tile_prims, sort_keys, prim_visible, tile_order, n_pairs, status, stream, nullptr);
}

extern "C" int pf_bin_generic_workspace_size(int64_t n_prims, int64_t pair_capacity, int32_t width, int32_t height,
                                             int32_t tile_width, size_t* bytes) {
    ConeTree ct{};
    int64_t n_cones = 0;
    if (!bytes || width < 2 || height < 2 || !cone_layout(height, width, tile_width, ct, &n_cones))
        return pf_fail(PF_ERR_ARGS, "pf_bin_generic_workspace_size: bad arguments (tile_width must be 2, 4, 8, ...)");
    const int64_t T = (int64_t)(1 + (height - 1) / tile_width) * (1 + (width - 1) / tile_width);
    size_t b = 0;
    int rc = pf_bin_workspace_size(n_prims, pair_capacity, T, &b);
    if (rc != PF_OK) return rc;
    *bytes = align_up(b) + align_up(16 * (size_t)n_cones);
    return PF_OK;
}

extern "C" int pf_bin_generic(const pf_camera* cam, const float* ray_maps, int32_t tile_width, const float* spheres,
                              int64_t n_prims, void* workspace, size_t workspace_bytes, int64_t pair_capacity,
                              int64_t* tile_offsets, int32_t* tile_prims, int64_t* sort_keys, uint8_t* prim_visible,
                              int32_t* tile_order, int64_t* n_pairs, int32_t* status, void* stream) {
    ConeTree ct{};
    int64_t n_cones = 0;
    if (!cam || !ray_maps || cam->width < 2 || cam->height < 2 ||
        !cone_layout(cam->height, cam->width, tile_width, ct, &n_cones))
        return pf_fail(PF_ERR_ARGS, "pf_bin_generic: bad camera, ray maps or tile width (2, 4, 8, ...)");
    size_t need = 0;
    int rc = pf_bin_generic_workspace_size(n_prims, pair_capacity, cam->width, cam->height, tile_width, &need);
    if (rc != PF_OK) return rc;
    if (!workspace || workspace_bytes < need) return pf_fail(PF_ERR_ARGS, "pf_bin_generic: workspace too small");
    const int64_t T = (int64_t)(1 + (cam->height - 1) / tile_width) * (1 + (cam->width - 1) / tile_width);
    const size_t bin_bytes = align_up(bin_layout(n_prims, pair_capacity, T).bytes);
    float4* cones = (float4*)((char*)workspace + bin_bytes);
    ct.cones = cones;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n_leaf = (int64_t)ct.dh[0] * ct.dw[0];
    cone_leaf_kernel<<<(unsigned)((n_leaf + 255) / 256), 256, 0, st>>>(ray_maps, cam->height, cam->width, ct.dw[0],
                                                                       n_leaf, cones);
    for (int l = 1; l < ct.n_levels; l++) {
        const int64_t n = (int64_t)ct.dh[l] * ct.dw[l];
        cone_merge_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(cones, ct.off[l], ct.off[l - 1], ct.dw[l],
                                                                       ct.dh[l - 1], ct.dw[l - 1], n);
    }
    return bin_impl(cam, tile_width, spheres, n_prims, workspace, bin_bytes, pair_capacity, tile_offsets, tile_prims,
                    sort_keys, prim_visible, tile_order, n_pairs, status, stream, &ct);
}

// ---------------------------------------------------------------------------
// Allocation-free binning.
//
// Some callers cannot allocate device memory at the moment they bin: a render
// callback running inside another application's frame (a viewer or plugin host
// that owns the CUDA context and its allocator), or code that must not call
// cudaMalloc while the device is busy with other work, since that call can
// synchronise the device.  pf_bin_noalloc serves them: the caller still passes
// the inputs and every output, and the binning scratch lives in the
// file-scope array below, so the call allocates nothing.
//
// Limits (the array is sized for them; larger problems are rejected with
// PF_ERR_ARGS): at most kNoAllocMaxPrims primitives, kNoAllocMaxPairs
// (tile, primitive) pairs of capacity and kNoAllocMaxTiles tiles.  The array
// (kNoAllocBytes = 7 MiB) is held on every GPU that loads the library, until
// the process exits.
//
// The first call on a device looks up the array's device address (with that
// device current) and caches it; make that first call before any stream
// capture.  The cached address belongs to the device's primary context: a
// cudaDeviceReset (or another context made current on that device) leaves it
// stale, and calls after one are not supported.  Every call shares the one array: calls whose work may overlap on
// the GPU (different streams, or different host threads, without ordering
// between them) race on it and must be serialised by the caller.  No part of
// the scratch needs to start at zero: every buffer in it is written before it
// is read.  The caller's *status word must be zero before the call, as for
// pf_bin.
namespace pf {
constexpr int64_t kNoAllocMaxPrims = 1 << 16;
constexpr int64_t kNoAllocMaxPairs = 1 << 18;
constexpr int64_t kNoAllocMaxTiles = 1 << 14;
constexpr size_t kNoAllocBytes = (size_t)7 << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_bin_scratch[kNoAllocBytes];

static std::mutex g_scratch_mu;
static void* g_scratch_ptr[kNoAllocMaxDevices];
}  // namespace pf

extern "C" int pf_bin_noalloc(const pf_camera* cam, int32_t tile_width, const float* spheres, int64_t n_prims,
                              int64_t pair_capacity, int64_t* tile_offsets, int32_t* tile_prims, int64_t* sort_keys,
                              uint8_t* prim_visible, int32_t* tile_order, int64_t* n_pairs, int32_t* status,
                              void* stream) {
    if (!cam || tile_width <= 0 || cam->width < 2 || cam->height < 2)
        return pf_fail(PF_ERR_ARGS, "pf_bin_noalloc: bad camera or tile width");
    const int64_t T = (int64_t)(1 + (cam->height - 1) / tile_width) * (1 + (cam->width - 1) / tile_width);
    if (n_prims < 0 || n_prims > kNoAllocMaxPrims)
        return pf_fail(PF_ERR_ARGS, "pf_bin_noalloc: n_prims exceeds the static scratch limit of 65536 primitives");
    if (pair_capacity < 0 || pair_capacity > kNoAllocMaxPairs)
        return pf_fail(PF_ERR_ARGS, "pf_bin_noalloc: pair_capacity exceeds the static scratch limit of 262144 pairs");
    if (T > kNoAllocMaxTiles)
        return pf_fail(PF_ERR_ARGS, "pf_bin_noalloc: the image has more than 16384 tiles");
    size_t need = 0;
    int rc = pf_bin_workspace_size(n_prims, pair_capacity, T, &need);
    if (rc != PF_OK) return rc;
    if (need > kNoAllocBytes) return pf_fail(PF_ERR_ARGS, "pf_bin_noalloc: problem does not fit the static scratch");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
        return pf_fail(PF_ERR_CUDA, "pf_bin_noalloc: no usable current device");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_bin_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return pf_fail(PF_ERR_CUDA, "pf_bin_noalloc: cudaGetSymbolAddress of the static scratch failed");
            }
            g_scratch_ptr[dev] = p;
        }
        scratch = g_scratch_ptr[dev];
    }
    return pf_bin(cam, tile_width, spheres, n_prims, scratch, kNoAllocBytes, pair_capacity, tile_offsets, tile_prims,
                  sort_keys, prim_visible, tile_order, n_pairs, status, stream);
}

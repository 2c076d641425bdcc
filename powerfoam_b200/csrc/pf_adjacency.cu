// pf_adjacency.cu -- Čech adjacency (overlapping balls) and Morton ordering.
//
// The reference builds the Čech adjacency by querying a Warp BVH over the
// spheres' AABBs (powerfoam/bvh.py:7-123): j is a neighbour of i iff their
// AABBs overlap and |c_i - c_j| < r_i + r_j, with c and r recovered from the
// AABB (c = (lo + hi) / 2, r = (hi.x - lo.x) / 2).  Here the same predicate is
// evaluated over a uniform grid of cell edge 2 * max r: primitives are sorted
// by cell with the library's radix sort, every primitive scans the 27 cells
// around its own, counts, a scan sizes the lists, a second pass writes them
// and each list is sorted ascending (the reference's order is the BVH
// traversal order; ascending order is the canonical form used everywhere
// here).  The pair count stays on the device: the caller passes a capacity
// and reads *n_edges to grow it, exactly as for binning.
//
// morton_sort follows powerfoam/geometry.py:7-85: 21-bit quantisation per
// axis over the bounding box, code = x << 2 | y << 1 | z interleaved, stable
// sort of the primitive ids by the 63-bit code.
#include <algorithm>

#include "pf_common.cuh"
#include "pf_sort.cuh"
#include "pf_api.h"
#include "pf_power.cuh"

namespace pf {


__global__ void bounds_kernel(const float* __restrict__ pts, const float* __restrict__ radii, int64_t N,
                              float* __restrict__ out /* lo3, hi3, rmax */) {
    __shared__ float s[7][32];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}, rm = 0.f;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; k++) {
            float v = pts[3 * i + k];
            lo[k] = fminf(lo[k], v);
            hi[k] = fmaxf(hi[k], v);
        }
        if (radii) rm = fmaxf(rm, radii[i]);
    }
    float v[7] = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], rm};
    for (int k = 0; k < 7; k++) {
        float x = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            float y = __shfl_xor_sync(0xffffffffu, x, o);
            x = k < 3 ? fminf(x, y) : fmaxf(x, y);
        }
        v[k] = x;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 7; k++) s[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++)
            for (int k = 0; k < 7; k++) v[k] = k < 3 ? fminf(v[k], s[k][w]) : fmaxf(v[k], s[k][w]);
        // float atomics on order-preserving ints
        for (int k = 0; k < 7; k++) {
            int* dst = (int*)&out[k];
            float x = v[k];
            int xi = __float_as_int(x);
            int key = xi >= 0 ? xi : (xi ^ 0x7fffffff);
            if (k < 3) atomicMin(dst, key);
            else atomicMax(dst, key);
        }
    }
}

PF_D float from_key(int key) { return __int_as_float(key >= 0 ? key : (key ^ 0x7fffffff)); }

__global__ void bounds_init_kernel(float* out) {
    int* o = (int*)out;
    int pinf = __float_as_int(INFINITY);
    int ninf_key = __float_as_int(-INFINITY) ^ 0x7fffffff;
    for (int k = 0; k < 3; k++) o[k] = pinf;
    for (int k = 3; k < 7; k++) o[k] = ninf_key;
    o[6] = 0;  // rmax >= 0
}

// grid from the bounds (device side, no host round trip)
__global__ void grid_kernel(const float* __restrict__ bkeys, int max_cells_log2, CechGrid* __restrict__ g) {
    const int* k = (const int*)bkeys;
    float lo[3], hi[3];
    for (int i = 0; i < 3; i++) {
        lo[i] = from_key(k[i]);
        hi[i] = from_key(k[3 + i]);
    }
    float rmax = from_key(k[6]);
    float h = fmaxf(2.0f * rmax * 1.0001f, 1e-6f);
    // bound the number of cells; a coarser grid only costs extra distance
    // tests.  Non-finite bounds (or a runaway) fall back to a single cell.
    g->nx = g->ny = g->nz = 1;
    for (int it = 0; it < 256; it++) {
        double nx = floor((double)(hi[0] - lo[0]) / h) + 1, ny = floor((double)(hi[1] - lo[1]) / h) + 1,
               nz = floor((double)(hi[2] - lo[2]) / h) + 1;
        if (!(nx * ny * nz < 1e30)) break;
        if (nx * ny * nz < (double)(1ll << max_cells_log2)) {
            g->nx = (int)nx;
            g->ny = (int)ny;
            g->nz = (int)nz;
            break;
        }
        h *= 1.25f;
    }
    if (g->nx == 1 && g->ny == 1 && g->nz == 1) h = INFINITY;
    g->lo_x = lo[0];
    g->lo_y = lo[1];
    g->lo_z = lo[2];
    g->inv_h = 1.0f / h;
}

PF_D int cell_coord(float v, float lo, float inv_h, int n) {
    float f = floorf((v - lo) * inv_h);
    int c = (f == f) ? __float2int_rz(f) : 0;
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__global__ void cell_key_kernel(const float* __restrict__ pts, int64_t N, const CechGrid* __restrict__ gp,
                                uint32_t* __restrict__ key, uint32_t* __restrict__ idx) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    CechGrid g = *gp;
    int cx = cell_coord(pts[3 * i], g.lo_x, g.inv_h, g.nx);
    int cy = cell_coord(pts[3 * i + 1], g.lo_y, g.inv_h, g.ny);
    int cz = cell_coord(pts[3 * i + 2], g.lo_z, g.inv_h, g.nz);
    key[i] = (uint32_t)((cz * g.ny + cy) * g.nx + cx);
    idx[i] = (uint32_t)i;
}

__global__ void cell_ranges_kernel(const uint32_t* __restrict__ key, int64_t N, const CechGrid* __restrict__ gp,
                                   int32_t* __restrict__ cell_start) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > N) return;
    CechGrid g = *gp;
    int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    int64_t lo = (i == 0) ? 0 : (int64_t)key[i - 1] + 1;
    int64_t hi = (i == N) ? ncell : (int64_t)key[i];
    for (int64_t c = lo; c <= hi; c++) cell_start[c] = (int32_t)i;
}

// bvh.py:7-69 predicate, with the AABB test of the BVH query
struct Ball {
    float lo[3], hi[3];
    v3 c;
    float r;
};

PF_D Ball make_ball(const float* pts, const float* radii, int64_t i) {
    Ball b;
    float r = radii[i];
    for (int k = 0; k < 3; k++) {
        float p = pts[3 * i + k];
        b.lo[k] = p - r;
        b.hi[k] = p + r;
    }
    b.c = mk(0.5f * (b.lo[0] + b.hi[0]), 0.5f * (b.lo[1] + b.hi[1]), 0.5f * (b.lo[2] + b.hi[2]));
    b.r = 0.5f * (b.hi[0] - b.lo[0]);
    return b;
}

PF_D bool overlaps(const Ball& a, const Ball& b) {
    for (int k = 0; k < 3; k++)
        if (!(a.lo[k] <= b.hi[k] && a.hi[k] >= b.lo[k])) return false;
    return length(a.c - b.c) < a.r + b.r;
}

template <bool WRITE>
__global__ void cech_kernel(const float* __restrict__ pts, const float* __restrict__ radii, int64_t N,
                            const CechGrid* __restrict__ gp, const int32_t* __restrict__ cell_start,
                            const uint32_t* __restrict__ sorted_idx, int32_t* __restrict__ counts,
                            const int64_t* __restrict__ offsets, const int64_t* __restrict__ total, int64_t capacity,
                            int32_t* __restrict__ adj) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (WRITE && *total > capacity) return;
    CechGrid g = *gp;
    Ball bi = make_ball(pts, radii, i);
    int cx = cell_coord(pts[3 * i], g.lo_x, g.inv_h, g.nx);
    int cy = cell_coord(pts[3 * i + 1], g.lo_y, g.inv_h, g.ny);
    int cz = cell_coord(pts[3 * i + 2], g.lo_z, g.inv_h, g.nz);
    int64_t pos = WRITE ? offsets[i] : 0;
    int n = 0;
    for (int dz = -1; dz <= 1; dz++) {
        int z = cz + dz;
        if (z < 0 || z >= g.nz) continue;
        for (int dy = -1; dy <= 1; dy++) {
            int y = cy + dy;
            if (y < 0 || y >= g.ny) continue;
            for (int dx = -1; dx <= 1; dx++) {
                int x = cx + dx;
                if (x < 0 || x >= g.nx) continue;
                int64_t c = ((int64_t)z * g.ny + y) * g.nx + x;
                for (int32_t s = cell_start[c]; s < cell_start[c + 1]; s++) {
                    int64_t j = sorted_idx[s];
                    if (j == i) continue;
                    Ball bj = make_ball(pts, radii, j);
                    if (overlaps(bi, bj)) {
                        if (WRITE) adj[pos + n] = (int32_t)j;
                        n++;
                    }
                }
            }
        }
    }
    if (!WRITE) {
        counts[i] = n;
    } else {
        // ascending order of each list
        int32_t* a = adj + pos;
        for (int u = 1; u < n; u++) {
            int32_t v = a[u];
            int w = u - 1;
            while (w >= 0 && a[w] > v) {
                a[w + 1] = a[w];
                w--;
            }
            a[w + 1] = v;
        }
    }
}

__global__ void offsets_i32_kernel(const int64_t* __restrict__ off64, int64_t N, const int64_t* __restrict__ total,
                                   int64_t capacity, int32_t* __restrict__ off32, int32_t* __restrict__ status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > N) return;
    int64_t t = *total;
    if (t > capacity) {
        off32[i] = 0;
        if (i == 0) atomicMax(status, PF_ERR_OVERFLOW);
        return;
    }
    off32[i] = (int32_t)(i == N ? t : off64[i]);
}

// ---------------------------------------------------------------------------
// Morton codes (geometry.py:7-47)
PF_D uint64_t expand_bits(uint64_t v) {
    v = v & 0x00000000001FFFFFull;
    v = (v | (v << 32)) & 0x001F00000000FFFFull;
    v = (v | (v << 16)) & 0x001F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void morton_kernel(const float* __restrict__ pts, int64_t N, const float* __restrict__ bkeys,
                              uint32_t* __restrict__ code_lo, uint32_t* __restrict__ code_hi,
                              uint32_t* __restrict__ idx) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int* k = (const int*)bkeys;
    float lower[3], dims[3];
    for (int a = 0; a < 3; a++) {
        lower[a] = from_key(k[a]);
        float upper = from_key(k[3 + a]);
        dims[a] = fmax_t(upper - lower[a], 1e-6f);
    }
    const float res = 2097152.0f;
    uint64_t q[3];
    for (int a = 0; a < 3; a++) {
        float nrm = (pts[3 * i + a] - lower[a]) / dims[a];
        float x = fmin_t(fmax_t(nrm * res, 0.0f), res - 1.0f);
        q[a] = expand_bits((uint64_t)x);
    }
    uint64_t code = q[0] * 4 + q[1] * 2 + q[2];
    code_lo[i] = (uint32_t)(code & 0xffffffffull);
    code_hi[i] = (uint32_t)(code >> 32);
    idx[i] = (uint32_t)i;
}

__global__ void gather_u32_kernel(const uint32_t* __restrict__ src, const uint32_t* __restrict__ perm, int64_t N,
                                  uint32_t* __restrict__ dst) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) dst[i] = src[perm[i]];
}

// ---------------------------------------------------------------------------
// Cell location: the power cell containing a point x is the primitive that
// minimises |x - p_i|^2 - r_i^2 (the cell of benchmark.py:320-324 for an
// arbitrary point).  Primitives are bucketed in a uniform grid of about four
// per cell (pts_per_cell); a query scans shells of grid cells around x's cell and stops once
// every unscanned primitive lies at least s * h away, i.e. its power distance
// is at least (s h)^2 - rmax^2 >= the best found.  Ties go to the lower index.
constexpr int kLocateMaxShell = 48;

__global__ void locate_grid_kernel(const float* __restrict__ bkeys, int64_t N, int max_cells_log2,
                                   CechGrid* __restrict__ g, float* __restrict__ rmax_out, float pts_per_cell) {
    const int* k = (const int*)bkeys;
    float lo[3], hi[3];
    for (int i = 0; i < 3; i++) {
        lo[i] = from_key(k[i]);
        hi[i] = from_key(k[3 + i]);
    }
    *rmax_out = from_key(k[6]);
    double vol = 1.0;
    for (int i = 0; i < 3; i++) vol *= fmax((double)(hi[i] - lo[i]), 1e-6);
    float h = (float)cbrt(vol * (double)pts_per_cell / (double)(N > 0 ? N : 1));
    h = fmaxf(h, 1e-6f);
    g->nx = g->ny = g->nz = 1;
    for (int it = 0; it < 256; it++) {
        double nx = floor((double)(hi[0] - lo[0]) / h) + 1, ny = floor((double)(hi[1] - lo[1]) / h) + 1,
               nz = floor((double)(hi[2] - lo[2]) / h) + 1;
        if (!(nx * ny * nz < 1e30)) break;
        if (nx * ny * nz < (double)(1ll << max_cells_log2)) {
            g->nx = (int)nx;
            g->ny = (int)ny;
            g->nz = (int)nz;
            break;
        }
        h *= 1.25f;
    }
    if (g->nx == 1 && g->ny == 1 && g->nz == 1) h = INFINITY;
    g->lo_x = lo[0];
    g->lo_y = lo[1];
    g->lo_z = lo[2];
    g->inv_h = 1.0f / h;
}

struct Locator {
    const float* pts;
    const float* radii;
    const CechGrid* grid;
    const int32_t* cell_start;
    const uint32_t* sorted;
    const float* rmax;
};

// returns the containing cell, or -1; *exact = false when the shell cap cut
// the search short
PF_D int32_t locate_point(const Locator& L, v3 x, bool* exact) {
    const CechGrid g = *L.grid;
    const float rmax = *L.rmax;
    const float h = 1.0f / g.inv_h;
    const int cx = cell_coord(x.x, g.lo_x, g.inv_h, g.nx);
    const int cy = cell_coord(x.y, g.lo_y, g.inv_h, g.ny);
    const int cz = cell_coord(x.z, g.lo_z, g.inv_h, g.nz);
    const int smax = imax(imax(g.nx, g.ny), g.nz);
    float best = INFINITY;
    int32_t best_i = -1;
    *exact = false;
    for (int s = 0; s <= kLocateMaxShell; s++) {
        for (int dz = -s; dz <= s; dz++) {
            const int z = cz + dz;
            if (z < 0 || z >= g.nz) continue;
            for (int dy = -s; dy <= s; dy++) {
                const int y = cy + dy;
                if (y < 0 || y >= g.ny) continue;
                const bool face = (dz == -s || dz == s || dy == -s || dy == s);
                const int step = (face || s == 0) ? 1 : 2 * s;
                for (int dx = -s; dx <= s; dx += step) {
                    const int xx = cx + dx;
                    if (xx < 0 || xx >= g.nx) continue;
                    const int64_t c = ((int64_t)z * g.ny + y) * g.nx + xx;
                    for (int32_t q = L.cell_start[c]; q < L.cell_start[c + 1]; q++) {
                        const int32_t j = (int32_t)L.sorted[q];
                        v3 dv = x - mk(L.pts[3 * j], L.pts[3 * j + 1], L.pts[3 * j + 2]);
                        const float rj = L.radii[j];
                        const float pd = dot(dv, dv) - rj * rj;
                        if (pd < best || (pd == best && j < best_i)) {
                            best = pd;
                            best_i = j;
                        }
                    }
                }
            }
        }
        const float reach = (float)s * h;
        if ((best_i >= 0 && reach * reach - rmax * rmax >= best) || s >= smax) {
            *exact = true;
            break;
        }
    }
    return best_i;
}

__global__ void locate_kernel(Locator L, const float* __restrict__ q, int64_t n, int32_t* __restrict__ out,
                              int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool exact;
    out[i] = locate_point(L, mk(q[3 * i], q[3 * i + 1], q[3 * i + 2]), &exact);
    if (!exact && status) atomicMax(status, PF_ERR_SEED);
}

// ---------------------------------------------------------------------------
// Point location by voxel map + walk (no counterpart in the reference, which
// only locates the camera, benchmark.py:320-324).  A res^3 grid over a box
// keeps the power cell of each voxel centre (exact, locate_point, built once
// per scene); a point then starts at its voxel's cell and walks along the
// segment from the voxel centre to the point across power faces -- the
// tracer's exit rule (raytrace.py:160-241) on exact float32 faces -- until the
// segment ends inside the current cell.
struct VoxelGrid {
    float lo[3];
    float h, inv_h;
    int res;
};

PF_D int64_t voxel_of(const VoxelGrid& g, v3 x, v3* centre) {
    const float xs[3] = {x.x, x.y, x.z};
    int c[3];
    for (int k = 0; k < 3; k++) {
        const float f = floorf((xs[k] - g.lo[k]) * g.inv_h);
        const int v = (f == f) ? __float2int_rz(fminf(fmaxf(f, -1.0f), (float)g.res)) : 0;
        c[k] = v < 0 ? 0 : (v >= g.res ? g.res - 1 : v);
    }
    *centre = mk(g.lo[0] + ((float)c[0] + 0.5f) * g.h, g.lo[1] + ((float)c[1] + 0.5f) * g.h,
                 g.lo[2] + ((float)c[2] + 0.5f) * g.h);
    return ((int64_t)c[2] * g.res + c[1]) * g.res + c[0];
}

__global__ void voxel_map_kernel(Locator L, VoxelGrid g, int32_t* __restrict__ cells, int32_t* __restrict__ status) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)g.res * g.res * g.res;
    if (v >= n) return;
    const int ix = (int)(v % g.res), iy = (int)((v / g.res) % g.res), iz = (int)(v / ((int64_t)g.res * g.res));
    const v3 c = mk(g.lo[0] + ((float)ix + 0.5f) * g.h, g.lo[1] + ((float)iy + 0.5f) * g.h,
                    g.lo[2] + ((float)iz + 0.5f) * g.h);
    bool exact;
    cells[v] = locate_point(L, c, &exact);
    if (!exact && status) atomicMax(status, PF_ERR_SEED);
}

// the cell containing x, walking from cell `c` (which contains p0) along
// p0 -> x; *ok = false when max_steps faces were crossed without reaching x
PF_D int32_t walk_to_point(const float* __restrict__ pts, const float* __restrict__ radii,
                           const int32_t* __restrict__ adj, const int32_t* __restrict__ adj_off, int64_t N,
                           int32_t c, v3 p0, v3 x, int max_steps, bool* ok) {
    const v3 u = x - p0;
    for (int step = 0; step <= max_steps; step++) {
        if (c < 0 || c >= N) break;
        const v3 ci = mk(__ldg(pts + 3 * c), __ldg(pts + 3 * c + 1), __ldg(pts + 3 * c + 2));
        const float ri = __ldg(radii + c);
        const float pi = dot(ci, ci) - ri * ri;
        float s_exit = 1.0f;  // the segment ends at x
        int32_t next = -1;
        const int32_t e1 = __ldg(adj_off + c + 1);
        for (int32_t e = __ldg(adj_off + c); e < e1; e++) {
            const int32_t j = __ldg(adj + e);
            const v3 cj = mk(__ldg(pts + 3 * j), __ldg(pts + 3 * j + 1), __ldg(pts + 3 * j + 2));
            const float rj = __ldg(radii + j);
            // power face between c and j: 2 x.(cj - ci) = (|cj|^2 - rj^2) - (|ci|^2 - ri^2)
            const v3 nrm = cj - ci;
            const float nu = dot(nrm, u);
            if (!(nu > 0.0f)) continue;
            const float s = (0.5f * ((dot(cj, cj) - rj * rj) - pi) - dot(nrm, p0)) / nu;
            if (s < s_exit) {
                s_exit = s;
                next = j;
            }
        }
        if (next < 0) {
            *ok = true;
            return c;
        }
        c = next;
    }
    *ok = false;
    return c;
}

// start cell of every pixel ray from the voxel map: the cell containing
// eye + t d where the proposal is confident (conf >= conf_thr, t > 0), else
// the default start (also when the walk needs more than max_steps faces)
__global__ void seed_vmap_kernel(const float* __restrict__ pts, const float* __restrict__ radii,
                                 const int32_t* __restrict__ adj, const int32_t* __restrict__ adj_off, int64_t N,
                                 const int32_t* __restrict__ vcells, VoxelGrid g, Cam cam,
                                 const float* __restrict__ t_entry, const float* __restrict__ conf, float conf_thr,
                                 int32_t default_start, int max_steps, int32_t* __restrict__ start_cells,
                                 int32_t* __restrict__ n_seeded) {
    const int64_t px = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)cam.W * cam.H;
    bool seeded = false;
    if (px < n) {
        int32_t cell = default_start;
        const float t = t_entry[px];
        if (conf[px] >= conf_thr && t > 0.0f) {
            const int pi = (int)(px / cam.W), pj = (int)(px % cam.W);
            const v3 x = cam.eye + t * ray_dir(cam, pi, pj);
            v3 p0;
            const int64_t v = voxel_of(g, x, &p0);
            bool ok;
            const int32_t c = walk_to_point(pts, radii, adj, adj_off, N, vcells[v], p0, x, max_steps, &ok);
            if (ok) {
                cell = c;
                seeded = true;
            }
        }
        start_cells[px] = cell;
    }
    const unsigned b = __ballot_sync(0xffffffffu, seeded);
    if ((threadIdx.x & 31) == 0 && b && n_seeded) atomicAdd(n_seeded, __popc(b));
}

// points located through the voxel map (as seed_vmap_kernel), -1 where the walk gave up
__global__ void locate_vmap_kernel(const float* __restrict__ pts, const float* __restrict__ radii,
                                   const int32_t* __restrict__ adj, const int32_t* __restrict__ adj_off, int64_t N,
                                   const int32_t* __restrict__ vcells, VoxelGrid g, const float* __restrict__ q,
                                   int64_t nq, int max_steps, int32_t* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const v3 x = mk(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    v3 p0;
    const int64_t v = voxel_of(g, x, &p0);
    bool ok;
    const int32_t c = walk_to_point(pts, radii, adj, adj_off, N, vcells[v], p0, x, max_steps, &ok);
    out[i] = ok ? c : -1;
}

// start cell of every pixel ray: the cell containing eye + t d where the
// proposal is confident (conf >= conf_thr, t > 0), else the default start
__global__ void seed_kernel(Locator L, Cam cam, const float* __restrict__ t_entry, const float* __restrict__ conf,
                            float conf_thr, int32_t default_start, int32_t* __restrict__ start_cells,
                            int32_t* __restrict__ n_seeded) {
    const int64_t px = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)cam.W * cam.H;
    bool seeded = false;
    if (px < n) {
        int32_t cell = default_start;
        const float t = t_entry[px];
        if (conf[px] >= conf_thr && t > 0.0f) {
            const int pi = (int)(px / cam.W), pj = (int)(px % cam.W);
            const v3 d = ray_dir(cam, pi, pj);
            bool exact;
            const int32_t c = locate_point(L, cam.eye + t * d, &exact);
            if (c >= 0 && exact) {
                cell = c;
                seeded = true;
            }
        }
        start_cells[px] = cell;
    }
    const unsigned b = __ballot_sync(0xffffffffu, seeded);
    if ((threadIdx.x & 31) == 0 && b && n_seeded) atomicAdd(n_seeded, __popc(b));
}

// ---------------------------------------------------------------------------
// Power-diagram adjacency (replaces build_power_adjacency, benchmark.py:25-83):
// every site clips its own power cell (pf_power.cuh) into a fixed slab of
// neighbours; edges seen from one side only are added to the other side (the
// hull's edges are undirected), the optional alpha_complex filter keeps the
// pairs whose balls overlap, and the lists are counted, scanned and written
// as CSR, ascending per site.

// per grid cell, the largest squared radius of its sites (non-negative
// floats order as their bit patterns)
__global__ void cell_weight_kernel(const float* __restrict__ pts, const float* __restrict__ radii, int64_t N,
                                   const CechGrid* __restrict__ gp, float* __restrict__ cell_w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const CechGrid g = *gp;
    const int cx = cell_coord(pts[3 * i], g.lo_x, g.inv_h, g.nx);
    const int cy = cell_coord(pts[3 * i + 1], g.lo_y, g.inv_h, g.ny);
    const int cz = cell_coord(pts[3 * i + 2], g.lo_z, g.inv_h, g.nz);
    const float w = radii[i] * radii[i];
    atomicMax((int*)cell_w + ((int64_t)cz * g.ny + cy) * g.nx + cx, __float_as_int(w));
}

// per block of kPcSuper^3 grid cells, the largest cell weight (-1 bits: no site)
__global__ void super_weight_kernel(const CechGrid* __restrict__ gp, const int32_t* __restrict__ cell_start,
                                    const float* __restrict__ cell_w, int* __restrict__ super_w) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const CechGrid g = *gp;
    if (c >= (int64_t)g.nx * g.ny * g.nz || cell_start[c] == cell_start[c + 1]) return;
    const int x = (int)(c % g.nx), y = (int)((c / g.nx) % g.ny), z = (int)(c / ((int64_t)g.nx * g.ny));
    const int snx = (g.nx + kPcSuper - 1) / kPcSuper, sny = (g.ny + kPcSuper - 1) / kPcSuper;
    atomicMax(super_w + ((int64_t)(z / kPcSuper) * sny + y / kPcSuper) * snx + x / kPcSuper,
              __float_as_int(cell_w[c]));
}

__global__ void __launch_bounds__(64) power_cell_kernel(PowerScene S, int64_t N, int32_t* __restrict__ slab,
                                                        int32_t* __restrict__ counts, int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    PowerCell C;
    bool full = false;
    counts[i] = power_site(S, i, C, slab + i * kPowerSlab, &full);
    if (full && status) atomicMax(status, PF_ERR_CELL);
}

PF_D bool slab_has(const int32_t* a, int n, int32_t v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && a[lo] == v;
}

// an edge i -> j that j's list lacks goes to j's extra slots
__global__ void power_symmetrize_kernel(const int32_t* __restrict__ slab, const int32_t* __restrict__ counts, int64_t N,
                                        int32_t* __restrict__ extra, int32_t* __restrict__ extra_n,
                                        int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int32_t* a = slab + i * kPowerSlab;
    for (int k = 0; k < counts[i]; k++) {
        const int32_t j = a[k];
        if (slab_has(slab + (int64_t)j * kPowerSlab, counts[j], (int32_t)i)) continue;
        const int slot = atomicAdd(extra_n + j, 1);
        if (slot < kPowerExtra) extra[(int64_t)j * kPowerExtra + slot] = (int32_t)i;
        else if (status) atomicMax(status, PF_ERR_CELL);
    }
}

// alpha_complex filter (benchmark.py:62-68): |p_i - p_j| < r_i + r_j
PF_D bool power_keep(const float* pts, const float* radii, int64_t i, int64_t j, bool alpha) {
    if (!alpha) return true;
    double d2 = 0.0;
    for (int k = 0; k < 3; k++) {
        const double e = (double)pts[3 * i + k] - (double)pts[3 * j + k];
        d2 += e * e;
    }
    return sqrt(d2) < (double)radii[i] + (double)radii[j];
}

// WRITE = false: the length of each final list; true: the lists
template <bool WRITE>
__global__ void power_emit_kernel(const float* __restrict__ pts, const float* __restrict__ radii,
                                  const int32_t* __restrict__ slab, const int32_t* __restrict__ counts,
                                  const int32_t* __restrict__ extra, const int32_t* __restrict__ extra_n, int64_t N,
                                  int alpha, int32_t* __restrict__ out_counts, const int64_t* __restrict__ offsets,
                                  const int64_t* __restrict__ total, int64_t capacity, int32_t* __restrict__ adj) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (WRITE && *total > capacity) return;
    const int32_t* a = slab + i * kPowerSlab;
    const int na = counts[i];
    const int nx = min(extra_n[i], kPowerExtra);
    int32_t ex[kPowerExtra];
    for (int k = 0; k < nx; k++) ex[k] = extra[i * kPowerExtra + k];
    for (int u = 1; u < nx; u++) {
        const int32_t v = ex[u];
        int w = u - 1;
        while (w >= 0 && ex[w] > v) {
            ex[w + 1] = ex[w];
            w--;
        }
        ex[w + 1] = v;
    }
    const int64_t pos = WRITE ? offsets[i] : 0;
    int n = 0, ia = 0, ix = 0;
    while (ia < na || ix < nx) {
        int32_t v;
        if (ix >= nx || (ia < na && a[ia] < ex[ix])) v = a[ia++];
        else v = ex[ix++];
        if (!power_keep(pts, radii, i, v, alpha != 0)) continue;
        if (WRITE) adj[pos + n] = v;
        n++;
    }
    if (!WRITE) out_counts[i] = n;
}

// ---------------------------------------------------------------------------
// Steiner points (benchmark.py:93-180).  Each round of get_steiner_points
// draws random samples, finds for each its 32 nearest primitive centres
// (scipy's cKDTree in the reference), takes the smallest dist - r over them
// as the sample's radius and the primitive that attains it, keeps samples
// whose radius is 2..6 times that primitive's, and thins them with a greedy
// minimum-overlap selection.  The nearest-neighbour query and the selection
// run here; distances are float64 rounded to float32, as the tree's are.

constexpr int kSteinerK = 32;

// k nearest centres of q (ascending distance), exact: grid shells until the
// shells scanned cover the k-th distance
__global__ void steiner_knn_kernel(Locator L, const float* __restrict__ queries, int64_t nq, int k,
                                   float* __restrict__ radius_out, int32_t* __restrict__ closest_out,
                                   int32_t* __restrict__ status) {
    const int64_t qi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    const CechGrid g = *L.grid;
    const double q[3] = {(double)queries[3 * qi], (double)queries[3 * qi + 1], (double)queries[3 * qi + 2]};
    const double h = 1.0 / (double)g.inv_h;
    const double glo[3] = {(double)g.lo_x, (double)g.lo_y, (double)g.lo_z};
    const int gn[3] = {g.nx, g.ny, g.nz};
    const int cc[3] = {cell_coord(queries[3 * qi], g.lo_x, g.inv_h, g.nx),
                       cell_coord(queries[3 * qi + 1], g.lo_y, g.inv_h, g.ny),
                       cell_coord(queries[3 * qi + 2], g.lo_z, g.inv_h, g.nz)};
    double bd[kSteinerK];
    int32_t bi[kSteinerK];
    int nb = 0;
    const int smax = imax(imax(g.nx, g.ny), g.nz);
    for (int s = 0; s <= smax; s++) {
        for (int dz = -s; dz <= s; dz++) {
            const int z = cc[2] + dz;
            if (z < 0 || z >= g.nz) continue;
            for (int dy = -s; dy <= s; dy++) {
                const int y = cc[1] + dy;
                if (y < 0 || y >= g.ny) continue;
                const bool face = (dz == -s || dz == s || dy == -s || dy == s);
                const int step = (face || s == 0) ? 1 : 2 * s;
                for (int dx = -s; dx <= s; dx += step) {
                    const int x = cc[0] + dx;
                    if (x < 0 || x >= g.nx) continue;
                    const int64_t c = ((int64_t)z * g.ny + y) * g.nx + x;
                    for (int32_t p = L.cell_start[c]; p < L.cell_start[c + 1]; p++) {
                        const int32_t j = (int32_t)L.sorted[p];
                        const double d0 = (double)L.pts[3 * j] - q[0], d1 = (double)L.pts[3 * j + 1] - q[1],
                                     d2 = (double)L.pts[3 * j + 2] - q[2];
                        const double d = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                        if (nb == k && !(d < bd[k - 1] || (d == bd[k - 1] && j < bi[k - 1]))) continue;
                        int w = nb < k ? nb++ : k - 1;
                        while (w > 0 && (bd[w - 1] > d || (bd[w - 1] == d && bi[w - 1] > j))) {
                            bd[w] = bd[w - 1];
                            bi[w] = bi[w - 1];
                            w--;
                        }
                        bd[w] = d;
                        bi[w] = j;
                    }
                }
            }
        }
        if (nb == k) {
            double reach = INFINITY;
            for (int a = 0; a < 3; a++) {
                if (cc[a] - s > 0) reach = fmin(reach, q[a] - (glo[a] + (cc[a] - s) * h));
                if (cc[a] + s < gn[a] - 1) reach = fmin(reach, glo[a] + (cc[a] + s + 1) * h - q[a]);
            }
            if (reach > bd[k - 1]) break;
        }
    }
    if (nb < k) {  // fewer primitives than neighbours asked for
        if (status) atomicMax(status, PF_ERR_ARGS);
        radius_out[qi] = NAN;
        closest_out[qi] = -1;
        return;
    }
    // (dists - all_radii[idxs]).min(dim=1), float32 as the reference
    float best = (float)bd[0] - L.radii[bi[0]];
    int32_t arg = bi[0];
    for (int a = 1; a < k; a++) {
        const float v = (float)bd[a] - L.radii[bi[a]];
        if (v < best) {
            best = v;
            arg = bi[a];
        }
    }
    radius_out[qi] = best;
    closest_out[qi] = arg;
}

constexpr int kSelectThreads = 1024;

PF_D float steiner_overlap(const float* p, const float* r, int64_t i, int64_t j) {
    const float sum_r = r[i] + r[j];
    const float dx = p[3 * i] - p[3 * j], dy = p[3 * i + 1] - p[3 * j + 1], dz = p[3 * i + 2] - p[3 * j + 2];
    const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
    return (sum_r - dist) / sum_r;
}

// _greedy_min_overlap_fps (benchmark.py:93-134) in one block: starting from
// `seed`, repeatedly select the sample whose largest overlap with the
// selected ones is smallest (first index on ties) while it is <= threshold.
// max_overlap is n floats of scratch.  At most n rounds.
__global__ void __launch_bounds__(kSelectThreads)
    steiner_select_kernel(const float* __restrict__ pts, const float* __restrict__ radii, int64_t n, int64_t seed,
                          float threshold, float* __restrict__ max_overlap, uint8_t* __restrict__ selected,
                          int32_t* __restrict__ n_selected) {
    __shared__ float sv[kSelectThreads / 32];
    __shared__ int64_t si[kSelectThreads / 32];
    __shared__ int64_t pick;
    __shared__ float pick_v;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int64_t i = t; i < n; i += blockDim.x) {
        selected[i] = 0;
        max_overlap[i] = steiner_overlap(pts, radii, i, seed);
    }
    __syncthreads();
    if (t == 0) {
        selected[seed] = 1;
        max_overlap[seed] = INFINITY;
    }
    int32_t count = 1;
    __syncthreads();
    for (int64_t round = 0; round < n; round++) {
        // block argmin, first index on ties; NaN compares as the reference's
        // torch.min: it wins (min propagates NaN)
        float bv = INFINITY;
        int64_t bidx = -1;
        for (int64_t i = t; i < n; i += blockDim.x) {
            const float v = max_overlap[i];
            if (bidx < 0 || v < bv || (v != v && bv == bv)) {
                bv = v;
                bidx = i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int64_t oi = __shfl_down_sync(0xffffffffu, bidx, o);
            const bool take = oi >= 0 && (bidx < 0 || (ov != ov && (bv == bv || oi < bidx)) ||
                                          (!(bv != bv) && (ov < bv || (ov == bv && oi < bidx))));
            if (take) {
                bv = ov;
                bidx = oi;
            }
        }
        if (lane == 0) {
            sv[w] = bv;
            si[w] = bidx;
        }
        __syncthreads();
        if (t == 0) {
            float v = sv[0];
            int64_t ix = si[0];
            for (int k = 1; k < (int)(blockDim.x / 32); k++) {
                const float ov = sv[k];
                const int64_t oi = si[k];
                const bool take = oi >= 0 && (ix < 0 || (ov != ov && (v == v || oi < ix)) ||
                                              (!(v != v) && (ov < v || (ov == v && oi < ix))));
                if (take) {
                    v = ov;
                    ix = oi;
                }
            }
            pick = ix;
            pick_v = v;
        }
        __syncthreads();
        const int64_t j = pick;
        if (j < 0 || pick_v > threshold) break;
        if (t == 0) {
            selected[j] = 1;
            max_overlap[j] = INFINITY;
        }
        count++;
        __syncthreads();
        for (int64_t i = t; i < n; i += blockDim.x) {
            const float nv = steiner_overlap(pts, radii, i, j);
            const float cur = max_overlap[i];
            max_overlap[i] = (cur != cur || nv != nv) ? NAN : fmaxf(cur, nv);  // torch.maximum propagates NaN
        }
        __syncthreads();
    }
    if (t == 0 && n_selected) *n_selected = count;
}

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct CechLayout {
    size_t bounds, grid, key0, idx0, key1, idx1, cell_start, counts, off64, spart, rhist, rpart, bytes;
};

constexpr int kMaxCellsLog2 = 22;

static CechLayout cech_layout(int64_t N) {
    CechLayout L;
    size_t o = 0;
    auto take = [&](size_t b) {
        size_t r = o;
        o = align_up(o + b);
        return r;
    };
    L.bounds = take(64);
    L.grid = take(sizeof(CechGrid));
    L.key0 = take(4 * (size_t)N);
    L.idx0 = take(4 * (size_t)N);
    L.key1 = take(4 * (size_t)N);
    L.idx1 = take(4 * (size_t)N);
    L.cell_start = take(4 * (((size_t)1 << kMaxCellsLog2) + 1));
    L.counts = take(4 * (size_t)N);
    L.off64 = take(8 * (size_t)(N + 1));
    L.spart = take(8 * (size_t)(scan_blocks(N) + 2));
    int64_t rb = radix_blocks(N);
    L.rhist = take(4 * (size_t)(256 * rb));
    L.rpart = take(4 * (size_t)(scan_blocks(256 * rb) + 1));
    L.bytes = o;
    return L;
}

}  // namespace pf

using namespace pf;

extern "C" int pf_cech_workspace_size(int64_t n_prims, size_t* bytes) {
    if (!bytes || n_prims < 0) return pf_fail(PF_ERR_ARGS, "pf_cech_workspace_size: bad arguments");
    *bytes = cech_layout(n_prims).bytes;
    return PF_OK;
}

extern "C" int pf_cech_adjacency(const float* points, const float* radii, int64_t n_prims, void* workspace,
                                 size_t workspace_bytes, int64_t edge_capacity, int32_t* adjacency,
                                 int32_t* adjacency_offsets, int64_t* n_edges, int32_t* status, void* stream) {
    if (n_prims <= 0 || !points || !radii || !adjacency_offsets || !n_edges || !status || edge_capacity < 0 ||
        edge_capacity >= ((int64_t)1 << 31) || (edge_capacity > 0 && !adjacency))
        return pf_fail(PF_ERR_ARGS, "pf_cech_adjacency: bad arguments");
    CechLayout L = cech_layout(n_prims);
    if (!workspace || workspace_bytes < L.bytes) return pf_fail(PF_ERR_ARGS, "pf_cech_adjacency: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    char* ws = (char*)workspace;
    float* bounds = (float*)(ws + L.bounds);
    CechGrid* grid = (CechGrid*)(ws + L.grid);
    uint32_t *key0 = (uint32_t*)(ws + L.key0), *idx0 = (uint32_t*)(ws + L.idx0);
    uint32_t *key1 = (uint32_t*)(ws + L.key1), *idx1 = (uint32_t*)(ws + L.idx1);
    int32_t* cell_start = (int32_t*)(ws + L.cell_start);
    int32_t* counts = (int32_t*)(ws + L.counts);
    int64_t* off64 = (int64_t*)(ws + L.off64);
    int64_t* spart = (int64_t*)(ws + L.spart);
    RadixScratch rs{(uint32_t*)(ws + L.rhist), (uint32_t*)(ws + L.rpart)};
    const int64_t N = n_prims;
    const unsigned gN = (unsigned)((N + 255) / 256);
    bounds_init_kernel<<<1, 1, 0, st>>>(bounds);
    bounds_kernel<<<(unsigned)std::min<int64_t>(gN, 148 * 8), 256, 0, st>>>(points, radii, N, bounds);
    grid_kernel<<<1, 1, 0, st>>>(bounds, kMaxCellsLog2, grid);
    cell_key_kernel<<<gN, 256, 0, st>>>(points, N, grid, key0, idx0);
    uint32_t* kf = radix_final_key_buffer(key0, key1, kMaxCellsLog2);
    uint32_t* vf = kf == key0 ? idx0 : idx1;
    radix_sort_pairs(key0, idx0, key1, idx1, kf, vf, N, nullptr, kMaxCellsLog2, rs, st);
    cell_ranges_kernel<<<(unsigned)((N + 1 + 255) / 256), 256, 0, st>>>(kf, N, grid, cell_start);
    cech_kernel<false><<<gN, 256, 0, st>>>(points, radii, N, grid, cell_start, vf, counts, nullptr, nullptr, 0,
                                           nullptr);
    exclusive_scan<int32_t, int64_t>(counts, off64, N, spart, n_edges, st);
    cech_kernel<true><<<gN, 256, 0, st>>>(points, radii, N, grid, cell_start, vf, nullptr, off64, n_edges,
                                          edge_capacity, adjacency);
    offsets_i32_kernel<<<(unsigned)((N + 1 + 255) / 256), 256, 0, st>>>(off64, N, n_edges, edge_capacity,
                                                                        adjacency_offsets, status);
    return pf_check_launch("pf_cech_adjacency");
}

// The locator keeps, in its workspace, the grid, the primitive ids sorted by
// grid cell and the per-cell ranges (the Čech layout without the edge lists).
static Locator locator_view(const float* points, const float* radii, int64_t N, char* ws) {
    CechLayout L = cech_layout(N);
    uint32_t* key0 = (uint32_t*)(ws + L.key0);
    uint32_t* key1 = (uint32_t*)(ws + L.key1);
    uint32_t* kf = radix_final_key_buffer(key0, key1, kMaxCellsLog2);
    Locator loc;
    loc.pts = points;
    loc.radii = radii;
    loc.grid = (const CechGrid*)(ws + L.grid);
    loc.cell_start = (const int32_t*)(ws + L.cell_start);
    loc.sorted = kf == key0 ? (const uint32_t*)(ws + L.idx0) : (const uint32_t*)(ws + L.idx1);
    loc.rmax = (const float*)(ws + L.bounds + 32);
    return loc;
}

extern "C" int pf_locator_workspace_size(int64_t n_prims, size_t* bytes) {
    return pf_cech_workspace_size(n_prims, bytes);
}

// grid over the bounds with about pts_per_cell primitives per cell, the ids
// sorted by cell and the per-cell ranges (the locator's and the power
// build's)
static void build_point_grid(const float* points, const float* radii, int64_t N, char* ws, float pts_per_cell,
                             cudaStream_t st) {
    const CechLayout L = cech_layout(N);
    float* bounds = (float*)(ws + L.bounds);
    CechGrid* grid = (CechGrid*)(ws + L.grid);
    uint32_t *key0 = (uint32_t*)(ws + L.key0), *idx0 = (uint32_t*)(ws + L.idx0);
    uint32_t *key1 = (uint32_t*)(ws + L.key1), *idx1 = (uint32_t*)(ws + L.idx1);
    int32_t* cell_start = (int32_t*)(ws + L.cell_start);
    RadixScratch rs{(uint32_t*)(ws + L.rhist), (uint32_t*)(ws + L.rpart)};
    const unsigned gN = (unsigned)((N + 255) / 256);
    bounds_init_kernel<<<1, 1, 0, st>>>(bounds);
    bounds_kernel<<<(unsigned)std::min<int64_t>(gN, 148 * 8), 256, 0, st>>>(points, radii, N, bounds);
    locate_grid_kernel<<<1, 1, 0, st>>>(bounds, N, kMaxCellsLog2, grid, bounds + 8, pts_per_cell);
    cell_key_kernel<<<gN, 256, 0, st>>>(points, N, grid, key0, idx0);
    uint32_t* kf = radix_final_key_buffer(key0, key1, kMaxCellsLog2);
    uint32_t* vf = kf == key0 ? idx0 : idx1;
    radix_sort_pairs(key0, idx0, key1, idx1, kf, vf, N, nullptr, kMaxCellsLog2, rs, st);
    cell_ranges_kernel<<<(unsigned)((N + 1 + 255) / 256), 256, 0, st>>>(kf, N, grid, cell_start);
}

extern "C" int pf_locator_build(const float* points, const float* radii, int64_t n_prims, void* workspace,
                                size_t workspace_bytes, void* stream) {
    if (n_prims <= 0 || n_prims >= ((int64_t)1 << 31) || !points || !radii)
        return pf_fail(PF_ERR_ARGS, "pf_locator_build: bad arguments");
    CechLayout L = cech_layout(n_prims);
    if (!workspace || workspace_bytes < L.bytes) return pf_fail(PF_ERR_ARGS, "pf_locator_build: workspace too small");
    build_point_grid(points, radii, n_prims, (char*)workspace, 4.0f, (cudaStream_t)stream);
    return pf_check_launch("pf_locator_build");
}

extern "C" int pf_locate_cells(const float* points, const float* radii, int64_t n_prims, const void* workspace,
                               const float* queries, int64_t n_queries, int32_t* cells, int32_t* status,
                               void* stream) {
    if (n_prims <= 0 || !points || !radii || !workspace || n_queries < 0 || (n_queries > 0 && (!queries || !cells)))
        return pf_fail(PF_ERR_ARGS, "pf_locate_cells: bad arguments");
    if (n_queries == 0) return PF_OK;
    Locator loc = locator_view(points, radii, n_prims, (char*)workspace);
    locate_kernel<<<(unsigned)((n_queries + 127) / 128), 128, 0, (cudaStream_t)stream>>>(loc, queries, n_queries,
                                                                                        cells, status);
    return pf_check_launch("pf_locate_cells");
}

extern "C" int pf_seed_start_cells(const float* points, const float* radii, int64_t n_prims, const void* workspace,
                                   const pf_camera* cam, const float* t_entry, const float* confidence,
                                   float conf_threshold, int32_t default_start, int32_t* start_cells,
                                   int32_t* n_seeded, void* stream) {
    if (n_prims <= 0 || !points || !radii || !workspace || !cam || !t_entry || !confidence || !start_cells ||
        cam->width < 2 || cam->height < 2 || default_start < 0 || default_start >= n_prims)
        return pf_fail(PF_ERR_ARGS, "pf_seed_start_cells: bad arguments");
    Locator loc = locator_view(points, radii, n_prims, (char*)workspace);
    const int64_t n = (int64_t)cam->width * cam->height;
    seed_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        loc, load_cam(*cam), t_entry, confidence, conf_threshold, default_start, start_cells, n_seeded);
    return pf_check_launch("pf_seed_start_cells");
}

// ---------------------------------------------------------------------------
// Occupancy seeding (no counterpart in the reference).  One bit per voxel of
// a res^3 grid over the primitives' box, set wherever the bounding box of a
// primitive whose density is not below sigma_min, grown by one voxel, reaches.
// The walk composites only inside spheres with density >= 1e-3
// (raytrace.py:201-206: a cell adds nothing unless its sphere is hit and
// sigma >= 1e-3), so a ray meets no compositing before the first set voxel on
// its path, and a walk seeded there composites what the plain walk does.
__global__ void occupancy_kernel(const float* __restrict__ pts, const float* __restrict__ radii,
                                 const float* __restrict__ density, int64_t N, VoxelGrid g, float sigma_min,
                                 uint32_t* __restrict__ bits, int32_t* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (density[i] < sigma_min) return;  // a NaN density counts as occupied, as the walk treats it
    const float c[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    const float r = radii[i];
    if (!isfinite(c[0]) || !isfinite(c[1]) || !isfinite(c[2]) || !isfinite(r)) {
        atomicMax(status, PF_ERR_NONFINITE);
        return;
    }
    int a[3], b[3];
    for (int k = 0; k < 3; k++) {
        const float fa = floorf((c[k] - r - g.lo[k]) * g.inv_h) - 1.0f;
        const float fb = floorf((c[k] + r - g.lo[k]) * g.inv_h) + 1.0f;
        a[k] = (int)fminf(fmaxf(fa, 0.0f), (float)(g.res - 1));
        b[k] = (int)fminf(fmaxf(fb, 0.0f), (float)(g.res - 1));
    }
    for (int z = a[2]; z <= b[2]; z++)
        for (int y = a[1]; y <= b[1]; y++)
            for (int x = a[0]; x <= b[0]; x++) {
                const int64_t v = ((int64_t)z * g.res + y) * g.res + x;
                atomicOr(&bits[v >> 5], 1u << (v & 31));
            }
}

// Per pixel ray: the distance at which it enters the first set voxel (a 3-D
// DDA from where it enters the grid's box), minus `margin`; rays that meet no
// set voxel get the box exit minus `margin`.  confidence = 1 where that skips
// part of the ray (t > 0 inside the box), else 0 (rays that miss the box, or
// start in a set voxel).
__global__ void occupancy_entry_kernel(const uint32_t* __restrict__ bits, VoxelGrid g, Cam cam, float margin,
                                       float* __restrict__ t_out, float* __restrict__ conf_out) {
    const int64_t px = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)cam.W * cam.H;
    if (px >= n) return;
    const int pi = (int)(px / cam.W), pj = (int)(px % cam.W);
    const v3 dv = ray_dir(cam, pi, pj);
    const float o[3] = {cam.eye.x, cam.eye.y, cam.eye.z}, d[3] = {dv.x, dv.y, dv.z};
    const float span = g.h * (float)g.res;
    float t0 = 0.0f, t1 = 3.0e38f;
    bool inside = true;
    for (int k = 0; k < 3; k++) {
        const float lo = g.lo[k], hi = g.lo[k] + span;
        if (d[k] == 0.0f) {
            if (o[k] < lo || o[k] > hi) inside = false;
        } else {
            float ta = (lo - o[k]) / d[k], tb = (hi - o[k]) / d[k];
            if (ta > tb) {
                const float tt = ta;
                ta = tb;
                tb = tt;
            }
            t0 = fmaxf(t0, ta);
            t1 = fminf(t1, tb);
        }
    }
    if (!inside || !(t1 > t0)) {
        t_out[px] = -1.0f;
        conf_out[px] = 0.0f;
        return;
    }
    int ix[3], step[3];
    float tmax[3], tdelta[3];
    for (int k = 0; k < 3; k++) {
        const float p = o[k] + t0 * d[k];
        const float f = floorf((p - g.lo[k]) * g.inv_h);
        ix[k] = (int)fminf(fmaxf(f, 0.0f), (float)(g.res - 1));
        if (d[k] > 0.0f) {
            step[k] = 1;
            tmax[k] = (g.lo[k] + (float)(ix[k] + 1) * g.h - o[k]) / d[k];
            tdelta[k] = g.h / d[k];
        } else if (d[k] < 0.0f) {
            step[k] = -1;
            tmax[k] = (g.lo[k] + (float)ix[k] * g.h - o[k]) / d[k];
            tdelta[k] = -g.h / d[k];
        } else {
            step[k] = 0;
            tmax[k] = 3.0e38f;
            tdelta[k] = 3.0e38f;
        }
    }
    float t = t0;
    bool hit = false;
    for (int it = 0; it < 3 * g.res + 3; it++) {  // a ray crosses at most 3 res voxels of the grid
        const int64_t v = ((int64_t)ix[2] * g.res + ix[1]) * g.res + ix[0];
        if ((__ldg(&bits[v >> 5]) >> (v & 31)) & 1u) {
            hit = true;
            break;
        }
        const int k = (tmax[0] < tmax[1]) ? (tmax[0] < tmax[2] ? 0 : 2) : (tmax[1] < tmax[2] ? 1 : 2);
        t = tmax[k];
        ix[k] += step[k];
        if (ix[k] < 0 || ix[k] >= g.res || t >= t1) break;
        tmax[k] += tdelta[k];
    }
    const float ts = (hit ? t : t1) - margin;
    t_out[px] = ts;
    conf_out[px] = ts > t0 ? 1.0f : 0.0f;
}

static bool voxel_grid(const float* lo, const float* hi, int32_t res, VoxelGrid* g) {
    if (!lo || !hi || res < 1 || res > 1024) return false;
    float ext = 0.f;
    for (int k = 0; k < 3; k++) {
        if (!(hi[k] >= lo[k])) return false;
        ext = fmaxf(ext, hi[k] - lo[k]);
    }
    ext = fmaxf(ext, 1e-6f);
    for (int k = 0; k < 3; k++) g->lo[k] = lo[k];
    g->h = ext / (float)res;
    g->inv_h = 1.0f / g->h;
    g->res = res;
    return true;
}

extern "C" int pf_voxel_map_build(const float* points, const float* radii, int64_t n_prims, const void* workspace,
                                  const float* box_lo, const float* box_hi, int32_t res, int32_t* cells,
                                  int32_t* status, void* stream) {
    VoxelGrid g;
    if (n_prims <= 0 || !points || !radii || !workspace || !cells || !voxel_grid(box_lo, box_hi, res, &g))
        return pf_fail(PF_ERR_ARGS, "pf_voxel_map_build: bad arguments");
    Locator loc = locator_view(points, radii, n_prims, (char*)workspace);
    const int64_t n = (int64_t)res * res * res;
    voxel_map_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(loc, g, cells, status);
    return pf_check_launch("pf_voxel_map_build");
}

extern "C" int pf_seed_start_cells_vmap(const float* points, const float* radii, int64_t n_prims,
                                        const int32_t* adjacency, const int32_t* adjacency_offsets,
                                        const int32_t* cells, const float* box_lo, const float* box_hi, int32_t res,
                                        const pf_camera* cam, const float* t_entry, const float* confidence,
                                        float conf_threshold, int32_t default_start, int32_t max_walk_steps,
                                        int32_t* start_cells, int32_t* n_seeded, void* stream) {
    VoxelGrid g;
    if (n_prims <= 0 || !points || !radii || !adjacency_offsets || !cells || !cam || !t_entry || !confidence ||
        !start_cells || cam->width < 2 || cam->height < 2 || default_start < 0 || default_start >= n_prims ||
        max_walk_steps < 0 || !voxel_grid(box_lo, box_hi, res, &g))
        return pf_fail(PF_ERR_ARGS, "pf_seed_start_cells_vmap: bad arguments");
    const int64_t n = (int64_t)cam->width * cam->height;
    seed_vmap_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        points, radii, adjacency, adjacency_offsets, n_prims, cells, g, load_cam(*cam), t_entry, confidence,
        conf_threshold, default_start, max_walk_steps, start_cells, n_seeded);
    return pf_check_launch("pf_seed_start_cells_vmap");
}

extern "C" int pf_locate_cells_vmap(const float* points, const float* radii, int64_t n_prims,
                                    const int32_t* adjacency, const int32_t* adjacency_offsets, const int32_t* cells,
                                    const float* box_lo, const float* box_hi, int32_t res, const float* queries,
                                    int64_t n_queries, int32_t max_walk_steps, int32_t* out, void* stream) {
    VoxelGrid g;
    if (n_prims <= 0 || !points || !radii || !adjacency_offsets || !cells || n_queries < 0 ||
        (n_queries > 0 && (!queries || !out)) || max_walk_steps < 0 || !voxel_grid(box_lo, box_hi, res, &g))
        return pf_fail(PF_ERR_ARGS, "pf_locate_cells_vmap: bad arguments");
    if (n_queries == 0) return PF_OK;
    locate_vmap_kernel<<<(unsigned)((n_queries + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        points, radii, adjacency, adjacency_offsets, n_prims, cells, g, queries, n_queries, max_walk_steps, out);
    return pf_check_launch("pf_locate_cells_vmap");
}

extern "C" int pf_morton_workspace_size(int64_t n_prims, size_t* bytes) {
    if (!bytes || n_prims < 0) return pf_fail(PF_ERR_ARGS, "pf_morton_workspace_size: bad arguments");
    int64_t rb = radix_blocks(n_prims);
    *bytes = align_up(64) + 6 * align_up(4 * (size_t)n_prims) + align_up(4 * (size_t)(256 * rb)) +
             align_up(4 * (size_t)(scan_blocks(256 * rb) + 1));
    return PF_OK;
}

extern "C" int pf_morton_sort(const float* points, int64_t n_prims, void* workspace, size_t workspace_bytes,
                              int32_t* permutation, void* stream) {
    size_t need = 0;
    if (pf_morton_workspace_size(n_prims, &need) != PF_OK) return PF_ERR_ARGS;
    if (n_prims <= 0 || !points || !permutation || !workspace || workspace_bytes < need)
        return pf_fail(PF_ERR_ARGS, "pf_morton_sort: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    char* ws = (char*)workspace;
    size_t o = 0;
    auto take = [&](size_t b) {
        char* r = ws + o;
        o += align_up(b);
        return r;
    };
    const int64_t N = n_prims;
    float* bounds = (float*)take(64);
    uint32_t* lo = (uint32_t*)take(4 * N);
    uint32_t* hi = (uint32_t*)take(4 * N);
    uint32_t* idx0 = (uint32_t*)take(4 * N);
    uint32_t* k1 = (uint32_t*)take(4 * N);
    uint32_t* idx1 = (uint32_t*)take(4 * N);
    uint32_t* hi_s = (uint32_t*)take(4 * N);
    int64_t rb = radix_blocks(N);
    RadixScratch rs{(uint32_t*)take(4 * 256 * rb), (uint32_t*)take(4 * (scan_blocks(256 * rb) + 1))};
    const unsigned gN = (unsigned)((N + 255) / 256);
    bounds_init_kernel<<<1, 1, 0, st>>>(bounds);
    bounds_kernel<<<(unsigned)std::min<int64_t>(gN, 148 * 8), 256, 0, st>>>(points, nullptr, N, bounds);
    morton_kernel<<<gN, 256, 0, st>>>(points, N, bounds, lo, hi, idx0);
    // LSD: low 32 bits (4 passes) then high 31 bits carried through a gather
    radix_sort_pairs(lo, idx0, k1, idx1, lo, idx0, N, nullptr, 32, rs, st);
    gather_u32_kernel<<<gN, 256, 0, st>>>(hi, idx0, N, hi_s);
    radix_sort_pairs(hi_s, idx0, k1, idx1, hi_s, (uint32_t*)permutation, N, nullptr, 32, rs, st);
    return pf_check_launch("pf_morton_sort");
}

struct PowerLayout {
    size_t slab, counts, extra, extra_n, cell_w, super_w, bytes;
};

static PowerLayout power_layout(int64_t N) {
    PowerLayout P;
    size_t o = cech_layout(N).bytes;
    auto take = [&](size_t b) {
        size_t r = o;
        o = align_up(o + b);
        return r;
    };
    P.slab = take(4 * (size_t)kPowerSlab * (size_t)N);
    P.counts = take(4 * (size_t)N);
    P.extra = take(4 * (size_t)kPowerExtra * (size_t)N);
    P.extra_n = take(4 * (size_t)N);
    P.cell_w = take(4 * ((size_t)1 << kMaxCellsLog2));
    P.super_w = take(4 * ((size_t)1 << kMaxCellsLog2));
    P.bytes = o;
    return P;
}

extern "C" int pf_power_workspace_size(int64_t n_prims, size_t* bytes) {
    if (!bytes || n_prims < 0 || n_prims >= ((int64_t)1 << 31))
        return pf_fail(PF_ERR_ARGS, "pf_power_workspace_size: bad arguments");
    *bytes = power_layout(n_prims).bytes;
    return PF_OK;
}

extern "C" int pf_power_adjacency(const float* points, const float* radii, int64_t n_prims, int32_t alpha_complex,
                                  void* workspace, size_t workspace_bytes, int64_t edge_capacity, int32_t* adjacency,
                                  int32_t* adjacency_offsets, int64_t* n_edges, int32_t* status, void* stream) {
    if (n_prims <= 0 || n_prims >= ((int64_t)1 << 31) || !points || !radii || !adjacency_offsets || !n_edges ||
        !status || edge_capacity < 0 || edge_capacity >= ((int64_t)1 << 31) || (edge_capacity > 0 && !adjacency))
        return pf_fail(PF_ERR_ARGS, "pf_power_adjacency: bad arguments");
    const PowerLayout P = power_layout(n_prims);
    if (!workspace || workspace_bytes < P.bytes) return pf_fail(PF_ERR_ARGS, "pf_power_adjacency: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    char* ws = (char*)workspace;
    const CechLayout L = cech_layout(n_prims);
    const int64_t N = n_prims;
    build_point_grid(points, radii, N, ws, kPowerPtsPerCell, st);
    const Locator loc = locator_view(points, radii, N, ws);
    float* cell_w = (float*)(ws + P.cell_w);
    int* super_w = (int*)(ws + P.super_w);
    int32_t* slab = (int32_t*)(ws + P.slab);
    int32_t* counts = (int32_t*)(ws + P.counts);
    int32_t* extra = (int32_t*)(ws + P.extra);
    int32_t* extra_n = (int32_t*)(ws + P.extra_n);
    int32_t* out_counts = (int32_t*)(ws + L.counts);
    int64_t* off64 = (int64_t*)(ws + L.off64);
    int64_t* spart = (int64_t*)(ws + L.spart);
    const size_t grid_bytes = 4 * ((size_t)1 << kMaxCellsLog2);
    if (cudaMemsetAsync(cell_w, 0, grid_bytes, st) != cudaSuccess ||
        cudaMemsetAsync(super_w, 0xff, grid_bytes, st) != cudaSuccess ||
        cudaMemsetAsync(extra_n, 0, 4 * (size_t)N, st) != cudaSuccess)
        return pf_check_launch("pf_power_adjacency");
    const unsigned gN = (unsigned)((N + 255) / 256);
    cell_weight_kernel<<<gN, 256, 0, st>>>(points, radii, N, loc.grid, cell_w);
    super_weight_kernel<<<(unsigned)(((int64_t)1 << kMaxCellsLog2) / 256), 256, 0, st>>>(loc.grid, loc.cell_start,
                                                                                          cell_w, super_w);
    PowerScene S{points, radii, loc.grid, loc.cell_start, loc.sorted, (const float*)(ws + L.bounds), cell_w,
                 (const float*)super_w};
    power_cell_kernel<<<(unsigned)((N + 63) / 64), 64, 0, st>>>(S, N, slab, counts, status);
    power_symmetrize_kernel<<<gN, 256, 0, st>>>(slab, counts, N, extra, extra_n, status);
    power_emit_kernel<false><<<gN, 256, 0, st>>>(points, radii, slab, counts, extra, extra_n, N, alpha_complex,
                                                 out_counts, nullptr, nullptr, 0, nullptr);
    exclusive_scan<int32_t, int64_t>(out_counts, off64, N, spart, n_edges, st);
    power_emit_kernel<true><<<gN, 256, 0, st>>>(points, radii, slab, counts, extra, extra_n, N, alpha_complex, nullptr,
                                                off64, n_edges, edge_capacity, adjacency);
    offsets_i32_kernel<<<(unsigned)((N + 1 + 255) / 256), 256, 0, st>>>(off64, N, n_edges, edge_capacity,
                                                                        adjacency_offsets, status);
    return pf_check_launch("pf_power_adjacency");
}

extern "C" int pf_steiner_knn(const float* points, const float* radii, int64_t n_prims, const void* workspace,
                              const float* samples, int64_t n_samples, int32_t k, float* sample_radius,
                              int32_t* closest, int32_t* status, void* stream) {
    if (n_prims <= 0 || !points || !radii || !workspace || n_samples < 0 || k < 1 || k > kSteinerK ||
        (n_samples > 0 && (!samples || !sample_radius || !closest)))
        return pf_fail(PF_ERR_ARGS, "pf_steiner_knn: bad arguments (k must be in [1, 32])");
    if (n_samples == 0) return PF_OK;
    Locator loc = locator_view(points, radii, n_prims, (char*)workspace);
    steiner_knn_kernel<<<(unsigned)((n_samples + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
        loc, samples, n_samples, k, sample_radius, closest, status);
    return pf_check_launch("pf_steiner_knn");
}

extern "C" int pf_steiner_select(const float* samples, const float* radii, int64_t n, int64_t seed, float threshold,
                                 float* scratch, uint8_t* selected, int32_t* n_selected, void* stream) {
    if (n < 0 || (n > 0 && (!samples || !radii || !scratch || !selected || seed < 0 || seed >= n)))
        return pf_fail(PF_ERR_ARGS, "pf_steiner_select: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0) {
        if (n_selected && cudaMemsetAsync(n_selected, 0, 4, st) != cudaSuccess)
            return pf_check_launch("pf_steiner_select");
        return PF_OK;
    }
    steiner_select_kernel<<<1, kSelectThreads, 0, st>>>(samples, radii, n, seed, threshold, scratch, selected,
                                                         n_selected);
    return pf_check_launch("pf_steiner_select");
}

extern "C" int pf_occupancy_words(int32_t res, int64_t* words) {
    if (res < 1 || res > 1024 || !words) return pf_fail(PF_ERR_ARGS, "pf_occupancy_words: res must be in [1, 1024]");
    *words = ((int64_t)res * res * res + 31) / 32;
    return PF_OK;
}

extern "C" int pf_occupancy_build(const float* points, const float* radii, const float* density, int64_t n_prims,
                                  const float* box_lo, const float* box_hi, int32_t res, float sigma_min,
                                  uint32_t* bits, int32_t* status, void* stream) {
    VoxelGrid g;
    if (n_prims < 0 || (n_prims > 0 && (!points || !radii || !density)) || !bits || !status ||
        !voxel_grid(box_lo, box_hi, res, &g))
        return pf_fail(PF_ERR_ARGS, "pf_occupancy_build: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t words = ((int64_t)res * res * res + 31) / 32;
    cudaMemsetAsync(bits, 0, sizeof(uint32_t) * (size_t)words, st);
    if (n_prims > 0)
        occupancy_kernel<<<(unsigned)((n_prims + 255) / 256), 256, 0, st>>>(points, radii, density, n_prims, g,
                                                                           sigma_min, bits, status);
    return pf_check_launch("pf_occupancy_build");
}

extern "C" int pf_occupancy_entry(const uint32_t* bits, const float* box_lo, const float* box_hi, int32_t res,
                                  const pf_camera* cam, float margin, float* t_entry, float* confidence,
                                  void* stream) {
    VoxelGrid g;
    if (!bits || !cam || !t_entry || !confidence || cam->width < 2 || cam->height < 2 || !(margin >= 0.0f) ||
        !voxel_grid(box_lo, box_hi, res, &g))
        return pf_fail(PF_ERR_ARGS, "pf_occupancy_entry: bad arguments");
    const int64_t n = (int64_t)cam->width * cam->height;
    occupancy_entry_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(bits, g, load_cam(*cam),
                                                                                          margin, t_entry, confidence);
    return pf_check_launch("pf_occupancy_entry");
}

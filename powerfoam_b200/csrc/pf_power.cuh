// pf_power.cuh -- one site's power cell by clipping (host + device code).
//
// The reference lifts (p, |p|^2 - r^2) to 4-D, takes the lower convex hull
// with Qhull on the host and keeps the tetrahedra's edges
// (benchmark.py:25-83).  Those edges are exactly the pairs whose power cells
// share a face (points in general position), so here every site computes its
// own power cell
//     C_i = { x : |x - p_i|^2 - r_i^2 <= |x - p_j|^2 - r_j^2  for all j }
// by clipping a box with the radical planes of candidate sites: the
// "meshless" construction of Ray, Sokolov, Lefebvre and Levy (Meshless
// Voronoi on the GPU, 2018), extended to weights.  The cell is kept in dual
// form -- planes, and one triangle of three plane indices per cell vertex,
// consistently oriented -- so a clip is: mark the vertices beyond the new
// plane, take the boundary edges of the marked triangles, fan new triangles
// from those edges to the new plane.
//
// Candidates come from a uniform grid (about one site per grid cell).  The
// cell is first clipped by the nearest radical planes among the 27
// surrounding grid cells (a warm start), then the grid is walked shell by
// shell.  A site can cut vertex v only if it lies inside v's power ball,
// |x - v|^2 < |v|^2 + r_j^2 - r_i^2, so a grid cell is scanned only if it
// meets one of those balls (bounded with the cell's largest r^2); cutting is
// monotone (a later cell is a subset of an earlier one), so a cell culled
// once never holds a cutter later.  The walk stops when the shells scanned
// cover the security radius rho + sqrt(rho^2 + max r^2 - r_i^2), rho the
// largest vertex distance.  After a few fine shells the walk continues over
// blocks of kPcSuper^3 grid cells, each culled as a whole first: the
// unbounded cells of hull sites reach the padded box and are only settled by
// the whole grid, which the blocks make cheap.  All geometry is in double
// precision relative to p_i with w = r^2 exact; the box is the scene's
// bounding box padded by kPowerPad times its extent, so the unbounded faces
// of hull sites cross it and are found.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace pf {

constexpr int kPcPlanes = 255;              // live planes of one cell (plane ids fit a byte)
constexpr int kPcTris = 2 * kPcPlanes - 4;  // vertices of a cell with kPcPlanes faces
constexpr int kPowerSlab = 192;             // neighbours written per site
constexpr int kPowerExtra = 4;              // one-sided edges added to a site's list
constexpr int kPcWarm = 32;                 // warm-start planes
constexpr int kPcSuper = 8;                 // grid cells per block edge in the coarse walk
constexpr int kPcLocalShells = 3;           // shells walked cell by cell before the coarse walk
constexpr double kPowerPad = 1.0e6;         // box padding, in scene extents
constexpr float kPowerPtsPerCell = 1.0f;    // grid density of the power build

// uniform grid: cell (x, y, z) covers lo + [x, x + 1) / inv_h per axis
struct CechGrid {
    float lo_x, lo_y, lo_z, inv_h;
    int nx, ny, nz;
};

struct PowerScene {
    const float* pts;
    const float* radii;
    const CechGrid* grid;
    const int32_t* cell_start;
    const uint32_t* sorted;
    const float* bounds;   // lo3, hi3 as order keys; rmax as a float at [8]
    const float* cell_w;   // per grid cell, the largest r^2 of its sites
    const float* super_w;  // per block of kPcSuper^3 cells, the same (negative: no site)
};

struct PowerCell {
    double n[kPcPlanes][3];  // plane n . x <= c, relative to the site
    double c[kPcPlanes];
    int32_t owner[kPcPlanes];  // the neighbour, -1 for box planes
    uint8_t tri[kPcTris][3];   // a vertex: three planes, det(n_a, n_b, n_c) > 0
    double v[kPcTris][3];
    double vn2[kPcTris];
    uint8_t out[kPcTris];
    uint16_t ol[kPcTris];  // triangles beyond the clipping plane
    uint8_t bnd[kPcTris * 3][2];
    double wkey[kPcWarm];  // warm-start candidates, nearest plane first
    int32_t wid[kPcWarm];
    int np, nt;
    double rho2;
    bool overflow;
};

__host__ __device__ __forceinline__ int pc_imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int pc_imax(int a, int b) { return a > b ? a : b; }

__host__ __device__ __forceinline__ void pc_vertex(PowerCell& C, int t) {
    const int a = C.tri[t][0], b = C.tri[t][1], q = C.tri[t][2];
    const double* na = C.n[a];
    const double* nb = C.n[b];
    const double* nq = C.n[q];
    const double bq[3] = {nb[1] * nq[2] - nb[2] * nq[1], nb[2] * nq[0] - nb[0] * nq[2], nb[0] * nq[1] - nb[1] * nq[0]};
    const double qa[3] = {nq[1] * na[2] - nq[2] * na[1], nq[2] * na[0] - nq[0] * na[2], nq[0] * na[1] - nq[1] * na[0]};
    const double ab[3] = {na[1] * nb[2] - na[2] * nb[1], na[2] * nb[0] - na[0] * nb[2], na[0] * nb[1] - na[1] * nb[0]};
    const double det = na[0] * bq[0] + na[1] * bq[1] + na[2] * bq[2];
    double v2 = 0.0;
    for (int k = 0; k < 3; k++) {
        const double x = (C.c[a] * bq[k] + C.c[b] * qa[k] + C.c[q] * ab[k]) / det;
        C.v[t][k] = x;
        v2 += x * x;
    }
    C.vn2[t] = v2;
}

__host__ __device__ __forceinline__ void pc_rho(PowerCell& C) {
    double r = 0.0;
    for (int t = 0; t < C.nt; t++) r = fmax(r, C.vn2[t]);
    C.rho2 = r;
}

// box [lo, hi] relative to the site: six planes, eight vertex triangles
__host__ __device__ __forceinline__ void pc_init(PowerCell& C, const double lo[3], const double hi[3]) {
    for (int k = 0; k < 3; k++) {
        for (int s = 0; s < 2; s++) {
            double* n = C.n[2 * k + s];
            n[0] = n[1] = n[2] = 0.0;
            n[k] = s == 0 ? 1.0 : -1.0;
            C.c[2 * k + s] = s == 0 ? hi[k] : -lo[k];
            C.owner[2 * k + s] = -1;
        }
    }
    C.np = 6;
    C.nt = 0;
    for (int sx = 0; sx < 2; sx++)
        for (int sy = 0; sy < 2; sy++)
            for (int sz = 0; sz < 2; sz++) {
                uint8_t a = (uint8_t)sx, b = (uint8_t)(2 + sy), q = (uint8_t)(4 + sz);
                // det(sgn_x e_x, sgn_y e_y, sgn_z e_z) = sgn_x sgn_y sgn_z
                if ((sx + sy + sz) & 1) {
                    const uint8_t t = a;
                    a = b;
                    b = t;
                }
                C.tri[C.nt][0] = a;
                C.tri[C.nt][1] = b;
                C.tri[C.nt][2] = q;
                pc_vertex(C, C.nt);
                C.nt++;
            }
    pc_rho(C);
    C.overflow = false;
}

// drop planes no triangle references; false if nothing was freed
static __host__ __device__ __noinline__ bool pc_compact_planes(PowerCell& C) {
    uint8_t map[kPcPlanes];
    for (int p = 0; p < C.np; p++) map[p] = 0xff;
    for (int t = 0; t < C.nt; t++)
        for (int k = 0; k < 3; k++) map[C.tri[t][k]] = 0;
    int m = 0;
    for (int p = 0; p < C.np; p++) {
        if (map[p] == 0xff) continue;
        if (m != p) {
            for (int k = 0; k < 3; k++) C.n[m][k] = C.n[p][k];
            C.c[m] = C.c[p];
            C.owner[m] = C.owner[p];
        }
        map[p] = (uint8_t)m++;
    }
    const bool freed = m < C.np;
    for (int t = 0; t < C.nt; t++)
        for (int k = 0; k < 3; k++) C.tri[t][k] = map[C.tri[t][k]];
    C.np = m;
    return freed;
}

// clip by n . x <= c (neighbour `owner`); true if the cell changed.  A plane
// must not be applied twice: the vertices it made lie on it up to rounding.
static __host__ __device__ __noinline__ bool pc_clip(PowerCell& C, double nx, double ny, double nz, double c,
                                              int32_t owner) {
    int n_out = 0;
    for (int t = 0; t < C.nt; t++) {
        const bool o = nx * C.v[t][0] + ny * C.v[t][1] + nz * C.v[t][2] > c;
        C.out[t] = o;
        if (o) C.ol[n_out++] = (uint16_t)t;
    }
    if (n_out == 0) return false;
    if (n_out == C.nt) {
        C.nt = 0;
        C.rho2 = 0.0;
        return true;
    }
    if (C.np == kPcPlanes && !pc_compact_planes(C)) {
        C.overflow = true;
        return false;
    }
    // boundary of the removed region: edges of removed triangles whose
    // reverse is not an edge of another removed triangle
    int m = 0;
    for (int a = 0; a < n_out; a++) {
        const int t = C.ol[a];
        for (int e = 0; e < 3; e++) {
            const uint8_t x = C.tri[t][e], y = C.tri[t][(e + 1) % 3];
            bool inner = false;
            for (int b = 0; b < n_out && !inner; b++) {
                const int u = C.ol[b];
                if (u == t) continue;
                for (int f = 0; f < 3; f++)
                    if (C.tri[u][f] == y && C.tri[u][(f + 1) % 3] == x) inner = true;
            }
            if (!inner) {
                C.bnd[m][0] = x;
                C.bnd[m][1] = y;
                m++;
            }
        }
    }
    if (C.nt - n_out + m > kPcTris) {
        C.overflow = true;
        return false;
    }
    const int q = C.np++;
    C.n[q][0] = nx;
    C.n[q][1] = ny;
    C.n[q][2] = nz;
    C.c[q] = c;
    C.owner[q] = owner;
    int w = 0;
    for (int t = 0; t < C.nt; t++) {
        if (C.out[t]) continue;
        if (w != t) {
            for (int k = 0; k < 3; k++) {
                C.tri[w][k] = C.tri[t][k];
                C.v[w][k] = C.v[t][k];
            }
            C.vn2[w] = C.vn2[t];
        }
        w++;
    }
    for (int e = 0; e < m; e++) {
        C.tri[w][0] = C.bnd[e][0];
        C.tri[w][1] = C.bnd[e][1];
        C.tri[w][2] = (uint8_t)q;
        pc_vertex(C, w);
        w++;
    }
    C.nt = w;
    pc_rho(C);
    return true;
}

// can a site inside the box [blo, bhi] (relative) cut a vertex?  dw bounds
// r_j^2 - r_i^2 for the sites of the box.
static __host__ __device__ __noinline__ bool pc_box_may_cut(const PowerCell& C, const double blo[3], const double bhi[3],
                                                     double dw) {
    for (int t = 0; t < C.nt; t++) {
        const double r2 = C.vn2[t] + dw;
        if (r2 <= 0.0) continue;
        double d2 = 0.0;
        for (int k = 0; k < 3; k++) {
            const double x = C.v[t][k];
            const double e = x < blo[k] ? blo[k] - x : (x > bhi[k] ? x - bhi[k] : 0.0);
            d2 += e * e;
        }
        if (d2 < r2) return true;
    }
    return false;
}

// box [blo, bhi] against the sphere |x| <= rho holding every vertex, then
// against each vertex's power ball
__host__ __device__ __forceinline__ bool pc_box_culled(const PowerCell& C, const double blo[3], const double bhi[3],
                                                       double dw) {
    double bd2 = 0.0;
    for (int k = 0; k < 3; k++) {
        const double e = blo[k] > 0.0 ? blo[k] : (bhi[k] < 0.0 ? -bhi[k] : 0.0);
        bd2 += e * e;
    }
    const double reach = sqrt(C.rho2) + sqrt(fmax(0.0, C.rho2 + dw));
    return bd2 >= reach * reach || !pc_box_may_cut(C, blo, bhi, dw);
}

__host__ __device__ __forceinline__ float pc_key_float(int key) {
    const int b = key >= 0 ? key : (key ^ 0x7fffffff);
    float f;
    memcpy(&f, &b, sizeof(f));
    return f;
}

// the grid cell of a coordinate (the assignment the cell sort uses)
__host__ __device__ __forceinline__ int pc_cell_coord(float v, float lo, float inv_h, int n) {
    const float f = floorf((v - lo) * inv_h);
    if (!(f == f) || f < 0.f) return 0;
    if (f >= (float)n) return n - 1;
    return (int)f;
}

struct PcSite {
    int64_t i;
    double p[3], wi, h, margin;
    double glo[3];
};

// clip by the sites of grid cell (x, y, z), culling the grid cell first if
// asked; warm-start sites (already applied) are skipped
static __host__ __device__ __noinline__ void pc_scan_cell(const PowerScene& S, const CechGrid& g, const PcSite& st, int x,
                                                   int y, int z, bool cull, PowerCell& C, int nk) {
    if (C.nt == 0 || C.overflow) return;
    const int64_t cell = ((int64_t)z * g.ny + y) * g.nx + x;
    if (S.cell_start[cell] == S.cell_start[cell + 1]) return;
    if (cull && g.inv_h > 0.f) {
        const int xyz[3] = {x, y, z};
        double clo[3], chi[3];
        for (int k = 0; k < 3; k++) {
            clo[k] = st.glo[k] + xyz[k] * st.h - st.margin - st.p[k];
            chi[k] = st.glo[k] + (xyz[k] + 1) * st.h + st.margin - st.p[k];
        }
        if (pc_box_culled(C, clo, chi, (double)S.cell_w[cell] - st.wi)) return;
    }
    for (int32_t qi = S.cell_start[cell]; qi < S.cell_start[cell + 1] && C.nt > 0 && !C.overflow; qi++) {
        const int64_t j = S.sorted[qi];
        if (j == st.i) continue;
        const double d0 = (double)S.pts[3 * j] - st.p[0];
        const double d1 = (double)S.pts[3 * j + 1] - st.p[1];
        const double d2 = (double)S.pts[3 * j + 2] - st.p[2];
        const double wj = (double)S.radii[j] * (double)S.radii[j];
        const double dd = d0 * d0 + d1 * d1 + d2 * d2;
        if (dd == 0.0) {
            if (wj > st.wi) {  // same centre, larger ball: the cell is empty
                C.nt = 0;
                C.rho2 = 0.0;
            }
            continue;
        }
        const double c = 0.5 * (dd - wj + st.wi);
        if (c >= 0.0 && c * c >= dd * C.rho2) continue;  // plane beyond every vertex
        bool seen = false;
        for (int k = 0; k < nk; k++) seen |= C.wid[k] == (int32_t)j;
        if (seen) continue;
        pc_clip(C, d0, d1, d2, c, (int32_t)j);
    }
}

// The power cell of site i; its neighbours (ascending, at most kPowerSlab)
// go to out, the count is returned, *full reports a capacity overflow.
static __host__ __device__ __noinline__ int power_site(const PowerScene& S, int64_t i, PowerCell& C, int32_t* out,
                                                bool* full) {
    const CechGrid g = *S.grid;
    const int* bk = (const int*)S.bounds;
    double lo[3], hi[3], ext = 0.0;
    for (int k = 0; k < 3; k++) {
        lo[k] = (double)pc_key_float(bk[k]);
        hi[k] = (double)pc_key_float(bk[3 + k]);
        ext = fmax(ext, hi[k] - lo[k]);
    }
    const double rmax = (double)S.bounds[8];
    const double pad = kPowerPad * fmax(ext, 1e-3);
    PcSite st;
    st.i = i;
    for (int k = 0; k < 3; k++) st.p[k] = (double)S.pts[3 * i + k];
    st.wi = (double)S.radii[i] * (double)S.radii[i];
    const double dw = rmax * rmax - st.wi;  // r_j^2 - r_i^2 bound over every site
    double blo[3], bhi[3];
    for (int k = 0; k < 3; k++) {
        blo[k] = lo[k] - pad - st.p[k];
        bhi[k] = hi[k] + pad - st.p[k];
    }
    pc_init(C, blo, bhi);
    st.h = 1.0 / (double)g.inv_h;
    st.glo[0] = (double)g.lo_x;
    st.glo[1] = (double)g.lo_y;
    st.glo[2] = (double)g.lo_z;
    st.margin = 1e-4 * (g.inv_h > 0.f ? st.h : 0.0) + 1e-6 * (ext + 1.0);
    const int gn[3] = {g.nx, g.ny, g.nz};
    const int cc[3] = {pc_cell_coord(S.pts[3 * i], g.lo_x, g.inv_h, g.nx),
                       pc_cell_coord(S.pts[3 * i + 1], g.lo_y, g.inv_h, g.ny),
                       pc_cell_coord(S.pts[3 * i + 2], g.lo_z, g.inv_h, g.nz)};
    const int smax = pc_imax(pc_imax(g.nx, g.ny), g.nz);

    // warm start: the nearest radical planes of the 27 surrounding cells
    int nk = 0;
    for (int z = pc_imax(cc[2] - 1, 0); z <= pc_imin(cc[2] + 1, g.nz - 1); z++)
        for (int y = pc_imax(cc[1] - 1, 0); y <= pc_imin(cc[1] + 1, g.ny - 1); y++)
            for (int x = pc_imax(cc[0] - 1, 0); x <= pc_imin(cc[0] + 1, g.nx - 1); x++) {
                const int64_t cell = ((int64_t)z * g.ny + y) * g.nx + x;
                for (int32_t qi = S.cell_start[cell]; qi < S.cell_start[cell + 1]; qi++) {
                    const int64_t j = S.sorted[qi];
                    if (j == i) continue;
                    const double d0 = (double)S.pts[3 * j] - st.p[0];
                    const double d1 = (double)S.pts[3 * j + 1] - st.p[1];
                    const double d2 = (double)S.pts[3 * j + 2] - st.p[2];
                    const double dd = d0 * d0 + d1 * d1 + d2 * d2;
                    if (dd == 0.0) continue;
                    const double wj = (double)S.radii[j] * (double)S.radii[j];
                    const double c = 0.5 * (dd - wj + st.wi);
                    // signed squared distance of the plane from the site
                    const double key = c < 0.0 ? -(c * c) / dd : (c * c) / dd;
                    if (nk == kPcWarm && key >= C.wkey[nk - 1]) continue;
                    int w = nk < kPcWarm ? nk++ : nk - 1;
                    while (w > 0 && C.wkey[w - 1] > key) {
                        C.wkey[w] = C.wkey[w - 1];
                        C.wid[w] = C.wid[w - 1];
                        w--;
                    }
                    C.wkey[w] = key;
                    C.wid[w] = (int32_t)j;
                }
            }
    for (int k = 0; k < nk && C.nt > 0 && !C.overflow; k++) {
        const int64_t j = C.wid[k];
        const double d0 = (double)S.pts[3 * j] - st.p[0];
        const double d1 = (double)S.pts[3 * j + 1] - st.p[1];
        const double d2 = (double)S.pts[3 * j + 2] - st.p[2];
        const double wj = (double)S.radii[j] * (double)S.radii[j];
        const double dd = d0 * d0 + d1 * d1 + d2 * d2;
        const double c = 0.5 * (dd - wj + st.wi);
        if (c >= 0.0 && c * c >= dd * C.rho2) continue;
        pc_clip(C, d0, d1, d2, c, (int32_t)j);
    }

    // fine walk: grid cells, shell by shell
    int s_done = -1;
    bool done = false;
    const int s_fine = pc_imin(smax, kPcLocalShells);
    for (int s = 0; s <= s_fine && C.nt > 0 && !C.overflow; s++) {
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
                    pc_scan_cell(S, g, st, x, y, z, s >= 1, C, nk);
                }
            }
        }
        s_done = s;
        if (C.nt == 0 || C.overflow) break;
        // radius covered by shells 0..s (a side at the grid edge is
        // unbounded: no site lies beyond it)
        double reach = INFINITY;
        for (int k = 0; k < 3; k++) {
            if (cc[k] - s > 0) reach = fmin(reach, st.p[k] - (st.glo[k] + (cc[k] - s) * st.h));
            if (cc[k] + s < gn[k] - 1) reach = fmin(reach, st.glo[k] + (cc[k] + s + 1) * st.h - st.p[k]);
        }
        if (reach - st.margin >= sqrt(C.rho2) + sqrt(fmax(0.0, C.rho2 + dw))) {
            done = true;
            break;
        }
    }

    // coarse walk: blocks of kPcSuper^3 grid cells, shell by shell
    if (!done && C.nt > 0 && !C.overflow) {
        const int F = kPcSuper;
        const int sn[3] = {(g.nx + F - 1) / F, (g.ny + F - 1) / F, (g.nz + F - 1) / F};
        const int sc[3] = {cc[0] / F, cc[1] / F, cc[2] / F};
        const int smax2 = pc_imax(pc_imax(sn[0], sn[1]), sn[2]);
        for (int s = 0; s <= smax2 && C.nt > 0 && !C.overflow; s++) {
            for (int dz = -s; dz <= s; dz++) {
                const int Z = sc[2] + dz;
                if (Z < 0 || Z >= sn[2]) continue;
                for (int dy = -s; dy <= s; dy++) {
                    const int Y = sc[1] + dy;
                    if (Y < 0 || Y >= sn[1]) continue;
                    const bool face = (dz == -s || dz == s || dy == -s || dy == s);
                    const int step = (face || s == 0) ? 1 : 2 * s;
                    for (int dx = -s; dx <= s && C.nt > 0 && !C.overflow; dx += step) {
                        const int X = sc[0] + dx;
                        if (X < 0 || X >= sn[0]) continue;
                        const float sw = S.super_w[((int64_t)Z * sn[1] + Y) * sn[0] + X];
                        if (!(sw >= 0.f)) continue;  // no site in the block
                        const int b0[3] = {X * F, Y * F, Z * F};
                        const int b1[3] = {pc_imin(b0[0] + F, g.nx), pc_imin(b0[1] + F, g.ny),
                                           pc_imin(b0[2] + F, g.nz)};
                        bool inside = true;  // wholly inside the finely walked shells
                        for (int k = 0; k < 3; k++) inside &= b0[k] >= cc[k] - s_done && b1[k] - 1 <= cc[k] + s_done;
                        if (inside) continue;
                        double blo2[3], bhi2[3];
                        for (int k = 0; k < 3; k++) {
                            blo2[k] = st.glo[k] + b0[k] * st.h - st.margin - st.p[k];
                            bhi2[k] = st.glo[k] + b1[k] * st.h + st.margin - st.p[k];
                        }
                        if (pc_box_culled(C, blo2, bhi2, (double)sw - st.wi)) continue;
                        for (int z = b0[2]; z < b1[2]; z++)
                            for (int y = b0[1]; y < b1[1]; y++)
                                for (int x = b0[0]; x < b1[0]; x++) {
                                    if (abs(x - cc[0]) <= s_done && abs(y - cc[1]) <= s_done &&
                                        abs(z - cc[2]) <= s_done)
                                        continue;
                                    pc_scan_cell(S, g, st, x, y, z, true, C, nk);
                                }
                    }
                }
            }
            if (C.nt == 0 || C.overflow) break;
            double reach = INFINITY;
            for (int k = 0; k < 3; k++) {
                if (sc[k] - s > 0) reach = fmin(reach, st.p[k] - (st.glo[k] + (double)(sc[k] - s) * F * st.h));
                if ((sc[k] + s + 1) * F < gn[k])
                    reach = fmin(reach, st.glo[k] + (double)(sc[k] + s + 1) * F * st.h - st.p[k]);
            }
            if (reach - st.margin >= sqrt(C.rho2) + sqrt(fmax(0.0, C.rho2 + dw))) break;
        }
    }

    // neighbours: owners of the planes that still bound the cell
    int cnt = 0;
    *full = C.overflow;
    if (C.nt > 0) {
        uint8_t used[kPcPlanes];
        for (int q = 0; q < C.np; q++) used[q] = 0;
        for (int t = 0; t < C.nt; t++)
            for (int k = 0; k < 3; k++) used[C.tri[t][k]] = 1;
        for (int q = 0; q < C.np; q++) {
            if (!used[q] || C.owner[q] < 0) continue;
            if (cnt == kPowerSlab) {
                *full = true;
                break;
            }
            const int32_t v = C.owner[q];
            int w = cnt - 1;
            while (w >= 0 && out[w] > v) {
                out[w + 1] = out[w];
                w--;
            }
            out[w + 1] = v;
            cnt++;
        }
    }
    return cnt;
}

}  // namespace pf

/*
 * pfoam.h -- C ABI of libpfoam, the B200 (sm_100a) implementation of the
 * Power Foam rendering hot path.
 *
 * Conventions (every entry point):
 *   - all array arguments are DEVICE pointers, C-contiguous, in the layouts
 *     stated beside each argument; sizes are int64 element counts;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *   - nothing is allocated and nothing synchronises with the host: scratch
 *     memory is passed in by the caller (see the *_workspace_size queries);
 *   - the return value is a host-side status (PF_OK or PF_ERR_*) covering
 *     argument validation and launch errors; conditions discovered on the
 *     device (buffer overflow, walk step cap, ...) are written to a device
 *     status word the caller reads when it chooses;
 *   - pf_last_error() describes the last non-zero return on this thread.
 *
 * Each entry point names the reference interface it replaces
 * (file:line inside theialab/powerfoam).
 */
#ifndef PFOAM_H
#define PFOAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_OK 0
#define PF_ERR_OVERFLOW 1  /* (tile, primitive) pairs exceeded the capacity */
#define PF_ERR_STEP_CAP 2  /* a cell walk reached max_steps */
#define PF_ERR_ARGS 3      /* invalid argument */
#define PF_ERR_CUDA 4      /* CUDA launch / runtime error */
#define PF_ERR_SEED 5      /* a proposal seed landed outside every cell */
#define PF_ERR_CELL 6      /* a power cell exceeded its plane / neighbour capacity */
#define PF_ERR_NONFINITE 7 /* a primitive attribute is NaN or infinite */

#define PF_ABI_VERSION 4

#if defined(__GNUC__)
#define PF_API __attribute__((visibility("default")))
#else
#define PF_API
#endif

/* Pinhole camera: powerfoam/camera.py:8-16 (WarpCamera) / :181-189
 * (TorchCamera).  |up| = tan(vfov/2), |right| = |up| * width / height and the
 * view direction is normalize(cross(up, right)). */
typedef struct pf_camera {
    float eye[3];
    float right[3];
    float up[3];
    int32_t width;
    int32_t height;
} pf_camera;

/* Inputs shared by the rasterizer entry points.  Replaces the argument list
 * of Rasterizer._forward / benchmark / visualize (powerfoam/rasterize.py:
 * 1587-1603, 1982-1996, 2133-2146) after their torch.cat packing. */
typedef struct pf_raster_inputs {
    pf_camera cam;
    int32_t tile_width;          /* tile edge in pixels (reference: 8) */
    int32_t n_sites;             /* texel sites per primitive, <= 8 */
    int64_t n_prims;
    const float *spheres;        /* (N,4) f32: centre xyz, radius */
    const void *nsigmas;         /* (N,4): normal xyz, density; f32 or f16 */
    const void *texel_sites;     /* (N,S,3) f32 or f16 */
    const void *texel_rgb;       /* (N,S,3) f32 or f16 */
    const void *texel_height;    /* (N,S)   f32 or f16 */
    int32_t attr_half;           /* 1: the four arrays above are f16 */
    const int32_t *adjacency;          /* (E) neighbour ids */
    const int32_t *adjacency_offsets;  /* (N+1) */
    const uint16_t *adjacency_diff;    /* (E,4) f16 bits; see each entry */
    const int64_t *tile_offsets; /* (T+1), T = ceil(H/tw)*ceil(W/tw) */
    const int32_t *tile_prims;   /* sorted primitive ids per tile */
    const float *depth_quantiles; /* (H,W,Q) or NULL */
    int32_t n_quantiles;
    const float *ray_gt;         /* (H,W,3) or NULL */
    float transmittance_threshold;
    const int32_t *tile_order;   /* (T) tile processing order (longest lists
                                    first, from pf_bin) or NULL */
    void *scratch;               /* >= 256 bytes of device scratch for the
                                    tile work queue, or NULL (one warp group
                                    per tile, no queue) */
    const float *ray_maps;       /* (H,W,6) f32 per-pixel ray origin and
                                    direction of a generic camera
                                    (TorchCamera.ray_maps, is_pinhole=False;
                                    rasterize.py:944-954) for the forward and
                                    backward, or NULL for the pinhole rays;
                                    the benchmark and viewer paths are
                                    pinhole only, as in the reference */
    float *segments;             /* optional segment records, one per hit
                                    (primitive, pixel) pair: a float4 with the
                                    sphere interval clipped by the power faces
                                    and the ids of the surfaces bounding it,
                                    then, with segment_planes, three float4 of
                                    the texture-plane result (64 bytes a
                                    record, else 16).  pf_raster_forward
                                    (tile widths 8 and 16) reserves the
                                    records of each warp's hits per 32
                                    primitives and writes them;
                                    pf_raster_backward reads them instead of
                                    clipping and evaluating the plane again.
                                    NULL: none.  16-byte aligned */
    uint32_t *segment_masks;     /* (pairs x tw^2 / 32) per pair and warp of
                                    32 pixels, the pixels whose ray hits the
                                    sphere */
    int32_t *segment_offsets;    /* (pairs x tw^2 / 32) per pair and warp,
                                    the index of its first record (the hits
                                    follow in pixel order), -1 when the
                                    buffer was full: the adjoint then clips
                                    again for that pair */
    int64_t *segment_count;      /* device counter of the records reserved;
                                    zero before the forward */
    int64_t segment_pairs;       /* pairs the mask and offset arrays hold
                                    (>= the pairs in tile_prims) */
    int64_t segment_capacity;    /* records the buffer holds (< 2^31) */
    int32_t segment_planes;      /* 1: the records hold the plane results */
} pf_raster_inputs;

/* ---------------------------------------------------------------------- */
PF_API int pf_abi_version(void);
PF_API const char *pf_last_error(void);

/* Pack per-primitive attributes into the float4 layouts the kernels read:
 * spheres = (points, radii), nsigmas = (normals, density).
 * Replaces the torch.cat calls of rasterize.py:1619-1620.  status (device,
 * may be NULL) is raised to PF_ERR_NONFINITE (atomic max, never lowered) when
 * any packed value is NaN or infinite; the reference has no such check (its
 * adjoint only zeroes non-finite gradients, rasterize.py:1954-1958). */
PF_API int pf_pack_prims(const float *points, const float *radii, const float *normals, const float *density,
                  int64_t n_prims, float *spheres, float *nsigmas, int32_t *status, void *stream);

/* ---------------------------------------------------------------------- */
/* Binning.  Replaces rasterize.py:1671-1768: count_visible_pinhole_kernel
 * (:140-200), torch.cumsum + offsets[-1].item() (:1713-1714),
 * write_visible_pinhole_kernel (:293-363), the prim_visible_mask scatter
 * (:1761-1765) and torch.argsort(sort_keys) + gather (:1767-1768).
 * Order: by tile, then by the float32 bits of |c - eye|^2 - r^2, then by
 * ascending primitive index (the reference leaves ties unordered).
 * On overflow (*n_pairs > pair_capacity) the tile lists are emptied and
 * *status is set to PF_ERR_OVERFLOW; *n_pairs always holds the true count. */
PF_API int pf_bin_workspace_size(int64_t n_prims, int64_t pair_capacity, int64_t n_tiles, size_t *bytes);
PF_API int pf_bin(const pf_camera *cam, int32_t tile_width, const float *spheres, int64_t n_prims, void *workspace,
           size_t workspace_bytes, int64_t pair_capacity, int64_t *tile_offsets, int32_t *tile_prims,
           int64_t *sort_keys /* (capacity) or NULL */, uint8_t *prim_visible /* (N) or NULL */,
           int32_t *tile_order /* (T) or NULL: tiles by decreasing list length */,
           int64_t *n_pairs /* device scalar */, int32_t *status /* device scalar */, void *stream);

/* Allocation-free binning: pf_bin with its scratch in a static device array
 * (7 MiB, held by every GPU that loads the library), for callers that cannot
 * allocate device memory while they render (a host application's frame
 * callback, code that must not synchronise the device through cudaMalloc).
 * No counterpart in the reference.  Limits: n_prims <= 65536,
 * pair_capacity <= 262144, at most 16384 tiles; larger problems return
 * PF_ERR_ARGS.  The first call on a device caches the array's address: make it
 * before any stream capture; a cudaDeviceReset afterwards leaves the cached
 * address stale and is not supported.  All calls share the array, so calls that may
 * overlap on the GPU race and must be serialised by the caller.  Outputs and
 * *status as for pf_bin. */
PF_API int pf_bin_noalloc(const pf_camera *cam, int32_t tile_width, const float *spheres, int64_t n_prims,
                          int64_t pair_capacity, int64_t *tile_offsets, int32_t *tile_prims, int64_t *sort_keys,
                          uint8_t *prim_visible, int32_t *tile_order, int64_t *n_pairs, int32_t *status,
                          void *stream);

/* Binning for a generic camera (TorchCamera.ray_maps with is_pinhole=False).
 * Replaces _precompute_cones, compute_leaf_cones_kernel, merge_cones_kernel
 * and count/write_visible_generic_kernel (rasterize.py:202-291, 365-569,
 * 1518-1585): ray cones over 2x2-pixel leaves merged level by level to one
 * root, each primitive descending into every cone its sphere meets
 * (camera.py:28-44) down to the level whose cones are the tiles.  ray_maps
 * is (H,W,6) f32 (origin, direction); tile_width must be a power of two
 * (8, 16 or 32 for the compositing kernels).  Outputs, ordering and *status
 * as for pf_bin; the workspace also holds the cones. */
PF_API int pf_bin_generic_workspace_size(int64_t n_prims, int64_t pair_capacity, int32_t width, int32_t height,
                                         int32_t tile_width, size_t *bytes);
PF_API int pf_bin_generic(const pf_camera *cam, const float *ray_maps, int32_t tile_width, const float *spheres,
                          int64_t n_prims, void *workspace, size_t workspace_bytes, int64_t pair_capacity,
                          int64_t *tile_offsets, int32_t *tile_prims, int64_t *sort_keys, uint8_t *prim_visible,
                          int32_t *tile_order, int64_t *n_pairs, int32_t *status, void *stream);

/* ---------------------------------------------------------------------- */
/* Neighbour encodings.
 * pf_adjacency_prefetch: (half(c_j - c_i), half(r_j)); replaces
 *   prefetch_adjacency_kernel, rasterize.py:580-606.
 * pf_adjacency_power_diff: (half(c_j - c_i), half(pm_j - pm_i)) with
 *   pm = (|c|^2 - r^2)/2; replaces benchmark.py:296-302. */
PF_API int pf_adjacency_prefetch(const float *spheres, const int32_t *adjacency, const int32_t *adjacency_offsets,
                          int64_t n_prims, uint16_t *adjacency_diff, void *stream);
PF_API int pf_adjacency_power_diff(const float *points, const float *radii, const int32_t *adjacency,
                            const int32_t *adjacency_offsets, int64_t n_prims, uint16_t *adjacency_diff,
                            void *stream);

/* Čech adjacency: j is a neighbour of i iff their AABBs overlap and
 * |c_i - c_j| < r_i + r_j with c, r recovered from the AABB.  Replaces
 * AABBTree.update + build_cech_complex (powerfoam/bvh.py:72-123, Warp BVH
 * query kernels :7-69); lists are in ascending neighbour order.  As for
 * binning, *n_edges always receives the true count and on overflow
 * (*n_edges > edge_capacity) the offsets are zeroed and *status is set to
 * PF_ERR_OVERFLOW. */
PF_API int pf_cech_workspace_size(int64_t n_prims, size_t *bytes);
PF_API int pf_cech_adjacency(const float *points, const float *radii, int64_t n_prims, void *workspace,
                             size_t workspace_bytes, int64_t edge_capacity, int32_t *adjacency /* (capacity) */,
                             int32_t *adjacency_offsets /* (N+1) */, int64_t *n_edges /* device */,
                             int32_t *status /* device */, void *stream);

/* Interpenetration penalty.  Replaces interpenetration_kernel and
 * InterpenetrationFunction (powerfoam/geometry.py:88-189).  spheres (N,4) =
 * (centre, radius), 16-byte aligned; for each i, areas[i] = sum over its list,
 * in list order, of (r_i + r_j - d)^2 where d = |c_i - c_j| < r_i + r_j
 * (bit-identical to the reference's loop, with pow(x, 2) as x * x).  The
 * backward writes dL/dspheres (N,4, zeroed first, 16-byte aligned) given
 * dL/dareas (N): per overlapping entry g = 2 (r_i + r_j - d) dL/dareas_i to
 * both radii and, when d > 0, -g (c_i - c_j) / d to c_i and its negative to
 * c_j (Warp's generated adjoint; summed in no fixed order).  n_edges is
 * the length of adjacency.  A neighbour index outside [0, N), or offsets that
 * decrease or leave [0, n_edges], are skipped (clamped) and set PF_ERR_ARGS
 * in *status (device, may be NULL); the reference has no such check. */
PF_API int pf_interpenetration(const float *spheres, const int32_t *adjacency, const int32_t *adjacency_offsets,
                               int64_t n_prims, int64_t n_edges, float *areas, int32_t *status, void *stream);
PF_API int pf_interpenetration_backward(const float *spheres, const int32_t *adjacency,
                                        const int32_t *adjacency_offsets, int64_t n_prims, int64_t n_edges,
                                        const float *grad_areas, float *grad_spheres, int32_t *status,
                                        void *stream);

/* Power-diagram (weighted Delaunay) adjacency on the GPU.  Replaces
 * build_power_adjacency (benchmark.py:25-83: lifted 4-D convex hull by Qhull
 * on the host, lower facets, tetrahedron edges, optional alpha_complex filter
 * |c_i - c_j| < r_i + r_j) by clipping each site's power cell with its
 * neighbours' radical planes in double precision.  The lists hold the
 * reference's neighbour sets, ascending and without the repeats its
 * torch.unique over unordered pairs leaves.  A cell with more than 96
 * neighbours or 128 live planes sets PF_ERR_CELL in *status; *n_edges and
 * edge overflow behave as in pf_cech_adjacency.  Exact duplicate sites (same
 * centre and radius) both keep their cells, where the hull keeps one. */
PF_API int pf_power_workspace_size(int64_t n_prims, size_t *bytes);
PF_API int pf_power_adjacency(const float *points, const float *radii, int64_t n_prims, int32_t alpha_complex,
                              void *workspace, size_t workspace_bytes, int64_t edge_capacity,
                              int32_t *adjacency /* (capacity) */, int32_t *adjacency_offsets /* (N+1) */,
                              int64_t *n_edges /* device */, int32_t *status /* device */, void *stream);

/* Steiner points (get_steiner_points, benchmark.py:93-180), the two steps
 * of a round that are not plumbing.  pf_steiner_knn: with a locator built
 * over the primitives (pf_locator_build), for each sample its k <= 32
 * nearest centres (scipy cKDTree.query in the reference; float64 distances
 * rounded to float32), the smallest dist - r over them -> sample_radius and
 * the primitive attaining it (first in distance order) -> closest.
 * pf_steiner_select: _greedy_min_overlap_fps (:93-134) from sample `seed`:
 * repeatedly select the sample with the smallest largest-overlap
 * (r_i + r_j - |p_i - p_j|) / (r_i + r_j) with the selected ones while it is
 * <= threshold; selected (n) gets 0/1, *n_selected (device, optional) the
 * count; scratch is n floats.  One block of 1024 threads. */
PF_API int pf_steiner_knn(const float *points, const float *radii, int64_t n_prims, const void *workspace,
                          const float *samples, int64_t n_samples, int32_t k, float *sample_radius,
                          int32_t *closest, int32_t *status, void *stream);
PF_API int pf_steiner_select(const float *samples, const float *radii, int64_t n, int64_t seed, float threshold,
                             float *scratch, uint8_t *selected, int32_t *n_selected, void *stream);

/* Spherical-Voronoi texel colour.  Replaces spherical_voronoi_fwd_kernel /
 * spherical_voronoi_bwd_kernel (powerfoam/color_fn.py:54-184): per point,
 * colour = max(sum_i w_i val_i / sum_i w_i + 0.5, 0) with
 * w_i = exp(-temp_i |normalize(p - origin) - axis_i|) over sv_dof sites, or
 * 0.5 grey (weight sum 0) when the direction is outside the camera cone
 * (dot(d, forward) < fov_cos_cutoff).  att_sites / att_values are
 * (sv_dof, N, 3), att_temps (sv_dof, N); f32, or f16 with attr_half = 1
 * (then value_out / weights_sum_out are f16 too).  The backward writes every
 * site gradient: zero where w / sum w < 1e-3 or outside the cone; the points
 * get no gradient (the reference's is disabled). */
PF_API int pf_sv_forward(const float *points, const float *camera_origin /* host, 3 */,
                         const float *camera_forward /* host, 3 */, float fov_cos_cutoff, const void *att_sites,
                         const void *att_values, const void *att_temps, int64_t n_points, int32_t sv_dof,
                         int32_t attr_half, void *value_out, void *weights_sum_out, void *stream);
PF_API int pf_sv_backward(const float *points, const float *camera_origin, const float *camera_forward,
                          float fov_cos_cutoff, const void *att_sites, const void *att_values, const void *att_temps,
                          const void *weights_sum, const void *values, const void *grad_values, int64_t n_points,
                          int32_t sv_dof, int32_t attr_half, void *grad_att_sites, void *grad_att_values,
                          void *grad_att_temps, void *stream);

/* Morton order of the primitives (stable on equal codes).  Replaces
 * morton_sort (powerfoam/geometry.py:7-85, Warp radix_sort_pairs). */
PF_API int pf_morton_workspace_size(int64_t n_prims, size_t *bytes);
PF_API int pf_morton_sort(const float *points, int64_t n_prims, void *workspace, size_t workspace_bytes,
                          int32_t *permutation, void *stream);

/* ---------------------------------------------------------------------- */
/* Differentiable rasterizer.  Replaces forward_kernel (rasterize.py:892-1146)
 * and the launch in Rasterizer._forward (:1795-1825).  adjacency_diff is the
 * pf_adjacency_prefetch encoding; attributes are f32.  Outputs (H,W[,3|Q]):
 * color, log_t, normal_distance, normal, quantile_depths (-1 where not
 * reached; NULL if no quantiles), err (the "surface" objective's per-pixel
 * expected squared error, rasterize.py:1076-1079, 1138-1141; NULL to skip);
 * contrib / point_err (N) (point_err may be NULL); early_stop (T) per-tile
 * stop index used by the backward; tile_contrib_pairs (T, optional) counts
 * the (tile, primitive) pairs in which at least one pixel composited. */
PF_API int pf_raster_forward(const pf_raster_inputs *in, int32_t return_point_err, float *color, float *log_t,
                      float *normal_distance, float *normal, float *quantile_depths, float *err, float *contrib,
                      float *point_err, int32_t *early_stop, int32_t *tile_contrib_pairs, void *stream);

/* Hand-written adjoint.  Replaces backward_kernel (rasterize.py:1150-1514) and
 * Rasterizer._backward (:1861-1980): dL/dlog_t = -dL/dopacity * exp(log_t),
 * gradients zeroed first and non-finite entries zeroed at the end.
 * grad_normal_distance / grad_normal / grad_quantile_depths / grad_contrib
 * may be NULL (treated as zero).  Outputs are written, not accumulated. */
PF_API int pf_raster_backward(const pf_raster_inputs *in, const int32_t *early_stop, const float *log_t,
                       const float *grad_color, const float *grad_opacity, const float *grad_normal_distance,
                       const float *grad_normal, const float *grad_quantile_depths, const float *grad_contrib,
                       float *grad_points, float *grad_radii, float *grad_normals, float *grad_density,
                       float *grad_texel_sites, float *grad_texel_rgb, float *grad_texel_height, void *stream);

/* Forward colour only.  Replaces benchmark_kernel (rasterize.py:614-734) as
 * launched by Rasterizer.benchmark (:2116-2131): adjacency_diff is the
 * pf_adjacency_power_diff encoding; attributes f32 or f16. */
PF_API int pf_raster_benchmark(const pf_raster_inputs *in, float *color, void *stream);

/* Viewer path, headless.  Replaces visualization_kernel (rasterize.py:738-888)
 * as launched by Rasterizer.visualize (:2133-2285). */
PF_API int pf_raster_visualize(const pf_raster_inputs *in, int32_t max_intersections, float depth_quantile,
                        float bkgd_r, float bkgd_g, float bkgd_b, float *color, float *depth, float *normal,
                        float *alpha, int32_t *intersections, void *stream);

/* ---------------------------------------------------------------------- */
/* Cell-walk ray tracer.  Replaces benchmark_kernel (powerfoam/raytrace.py:
 * 115-241) launched by RayTracer.benchmark (:247-309).  Adds: per-ray start
 * cells (start_cells, NULL = every ray starts at start_idx), a step cap
 * (PF_ERR_STEP_CAP in *status), depth / normal / log_t outputs and an
 * optional visited-cell log (visit_cap entries per ray, -1 padded). */
typedef struct pf_trace_inputs {
    pf_camera cam;
    int32_t n_sites;
    int32_t attr_half;
    int64_t n_prims;
    const float *spheres;
    const void *nsigmas;
    const void *texel_sites;
    const void *texel_rgb;
    const void *texel_height;
    const int32_t *adjacency;
    const int32_t *adjacency_offsets;
    const uint16_t *adjacency_diff;   /* pf_adjacency_power_diff encoding */
    int32_t start_idx;
    const int32_t *start_cells;       /* (H*W) or NULL */
    float transmittance_threshold;
    int32_t max_steps;
    float depth_quantile;
} pf_trace_inputs;

PF_API int pf_trace_forward(const pf_trace_inputs *in, float *color, float *log_t, float *depth, float *normal,
                     int32_t *depth_seg, float *depth_sigma, int32_t *visit_log, int32_t visit_cap,
                     int32_t *visit_count, int32_t *status, void *stream);

/* Adjoint of pf_trace_forward (no counterpart in the reference: its tracer
 * is forward-only).  Takes the forward's colour, normal, depth_seg and
 * depth_sigma and the upstream gradients of colour (H,W,3), log
 * transmittance (H,W), depth (H,W) and normal (H,W,3) (any of the four may
 * be NULL); writes (zeroes first) the gradients of every primitive attribute
 * and zeroes non-finite entries.  Attributes must be f32.  The walk is
 * repeated (transmittance recomputed, nothing kept from the forward); up to
 * segments_per_ray segments of each ray are recorded in the workspace
 * (256-byte aligned, pf_trace_backward_workspace_size bytes, about
 * 48 * segments_per_ray + 60 bytes per pixel) for the gradient launch, and
 * rays with more are finished by a launch that walks them on from there.
 * Any segments_per_ray in [0, 65535] gives the same gradients. */
PF_API int pf_trace_backward_workspace_size(const pf_trace_inputs *in, int32_t segments_per_ray, size_t *bytes);
PF_API int pf_trace_backward(const pf_trace_inputs *in, const float *color, const float *normal,
                             const int32_t *depth_seg, const float *depth_sigma, const float *grad_color,
                             const float *grad_log_t, const float *grad_depth, const float *grad_normal,
                             float *grad_points, float *grad_radii, float *grad_normals, float *grad_density,
                             float *grad_texel_sites, float *grad_texel_rgb, float *grad_texel_height,
                             int32_t segments_per_ray, void *workspace, size_t workspace_bytes, void *stream);

/* The walk of pf_trace_forward (f32 attributes, no visit log) that also
 * writes the adjoint's segment records into `workspace` (the layout and size
 * of pf_trace_backward_workspace_size for segments_per_ray): up to
 * segments_per_ray records per ray and the walk state of each ray with more.
 * pf_trace_backward_recorded then starts the adjoint from those records, so
 * the walk is not repeated.  No counterpart in the reference (its tracer has
 * no adjoint); outputs as pf_trace_forward. */
PF_API int pf_trace_forward_record(const pf_trace_inputs *in, float *color, float *log_t, float *depth, float *normal,
                                   int32_t *depth_seg, float *depth_sigma, int32_t *visit_count, int32_t *status,
                                   int32_t segments_per_ray, void *workspace, size_t workspace_bytes, void *stream);
/* pf_trace_backward without its walk: `workspace` holds the records that
 * pf_trace_forward_record wrote with the same inputs and segments_per_ray
 * (the workspace is only read).  Same arguments and gradients as
 * pf_trace_backward. */
PF_API int pf_trace_backward_recorded(const pf_trace_inputs *in, const float *color, const float *normal,
                                      const int32_t *depth_seg, const float *depth_sigma, const float *grad_color,
                                      const float *grad_log_t, const float *grad_depth, const float *grad_normal,
                                      float *grad_points, float *grad_radii, float *grad_normals,
                                      float *grad_density, float *grad_texel_sites, float *grad_texel_rgb,
                                      float *grad_texel_height, int32_t segments_per_ray, const void *workspace,
                                      size_t workspace_bytes, void *stream);

/* Training labels of the ray-proposal network (no counterpart in the
 * reference): the walk of pf_trace_forward (f32 attributes) writing, per
 * pixel ray, the colour and the first cell after whose compositing the
 * transmittance is below label_threshold: the t at which the ray enters it
 * (label_t), the cell (label_cell) and the cells walked before it
 * (label_step), all -1 when the transmittance never falls below the
 * threshold. */
PF_API int pf_trace_labels(const pf_trace_inputs *in, float label_threshold, float *color, float *label_t,
                           int32_t *label_cell, int32_t *label_step, int32_t *visit_count, int32_t *status,
                           void *stream);

/* Start cell of benchmark.py:320-324: argmin_i |p_i - eye|^2 - r_i^2 (first
 * index on ties).  workspace: pf_start_cell_workspace_size bytes. */
PF_API int pf_start_cell_workspace_size(int64_t n_prims, size_t *bytes);
PF_API int pf_start_cell(const float *points, const float *radii, int64_t n_prims, const float *eye_host,
                  void *workspace, size_t workspace_bytes, int32_t *out_idx, void *stream);

/* ---------------------------------------------------------------------- */
/* Point location in the power diagram: the cell containing x is
 * argmin_i |x - p_i|^2 - r_i^2 (the start-cell rule of benchmark.py:320-324
 * applied to any point; lowest index on ties).  pf_locator_build buckets the
 * primitives in a uniform grid kept in the caller's workspace
 * (pf_locator_workspace_size bytes); queries scan grid shells until no
 * unscanned primitive can win.  A query cut short by the shell cap raises
 * PF_ERR_SEED in *status.  No counterpart in the reference (its start cell
 * is a brute-force argmin for the camera eye only). */
PF_API int pf_locator_workspace_size(int64_t n_prims, size_t *bytes);
PF_API int pf_locator_build(const float *points, const float *radii, int64_t n_prims, void *workspace,
                            size_t workspace_bytes, void *stream);
PF_API int pf_locate_cells(const float *points, const float *radii, int64_t n_prims, const void *workspace,
                           const float *queries /* (n,3) */, int64_t n_queries, int32_t *cells, int32_t *status,
                           void *stream);
/* Proposal-seeded start cells for every pixel ray of `cam`: where
 * confidence >= conf_threshold and t_entry > 0 the cell containing
 * eye + t_entry * dir (the ray's walk then skips the cells before it), else
 * default_start.  *n_seeded (optional) accumulates the seeded rays. */
PF_API int pf_seed_start_cells(const float *points, const float *radii, int64_t n_prims, const void *workspace,
                               const pf_camera *cam, const float *t_entry, const float *confidence,
                               float conf_threshold, int32_t default_start, int32_t *start_cells,
                               int32_t *n_seeded, void *stream);

/* Point location by voxel map (no counterpart in the reference).
 * pf_voxel_map_build: for a res^3 grid of cubic voxels over the box
 * [box_lo, box_hi] (host, 3 floats each; edge max extent / res, res <= 1024),
 * the power cell of every voxel centre (pf_locate_cells' rule; workspace: a
 * built locator), cells (res^3) x-fastest; PF_ERR_SEED in *status (device,
 * optional) if a centre was not settled.  Once per scene.
 * pf_seed_start_cells_vmap: pf_seed_start_cells from the map: a seed point
 * starts at its voxel's cell and walks along the segment from the voxel
 * centre to the point across the power faces of `adjacency` (the tracer's
 * exit rule on exact float32 faces) until the segment ends in the current
 * cell; more than max_walk_steps crossings leave the ray unseeded.
 * pf_locate_cells_vmap: the same location for points (n,3); -1 where the
 * walk gave up. */
PF_API int pf_voxel_map_build(const float *points, const float *radii, int64_t n_prims, const void *workspace,
                              const float *box_lo, const float *box_hi, int32_t res, int32_t *cells, int32_t *status,
                              void *stream);
PF_API int pf_seed_start_cells_vmap(const float *points, const float *radii, int64_t n_prims,
                                    const int32_t *adjacency, const int32_t *adjacency_offsets, const int32_t *cells,
                                    const float *box_lo, const float *box_hi, int32_t res, const pf_camera *cam,
                                    const float *t_entry, const float *confidence, float conf_threshold,
                                    int32_t default_start, int32_t max_walk_steps, int32_t *start_cells,
                                    int32_t *n_seeded, void *stream);
PF_API int pf_locate_cells_vmap(const float *points, const float *radii, int64_t n_prims, const int32_t *adjacency,
                                const int32_t *adjacency_offsets, const int32_t *cells, const float *box_lo,
                                const float *box_hi, int32_t res, const float *queries, int64_t n_queries,
                                int32_t max_walk_steps, int32_t *out, void *stream);

/* Occupancy seeding (no counterpart in the reference): a conservative,
 * unlearned proposal.  pf_occupancy_build sets one bit per voxel of a res^3
 * grid over [box_lo, box_hi] (cubic voxels of the largest extent / res, bit
 * v = (z res + y) res + x) wherever the bounding box of a primitive with
 * density >= sigma_min (NaN counts), grown by one voxel, reaches; `bits` holds
 * pf_occupancy_words(res) words and is cleared first; a non-finite centre or
 * radius raises PF_ERR_NONFINITE in *status.  The walk composites only inside
 * spheres of density >= 1e-3 (raytrace.py:201-206), so with sigma_min <= 1e-3
 * a ray meets nothing before the first set voxel on its path.
 * pf_occupancy_entry: per pixel ray of `cam`, the distance at which it enters
 * the first set voxel (3-D DDA from where it enters the box), or the box exit
 * when it meets none, minus `margin`; confidence 1 where that skips part of
 * the ray, 0 where it does not (rays that miss the box or start in a set
 * voxel; t_entry -1 for a miss).  The two outputs are pf_seed_start_cells_vmap's
 * t_entry and confidence (threshold 0.5). */
PF_API int pf_occupancy_words(int32_t res, int64_t *words);
PF_API int pf_occupancy_build(const float *points, const float *radii, const float *density, int64_t n_prims,
                              const float *box_lo, const float *box_hi, int32_t res, float sigma_min, uint32_t *bits,
                              int32_t *status, void *stream);
PF_API int pf_occupancy_entry(const uint32_t *bits, const float *box_lo, const float *box_hi, int32_t res,
                              const pf_camera *cam, float margin, float *t_entry, float *confidence, void *stream);

/* ---------------------------------------------------------------------- */
/* Ray-proposal network (no counterpart in the reference): 6-frequency
 * positional encoding of (origin / 3, unit direction) -> 3 x 64 ReLU -> (entry
 * distance, confidence), BF16 tcgen05 GEMMs with FP32 accumulation in tensor
 * memory.  Parameters: pf_mlp_param_count() FP32 values, four row-major
 * (out x 80) matrices (64, 64, 64 and 16 rows; input column 78 of layer 1 and
 * 64 of layers 2-4 carry the bias, other pad columns and rows 2..15 of layer
 * 4 are zero); the kernels read a BF16 image of pf_mlp_image_bytes() bytes
 * that pf_mlp_pack (or pf_mlp_adam) writes.
 * pf_mlp_forward: rays (n,6) = origin, unit direction, or every pixel ray of
 *   `cam` when rays is NULL; writes t_entry (world units) and confidence.
 * pf_mlp_train_step: one minibatch of `batch` rays drawn (hashed with *step
 *   and seed) from rays (n,8) = origin, direction, label t (< 0: no label),
 *   no-hit flag (nonzero: the ray never reaches a significant cell and t is
 *   where it leaves the primitives' box); loss = asymmetric squared error of
 *   t / 6 (overshoot_weight on over-estimates of unflagged rays) +
 *   cross-entropy of the confidence against "seed is safe" (t >= 0 and either
 *   flagged or t_pred - margin <= t); ADDS the mean-loss gradient into grad and
 *   the loss sums into loss[0..1] (may be NULL).
 * pf_mlp_adam: Adam on the master weights, clears grad, writes the image and
 *   advances *step (done: a device word, zero before the first call).
 * pf_mlp_gemm_selftest: D (128 x 80 f32) = A (128 x 128) B^T (B 80 x 128),
 *   BF16 row-major inputs, through the tensor-core path with mode 0: both
 *   K-major, 1: B MN-major, 2: both MN-major (the three operand arrangements
 *   the network uses). */
PF_API int pf_mlp_param_count(void);
PF_API int pf_mlp_image_bytes(void);
PF_API int pf_mlp_pack(const float *weights, uint8_t *image, void *stream);
PF_API int pf_mlp_forward(const uint8_t *image, const float *rays, int64_t n_rays, const pf_camera *cam,
                          float *t_entry, float *confidence, int32_t *status, void *stream);
PF_API int pf_mlp_train_step(const uint8_t *image, const float *rays, int64_t n_rays, int32_t batch,
                             const int32_t *step, uint32_t seed, float overshoot_weight, float margin, float *grad,
                             float *loss, int32_t *status, void *stream);
PF_API int pf_mlp_adam(float *weights, float *m, float *v, float *grad, uint8_t *image, int32_t *step,
                       uint32_t *done, float lr, float beta1, float beta2, float eps, void *stream);
PF_API int pf_mlp_gemm_selftest(const uint16_t *a, const uint16_t *b, int32_t mode, float *d, int32_t *status,
                                void *stream);

/* ---------------------------------------------------------------------- */
/* Batched multi-view training step.  No counterpart in the reference, whose
 * scene renders one view per Rasterizer.forward call (scene.py:314-353).  For
 * every view: the forward of pf_raster_forward, the L2 loss
 * sum((color - target)^2), dL/dcolor = 2 (color - target) and the adjoint of
 * pf_raster_backward, with the gradients of all views summed into one set of
 * primitive gradients (texel_rgb gradients per view, since the colours are
 * per view).  A persistent launch takes (view, tile) work items from a
 * device queue, `chunk` items per pop, in the order `order` selects; fused
 * (split = 0), each tile's adjoint runs right after its own forward in the
 * same launch; split (split = 1), one persistent launch runs every tile's
 * forward and loss gradient, then a second every tile's adjoint.  Views are binned
 * beforehand with pf_bin at the batch's tile width (8, 16 or 32).  Nothing is
 * allocated and nothing synchronises, so the call can be captured in a CUDA
 * graph.  Images are bit-identical to pf_raster_forward per view; gradients
 * equal the sum of the per-view pf_raster_backward results up to the order of
 * the float additions. */
#define PF_BATCH_MAX_VIEWS 64
#define PF_BATCH_ORDER_LONGEST 0 /* all views' tiles by decreasing list length */
#define PF_BATCH_ORDER_VIEW 1    /* view by view, tiles in index order */

typedef struct pf_batch_scene {
    int32_t n_sites;
    int64_t n_prims;
    const float *spheres;              /* (N,4) */
    const float *nsigmas;              /* (N,4) */
    const float *texel_sites;          /* (N,S,3) */
    const float *texel_height;         /* (N,S) */
    const int32_t *adjacency;          /* (E) */
    const int32_t *adjacency_offsets;  /* (N+1) */
    const uint16_t *adjacency_diff;    /* (E,4) pf_adjacency_prefetch encoding */
    float transmittance_threshold;
    /* optional segment records (tile widths 8 and 16), as
     * pf_raster_inputs.segments: the forward launch writes them, the adjoint
     * reads them; the masks and offsets of view v start at its
     * segment_pair_base (in pairs).  The views render in record groups
     * (pf_batch_view.segment_group: 0 for the first view, then the previous
     * view's group or the next one), one group after the other, each reusing
     * the record buffer with its own counter: segment_count holds one int64
     * per group (the last view's group + 1), zeroed by the call */
    float *segments;
    uint32_t *segment_masks;
    int32_t *segment_offsets;
    int64_t *segment_count;
    int64_t segment_capacity;          /* records (< 2^31) */
    int32_t segment_planes;            /* 1: records hold the plane results */
} pf_batch_scene;

typedef struct pf_batch_view {
    pf_camera cam;
    const int64_t *tile_offsets;   /* (T+1) from pf_bin at the batch tile width */
    const int32_t *tile_prims;
    const float *texel_rgb;        /* (N,S,3) this view's texel colours */
    const float *target;           /* (H,W,3) */
    float *color;                  /* (H,W,3) */
    float *log_t;                  /* (H,W) */
    float *normal_distance;        /* (H,W) */
    float *normal;                 /* (H,W,3) */
    float *grad_color;             /* (H,W,3) written: 2 (color - target) */
    float *contrib;                /* (N); views may share one array (summed) */
    int32_t *early_stop;           /* (T) */
    int32_t *tile_contrib_pairs;   /* (T) or NULL */
    float *grad_texel_rgb;         /* (N,S,3); views may share one array (summed) */
    int64_t segment_pair_base;     /* with segments: the view's first pair in the mask / offset arrays */
    int64_t segment_pairs;         /* its pairs there (>= the pairs in tile_prims) */
    int32_t segment_group;         /* with segments: its record group (see pf_batch_scene) */
} pf_batch_view;

/* tile_loss holds one float per tile of every view, the views' tiles
 * concatenated in view order: the loss of view v is the sum of its slice. */
PF_API int pf_batch_workspace_size(const pf_batch_view *views, int32_t n_views, int32_t tile_width, size_t *bytes);
PF_API int pf_batch_render(const pf_batch_scene *scene, const pf_batch_view *views, int32_t n_views,
                           int32_t tile_width, int32_t chunk, int32_t order,
                           int32_t split /* 0: one fused launch; 1: a forward launch, then an adjoint launch */,
                           void *workspace, size_t workspace_bytes,
                           float *tile_loss, float *grad_points, float *grad_radii, float *grad_normals,
                           float *grad_density, float *grad_texel_sites, float *grad_texel_height,
                           int32_t *status, void *stream);

/* Schedule tuner for pf_batch_render at one tile width (the views binned at
 * that width): for each candidate, `warmup` untimed calls, then `iters` calls
 * timed with CUDA events on `stream`; writes each candidate's mean ms and the
 * index of the fastest into *best.  The host waits for every candidate's
 * events (not capturable); the outputs hold the last call's results.  The
 * tile width itself is swept by the caller, which bins the views at each
 * width (powerfoam_b200/batch.py autotune). */
typedef struct pf_batch_schedule {
    int32_t chunk;
    int32_t order; /* PF_BATCH_ORDER_* */
    int32_t split;
    float ms;      /* written */
} pf_batch_schedule;

PF_API int pf_batch_autotune(const pf_batch_scene *scene, const pf_batch_view *views, int32_t n_views,
                             int32_t tile_width, pf_batch_schedule *candidates, int32_t n_candidates,
                             int32_t warmup, int32_t iters, void *workspace, size_t workspace_bytes,
                             float *tile_loss, float *grad_points, float *grad_radii, float *grad_normals,
                             float *grad_density, float *grad_texel_sites, float *grad_texel_height,
                             int32_t *status, int32_t *best, void *stream);

/* ---------------------------------------------------------------------- */
/* Texel colour pre-step for the synthetic scenes: degree-3 real SH (16
 * coefficients per channel, constants of powerfoam/sh_utils.py:4-50) at
 * normalize(p - eye), + 0.5, clamped at 0, broadcast to the S sites.
 * Stands where the reference evaluates its per-view colour function
 * (scene.py:331-335 / benchmark.py:390-399). */
PF_API int pf_sh_texel_rgb(const float *points, const float *sh /* (N,16,3) */, int64_t n_prims, int32_t n_sites,
                    const float *eye_host, float *texel_rgb, void *stream);
/* Adjoint of pf_sh_texel_rgb with respect to the coefficients: ADDS
 * basis(dir) * sum_s dL/dtexel_rgb[s] into grad_sh (N,16,3) wherever the
 * pre-clamp colour is positive (no gradient reaches the points through the
 * view direction).  Successive calls for several views accumulate. */
PF_API int pf_sh_texel_rgb_backward(const float *points, const float *sh, int64_t n_prims, int32_t n_sites,
                                    const float *eye_host, const float *grad_texel_rgb, float *grad_sh,
                                    void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PFOAM_H */

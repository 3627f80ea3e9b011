/*
 * tg2dgs.h -- C ABI of the B200 textured 2DGS rasterization path.
 *
 * Plain pointers and sizes only.  Every buffer (inputs, outputs, workspace) is
 * allocated and owned by the caller; every entry point enqueues work on the
 * given CUDA stream and returns 0 on success or a negative TG_ERR_* code (the
 * message is available from tg_last_error()).  Entry points are safe to call
 * concurrently from several host threads on distinct streams.
 *
 * Each entry point names the reference interface it replaces (paths inside the
 * Camak2441/textured_gaussians project).
 */
#ifndef TG2DGS_H
#define TG2DGS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* tg_stream_t; /* same type as cudaStream_t */

#if defined(__GNUC__)
#define TG_API __attribute__((visibility("default")))
#else
#define TG_API
#endif

#define TG_OK 0
#define TG_ERR_INVALID_ARG (-1)   /* null pointer, bad size, misaligned buffer */
#define TG_ERR_UNSUPPORTED (-2)   /* channel count / texture format / tile size (8, 16, 32) not supported */
#define TG_ERR_CUDA (-3)          /* a CUDA launch or runtime call failed */
#define TG_ERR_WORKSPACE (-4)     /* workspace smaller than tg_sort_workspace_bytes() */
#define TG_ERR_TIMEOUT (-5)       /* a bounded device-side wait gave up */

/* texture storage formats (textures are [G, ry, rx, 4] RGBA texels) */
#define TG_TEX_NONE 0  /* plain 2DGS compositor, no textures */
#define TG_TEX_F32 1
#define TG_TEX_BF16 2
#define TG_TEX_F16 3
#define TG_TEX_FP8_E4M3 4 /* plus one float scale per Gaussian: texel = fp8 * scale */

/* compositor adjoint forms */
#define TG_ADJ_REFERENCE 0 /* "bilinear": texture lookup not differentiated w.r.t. geometry */
#define TG_ADJ_BWD2 1      /* "bilinear_bwd2": reference UV term (du/ds factor (R-1)/range) */
#define TG_ADJ_EXACT 2     /* exact derivative of the forward ((R-1)/(2*range)) */

/* Texture filters of the compositor (tg_raster_fwd_args.filter).  mipmapped2
 * is selected by mip_levels > 0 (filter 0 or TG_FILTER_MIPMAPPED2). */
#define TG_FILTER_BILINEAR 0
#define TG_FILTER_MIPMAPPED2 1
#define TG_FILTER_ANISO_BILINEAR 2

/* ------------------------------------------------------------------ batching form
 * Views of uneven size in one call (no counterpart in the reference, which
 * renders C cameras of one size per call).  A batch of C views is described by
 * a device array tg_view[C]; the tiles of all views form one flat list (view c
 * owns tiles [tile_base, tile_base + tile_width*tile_height), row-major), and
 * the per-pixel outputs are flat over all views (view c owns pixels
 * [pix_base, pix_base + width*height), row-major).  tile_view[t] is the view of
 * flat tile t.  Kernels bounds-check every pixel and tile index against the
 * totals passed beside the table. */
typedef struct {
    int32_t width, height;           /* image size of the view */
    int32_t tile_width, tile_height; /* its tile grid: ceil(width / tile_size), ceil(height / tile_size) */
    int64_t tile_base;               /* first flat tile of the view */
    int64_t pix_base;                /* first flat pixel of the view */
} tg_view;

TG_API int tg_version(void);
TG_API const char* tg_last_error(void);
/* Number of kernels this library has launched in this process (all devices,
 * all threads); lets a harness count the launches inside a timed region.
 * No counterpart in the reference. */
TG_API uint64_t tg_kernel_launch_count(void);

/* ------------------------------------------------------------------ projection
 * Replaces fully_fused_projection_fwd_2dgs_tensor
 * (textured_gaussians/cuda/csrc/fully_fused_projection_2dgs_fwd.cu:247-304).
 * All float arrays are FP32, row-major.  Entries that are culled get radii 0
 * and zeros elsewhere. */
typedef struct {
    int32_t C, N;
    const float* means;    /* [N,3] */
    const float* quats;    /* [N,4] wxyz, not necessarily normalised */
    const float* scales;   /* [N,3] (third unused) */
    const float* viewmats; /* [C,4,4] world-to-camera */
    const float* Ks;       /* [C,3,3] */
    int32_t width, height;
    float near_plane, far_plane, radius_clip;
    int32_t* radii;        /* [C,N] */
    float* means2d;        /* [C,N,2] */
    float* depths;         /* [C,N] */
    float* ray_transforms; /* [C,N,3,3] rows of K*[R*s0*q0, R*s1*q1, mean_c] */
    float* normals;        /* [C,N,3] */
    /* Fused SH colours (sh_coeffs NULL: not computed), replacing the
     * reference's spherical_harmonics + clamp glue (rendering.py:1573-1583):
     * colors[c,n] = max(SH(sh_degree, mean_n - centre_c) + 0.5, 0) for visible
     * entries, 0.5 elsewhere; centre_c = -R_c^-1 t_c from viewmats[c]. */
    int32_t sh_degree, sh_K;     /* degree <= 4, (degree+1)^2 <= K */
    const float* sh_coeffs;      /* [N,K,3] */
    float* colors;               /* [C,N,3] */
} tg_project_fwd_args;
TG_API int tg_project_fwd(const tg_project_fwd_args* a, tg_stream_t stream);

/* Replaces fully_fused_projection_bwd_2dgs_tensor / fully_fused_projection_bwd2_2dgs_tensor
 * (textured_gaussians/cuda/csrc/fully_fused_projection_2dgs_bwd.cu:150-222, ..._bwd2.cu).
 * mode: 0 reference, 1 norm_rot_grad (bwd2), 2 exact.  v_means/v_quats/v_scales
 * are overwritten (zeroed, then accumulated). */
typedef struct {
    int32_t C, N;
    const float* means;
    const float* quats;
    const float* scales;
    const float* viewmats;
    const float* Ks;
    const int32_t* radii;          /* [C,N] */
    const float* ray_transforms;   /* [C,N,9] */
    const float* v_means2d;        /* [C,N,2] */
    const float* v_depths;         /* [C,N] */
    const float* v_normals;        /* [C,N,3] */
    const float* v_ray_transforms; /* [C,N,9] */
    int32_t mode;
    float* v_means;  /* [N,3] */
    float* v_quats;  /* [N,4] */
    float* v_scales; /* [N,3] */
    /* Fused SH adjoint (sh_coeffs NULL: none): v_colors [C,N,3] in;
     * v_sh_coeffs [N,K,3] out (overwritten); the direction's gradient is
     * added into v_means. */
    int32_t sh_degree, sh_K;
    const float* sh_coeffs;
    const float* v_colors;
    float* v_sh_coeffs;
} tg_project_bwd_args;
TG_API int tg_project_bwd(const tg_project_bwd_args* a, tg_stream_t stream);

/* ------------------------------------------------------------------ packed projection
 * Replaces fully_fused_projection_packed_fwd_2dgs_tensor
 * (textured_gaussians/cuda/csrc/fully_fused_projection_packed_2dgs_fwd.cu:232-324),
 * split at the one host synchronisation the reference also has (:274-275):
 * tg_project_packed_count projects every (camera, Gaussian), counts the visible
 * entries, and writes their total *nnz (device int64) and indptr[C+1]; the
 * caller reads nnz, allocates the packed outputs and calls
 * tg_project_packed_emit with the same arguments plus nnz_host and the output
 * pointers.  Entries are ordered by camera, then Gaussian.  C <= 65535 and
 * nnz < 2^31 (indptr is int32, as in the reference).  Each camera uses its own
 * intrinsics Ks[c], as the dense forward and the packed backward do (the
 * reference's packed forward reads Ks[0] for every camera, :103). */
typedef struct {
    int32_t C, N;
    const float* means;    /* [N,3] */
    const float* quats;    /* [N,4] */
    const float* scales;   /* [N,3] */
    const float* viewmats; /* [C,4,4] */
    const float* Ks;       /* [C,3,3] */
    int32_t width, height;
    float near_plane, far_plane, radius_clip;
    void* workspace;        /* tg_project_packed_workspace_bytes(C, N) bytes, kept between the two calls */
    int64_t* nnz;           /* [1] device, written by count */
    int32_t* indptr;        /* [C+1], written by count */
    int64_t nnz_host;       /* emit: the value of *nnz */
    int64_t* camera_ids;    /* [nnz] (emit) */
    int64_t* gaussian_ids;  /* [nnz] (emit) */
    int32_t* radii;         /* [nnz] (emit) */
    float* means2d;         /* [nnz,2] (emit) */
    float* depths;          /* [nnz] (emit) */
    float* ray_transforms;  /* [nnz,3,3] (emit) */
    float* normals;         /* [nnz,3] (emit) */
    /* Batching form (NULL / 0 otherwise): camera c projects only Gaussians
     * [gauss_ranges[2c], gauss_ranges[2c+1]) (its scene inside the concatenated
     * Gaussian arrays; max_range = the longest range) onto an image of
     * views[c].width x views[c].height.  N is then the total Gaussian count. */
    const tg_view* views;         /* [C] or NULL */
    const int64_t* gauss_ranges;  /* [C,2] or NULL */
    int32_t max_range;
    /* Capacity mode (overflow != NULL, for CUDA-graph capture): nnz_host is the
     * capacity of the output arrays rather than *nnz; emit zeroes all of them
     * (radii 0: the unused tail intersects nothing; its Gaussian ids are spread
     * over [0, N) so gathers over the tail do not collide), writes the first
     * min(*nnz, capacity) entries and sets *overflow to 1 if *nnz > capacity.
     * The caller zeroes *overflow. */
    uint32_t* overflow;
    /* Fused SH colours as in tg_project_fwd_args (emit): colors [nnz,3]. */
    int32_t sh_degree, sh_K;
    const float* sh_coeffs;
    float* colors;
} tg_project_packed_args;
TG_API size_t tg_project_packed_workspace_bytes(int32_t C, int32_t N);
TG_API int tg_project_packed_count(const tg_project_packed_args* a, tg_stream_t stream);
TG_API int tg_project_packed_emit(const tg_project_packed_args* a, tg_stream_t stream);

/* Replaces fully_fused_projection_packed_bwd_2dgs_tensor / fully_fused_projection_packed_bwd2_2dgs_tensor
 * (textured_gaussians/cuda/csrc/fully_fused_projection_packed_2dgs_bwd.cu:172-266, ..._bwd2.cu).
 * One thread per packed entry; mode as in tg_project_bwd.  sparse_grad = 1:
 * v_means [nnz,3], v_quats [nnz,4], v_scales [nnz,3] hold each entry's own
 * gradient (overwritten).  sparse_grad = 0: they are [N,...] and hold the sum
 * over each Gaussian's entries (zeroed, then accumulated with atomics).
 * Entries whose camera or Gaussian id is out of range are skipped. */
typedef struct {
    int32_t C, N;
    int64_t nnz;
    const float* means;
    const float* quats;
    const float* scales;
    const float* viewmats;
    const float* Ks;
    const int64_t* camera_ids;     /* [nnz] */
    const int64_t* gaussian_ids;   /* [nnz] */
    const float* ray_transforms;   /* [nnz,9] */
    const float* v_means2d;        /* [nnz,2] */
    const float* v_depths;         /* [nnz] */
    const float* v_normals;        /* [nnz,3] */
    const float* v_ray_transforms; /* [nnz,9] */
    int32_t mode, sparse_grad;
    float* v_means;
    float* v_quats;
    float* v_scales;
    /* Fused SH adjoint as in tg_project_bwd_args: v_colors [nnz,3] in;
     * v_sh_coeffs [N,K,3] out (zeroed, then accumulated with atomics); the
     * direction's gradient is added into v_means (the entry's row when
     * sparse_grad). */
    int32_t sh_degree, sh_K;
    const float* sh_coeffs;
    const float* v_colors;
    float* v_sh_coeffs;
} tg_project_packed_bwd_args;
TG_API int tg_project_packed_bwd(const tg_project_packed_bwd_args* a, tg_stream_t stream);

/* ------------------------------------------------------------------ tile intersection
 * Replaces isect_tiles_tensor (textured_gaussians/cuda/csrc/isect_tiles.cu:107-307),
 * split at the one host synchronisation the reference also has (:200-201):
 * tg_isect_count writes tiles_per_gauss, the inclusive prefix sum cum_tiles and
 * the total *n_isects (device scalar); tg_isect_emit then writes the unsorted
 * keys cam<<(32+tile_bits) | tile<<32 | bits(depth) and flatten ids. */
typedef struct {
    int64_t n_elems;            /* C*N dense, nnz packed */
    int64_t N;                  /* dense: Gaussians per camera; packed: 0 */
    const int64_t* camera_ids;  /* packed: [nnz]; dense: NULL */
    const float* means2d;       /* [n_elems,2] */
    const int32_t* radii;       /* [n_elems] */
    const float* depths;        /* [n_elems] */
    int32_t tile_size, tile_width, tile_height, n_cameras;
    int32_t* tiles_per_gauss;   /* [n_elems] */
    int64_t* cum_tiles;         /* [n_elems] inclusive prefix sum */
    int64_t* n_isects;          /* [1] device */
    void* scan_workspace;       /* tg_scan_workspace_bytes(n_elems) bytes */
    int64_t* isect_ids;         /* [n_isects] (emit only) */
    int32_t* flatten_ids;       /* [n_isects] (emit only) */
    /* Batching form: per-camera tile grids (tile_width/tile_height above are
     * then the largest grid's, which sets the tile bits of the keys); tile ids
     * in the keys are local to the camera.  NULL: one grid for all cameras. */
    const tg_view* views;       /* [n_cameras] or NULL */
    /* Capacity mode (overflow != NULL; for CUDA-graph capture, where the count
     * cannot be read back between the two calls): isect_ids / flatten_ids hold
     * `capacity` entries, emit writes the first min(*n_isects, capacity),
     * sets *overflow to 1 if *n_isects > capacity, and fills the rest of the
     * keys with 2^(32+tile_bits+camera_bits) - 1, which sorts after every real
     * key.  The caller zeroes *overflow. */
    int64_t capacity;
    uint32_t* overflow;
} tg_isect_args;
TG_API size_t tg_scan_workspace_bytes(int64_t n_elems);
TG_API int tg_isect_count(const tg_isect_args* a, tg_stream_t stream);
TG_API int tg_isect_emit(const tg_isect_args* a, tg_stream_t stream);

/* Stable LSD onesweep radix sort of (int64 key, int32 value) pairs on key bits
 * [0, end_bit), ping-ponging between (keys, vals) and (keys_alt, vals_alt).
 * Replaces cub::DeviceRadixSort::SortPairs as called at
 * textured_gaussians/cuda/csrc/isect_tiles.cu:246-300.  *result_in_alt (host
 * int) is set to 1 when the sorted data ends in the *_alt buffers. */
TG_API size_t tg_sort_workspace_bytes(int64_t n, int32_t end_bit);
TG_API int tg_sort_pairs(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n, int32_t end_bit,
                  void* workspace, size_t workspace_bytes, int32_t* result_in_alt, tg_stream_t stream);

/* Waits for `stream`, then reports whether any bounded look-back wait of the
 * last tg_sort_pairs call that used `workspace` (with the same n and end_bit)
 * gave up: TG_ERR_TIMEOUT if so, TG_OK otherwise.  Synchronising; for
 * diagnostics and tests.  No counterpart in the reference. */
TG_API int tg_sort_status(const void* workspace, int64_t n, int32_t end_bit, tg_stream_t stream);

/* Diagnostic self-test of the sort's bounded waits (no counterpart in the
 * reference): one pass over 8192 pairs (8 key bits) of keys/vals into
 * keys_alt/vals_alt, run by a single CTA that is made to wait for a
 * predecessor tile that never publishes.  The wait gives up after its poll
 * limit (about a second), raises the error flag and the kernel returns; the
 * call then synchronises and returns TG_ERR_TIMEOUT -- the expected outcome --
 * with the CUDA context still usable.  workspace: tg_sort_workspace_bytes(8192, 8). */
TG_API int tg_sort_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt,
                                     void* workspace, size_t workspace_bytes, tg_stream_t stream);

/* The same sort, for callers that cannot allocate device memory (a plugin host
 * that owns all GPU memory, a real-time loop that must not call cudaMalloc, a
 * host without a caching allocator).  No counterpart in the reference.  The
 * caller passes only keys, values and their ping-pong buffers; the scratch the
 * sort needs lives in a static device array of this library (8 MiB + 16 KiB
 * held on every GPU that loads it, until exit), so n is limited to
 * TG_SORT_NOALLOC_MAX_PAIRS -- larger n is rejected with TG_ERR_INVALID_ARG.
 * Calls share that array: those that overlap on one GPU race and must be
 * serialised by the caller.  The first call on a device looks up the array's
 * address with that device current; make it before any stream capture (the
 * address is looked up again if the device's context has changed since). */
#define TG_SORT_NOALLOC_MAX_PAIRS 4194304
TG_API int tg_sort_pairs_noalloc(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n,
                                 int32_t end_bit, int32_t* result_in_alt, tg_stream_t stream);

/* Waits for `stream`, then reports whether a bounded look-back wait of the last
 * tg_sort_pairs_noalloc call on the current device gave up: TG_ERR_TIMEOUT if
 * so, TG_OK otherwise (the flag lives in the static scratch and is cleared by
 * every call).  Synchronising; for diagnostics and tests.  No counterpart in
 * the reference. */
TG_API int tg_sort_noalloc_status(tg_stream_t stream);

/* tg_sort_lookback_selftest run on the static scratch of tg_sort_pairs_noalloc
 * (8192 pairs of keys/vals into keys_alt/vals_alt): returns TG_ERR_TIMEOUT by
 * design, and leaves the flag set for tg_sort_noalloc_status until the next
 * sort.  No counterpart in the reference. */
TG_API int tg_sort_noalloc_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt,
                                             tg_stream_t stream);

/* Replaces isect_offset_encode_tensor (textured_gaussians/cuda/csrc/isect_tiles.cu:357-390):
 * offsets[c,ty,tx] = index of the first sorted intersection of tile (c,ty,tx)
 * or of the next non-empty tile. */
TG_API int tg_isect_offset_encode(const int64_t* isect_ids, int64_t n_isects, int32_t n_cameras, int32_t tile_width,
                           int32_t tile_height, int32_t* offsets, tg_stream_t stream);

/* Batching form of tg_isect_offset_encode: offsets[t] for every flat tile t of
 * the views (n_tiles in total, tile_view[t] its view); max_tiles_per_view sets
 * the tile bits of the keys, as in tg_isect_args.  No counterpart in the
 * reference. */
TG_API int tg_isect_offset_encode_views(const int64_t* isect_ids, int64_t n_isects, int32_t n_cameras,
                                        int64_t max_tiles_per_view, const tg_view* views, const int32_t* tile_view,
                                        int64_t n_tiles, int32_t* offsets, tg_stream_t stream);

/* ------------------------------------------------------------------ compositor
 * Replaces rasterize_to_pixels_fwd_textured_gaussians_tensor
 * (textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_gaussians_2dgs_fwd.cu:618-690)
 * and, with tex_format TG_TEX_NONE, rasterize_to_pixels_fwd_2dgs_tensor
 * (textured_gaussians/cuda/csrc/rasterize_to_pixels_2dgs_fwd.cu:566-631).
 * Element arrays are [E,...] with E = C*N (dense) or nnz (packed).  The
 * texture row of element e is gaussian_ids[e] when gaussian_ids != NULL
 * (packed) and e % N otherwise. */
typedef struct {
    int32_t C, N, D;            /* cameras, Gaussians, colour channels (1..5) */
    int32_t width, height, tile_size, tile_width, tile_height;
    int64_t n_isects;
    const float* means2d;       /* [E,2] */
    const float* ray_transforms;/* [E,9] */
    const float* colors;        /* [E,D] */
    const float* opacities;     /* [E] */
    const float* normals;       /* [E,3] */
    int32_t tex_format;         /* TG_TEX_* */
    const void* textures;       /* [G,ry,rx,4] in tex_format */
    const float* tex_scales;    /* [G] (fp8 only) */
    int32_t tex_ry, tex_rx;
    float range_x, range_y;
    const float* backgrounds;   /* [C,D] or NULL */
    const uint8_t* masks;       /* [C,tile_height,tile_width] or NULL */
    const int32_t* tile_offsets;/* [C,tile_height,tile_width] */
    const int32_t* flatten_ids; /* [n_isects] */
    const int64_t* gaussian_ids;/* [E] or NULL */
    float contrib_threshold, g_weight;
    int32_t n_contrib;          /* length of contrib_sum/count (N, or G when packed) */
    float* out_colors;          /* [C,H,W,D] */
    float* out_alphas;          /* [C,H,W] */
    float* out_normals;         /* [C,H,W,3] */
    float* out_distort;         /* [C,H,W] */
    float* out_median;          /* [C,H,W] */
    int32_t* last_ids;          /* [C,H,W] */
    int32_t* median_ids;        /* [C,H,W] */
    float* contrib_sum;         /* [n_contrib] (zeroed by the call) */
    float* contrib_count;       /* [n_contrib] (zeroed by the call) */
    /* Work order and batching form (all NULL / 0 for one image size in CTA order).
     * tile_order: [n tiles] permutation giving the order in which tiles are
     * taken (e.g. heaviest first), or NULL.  views / tile_view: the view table
     * above; tile_offsets and masks are then [n_tiles] over the flat tile list,
     * the per-pixel outputs [n_pixels, ...] over the flat pixels, backgrounds
     * [C,D], and width/height/tile_width/tile_height are ignored. */
    const int32_t* tile_order;
    const tg_view* views;
    const int32_t* tile_view;
    int64_t n_tiles, n_pixels;
    /* Capacity mode: device count of valid intersections (flatten_ids then
     * holds n_isects >= *n_isects_dev entries, the tail unused), or NULL. */
    const int64_t* n_isects_dev;
    /* Splats staged in shared memory per batch: 0 = tile_size^2 (the
     * reference's batch), else a multiple of 32 up to 1024. */
    int32_t batch_depth;
    /* Persistent launch: one device uint32 the call zeroes; a grid of as many
     * CTAs as fit on the device takes work items (tiles, in tile_order) from
     * it until none is left.  NULL: one CTA per work item. */
    uint32_t* work_queue;
    /* The mipmapped2 filter (mip_levels = L > 0; rasterize_to_pixels_mip2_
     * textured_gaussians_2dgs_fwd.cu of the reference): textures are 2^L x 2^L (L <= 13)
     * (tex_ry = tex_rx = 2^L) and tex_coarse holds their coarser levels,
     * [G, (4^L - 1) / 3, 4] FP32 in the reference's pyramid order (coarsest
     * first, as made by tg_generate_mipmap); level 0 is read from `textures`.
     * Supported with F32 / BF16 storage, 3 or 4 channels, tile 8 or 16, no
     * persistent launch, and the reference adjoint. */
    int32_t mip_levels;
    const float* tex_coarse;
    /* TG_FILTER_ANISO_BILINEAR: the anisotropic_bilinear filter
     * (rasterize_to_pixels_aniso_bilinear_textured_gaussians_2dgs_{fwd,bwd}.cu
     * of the reference): each pixel's footprint quad in texel space integrates
     * the bilinear interpolant (cell by cell, or along the footprint's boundary
     * when aniso_prefix is given).  Same support as mipmapped2
     * (F32 / BF16 storage, 3 or 4 channels, tile 8 or 16, one CTA per tile,
     * reference adjoint). */
    int32_t filter;
    /* Transmittance checkpoints (NULL: none; no counterpart in the reference,
     * whose adjoint recovers each splat's transmittance by dividing the final
     * one by (1 - alpha) back to front, rasterize_to_pixels_textured_gaussians_
     * 2dgs_bwd.cu:160, :456-457).  When set, the forward writes every pixel's
     * transmittance at the end of each batch of its tile, and the adjoint,
     * given the same pointer, restarts the division from that exact value at
     * every batch, so rounding accumulates over one batch of splats instead of
     * the whole list.  FP32, [n_tiles + n_isects / bs + 1, tile_size^2] with
     * bs the batch depth (tile_size^2 when batch_depth is 0); row
     * t + tile_offsets[t] / bs + k holds batch k of tile t. */
    float* t_checkpoints;
    /* TG_FILTER_ANISO_BILINEAR only: the row-prefix table of the textures,
     * [G,ry,rx,4] FP32 as made by tg_aniso_prefix, or NULL.  When set, a
     * footprint whose corner rays meet the splat plane on one side (a convex
     * quad) is integrated along its boundary (Green's theorem over the rows'
     * prefix integrals: work in proportion to its perimeter in texel cells)
     * instead of cell by cell as the reference does; the same integral up to
     * FP32 rounding.  No counterpart in the reference. */
    const float* aniso_prefix;
    /* With aniso_prefix: records of the footprint integrals the forward
     * computes, per pixel in the order it computes them: aniso_records
     * [n_pixels, aniso_record_cap, 4] FP32 (the first aniso_record_cap of
     * each pixel's) and aniso_record_count [n_pixels] int32 (how many of them
     * the pixel had up to its last contributor).  Given the same pointers the
     * adjoint reads these integrals instead of integrating the footprints
     * again (those past the capacity it integrates again).  NULL / 0: none.
     * No counterpart in the reference. */
    float* aniso_records;
    int32_t* aniso_record_count;
    int32_t aniso_record_cap;
} tg_raster_fwd_args;
TG_API int tg_rasterize_fwd(const tg_raster_fwd_args* a, tg_stream_t stream);

/* Replaces rasterize_to_pixels_bwd_textured_gaussians_tensor
 * (textured_gaussians/cuda/csrc/rasterize_to_pixels_textured_gaussians_2dgs_bwd.cu:890-984),
 * the bwd2 variant (..._bwd2.cu) and rasterize_to_pixels_bwd_2dgs_tensor
 * (textured_gaussians/cuda/csrc/rasterize_to_pixels_2dgs_bwd.cu).  All
 * gradient outputs are zeroed by the call, then accumulated.  v_densify is
 * written after the accumulation completes. */
typedef struct {
    tg_raster_fwd_args f;        /* forward inputs (output pointers unused) */
    const float* render_colors;  /* [C,H,W,D] forward outputs */
    const float* render_alphas;  /* [C,H,W] */
    const int32_t* last_ids;     /* [C,H,W] */
    const int32_t* median_ids;   /* [C,H,W] */
    const float* v_render_colors;  /* [C,H,W,D] */
    const float* v_render_alphas;  /* [C,H,W] */
    const float* v_render_normals; /* [C,H,W,3] */
    const float* v_render_distort; /* [C,H,W] */
    const float* v_render_median;  /* [C,H,W] */
    int32_t adjoint;             /* TG_ADJ_* */
    int64_t n_elems;             /* E */
    float* v_means2d;            /* [E,2] */
    float* v_means2d_abs;        /* [E,2] or NULL */
    float* v_ray_transforms;     /* [E,9] */
    float* v_colors;             /* [E,D] */
    float* v_opacities;          /* [E] */
    float* v_normals;            /* [E,3] */
    float* v_textures;           /* [G,ry,rx,4] FP32 or NULL */
    float* v_densify;            /* [E,2] */
    float* v_tex_coarse;         /* mipmapped2: [G, (4^L - 1) / 3, 4] gradient of tex_coarse (zeroed by the call) */
    /* anisotropic_bilinear with f.aniso_prefix set and v_textures requested:
     * [G,ry,rx,4] FP32 scratch for the gradient of the row-prefix table; the
     * call zeroes it and folds it into v_textures after the accumulation. */
    float* v_aniso_prefix;
} tg_raster_bwd_args;
TG_API int tg_rasterize_bwd(const tg_raster_bwd_args* a, tg_stream_t stream);

/* ------------------------------------------------------------------ spherical harmonics
 * Replaces compute_sh_fwd_tensor / compute_sh_bwd_tensor
 * (textured_gaussians/cuda/csrc/compute_sh_fwd.cu, compute_sh_bwd.cu).
 * colors[i,3] = sum_k basis_k(normalize(dirs[i])) coeffs[i % coeff_rows,k,:]
 * for i < n; masked-out elements are written as zeros.  coeff_rows < n lets
 * C cameras share one [N,K,3] coefficient table without materialising C
 * copies (n = C*N, coeff_rows = N).  Backward overwrites v_coeffs
 * ([coeff_rows,K,3], summed over the elements sharing a row, deterministic)
 * and, if non-NULL, v_dirs ([n,3]). */
TG_API int tg_sh_fwd(int64_t n, int64_t coeff_rows, int32_t degree, int32_t K, const float* dirs, const float* coeffs,
                     const uint8_t* masks, float* colors, tg_stream_t stream);
TG_API int tg_sh_bwd(int64_t n, int64_t coeff_rows, int32_t degree, int32_t K, const float* dirs, const float* coeffs,
                     const uint8_t* masks, const float* v_colors, float* v_coeffs, float* v_dirs, tg_stream_t stream);

/* ------------------------------------------------------------------ mip pyramid
 * Replaces generate_mipmap_fwd / generate_mipmap_bwd
 * (textured_gaussians/cuda/csrc/generate_mipmap_{fwd,bwd}.cu): coarse[g] holds
 * levels 1..L of the 2^L x 2^L RGBA texture g, coarsest first (level t, side
 * 2^(L-t), starts at texel (4^(L-t) - 1) / 3), each texel the mean of its
 * four children summed in the reference's order ((a + b) + c) + d, then / 4.
 * The reference also copies level 0 into its pyramid; here the compositor
 * reads level 0 from the texture storage itself.  The adjoint adds each coarse
 * gradient / 4 into its four children, coarsest to finest, ending in
 * v_textures (accumulated, not overwritten); v_coarse is scratch (levels 5,
 * 10, ... are modified when L > 5).  1 <= L <= 13. */
TG_API int tg_generate_mipmap(const float* textures, float* coarse, int64_t G, int32_t L, tg_stream_t stream);
TG_API int tg_generate_mipmap_bwd(float* v_coarse, float* v_textures, int64_t G, int32_t L, tg_stream_t stream);

/* ------------------------------------------------------------------ anisotropic_bilinear row prefixes
 * The table tg_raster_fwd_args.aniso_prefix points to: for texture g, row r
 * and column u, prefix[g,r,u] = sum_{k<u} (t(g,r,k) + t(g,r,k+1)) / 2 (the
 * integral of the row's linear interpolant from column 0 to u; 0 at u = 0),
 * per channel, FP32 [G,ry,rx,4], decoded from `textures` in tex_format
 * (TG_TEX_F32/BF16/F16/FP8_E4M3, tex_scales [G] for fp8).  Rebuild it
 * whenever the textures change.  No counterpart in the reference. */
TG_API int tg_aniso_prefix(const void* textures, int32_t tex_format, const float* tex_scales, int64_t G, int32_t ry,
                           int32_t rx, float* prefix, tg_stream_t stream);

/* ------------------------------------------------------------------ gradient consumers
 * Replaces selective_adam_update (textured_gaussians/cuda/csrc/adam.cu:17-89):
 * for every row r < N (M floats each) with visibility[r] != 0,
 *   m = b1 m + (1-b1) g;  v = b2 v + (1-b2) g^2;  p += -lr m / (sqrt(v) + eps)
 * (no bias correction, as in the reference); other rows are not touched.
 * shadow_format TG_TEX_BF16 / TG_TEX_F16 additionally writes each updated
 * row into `shadow` ([N*M] in that format: the texture storage the compositor
 * samples) in the same pass; TG_TEX_NONE: no shadow. */
TG_API int tg_selective_adam(float* param, const float* grad, float* exp_avg, float* exp_avg_sq,
                             const uint8_t* visibility, float lr, float b1, float b2, float eps, int64_t N, int64_t M,
                             int32_t shadow_format, void* shadow, tg_stream_t stream);

/* Replaces the running-statistics update of DefaultStrategy._update_state
 * (textured_gaussians/strategy/default.py:213-261): for every entry with
 * radius > 0, grad2d[g] += |(gx * width/2 * C, gy * height/2 * C)|,
 * count[g] += 1 and (if max_radii != NULL) max_radii[g] = max(max_radii[g],
 * radius / max(width, height)) -- a true maximum (the reference's indexed
 * assignment keeps the last camera's value when a Gaussian is seen by several).
 * Dense: entries [C,N], g = n; packed: gaussian_ids[e].  max_radii must hold
 * non-negative values. */
typedef struct {
    int32_t C;
    int64_t N;                  /* Gaussians */
    int64_t n_elems;            /* packed: nnz (dense: C*N, unused) */
    const float* grads2d;       /* [E,2] gradient of the 2D means (or its absolute value) */
    const int32_t* radii;       /* [E] */
    const int64_t* gaussian_ids;/* packed: [nnz]; dense: NULL */
    int32_t width, height;
    float* grad2d;              /* [N] accumulated */
    float* count;               /* [N] accumulated */
    float* max_radii;           /* [N] or NULL */
} tg_densify_stats_args;
TG_API int tg_densify_stats(const tg_densify_stats_args* a, tg_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* TG2DGS_H */

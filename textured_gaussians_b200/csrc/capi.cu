// extern "C" entry points of libtg2dgs.so (declared in include/tg2dgs.h).
//
// Each entry point validates its arguments (null pointers, sizes, alignment of
// vector-loaded buffers, supported channel counts / formats / tile sizes),
// enqueues its kernels on the caller's stream and maps failures to TG_ERR_*
// codes with a per-thread message.  Nothing here allocates device memory:
// every buffer, including scratch workspaces, comes from the caller.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "tg_common.cuh"

namespace tg {
cudaError_t launch_project_fwd(const tg_project_fwd_args& a, cudaStream_t s);
cudaError_t launch_project_bwd(const tg_project_bwd_args& a, cudaStream_t s);
size_t project_packed_workspace_bytes(int32_t C, int32_t N);
cudaError_t launch_project_packed_count(const tg_project_packed_args& a, cudaStream_t s);
cudaError_t launch_project_packed_emit(const tg_project_packed_args& a, cudaStream_t s);
cudaError_t launch_project_packed_bwd(const tg_project_packed_bwd_args& a, cudaStream_t s);
size_t scan_workspace_bytes(int64_t n_elems);
cudaError_t launch_isect_count(const tg_isect_args& a, cudaStream_t s);
cudaError_t launch_isect_emit(const tg_isect_args& a, int tile_n_bits, int end_bit, cudaStream_t s);
uint32_t* sort_error_flag(void* workspace, int64_t n, int end_bit);
int sort_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, void* workspace,
                           size_t ws_bytes, cudaStream_t s, cudaError_t& cerr);
size_t sort_workspace_bytes(int64_t n, int end_bit);
int sort_pairs(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n, int end_bit,
               void* workspace, size_t ws_bytes, int32_t* result_in_alt, cudaStream_t s, cudaError_t& cerr);
cudaError_t launch_offset_encode(const int64_t* keys, int64_t n, int C, int tw, int th, int tile_n_bits, int end_bit,
                                 int32_t* offsets, cudaStream_t s);
cudaError_t launch_offset_encode_views(const int64_t* keys, int64_t n, int C, int64_t n_tiles, const tg_view* views,
                                       const int32_t* tile_view, int tile_n_bits, int end_bit, int32_t* offsets,
                                       cudaStream_t s);
cudaError_t launch_raster_fwd(const tg_raster_fwd_args& a, cudaStream_t s);
cudaError_t launch_raster_bwd(const tg_raster_bwd_args& a, cudaStream_t s);
cudaError_t launch_sh_fwd(int64_t n, int64_t rows, int degree, int K, const float* dirs, const float* coeffs,
                          const uint8_t* masks, float* colors, cudaStream_t s);
cudaError_t launch_sh_bwd(int64_t n, int64_t rows, int degree, int K, const float* dirs, const float* coeffs,
                          const uint8_t* masks, const float* v_colors, float* v_coeffs, float* v_dirs,
                          cudaStream_t s);
cudaError_t launch_selective_adam(float* param, const float* grad, float* m, float* v, const uint8_t* vis, float lr,
                                  float b1, float b2, float eps, int64_t N, int64_t M, int shadow_format, void* shadow,
                                  cudaStream_t s);
cudaError_t launch_densify_stats(const tg_densify_stats_args& a, cudaStream_t s);
cudaError_t launch_generate_mipmap(const float* textures, float* coarse, int64_t G, int L, cudaStream_t s);
cudaError_t launch_generate_mipmap_bwd(float* v_coarse, float* v_textures, int64_t G, int L, cudaStream_t s);
cudaError_t launch_aniso_prefix(const void* textures, int tex_format, const float* tex_scales, int64_t G, int ry,
                                int rx, float* prefix, cudaStream_t s);
cudaError_t launch_aniso_prefix_fold(const float* v_prefix, int64_t G, int ry, int rx, float* v_textures,
                                     cudaStream_t s);
int fail_with(int code, const char* msg);
}  // namespace tg

namespace {
std::atomic<uint64_t> g_launches{0};
}  // namespace
void tg::note_launches(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return TG_OK;
    return fail(TG_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

int bit_width(int64_t n) {  // floor(log2(n)) + 1, as the reference computes it
    int b = 0;
    while (n > 0) { ++b; n >>= 1; }
    return b;
}

}  // namespace

int tg::fail_with(int code, const char* msg) { return fail(code, "%s", msg); }

namespace {

#define TG_REQUIRE(cond, code, ...) \
    do {                            \
        if (!(cond)) return fail(code, __VA_ARGS__); \
    } while (0)

int64_t raster_pixels(const tg_raster_fwd_args& a) {
    return a.views ? a.n_pixels : (int64_t)a.C * a.height * a.width;
}

int check_sh(int32_t degree, int32_t K, const float* coeffs, const void* out) {
    if (coeffs == nullptr) return TG_OK;
    TG_REQUIRE(degree >= 0 && degree <= 4 && (degree + 1) * (degree + 1) <= K && K <= 25, TG_ERR_INVALID_ARG,
               "bad fused SH degree %d for %d bases", degree, K);
    TG_REQUIRE(out != nullptr, TG_ERR_INVALID_ARG, "fused SH needs its output buffer");
    return TG_OK;
}

int check_raster_common(const tg_raster_fwd_args& a) {
    TG_REQUIRE(a.C >= 0 && a.width >= 0 && a.height >= 0, TG_ERR_INVALID_ARG, "negative sizes");
    TG_REQUIRE(a.tile_size == 8 || a.tile_size == 16 || a.tile_size == 32, TG_ERR_UNSUPPORTED,
               "tile_size %d not supported (8, 16 or 32)", a.tile_size);
    TG_REQUIRE(a.batch_depth == 0 || (a.batch_depth >= 32 && a.batch_depth <= 1024 && a.batch_depth % 32 == 0),
               TG_ERR_UNSUPPORTED, "batch_depth %d not supported (0, or a multiple of 32 up to 1024)", a.batch_depth);
    TG_REQUIRE(a.D >= 1 && a.D <= 5, TG_ERR_UNSUPPORTED, "unsupported number of channels: %d", a.D);
    if (a.views) {
        TG_REQUIRE(a.tile_view && a.n_tiles >= 0 && a.n_tiles < (int64_t(1) << 31) && a.n_pixels >= 0,
                   TG_ERR_INVALID_ARG, "view table needs tile_view, n_tiles and n_pixels");
    } else {
        TG_REQUIRE((int64_t)a.tile_width * a.tile_size >= a.width && (int64_t)a.tile_height * a.tile_size >= a.height,
                   TG_ERR_INVALID_ARG, "tile grid %dx%d does not cover the image", a.tile_width, a.tile_height);
        TG_REQUIRE((int64_t)a.C * a.tile_width * a.tile_height < (int64_t(1) << 31), TG_ERR_INVALID_ARG,
                   "too many tiles");
    }
    TG_REQUIRE(a.n_isects >= 0 && a.n_isects < (int64_t(1) << 31), TG_ERR_INVALID_ARG, "n_isects out of range");
    TG_REQUIRE(a.tile_offsets && (a.n_isects == 0 || a.flatten_ids), TG_ERR_INVALID_ARG, "null offsets/flatten ids");
    TG_REQUIRE(a.means2d && a.ray_transforms && a.colors && a.opacities && a.normals, TG_ERR_INVALID_ARG,
               "null splat array");
    TG_REQUIRE(aligned(a.means2d, 8), TG_ERR_INVALID_ARG, "means2d must be 8-byte aligned");
    TG_REQUIRE(a.gaussian_ids != nullptr || a.N > 0 || a.n_isects == 0, TG_ERR_INVALID_ARG, "N must be > 0");
    switch (a.tex_format) {
        case TG_TEX_NONE: break;
        case TG_TEX_F32:
            TG_REQUIRE(a.textures && aligned(a.textures, 16), TG_ERR_INVALID_ARG, "FP32 textures must be 16-byte aligned");
            break;
        case TG_TEX_BF16:
        case TG_TEX_F16:
            TG_REQUIRE(a.textures && aligned(a.textures, 8), TG_ERR_INVALID_ARG, "16-bit textures must be 8-byte aligned");
            TG_REQUIRE(a.D == 3 || a.D == 4, TG_ERR_UNSUPPORTED, "16-bit textures support 3 or 4 channels");
            break;
        case TG_TEX_FP8_E4M3:
            TG_REQUIRE(a.textures && aligned(a.textures, 4) && a.tex_scales, TG_ERR_INVALID_ARG,
                       "FP8 textures need 4-byte alignment and per-Gaussian scales");
            TG_REQUIRE(a.D == 3 || a.D == 4, TG_ERR_UNSUPPORTED, "FP8 textures support 3 or 4 channels");
            break;
        default: return fail(TG_ERR_UNSUPPORTED, "unknown texture format %d", a.tex_format);
    }
    if (a.tex_format != TG_TEX_NONE)
        TG_REQUIRE(a.tex_rx >= 1 && a.tex_ry >= 1 && a.range_x > 0.f && a.range_y > 0.f, TG_ERR_INVALID_ARG,
                   "bad texture size or range");
    TG_REQUIRE(a.mip_levels >= 0 && a.mip_levels <= 13, TG_ERR_INVALID_ARG, "bad mip_levels %d", a.mip_levels);
    if (a.mip_levels > 0) {
        TG_REQUIRE(a.tex_format == TG_TEX_F32 || a.tex_format == TG_TEX_BF16, TG_ERR_UNSUPPORTED,
                   "the mipmapped2 filter supports FP32 and BF16 texture storage");
        TG_REQUIRE(a.D == 3 || a.D == 4, TG_ERR_UNSUPPORTED, "the mipmapped2 filter supports 3 or 4 channels");
        TG_REQUIRE(a.tex_rx == (1 << a.mip_levels) && a.tex_ry == a.tex_rx, TG_ERR_INVALID_ARG,
                   "mipmapped2 textures must be 2^L x 2^L (got %d x %d for L = %d)", a.tex_ry, a.tex_rx, a.mip_levels);
        TG_REQUIRE(a.tex_coarse && aligned(a.tex_coarse, 16), TG_ERR_INVALID_ARG,
                   "mipmapped2 needs the 16-byte aligned coarse pyramid");
        TG_REQUIRE(a.tile_size <= 16 && a.work_queue == nullptr, TG_ERR_UNSUPPORTED,
                   "the mipmapped2 filter runs with tile 8 or 16 and one CTA per tile");
    }
    TG_REQUIRE(a.filter == TG_FILTER_BILINEAR || a.filter == TG_FILTER_MIPMAPPED2 ||
                   a.filter == TG_FILTER_ANISO_BILINEAR, TG_ERR_INVALID_ARG, "unknown filter %d", a.filter);
    TG_REQUIRE(a.filter != TG_FILTER_MIPMAPPED2 || a.mip_levels > 0, TG_ERR_INVALID_ARG,
               "TG_FILTER_MIPMAPPED2 needs mip_levels > 0");
    if (a.filter == TG_FILTER_ANISO_BILINEAR) {
        TG_REQUIRE(a.mip_levels == 0, TG_ERR_INVALID_ARG, "anisotropic_bilinear takes no mip levels");
        TG_REQUIRE(a.tex_format == TG_TEX_F32 || a.tex_format == TG_TEX_BF16, TG_ERR_UNSUPPORTED,
                   "the anisotropic_bilinear filter supports FP32 and BF16 texture storage");
        TG_REQUIRE(a.D == 3 || a.D == 4, TG_ERR_UNSUPPORTED, "the anisotropic_bilinear filter supports 3 or 4 channels");
        TG_REQUIRE(a.tile_size <= 16 && a.work_queue == nullptr, TG_ERR_UNSUPPORTED,
                   "the anisotropic_bilinear filter runs with tile 8 or 16 and one CTA per tile");
        TG_REQUIRE(a.aniso_prefix == nullptr || aligned(a.aniso_prefix, 16), TG_ERR_INVALID_ARG,
                   "aniso_prefix must be 16-byte aligned");
        TG_REQUIRE(a.aniso_records == nullptr ||
                       (a.aniso_record_count != nullptr && a.aniso_record_cap > 0 && aligned(a.aniso_records, 16)),
                   TG_ERR_INVALID_ARG, "aniso_records needs a 16-byte aligned buffer, counts and a capacity");
    }
    return TG_OK;
}
}  // namespace

extern "C" {

int tg_version(void) { return 1; }

const char* tg_last_error(void) { return g_last_error.c_str(); }

uint64_t tg_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int tg_project_fwd(const tg_project_fwd_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    TG_REQUIRE(a->C >= 0 && a->N >= 0, TG_ERR_INVALID_ARG, "negative sizes");
    if ((int64_t)a->C * a->N == 0) return TG_OK;
    TG_REQUIRE(a->means && a->quats && a->scales && a->viewmats && a->Ks && a->radii && a->means2d && a->depths &&
                   a->ray_transforms && a->normals,
               TG_ERR_INVALID_ARG, "null pointer");
    TG_REQUIRE(aligned(a->quats, 16) && aligned(a->means2d, 8), TG_ERR_INVALID_ARG,
               "quats must be 16-byte and means2d 8-byte aligned");
    const int rc = check_sh(a->sh_degree, a->sh_K, a->sh_coeffs, a->colors);
    if (rc != TG_OK) return rc;
    return cuda_status(tg::launch_project_fwd(*a, stream), "tg_project_fwd");
}

int tg_project_bwd(const tg_project_bwd_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    TG_REQUIRE(a->C >= 0 && a->N >= 0, TG_ERR_INVALID_ARG, "negative sizes");
    TG_REQUIRE(a->mode >= 0 && a->mode <= 2, TG_ERR_INVALID_ARG, "bad mode %d", a->mode);
    if (a->N == 0) return TG_OK;
    TG_REQUIRE(a->means && a->quats && a->scales && a->viewmats && a->Ks && a->radii && a->ray_transforms &&
                   a->v_means2d && a->v_depths && a->v_normals && a->v_ray_transforms && a->v_means && a->v_quats &&
                   a->v_scales,
               TG_ERR_INVALID_ARG, "null pointer");
    TG_REQUIRE(aligned(a->quats, 16) && aligned(a->v_quats, 16), TG_ERR_INVALID_ARG, "quats must be 16-byte aligned");
    int rc = check_sh(a->sh_degree, a->sh_K, a->sh_coeffs, a->v_sh_coeffs);
    if (rc != TG_OK) return rc;
    if (a->sh_coeffs) TG_REQUIRE(a->v_colors != nullptr, TG_ERR_INVALID_ARG, "fused SH adjoint needs v_colors");
    return cuda_status(tg::launch_project_bwd(*a, stream), "tg_project_bwd");
}

namespace {
int check_packed_common(const tg_project_packed_args* a) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    TG_REQUIRE(a->C >= 0 && a->N >= 0, TG_ERR_INVALID_ARG, "negative sizes");
    TG_REQUIRE(a->C <= 65535, TG_ERR_UNSUPPORTED, "at most 65535 cameras (got %d)", a->C);
    TG_REQUIRE(a->workspace && a->nnz && a->indptr, TG_ERR_INVALID_ARG, "null workspace / nnz / indptr");
    TG_REQUIRE(a->gauss_ranges == nullptr || a->max_range >= 0, TG_ERR_INVALID_ARG, "negative max_range");
    if ((int64_t)a->C * a->N == 0) return TG_OK;
    TG_REQUIRE(a->means && a->quats && a->scales && a->viewmats && a->Ks, TG_ERR_INVALID_ARG, "null pointer");
    TG_REQUIRE(aligned(a->quats, 16), TG_ERR_INVALID_ARG, "quats must be 16-byte aligned");
    return TG_OK;
}
}  // namespace

size_t tg_project_packed_workspace_bytes(int32_t C, int32_t N) { return tg::project_packed_workspace_bytes(C, N); }

int tg_project_packed_count(const tg_project_packed_args* a, tg_stream_t stream) {
    const int rc = check_packed_common(a);
    if (rc != TG_OK) return rc;
    return cuda_status(tg::launch_project_packed_count(*a, stream), "tg_project_packed_count");
}

int tg_project_packed_emit(const tg_project_packed_args* a, tg_stream_t stream) {
    const int rc = check_packed_common(a);
    if (rc != TG_OK) return rc;
    TG_REQUIRE(a->nnz_host >= 0, TG_ERR_INVALID_ARG, "negative nnz");
    TG_REQUIRE(a->nnz_host < (int64_t(1) << 31), TG_ERR_UNSUPPORTED, "nnz %lld does not fit the int32 indptr",
               (long long)a->nnz_host);
    if (a->nnz_host == 0 || (int64_t)a->C * a->N == 0) return TG_OK;
    TG_REQUIRE(a->camera_ids && a->gaussian_ids && a->radii && a->means2d && a->depths && a->ray_transforms &&
                   a->normals,
               TG_ERR_INVALID_ARG, "null output pointer");
    TG_REQUIRE(aligned(a->means2d, 8), TG_ERR_INVALID_ARG, "means2d must be 8-byte aligned");
    const int rc_sh = check_sh(a->sh_degree, a->sh_K, a->sh_coeffs, a->colors);
    if (rc_sh != TG_OK) return rc_sh;
    if (a->sh_coeffs && a->overflow) {  // the unused tail's colours are zeroed (never rendered)
        const cudaError_t e = cudaMemsetAsync(a->colors, 0, 12 * (size_t)a->nnz_host, stream);
        if (e != cudaSuccess) return cuda_status(e, "tg_project_packed_emit memset");
    }
    if (a->overflow) {  // capacity mode: every output zeroed, so the unused tail is inert
        const size_t n = (size_t)a->nnz_host;
        struct Z { void* p; size_t b; } zs[] = {{a->camera_ids, 8 * n}, {a->gaussian_ids, 8 * n}, {a->radii, 4 * n},
                                                {a->means2d, 8 * n},    {a->depths, 4 * n},       {a->ray_transforms, 36 * n},
                                                {a->normals, 12 * n}};
        for (const Z& z : zs) {
            const cudaError_t e = cudaMemsetAsync(z.p, 0, z.b, stream);
            if (e != cudaSuccess) return cuda_status(e, "tg_project_packed_emit memset");
        }
    }
    return cuda_status(tg::launch_project_packed_emit(*a, stream), "tg_project_packed_emit");
}

int tg_project_packed_bwd(const tg_project_packed_bwd_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    TG_REQUIRE(a->C >= 0 && a->N >= 0 && a->nnz >= 0, TG_ERR_INVALID_ARG, "negative sizes");
    TG_REQUIRE(a->mode >= 0 && a->mode <= 2, TG_ERR_INVALID_ARG, "bad mode %d", a->mode);
    TG_REQUIRE(a->nnz < (int64_t(1) << 31), TG_ERR_UNSUPPORTED, "nnz out of range");
    const int64_t rows = a->sparse_grad ? a->nnz : a->N;
    if (rows > 0) TG_REQUIRE(a->v_means && a->v_quats && a->v_scales, TG_ERR_INVALID_ARG, "null gradient output");
    if (rows > 0) TG_REQUIRE(aligned(a->v_quats, 16), TG_ERR_INVALID_ARG, "v_quats must be 16-byte aligned");
    if (rows > 0) {  // zeroed in both layouts, so skipped entries read as zero
        cudaError_t e = cudaMemsetAsync(a->v_means, 0, sizeof(float) * 3 * (size_t)rows, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(a->v_quats, 0, sizeof(float) * 4 * (size_t)rows, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(a->v_scales, 0, sizeof(float) * 3 * (size_t)rows, stream);
        if (e != cudaSuccess) return cuda_status(e, "tg_project_packed_bwd");
    }
    const int rc_sh = check_sh(a->sh_degree, a->sh_K, a->sh_coeffs, a->v_sh_coeffs);
    if (rc_sh != TG_OK) return rc_sh;
    if (a->sh_coeffs && a->N > 0) {
        TG_REQUIRE(a->v_colors != nullptr, TG_ERR_INVALID_ARG, "fused SH adjoint needs v_colors");
        const cudaError_t e = cudaMemsetAsync(a->v_sh_coeffs, 0, sizeof(float) * 3 * a->sh_K * (size_t)a->N, stream);
        if (e != cudaSuccess) return cuda_status(e, "tg_project_packed_bwd memset");
    }
    if (a->nnz == 0) return TG_OK;
    TG_REQUIRE(a->means && a->quats && a->scales && a->viewmats && a->Ks && a->camera_ids && a->gaussian_ids &&
                   a->ray_transforms && a->v_means2d && a->v_depths && a->v_normals && a->v_ray_transforms,
               TG_ERR_INVALID_ARG, "null pointer");
    TG_REQUIRE(aligned(a->quats, 16), TG_ERR_INVALID_ARG, "quats must be 16-byte aligned");
    return cuda_status(tg::launch_project_packed_bwd(*a, stream), "tg_project_packed_bwd");
}

size_t tg_scan_workspace_bytes(int64_t n_elems) { return tg::scan_workspace_bytes(n_elems); }

int tg_isect_count(const tg_isect_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    TG_REQUIRE(a->n_elems >= 0 && a->n_elems < (int64_t(1) << 31), TG_ERR_INVALID_ARG, "n_elems out of range");
    TG_REQUIRE(a->tile_size > 0 && a->tile_width > 0 && a->tile_height > 0 && a->n_cameras > 0, TG_ERR_INVALID_ARG,
               "bad tile grid");
    TG_REQUIRE(bit_width((int64_t)a->tile_width * a->tile_height) + bit_width(a->n_cameras) <= 32, TG_ERR_INVALID_ARG,
               "camera and tile ids need more than 32 bits");
    TG_REQUIRE(a->n_isects && a->scan_workspace, TG_ERR_INVALID_ARG, "null n_isects / workspace");
    if (a->n_elems > 0)
        TG_REQUIRE(a->means2d && a->radii && a->tiles_per_gauss && a->cum_tiles && aligned(a->means2d, 8),
                   TG_ERR_INVALID_ARG, "null or misaligned pointer");
    return cuda_status(tg::launch_isect_count(*a, stream), "tg_isect_count");
}

int tg_isect_emit(const tg_isect_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    if (a->overflow) {
        TG_REQUIRE(a->capacity >= 0 && a->capacity < (int64_t(1) << 31), TG_ERR_INVALID_ARG, "bad capacity");
        TG_REQUIRE(a->n_isects && (a->capacity == 0 || (a->isect_ids && a->flatten_ids)), TG_ERR_INVALID_ARG,
                   "capacity mode needs n_isects and the key / id buffers");
    }
    if (a->n_elems == 0 && !(a->overflow && a->capacity > 0)) return TG_OK;
    if (a->n_elems > 0) {
        TG_REQUIRE(a->means2d && a->radii && a->depths && a->cum_tiles && a->isect_ids && a->flatten_ids,
                   TG_ERR_INVALID_ARG, "null pointer");
        TG_REQUIRE(a->camera_ids != nullptr || a->N > 0, TG_ERR_INVALID_ARG, "dense layout needs N > 0");
    }
    const int tb = bit_width((int64_t)a->tile_width * a->tile_height);
    const int cb = bit_width(a->n_cameras);
    return cuda_status(tg::launch_isect_emit(*a, tb, 32 + tb + cb, stream), "tg_isect_emit");
}

int tg_sort_lookback_selftest(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, void* workspace,
                              size_t workspace_bytes, tg_stream_t stream) {
    TG_REQUIRE(keys && vals && keys_alt && vals_alt && workspace, TG_ERR_INVALID_ARG, "null pointer");
    cudaError_t cerr;
    const int rc = tg::sort_lookback_selftest(keys, vals, keys_alt, vals_alt, workspace, workspace_bytes, stream, cerr);
    if (rc == TG_ERR_CUDA) return cuda_status(cerr, "tg_sort_lookback_selftest");
    if (rc == TG_ERR_WORKSPACE) return fail(rc, "workspace smaller than tg_sort_workspace_bytes(8192, 8)");
    if (rc == TG_ERR_TIMEOUT) return fail(rc, "look-back wait gave up (the expected outcome of this self-test)");
    return rc;
}

int tg_sort_status(const void* workspace, int64_t n, int32_t end_bit, tg_stream_t stream) {
    TG_REQUIRE(n >= 0 && end_bit >= 0 && end_bit <= 64, TG_ERR_INVALID_ARG, "bad sizes");
    if (n <= 1 || end_bit == 0) return TG_OK;
    TG_REQUIRE(workspace != nullptr, TG_ERR_INVALID_ARG, "null workspace");
    const uint32_t* flag = tg::sort_error_flag(const_cast<void*>(workspace), n, end_bit);
    uint32_t h = 0;
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(&h, flag, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "tg_sort_status");
    if (h) return fail(TG_ERR_TIMEOUT, "a look-back wait of the pair sort gave up");
    return TG_OK;
}

size_t tg_sort_workspace_bytes(int64_t n, int32_t end_bit) { return tg::sort_workspace_bytes(n, end_bit); }

int tg_sort_pairs(int64_t* keys, int32_t* vals, int64_t* keys_alt, int32_t* vals_alt, int64_t n, int32_t end_bit,
                  void* workspace, size_t workspace_bytes, int32_t* result_in_alt, tg_stream_t stream) {
    TG_REQUIRE(result_in_alt != nullptr, TG_ERR_INVALID_ARG, "null result_in_alt");
    *result_in_alt = 0;
    TG_REQUIRE(n >= 0 && n < (int64_t(1) << 30), TG_ERR_INVALID_ARG, "sort supports up to 2^30 pairs");
    TG_REQUIRE(end_bit >= 0 && end_bit <= 64, TG_ERR_INVALID_ARG, "bad end_bit %d", end_bit);
    if (n <= 1) return TG_OK;
    TG_REQUIRE(keys && vals && keys_alt && vals_alt && workspace, TG_ERR_INVALID_ARG, "null pointer");
    cudaError_t cerr;
    const int rc = tg::sort_pairs(keys, vals, keys_alt, vals_alt, n, end_bit, workspace, workspace_bytes,
                                  result_in_alt, stream, cerr);
    if (rc == TG_ERR_CUDA) return cuda_status(cerr, "tg_sort_pairs");
    if (rc == TG_ERR_WORKSPACE) return fail(rc, "workspace of %zu bytes is smaller than %zu", workspace_bytes,
                                            tg::sort_workspace_bytes(n, end_bit));
    if (rc != TG_OK) return fail(rc, "tg_sort_pairs: invalid argument");
    return TG_OK;
}

int tg_isect_offset_encode(const int64_t* isect_ids, int64_t n_isects, int32_t n_cameras, int32_t tile_width,
                           int32_t tile_height, int32_t* offsets, tg_stream_t stream) {
    TG_REQUIRE(n_cameras > 0 && tile_width > 0 && tile_height > 0 && offsets, TG_ERR_INVALID_ARG, "bad arguments");
    TG_REQUIRE(n_isects >= 0 && (n_isects == 0 || isect_ids), TG_ERR_INVALID_ARG, "null isect_ids");
    const int tb = bit_width((int64_t)tile_width * tile_height);
    const int cb = bit_width(n_cameras);
    return cuda_status(tg::launch_offset_encode(isect_ids, n_isects, n_cameras, tile_width, tile_height, tb,
                                                32 + tb + cb, offsets, stream),
                       "tg_isect_offset_encode");
}

int tg_isect_offset_encode_views(const int64_t* isect_ids, int64_t n_isects, int32_t n_cameras,
                                 int64_t max_tiles_per_view, const tg_view* views, const int32_t* tile_view,
                                 int64_t n_tiles, int32_t* offsets, tg_stream_t stream) {
    TG_REQUIRE(n_cameras > 0 && max_tiles_per_view > 0 && n_tiles >= 0 && n_tiles < (int64_t(1) << 31),
               TG_ERR_INVALID_ARG, "bad sizes");
    TG_REQUIRE(n_isects >= 0 && (n_isects == 0 || isect_ids), TG_ERR_INVALID_ARG, "null isect_ids");
    if (n_tiles == 0) return TG_OK;
    TG_REQUIRE(views && tile_view && offsets, TG_ERR_INVALID_ARG, "null view table or offsets");
    const int tb = bit_width(max_tiles_per_view);
    const int cb = bit_width(n_cameras);
    TG_REQUIRE(tb + cb <= 32, TG_ERR_INVALID_ARG, "camera and tile ids need more than 32 bits");
    return cuda_status(tg::launch_offset_encode_views(isect_ids, n_isects, n_cameras, n_tiles, views, tile_view, tb,
                                                      32 + tb + cb, offsets, stream),
                       "tg_isect_offset_encode_views");
}

int tg_rasterize_fwd(const tg_raster_fwd_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    int rc = check_raster_common(*a);
    if (rc != TG_OK) return rc;
    const int64_t pixels = raster_pixels(*a);
    if (pixels > 0)
        TG_REQUIRE(a->out_colors && a->out_alphas && a->out_normals && a->out_distort && a->out_median &&
                       a->last_ids && a->median_ids,
                   TG_ERR_INVALID_ARG, "null output");
    TG_REQUIRE(a->n_contrib >= 0 && (a->n_contrib == 0 || (a->contrib_sum && a->contrib_count)), TG_ERR_INVALID_ARG,
               "null contribution buffers");
    cudaError_t e = cudaSuccess;
    if (a->n_contrib > 0) {
        e = cudaMemsetAsync(a->contrib_sum, 0, sizeof(float) * a->n_contrib, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(a->contrib_count, 0, sizeof(float) * a->n_contrib, stream);
        if (e != cudaSuccess) return cuda_status(e, "tg_rasterize_fwd memset");
    }
    return cuda_status(tg::launch_raster_fwd(*a, stream), "tg_rasterize_fwd");
}

int tg_rasterize_bwd(const tg_raster_bwd_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    int rc = check_raster_common(a->f);
    if (rc != TG_OK) return rc;
    TG_REQUIRE(a->adjoint >= 0 && a->adjoint <= 2, TG_ERR_INVALID_ARG, "bad adjoint %d", a->adjoint);
    TG_REQUIRE(a->f.mip_levels == 0 || a->adjoint == TG_ADJ_REFERENCE, TG_ERR_UNSUPPORTED,
               "the mipmapped2 filter has the reference adjoint only");
    TG_REQUIRE(a->f.filter != TG_FILTER_ANISO_BILINEAR || a->adjoint == TG_ADJ_REFERENCE, TG_ERR_UNSUPPORTED,
               "the anisotropic_bilinear filter has the reference adjoint only");
    if (a->f.mip_levels > 0 && a->v_textures)
        TG_REQUIRE(a->v_tex_coarse && aligned(a->v_tex_coarse, 16), TG_ERR_INVALID_ARG,
                   "mipmapped2 texture gradients need v_tex_coarse");
    TG_REQUIRE(a->n_elems >= 0, TG_ERR_INVALID_ARG, "negative n_elems");
    TG_REQUIRE(a->render_colors && a->render_alphas && a->last_ids && a->median_ids && a->v_render_colors &&
                   a->v_render_alphas && a->v_render_normals && a->v_render_distort && a->v_render_median,
               TG_ERR_INVALID_ARG, "null forward output or upstream gradient");
    TG_REQUIRE(a->v_means2d && a->v_ray_transforms && a->v_colors && a->v_opacities && a->v_normals && a->v_densify,
               TG_ERR_INVALID_ARG, "null gradient output");
    if (a->v_textures) TG_REQUIRE(aligned(a->v_textures, 16), TG_ERR_INVALID_ARG, "v_textures must be 16-byte aligned");
    // the boundary-integral adjoint accumulates the row-prefix gradient, folded into v_textures afterwards
    const bool fold = a->f.filter == TG_FILTER_ANISO_BILINEAR && a->f.aniso_prefix != nullptr &&
                      a->v_textures != nullptr;
    if (fold)
        TG_REQUIRE(a->v_aniso_prefix && aligned(a->v_aniso_prefix, 16), TG_ERR_INVALID_ARG,
                   "anisotropic_bilinear with aniso_prefix needs a 16-byte aligned v_aniso_prefix");
    const int64_t E = a->n_elems;
    const int D = a->f.D;
    const size_t tex_bytes = a->f.tex_format == TG_TEX_NONE || a->v_textures == nullptr
                                 ? 0
                                 : sizeof(float) * 4 * (size_t)a->f.tex_ry * a->f.tex_rx * (size_t)a->f.n_contrib;
    struct Z { void* p; size_t n; } zs[] = {
        {a->v_means2d, sizeof(float) * 2 * E}, {a->v_ray_transforms, sizeof(float) * 9 * E},
        {a->v_colors, sizeof(float) * D * E},  {a->v_opacities, sizeof(float) * E},
        {a->v_normals, sizeof(float) * 3 * E}, {a->v_means2d_abs, a->v_means2d_abs ? sizeof(float) * 2 * E : 0},
        {a->v_textures, tex_bytes},            {a->v_densify, sizeof(float) * 2 * E},
        {a->v_tex_coarse, a->f.mip_levels > 0 && a->v_textures
                              ? sizeof(float) * 4 * (size_t)(((int64_t(1) << (2 * a->f.mip_levels)) - 1) / 3) *
                                    (size_t)a->f.n_contrib
                              : 0},
        {fold ? a->v_aniso_prefix : nullptr, tex_bytes}};
    for (const Z& z : zs)
        if (z.p && z.n) {
            cudaError_t e = cudaMemsetAsync(z.p, 0, z.n, stream);
            if (e != cudaSuccess) return cuda_status(e, "tg_rasterize_bwd memset");
        }
    tg_raster_bwd_args b = *a;
    if (!fold) b.v_aniso_prefix = nullptr;
    cudaError_t e = tg::launch_raster_bwd(b, stream);
    if (e == cudaSuccess && fold)
        e = tg::launch_aniso_prefix_fold(a->v_aniso_prefix, a->f.n_contrib, a->f.tex_ry, a->f.tex_rx, a->v_textures,
                                         stream);
    return cuda_status(e, "tg_rasterize_bwd");
}

int tg_sh_fwd(int64_t n, int64_t coeff_rows, int32_t degree, int32_t K, const float* dirs, const float* coeffs,
              const uint8_t* masks, float* colors, tg_stream_t stream) {
    TG_REQUIRE(n >= 0 && degree >= 0 && degree <= 4 && (degree + 1) * (degree + 1) <= K, TG_ERR_INVALID_ARG,
               "bad SH degree %d for %d bases", degree, K);
    if (n == 0) return TG_OK;
    TG_REQUIRE(coeff_rows > 0 && n % coeff_rows == 0, TG_ERR_INVALID_ARG, "coeff_rows must divide n");
    TG_REQUIRE(dirs && coeffs && colors, TG_ERR_INVALID_ARG, "null pointer");
    return cuda_status(tg::launch_sh_fwd(n, coeff_rows, degree, K, dirs, coeffs, masks, colors, stream), "tg_sh_fwd");
}

int tg_sh_bwd(int64_t n, int64_t coeff_rows, int32_t degree, int32_t K, const float* dirs, const float* coeffs,
              const uint8_t* masks, const float* v_colors, float* v_coeffs, float* v_dirs, tg_stream_t stream) {
    TG_REQUIRE(n >= 0 && degree >= 0 && degree <= 4 && (degree + 1) * (degree + 1) <= K, TG_ERR_INVALID_ARG,
               "bad SH degree %d for %d bases", degree, K);
    if (n == 0) return TG_OK;
    TG_REQUIRE(coeff_rows > 0 && n % coeff_rows == 0, TG_ERR_INVALID_ARG, "coeff_rows must divide n");
    TG_REQUIRE(dirs && coeffs && v_colors && v_coeffs, TG_ERR_INVALID_ARG, "null pointer");
    return cuda_status(
        tg::launch_sh_bwd(n, coeff_rows, degree, K, dirs, coeffs, masks, v_colors, v_coeffs, v_dirs, stream),
        "tg_sh_bwd");
}

int tg_selective_adam(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, const uint8_t* visibility,
                      float lr, float b1, float b2, float eps, int64_t N, int64_t M, int32_t shadow_format,
                      void* shadow, tg_stream_t stream) {
    TG_REQUIRE(N >= 0 && M >= 0, TG_ERR_INVALID_ARG, "negative sizes");
    TG_REQUIRE(shadow_format == TG_TEX_NONE || shadow_format == TG_TEX_BF16 || shadow_format == TG_TEX_F16,
               TG_ERR_UNSUPPORTED, "shadow format %d not supported (none, BF16, FP16)", shadow_format);
    if (N * M == 0) return TG_OK;
    TG_REQUIRE(param && grad && exp_avg && exp_avg_sq && visibility, TG_ERR_INVALID_ARG, "null pointer");
    TG_REQUIRE(shadow_format == TG_TEX_NONE || shadow != nullptr, TG_ERR_INVALID_ARG, "null shadow");
    return cuda_status(tg::launch_selective_adam(param, grad, exp_avg, exp_avg_sq, visibility, lr, b1, b2, eps, N, M,
                                                 shadow_format, shadow, stream),
                       "tg_selective_adam");
}

int tg_generate_mipmap(const float* textures, float* coarse, int64_t G, int32_t L, tg_stream_t stream) {
    TG_REQUIRE(G >= 0 && L >= 1 && L <= 13, TG_ERR_INVALID_ARG, "bad sizes (G %lld, L %d)", (long long)G, L);
    if (G == 0) return TG_OK;
    TG_REQUIRE(textures && coarse && aligned(textures, 16) && aligned(coarse, 16), TG_ERR_INVALID_ARG,
               "null or misaligned pointer");
    return cuda_status(tg::launch_generate_mipmap(textures, coarse, G, L, stream), "tg_generate_mipmap");
}

int tg_generate_mipmap_bwd(float* v_coarse, float* v_textures, int64_t G, int32_t L, tg_stream_t stream) {
    TG_REQUIRE(G >= 0 && L >= 1 && L <= 13, TG_ERR_INVALID_ARG, "bad sizes (G %lld, L %d)", (long long)G, L);
    if (G == 0) return TG_OK;
    TG_REQUIRE(v_coarse && v_textures && aligned(v_coarse, 16) && aligned(v_textures, 16), TG_ERR_INVALID_ARG,
               "null or misaligned pointer");
    return cuda_status(tg::launch_generate_mipmap_bwd(v_coarse, v_textures, G, L, stream), "tg_generate_mipmap_bwd");
}

int tg_aniso_prefix(const void* textures, int32_t tex_format, const float* tex_scales, int64_t G, int32_t ry,
                    int32_t rx, float* prefix, tg_stream_t stream) {
    TG_REQUIRE(G >= 0 && ry >= 1 && rx >= 1, TG_ERR_INVALID_ARG, "bad sizes (G %lld, ry %d, rx %d)", (long long)G, ry,
               rx);
    TG_REQUIRE(tex_format == TG_TEX_F32 || tex_format == TG_TEX_BF16 || tex_format == TG_TEX_F16 ||
                   tex_format == TG_TEX_FP8_E4M3,
               TG_ERR_INVALID_ARG, "bad texture format %d", tex_format);
    if (G == 0) return TG_OK;
    TG_REQUIRE(textures && prefix && aligned(prefix, 16) && aligned(textures, tex_format == TG_TEX_F32 ? 16 : 8),
               TG_ERR_INVALID_ARG, "null or misaligned pointer");
    TG_REQUIRE(tex_format != TG_TEX_FP8_E4M3 || tex_scales != nullptr, TG_ERR_INVALID_ARG, "fp8 needs tex_scales");
    return cuda_status(tg::launch_aniso_prefix(textures, tex_format, tex_scales, G, ry, rx, prefix, stream),
                       "tg_aniso_prefix");
}

int tg_densify_stats(const tg_densify_stats_args* a, tg_stream_t stream) {
    TG_REQUIRE(a != nullptr, TG_ERR_INVALID_ARG, "null args");
    TG_REQUIRE(a->C >= 0 && a->N >= 0 && a->n_elems >= 0 && a->width > 0 && a->height > 0, TG_ERR_INVALID_ARG,
               "bad sizes");
    if (a->N == 0 || (a->gaussian_ids && a->n_elems == 0) || (!a->gaussian_ids && a->C == 0)) return TG_OK;
    TG_REQUIRE(a->grads2d && a->radii && a->grad2d && a->count, TG_ERR_INVALID_ARG, "null pointer");
    return cuda_status(tg::launch_densify_stats(*a, stream), "tg_densify_stats");
}

}  // extern "C"

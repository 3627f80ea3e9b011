// Coarse mip levels of the per-Gaussian textures (for the mipmapped2 filter)
// and their adjoint, for sm_100a.
//
// Follows generate_mipmap_fwd.cu / generate_mipmap_bwd.cu of the reference:
// level t (side 2^(L-t)) of texture g sits at texel (4^(L-t) - 1) / 3 of the
// pyramid, coarsest first; a texel is ((a + b) + c + d) / 4 of its four
// children in the reference's order.  B200 form: level 0 is not copied into
// the pyramid (the compositor reads it from the texture storage), and each
// level is one grid-stride launch over all textures (a level needs the one
// below it), float4 per texel.
#include "tg_common.cuh"

namespace tg {

__device__ __forceinline__ int64_t level_base(int L, int t) { return (((int64_t)1 << (2 * (L - t))) - 1) / 3; }

// Level t >= 1 from level t - 1 (the texture itself when t == 1).
__global__ void __launch_bounds__(256) mip_level_fwd_kernel(const float4* __restrict__ tex, float4* __restrict__ coarse,
                                                            int64_t G, int L, int t) {
    const int side = 1 << (L - t), child_side = side << 1;
    const int64_t per = (int64_t)side * side, clen = level_base(L, 0);
    const int64_t total = G * per;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = i / per;
        const int r = (int)(i - g * per), v = r / side, u = r - v * side;
        const float4* src = t == 1 ? tex + g * (int64_t)child_side * child_side : coarse + g * clen + level_base(L, t - 1);
        const float4 a = src[(2 * v) * child_side + 2 * u], b = src[(2 * v) * child_side + 2 * u + 1];
        const float4 c = src[(2 * v + 1) * child_side + 2 * u], d = src[(2 * v + 1) * child_side + 2 * u + 1];
        coarse[g * clen + level_base(L, t) + r] =
            make_float4((a.x + b.x + c.x + d.x) * 0.25f, (a.y + b.y + c.y + d.y) * 0.25f,
                        (a.z + b.z + c.z + d.z) * 0.25f, (a.w + b.w + c.w + d.w) * 0.25f);
    }
}

// Children at level t - 1 receive a quarter of their parent's gradient at level t.
__global__ void __launch_bounds__(256) mip_level_bwd_kernel(float4* __restrict__ v_coarse,
                                                            float4* __restrict__ v_tex, int64_t G, int L, int t) {
    const int child_side = 1 << (L - t + 1), side = child_side >> 1;
    const int64_t per = (int64_t)child_side * child_side, clen = level_base(L, 0);
    const int64_t total = G * per;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = i / per;
        const int r = (int)(i - g * per), v = r / child_side, u = r - v * child_side;
        const float4 p = v_coarse[g * clen + level_base(L, t) + (v >> 1) * side + (u >> 1)];
        float4* dst = t == 1 ? v_tex + g * per + r : v_coarse + g * clen + level_base(L, t - 1) + r;
        float4 q = *dst;
        q.x += p.x * 0.25f;
        q.y += p.y * 0.25f;
        q.z += p.z * 0.25f;
        q.w += p.w * 0.25f;
        *dst = q;
    }
}

static unsigned grid_for(int64_t work) {
    return (unsigned)std::min<int64_t>(std::max<int64_t>((work + 255) / 256, 1), (int64_t)kNumSMs * 64);
}

cudaError_t launch_generate_mipmap(const float* textures, float* coarse, int64_t G, int L, cudaStream_t s) {
    for (int t = 1; t <= L; ++t) {
        const int64_t side = (int64_t)1 << (L - t);
        mip_level_fwd_kernel<<<grid_for(G * side * side), 256, 0, s>>>(reinterpret_cast<const float4*>(textures),
                                                                       reinterpret_cast<float4*>(coarse), G, L, t);
        note_launches(1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_generate_mipmap_bwd(float* v_coarse, float* v_textures, int64_t G, int L, cudaStream_t s) {
    for (int t = L; t >= 1; --t) {
        const int64_t cs = (int64_t)1 << (L - t + 1);
        mip_level_bwd_kernel<<<grid_for(G * cs * cs), 256, 0, s>>>(reinterpret_cast<float4*>(v_coarse),
                                                                   reinterpret_cast<float4*>(v_textures), G, L, t);
        note_launches(1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace tg

// Test infrastructure only: Python bindings for the reference's own CUDA ops,
// compiled from the unmodified reference sources by oracle/build_ref.py into
// oracle/_ref/ (never shipped, never linked by the package).  The functions are
// declared by the reference's textured_gaussians/cuda/csrc/bindings.h; the op
// names are the ones textured_gaussians/cuda/csrc/ext.cpp registers for them.
#include "bindings.h"

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
    m.def("compute_sh_fwd", &gsplat::compute_sh_fwd_tensor);
    m.def("compute_sh_bwd", &gsplat::compute_sh_bwd_tensor);
    m.def("fully_fused_projection_fwd_2dgs", &gsplat::fully_fused_projection_fwd_2dgs_tensor);
    m.def("fully_fused_projection_bwd_2dgs", &gsplat::fully_fused_projection_bwd_2dgs_tensor);
    m.def("isect_tiles", &gsplat::isect_tiles_tensor);
    m.def("isect_offset_encode", &gsplat::isect_offset_encode_tensor);
    m.def("rasterize_to_pixels_fwd_2dgs", &gsplat::rasterize_to_pixels_fwd_2dgs_tensor);
    m.def("rasterize_to_pixels_bwd_2dgs", &gsplat::rasterize_to_pixels_bwd_2dgs_tensor);
    m.def("rasterize_to_pixels_fwd_textured_gaussians", &gsplat::rasterize_to_pixels_fwd_textured_gaussians_tensor);
    m.def("rasterize_to_pixels_bwd_textured_gaussians", &gsplat::rasterize_to_pixels_bwd_textured_gaussians_tensor);
    m.def("rasterize_to_pixels_bwd2_textured_gaussians", &gsplat::rasterize_to_pixels_bwd2_textured_gaussians_tensor);
    m.def("generate_mipmap_fwd", &gsplat::generate_mipmap_fwd_tensor);
    m.def("generate_mipmap_bwd", &gsplat::generate_mipmap_bwd_tensor);
    m.def("rasterize_to_pixels_fwd_mip2_textured_gaussians",
          &gsplat::rasterize_to_pixels_fwd_mip2_textured_gaussians_tensor);
    m.def("rasterize_to_pixels_bwd_mip2_textured_gaussians",
          &gsplat::rasterize_to_pixels_bwd_mip2_textured_gaussians_tensor);
    m.def("rasterize_to_pixels_fwd_aniso_bilinear_textured_gaussians",
          &gsplat::rasterize_to_pixels_fwd_aniso_bilinear_textured_gaussians_tensor);
    m.def("rasterize_to_pixels_bwd_aniso_bilinear_textured_gaussians",
          &gsplat::rasterize_to_pixels_bwd_aniso_bilinear_textured_gaussians_tensor);
}

"""Op surface mirroring textured_gaussians.cuda (see _wrapper.py)."""
from ._wrapper import (
    densify_stats,
    fully_fused_projection_2dgs,
    isect_offset_encode,
    isect_offset_encode_views,
    isect_tiles,
    make_texture_storage,
    rasterize_to_pixels_2dgs,
    rasterize_to_pixels_textured_gaussians,
    selective_adam_update,
    sort_pairs,
    spherical_harmonics,
    spherical_harmonics_shared,
    tile_order_heaviest_first,
)

__all__ = [
    "densify_stats",
    "fully_fused_projection_2dgs",
    "isect_offset_encode",
    "isect_offset_encode_views",
    "isect_tiles",
    "make_texture_storage",
    "rasterize_to_pixels_2dgs",
    "rasterize_to_pixels_textured_gaussians",
    "selective_adam_update",
    "sort_pairs",
    "spherical_harmonics",
    "spherical_harmonics_shared",
    "tile_order_heaviest_first",
]

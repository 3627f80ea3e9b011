"""Host logic of the batching form (no GPU): the view table's flat tile and
pixel bases, the tile -> view map and the byte layout of tg_view."""
import ctypes

import numpy as np

from textured_gaussians_b200.batch import TG_VIEW, ViewTable


class CView(ctypes.Structure):  # tg_view as declared in include/tg2dgs.h
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("tile_width", ctypes.c_int32),
                ("tile_height", ctypes.c_int32), ("tile_base", ctypes.c_int64), ("pix_base", ctypes.c_int64)]


def test_tg_view_layout_matches_c():
    assert ctypes.sizeof(CView) == TG_VIEW.itemsize == 32
    for name, _ in CView._fields_:
        assert getattr(CView, name).offset == TG_VIEW.fields[name][1], name


def test_view_table_bases_and_tile_map():
    widths, heights = [1600, 400, 1297, 800], [1200, 300, 840, 600]
    vt = ViewTable(widths, heights, 16, "cpu")
    tw = [100, 25, 82, 50]
    th = [75, 19, 53, 38]
    tiles = [a * b for a, b in zip(tw, th)]
    assert vt.tile_w == tw and vt.tile_h == th
    assert vt.tile_base == [0, tiles[0], tiles[0] + tiles[1], tiles[0] + tiles[1] + tiles[2]]
    assert vt.n_tiles == sum(tiles) and vt.key_tiles == max(tiles)
    px = [w * h for w, h in zip(widths, heights)]
    assert vt.pix_base == [0, px[0], px[0] + px[1], px[0] + px[1] + px[2]] and vt.n_pixels == sum(px)
    arr = vt.views.numpy().view(TG_VIEW)
    assert arr["tile_width"].tolist() == tw and arr["pix_base"].tolist() == vt.pix_base
    tv = vt.tile_view.numpy()
    for c in range(4):
        seg = tv[vt.tile_base[c]:vt.tile_base[c] + tiles[c]]
        assert (seg == c).all()
    flat = np.arange(vt.n_pixels)
    import torch
    parts = vt.split(torch.from_numpy(flat))
    assert [tuple(p.shape) for p in parts] == [(h, w) for w, h in zip(widths, heights)]
    assert int(parts[2][0, 0]) == vt.pix_base[2] and int(parts[2][1, 0]) == vt.pix_base[2] + widths[2]

"""CPU checks of the oracle's mip pyramid (the mipmapped2 filter's texture
levels): each coarse texel is the mean of its 2^t x 2^t block of level 0, and
the pyramid adjoint is the transpose of the pyramid (dot-product test)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("L", [1, 3, 5])
def test_levels_are_block_means(L):
    rng = np.random.default_rng(L)
    R = 1 << L
    tex = rng.uniform(-1, 1, size=(7, R, R, 4))
    pyr = O.generate_mipmap(tex)
    assert pyr.shape == (7, (4 ** (L + 1) - 1) // 3, 4)
    for t in range(L + 1):
        side = R >> t
        lvl = pyr[:, O.mip_level_base(L, t):O.mip_level_base(L, t) + side * side].reshape(7, side, side, 4)
        ref = tex.reshape(7, side, 1 << t, side, 1 << t, 4).mean(axis=(2, 4))
        np.testing.assert_allclose(lvl, ref, rtol=0, atol=1e-14)


@pytest.mark.parametrize("L", [1, 2, 4])
def test_adjoint_is_the_transpose(L):
    rng = np.random.default_rng(10 + L)
    R = 1 << L
    x = rng.normal(size=(5, R, R, 4))
    v = rng.normal(size=(5, (4 ** (L + 1) - 1) // 3, 4))
    lhs = float((O.generate_mipmap(x) * v).sum())
    rhs = float((O.generate_mipmap_bwd(v, L) * x).sum())
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_float32_pyramid_sums_in_the_reference_order():
    # ((a + b) + c + d) / 4 in FP32, not the FP64 mean rounded once
    tex = np.array([1.0, 2.0 ** -24, 2.0 ** -24, 2.0 ** -24], np.float32).reshape(1, 2, 2, 1).repeat(4, -1)
    pyr = O.generate_mipmap(tex)
    a, b, c, d = (np.float32(x) for x in tex[0].reshape(4, 4)[:, 0])
    assert pyr[0, 0, 0] == ((a + b) + c + d) / np.float32(4)

"""FP64 finite differences against the oracle's spherical-harmonics adjoint
(the restatement of compute_sh_bwd.cu / spherical_harmonics.cuh:17-387),
degrees 0 to 4: the coefficient gradient (the colour is linear in the
coefficients) and the direction gradient (through the normalisation of the
view direction), plus masked entries, which have neither output nor gradient
(the reference leaves a masked entry's colour uninitialised,
compute_sh_fwd.cu:56; the oracle and the kernels write 0).
"""
import numpy as np
import pytest

from oracle import oracle as O

F64 = np.float64


def _case(degree, n=64, seed=0):
    rng = np.random.default_rng(seed + degree)
    K = (degree + 1) ** 2
    dirs = rng.normal(size=(n, 3)) * rng.uniform(0.5, 3.0, size=(n, 1))  # not unit length: normalised inside
    coeffs = rng.normal(size=(n, K, 3))
    w = rng.normal(size=(n, 3))
    return dirs, coeffs, w


def _loss(degree, dirs, coeffs, w, masks=None):
    return float((O.sh_fwd(degree, dirs, coeffs, masks, dtype=F64) * w).sum())


@pytest.mark.parametrize("degree", range(5))
def test_coefficient_gradient_matches_finite_differences(degree):
    dirs, coeffs, w = _case(degree)
    v_coeffs, _ = O.sh_bwd(degree, dirs, coeffs, w, dtype=F64)
    d = np.random.default_rng(1).normal(size=coeffs.shape)
    h = 0.1
    fd = (_loss(degree, dirs, coeffs + h * d, w) - _loss(degree, dirs, coeffs - h * d, w)) / (2 * h)
    assert abs(fd - (v_coeffs * d).sum()) <= 1e-11 * max(1.0, abs(fd))


@pytest.mark.parametrize("degree", range(1, 5))
def test_direction_gradient_matches_finite_differences(degree):
    dirs, coeffs, w = _case(degree)
    _, v_dirs = O.sh_bwd(degree, dirs, coeffs, w, dtype=F64)
    rng = np.random.default_rng(2)
    h = 1e-6
    for _ in range(4):
        d = rng.normal(size=dirs.shape)
        fd = (_loss(degree, dirs + h * d, coeffs, w) - _loss(degree, dirs - h * d, coeffs, w)) / (2 * h)
        an = float((v_dirs * d).sum())
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (degree, fd, an)


def test_degree_zero_has_no_direction_gradient():
    dirs, coeffs, w = _case(0)
    _, v_dirs = O.sh_bwd(0, dirs, coeffs, w, dtype=F64)
    assert not v_dirs.any()


@pytest.mark.parametrize("degree", [1, 3])
def test_masked_entries_have_no_output_or_gradient(degree):
    dirs, coeffs, w = _case(degree)
    masks = np.arange(len(dirs)) % 3 != 0
    out = O.sh_fwd(degree, dirs, coeffs, masks, dtype=F64)
    v_coeffs, v_dirs = O.sh_bwd(degree, dirs, coeffs, w, masks, dtype=F64)
    assert not out[~masks].any() and not v_coeffs[~masks].any() and not v_dirs[~masks].any()
    assert out[masks].any() and v_dirs[masks].any()

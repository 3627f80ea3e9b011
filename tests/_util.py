"""Comparison helpers shared by the parity tests."""
import numpy as np


def to_np(t):
    return t.detach().float().cpu().numpy() if hasattr(t, "detach") else np.asarray(t)


def close_report(a, b, atol, rtol):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    err = np.abs(a - b)
    bad = err > atol + rtol * np.abs(b)
    return int(bad.sum()), float(err.max() if err.size else 0.0)


def assert_close(a, b, atol, rtol=0.0, max_bad_frac=0.0, name=""):
    """Elementwise |a-b| <= atol + rtol*|b|, allowing a stated fraction of
    outliers (pixels whose discrete branch -- the 1/255 alpha cut, the 1e-4
    transmittance stop, a bilinear tap switch -- flips on a 1-ulp input change)."""
    nbad, emax = close_report(a, b, atol, rtol)
    n = max(np.asarray(b).size, 1)
    assert nbad <= max_bad_frac * n, f"{name}: {nbad}/{n} elements outside atol={atol} rtol={rtol} (max err {emax})"


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def cosine(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-300))

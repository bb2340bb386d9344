"""Shared helpers of the parity tests."""
import numpy as np


def rel_max_err(a, b):
    """max_i |a_i - b_i| / max_i |b_i| per variable (columns), maximum over
    variables: the residual parity metric (a per-cell relative error is
    meaningless where R ~ 0 in uniform flow)."""
    a = np.asarray(a).reshape(-1, 4)
    b = np.asarray(b).reshape(-1, 4)
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return float("inf")
    a = np.nan_to_num(a)
    b = np.nan_to_num(b)
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return float((np.abs(a - b).max(axis=0) / scale).max())


def l1_linf(a, b):
    d = np.abs(np.asarray(a) - np.asarray(b))
    return float(d.mean()), float(d.max())


def sod_frobenius(case, prim, gold):
    """check/check.py:33-36 metric: Frobenius norm of (x, rho, u) differences
    against the golden CSV (CSV rows sorted by x)."""
    x = case.mesh()["cell_bary"][:, 0]
    o = np.argsort(x, kind="stable")
    out = np.stack([x[o], prim[o, 0], prim[o, 1]], 1)
    g = np.stack([gold["x"], gold["rho"], gold["u"]], 1)
    return float(np.sqrt(((g - out) ** 2).sum()))

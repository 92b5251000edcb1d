"""Comparison helpers shared by the parity tests."""
import numpy as np


def split_packed(hs, hsdiag):
    """The four regions of the packed state: H strict lower, H diagonal
    (in HS), S strict upper, S diagonal (HSDIAG)."""
    n = hs.shape[0]
    il = np.tril_indices(n, -1)
    iu = np.triu_indices(n, 1)
    return {"H_lower": hs[il], "H_diag": np.diag(hs).copy(), "S_upper": hs[iu], "S_diag": hsdiag.copy()}


def rel_errors(hs, hsd, hs_ref, hsd_ref):
    """max |x - ref| / max |ref| for H (lower + diagonal) and S (upper +
    HSDIAG): the per-matrix relative error the parity tolerance is on."""
    a = split_packed(hs, hsd)
    b = split_packed(hs_ref, hsd_ref)
    out = {}
    for m, keys in (("H", ("H_lower", "H_diag")), ("S", ("S_upper", "S_diag"))):
        num = max(float(np.max(np.abs(a[k] - b[k]))) if b[k].size else 0.0 for k in keys)
        den = max(float(np.max(np.abs(b[k]))) if b[k].size else 0.0 for k in keys)
        out[m] = num / den if den > 0 else num
    return out

"""Known answers from the reference's own shipped MgO runs (CPU only).

tests/golden/mgo_golden.json was extracted by tests/golden/make_golden.py
from SRC_elast/example-MgO/elast/{tetra,eos,rhomb}: the lapw1 MATRIX SIZE
of every k-point and the star expansion SETWAR printed for the warped
interstitial potential.
"""
import json
import os

import numpy as np
import pytest

from hack_wein2k_b200 import lattice, warp

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mgo_golden.json")))


def _case(name):
    return GOLD["cases"][name]


@pytest.mark.parametrize("name", ["tetra", "eos", "rhomb"])
def test_basis_size_per_kpoint(name):
    """COORS reproduces the plane-wave count NV the reference printed at
    every k ('MATRIX SIZE' of the 2001 build's PRTKPT) and NV + NLO the
    size its solver printed ('matrix size')."""
    c = _case(name)
    st, in1 = c["struct"], c["in1"]
    br2, ortho, pia = lattice.latgen(st["lattic"], *st["abc"], *st["angles"])
    rmin = min(a["rmt"] for a in st["atoms"])
    rkm = in1["rkmax"] / rmin
    nlo = sum((2 * l + 1) * a["mult"] for a, los in zip(st["atoms"], in1["lo_l"]) for l in los)
    assert len(c["kpoints"]) == c["n_klist"]
    bad = []
    for e in c["kpoints"]:
        ix, iy, iz, idv = e["k"]
        kzz, xk, yk, zk, rk = lattice.coors(rkm, np.array([ix, iy, iz]) / idv, br2, ortho, pia, st["lattic"])
        if len(rk) != e["nv"] or (e["hsrows"] is not None and len(rk) + nlo != e["hsrows"]):
            bad.append((e["k"], len(rk), nlo, e["nv"], e["hsrows"]))
    assert not bad, bad[:5]
    assert sum(e["hsrows"] is not None for e in c["kpoints"]) > 0.9 * len(c["kpoints"])


def test_lopw_rows_for_tetra_gamma():
    """LOPW picks the NLO rows at Gamma without exhausting the plane waves;
    HSROWS = NV + NLO = 199 + 5, the sizes the reference printed."""
    c = _case("tetra")
    st, in1 = c["struct"], c["in1"]
    br2, ortho, pia = lattice.latgen(st["lattic"], *st["abc"], *st["angles"])
    rkm = in1["rkmax"] / min(a["rmt"] for a in st["atoms"])
    mult = [a["mult"] for a in st["atoms"]]
    ilo = np.zeros((len(mult), 4), dtype=int)
    for i, los in enumerate(in1["lo_l"]):
        for l in los:
            ilo[i, l] += 1
    pos = np.array([p for a in st["atoms"] for p in a["pos"]])
    rot = np.stack([np.eye(3)] * len(pos))
    nv, kzz, xk, yk, zk, rk = lattice.basis(rkm, np.zeros(3), br2, ortho, pia, st["lattic"], mult, ilo, pos,
                                            rot, np.stack([np.eye(3)] * len(mult)))
    assert nv == 199 and len(rk) == 204


@pytest.mark.parametrize("name", ["tetra", "eos", "rhomb"])
def test_setwar_star_expansion(name):
    """STERN members in the printed order, their tau phases and
    WARPING = POTK conj(TAUP) (printed to 5 decimals)."""
    c = _case(name)
    imat, tau = warp.symops_from_struct(c["struct"]["symops"])
    stars = c["stars"]
    potk = {tuple(p[:3]): complex(p[3], p[4]) for p in c["potk"]}
    checked = 0
    for s in stars:
        k = tuple(s["k"])
        kkk, taup = warp.stern(list(k), imat, tau)
        assert len(kkk) == s["ind"]
        for m, (kk, tp) in enumerate(zip(kkk, taup)):
            if m >= len(s["members"]):
                break
            g = s["members"][m]
            assert kk == g["wave"], (k, m, kk, g["wave"])
            assert abs(tp.real - g["taup"][0]) <= 6e-6 and abs(tp.imag - g["taup"][1]) <= 6e-6
            if k in potk:
                w = potk[k] * np.conj(tp)
                assert abs(w.real - g["warping"][0]) <= 6e-6 and abs(w.imag - g["warping"][1]) <= 6e-6
                checked += 1
    assert checked > 0


def test_setwar_table_is_hermitian_for_centrosymmetric_mgo():
    """The star-expanded table of MgO (inversion symmetric) is real and
    symmetric under G -> -G, as the REAL build of the reference assumes."""
    c = _case("eos")
    imat, tau = warp.symops_from_struct(c["struct"]["symops"])
    pk = [(p[0], p[1], p[2], complex(p[3], p[4])) for p in c["potk"]]
    tab, (w1, w2, w3), _ = warp.setwar(pk, imat, tau)
    assert np.allclose(tab, tab[::-1, ::-1, ::-1].conj(), atol=1e-12)

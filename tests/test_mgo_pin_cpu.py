"""End-to-end pin of the H/S setup against the reference's own MgO runs (CPU).

tests/golden/mgo_atpar.json holds the input files of the reference's
shipped MgO SCF runs (SRC_elast/example-MgO/elast/{eos,rhomb,tetra}: case.struct,
case.in1, case.klist and the case.vsp / case.vns potentials of the cycle
whose lapw1 output is kept) and the numbers that lapw1 printed:
  * the searched energy parameters, the POTENTIAL PARAMETERS table
    (U, U', Udot, Udot', |Udot|^2 per l, 6 significant digits), the LO
    coefficients (5 decimals) and the Gaunt factors and radial integrals of
    the non-spherical potential (8 decimals), all from ATPAR;
  * the eigenvalues of every k-point (7 decimals).
The host ATPAR (hack_wein2k_b200.atpar) is checked against the first list
to the printed precision, and the full chain (case files -> ATPAR -> COORS
/ LOPW -> HAMILT + HNS in the oracle -> generalized eigen-solve) against the
eigenvalues.  The runs were made in 2001 with the REAL build of an older
lapw1 (its LO-row print differs from this tree's source); the eigenvalues
agree to 2.5e-5 Ry, and the tolerance is 5e-5 Ry.
"""
import json
import os

import numpy as np
import pytest
import scipy.linalg

from hack_wein2k_b200 import atpar as AP
from hack_wein2k_b200 import case_files as CF
from hack_wein2k_b200.problem import hermitian_from_packed
from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mgo_atpar.json")))
TOL_EIG_RY = 5.0e-5


class Case:
    def __init__(self, name):
        c = GOLD["cases"][name]
        f = c["files"]
        self.name = name
        self.struct = CF.read_struct(f["struct"])
        nat = len(self.struct.atoms)
        self.in1 = CF.read_in1(f["in1"], nat)
        npts = [a.jrj for a in self.struct.atoms]
        self.vsp = CF.read_vsp(f["vsp"], npts)
        self.vns = CF.read_vns(f["vns"], npts)
        self.klist = CF.read_klist(f["klist"])
        self.printed = c["atpar"]
        self.eig = c["eigenvalues"]
        self.rads = AP.atpar(self.struct, self.in1, self.vsp, self.vns, self.in1.lmax + 1, self.in1.lnsmax)

    def kpoint(self, block):
        """The klist k of an eigenvalue block (matched on the printed k)."""
        kp = np.array(self.eig[block]["kprint"])
        best = min(self.klist, key=lambda e: float(np.abs(np.array(e[1]) / e[2] - kp).sum()))
        k = np.array(best[1], dtype=np.float64) / best[2]
        assert np.abs(k - kp).max() < 1e-5
        return k

    def problem(self, block, tns=None):
        return AP.problem_from_case(self.struct, self.in1, self.vsp, self.vns, self.kpoint(block), rads=self.rads,
                                    tns=tns, name=f"{self.name}-k{block}")


# per run: lattice, symmetry operations, LM terms of the potential per atom, k-points
RUNS = {"eos": ("F", 48, 4, 165), "rhomb": ("R", 12, 6, 489), "tetra": ("F", 16, 5, 405)}


@pytest.fixture(scope="module", params=sorted(RUNS))
def case(request):
    return Case(request.param)


def test_case_file_readers(case):
    st = case.struct
    assert len(st.atoms) == 2 and [a.name for a in st.atoms] == ["Mg", "O"]
    assert all(a.jrj == 781 and abs(a.rmt - 1.7) < 1e-12 for a in st.atoms)
    lattic, nsym, nlm, nk = RUNS[case.name]
    assert st.lattic == lattic
    assert len(st.imat) == nsym
    assert case.in1.rkmax == 8.0 and case.in1.lmax == 10 and case.in1.lnsmax == 4
    assert (case.in1.emin, case.in1.emax) == (-7.0, 1.5)
    assert all(len(v) == 781 for v in case.vsp)
    assert [len(x) for x in case.vns.lm] == [nlm, nlm]
    assert len(case.vns.potk) > 50 and case.vns.potk[0][:3] == (0, 0, 0)
    assert len(case.klist) == nk


def test_energy_search_matches_printed(case):
    for rad, pr in zip(case.rads, case.printed):
        searched = [e for e in pr["energies"] if e["bottom"] is not None]
        assert len(searched) == len(rad.searched)
        for (l, e, eb, et), p in zip(rad.searched, searched):
            assert l == p["l"]
            assert abs(e - p["e"]) < 6e-5 and abs(eb - p["bottom"]) < 6e-4 and abs(et - p["top"]) < 6e-4


def test_radial_parameters_match_printed(case):
    """U(R), U'(R), DU/DE, DU'/DE, NORM-U' per l to the printed 6 digits."""
    lt = case.in1.lmax + 1
    for rad, pr in zip(case.rads, case.printed):
        for row in pr["params"][:lt]:
            l = row[0]
            mine = [rad.p[l], rad.dp[l], rad.pe[l], rad.dpe[l], rad.pei[l]]
            for x, y in zip(mine, row[1:6]):
                assert abs(x - y) <= 6e-6 * abs(y) + 1e-12, (l, mine, row)
            assert tuple(rad.nodes[l]) == tuple(row[6:9])


def test_local_orbitals_match_printed(case):
    for rad, pr in zip(case.rads, case.printed):
        # the LO rows print U(R) and U'(R) of the LO function first
        for row in pr["params"][case.in1.lmax + 1:]:
            l = row[0]
            assert abs(rad.plo[l] - row[1]) <= 6e-6 * abs(row[1]) and abs(rad.dplo[l] - row[2]) <= 6e-6 * abs(row[2])
        assert len(pr["lo_coef"]) == int(rad.ilo.sum())
        for l, a, b, c in pr["lo_coef"]:
            assert abs(rad.alo[0, l] - a) < 6e-6 and abs(rad.blo[0, l] - b) < 6e-6 and abs(rad.clo[0, l] - c) < 6e-6


def test_gaunt_factors_and_radial_integrals_match_printed(case):
    """GNT and U V U, UE V UE, U V UE (and the LO integrals) to 8 decimals."""
    n = 0
    for rad, pr in zip(case.rads, case.printed):
        gmap = {}
        for (l0, ll, lp, lmx, m, mp, g) in rad.gaunts:
            gmap.setdefault((l0, ll, lp, m, mp), []).append(g)
        for e in pr["nonspherical"]:
            l0, ll, lp, m, _mm, mp = e["idx"]
            cands = gmap.get((l0, ll, lp, m, mp), [])
            assert any(abs(g.real - e["gnt"][0]) < 6e-9 and abs(g.imag - e["gnt"][1]) < 6e-9 for g in cands), e
            if "v" in e:
                got = (rad.vnslo if e["lo"] else rad.vns)[(l0, e["lm1"], lp)]
                assert max(abs(x - y) for x, y in zip(got, e["v"])) < 6e-9, (e, got)
                n += 1
    assert n > 40


@pytest.mark.parametrize("block", [0, 1, 7, 40])
def test_eigenvalues_match_printed_through_the_oracle(case, block):
    """case files -> ATPAR -> basis -> oracle HAMILT + HNS -> eigen-solve:
    every eigenvalue lapw1 printed in the window [EMIN, EMAX] within 5e-5 Ry,
    and the plane-wave count it printed (MATRIX SIZE)."""
    p = case.problem(block)
    assert p.nv == case.eig[block]["size"]
    hs, hsd = O.setup(p)
    H, S = hermitian_from_packed(hs, hsd)
    w = scipy.linalg.eigh(H, S, eigvals_only=True)
    w = w[(w > case.in1.emin) & (w < case.in1.emax)]
    e0 = np.array(case.eig[block]["eig"])
    assert len(w) == len(e0)
    assert np.abs(w - e0).max() <= TOL_EIG_RY, np.abs(w - e0).max()


def test_vector_file_round_trip(case):
    """case.vector as lapw1 writes it (inilpw.f:440-445, tapewf.F:44-59):
    the header records of every atom, then per k-point the k line, the KZZ
    of all HSROWS rows and each state's energy and conjugated eigenvector,
    every record framed by its 4-byte length; read back unchanged."""
    import io
    import struct

    from hack_wein2k_b200 import vector_file as VF
    p = case.problem(0)
    hs, hsd = O.setup(p)
    H, S = hermitian_from_packed(hs, hsd)
    w, Z = scipy.linalg.eigh(H, S)
    sel = (w > case.in1.emin) & (w < case.in1.emax)
    w, Z = w[sel], Z[:, sel]
    buf = io.BytesIO()
    VF.write_header(buf, p.e, p.elo)
    VF.write_kpoint(buf, p.meta["k"], "1", p.kzz, w, Z, 1.0, "")
    raw = buf.getvalue()
    assert struct.unpack("<i", raw[:4])[0] == 8 * p.e.shape[1]          # E(1:LMAX) of atom 1
    head, kps = VF.read_vector(io.BytesIO(raw), p.nat)
    assert np.array_equal(head[0][0], p.e[0]) and np.array_equal(head[1][1], p.elo[1].reshape(-1))
    (kp,) = kps
    assert kp["kzz"].shape == (p.n, 3) and np.array_equal(kp["kzz"], p.kzz)
    assert np.array_equal(kp["eig"], w) and np.array_equal(kp["z"], Z)
    lines = VF.energy_lines(p.meta["k"], "1", p.n, w, 1.0)
    assert len(lines) == 1 + len(w) and len(lines[0]) == 3 * 19 + 10 + 12 + 5 + 3


def test_nsh_file_round_trip(case):
    """case.nsh as ATPAR/FORFHS write it for lapw2's forces (atpar.f:112,
    345, 563-570; forfhs.f:26-69): one entry per LQNS Gaunt factor of each
    atom, GFAC times the radial integrals, LO lines where l0 or lp <= LOMAX;
    read back to the 12 printed digits.  The factors themselves are pinned
    to lapw1's own print by the Gaunt/integral test above."""
    import io

    from hack_wein2k_b200 import vector_file as VF
    buf = io.StringIO()
    VF.write_nsh(buf, case.rads)
    text = buf.getvalue()
    assert text.splitlines()[0].startswith(" non-spherical Matrixelements x Gaunt-Coefficient")
    got = VF.read_nsh(io.StringIO(text))
    assert sorted(got) == [1, 2]
    for ja, rad in enumerate(case.rads):
        ents = got[ja + 1]
        assert len(ents) == len(rad.gaunts) > 0
        for e, (l0, ll, lp, lm1, m, mp, g) in zip(ents, rad.gaunts):
            assert e["idx"] == (l0, ll, lp, m, rad.lm[lm1 - 1][1], mp)
            uvu, dvd, uvd = rad.vns[(l0, lm1, lp)]
            want = [g * uvu, g * dvd, g * uvd, g * rad.vns[(lp, lm1, l0)][2]]
            assert all(abs(x - y) <= 1e-11 * max(1.0, abs(y)) for x, y in zip(e["t"], want)), (e, want)
            assert (e["lo"] is not None) == (l0 <= 3 or lp <= 3)
            if e["lo"] is not None and l0 <= 3 and rad.loor[l0]:
                assert abs(e["lo"][0] - g * rad.vnslo[(l0, lm1, lp)][0]) <= 1e-11 * max(1.0, abs(e["lo"][0]))

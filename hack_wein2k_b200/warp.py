"""Interstitial warped-potential table: SETWAR / STERN on the host.

The drop-in takes the WARP(-W1:W1,-W2:W2,-W3:W3) table the Fortran host
builds once per run (INIKPT -> SETWAR); this module builds the same table
from the interstitial plane-wave list of case.vns:

  rdswar  SRC_lapw1/rdswar.f:19-30   read JA,JB,JC,POTK of the star heads
  stern   SRC_lapw1/stern.F:44-91    star of one reciprocal vector and its
                                     tau phases (averaged over the group
                                     operations that map onto a member)
  setwar  SRC_lapw1/setwar.f:83-117  WARP(KKK) = POTK * conj(TAUP)
"""
from __future__ import annotations

import math

import numpy as np


def stern(g, imat, tau):
    """Members and tau phases of the star of g.

    imat[i][j][l] = IMAT(j+1, l+1, i+1), tau[i][j] = TAU(j+1, i+1)."""
    tpi = 8.0 * math.atan(1.0)
    kkk, taup, index = [], [], []
    for i in range(len(imat)):
        tk = 0.0
        k = [0, 0, 0]
        for j in range(3):
            tk = tk + tau[i][j] * g[j] * tpi
            s = 0
            for l in range(3):
                s = imat[i][j][l] * g[l] + s
            k[j] = s
        found = -1
        for m in range(len(kkk)):
            if kkk[m] == k:
                found = m
                break
        if found >= 0:
            taup[found] = taup[found] + complex(math.cos(tk), math.sin(tk))
            index[found] += 1
        else:
            kkk.append(k)
            taup.append(complex(math.cos(tk), math.sin(tk)))
            index.append(1)
    taup = [t / c for t, c in zip(taup, index)]
    return kkk, taup


def symops_from_struct(ops):
    """[{imat: rows as written in case.struct, tau}] -> (imat[i][j][l], tau[i][j]).

    case.struct writes operation i as three lines r = 1..3 holding
    IMAT(1..3, r) and TAU(r) (latgen.f:311-315)."""
    imat = []
    tau = []
    for op in ops:
        m = [[0] * 3 for _ in range(3)]
        for r in range(3):
            for j1 in range(3):
                m[j1][r] = op["imat"][r][j1]
        imat.append(m)
        tau.append(list(op["tau"]))
    return imat, tau


def setwar(potk, imat, tau):
    """Star-expanded WARP table.  potk: [(ja, jb, jc, complex)].  Returns
    (warp [2w3+1, 2w2+1, 2w1+1] complex, (w1, w2, w3), stars) where stars
    lists the members and phases per input vector in setwar.f's order."""
    entries = {}
    stars = []
    for ja, jb, jc, v in potk:
        kkk, taup = stern([ja, jb, jc], imat, tau)
        stars.append((kkk, taup))
        for k, t in zip(kkk, taup):
            entries[tuple(k)] = v * np.conj(t)
    w = [max(abs(k[c]) for k in entries) if entries else 0 for c in range(3)]
    warp = np.zeros((2 * w[2] + 1, 2 * w[1] + 1, 2 * w[0] + 1), dtype=np.complex128)
    for (x, y, z), v in entries.items():
        warp[z + w[2], y + w[1], x + w[0]] = v
    return warp, tuple(w), stars

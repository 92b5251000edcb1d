"""Host-side basis construction: lattice, |k+G| plane-wave list, LO rows.

These are the callers on the input side of the H/S setup.  They stay on the
host in the drop-in (the boundary takes KZZ/XK/YK/ZK/RK as given and never
re-sorts them), so they are written with numpy here:

  latgen  SRC_lapw1/latgen.f:39-301   reciprocal basis BR2, ORTHO flag
  coors   SRC_lapw1/coors.f:47-210    k+G list with |k+G| <= RKM, sorted by
                                      length (ties keep generation order)
  lopw    SRC_lapw1/lopw.f:42-128     one k+G per local-orbital row, chosen
                                      by Gram-Schmidt on phase x Y_lm
  ylm     SRC_lapw1/ylm.f:162-263     Condon-Shortley Y_lm, vectorised
"""
from __future__ import annotations

import math

import numpy as np

TPI = 2.0 * math.pi


def latgen(lattic: str, a: float, b: float, c: float,
           alpha: float = 90.0, beta: float = 90.0, gamma: float = 90.0):
    """Reciprocal basis BR2 (columns = reciprocal vectors, Cartesian, 1/bohr),
    ORTHO flag and PIA = 2 pi / (a, b, c) as latgen.f:39-301 builds them.
    Angles in degrees."""
    pi = 4.0 * math.atan(1.0)
    al = np.array([alpha, beta, gamma]) * pi / 180.0
    pia = np.array([2.0 * pi / a, 2.0 * pi / b, 2.0 * pi / c])
    lat = lattic.strip().upper()
    normalize = True
    if lat[0] == "H":
        br2 = np.array([[2 / math.sqrt(3), 1 / math.sqrt(3), 0], [0, 1, 0], [0, 0, 1.0]])
        ortho = False
    elif lat[0] in "SP":
        right = [abs(x - pi / 2) <= 1e-4 for x in al]
        if all(right):
            br2 = np.eye(3)
            ortho = True
        elif not right[0] or (not right[1] and not right[2]):
            sinbc, cosab, cosac, cosbc = math.sin(al[0]), math.cos(al[2]), math.cos(al[1]), math.cos(al[0])
            wurzel = math.sqrt(sinbc ** 2 - cosac ** 2 - cosab ** 2 + 2 * cosbc * cosac * cosab)
            br2 = np.array([
                [sinbc / wurzel * pia[0], (-cosab + cosbc * cosac) / (sinbc * wurzel) * pia[1],
                 (cosbc * cosab - cosac) / (sinbc * wurzel) * pia[2]],
                [0.0, pia[1] / sinbc, -pia[2] * cosbc / sinbc],
                [0.0, 0.0, pia[2]]])
            ortho, normalize = False, False
        elif not right[2]:
            s, co = math.sin(al[2]), math.cos(al[2])
            br2 = np.array([[pia[0] / s, -pia[1] * co / s, 0], [0, pia[1], 0], [0, 0, pia[2]]])
            ortho, normalize = False, False
        else:
            s, co = math.sin(al[1]), math.cos(al[1])
            br2 = np.array([[pia[0] / s, 0, -pia[2] * co / s], [0, pia[1], 0], [0, 0, pia[2]]])
            ortho, normalize = False, False
    elif lat[0] == "F":
        br2 = np.array([[-1.0, 1, 1], [1, -1, 1], [1, 1, -1]])
        ortho = True
    elif lat[0] == "B":
        br2 = np.array([[0.0, 1, 1], [1, 0, 1], [1, 1, 0]])
        ortho = True
    elif lat[0] == "C":
        if lat[1:3] == "XZ":
            br2 = np.array([[1.0, 0, 1], [0, 1, 0], [-1, 0, 1]])
            ortho = True
        elif lat[1:3] == "YZ":
            br2 = np.array([[1.0, 0, 0], [0, 1, 1], [0, -1, 1]])
            ortho = True
        else:
            br2 = np.array([[1.0, 1, 0], [-1, 1, 0], [0, 0, 1]])
            ortho = True
    elif lat[0] == "R":
        r3 = math.sqrt(3.0)
        br2 = np.array([[1 / r3, 1 / r3, -2 / r3], [-1, 1, 0], [1, 1, 1.0]])
        ortho = False
    else:
        raise ValueError(f"unknown lattice type {lattic!r}")
    br2 = np.array(br2, dtype=np.float64)
    if normalize:
        br2 = br2 * pia[:, None]
    return br2, ortho, pia


def ylm(v: np.ndarray, lmax: int) -> np.ndarray:
    """Y_lm for vectors v[..., 3]; returns [..., (lmax+1)^2] complex, index
    l*l+l+m, following the recursion of ylm.f:162-263."""
    v = np.asarray(v, dtype=np.float64)
    sh = v.shape[:-1]
    v = v.reshape(-1, 3)
    npt = v.shape[0]
    pi = 4.0 * math.atan(1.0)
    Y = np.zeros((npt, (lmax + 1) ** 2 + 1), dtype=np.complex128)   # 1-based like the Fortran
    yllr = 1.0 / math.sqrt(4.0 * pi)
    Y[:, 1] = yllr
    if lmax > 0:
        abmax = np.maximum(np.abs(v[:, 0]), np.abs(v[:, 1]))
        with np.errstate(invalid="ignore", divide="ignore"):
            a = v[:, 0] / abmax
            b = v[:, 1] / abmax
            ab = np.sqrt(a * a + b * b)
            cosph = np.where(abmax > 0, a / ab, 1.0)
            sinph = np.where(abmax > 0, b / ab, 0.0)
            abcmax = np.maximum(abmax, np.abs(v[:, 2]))
            a = v[:, 0] / abcmax
            b = v[:, 1] / abcmax
            c = v[:, 2] / abcmax
            ab = a * a + b * b
            abc = np.sqrt(ab + c * c)
            costh = np.where(abcmax > 0, c / abc, 1.0)
            sinth = np.where(abcmax > 0, np.sqrt(ab) / abc, 0.0)
        Y[:, 3] = math.sqrt(3.0) * yllr * costh
        t1 = -math.sqrt(1.5) * yllr * sinth
        Y[:, 4] = t1 * cosph + 1j * (t1 * sinph)
        Y[:, 2] = -np.conj(Y[:, 4])
        for l in range(2, lmax + 1):
            index = l * l + 1
            index2 = index + 2 * l
            msign = 1 - 2 * (l % 2)
            r1, i1 = Y[:, index - 1].real.copy(), Y[:, index - 1].imag.copy()
            t1 = -math.sqrt((2 * l + 1) / (2 * l)) * sinth
            Y[:, index2] = t1 * (cosph * r1 - sinph * i1) + 1j * (t1 * (cosph * i1 + sinph * r1))
            Y[:, index] = msign * np.conj(Y[:, index2])
            index2 -= 1
            index += 1
            t2 = math.sqrt(2 * l + 1) * costh
            Y[:, index2] = t2 * r1 + 1j * (t2 * i1)
            Y[:, index] = -msign * np.conj(Y[:, index2])
            index2 -= 1
            index += 1
            i4l2 = index2 - 4 * l + 2
            i2l = index2 - 2 * l
            d4ll1c = costh * math.sqrt(4 * l * l - 1)
            d2l13 = -math.sqrt((2 * l + 1) / (2 * l - 3))
            for m in range(l - 2, -1, -1):
                tt1 = 1.0 / math.sqrt((l + m) * (l - m))
                tt2 = d4ll1c * tt1
                tt3 = d2l13 * math.sqrt((l + m - 1) * (l - m - 1)) * tt1
                yr = tt2 * Y[:, i2l].real + tt3 * Y[:, i4l2].real
                yi = tt2 * Y[:, i2l].imag + tt3 * Y[:, i4l2].imag
                Y[:, index2] = yr + 1j * yi
                Y[:, index] = msign * np.conj(Y[:, index2])
                msign = -msign
                index2 -= 1
                index += 1
                i4l2 -= 1
                i2l -= 1
    return Y[:, 1:].reshape(sh + ((lmax + 1) ** 2,))


def rotate(vec: np.ndarray, rotmat_c: np.ndarray) -> np.ndarray:
    """rotate.f:22-28 with ROTMAT given in the C view [col][row] of the
    Fortran ROTMAT(3,3): out_jc = sum_j vec_j ROTMAT(jc, j)."""
    m = np.asarray(rotmat_c).T            # m[row, col] = ROTMAT(row, col)
    out = np.zeros_like(vec)
    for jc in range(3):
        d = 0.0
        for j in range(3):
            d = d + vec[..., j] * m[jc, j]
        out[..., jc] = d
    return out


def coors(rkm: float, sk: np.ndarray, br2: np.ndarray, ortho: bool, pia: np.ndarray,
          lattic: str = "P", nmax: int | None = None):
    """Plane-wave list of coors.f:47-210.  `sk` is the k-point as SETKPT
    stores it (SX1,SY1,SZ1).  Returns kzz [nv,3] int32, xk, yk, zk, rk."""
    sx, sy, sz = (float(x) for x in sk)
    if ortho:
        skx, sky, skz = sx * pia[0], sy * pia[1], sz * pia[2]
    else:
        skx = sx * br2[0, 0] + sy * br2[0, 1] + sz * br2[0, 2]
        sky = sx * br2[1, 0] + sy * br2[1, 1] + sz * br2[1, 2]
        skz = sx * br2[2, 0] + sy * br2[2, 1] + sz * br2[2, 2]
    # box large enough for every |k+G| <= rkm (the reference doubles NVEC
    # until its check at coors.f:172-201 passes; any large enough box gives
    # the same list, generation order being lexicographic in (JA,JB,JC))
    binv = np.linalg.inv(br2)
    kk = math.sqrt(skx * skx + sky * sky + skz * skz)
    ext = [int(math.ceil(np.linalg.norm(binv[i]) * (rkm + kk))) + 2 for i in range(3)]
    ja = np.arange(-ext[0], ext[0] + 1)
    jb = np.arange(-ext[1], ext[1] + 1)
    jc = np.arange(-ext[2], ext[2] + 1)
    JA, JB, JC = np.meshgrid(ja, jb, jc, indexing="ij")
    JA, JB, JC = JA.ravel(), JB.ravel(), JC.ravel()
    sbx = skx + JA * br2[0, 0] + JB * br2[0, 1] + JC * br2[0, 2]
    sby = sky + JA * br2[1, 0] + JB * br2[1, 1] + JC * br2[1, 2]
    sbz = skz + JA * br2[2, 0] + JB * br2[2, 1] + JC * br2[2, 2]
    rkq = np.sqrt(sbx * sbx + sby * sby + sbz * sbz)
    sel = np.nonzero(rkq <= rkm)[0]
    order = sel[np.argsort(rkq[sel], kind="stable")]
    if nmax is not None and len(order) > nmax:
        raise ValueError(f"basis of {len(order)} plane waves exceeds NMATMAX-NLO={nmax}")
    sbx, sby, sbz, rkq = sbx[order], sby[order], sbz[order], rkq[order]
    if ortho:
        kzz = np.empty((len(order), 3), dtype=np.int32)
        for c, (s, sv) in enumerate(((sbx, sx), (sby, sy), (sbz, sz))):
            q = s / pia[c] - sv
            kzz[:, c] = np.trunc(q + np.copysign(1.0e-2, q)).astype(np.int32)
    else:
        kzz = np.stack([JA[order], JB[order], JC[order]], axis=1).astype(np.int32)
        if lattic.strip().upper().startswith("CXZ"):
            a_, b_, c_ = kzz[:, 0].copy(), kzz[:, 1].copy(), kzz[:, 2].copy()
            kzz = np.stack([a_ + c_, b_, -a_ + c_], axis=1).astype(np.int32)
    return kzz, sbx.copy(), sby.copy(), sbz.copy(), rkq.copy()


def lopw(nv: int, kzz, xk, yk, zk, mult, ilo, pos, rotij, rotloc, lomax: int = 3):
    """Local-orbital rows of lopw.f:42-128: for each (atom type, l, jlo) and
    each (equivalent atom, m) the next plane wave whose phase x Y_lm vector
    is linearly independent (Gram-Schmidt norm > 1e-3) of those taken."""
    kzz = np.asarray(kzz)
    out_k, out_x, out_y, out_z = [], [], [], []
    tpi = 8.0 * math.atan(1.0)
    ia1 = 0
    nat = len(mult)
    for n in range(nat):
        for l in range(lomax + 1):
            for _jlo in range(int(ilo[n][l])):
                lmdn, lmup = l * l + 1, (l + 1) * (l + 1)
                index = 0
                nbm = int(mult[n]) * (1 + lmup - lmdn)
                hh = np.zeros((nbm, nbm), dtype=np.complex128)
                nb = 0
                for _ieq in range(int(mult[n])):
                    for _lm in range(lmdn, lmup + 1):
                        nb += 1
                        while True:
                            index += 1
                            if index > nv:
                                raise RuntimeError("LOPW: plane waves exhausted")
                            kk = kzz[index - 1]
                            vec = np.array([xk[index - 1], yk[index - 1], zk[index - 1]])
                            if nbm == 1:
                                break
                            rkgm = math.sqrt(vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2])
                            col = np.zeros(nbm, dtype=np.complex128)
                            iix = 0
                            for natx in range(int(mult[n])):
                                natxx = ia1 + natx
                                sxp = kk[0] * pos[natxx][0] + kk[1] * pos[natxx][1] + kk[2] * pos[natxx][2]
                                sf = complex(math.cos(tpi * sxp), math.sin(tpi * sxp))
                                if rkgm <= 1.0e-5:
                                    yl = np.zeros((lomax + 1) ** 2, dtype=np.complex128)
                                    yl[0] = 1.0
                                else:
                                    r1 = rotate(vec, rotij[natxx])
                                    r2 = rotate(r1, rotloc[n])
                                    yl = ylm(r2, lomax)
                                for lmx in range(lmdn, lmup + 1):
                                    col[iix] = sf * yl[lmx - 1]
                                    iix += 1
                            for j in range(nb - 1):
                                cc = np.sum(col * np.conj(hh[:, j]))
                                col = col - cc * hh[:, j]
                            hl = float(np.sum(np.conj(col) * col).real)
                            if hl > 1.0e-3:
                                hh[:, nb - 1] = col / math.sqrt(hl)
                                break
                        out_k.append(kzz[index - 1].copy())
                        out_x.append(xk[index - 1])
                        out_y.append(yk[index - 1])
                        out_z.append(zk[index - 1])
        ia1 += int(mult[n])
    if not out_k:
        return (np.zeros((0, 3), np.int32),) + (np.zeros(0),) * 3
    return (np.array(out_k, dtype=np.int32), np.array(out_x), np.array(out_y), np.array(out_z))


def kzz_matrix(br2, ortho, pia, lattic="P"):
    """B with Cartesian k+G = k + B @ KZZ for the KZZ convention of COORS:
    conventional indices (B = diag PIA) for ORTHO lattices (coors.f:123-129),
    BR2 otherwise, with the CXZ relabelling of coors.f:135-139 folded in."""
    if ortho:
        return np.diag(np.asarray(pia, dtype=np.float64))
    b = np.asarray(br2, dtype=np.float64)
    if lattic.strip().upper().startswith("CXZ"):
        t = np.array([[0.5, 0.0, -0.5], [0.0, 1.0, 0.0], [0.5, 0.0, 0.5]])
        b = b @ t
    return b


def basis(rkm, sk, br2, ortho, pia, lattic, mult, ilo, pos, rotij, rotloc):
    """COORS followed by LOPW: all HSROWS rows."""
    kzz, xk, yk, zk, rk = coors(rkm, sk, br2, ortho, pia, lattic)
    nv = len(rk)
    lk, lx, ly, lz = lopw(nv, kzz, xk, yk, zk, mult, ilo, pos, rotij, rotloc)
    lr = np.sqrt(lx * lx + ly * ly + lz * lz)
    return (nv, np.concatenate([kzz, lk]), np.concatenate([xk, lx]), np.concatenate([yk, ly]),
            np.concatenate([zk, lz]), np.concatenate([rk, lr]))

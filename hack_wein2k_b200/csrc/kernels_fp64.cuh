// kernels_fp64.cuh -- FP64 kernels of the lapw1 H/S setup (sm_100a).
//
// Data layout in HBM for one k-point (rows = HSROWS = nv + nlo, padded):
//   al, bl     [nat][ltop][nvpad]  f64    matching coefficients (K-a)
//   phase      [ndf][npad]         c128   exp(2 pi i K_n . r_a) of every row
//   tab        [(2d3+1)(2d2+1)(2d1+1)] 2 x c128: (Theta(dK), WARP(dK))
//   hns L / R  [ndf*2*nsl2][npad]  c128   HNS left (A2,B2) / right (ALM,BLM)
//   hs         n x n c128, column-major (the caller's HS), hsdiag n c128
#pragma once
#include "common.cuh"

struct DevProb {
  int n, nv, nlo, nat, ndf, ltop, ldl, lnsmax, ins;
  int nvpad, npad;
  double vi;
  // structure
  const int* mult;
  const int* atype;     // [ndf] 0-based type of atom a
  const int* afirst;    // [nat] first atom index of type
  const double* rmt;
  const double* v;
  const double* pos;    // [ndf][3]
  const double* rotij;  // [ndf][9]
  const double* rotloc; // [nat][9]
  // rows
  const int* kzz;       // [n][3]
  const double* xk;
  const double* yk;
  const double* zk;
  const double* rk;
  // radial [nat][ldl]
  const double* p;
  const double* pe;
  const double* dp;
  const double* dpe;
  const double* pei;
  const double* e;
  const int* lapw;
  // LO
  const int* ilo;
  const int* loor;
  const double* alo;
  const double* blo;
  const double* clo;
  const double* elo;
  const double* pi12lo;
  const double* pe12lo;
  const double* dplo;
  // derived
  double* al;
  double* bl;
  double2* phase;
};

// ---------------------------------------------------------------------
// K-a: AL/BL (hamilt.F:160-175), one thread per (row n < nv, atom type)
// ---------------------------------------------------------------------
__global__ void k_albl(DevProb P, int* status) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  int jn = blockIdx.y;
  if (n >= P.nvpad) return;
  const int ltop = P.ltop;
  double* al = P.al + ((size_t)jn * ltop) * P.nvpad + n;
  double* bl = P.bl + ((size_t)jn * ltop) * P.nvpad + n;
  if (n >= P.nv) {
    for (int l = 0; l < ltop; l++) {
      al[(size_t)l * P.nvpad] = 0.0;
      bl[(size_t)l * P.nvpad] = 0.0;
    }
    return;
  }
  double fj[L1G_MAXL + 2], dfj[L1G_MAXL + 2];
  double rkn = P.rk[n], r = P.rmt[jn];
  int st = dev_sphbes(ltop - 1, r * rkn, fj);
  if (st) atomicOr(status, st);
  dev_dvbes1(fj, dfj, rkn, r, ltop);
  const double* U = P.p + jn * P.ldl;
  const double* UP = P.pe + jn * P.ldl;
  const double* DU = P.dp + jn * P.ldl;
  const double* DUP = P.dpe + jn * P.ldl;
  const int* LAPW = P.lapw + jn * P.ldl;
  for (int l = 0; l < ltop; l++) {
    double a, b;
    if (LAPW[l]) {
      a = rkn * dfj[l] * UP[l] - fj[l] * DUP[l];
      b = fj[l] * DU[l] - rkn * dfj[l] * U[l];
    } else {
      a = fj[l] / U[l] / (r * r);
      b = 0.0;
    }
    al[(size_t)l * P.nvpad] = a;
    bl[(size_t)l * P.nvpad] = b;
  }
}

// structure-factor phases of every row for every atom (hns.F:171-174)
__global__ void k_phase(DevProb P) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  int a = blockIdx.y;
  if (n >= P.npad) return;
  double2 v = cmk(0.0, 0.0);
  if (n < P.n) {
    const double* r = P.pos + 3 * a;
    const int* k = P.kzz + 3 * n;
    double s = r[0] * (double)k[0] + r[1] * (double)k[1] + r[2] * (double)k[2];
    v = cexp2pi(s);
  }
  P.phase[(size_t)a * P.npad + n] = v;
}

// ---------------------------------------------------------------------
// K-c table: Theta(dK) and WARP(dK) on the integer box of row differences.
//   INS == 0: Theta(dK != 0) = sum_type 3 V PHASE BESR  (hamilt.F:297-326)
//             Theta(0)       = sum_type (1/NAT - V MULT) (hamilt.F:328-329)
//   INS != 0: USTPHX (ustphx.F:31-52); no warp term (hamilt.F:349-365)
// ---------------------------------------------------------------------
struct TabDesc {
  int d1, d2, d3;       // half extents
  int w1, w2, w3;       // WARP half extents
  double bk[9];         // Cartesian dK = bk * dKZZ  (bk row-major [3][3])
};

__global__ void k_table(DevProb P, TabDesc T, const double2* warp, double2* tab) {
  int nx = 2 * T.d1 + 1, ny = 2 * T.d2 + 1, nz = 2 * T.d3 + 1;
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nx * ny * nz) return;
  int ix = idx % nx, iy = (idx / nx) % ny, iz = idx / (nx * ny);
  int d[3] = {ix - T.d1, iy - T.d2, iz - T.d3};
  double g0 = T.bk[0] * d[0] + T.bk[1] * d[1] + T.bk[2] * d[2];
  double g1 = T.bk[3] * d[0] + T.bk[4] * d[1] + T.bk[5] * d[2];
  double g2 = T.bk[6] * d[0] + T.bk[7] * d[1] + T.bk[8] * d[2];
  double slen = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
  bool zero = (d[0] == 0 && d[1] == 0 && d[2] == 0);
  double2 th = cmk(0.0, 0.0);
  if (P.ins == 0) {
    for (int jn = 0; jn < P.nat; jn++) {
      if (zero) {
        th.x = th.x + 1.0 / (double)P.nat - P.v[jn] * (double)P.mult[jn];
      } else {
        double2 ph = cmk(0.0, 0.0);
        int a0 = P.afirst[jn];
        for (int q = 0; q < P.mult[jn]; q++) {
          const double* r = P.pos + 3 * (a0 + q);
          ph = cadd(ph, cexp2pi(r[0] * d[0] + r[1] * d[1] + r[2] * d[2]));
        }
        double h = slen * P.rmt[jn];
        double sn, cs;
        sincos(h, &sn, &cs);
        double besr = (h * cs - sn) * (1.0 / (h * h * h));
        double v3 = 3.0 * P.v[jn];
        th = cadd(th, cscale(cscale(ph, v3), besr));
      }
    }
  } else {
    if (slen > 1.0e-10) {
      double2 u = cmk(0.0, 0.0);
      for (int jn = 0; jn < P.nat; jn++) {
        double2 ph = cmk(0.0, 0.0);
        int a0 = P.afirst[jn];
        for (int q = 0; q < P.mult[jn]; q++) {
          const double* r = P.pos + 3 * (a0 + q);
          ph = cadd(ph, cexp2pi(r[0] * d[0] + r[1] * d[1] + r[2] * d[2]));
        }
        double qq = slen * P.rmt[jn];
        double sn, cs;
        sincos(qq, &sn, &cs);
        double besr = (qq * cs - sn) / (qq * qq * qq);
        u = cadd(u, cscale(cscale(ph, P.v[jn]), besr));
      }
      th = cscale(u, 3.0);
    } else {
      double u = 0.0;
      for (int jn = 0; jn < P.nat; jn++) u = u + P.v[jn] * (double)P.mult[jn];
      th = cmk(1.0 - u, 0.0);
    }
  }
  double2 w = cmk(0.0, 0.0);
  if (P.ins == 0 && abs(d[0]) <= T.w1 && abs(d[1]) <= T.w2 && abs(d[2]) <= T.w3) {
    size_t wi = ((size_t)(d[2] + T.w3) * (2 * T.w2 + 1) + (size_t)(d[1] + T.w2)) * (2 * T.w1 + 1) +
                (size_t)(d[0] + T.w1);
    w = warp[wi];
  }
  tab[2 * (size_t)idx] = th;
  tab[2 * (size_t)idx + 1] = w;
}

// ---------------------------------------------------------------------
// K-b + K-c: PW x PW block of H and S (hamilt.F:188-466 + ZSWAP).
//
// Per pair (J <= I), the reference accumulates, atom type by atom type,
//   t_S = sum_l (2l+1) P_l(x_JI) [AL_J AL_I + CHN BL_J BL_I]
//   t_H = sum_l (2l+1) P_l(x_JI) [AL_J hA_I + BL_J hB_I]
// with hA/hB the non-symmetric 2x2 block of hamilt.F:386-424 (surface
// kinetic terms included) applied on the column side, and adds
// VIF * PHASE * t to S and H, PHASE = sum_eq exp(2 pi i (K_J - K_I) r_eq).
// This kernel keeps that loop order: the Legendre weights w_l = (2l+1) P_l
// of each pair are computed once with the reference's recursion (UTOP
// branch included, hamilt.F:250-281) and held in registers; per atom type
// the J-side {AL, BL} and the I-side VIF {AL, CHN BL, hA, hB} are staged in
// shared memory; PHASE is formed as sum_eq phi_a(J) conj(phi_a(I)) from the
// per-row phases.  That is 6 FMA per (pair, type, l) plus the phase
// products, instead of 16 for the same sum as a GEMM over explicit (l, r).
// Thread (tj, ti) owns rows J = j0 + tj + 16u and columns I = i0 + ti + 16v
// (u, v in {0,1}), so shared-memory reads are conflict-free.
// ---------------------------------------------------------------------
#define SPH_T 32
#define SPH_TC 8
#define SPH_THREADS 256
#define SPH_LMAX 13
#define SPH_MAXA 32  // equivalent atoms whose phases one chunk stages
// dynamic shared memory: per staged type 1 J-side and 2 I-side double2 per
// (l, row), plus the J and I phases of up to SPH_MAXA atoms
#define SPH_DYN_SMEM ((3 * SPH_TC * SPH_LMAX * SPH_T + 2 * SPH_MAXA * SPH_T) * 16)

struct SphCoef {  // per (type, l)
  double vif, chn, mAA, mAB, mBA, mBB;
};

__global__ void k_sph_coef(DevProb P, SphCoef* coef) {
  int l = threadIdx.x, jn = blockIdx.x;
  if (l >= P.ltop) return;
  const double pi = 3.141592653589793238462643;
  double r = P.rmt[jn];
  double r2 = r * r;
  int o = jn * P.ldl + l;
  double U = P.p[o], UP = P.pe[o], DU = P.dp[o], DUP = P.dpe[o], CHN = P.pei[o], E = P.e[o];
  SphCoef c;
  c.vif = 4.0 * pi * P.vi * (r2 * r2);
  c.chn = P.lapw[o] ? CHN : 0.0;
  c.mAA = E + r2 * (U * DU);
  c.mAB = r2 * (UP * DU);
  c.mBA = 1.0 + r2 * (U * DUP);
  c.mBB = E * CHN + r2 * (UP * DUP);
  coef[jn * P.ltop + l] = c;
}

__global__ void __launch_bounds__(SPH_THREADS, 1)
    k_spherical(DevProb P, const int2* __restrict__ tiles, const SphCoef* __restrict__ coef,
                const double2* __restrict__ tab, TabDesc T, double2* __restrict__ hs, int ld,
                double2* __restrict__ hsdiag) {
  extern __shared__ double2 sm2[];
  // staged per type chunk: J side (AL, BL) [tc][l][32], I side VIF-scaled
  // (AL, CHN BL) and (hA, hB) [tc][l][32][2], phases [atom][32] for J and I
  double2* sJ = sm2;
  double2* sI = sJ + SPH_TC * SPH_LMAX * SPH_T;
  double2* sPJ = sI + 2 * SPH_TC * SPH_LMAX * SPH_T;
  double2* sPI = sPJ + SPH_MAXA * SPH_T;
  const int tid = threadIdx.x;
  const int tj = tid & 15, ti = tid >> 4;
  const int2 t = tiles[blockIdx.x];
  const int i0 = t.x * SPH_T, j0 = t.y * SPH_T;
  const int nv = P.nv, ltop = P.ltop, nat = P.nat;

  // Legendre weights (2l+1) P_l(x_JI) of the four owned pairs
  double w[4][SPH_LMAX];
#pragma unroll
  for (int u = 0; u < 2; u++)
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const int q = u * 2 + v;
      const int J = j0 + tj + 16 * u, I = i0 + ti + 16 * v;
      double x = 0.0;
      if (J < nv && I < nv) {
        x = P.xk[I] * P.xk[J] + P.yk[I] * P.yk[J] + P.zk[I] * P.zk[J];
        double den = P.rk[I] * P.rk[J];
        if (den > 1.0e-8) x = x / den;
      }
      const bool top = !(fabs(x) < 0.9999999);
      double pm2 = 1.0, pm1 = x;
      w[q][0] = 1.0;
      w[q][1] = 3.0 * x;
#pragma unroll
      for (int l = 2; l < SPH_LMAX; l++) {
        double pl;
        if (!top) {
          const double pplx = x * pm1;
          const double pply = pplx - pm2;
          pl = pplx + ((double)(l - 1) / (double)l) * pply;
        } else {
          pl = x * pm1;
        }
        pm2 = pm1;
        pm1 = pl;
        w[q][l] = (double)(2 * l + 1) * pl;
      }
    }

  double2 aS[4], aH[4];
#pragma unroll
  for (int q = 0; q < 4; q++) aS[q] = aH[q] = cmk(0.0, 0.0);

  for (int t0 = 0; t0 < nat;) {
    // chunk of types whose equivalent atoms fit the staged phase rows
    int ntc = 0, na = 0;
    while (ntc < SPH_TC && t0 + ntc < nat && na + P.mult[t0 + ntc] <= SPH_MAXA) na += P.mult[t0 + ntc++];
    const bool staged = ntc > 0;
    if (!staged) ntc = 1;  // one type with more atoms than SPH_MAXA: phases from global memory
    const int a0c = P.afirst[t0];
    __syncthreads();
    for (int idx = tid; idx < ntc * ltop * SPH_T; idx += SPH_THREADS) {
      const int r = idx % SPH_T, l = (idx / SPH_T) % ltop, tc = idx / (SPH_T * ltop);
      const int jn = t0 + tc;
      const size_t ob = ((size_t)jn * ltop + l) * P.nvpad;
      const int J = j0 + r, I = i0 + r;
      double aj = 0.0, bj = 0.0, ai = 0.0, bi = 0.0;
      if (J < nv) {
        aj = P.al[ob + J];
        bj = P.bl[ob + J];
      }
      if (I < nv) {
        ai = P.al[ob + I];
        bi = P.bl[ob + I];
      }
      const SphCoef c = coef[jn * ltop + l];
      const int s = (tc * SPH_LMAX + l) * SPH_T + r;
      sJ[s] = cmk(aj, bj);
      sI[2 * s] = cmk(c.vif * ai, c.vif * (c.chn * bi));
      sI[2 * s + 1] = cmk(c.vif * (c.mAA * ai + c.mAB * bi), c.vif * (c.mBA * ai + c.mBB * bi));
    }
    if (staged)
      for (int idx = tid; idx < na * SPH_T; idx += SPH_THREADS) {
        const int r = idx % SPH_T, e = idx / SPH_T;
        const double2* pa = P.phase + (size_t)(a0c + e) * P.npad;
        sPJ[idx] = pa[j0 + r];
        sPI[idx] = pa[i0 + r];
      }
    __syncthreads();
    for (int tc = 0; tc < ntc; tc++) {
      const int jn = t0 + tc;
      double tS[4], tH[4];
#pragma unroll
      for (int q = 0; q < 4; q++) tS[q] = tH[q] = 0.0;
#pragma unroll
      for (int l = 0; l < SPH_LMAX; l++) {
        if (l < ltop) {
          const int s = (tc * SPH_LMAX + l) * SPH_T;
          double2 jv[2], is[2], ih[2];
#pragma unroll
          for (int u = 0; u < 2; u++) jv[u] = sJ[s + tj + 16 * u];
#pragma unroll
          for (int v = 0; v < 2; v++) {
            is[v] = sI[2 * (s + ti + 16 * v)];
            ih[v] = sI[2 * (s + ti + 16 * v) + 1];
          }
#pragma unroll
          for (int u = 0; u < 2; u++)
#pragma unroll
            for (int v = 0; v < 2; v++) {
              const int q = u * 2 + v;
              const double sv = fma(jv[u].y, is[v].y, jv[u].x * is[v].x);
              const double hv = fma(jv[u].y, ih[v].y, jv[u].x * ih[v].x);
              tS[q] = fma(w[q][l], sv, tS[q]);
              tH[q] = fma(w[q][l], hv, tH[q]);
            }
        }
      }
      // PHASE = sum over the equivalent atoms of this type
      double2 ph[4];
#pragma unroll
      for (int q = 0; q < 4; q++) ph[q] = cmk(0.0, 0.0);
      const int ae = P.afirst[jn], me = P.mult[jn];
      for (int e = 0; e < me; e++) {
        double2 fj[2], fi[2];
        if (staged) {
          const int b = (ae - a0c + e) * SPH_T;
#pragma unroll
          for (int u = 0; u < 2; u++) fj[u] = sPJ[b + tj + 16 * u];
#pragma unroll
          for (int v = 0; v < 2; v++) fi[v] = sPI[b + ti + 16 * v];
        } else {
          const double2* pa = P.phase + (size_t)(ae + e) * P.npad;
#pragma unroll
          for (int u = 0; u < 2; u++) fj[u] = pa[j0 + tj + 16 * u];
#pragma unroll
          for (int v = 0; v < 2; v++) fi[v] = pa[i0 + ti + 16 * v];
        }
#pragma unroll
        for (int u = 0; u < 2; u++)
#pragma unroll
          for (int v = 0; v < 2; v++) {
            const int q = u * 2 + v;
            ph[q].x = fma(fj[u].x, fi[v].x, fma(fj[u].y, fi[v].y, ph[q].x));
            ph[q].y = fma(fj[u].y, fi[v].x, fma(-fj[u].x, fi[v].y, ph[q].y));
          }
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        aS[q].x = fma(ph[q].x, tS[q], aS[q].x);
        aS[q].y = fma(ph[q].y, tS[q], aS[q].y);
        aH[q].x = fma(ph[q].x, tH[q], aH[q].x);
        aH[q].y = fma(ph[q].y, tH[q], aH[q].y);
      }
    }
    t0 += ntc;
  }
  // interstitial + write (hamilt.F:289-345, 459-466, calkpt.F:164)
  const int nx = 2 * T.d1 + 1, ny = 2 * T.d2 + 1;
#pragma unroll
  for (int v = 0; v < 2; v++) {
    const int I = i0 + ti + 16 * v;
    if (I >= nv) continue;
    const int k1 = P.kzz[3 * I], k2 = P.kzz[3 * I + 1], k3 = P.kzz[3 * I + 2];
    const double xi = P.xk[I], yi = P.yk[I], zi = P.zk[I];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int J = j0 + tj + 16 * u;
      if (J > I) continue;
      const int q = u * 2 + v;
      const double x2 = P.xk[J] * xi + P.yk[J] * yi + P.zk[J] * zi;
      const int d1 = P.kzz[3 * J] - k1 + T.d1, d2 = P.kzz[3 * J + 1] - k2 + T.d2, d3 = P.kzz[3 * J + 2] - k3 + T.d3;
      const size_t c = ((size_t)d3 * ny + d2) * nx + d1;
      const double2 th = tab[2 * c], wp = tab[2 * c + 1];
      const double2 s = cadd(th, aS[q]);
      const double2 h = cadd(cadd(cscale(th, x2), wp), aH[q]);
      if (J == I) {
        hs[(size_t)I * ld + I] = h;
        hsdiag[I] = s;
      } else {
        hs[(size_t)I * ld + J] = s;  // S upper: HS(J,I)
        hs[(size_t)J * ld + I] = h;  // H lower: HS(I,J)
      }
    }
  }
}

// ---------------------------------------------------------------------
// K-b': local-orbital columns (hamilt.F:475-818).  One block row per LO
// column, threads over rows J <= I.
// ---------------------------------------------------------------------
struct LoCol {
  int jn, l, jlo, jeqo, mo1, nnlo, a0;  // a0: first atom of the type
  double clr, cli;                       // i^l
};

// status: when non-null, a non-finite written element sets
// L1G_STATUS_NONFINITE (the split path's writers check what they write)
__global__ void k_lo(DevProb P, const LoCol* __restrict__ cols, double2* __restrict__ hs, int ld,
                     double2* __restrict__ hsdiag, int* __restrict__ status) {
  const LoCol c = cols[blockIdx.y];
  const int nv = P.nv;
  const int I = nv + c.nnlo - 1;  // 0-based row/column of this LO
  int J = blockIdx.x * blockDim.x + threadIdx.x;
  const int jn = c.jn, l = c.l, jlo = c.jlo, jeqo = c.jeqo, mo1 = c.mo1, mult = P.mult[jn];
  // the LO row's Y_lm per equivalent atom, shared by the block (I is the
  // block's), in chunks of LO_YCH atoms
  constexpr int LO_YCH = 16;
  __shared__ double2 syi[LO_YCH][16];
  const bool active = J <= I;
  if (!active && (blockIdx.x * blockDim.x) > I) return;  // the whole block is past the row (block-uniform)
  const double pi = 3.141592653589793238462643;
  const double r = P.rmt[jn], r2 = r * r;
  const double pi4r2v = 4.0 * pi * sqrt(P.vi) * r * r;
  const int o = jn * P.ldl + l;
  const double U = P.p[o], UP = P.pe[o], DU = P.dp[o], DUP = P.dpe[o], CHN = P.pei[o], E = P.e[o];
  const int lo4 = jn * (L1G_LOMAX + 1) + l;
#define LOV(arr, jj) P.arr[(jn * L1G_NLOAT + (jj)-1) * (L1G_LOMAX + 1) + l]
  const double ALO = LOV(alo, jlo), BLO = LOV(blo, jlo), CLO = LOV(clo, jlo), ELO = LOV(elo, jlo);
  const double PI12 = P.pi12lo[lo4], PE12 = P.pe12lo[lo4], DPL = P.dplo[lo4];
  const double c1r = ALO + PI12 * CLO;
  const double c2r = BLO * CHN + PE12 * CLO;
  const double c11r = ALO * E + 0.5 * (BLO + CLO * PI12 * (ELO + E));
  const double c12r = BLO * CHN * E + 0.5 * (ALO + CLO * PI12 + CLO * PE12 * (ELO + E));
  const double c3r = CLO + PE12 * BLO + ALO * PI12;
  const double c13r = CLO * ELO + 0.5 * (BLO * PI12 + (ELO + E) * (ALO * PI12 + PE12 * BLO));
  const double akinlor = 0.5 * r2 * (ALO * DU + BLO * DUP + CLO * DPL);
  const double clr = c.clr, cli = c.cli;

  // LO-LO row ranges (hamilt.F:677-680), 1-based NNLO arithmetic
  bool inlo[L1G_NLOAT + 1];
  int Jf = J + 1;  // 1-based row
  bool any_lo = false;
  for (int jlop = 1; jlop <= jlo; jlop++) {
    int jbeg = nv + c.nnlo - (mo1 + l) - (2 * l + 1) * (jeqo - 1) - (jlo - jlop) * (2 * l + 1) * mult;
    int jend = nv + c.nnlo - (jlo - jlop) * (mo1 + l + 1) - (jlo - jlop) * (jeqo - 1) * (2 * l + 1);
    inlo[jlop] = (Jf >= jbeg && Jf <= jend);
    any_lo |= inlo[jlop];
  }
  double2 S = cmk(0.0, 0.0), H = cmk(0.0, 0.0);
  const bool work = active && (J < nv || any_lo);
  {
    double alj = 0.0, blj = 0.0;
    if (work && J < nv) {
      size_t oo = ((size_t)jn * P.ltop + l) * P.nvpad + J;
      alj = P.al[oo];
      blj = P.bl[oo];
    }
    for (int jeq = 0; jeq < mult; jeq++) {
      if (jeq % LO_YCH == 0) {  // block-uniform: the next chunk's Y_lm of the LO row
        __syncthreads();
        const int q = threadIdx.x;
        if (q < LO_YCH && jeq + q < mult)
          dev_ylm_row<3>(P.xk[I], P.yk[I], P.zk[I], P.rotij + 9 * (c.a0 + jeq + q), P.rotloc + 9 * jn, l, syi[q]);
        __syncthreads();
      }
      if (!work) continue;
      const int a = c.a0 + jeq;
      const double* ra = P.pos + 3 * a;
      double s = ra[0] * (double)(P.kzz[3 * I] - P.kzz[3 * J]) + ra[1] * (double)(P.kzz[3 * I + 1] - P.kzz[3 * J + 1]) +
                 ra[2] * (double)(P.kzz[3 * I + 2] - P.kzz[3 * J + 2]);
      const double2 ph = cconj(cexp2pi(s));
      double2 yj[16];
      const double2* yi = syi[jeq % LO_YCH];
      dev_ylm_row<3>(P.xk[J], P.yk[J], P.zk[J], P.rotij + 9 * a, P.rotloc + 9 * jn, l, yj);
      for (int mo2 = -l; mo2 <= l; mo2++) {
        const int lm = l * (l + 1) + mo2;
        const double clylnr = clr * yi[lm].x + cli * yi[lm].y;
        const double clylni = cli * yi[lm].x - clr * yi[lm].y;
        const double c1rup = c1r * clylnr * pi4r2v, c1iup = c1r * clylni * pi4r2v;
        const double c2rup = c2r * clylnr * pi4r2v, c2iup = c2r * clylni * pi4r2v;
        const double c3rup = c3r * clylnr * pi4r2v, c3iup = c3r * clylni * pi4r2v;
        const double c11rup = c11r * clylnr * pi4r2v, c11iup = c11r * clylni * pi4r2v;
        const double c12rup = c12r * clylnr * pi4r2v, c12iup = c12r * clylni * pi4r2v;
        const double c13rup = c13r * clylnr * pi4r2v, c13iup = c13r * clylni * pi4r2v;
        const double akinlorup = akinlor * clylnr * pi4r2v, akinloiup = akinlor * clylni * pi4r2v;
        const double clylr = clr * yj[lm].x + cli * yj[lm].y;
        const double clyli = cli * yj[lm].x - clr * yj[lm].y;
        if (J < nv) {
          const double c6r = clylr * alj * pi4r2v, c6i = clyli * alj * pi4r2v;
          const double c7r = clylr * blj * pi4r2v, c7i = clyli * blj * pi4r2v;
          double cabr = c6r * c1rup + c7r * c2rup + c6i * c1iup + c7i * c2iup;
          double cabi = -c6i * c1rup - c7i * c2rup + c6r * c1iup + c7r * c2iup;
          S = cadd(S, cmk(cabr * ph.x - cabi * ph.y, cabr * ph.y + cabi * ph.x));
          cabr = c6r * c11rup + c7r * c12rup + c6i * c11iup + c7i * c12iup;
          cabi = -c6i * c11rup - c7i * c12rup + c6r * c11iup + c7r * c12iup;
          const double ua = c6r * U + c7r * UP, ub = c6i * U + c7i * UP;
          const double akinbr = ua * akinlorup + ub * akinloiup;
          const double akinbi = ua * akinloiup - ub * akinlorup;
          H = cadd(H, cmk(cabr * ph.x - cabi * ph.y, cabr * ph.y + cabi * ph.x));
          H = cadd(H, cmk(akinbr * ph.x - akinbi * ph.y, akinbr * ph.y + akinbi * ph.x));
        } else {
          for (int jlop = 1; jlop <= jlo; jlop++) {
            if (!inlo[jlop]) continue;
            const double alop = LOV(alo, jlop), blop = LOV(blo, jlop), clop = LOV(clo, jlop);
            const double c6r = clylr * alop * pi4r2v, c6i = clyli * alop * pi4r2v;
            const double c7r = clylr * blop * pi4r2v, c7i = clyli * blop * pi4r2v;
            const double c8r = clylr * clop * pi4r2v, c8i = clyli * clop * pi4r2v;
            double cr = c6r * c1rup + c6i * c1iup + c7r * c2rup + c7i * c2iup + c8r * c3rup + c8i * c3iup;
            double ci = -c6i * c1rup + c6r * c1iup - c7i * c2rup + c7r * c2iup - c8i * c3rup + c8r * c3iup;
            S = cadd(S, cmk(cr * ph.x - ci * ph.y, cr * ph.y + ci * ph.x));
            cr = c6r * c11rup + c6i * c11iup + c7r * c12rup + c7i * c12iup + c8r * c13rup + c8i * c13iup;
            ci = -c6i * c11rup + c6r * c11iup - c7i * c12rup + c7r * c12iup - c8i * c13rup + c8r * c13iup;
            H = cadd(H, cmk(cr * ph.x - ci * ph.y, cr * ph.y + ci * ph.x));
          }
        }
      }
    }
  }
#undef LOV
  if (!active) return;
  if (J == I) {
    hs[(size_t)I * ld + I] = H;
    hsdiag[I] = S;
  } else {
    hs[(size_t)I * ld + J] = S;
    hs[(size_t)J * ld + I] = H;
  }
  if (status && (l1g_nonfinite(S) || l1g_nonfinite(H))) atomicOr(status, L1G_STATUS_NONFINITE);
}

// ---------------------------------------------------------------------
// K-ns operands (hns.F:165-437).  For atom a, k = (a*2 + r)*nsl2 + lm:
//   R[k][i] = {ALM, BLM}(i, lm)            (hns.F:190-259; r = 0, 1)
//   L[k][i] = {A2, B2}(i, lm)              (hns.F:381-434)
// with A2 = sum_b TUU conj(ALM) + TDU conj(BLM) + TUU21 conj(CLM), B2 the
// same with TUD, TDD, TUD21 (the TMP sums of hns.F:387-417: T times the
// conjugate).  CLM is non-zero only on the atom's own LO rows, so
//   k_hns_alm     builds R (and CLM, C-side of the LO rows) per row,
//   k_hns_tmul    forms L = M conj(R) per atom as a small complex GEMM,
//                 M = [[TUU, TDU], [TUD, TDD]] (2 nsl2 x 2 nsl2),
//   k_hns_lo_ops  adds the CLM terms of the LO rows and their C2.
// ---------------------------------------------------------------------
struct LoRange {
  int jn, l, jlo, i1, i2;  // rows nv+i1..nv+i2 (1-based LO indices)
};

__global__ void k_hns_alm(DevProb P, const LoRange* __restrict__ lor, int nlor, double2* __restrict__ Rop,
                          double2* __restrict__ Clo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // row
  const int a = blockIdx.y;                              // atom
  const int nsl = P.lnsmax + 1, nsl2 = nsl * nsl;
  if (i >= P.npad) return;
  const size_t Kst = (size_t)P.npad;
  double2* RA = Rop + ((size_t)(a * 2 + 0) * nsl2) * Kst + i;
  double2* RB = Rop + ((size_t)(a * 2 + 1) * nsl2) * Kst + i;
  if (i >= P.n) {
    for (int lm = 0; lm < nsl2; lm++) RA[lm * Kst] = RB[lm * Kst] = cmk(0.0, 0.0);
    return;
  }
  const int jn = P.atype[a];
  const double pi = 3.141592653589793238462643;
  const double rhoatm = 4.0 * pi * sqrt(P.vi) * P.rmt[jn] * P.rmt[jn];
  const double2 ph = P.phase[(size_t)a * P.npad + i];
  double2 y[25];
  dev_ylm_row<4>(P.xk[i], P.yk[i], P.zk[i], P.rotij + 9 * a, P.rotloc + 9 * jn, nsl - 1, y);
  // LO identity of this row for this atom's type (hns.F:223-255, LOHNS)
  int myl = -1, myjlo = 0;
  if (i >= P.nv) {
    const int li = i - P.nv + 1;
    for (int q = 0; q < nlor; q++)
      if (lor[q].jn == jn && li >= lor[q].i1 && li <= lor[q].i2) {
        myl = lor[q].l;
        myjlo = lor[q].jlo;
      }
  }
  double2 cil = cmk(1.0, 0.0);
  int lm = 0;
  for (int l0 = 0; l0 < nsl; l0++) {
    for (int m0 = -l0; m0 <= l0; m0++, lm++) {
      const double2 tt = cmul(cmul(cil, ph), cconj(y[lm]));
      const double almr = rhoatm * tt.x, almi = rhoatm * tt.y;
      double2 A = cmk(0.0, 0.0), B = A, Cc = A;
      if (i < P.nv) {
        const size_t o = ((size_t)jn * P.ltop + l0) * P.nvpad + i;
        const double alv = P.al[o], blv = P.bl[o];
        B = cmk(blv * almr, blv * almi);
        A = cmk(alv * almr, alv * almi);
      } else if (l0 == myl) {
        const int oo = (jn * L1G_NLOAT + myjlo - 1) * (L1G_LOMAX + 1) + l0;
        B = cmk(P.blo[oo] * almr, P.blo[oo] * almi);
        Cc = cmk(P.clo[oo] * almr, P.clo[oo] * almi);
        A = cmk(P.alo[oo] * almr, P.alo[oo] * almi);
      }
      RA[lm * Kst] = A;
      RB[lm * Kst] = B;
      if (i >= P.nv) Clo[((size_t)a * nsl2 + lm) * (size_t)P.nlo + (i - P.nv)] = Cc;
    }
    cil = cmk(-cil.y, cil.x);
  }
}

// 16-byte global -> shared copy that bypasses registers (cp.async), so that
// a block's staging has all its loads in flight at once
__device__ __forceinline__ void l1g_cp16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void l1g_cp_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

#define TMUL_I 64        // columns (basis rows i) per work item
#define TMUL_ROWS 10     // rows of L per thread (one warp: 10 rows x 64 columns)
#define TMUL_WARPS 5     // 5 x 10 >= 2 NSL2 = 50 rows
#define TMUL_SMEM ((2 * L1G_NSL2) * (2 * L1G_NSL2) * 16 + (2 * L1G_NSL2) * TMUL_I * 16)
// L[(a, r_out, la)][i] = sum_{(r, b)} M[(r_out, la)][(r, b)] conj(R[(a, r, b)][i])
// A work item is (atom, 64 columns i); block b takes the contiguous items
// [b per, (b+1) per) (one atom for most of them: M is staged again only
// when the atom changes).  Thread (warp w, lane): rows 10 w .. 10 w + 9 and
// columns lane, lane + 32 of the item, 20 complex accumulators; per k two
// R values (conflict-free rows of smem) and ten broadcast M values.
__global__ void __launch_bounds__(32 * TMUL_WARPS, 2) k_hns_tmul(int npad, int nsl2, int ndf, int per,
                                                              const int* __restrict__ atype,
                                                              const double2* __restrict__ tns,
                                                              const double2* __restrict__ Rop,
                                                              double2* __restrict__ Lop) {
  extern __shared__ double2 tm[];
  const int K = 2 * nsl2;
  double2* sM = tm;          // [K][K]
  double2* sR = tm + K * K;  // [K][TMUL_I]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nch = (npad + TMUL_I - 1) / TMUL_I, nitem = nch * ndf;
  const int it0 = blockIdx.x * per, it1 = min(nitem, it0 + per);
  int staged = -1;
  for (int item = it0; item < it1; item++) {
    const int a = item / nch, i0 = (item % nch) * TMUL_I;
    __syncthreads();  // the previous item's smem reads are done
    if (a != staged) {
      const double2* T = tns + (size_t)atype[a] * LAPW1GPU_NTNS * L1G_NSL2 * L1G_NSL2;
      for (int idx = tid; idx < K * K; idx += 32 * TMUL_WARPS) {
        const int row = idx / K, col = idx % K;
        const int ro = row / nsl2, la = row % nsl2, r = col / nsl2, b = col % nsl2;
        const int blk = ro == 0 ? (r == 0 ? 0 : 1) : (r == 0 ? 3 : 4);  // TUU TDU / TUD TDD
        l1g_cp16(&sM[idx], &T[((size_t)blk * L1G_NSL2 + la) * L1G_NSL2 + b]);
      }
      staged = a;
    }
    const double2* R = Rop + (size_t)a * K * npad;
    for (int idx = tid; idx < K * TMUL_I; idx += 32 * TMUL_WARPS) {
      const int k = idx / TMUL_I, c = idx % TMUL_I;
      if (i0 + c < npad)
        l1g_cp16(&sR[idx], &R[(size_t)k * npad + i0 + c]);
      else
        sR[idx] = make_double2(0.0, 0.0);
    }
    l1g_cp_wait_all();
    __syncthreads();
    const int r0 = w * TMUL_ROWS;
    if (r0 < K) {  // warp-uniform
      double2 acc[TMUL_ROWS][2];
#pragma unroll
      for (int r = 0; r < TMUL_ROWS; r++) acc[r][0] = acc[r][1] = cmk(0.0, 0.0);
#pragma unroll 2
      for (int k = 0; k < K; k++) {
        const double2 x0 = sR[k * TMUL_I + lane], x1 = sR[k * TMUL_I + lane + 32];
#pragma unroll
        for (int r = 0; r < TMUL_ROWS; r++) {
          const double2 m = sM[min(r0 + r, K - 1) * K + k];  // rows past K: computed, not stored
          acc[r][0].x = fma(m.x, x0.x, fma(m.y, x0.y, acc[r][0].x));
          acc[r][0].y = fma(m.y, x0.x, fma(-m.x, x0.y, acc[r][0].y));
          acc[r][1].x = fma(m.x, x1.x, fma(m.y, x1.y, acc[r][1].x));
          acc[r][1].y = fma(m.y, x1.x, fma(-m.x, x1.y, acc[r][1].y));
        }
      }
      double2* L = Lop + (size_t)a * K * npad;
#pragma unroll
      for (int r = 0; r < TMUL_ROWS; r++) {
        const int row = r0 + r;
        if (row < K) {
          if (i0 + lane < npad) L[(size_t)row * npad + i0 + lane] = acc[r][0];
          if (i0 + lane + 32 < npad) L[(size_t)row * npad + i0 + lane + 32] = acc[r][1];
        }
      }
    }
  }
}

// LO rows: A2 += TUU21 conj(CLM), B2 += TUD21 conj(CLM),
// C2 = TUU12 conj(ALM) + TDU12 conj(BLM) + TUU22 conj(CLM)  (hns.F:391-433).
// One thread per (la, 4 LO rows) of an atom: block (32 la, 8) over 32 rows,
// the rows' ALM, BLM, CLM staged in shared memory; each T element read is
// used for the 4 rows.
// cj: Lop holds conj(L) (the library product of the split path), so the
// LO terms are added conjugated.
#define LOOPS_ROWS 32
__global__ void __launch_bounds__(256) k_hns_lo_ops(DevProb P, const double2* __restrict__ tns,
                                                    double2* __restrict__ Lop, const double2* __restrict__ Rop,
                                                    const double2* __restrict__ Clo, double2* __restrict__ C2lo,
                                                    int cj) {
  __shared__ double2 sX[LOOPS_ROWS][3][L1G_NSL2];
  const int la = threadIdx.x, cy = threadIdx.y;
  const int c0 = blockIdx.x * LOOPS_ROWS;  // first LO row of the block
  const int a = blockIdx.y;
  const int nsl2 = (P.lnsmax + 1) * (P.lnsmax + 1);
  const size_t npad = P.npad;
  for (int q = threadIdx.y * 32 + threadIdx.x; q < LOOPS_ROWS * 3 * nsl2; q += 256) {
    const int r = q / (3 * nsl2), w = (q / nsl2) % 3, b = q % nsl2;
    const int cc = c0 + r;
    double2 v = cmk(0.0, 0.0);
    if (cc < P.nlo) {
      const size_t i = P.nv + cc;
      if (w < 2)
        v = Rop[((size_t)(a * 2 + w) * nsl2 + b) * npad + i];
      else
        v = Clo[((size_t)a * nsl2 + b) * P.nlo + cc];
    }
    sX[r][w][b] = v;
  }
  __syncthreads();
  if (la >= nsl2 || c0 + cy >= P.nlo) return;
  const double2* T = tns + (size_t)P.atype[a] * LAPW1GPU_NTNS * L1G_NSL2 * L1G_NSL2;
  double2 da[4], db[4], dc[4];
#pragma unroll
  for (int u = 0; u < 4; u++) da[u] = db[u] = dc[u] = cmk(0, 0);
  for (int b = 0; b < nsl2; b++) {
#define TT(blk) __ldg(T + ((size_t)(blk)*L1G_NSL2 + la) * L1G_NSL2 + b)
    const double2 tuu21 = TT(2), tud21 = TT(5), tuu12 = TT(6), tdu12 = TT(7), tuu22 = TT(8);
#undef TT
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int r = cy + 8 * u;
      const double2 A = sX[r][0][b], B = sX[r][1][b], Cc = sX[r][2][b];
      da[u] = cadd(da[u], cmul(tuu21, cconj(Cc)));
      db[u] = cadd(db[u], cmul(tud21, cconj(Cc)));
      dc[u] = cadd(dc[u], cadd(cadd(cmul(tuu12, cconj(A)), cmul(tdu12, cconj(B))), cmul(tuu22, cconj(Cc))));
    }
  }
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int c = c0 + cy + 8 * u;
    if (c >= P.nlo) break;
    const size_t i = P.nv + c;
    double2* LA = Lop + ((size_t)(a * 2 + 0) * nsl2 + la) * npad + i;
    double2* LB = Lop + ((size_t)(a * 2 + 1) * nsl2 + la) * npad + i;
    *LA = cadd(*LA, cj ? cconj(da[u]) : da[u]);
    *LB = cadd(*LB, cj ? cconj(db[u]) : db[u]);
    C2lo[((size_t)a * nsl2 + la) * P.nlo + c] = dc[u];
  }
}


// HS(i,j) += sum_k Lop[k][i] * Rop[k][j] on the lower triangle i >= j
// (zher2m.f:69-80, 'L','N','T').  64x64 tiles, 4x4 complex per thread.
#define HNS_T 64
#define HNS_KT 16
__global__ void __launch_bounds__(256, 2)
    k_hns_gemm(int n, int npad, int K, const int2* __restrict__ tiles, const double2* __restrict__ Lop,
               const double2* __restrict__ Rop, double2* __restrict__ hs, int ld) {
  __shared__ double2 sL[HNS_KT][HNS_T];
  __shared__ double2 sR[HNS_KT][HNS_T];
  const int tid = threadIdx.x, ti = tid & 15, tj = tid >> 4;
  const int2 t = tiles[blockIdx.x];
  const int i0 = t.x * HNS_T, j0 = t.y * HNS_T;
  double2 acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) acc[u][v] = cmk(0.0, 0.0);
  for (int k0 = 0; k0 < K; k0 += HNS_KT) {
    __syncthreads();
    for (int idx = tid; idx < HNS_KT * HNS_T; idx += 256) {
      int kk = idx / HNS_T, r = idx % HNS_T;
      int k = k0 + kk;
      double2 lv = cmk(0.0, 0.0), rv = cmk(0.0, 0.0);
      if (k < K) {
        lv = Lop[(size_t)k * npad + i0 + r];
        rv = Rop[(size_t)k * npad + j0 + r];
      }
      sL[kk][r] = lv;
      sR[kk][r] = rv;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < HNS_KT; kk++) {
      // thread (ti, tj) owns rows i0 + ti + 16u and columns j0 + tj + 16v:
      // consecutive threads read consecutive shared-memory words
      double2 lv[4], rv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) lv[u] = sL[kk][ti + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; v++) rv[v] = sR[kk][tj + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          acc[u][v].x = fma(lv[u].x, rv[v].x, acc[u][v].x);
          acc[u][v].x = fma(-lv[u].y, rv[v].y, acc[u][v].x);
          acc[u][v].y = fma(lv[u].x, rv[v].y, acc[u][v].y);
          acc[u][v].y = fma(lv[u].y, rv[v].x, acc[u][v].y);
        }
    }
  }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    int j = j0 + tj + 16 * v;
    if (j >= n) continue;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      int i = i0 + ti + 16 * u;
      if (i >= n || i < j) continue;
      double2* dst = hs + (size_t)j * ld + i;
      *dst = cadd(*dst, acc[u][v]);
    }
  }
}

// LO block of HNS through a library product: HS(nv+i, nv+j) += T(i, j) on
// the lower triangle i >= j, T = C2^T CLM computed into a scratch block
__global__ void k_add_lower(int nv, int nlo, const double2* __restrict__ T, double2* __restrict__ hs, int ld,
                            int* __restrict__ status) {
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  const int cj = blockIdx.y;
  if (ci >= nlo || ci < cj) return;
  double2* dst = hs + (size_t)(nv + cj) * ld + (nv + ci);
  const double2 v = cadd(*dst, T[(size_t)cj * nlo + ci]);
  *dst = v;
  if (status && l1g_nonfinite(v)) atomicOr(status, L1G_STATUS_NONFINITE);
}

// LO block of HNS: HS(i,j) += sum C2[k][i] CLM[k][j], nv <= j <= i < n
__global__ void k_hns_lo(int nv, int nlo, int K, const double2* __restrict__ C2lo, const double2* __restrict__ Clo,
                         double2* __restrict__ hs, int ld) {
  int ci = blockIdx.x * blockDim.x + threadIdx.x;
  int cj = blockIdx.y;
  if (ci >= nlo || ci < cj) return;
  double2 s = cmk(0.0, 0.0);
  for (int k = 0; k < K; k++) {
    double2 a = C2lo[(size_t)k * nlo + ci], b = Clo[(size_t)k * nlo + cj];
    s = cadd(s, cmul(a, b));
  }
  double2* dst = hs + (size_t)(nv + cj) * ld + (nv + ci);
  *dst = cadd(*dst, s);
}

// ---------------------------------------------------------------------
// K-orb: HORB (horb.F:98-297) for one (U-atom a, l = lvor)
// ---------------------------------------------------------------------
__global__ void k_horb_rows(DevProb P, int a, int lvor, const double2* __restrict__ pot /*[7][7] pot(m2,m1)*/,
                            const LoRange* __restrict__ lor, int nlor, double2* __restrict__ alm,
                            double2* __restrict__ blm, double2* __restrict__ clm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const int jn = P.atype[a];
  const double pi = 3.141592653589793238462643;
  const double rhoatm = 4.0 * pi * sqrt(P.vi) * P.rmt[jn] * P.rmt[jn];
  const double* r = P.pos + 3 * a;
  double arg = (r[0] * P.kzz[3 * i] + r[1] * P.kzz[3 * i + 1] + r[2] * P.kzz[3 * i + 2]);
  double2 ph = cexp2pi(arg);
  double2 y[16];
  dev_ylm_row<3>(P.xk[i], P.yk[i], P.zk[i], P.rotij + 9 * a, P.rotloc + 9 * jn, lvor, y);
  double2 cil = cmk(1.0, 0.0);
  for (int q = 0; q < lvor; q++) cil = cmk(-cil.y, cil.x);
  int myjlo = 0;
  if (i >= P.nv) {
    int li = i - P.nv + 1;
    for (int q = 0; q < nlor; q++)
      if (lor[q].jn == jn && lor[q].l == lvor && li >= lor[q].i1 && li <= lor[q].i2) myjlo = lor[q].jlo;
  }
  for (int m = -3; m <= 3; m++) {
    double2 A = cmk(0, 0), B = A, Cc = A;
    if (m >= -lvor && m <= lvor) {
      int lm = lvor * (lvor + 1) + m;
      double2 t1 = cmul(cmul(cscale(cil, rhoatm), ph), cconj(y[lm]));
      if (i < P.nv) {
        size_t o = ((size_t)jn * P.ltop + lvor) * P.nvpad + i;
        A = cscale(t1, P.al[o]);
        B = cscale(t1, P.bl[o]);
      } else if (myjlo > 0) {
        int oo = (jn * L1G_NLOAT + myjlo - 1) * (L1G_LOMAX + 1) + lvor;
        B = cscale(t1, P.blo[oo]);
        Cc = cscale(t1, P.clo[oo]);
        A = cscale(t1, P.alo[oo]);
      }
    }
    alm[(size_t)i * 7 + m + 3] = A;
    blm[(size_t)i * 7 + m + 3] = B;
    clm[(size_t)i * 7 + m + 3] = Cc;
  }
}

__global__ void k_horb_pairs(DevProb P, int a, int lvor, const double2* __restrict__ pot, const LoRange* __restrict__ lor,
                             int nlor, const double2* __restrict__ alm, const double2* __restrict__ blm,
                             const double2* __restrict__ clm, double2* __restrict__ hs, int ld) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (i >= P.n || i < j) return;
  const int jn = P.atype[a], nv = P.nv;
  const int o = jn * P.ldl + lvor;
  const double peil = P.pei[o];
  const double pi12 = lvor <= L1G_LOMAX ? P.pi12lo[jn * (L1G_LOMAX + 1) + lvor] : 0.0;
  const double pe12 = lvor <= L1G_LOMAX ? P.pe12lo[jn * (L1G_LOMAX + 1) + lvor] : 0.0;
#define POT(m1, m0) pot[((m1) + 3) * 7 + (m0) + 3]
#define AL7(mm, r) alm[(size_t)(r)*7 + (mm) + 3]
#define BL7(mm, r) blm[(size_t)(r)*7 + (mm) + 3]
#define CL7(mm, r) clm[(size_t)(r)*7 + (mm) + 3]
  double2 add = cmk(0.0, 0.0);
  bool hit = false;
  if (i < nv && j < nv) {
    double2 t4 = cmk(0, 0), t5 = cmk(0, 0);
    for (int m0 = -lvor; m0 <= lvor; m0++) {
      double2 t1 = cmk(0, 0), t2 = cmk(0, 0);
      for (int m1 = -lvor; m1 <= lvor; m1++) {
        t1 = cadd(t1, cmul(POT(m1, m0), AL7(m1, j)));
        t2 = cadd(t2, cmul(POT(m1, m0), BL7(m1, j)));
      }
      t2 = cscale(t2, peil);
      t4 = cadd(t4, cmul(t1, cconj(AL7(m0, i))));
      t5 = cadd(t5, cmul(t2, cconj(BL7(m0, i))));
    }
    add = cadd(t4, t5);
    hit = true;
  } else if (i >= nv && lvor <= L1G_LOMAX) {
    int li = i - nv + 1, lj = j - nv + 1;
    int jlo_i = 0, i22 = 0, jlo_j = 0;
    for (int q = 0; q < nlor; q++) {
      if (lor[q].jn == jn && lor[q].l == lvor && li >= lor[q].i1 && li <= lor[q].i2) jlo_i = lor[q].jlo;
      if (j >= nv && lor[q].jn == jn && lor[q].l == lvor && lj >= lor[q].i1 && lj <= lor[q].i2) {
        jlo_j = lor[q].jlo;
        i22 = lor[q].i2;
      }
    }
    if (jlo_i > 0 && j < nv) {  // <APW||LO>
      double2 t4 = cmk(0, 0), t5 = t4, t6 = t4, t7 = t4;
      for (int m0 = -lvor; m0 <= lvor; m0++) {
        double2 t1 = cmk(0, 0), t2 = cmk(0, 0);
        for (int m1 = -lvor; m1 <= lvor; m1++) {
          t1 = cadd(t1, cmul(AL7(m1, j), POT(m1, m0)));
          t2 = cadd(t2, cmul(BL7(m1, j), POT(m1, m0)));
        }
        t4 = cadd(t4, cmul(t1, cconj(AL7(m0, i))));
        t5 = cadd(t5, cmul(t2, cconj(BL7(m0, i))));
        t6 = cadd(t6, cmul(t1, cconj(CL7(m0, i))));
        t7 = cadd(t7, cmul(t2, cconj(CL7(m0, i))));
      }
      add = cadd(cadd(cadd(t4, cscale(t5, peil)), cscale(t6, pi12)), cscale(t7, pe12));
      hit = true;
    } else if (jlo_i > 0 && jlo_j > 0 && jlo_j <= jlo_i && lj <= i22) {  // <LO||LO>
      double2 t4 = cmk(0, 0), t5 = t4, t6 = t4, t7 = t4;
      for (int m0 = -lvor; m0 <= lvor; m0++) {
        double2 t1 = cmk(0, 0), t2 = t1, t3 = t1;
        for (int m1 = -lvor; m1 <= lvor; m1++) {
          t1 = cadd(t1, cmul(POT(m1, m0), AL7(m1, j)));
          t2 = cadd(t2, cmul(POT(m1, m0), BL7(m1, j)));
          t3 = cadd(t3, cmul(POT(m1, m0), CL7(m1, j)));
        }
        t4 = cadd(cadd(t4, cmul(t1, cconj(AL7(m0, i)))), cmul(cconj(CL7(m0, i)), t3));
        t5 = cadd(t5, cmul(cconj(BL7(m0, i)), t2));
        t6 = cadd(cadd(t6, cmul(cconj(CL7(m0, i)), t1)), cmul(cconj(AL7(m0, i)), t3));
        t7 = cadd(cadd(t7, cmul(cconj(BL7(m0, i)), t3)), cmul(cconj(CL7(m0, i)), t2));
      }
      add = cadd(cadd(cadd(cscale(t5, peil), cscale(t6, pi12)), cscale(t7, pe12)), t4);
      hit = true;
    }
  }
#undef POT
#undef AL7
#undef BL7
#undef CL7
  if (hit) {
    double2* dst = hs + (size_t)j * ld + i;
    *dst = cadd(*dst, add);
  }
}

// non-finite scan of the n x n block and hsdiag (hsdiag may be null)
__global__ void k_check_finite(int n, const double2* __restrict__ hs, int ld, const double2* __restrict__ hsdiag,
                               int* status) {
  // a component is non-finite when its exponent bits are all ones
  unsigned bad = 0;
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const double2* col = hs + (size_t)j * ld;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double2 v = col[i];
      bad |= ((unsigned)(__double_as_longlong(v.x) >> 52) & 0x7ffu) == 0x7ffu;
      bad |= ((unsigned)(__double_as_longlong(v.y) >> 52) & 0x7ffu) == 0x7ffu;
    }
  }
  if (blockIdx.x == 0 && hsdiag)
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double2 d = hsdiag[i];
      bad |= ((unsigned)(__double_as_longlong(d.x) >> 52) & 0x7ffu) == 0x7ffu;
      bad |= ((unsigned)(__double_as_longlong(d.y) >> 52) & 0x7ffu) == 0x7ffu;
    }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, L1G_STATUS_NONFINITE);
}

// The generalized problem SECLR4 solves (seclr4.F:158-345), unpacked from
// the packed state: H(i,j) = conj(HS(i,j)) and S(i,j) = conj(HS(j,i)) for
// i > j (ZHCGST factors S**T), real diagonals from HS(i,i) and HSDIAG(i);
// the lower triangles of H and S, column-major n x n (ld n).
__global__ void k_unpack_seclr(int n, const double2* __restrict__ hs, int ld, const double2* __restrict__ hsdiag,
                               double2* __restrict__ H, double2* __restrict__ S) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // row
  const int j = blockIdx.y;                             // column
  if (i >= n || i < j) return;
  const size_t o = (size_t)j * n + i;
  if (i == j) {
    H[o] = cmk(hs[(size_t)i * ld + i].x, 0.0);
    S[o] = cmk(hsdiag[i].x, 0.0);
  } else {
    H[o] = cconj(hs[(size_t)j * ld + i]);
    S[o] = cconj(hs[(size_t)i * ld + j]);
  }
}

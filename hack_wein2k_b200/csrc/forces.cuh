// forces.cuh -- adjoint of the H/S setup: band-energy gradients on the atoms.
//
// E = sum_n f_n eps_n of the generalized problem H c = eps S c that SECLR4
// solves from the packed state: H from conj of the lower triangle, S the
// transpose of the conj of the upper one (ZHCGST factors S**T), so that
// H(I,J) = conj(HS(I,J)) and S(I,J) = conj(HS(J,I)) for I > J.
// Hellmann-Feynman for that problem gives
//   dE/dr = sum_n f_n c_n^H (dH/dr - eps_n dS/dr) c_n.
// Atom positions r_a (POS, lattice coordinates) enter the setup only through
// the structure-factor phases exp(2 pi i KZZ . r_a): every contribution of
// atom a to the packed element HS(I,J), I > J (lower, H) or HS(J,I) (upper,
// S) carries exp(2 pi i (KZZ_J - KZZ_I) . r_a).  With D = 2 pi (KZZ_I -
// KZZ_J), h = conj(HS_a(I,J)) and s = conj(HS_a(J,I)) the pair adds
//   dE/dr_a,c += -2 D_c [ Im(h rho(J,I)) - Im(s rhoE(J,I)) ]
// where rho(J,I) = sum_n f_n c_n(J) conj(c_n(I)) and rhoE carries f_n eps_n.
// Diagonal elements do not depend on the positions (D = 0).  Radial
// functions, rotations (ROTIJ, ROTLOC) and the warped potential are held
// fixed: the result is the gradient of the setup as a function of POS.
//   k_force_sph   PW x PW pairs: the spherical sums of k_spherical; the
//                 step-function term 3 V BESR of each atom (k_table) depends
//                 on the pair only through dK, so the pairs are binned by dK
//                 and k_force_step sums the bins per atom
//   k_force_rsph, k_force_pre, k_force_bins  (split precision) the PW x PW
//                 pairs of two different row blocks as int8 projections by
//                 the addition theorem, against a running prefix; the pairs
//                 inside a block stay on k_force_sph (see below k_force_step)
//   k_force_lo    local-orbital columns, per equivalent atom (k_lo's terms)
//   k_force_hns_reduce  the HNS update through its factors.  HNS adds
//                 A(I,J) = X_J^T T conj(X_I) with X = (ALM, BLM, CLM) per atom
//                 and T the Hermitian 3x3 block of (TUU TDU TUU21 / TUD TDD
//                 TUD21 / TUU12 TDU12 TUU22), so A is Hermitian, the summand
//                 is symmetric in (I, J) and the lower-triangle sum is half
//                 the full one, which factors as
//                   -Im sum_n f_n sum_k [Y0 conj(Zc) - Yc conj(Z0)],
//                 Y = conj(X)^T (G c), Z = T Y.  Y = R^H (G c) for the
//                 (ALM, BLM) rows and CLM^H (G c) over the LO rows (library
//                 ZGEMMs); Z = T Y per atom (k_force_hns_z, zc = 0 and 1):
//                 for the CLM rows this is the CLM row of T applied to
//                 plane-wave rows too, which the lower triangle never uses
#pragma once
#include "kernels_fp64.cuh"

#define FRC_2PI 6.283185307179586476925287

// Rows of the spherical force operands, per (type, l, row): the J side
// (a, b) and the I side, S = vif (a, chn b) and H = vif (mAA a + mAB b,
// mBA a + mBB b), so that each l term of a pair is one 2-vector dot
// product per side.  Rows nv..nvpad-1 are zero (k_albl zeroes them).
__global__ void k_force_rows(DevProb P, const SphCoef* __restrict__ coef, double2* __restrict__ rowJ,
                             double2* __restrict__ rowI) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, tl = blockIdx.y;  // tl = type * ltop + l
  if (r >= P.nvpad) return;
  const size_t o = (size_t)tl * P.nvpad + r;
  const double a = P.al[o], b = P.bl[o];
  const SphCoef c = coef[tl];
  rowJ[o] = cmk(a, b);
  rowI[2 * o] = cmk(c.vif * a, c.vif * (c.chn * b));
  rowI[2 * o + 1] = cmk(c.vif * (c.mAA * a + c.mAB * b), c.vif * (c.mBA * a + c.mBB * b));
}

#define FRC_THREADS 256
#define FRC_MAXA 16  // equivalent atoms per staged chunk (a type with more reads its phases from global)
#define FRC_LT 11    // l count of the specialised kernel (lmax = 10)

// types per staged chunk: as many as the shared memory holds twice
__host__ __device__ constexpr int frc_tc(int lt) { return lt <= FRC_LT ? 5 : 4; }

__device__ __forceinline__ void frc_cp16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void frc_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void frc_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A chunk of types from t0: up to TC types whose equivalent atoms fit
// FRC_MAXA; a single type with more atoms forms a chunk of its own whose
// phases are not staged.
struct FrcChunk {
  int ntc, na, staged;
};
template <int TC>
__device__ __forceinline__ FrcChunk frc_chunk(const DevProb& P, int t0) {
  FrcChunk c{0, 0, 1};
  while (c.ntc < TC && t0 + c.ntc < P.nat && c.na + P.mult[t0 + c.ntc] <= FRC_MAXA) c.na += P.mult[t0 + c.ntc++];
  if (c.ntc == 0) c = FrcChunk{1, 0, 0};
  return c;
}

// dynamic shared memory: two stages of type rows (J: 1, I: 2 double2 per
// row and l) and of phases, two buffers of the per-warp force totals of a
// chunk's atoms (one per warp and component), and -4 pi KZZ of the tile's
// 64 rows
#define FRC_WARPS (FRC_THREADS / 32)
__host__ __device__ constexpr int frc_smem_bytes(int lt) {
  return (2 * frc_tc(lt) * lt * SPH_T * 3 + 2 * 2 * FRC_MAXA * SPH_T) * 16 + 2 * FRC_MAXA * 3 * FRC_WARPS * 8 +
         2 * SPH_T * 4 * 8;
}

// One block per 32 x 32 pair tile, 256 threads.  Thread (warp, lane) owns
// the 2 x 2 pairs J = j0 + jl0 + {0, 8}, I = i0 + il0 + {0, 4} with
// jl0 = 16 (warp & 1) + (lane & 7), il0 = 8 (warp >> 1) + (lane >> 3):
// a warp reads 8 distinct J rows and 4 distinct I rows per l, so that the
// shared-memory reads (about one cycle each: the addresses of a read are
// 8 or 4 distinct 16-byte words) stay below the FP64 pipe's rate.  The
// Legendre weights, rho, rhoE and dK of the four pairs stay in registers
// for all types.  The type rows (k_force_rows) and the phases of a chunk
// are copied into shared memory by cp.async one chunk ahead (double
// buffer), one warp per 32-row segment.  One block barrier per chunk: the
// per-warp force totals of a chunk go to one of two buffers and are summed
// over the warps (and added to F) after the next chunk's barrier.
template <int LT, bool GUARD>
__global__ void __launch_bounds__(FRC_THREADS, 1)
    k_force_sph(DevProb P, const int2* __restrict__ tiles, const double2* __restrict__ rowJ,
                const double2* __restrict__ rowI, TabDesc T, const double2* __restrict__ rho,
                const double2* __restrict__ rhoe, int ldr, int rt, double* __restrict__ F, double* __restrict__ bins) {
  constexpr int TC = frc_tc(LT);
  extern __shared__ double2 sm2[];
  double2* sJ = sm2;                       // [2][TC][LT][SPH_T]
  double2* sI = sJ + 2 * TC * LT * SPH_T;  // [2][TC][LT][SPH_T][S, H]
  double2* sP = sI + 4 * TC * LT * SPH_T;  // [2][J, I][FRC_MAXA][SPH_T]
  double* red = reinterpret_cast<double*>(sP + 4 * FRC_MAXA * SPH_T);  // [2][FRC_MAXA][3][warps]
  double* sK = red + 2 * FRC_MAXA * 3 * FRC_WARPS;                       // [J 0..31, I 32..63][4]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int2 t = tiles[blockIdx.x];
  const int i0 = t.x * SPH_T, j0 = t.y * SPH_T;
  const int nv = P.nv, ltop = P.ltop, nat = P.nat, nvpad = P.nvpad;
  const int jl0 = (warp & 1) * 16 + (lane & 7), il0 = (warp >> 1) * 8 + (lane >> 3);

  // (type, l) rows of consecutive types are consecutive in rowJ / rowI:
  // the chunk's rows are k = 0 .. ntc ltop - 1 from row t0 ltop, and with
  // ltop = LT also consecutive in shared memory
  auto stage = [&](int st, int t0, const FrcChunk& ch) {
    double2* dJ = sJ + st * TC * LT * SPH_T;
    double2* dI = sI + st * 2 * TC * LT * SPH_T;
    const size_t g0 = (size_t)t0 * ltop;
    for (int k = warp; k < ch.ntc * ltop; k += FRC_THREADS / 32) {
      const int ks = GUARD ? (k / ltop) * LT + k % ltop : k;
      const double2* src = rowJ + (g0 + k) * nvpad + j0;
      frc_cp16(dJ + ks * SPH_T + lane, src + lane);
      const double2* srci = rowI + 2 * ((g0 + k) * nvpad + i0);
      frc_cp16(dI + ks * 2 * SPH_T + lane, srci + lane);
      frc_cp16(dI + ks * 2 * SPH_T + SPH_T + lane, srci + SPH_T + lane);
    }
    if (ch.staged) {
      double2* dP = sP + st * 2 * FRC_MAXA * SPH_T;
      const int a0c = P.afirst[t0];
      for (int k = warp; k < ch.na * 2; k += FRC_THREADS / 32) {
        const int side = k & 1, e = k >> 1;
        frc_cp16(dP + (side * FRC_MAXA + e) * SPH_T + lane,
                 P.phase + (size_t)(a0c + e) * P.npad + (side ? i0 : j0) + lane);
      }
    }
    frc_commit();
  };

  FrcChunk ch = frc_chunk<TC>(P, 0);
  stage(0, 0, ch);
  // the pair term carries -2 (2 pi dK) = -4 pi (KZZ_I - KZZ_J): per row
  // -4 pi KZZ, read once per atom
  if (tid < 2 * SPH_T) {
    const int R = (tid < SPH_T ? j0 : i0 - SPH_T) + tid;
    const bool in = R < nv;
#pragma unroll
    for (int c = 0; c < 3; c++) sK[tid * 4 + c] = in ? -2.0 * FRC_2PI * P.kzz[3 * R + c] : 0.0;
    sK[tid * 4 + 3] = 0.0;
  }

  double w[4][LT];
  double2 rj[4], re[4];  // rho(J,I) and rhoE(J,I) of the owned pairs; zero for inactive pairs
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int J = j0 + jl0 + 8 * (q >> 1), I = i0 + il0 + 4 * (q & 1);
    const bool act = (J < nv && I < nv && J < I);
    double x = 0.0;
    rj[q] = re[q] = cmk(0.0, 0.0);
    if (act) {
      x = P.xk[I] * P.xk[J] + P.yk[I] * P.yk[J] + P.zk[I] * P.zk[J];
      double den = P.rk[I] * P.rk[J];
      if (den > 1.0e-8) x = x / den;
      const int d0 = P.kzz[3 * I] - P.kzz[3 * J], d1 = P.kzz[3 * I + 1] - P.kzz[3 * J + 1],
                d2 = P.kzz[3 * I + 2] - P.kzz[3 * J + 2];
      // rt: the density matrices hold conj(rho(J,I)) at (I, J) instead
      rj[q] = rt ? cconj(rho[(size_t)J * ldr + I]) : rho[(size_t)I * ldr + J];
      re[q] = rt ? cconj(rhoe[(size_t)J * ldr + I]) : rhoe[(size_t)I * ldr + J];
      // the step-function term depends on the pair only through dK =
      // KZZ_I - KZZ_J: bin x2 rho - rhoE by dK (k_force_step finishes it)
      const size_t b = (((size_t)(d2 + T.d3) * (2 * T.d2 + 1)) + (d1 + T.d2)) * (2 * T.d1 + 1) + (d0 + T.d1);
      const double x2q = P.xk[J] * P.xk[I] + P.yk[J] * P.yk[I] + P.zk[J] * P.zk[I];
      atomicAdd(&bins[2 * b], x2q * rj[q].x - re[q].x);
      atomicAdd(&bins[2 * b + 1], x2q * rj[q].y - re[q].y);
    }
    const bool top = !(fabs(x) < 0.9999999);
    double pm2 = 1.0, pm1 = x;
    w[q][0] = 1.0;
    if (LT > 1) w[q][1] = 3.0 * x;
#pragma unroll
    for (int l = 2; l < LT; l++) {
      double pl;
      if (!top) {
        const double pplx = x * pm1;
        pl = pplx + ((double)(l - 1) / (double)l) * (pplx - pm2);
      } else {
        pl = x * pm1;
      }
      pm2 = pm1;
      pm1 = pl;
      w[q][l] = (double)(2 * l + 1) * pl;
    }
  }

  // sum over the warps of a staged chunk's per-warp totals (red buffer rb),
  // one thread per (atom, component)
  auto flush = [&](int rb, int a0, int na) {
    if (tid < na * 3) {
      const double* r = red + ((size_t)rb * FRC_MAXA * 3 + tid) * FRC_WARPS;
      double sacc = 0.0;
#pragma unroll
      for (int w = 0; w < FRC_WARPS; w++) sacc += r[w];
      atomicAdd(&F[(a0 + tid / 3) * 3 + tid % 3], sacc);
    }
  };
  int st = 0;
  int pa0 = 0, pna = 0;  // atoms of the previous chunk, flushed after this chunk's barrier
  for (int t0 = 0; t0 < nat;) {
    const int t1 = t0 + ch.ntc;
    frc_wait<0>();    // this thread's copies of the chunk (issued one chunk earlier)
    __syncthreads();  // every thread's copies landed; every warp is past the previous chunk
    FrcChunk nx{0, 0, 1};
    if (t1 < nat) {  // into the stage the previous chunk read
      nx = frc_chunk<TC>(P, t1);
      stage(st ^ 1, t1, nx);
    }
    flush(st ^ 1, pa0, pna);
    const double2* cJ = sJ + st * TC * LT * SPH_T;
    const double2* cI = sI + st * 2 * TC * LT * SPH_T;
    const double2* cPJ = sP + st * 2 * FRC_MAXA * SPH_T;
    const double2* cPI = cPJ + FRC_MAXA * SPH_T;
    const int a0c = P.afirst[t0];
    // l sums of type tc for the four pairs
    auto lsum = [&](int tc, double(&tS)[4], double(&tH)[4]) {
      const double2* bJ = cJ + tc * LT * SPH_T + jl0;
      const double2* bI = cI + tc * LT * 2 * SPH_T + 2 * il0;
      // the row values of l + 1 are read while l is summed
      double2 av[2] = {bJ[0], bJ[8]}, sv[2] = {bI[0], bI[8]}, hv[2] = {bI[1], bI[9]};
#pragma unroll
      for (int l = 0; l < LT; l++) {
        if (GUARD && l >= ltop) break;
        const double2 a0 = av[0], a1 = av[1], s0 = sv[0], s1 = sv[1], h0 = hv[0], h1 = hv[1];
        if (l + 1 < LT) {
          const int o = (l + 1) * SPH_T;
          av[0] = bJ[o];
          av[1] = bJ[o + 8];
          sv[0] = bI[2 * o];
          sv[1] = bI[2 * o + 8];
          hv[0] = bI[2 * o + 1];
          hv[1] = bI[2 * o + 9];
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const double2 a = (q >> 1) ? a1 : a0, s = (q & 1) ? s1 : s0, h = (q & 1) ? h1 : h0;
          if (l == 0) {  // w_0 = P_0 = 1
            tS[q] = fma(a.y, s.y, a.x * s.x);
            tH[q] = fma(a.y, h.y, a.x * h.x);
          } else {
            tS[q] = fma(w[q][l], fma(a.y, s.y, a.x * s.x), tS[q]);
            tH[q] = fma(w[q][l], fma(a.y, h.y, a.x * h.x), tH[q]);
          }
        }
      }
    };
    // one atom's force over the warp's pairs (phases fj of the J rows, fi
    // of the I rows): returns, in lanes 0, 8 and 16, the warp's total of
    // components 0, 1 and 2 (a transposed reduction: six shuffles for the
    // three components)
    auto fterm = [&](const double2(&fj)[2], const double2(&fi)[2], const double(&tS)[4],
                     const double(&tH)[4]) -> double {
      double g[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        // cP = conj(phi_J) phi_I = conj(PHASE_a(J,I)); inactive pairs have
        // rho = rhoE = 0 and add nothing
        const double2 pj = fj[q >> 1], pi = fi[q & 1];
        const double cpr = fma(pj.x, pi.x, pj.y * pi.y);
        const double cpi = fma(pj.x, pi.y, -(pj.y * pi.x));
        const double uim = fma(cpr, rj[q].y, cpi * rj[q].x);  // Im(cP rho(J,I))
        const double vim = fma(cpr, re[q].y, cpi * re[q].x);  // Im(cP rhoE(J,I))
        g[q] = fma(tH[q], uim, -(tS[q] * vim));
      }
      // sum_q g_q (K_I - K_J): by I row and by J row
      const double gi0 = g[0] + g[2], gi1 = g[1] + g[3], gj0 = g[0] + g[1], gj1 = g[2] + g[3];
      const double2* k2 = reinterpret_cast<const double2*>(sK);  // row r: k2[2r] = (x, y), k2[2r + 1].x = z
      const double2 kI0 = k2[2 * (SPH_T + il0)], kI1 = k2[2 * (SPH_T + il0 + 4)];
      const double2 kJ0 = k2[2 * jl0], kJ1 = k2[2 * (jl0 + 8)];
      const double zI0 = k2[2 * (SPH_T + il0) + 1].x, zI1 = k2[2 * (SPH_T + il0 + 4) + 1].x;
      const double zJ0 = k2[2 * jl0 + 1].x, zJ1 = k2[2 * (jl0 + 8) + 1].x;
      const double f0 = fma(gi0, kI0.x, fma(gi1, kI1.x, -fma(gj0, kJ0.x, gj1 * kJ1.x)));
      const double f1 = fma(gi0, kI0.y, fma(gi1, kI1.y, -fma(gj0, kJ0.y, gj1 * kJ1.y)));
      const double f2 = fma(gi0, zI0, fma(gi1, zI1, -fma(gj0, zJ0, gj1 * zJ1)));
      // lanes 0..15 keep components (0, 1), lanes 16..31 (2, none); then
      // lanes with bit 3 clear keep the first, the others the second; then
      // the sum over lane & 7
      const bool lo16 = (lane & 16) == 0, lo8 = (lane & 8) == 0;
      const double k0 = (lo16 ? f0 : f2) + __shfl_xor_sync(0xffffffffu, lo16 ? f2 : f0, 16);
      const double k1 = (lo16 ? f1 : 0.0) + __shfl_xor_sync(0xffffffffu, lo16 ? 0.0 : f1, 16);
      double v = (lo8 ? k0 : k1) + __shfl_xor_sync(0xffffffffu, lo8 ? k1 : k0, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      return v;
    };
    // staged atom slot e of the chunk: the warp's totals into red buffer st
    auto fstaged = [&](int e, const double(&tS)[4], const double(&tH)[4]) {
      const int b = e * SPH_T;
      const double2 fj[2] = {cPJ[b + jl0], cPJ[b + jl0 + 8]}, fi[2] = {cPI[b + il0], cPI[b + il0 + 4]};
      const double v = fterm(fj, fi, tS, tH);
      if ((lane & 7) == 0 && lane < 24) red[(((size_t)st * FRC_MAXA + e) * 3 + (lane >> 3)) * FRC_WARPS + warp] = v;
    };
    if (ch.staged && ch.na == ch.ntc) {
      // one atom per type (slot tc): the force terms of type tc - 1 are
      // formed in the same straight-line block as the l sums of type tc,
      // so that the reduction's latency overlaps the sums
      double pS[4], pH[4];
      lsum(0, pS, pH);
      for (int tc = 1; tc < ch.ntc; tc++) {
        double tS[4], tH[4];
        lsum(tc, tS, tH);
        fstaged(tc - 1, pS, pH);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          pS[q] = tS[q];
          pH[q] = tH[q];
        }
      }
      fstaged(ch.ntc - 1, pS, pH);
    } else {
      for (int tc = 0; tc < ch.ntc; tc++) {
        double tS[4], tH[4];
        lsum(tc, tS, tH);
        const int jn = t0 + tc, ae = P.afirst[jn], me = P.mult[jn];
        for (int e = 0; e < me; e++) {
          if (ch.staged) {
            fstaged(ae - a0c + e, tS, tH);
          } else {
            const double2* pa = P.phase + (size_t)(ae + e) * P.npad;
            const double2 fj[2] = {pa[j0 + jl0], pa[j0 + jl0 + 8]}, fi[2] = {pa[i0 + il0], pa[i0 + il0 + 4]};
            const double v = fterm(fj, fi, tS, tH);
            if ((lane & 7) == 0 && lane < 24) atomicAdd(&F[(ae + e) * 3 + (lane >> 3)], v);
          }
        }
      }
    }
    pa0 = a0c;
    pna = ch.staged ? ch.na : 0;
    t0 = t1;
    ch = nx;
    st ^= 1;
  }
  __syncthreads();
  flush(st ^ 1, pa0, pna);
}

// Step-function part of the spherical force: with B(dK) = sum over pairs
// J < I with KZZ_I - KZZ_J = dK of (x2 rho(J,I) - rhoE(J,I)) (binned by
// k_force_sph), atom a of type t gets
//   dE/dr_a,c += sum_dK -2 (3 V_t) BESR(|dK| R_t) Im(exp(2 pi i dK.r_a) B(dK)) 2 pi dK_c
// (the 3 V BESR term of k_table for that atom).  One block per atom.
__global__ void __launch_bounds__(256) k_force_step(DevProb P, TabDesc T, const double* __restrict__ bins,
                                                    double* __restrict__ F) {
  __shared__ double red[3][256];
  const int a = blockIdx.x, jn = P.atype[a];
  const double v3 = 3.0 * P.v[jn], rt = P.rmt[jn];
  const double* r = P.pos + 3 * a;
  const int nx = 2 * T.d1 + 1, ny = 2 * T.d2 + 1, nz = 2 * T.d3 + 1;
  const long nb = (long)nx * ny * nz;
  double acc[3] = {0.0, 0.0, 0.0};
  for (long q = threadIdx.x; q < nb; q += blockDim.x) {
    const double bx = bins[2 * q], by = bins[2 * q + 1];
    if (bx == 0.0 && by == 0.0) continue;
    const int d0 = (int)(q % nx) - T.d1, d1 = (int)((q / nx) % ny) - T.d2, d2 = (int)(q / ((long)nx * ny)) - T.d3;
    const double g0 = T.bk[0] * d0 + T.bk[1] * d1 + T.bk[2] * d2;
    const double g1 = T.bk[3] * d0 + T.bk[4] * d1 + T.bk[5] * d2;
    const double g2 = T.bk[6] * d0 + T.bk[7] * d1 + T.bk[8] * d2;
    const double h = sqrt(g0 * g0 + g1 * g1 + g2 * g2) * rt;
    double sn, cs;
    sincos(h, &sn, &cs);
    const double besr = (h * cs - sn) * (1.0 / (h * h * h));
    const double2 ph = cexp2pi(r[0] * d0 + r[1] * d1 + r[2] * d2);
    const double im = ph.x * by + ph.y * bx;  // Im(exp(2 pi i dK.r) B)
    const double gq = -2.0 * v3 * besr * im * FRC_2PI;
    acc[0] = fma(gq, (double)d0, acc[0]);
    acc[1] = fma(gq, (double)d1, acc[1]);
    acc[2] = fma(gq, (double)d2, acc[2]);
  }
  for (int c = 0; c < 3; c++) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 3; c++) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) atomicAdd(&F[a * 3 + threadIdx.x], red[threadIdx.x][0]);
}

// ---------------------------------------------------------------------
// The spherical pair sums as projections (split precision).
//
// By the addition theorem (2l+1) P_l(u.v) = sum_m Z_lm(u) Z_lm(v) for the
// real spherical harmonics Z_lm scaled as below, so the type term of a pair
// factors into row vectors: tH(I,J) = sum_(l,m) sum_(alpha,beta)
// A^alpha_J Z_lm(J) M^(alpha beta)_l A^beta_I Z_lm(I) with A = (al, bl),
// M_H = vif (mAA mAB / mBA mBB), M_S = vif diag(1, chn).  With y_b(I) =
// conj(phase_a(I)) c_b(I), conj(phase_J) phase_I rho(J,I) = sum_b f_b y_b(J)
// conj(y_b(I)), and with kappa = 2 pi KZZ the pair weight -4 pi (KZZ_I -
// KZZ_J) = -2 (kappa_I - kappa_J), so that the PW x PW part of atom a's
// gradient over pairs J < I with J in a set Jset and I in a set Iset is
//   -2 sum_(l,m,alpha,beta,b) M^(alpha beta)_l (f_b | f_b eps_b) Im(
//       Pj_alpha conj(Yk_beta) - Pk_alpha conj(Y_beta))
// where P = sum_(J in Jset) A^alpha Z_lm conj(phase_a) (c, kappa c)(J) and Y
// the same over Iset.  J < I is a triangle, not a product of two sets: the
// PW rows are cut into blocks of B rows; the pairs of two different blocks
// are the projections of block p (Y) against the sum of the projections of
// the blocks before it (the prefix P), the pairs inside a block go through
// k_force_sph on the diagonal tiles.  The projections are int8 slice
// products (k_split_gemm) of the left operand of k_force_rsph with (G c)^T.
// Rows whose |k| is 0 use the direction z (their al, bl vanish for l > 0).
// The pair kernel uses P_l = x P_(l-1) for |x| >= 0.9999999 (hamilt.F's
// UTOP branch); the projections use P_l itself (the same value at |x| = 1).

// Z_lm(u) for the unit vector u, lm = l l + l + m: m = 0: N_l0 Q_l0(uz);
// m > 0 and m < 0: sqrt(2) N_l|m| Q_l|m|(uz) times Re and Im of (ux + i uy)^|m|,
// with P_l^m = (1 - uz^2)^(m/2) Q_lm (no Condon-Shortley phase; Q_mm =
// (2m-1)!!, Q_(m+1)m = (2m+1) uz Q_mm, then the three-term recursion in l)
// and N_lm = sqrt((2l+1) (l-m)!/(l+m)!), so that sum_m Z_lm(u) Z_lm(v) =
// (2l+1) P_l(u.v).
__device__ double frc_zlm(double ux, double uy, double uz, int l, int m) {
  const int am = m < 0 ? -m : m;
  double q0 = 1.0;
  for (int k = 1; k <= am; k++) q0 *= (double)(2 * k - 1);
  double q = q0;
  if (l > am) {
    double qm2 = q0, qm1 = (double)(2 * am + 1) * uz * q0;
    for (int ll = am + 2; ll <= l; ll++) {
      const double qn = ((double)(2 * ll - 1) * uz * qm1 - (double)(ll + am - 1) * qm2) / (double)(ll - am);
      qm2 = qm1;
      qm1 = qn;
    }
    q = qm1;
  }
  double fr = 1.0;
  for (int k = l - am + 1; k <= l + am; k++) fr /= (double)k;
  const double nrm = sqrt((double)(2 * l + 1) * fr);
  if (am == 0) return nrm * q;
  double cr = 1.0, ci = 0.0;
  for (int k = 0; k < am; k++) {
    const double tr = cr * ux - ci * uy;
    ci = cr * uy + ci * ux;
    cr = tr;
  }
  return 1.4142135623730951 * nrm * q * (m > 0 ? cr : ci);
}

__device__ __forceinline__ int frc_lof(int lm) {
  int l = (int)sqrt((double)lm);
  while (l * l > lm) l--;
  while ((l + 1) * (l + 1) <= lm) l++;
  return l;
}

// Left operand of the projections, k-major: row I < NV of Lt (stride ld)
// holds, at r = (a 2 + alpha) ltop^2 + lm, A^alpha_(t l)(I) Z_lm(k_I)
// conj(phase_a(I)) for atom a of type t (alpha 0: al, 1: bl).  One block
// per row.
__global__ void __launch_bounds__(256) k_force_rsph(DevProb P, double2* __restrict__ Lt, int ld) {
  __shared__ double z[L1G_MAXL * L1G_MAXL];
  __shared__ unsigned char lof[L1G_MAXL * L1G_MAXL];
  const int I = blockIdx.x;
  const int L2 = P.ltop * P.ltop;
  if ((int)threadIdx.x < L2) {
    double ux = 0.0, uy = 0.0, uz = 1.0;
    const double r = P.rk[I];
    if (r > 0.0) {
      ux = P.xk[I] / r;
      uy = P.yk[I] / r;
      uz = P.zk[I] / r;
    }
    const int lm = threadIdx.x, l = frc_lof(lm);
    z[lm] = frc_zlm(ux, uy, uz, l, lm - l * l - l);
    lof[lm] = (unsigned char)l;
  }
  __syncthreads();
  const int per = 2 * L2, K = P.ndf * per;
  double2* out = Lt + (size_t)I * ld;
  for (int r = threadIdx.x; r < K; r += blockDim.x) {
    const int a = r / per, rem = r - a * per, alpha = rem >= L2 ? 1 : 0, lm = rem - alpha * L2;
    const size_t o = ((size_t)P.atype[a] * P.ltop + lof[lm]) * P.nvpad + I;
    const double v = (alpha ? P.bl[o] : P.al[o]) * z[lm];
    const double2 ph = P.phase[(size_t)a * P.npad + I];
    out[r] = cmk(v * ph.x, -v * ph.y);
  }
}

// One block of rows against the prefix: Y and Pre are K x 4nb column-major
// (stride ld; column g nb + b: g = 0 the plain projection of band b, g =
// 1..3 the kappa_g-weighted one), rows r = (a 2 + alpha) ltop^2 + lm.
// Adds block p's cross-block pair sums to F and, with update, Pre += Y.
// One block per (atom, FRC_PB bands); thread = lm, both alpha rows.
#define FRC_PB 8
// the default (lapw1gpu_set_force_projection slices -1): 6 slices (at 5 the
// c1 adjoint's error grew from 2.5e-8 to 1.2e-5 of its largest component),
// on when the PW rows span 6 blocks (at c1, 4.5 blocks of 1024 rows, the
// projections took 6.97 ms against 6.09 for the pair kernel alone; at c4,
// 11.6 blocks, 57.3 against 73.7 ms for the whole adjoint)
#define L1G_FSP_SLICES 6
#define L1G_FSP_MIN_BLOCKS 6
__global__ void __launch_bounds__(128) k_force_pre(DevProb P, const SphCoef* __restrict__ coef,
                                                   const double2* __restrict__ Y, double2* __restrict__ Pre, int ld,
                                                   int nb, const double* __restrict__ f,
                                                   const double* __restrict__ eps, int update,
                                                   double* __restrict__ F) {
  __shared__ double red[4][3];
  const int a = blockIdx.x, b0 = blockIdx.y * FRC_PB, b1 = min(nb, b0 + FRC_PB);
  const int L2 = P.ltop * P.ltop, t = P.atype[a];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int lm = threadIdx.x; lm < L2; lm += blockDim.x) {
    const SphCoef cf = coef[t * P.ltop + frc_lof(lm)];
    const double hAA = cf.vif * cf.mAA, hAB = cf.vif * cf.mAB, hBA = cf.vif * cf.mBA, hBB = cf.vif * cf.mBB;
    const double sAA = cf.vif, sBB = cf.vif * cf.chn;
    const size_t r0 = (size_t)a * 2 * L2 + lm, r1 = r0 + L2;
    for (int b = b0; b < b1; b++) {
      double2 p[2][4], y[2][4];
#pragma unroll
      for (int g = 0; g < 4; g++) {
        const size_t o = (size_t)(g * nb + b) * ld;
        p[0][g] = Pre[o + r0];
        p[1][g] = Pre[o + r1];
        y[0][g] = Y[o + r0];
        y[1][g] = Y[o + r1];
      }
      const double fb = f[b], fe = f[b] * eps[b];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        double X[2][2];
#pragma unroll
        for (int al = 0; al < 2; al++)
#pragma unroll
          for (int be = 0; be < 2; be++) {
            // Im(p conj(y)) = p.y y.x - p.x y.y
            const double2 p0 = p[al][0], pk = p[al][c + 1], y0 = y[be][0], yk = y[be][c + 1];
            X[al][be] = fma(p0.y, yk.x, -(p0.x * yk.y)) - fma(pk.y, y0.x, -(pk.x * y0.y));
          }
        const double tH = fma(hAA, X[0][0], fma(hAB, X[0][1], fma(hBA, X[1][0], hBB * X[1][1])));
        const double tS = fma(sAA, X[0][0], sBB * X[1][1]);
        acc[c] = fma(-2.0, fma(fb, tH, -(fe * tS)), acc[c]);
      }
      if (update) {
#pragma unroll
        for (int g = 0; g < 4; g++) {
          const size_t o = (size_t)(g * nb + b) * ld;
          Pre[o + r0] = cadd(p[0][g], y[0][g]);
          Pre[o + r1] = cadd(p[1][g], y[1][g]);
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w][threadIdx.x];
    atomicAdd(&F[a * 3 + threadIdx.x], v);
  }
}

// The step-function bins of k_force_sph alone, for the tiles whose pairs
// the projections cover (same thread-to-pair map, same bins).
__global__ void __launch_bounds__(FRC_THREADS) k_force_bins(DevProb P, const int2* __restrict__ tiles, TabDesc T,
                                                            const double2* __restrict__ rho,
                                                            const double2* __restrict__ rhoe, int ldr, int rt,
                                                            double* __restrict__ bins) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int2 t = tiles[blockIdx.x];
  const int i0 = t.x * SPH_T, j0 = t.y * SPH_T;
  const int nv = P.nv;
  const int jl0 = (warp & 1) * 16 + (lane & 7), il0 = (warp >> 1) * 8 + (lane >> 3);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int J = j0 + jl0 + 8 * (q >> 1), I = i0 + il0 + 4 * (q & 1);
    if (!(J < nv && I < nv && J < I)) continue;
    const double2 rj = rt ? cconj(rho[(size_t)J * ldr + I]) : rho[(size_t)I * ldr + J];
    const double2 re = rt ? cconj(rhoe[(size_t)J * ldr + I]) : rhoe[(size_t)I * ldr + J];
    const int d0 = P.kzz[3 * I] - P.kzz[3 * J], d1 = P.kzz[3 * I + 1] - P.kzz[3 * J + 1],
              d2 = P.kzz[3 * I + 2] - P.kzz[3 * J + 2];
    const size_t b = (((size_t)(d2 + T.d3) * (2 * T.d2 + 1)) + (d1 + T.d2)) * (2 * T.d1 + 1) + (d0 + T.d1);
    const double x2q = P.xk[J] * P.xk[I] + P.yk[J] * P.yk[I] + P.zk[J] * P.zk[I];
    atomicAdd(&bins[2 * b], x2q * rj.x - re.x);
    atomicAdd(&bins[2 * b + 1], x2q * rj.y - re.y);
  }
}

// local-orbital columns: k_lo's terms per equivalent atom, reduced per warp
__global__ void k_force_lo(DevProb P, const LoCol* __restrict__ cols, const double2* __restrict__ rho,
                           const double2* __restrict__ rhoe, int ldr, int rt, double* __restrict__ F) {
  const LoCol c = cols[blockIdx.y];
  const int nv = P.nv;
  const int I = nv + c.nnlo - 1;
  if ((int)(blockIdx.x * blockDim.x) >= I) return;  // no pair J < I in the block (block-uniform)
  const int J = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int jn = c.jn, l = c.l, jlo = c.jlo, jeqo = c.jeqo, mo1 = c.mo1, mult = P.mult[jn];
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
  bool inlo[L1G_NLOAT + 1];
  const int Jf = J + 1;
  bool any_lo = false;
  for (int jlop = 1; jlop <= jlo; jlop++) {
    int jbeg = nv + c.nnlo - (mo1 + l) - (2 * l + 1) * (jeqo - 1) - (jlo - jlop) * (2 * l + 1) * mult;
    int jend = nv + c.nnlo - (jlo - jlop) * (mo1 + l + 1) - (jlo - jlop) * (jeqo - 1) * (2 * l + 1);
    inlo[jlop] = (Jf >= jbeg && Jf <= jend);
    any_lo |= inlo[jlop];
  }
  const bool act = (J < I) && (J < nv || any_lo);
  double dxc[3] = {0.0, 0.0, 0.0};
  double2 rj = cmk(0.0, 0.0), re = cmk(0.0, 0.0);
  double alj = 0.0, blj = 0.0;
  if (act) {
    dxc[0] = FRC_2PI * (P.kzz[3 * I] - P.kzz[3 * J]);
    dxc[1] = FRC_2PI * (P.kzz[3 * I + 1] - P.kzz[3 * J + 1]);
    dxc[2] = FRC_2PI * (P.kzz[3 * I + 2] - P.kzz[3 * J + 2]);
    rj = rt ? cconj(rho[(size_t)J * ldr + I]) : rho[(size_t)I * ldr + J];
    re = rt ? cconj(rhoe[(size_t)J * ldr + I]) : rhoe[(size_t)I * ldr + J];
    if (J < nv) {
      size_t oo = ((size_t)jn * P.ltop + l) * P.nvpad + J;
      alj = P.al[oo];
      blj = P.bl[oo];
    }
  }
  // the LO row's Y_lm per equivalent atom, shared by the block (I is the
  // block's), in chunks of FRC_YCH atoms
  constexpr int FRC_YCH = 16;
  __shared__ double2 syi[FRC_YCH][16];
  for (int jeq = 0; jeq < mult; jeq++) {
    const int a = c.a0 + jeq;
    if (jeq % FRC_YCH == 0) {  // block-uniform
      __syncthreads();
      const int q = threadIdx.x;
      if (q < FRC_YCH && jeq + q < mult)
        dev_ylm_row<3>(P.xk[I], P.yk[I], P.zk[I], P.rotij + 9 * (a + q), P.rotloc + 9 * jn, l, syi[q]);
      __syncthreads();
    }
    double2 S = cmk(0.0, 0.0), H = cmk(0.0, 0.0);
    if (act) {
      const double* ra = P.pos + 3 * a;
      double s = ra[0] * (double)(P.kzz[3 * I] - P.kzz[3 * J]) + ra[1] * (double)(P.kzz[3 * I + 1] - P.kzz[3 * J + 1]) +
                 ra[2] * (double)(P.kzz[3 * I + 2] - P.kzz[3 * J + 2]);
      const double2 ph = cconj(cexp2pi(s));
      double2 yj[16];
      const double2* yi = syi[jeq % FRC_YCH];
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
    // HS(I,J) = H (lower), HS(J,I) = S (upper): h = conj(H), s = conj(S)
    const double uim = H.x * rj.y - H.y * rj.x;  // Im(conj(H) rho(J,I))
    const double vim = S.x * re.y - S.y * re.x;  // Im(conj(S) rhoE(J,I))
    const double g = act ? -2.0 * (uim - vim) : 0.0;
    // the block's sum (every block of a column belongs to one atom): warp
    // sums, then one atomic per component and block
    __shared__ double wsum[4][3];  // blockDim.x = 128: 4 warps
#pragma unroll
    for (int cc = 0; cc < 3; cc++) {
      double v = g * dxc[cc];
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_down_sync(0xffffffffu, v, o2);
      if (lane == 0) wsum[threadIdx.x >> 5][cc] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicAdd(&F[a * 3 + threadIdx.x], wsum[0][threadIdx.x] + wsum[1][threadIdx.x] +
                                                          wsum[2][threadIdx.x] + wsum[3][threadIdx.x]);
    __syncthreads();  // wsum is rewritten by the next equivalent atom
  }
#undef LOV
}

// GC[g][b][i] = G_g(i) C(i, b): g = 0 the plain block, g = 1..3 the rows
// scaled by 2 pi KZZ_g(i), for the HNS gradient GEMMs
__global__ void k_force_gscale(int n, int nb, const int* __restrict__ kzz, const double2* __restrict__ C, int ldc,
                               double2* __restrict__ GC) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= n) return;
  const double2 v = C[(size_t)b * ldc + i];
  GC[(size_t)b * n + i] = v;
#pragma unroll
  for (int c = 0; c < 3; c++) GC[((size_t)(c + 1) * nb + b) * n + i] = cscale(v, FRC_2PI * kzz[3 * i + c]);
}

// occupation- and energy-weighted copies of the eigenvector block
// out[c][r] = in[r][c] (conjugated when cj): in is rows x cols with row
// stride ldi, out cols x rows with row stride ldo; 32 x 32 tiles through
// shared memory, both sides coalesced
__global__ void __launch_bounds__(256) k_force_trans(const double2* __restrict__ in, int ldi, int rows, int cols,
                                                     int cj, double2* __restrict__ out, int ldo) {
  __shared__ double2 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int y = ty; y < 32; y += 8) {
    const int r = r0 + y, c = c0 + tx;
    double2 v = (r < rows && c < cols) ? in[(size_t)r * ldi + c] : cmk(0.0, 0.0);
    t[y][tx] = cj ? cconj(v) : v;
  }
  __syncthreads();
  for (int y = ty; y < 32; y += 8) {
    const int c = c0 + y, r = r0 + tx;
    if (c < cols && r < rows) out[(size_t)c * ldo + r] = t[tx][y];
  }
}

// Cf = f c, Ce = f eps c per band (cj: their conjugates, for the split
// path's products C conj(Cf)^T, which take no conjugate themselves)
__global__ void k_force_weight(int n, int nb, const double2* __restrict__ C, int ldc, const double* __restrict__ f,
                               const double* __restrict__ eps, int cj, double2* __restrict__ Cf,
                               double2* __restrict__ Ce) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (i >= n) return;
  double2 v = C[(size_t)b * ldc + i];
  if (cj) v = cconj(v);
  Cf[(size_t)b * n + i] = cscale(v, f[b]);
  Ce[(size_t)b * n + i] = cscale(v, f[b] * eps[b]);
}

// Z = T Y per atom: the product L^T (G c) through the small T of each atom
// instead of a second N x K GEMM, because L = M conj(R) (+ the CLM terms of
// the LO rows).  FRC_ZCOLS columns of Y per block: the atom type's T blocks
// and the columns' Y entries of the atom are staged in shared memory once;
// lane = column (the T entries a warp reads are one broadcast word, the
// columns' Y rows lie 3 NSL2 = 75 double2 apart: odd, so a warp's 16-byte
// reads do not conflict) and each thread keeps the NSL2 outputs of one T
// row (r) of its column in registers.  Y: [col][K] (k = (a*2 + r)*nsl2 + b), Yc, Zc: [col][Kc]
// (k = a*nsl2 + lm), col < ncol = 4 nb.
//   zc = 0: Z[a][(r, lm)] = sum_b T_(r,A)[lm][b] Y_A[b] + T_(r,B)[lm][b] Y_B[b]
//           (+ T_(r,C)[lm][b] Yc[b] with LOs), with (A, B, C) = (TUU, TDU,
//           TUU21) for r = 0 and (TUD, TDD, TUD21) for r = 1;
//   zc = 1: Zc[a][lm] = sum_b TUU12[lm][b] Y_A[b] + TDU12[lm][b] Y_B[b] +
//           TUU22[lm][b] Yc[b]: the CLM row of T applied to Y over all rows.
#define FRC_ZCOLS 128
#define FRC_ZSMEM ((6 * L1G_NSL2 * L1G_NSL2 + FRC_ZCOLS * 3 * L1G_NSL2) * 16)
__global__ void __launch_bounds__(256, 1) k_force_hns_z(int zc, int nsl2, int K, int Kc, int ncol,
                                                     const int* __restrict__ atype, const double2* __restrict__ tns,
                                                     const double2* __restrict__ Y, const double2* __restrict__ Yc,
                                                     double2* __restrict__ Z, double2* __restrict__ Zc) {
  extern __shared__ double2 zsm[];
  double2* sT = zsm;                            // [6 blocks][L1G_NSL2][L1G_NSL2]
  double2* sY = sT + 6 * L1G_NSL2 * L1G_NSL2;  // [FRC_ZCOLS][A, B, C][L1G_NSL2]
  const int a = blockIdx.y, c0 = blockIdx.x * FRC_ZCOLS, tid = threadIdx.x;
  const int nc = min(FRC_ZCOLS, ncol - c0);
  const double2* T = tns + (size_t)atype[a] * LAPW1GPU_NTNS * L1G_NSL2 * L1G_NSL2;
  const int nb = zc ? 3 : 6, b0 = zc ? 6 : 0;  // T blocks used
  // staging by cp.async (every copy in flight at once; the block has one
  // wave of work after it)
  for (int i = tid; i < nb * nsl2 * nsl2; i += blockDim.x) {
    const int blk = i / (nsl2 * nsl2), r = i % (nsl2 * nsl2), lm = r / nsl2, b = r % nsl2;
    frc_cp16(&sT[(blk * L1G_NSL2 + lm) * L1G_NSL2 + b], &T[((size_t)(b0 + blk) * L1G_NSL2 + lm) * L1G_NSL2 + b]);
  }
  for (int i = tid; i < nc * 3 * nsl2; i += blockDim.x) {
    const int cl = i / (3 * nsl2), r = i % (3 * nsl2), part = r / nsl2, b = r % nsl2;
    double2* dst = &sY[(cl * 3 + part) * L1G_NSL2 + b];
    if (part < 2)
      frc_cp16(dst, &Y[(size_t)(c0 + cl) * K + (size_t)a * 2 * nsl2 + part * nsl2 + b]);
    else if (Yc)
      frc_cp16(dst, &Yc[(size_t)(c0 + cl) * Kc + (size_t)a * nsl2 + b]);
    else
      *dst = cmk(0.0, 0.0);
  }
  frc_commit();
  frc_wait<0>();
  __syncthreads();
  // warp w: columns 32 (w % 4) + lane, outputs: zc = 0 the row r = w / 4
  // (lm = 0 .. nsl2-1), zc = 1 the lm half w / 4 of the single row
  const int lane = tid & 31, w = tid >> 5, cl = (w & 3) * 32 + lane, oh = w >> 2;
  const int half = (nsl2 + 1) / 2;
  const int ro = zc ? 0 : oh, lm0 = (zc && oh) ? half : 0, nlm = zc ? (oh ? nsl2 - half : half) : nsl2;
  const double2* tR = sT + (3 * ro) * L1G_NSL2 * L1G_NSL2;    // blocks (A, B, C) of row ro
  const double2* y = sY + (size_t)min(cl, nc - 1) * 3 * L1G_NSL2;  // columns past nc: computed, not stored
  double2 z[L1G_NSL2];
#pragma unroll
  for (int q = 0; q < L1G_NSL2; q++) z[q] = cmk(0.0, 0.0);
  for (int b = 0; b < nsl2; b++) {
    const double2 yA = y[b], yB = y[L1G_NSL2 + b], yC = y[2 * L1G_NSL2 + b];  // yC zero without LOs
#pragma unroll
    for (int q = 0; q < L1G_NSL2; q++) {
      if (q < nlm) {
        const double2* t = tR + (lm0 + q) * L1G_NSL2 + b;
        z[q] = cadd(z[q], cmul(t[0], yA));
        z[q] = cadd(z[q], cmul(t[L1G_NSL2 * L1G_NSL2], yB));
        z[q] = cadd(z[q], cmul(t[2 * L1G_NSL2 * L1G_NSL2], yC));
      }
    }
  }
  if (cl < nc) {
#pragma unroll
    for (int q = 0; q < L1G_NSL2; q++) {
      if (q < nlm) {
        const int lm = lm0 + q;
        if (zc)
          Zc[(size_t)(c0 + cl) * Kc + (size_t)a * nsl2 + lm] = z[q];
        else
          Z[(size_t)(c0 + cl) * K + (size_t)a * 2 * nsl2 + ro * nsl2 + lm] = z[q];
      }
    }
  }
}

// F_a,c -= Im sum_n f_n sum_{k in a} [Y0 conj(Zc) - Yc conj(Z0)]; Y*, Z* are
// [4][nb][K] (index 0: no G, 1..3: G_x, G_y, G_z), K = kper per atom
__global__ void k_force_hns_reduce(int kper, int K, int nb, const double2* __restrict__ Y, const double2* __restrict__ Z,
                                   const double* __restrict__ f, double* __restrict__ F) {
  const int a = blockIdx.x;
  __shared__ double red[3][256];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int q = threadIdx.x; q < kper * nb; q += blockDim.x) {
    const int kk = a * kper + q % kper, b = q / kper;
    const size_t o0 = (size_t)b * K + kk;
    const double2 y0 = Y[o0], z0 = Z[o0];
    const double fb = f[b];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const size_t oc = ((size_t)(c + 1) * nb + b) * K + kk;
      const double2 yc = Y[oc], zc = Z[oc];
      // Im(y0 conj(zc) - yc conj(z0))
      const double im = (y0.y * zc.x - y0.x * zc.y) - (yc.y * z0.x - yc.x * z0.y);
      acc[c] -= fb * im;
    }
  }
  for (int c = 0; c < 3; c++) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int c = 0; c < 3; c++) red[c][threadIdx.x] += red[c][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 3) atomicAdd(&F[a * 3 + threadIdx.x], red[threadIdx.x][0]);
}

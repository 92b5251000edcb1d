// sph_tc.cuh -- the spherical muffin-tin part of H and S (hamilt.F:371-440)
// on the 5th-generation tensor cores, split precision, sm_100a.
//
// For a pair (J <= I) HAMILT accumulates, per atom type and l,
//   S(J,I) += PHASE(J,I) (2l+1) P_l(x_JI) VIF [AL_J AL_I + CHN BL_J BL_I]
// and the same with the non-symmetric 2x2 block for H.  With PHASE =
// sum_eq phi_a(J) conj(phi_a(I)) the type and equivalent-atom sums at fixed
// l are one complex GEMM over k = (atom a, r in {AL, BL}):
//   G_l(J, I) = sum_k u_l(J,k) conj(v_l(I,k)),
//   u_l(J, (a,r)) = phi_a(J) {AL, BL}_(type a, l, J),
//   v_l(I, (a,r)) = phi_a(I) VIF {AL, CHN BL} (S) or VIF {hA, hB} (H),
// and the Legendre weight w_l(J,I) = (2l+1) P_l(x_JI), which couples J and I
// non-separably, is applied per pair as G_l leaves the accumulator:
//   aS(J,I) = sum_l w_l(J,I) G^S_l(J,I), aH likewise.
// The GEMMs run as Ozaki int8 slice products (the scheme of split_tc.cuh:
// power-of-two row scales, S slices, one exact int32 TMEM accumulator per
// level p+q-2 < S) with kind::i8 tcgen05.mma, M = 128 rows J, N = 4 real
// columns per I (S re, S im, H re, H im).  The accumulator is double
// buffered over l (2 x S levels x N columns of TMEM), so the FP64 epilogue
// of l (combine levels, scale, weight, accumulate per pair in registers)
// overlaps the MMAs of l+1.  After the last l the interstitial terms are
// gathered from the Theta/WARP table and HS is written as k_spherical does.
//
// Warp roles: warps 0..4 EG-1 epilogue (warp w reads TMEM lanes 32 (w%4)..
// and the I group w/4 of 4 I), warp 4 EG lane 0 issues the MMAs, warp
// 4 EG + 1 lane 0 the TMA loads (a full ring ahead of the MMAs, whatever
// they wait on).  Every
// mbarrier wait is bounded; a timeout sets a status bit and ends the CTA's
// work cleanly (copies drained, MMAs complete, TMEM freed).
#pragma once

namespace sphtc {

using split::desc_kblock;
using split::digit7;
using split::digit_scale;
using split::i2d_exact;
using split::idesc_i8;
using split::mbar_expect_tx;
using split::mbar_init;
using split::mbar_try_wait;
using split::mbar_wait;
using split::smem_u32;
using split::tc_fence_after;
using split::tc_fence_before;
using split::tma_load_3d;

// KB: bytes of K per pipeline stage and row (64: 64-byte swizzled rows, a
// deep ring; 128: 128-byte swizzled rows, half the TMA row requests per
// byte, two stages) -- a tunable tile shape
template <int S, int KB = 64>
struct Cfg {
  // real columns per level of one accumulator buffer: 4 per I, at most 48
  // (12 I: three epilogue warp groups of 4 I)
  static constexpr int NMAX = ((512 / (2 * S)) / 16) * 16;
  static constexpr int N = NMAX > 48 ? 48 : NMAX;
  static_assert(S * N <= 256, "one MMA per A slice needs (S - p) N <= 256 columns");
  static constexpr int IT = N / 4;   // I per tile
  static constexpr int IPT = 4;      // I per epilogue thread
  static constexpr int EG = IT / IPT;  // epilogue warp groups (4 warps each: the 4 TMEM lane quarters)
  static_assert(EG * IPT == IT, "I per tile must be a multiple of 4");
  static constexpr int EPI = 128 * EG;  // epilogue threads
  // one pipeline stage: all S slices of a KB-byte K block of A (128 rows)
  // and of B (N rows)
  static_assert(KB == 64 || KB == 128, "K block of 64 or 128 bytes");
  static constexpr int KSTEPS = KB / 32;  // 32-byte MMA K steps per stage
  static constexpr int A_BYTES = S * 128 * KB;
  static constexpr int B_BYTES = S * N * KB;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  // per-tile exponent tables: eA - 12 per (l, J) and eB per (l, I, S|H), int16
  static constexpr int SCALE_BYTES = (SPH_LMAX * 128 + SPH_LMAX * 2 * IT) * 2;
  static constexpr int STAGES_FIT = (227 * 1024 - SCALE_BYTES - 1024) / STAGE;
  static constexpr int STAGES = STAGES_FIT > 8 ? 8 : STAGES_FIT;
  static_assert(STAGES >= 2, "the ring needs two stages");
  static constexpr int SMEM = STAGES * STAGE + SCALE_BYTES + 1024;
  static constexpr int THREADS = EPI + 64;  // + the MMA warp and the TMA warp
};

// Operand rows of one l, built from AL/BL, phases and the per-(type, l)
// coefficients, then cut into S int8 slices with a power-of-two scale per
// complex row.  isB = 0: complex row J -> real row J = [Re u | Im u].
// isB = 1: complex row c = 2 I + m (m = 0 S, 1 H) -> real rows 2c =
// [Re v | Im v] and 2c+1 = [-Im v | Re v], so that a real dot product with
// [Re u | Im u] gives Re and Im of u conj(v).  out: [S][L][rows][Kp] int8,
// Kp = 2 Kcp; ex: [L][complex rows] exponents.  32 complex rows per block.
template <int S>
// A non-finite operand value sets L1G_STATUS_NONFINITE in status (int8
// slices cannot carry it into the products).
__global__ void __launch_bounds__(256, 2) k_sph_slice(DevProb P, const SphCoef* __restrict__ coef, int isB, int Kcp,
                                                      int ncrow, int8_t* __restrict__ out, int* __restrict__ ex,
                                                      int* __restrict__ status) {
  extern __shared__ double2 tile[];  // [Kc][33]
  __shared__ double red[8][32];
  __shared__ int rexp[32];
  const int l = blockIdx.y, L = P.ltop;
  const int rc0 = blockIdx.x * 32;
  const int tid = threadIdx.x;
  const int Kc = 2 * P.ndf, Kp = 2 * Kcp;
  const int nrow_real = isB ? 2 * ncrow : ncrow;  // real rows per l
  // values: one (row, atom) per thread and pass, AL/BL and the phase read
  // once for the atom's two k (and, for B, for both the S and H rows of I)
  const int nrr = isB ? 16 : 32;  // distinct basis rows of the block
  for (int idx = tid; idx < nrr * P.ndf; idx += 256) {
    const int rr = idx % nrr, a = idx / nrr;
    const int row = isB ? (rc0 >> 1) + rr : rc0 + rr;  // J or I
    double al = 0.0, bl = 0.0;
    double2 ph = make_double2(0.0, 0.0);
    const int t = P.atype[a];
    if (row < P.nv) {
      const size_t o = ((size_t)t * L + l) * P.nvpad + row;
      al = P.al[o];
      bl = P.bl[o];
      ph = P.phase[(size_t)a * P.npad + row];
    }
    if (!isB) {
      const bool in = rc0 + rr < ncrow;
      tile[(2 * a) * 33 + rr] = in ? make_double2(ph.x * al, ph.y * al) : make_double2(0.0, 0.0);
      tile[(2 * a + 1) * 33 + rr] = in ? make_double2(ph.x * bl, ph.y * bl) : make_double2(0.0, 0.0);
    } else {
      const SphCoef c = coef[t * L + l];
      const double xs0 = c.vif * al, xs1 = c.vif * (c.chn * bl);                                  // S row
      const double xh0 = c.vif * (c.mAA * al + c.mAB * bl), xh1 = c.vif * (c.mBA * al + c.mBB * bl);  // H row
      const bool in0 = rc0 + 2 * rr < ncrow, in1 = rc0 + 2 * rr + 1 < ncrow;
      tile[(2 * a) * 33 + 2 * rr] = in0 ? make_double2(ph.x * xs0, ph.y * xs0) : make_double2(0.0, 0.0);
      tile[(2 * a + 1) * 33 + 2 * rr] = in0 ? make_double2(ph.x * xs1, ph.y * xs1) : make_double2(0.0, 0.0);
      tile[(2 * a) * 33 + 2 * rr + 1] = in1 ? make_double2(ph.x * xh0, ph.y * xh0) : make_double2(0.0, 0.0);
      tile[(2 * a + 1) * 33 + 2 * rr + 1] = in1 ? make_double2(ph.x * xh1, ph.y * xh1) : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  {
    bool bad = false;
    for (int idx = tid; idx < 32 * Kc; idx += 256) bad |= l1g_nonfinite(tile[(idx >> 5) * 33 + (idx & 31)]);
    if (bad) atomicOr(status, L1G_STATUS_NONFINITE);
  }
  {
    const int r = tid & 31, part = tid >> 5;
    double m = 0.0;
    for (int k = part; k < Kc; k += 8) {
      const double2 v = tile[k * 33 + r];
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
    red[part][r] = m;
    __syncthreads();
    if (tid < 32) {
      double mm = 0.0;
      for (int q = 0; q < 8; q++) mm = fmax(mm, red[q][tid]);
      const int e = (mm > 0.0) ? ilogb(mm) + 1 : 0;
      rexp[tid] = e;
      if (rc0 + tid < ncrow) ex[(size_t)l * ncrow + rc0 + tid] = e;
    }
    __syncthreads();
  }
  // one element per thread and pass, lanes along k: conflict-free tile
  // reads (stride 33) and byte stores coalesced along each row
  const size_t plane = (size_t)L * nrow_real * Kp;  // one slice plane
  int8_t* lbase = out + (size_t)l * nrow_real * Kp;
  for (int idx = tid; idx < 32 * Kcp; idx += 256) {
    const int rr = idx / Kcp, k = idx - rr * Kcp;
    const int rc = rc0 + rr;
    if (rc >= ncrow) continue;
    const int e = rexp[rr];
    const double2 v = (k < Kc) ? tile[k * 33 + rr] : make_double2(0.0, 0.0);
    double tr = digit_scale(v.x, e), ti = digit_scale(v.y, e);
#pragma unroll
    for (int p = 0; p < S; p++) {
      const int8_t ar = (int8_t)digit7(tr), ai = (int8_t)digit7(ti);
      int8_t* base = lbase + (size_t)p * plane;
      if (!isB) {
        base[(size_t)rc * Kp + k] = ar;
        base[(size_t)rc * Kp + Kcp + k] = ai;
      } else {
        base[(size_t)(2 * rc) * Kp + k] = ar;
        base[(size_t)(2 * rc) * Kp + Kcp + k] = ai;
        base[(size_t)(2 * rc + 1) * Kp + k] = (int8_t)(-ai);
        base[(size_t)(2 * rc + 1) * Kp + Kcp + k] = ar;
      }
    }
  }
}

// 2^e as a double from its exponent bits: exact for -1022 <= e <= 1023,
// 0 below that range and infinity above it (no branch)
__device__ __forceinline__ double pow2i(int e) {
  const double v = __longlong_as_double((long long)(min(max(e, -1023), 1024) + 1023) << 52);
  return e < -1022 ? 0.0 : v;
}

// Level sum of one accumulator column, sum_d c_d 2^(-7d), in one of three
// exact forms (LS, chosen on the host from the bound on |c_d|):
//   LS = 2: levels paired in int32 (c_d 128 + c_(d+1)), the pairs combined
//           in int64 into V = sum_d c_d 2^(7(S-1-d)), |V| < 2^51, and V
//           converted by one add (returns V: the caller's scale carries
//           2^(-7(S-1)));
//   LS = 1: pairs in int32, each pair converted and accumulated in FP64;
//   LS = 0: every level converted and accumulated in FP64.
template <int S, int LS>
__device__ __forceinline__ double level_sum(const uint32_t (&r)[S]) {
  if (LS == 2) {
    long long V = 0;
#pragma unroll
    for (int d = 0; d < S; d += 2) {
      if (d + 1 < S)
        V = V * 16384 + (long long)((int)r[d] * 128 + (int)r[d + 1]);
      else
        V = V * 128 + (long long)(int)r[d];
    }
    // 1.5 2^52 + V has V in its low mantissa bits for |V| < 2^51
    return __longlong_as_double(V + 0x4338000000000000LL) - 6755399441055744.0;
  }
  double v = 0.0, w = 1.0;
  if (LS == 1) {
#pragma unroll
    for (int d = 0; d < S; d += 2) {
      if (d + 1 < S) {
        const int pr = (int)r[d] * 128 + (int)r[d + 1];
        v = fma(i2d_exact((uint32_t)pr), w * 0.0078125, v);
      } else {
        v = fma(i2d_exact(r[d]), w, v);
      }
      w *= 6.103515625e-05;  // 2^-14
    }
  } else {
#pragma unroll
    for (int d = 0; d < S; d++) {
      v = fma(i2d_exact(r[d]), w, v);
      w *= 0.0078125;
    }
  }
  return v;
}

// S levels x 4 columns of this warp's TMEM lanes into registers (async until
// tmem_wait4)
template <int S>
__device__ __forceinline__ void tmem_ld4(uint32_t (&r)[S][4], uint32_t addr, int N) {
#pragma unroll
  for (int d = 0; d < S; d++)
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[d][0]), "=r"(r[d][1]), "=r"(r[d][2]), "=r"(r[d][3])
                 : "r"(addr + (uint32_t)(d * N)));
}
// wait for this thread's TMEM loads; the registers pass through an empty asm
// so that no use of them is scheduled before the wait
template <int S>
__device__ __forceinline__ void tmem_wait4(uint32_t (&r)[S][4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int d = 0; d < S; d++) asm volatile("" : "+r"(r[d][0]), "+r"(r[d][1]), "+r"(r[d][2]), "+r"(r[d][3]));
}
// bounded wait that also gives up once another role has raised the abort flag
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, const int* flag) {
  long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (*(volatile const int*)flag || clock64() - t0 > (1LL << 31)) return false;
  return true;
}

// Persistent: CTA b takes tiles b, b + gridDim.x, ... of the list.  The
// stage ring and the two accumulator buffers run on counters that continue
// across tiles, so the loads and MMAs of a tile's first l overlap the
// previous tile's last epilogue, interstitial gather and HS writes.
template <int S, int LS, int KB>
__global__ void __launch_bounds__(Cfg<S, KB>::THREADS, 1)
    k_sph_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, DevProb P,
             const int2* __restrict__ tiles, int ntile, int nkb, int klast, int npA, int npB,
             const int* __restrict__ exA, const int* __restrict__ exB, const double2* __restrict__ tab, TabDesc T,
             double2* __restrict__ hs, int ld, double2* __restrict__ hsdiag, int* __restrict__ status,
             int never_wait) {
  using C = Cfg<S, KB>;
  constexpr int N = C::N, IT = C::IT, STAGES = C::STAGES, HALF = C::IPT, EPI = C::EPI;
  constexpr int MMA_WARP = 4 * C::EG, TMA_WARP = 4 * C::EG + 1;
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t full[STAGES], empty[STAGES], tfull[2], tempty[2], accbar, ebar, never;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int L = P.ltop, nv = P.nv;
  const int nit = L * nkb;  // pipeline iterations per tile

  if (warp == MMA_WARP) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4 * C::EG);  // one arrival per epilogue warp
    }
    mbar_init(&accbar, 1);
    mbar_init(&ebar, EPI);  // the epilogue threads' barrier (bounded waits)
    mbar_init(&never, 1);   // nothing arrives here (the never_wait test hook)
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == TMA_WARP) {
    // ---- TMA producer: a full ring ahead of the MMAs ----
    if (lane == 0) {
      long g = 0;  // iterations issued over all tiles
      bool ok = true;
      for (int t = blockIdx.x; t < ntile && ok; t += gridDim.x) {
        const int2 tt = tiles[t];
        const int j0 = tt.x * 128, i0 = tt.y * IT;
        for (int it = 0; it < nit; it++, g++) {
          const int st = (int)(g % STAGES);
          if (g >= STAGES) {  // the MMAs of g - STAGES have released the stage
            const uint32_t par = (uint32_t)((g - STAGES) / STAGES) & 1;
            long long t0 = clock64();
            while (!mbar_try_wait(&empty[st], par)) {
              if (*(volatile int*)&abort_flag || clock64() - t0 > (1LL << 31)) {
                ok = false;
                break;
              }
            }
            if (!ok) break;
          }
          const int l = it / nkb, kb = it % nkb;
          uint8_t* a = smem + st * C::STAGE;
          uint8_t* b = a + C::A_BYTES;
          mbar_expect_tx(&full[st], C::STAGE);
          tma_load_3d(a, &tmA, &full[st], kb * KB, l * npA + j0, 0);
          tma_load_3d(b, &tmB, &full[st], kb * KB, l * 4 * npB + 4 * i0, 0);
        }
      }
      if (!ok) atomicOr(status, L1G_STATUS_TIMEOUT);
      // the copies in flight land before the CTA's shared memory is released
      // (the MMA issuer may stop early; consumed stages return at once)
      for (long q = g - STAGES > 0 ? g - STAGES : 0; q < g; q++)
        mbar_wait(&full[q % STAGES], (uint32_t)(q / STAGES) & 1);
    }
    __syncwarp();
  } else if (warp == MMA_WARP) {
    // ---- MMA issuer ----
    if (lane == 0) {
      long g = 0;   // pipeline iterations over all tiles
      long gl = 0;  // accumulations (tile, l) over all tiles
      bool ok = true;
      if (never_wait) {
        // test hook: the consumer waits on a barrier that nothing arrives
        // at, with a short bound (about half a millisecond), and takes the
        // timeout path below (the other roles' waits keep their full bound)
        const long long t0 = clock64();
        while (!mbar_try_wait(&never, 0))
          if (clock64() - t0 > (1LL << 20)) {
            ok = false;
            break;
          }
      }
      for (int t = blockIdx.x; t < ntile && ok; t += gridDim.x) {
        for (int it = 0; it < nit; it++, g++) {
          const int st = (int)(g % STAGES), kb = it % nkb, buf = (int)(gl & 1);
          if (kb == 0 && gl >= 2 && !wait_or_abort(&tempty[buf], (uint32_t)((gl - 2) >> 1) & 1, &abort_flag)) {
            ok = false;
            break;
          }
          if (!wait_or_abort(&full[st], (uint32_t)(g / STAGES) & 1, &abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a0 = smem_u32(smem + st * C::STAGE);
          const uint32_t b0 = a0 + C::A_BYTES;
          // The S slices of B lie one after another in shared memory (one
          // (S N)-row K-major tile) and the level accumulators N columns
          // apart in TMEM, so A slice p times B slices 0..S-1-p is ONE MMA
          // of width (S-p) N whose columns land on levels p..S-1.  The last
          // block holds klast valid 32-byte steps (TMA zero-fills the rest;
          // their MMAs are skipped).
          const int nh = (kb == nkb - 1) ? klast : C::KSTEPS;
#pragma unroll
          for (int p = 0; p < S; p++)
#pragma unroll
            for (int h = 0; h < C::KSTEPS; h++) {
              if (h >= nh) continue;
              const uint64_t ad = desc_kblock<KB>(a0 + p * 128 * KB + h * 32);
              const uint64_t bd = desc_kblock<KB>(b0 + h * 32);
              const uint32_t acc = (kb > 0 || h > 0 || p > 0) ? 1u : 0u;
              const uint32_t d = tmem + (uint32_t)(buf * S * N + p * N);
              asm volatile(
                  "{\n\t.reg .pred pa;\n\t"
                  "setp.ne.b32 pa, %4, 0;\n\t"
                  "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, pa;\n\t}" ::"r"(d),
                  "l"(ad), "l"(bd), "r"(idesc_i8(128, (S - p) * N)), "r"(acc)
                  : "memory");
            }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_u32(&empty[st]))
                       : "memory");
          if (kb == nkb - 1) {
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&tfull[buf]))
                         : "memory");
            gl++;
          }
        }
      }
      if (!ok) {
        atomicOr(status, L1G_STATUS_TIMEOUT);
        *(volatile int*)&abort_flag = 1;
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&accbar))
                   : "memory");
    }
    __syncwarp();
  } else {
    // ---- epilogue warps ----
    int16_t* sA = (int16_t*)(smem + STAGES * C::STAGE);  // [l][128]: eA - 12
    int16_t* sB = sA + SPH_LMAX * 128;                    // [l][IT][2]: eB
    const int g4 = warp & 3, hh = warp >> 2;
    const uint32_t trow = tmem + ((uint32_t)(32 * g4) << 16);
    long gl = 0;  // accumulations consumed over all tiles
    bool ok = true;
    uint32_t ephase = 0;
    // barrier of the epilogue threads on an mbarrier, every wait bounded
    // (a warp that gave up leaves the others to time out, not to hang);
    // warp-uniform outcome
    auto epi_sync = [&]() -> bool {
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&ebar)) : "memory");
      const bool r = __all_sync(0xffffffffu, wait_or_abort(&ebar, ephase & 1, &abort_flag));
      ephase++;
      return r;
    };
    // this thread's share of a tile's scale tables, fetched into registers
    // one tile ahead (behind the previous tile's interstitial part)
    constexpr int QA = (SPH_LMAX * 128 + EPI - 1) / EPI, QB = (SPH_LMAX * 2 * IT + EPI - 1) / EPI;
    int16_t pa[QA], pb[QB];
    auto fetch = [&](int t) {  // volatile loads: issued here, ahead of their use
      const int j0 = split::ld_early(&tiles[t].x) * 128, i0 = split::ld_early(&tiles[t].y) * IT;
#pragma unroll
      for (int k = 0; k < QA; k++) {
        const int q = tid + k * EPI, l = q >> 7, J = j0 + (q & 127);
        pa[k] = (int16_t)((q < L * 128 && J < nv) ? split::ld_early(&exA[(size_t)l * npA + J]) - 12
                                                   : -2000);  // -2000: a zero scale
      }
#pragma unroll
      for (int k = 0; k < QB; k++) {
        const int q = tid + k * EPI, l = q / (2 * IT), r = q % (2 * IT), I = i0 + (r >> 1);
        pb[k] = (int16_t)((q < L * 2 * IT && I < nv) ? split::ld_early(&exB[(size_t)l * 2 * npB + 2 * I + (r & 1)])
                                                      : -2000);
      }
    };
    if (blockIdx.x < ntile) fetch(blockIdx.x);
    for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
      const int2 tt = tiles[t];
      const int j0 = tt.x * 128, i0 = tt.y * IT;
      // scale tables of this tile for every l, written once the previous
      // tile's readers are past the first barrier
      if (!epi_sync()) {
        ok = false;
        break;
      }
#pragma unroll
      for (int k = 0; k < QA; k++)
        if (tid + k * EPI < L * 128) sA[tid + k * EPI] = pa[k];
#pragma unroll
      for (int k = 0; k < QB; k++)
        if (tid + k * EPI < L * 2 * IT) sB[tid + k * EPI] = pb[k];
      if (!epi_sync()) {
        ok = false;
        break;
      }
      const int J = j0 + 32 * g4 + lane;
      const bool jin = J < nv;
      const double xj = jin ? P.xk[J] : 0.0, yj = jin ? P.yk[J] : 0.0, zj = jin ? P.zk[J] : 0.0;
      const double rj = jin ? P.rk[J] : 0.0;
      double x[HALF], pm1[HALF], pm2[HALF];
      double2 aS[HALF], aH[HALF];
#pragma unroll
      for (int u = 0; u < HALF; u++) {
        const int I = i0 + hh * HALF + u;
        double xx = 0.0;
        if (jin && I < nv) {
          xx = P.xk[I] * xj + P.yk[I] * yj + P.zk[I] * zj;
          const double den = P.rk[I] * rj;
          if (den > 1.0e-8) xx = xx / den;
        }
        x[u] = xx;
        pm1[u] = xx;   // P_1
        pm2[u] = 1.0;  // P_0
        aS[u] = aH[u] = make_double2(0.0, 0.0);
      }
      for (int l = 0; l < L; l++, gl++) {
        const int buf = (int)(gl & 1);
        // warp-uniform outcome: the TMEM loads below are .sync.aligned
        if (!__all_sync(0xffffffffu, wait_or_abort(&tfull[buf], (uint32_t)(gl >> 1) & 1, &abort_flag))) {
          ok = false;
          if (lane == 0) atomicOr(status, L1G_STATUS_TIMEOUT);
          break;
        }
        if (__any_sync(0xffffffffu, *(volatile int*)&abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int ea = sA[l * 128 + 32 * g4 + lane] + (LS == 2 ? -7 * (S - 1) : 0);
        const double cl = (l >= 2) ? (double)(l - 1) / (double)l : 0.0, fl = (double)(2 * l + 1);
        // 4 real columns per I: S re, S im, H re, H im; this thread's HALF I
        // start at column 4 HALF hh; one I (4 columns x S levels) per load
        const uint32_t tcol = trow + (uint32_t)(buf * S * N + 4 * HALF * hh);
#pragma unroll
        for (int u = 0; u < HALF; u++) {
          uint32_t r[S][4];
          tmem_ld4<S>(r, tcol + 4 * u, N);
          tmem_wait4<S>(r);
          if (u == HALF - 1) {
            // all columns of this buffer read: hand it back to the MMA issuer
            tc_fence_before();
            __syncwarp();
            if (lane == 0)
              asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[buf])) : "memory");
          }
          double v[4];
#pragma unroll
          for (int m = 0; m < 4; m++) {
            uint32_t rr[S];
#pragma unroll
            for (int d = 0; d < S; d++) rr[d] = r[d][m];
            v[m] = level_sum<S, LS>(rr);
          }
          // Legendre weight (hamilt.F:250-281 recursion, UTOP branch)
          double pl;
          if (l == 0)
            pl = 1.0;
          else if (l == 1)
            pl = x[u];
          else {
            if (fabs(x[u]) < 0.9999999) {
              const double pplx = x[u] * pm1[u];
              pl = pplx + cl * (pplx - pm2[u]);
            } else {
              pl = x[u] * pm1[u];
            }
            pm2[u] = pm1[u];
            pm1[u] = pl;
          }
          const double wl = fl * pl;
          const int16_t* sb = sB + (l * IT + hh * HALF + u) * 2;
          const double sS = wl * pow2i(ea + sb[0]), sH = wl * pow2i(ea + sb[1]);
          aS[u].x = fma(v[0], sS, aS[u].x);
          aS[u].y = fma(v[1], sS, aS[u].y);
          aH[u].x = fma(v[2], sH, aH[u].x);
          aH[u].y = fma(v[3], sH, aH[u].y);
        }
      }
      if (!ok) {
        *(volatile int*)&abort_flag = 1;
        break;
      }
      if (t + (int)gridDim.x < ntile) fetch(t + gridDim.x);
      // interstitial + write (hamilt.F:289-345, 459-466, calkpt.F:164): every
      // load of the HALF pairs first (the HS stores might alias them), then
      // the stores; I past NV reads a valid row and stores nothing
      if (jin) {
        const int nx = 2 * T.d1 + 1, ny = 2 * T.d2 + 1;
        const int k1 = P.kzz[3 * J], k2 = P.kzz[3 * J + 1], k3 = P.kzz[3 * J + 2];
        double2 th[HALF], wp[HALF];
        double x2[HALF];
#pragma unroll
        for (int u = 0; u < HALF; u++) {
          const int I = min(i0 + hh * HALF + u, nv - 1);
          x2[u] = xj * P.xk[I] + yj * P.yk[I] + zj * P.zk[I];
          const int d1 = k1 - P.kzz[3 * I] + T.d1, d2 = k2 - P.kzz[3 * I + 1] + T.d2,
                    d3 = k3 - P.kzz[3 * I + 2] + T.d3;
          const size_t ci = ((size_t)d3 * ny + d2) * nx + d1;
          th[u] = tab[2 * ci];
          wp[u] = tab[2 * ci + 1];
        }
        bool bad = false;  // a written element is not finite
#pragma unroll
        for (int u = 0; u < HALF; u++) {
          const int I = i0 + hh * HALF + u;
          if (I >= nv || J > I) continue;
          const double2 s = cadd(th[u], aS[u]);
          const double2 h = cadd(cadd(cscale(th[u], x2[u]), wp[u]), aH[u]);
          if (J == I) {
            hs[(size_t)I * ld + I] = h;
            hsdiag[I] = s;
          } else {
            hs[(size_t)I * ld + J] = s;  // S upper: HS(J,I)
            hs[(size_t)J * ld + I] = h;  // H lower: HS(I,J)
          }
          bad |= l1g_nonfinite(s) | l1g_nonfinite(h);
        }
        if (bad) atomicOr(status, L1G_STATUS_NONFINITE);
      }
    }
    if (!ok) {
      *(volatile int*)&abort_flag = 1;
      if (lane == 0) atomicOr(status, L1G_STATUS_TIMEOUT);
    }
  }
  // every MMA issued has completed before TMEM is freed
  if (warp == MMA_WARP) mbar_wait(&accbar, 0);
  tc_fence_before();
  __syncthreads();
  if (warp == MMA_WARP) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

}  // namespace sphtc

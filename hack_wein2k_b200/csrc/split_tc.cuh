// split_tc.cuh -- split-precision HNS contraction on the 5th-generation
// tensor cores (tcgen05, kind::i8), sm_100a.
//
// The HNS update of the lower triangle (hns.F:449-467, zher2m.f:69-80),
//   HS(i,j) += sum_k L(i,k) R(j,k),  i >= j,   K = 2*NDF*(lnsmax+1)^2 complex,
// is computed as an Ozaki-style sum of exact integer products:
//   * every row of L (and of R) gets a power-of-two scale 2^e, e = ilogb(max)+1,
//     so the scaled row lies in (-1, 1);
//   * the scaled row is cut into S int8 slices, l = sum_p a_p 2^(-6-7(p-1)),
//     |a_p| <= 64 (first slice 6 bits + sign, then 7 bits each); the cut is
//     exact in FP64 (power-of-two scalings and Sterbenz subtractions);
//   * slice products a_p b_q with p+q-2 = d < S are accumulated EXACTLY in one
//     int32 TMEM accumulator per level d (|sum| <= 64*64*2K < 2^31);
//   * the epilogue combines the levels in FP64, sum_d c_d 2^(-7d), scales by
//     2^(e_i + f_j - 12) and adds into HS.
// The dropped products (p+q-2 >= S) bound the error by ~(S+1) 2^(-7S) of
// max|L_i| max|R_j| K per element: S=7 is FP64-class (2^-49).
//
// Complex arithmetic as one real GEMM with K' = 2K (a Kcp-padded real half
// and imaginary half per row): A row i = [Re L_i | Im L_i],
// B rows 2j = [Re R_j | -Im R_j] (-> Re C), 2j+1 = [Im R_j | Re R_j] (-> Im C),
// so the accumulator columns alternate Re/Im of consecutive j.
//
// Kernel shape: one CTA per (128-row, N/2-column) tile of the triangle,
// M=128, N = 512/S rounded down to 16 (all S levels fit the 512 TMEM
// columns), 64-byte K blocks with 64B-swizzled TMA tiles of all S slices
// in one 3-D box, 2-3 pipeline stages.  Thread 0 issues TMA and MMA; all
// four warps run the epilogue.  Every mbarrier wait is bounded (about one
// second of clock64); a timeout sets a status bit, skips the writes,
// drains the copies in flight (bounded) and frees TMEM before returning.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#define L1G_MAX_SLICES 8
#define L1G_STATUS_TIMEOUT 8

namespace split {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait (~1 s of SM clock); false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > (1LL << 31)) return false;
  return true;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}
// int32 -> double, exact: the bits (0x43300000, x + 2^31) are the double
// 2^52 + 2^31 + x, so one add recovers x (an FP64 add issues at the full
// FP64 rate, the integer-to-double conversion at a fraction of it)
__device__ __forceinline__ double i2d_exact(uint32_t x) {
  return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 4503601774854144.0;
}

// x 2^(6 - e): the first int8 digit's scale for a row of exponent e (one
// multiply by the exact power of two in the normal range, ldexp outside it)
__device__ __forceinline__ double digit_scale(double x, int e) {
  const int k = 6 - e;
  return (k >= -1022 && k <= 1023) ? x * __longlong_as_double((long long)(k + 1023) << 52) : ldexp(x, k);
}
// a global load issued where it stands (volatile: not sunk to its use)
__device__ __forceinline__ int ld_early(const int* p) {
  int v;
  asm volatile("ld.global.nc.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
// 2^e exactly: exponent bits in the normal range, ldexp outside it
__device__ __forceinline__ double pow2_exact(int e) {
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}
// One int8 digit of the slicing: t rounded to the nearest integer (ties to
// even, as rint) by adding 1.5 2^52, whose low mantissa bits then hold the
// integer; t becomes the exact remainder scaled by 2^7 for the next digit.
__device__ __forceinline__ int digit7(double& t) {
  const double sh = t + 6755399441055744.0;
  const int d = __double2loint(sh);
  t = (t - (sh - 6755399441055744.0)) * 128.0;
  return d;
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// K-major operand tile, 64-byte swizzle: rows of 64 B, 8-row groups 512 B apart
__device__ __forceinline__ uint64_t desc_sw64(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;     // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;              // descriptor version (sm100)
  d |= (uint64_t)4 << 61;              // SWIZZLE_64B
  return d;
}
// K-major operand tile, 128-byte swizzle: rows of 128 B, 8-row groups 1024 B
// apart (the tile base 1024-byte aligned; a K step inside the row advances
// the start address by 32 B, the swizzle acting on the absolute address)
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;  // SWIZZLE_128B
  return d;
}
// the descriptor of a K block of KB bytes per row (64 or 128)
template <int KB>
__device__ __forceinline__ uint64_t desc_kblock(uint32_t saddr) {
  return KB == 128 ? desc_sw128(saddr) : desc_sw64(saddr);
}
// instruction descriptor: D s32, A s8, B s8, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

template <int S>
struct Cfg {
  static constexpr int N = ((512 / S) / 16) * 16 > 128 ? 128 : ((512 / S) / 16) * 16;  // real columns
  static constexpr int JT = N / 2;                                                     // complex columns
  static constexpr int A_BYTES = S * 128 * 64;
  static constexpr int B_BYTES = S * N * 64;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int STAGES = (3 * STAGE + 1024 <= 220 * 1024) ? 3 : 2;
  static constexpr int SMEM = STAGES * STAGE + 1024;
};

// FP64 -> int8 slices.  X: [Kc][npad] complex (k-major planes, the HNS
// operand layout).  Out: [S][rows][Kp] int8 with Kp = 2*Kcp; for the left
// operand (isB = 0) rows = np, row i = [Re | Im]; for the right operand
// rows = 2*np, row 2j = [Re | -Im], row 2j+1 = [Im | Re].  ex[row of X] =
// the power-of-two exponent of the row's largest component.
// Row exponents for the slicing, in parallel over rows and K chunks:
// ex[row] = max over k of ilogb(max(|Re|, |Im|)) + 1 (ex starts at a very
// negative value, so all-zero rows keep a zero scale).  One thread per row,
// 64 k per block.
__global__ void __launch_bounds__(128) k_rowexp(const double2* __restrict__ X, int Kc, int npad,
                                                int* __restrict__ ex) {
  const int row = blockIdx.x * 128 + threadIdx.x;
  const int k0 = blockIdx.y * 64;
  if (row >= npad) return;
  double m = 0.0;
  for (int k = k0; k < min(Kc, k0 + 64); k++) {
    const double2 v = X[(size_t)k * npad + row];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  if (m > 0.0) atomicMax(&ex[row], ilogb(m) + 1);
}

// FP64 -> int8 slices with the exponents of k_rowexp, one block per 32 rows
// x 64 k: every output byte of [0, np) x [0, 2 Kcp) is written (zeros for
// the padding rows and columns), so the operand buffers need no clearing.
template <int S>
// A non-finite operand value sets L1G_STATUS_NONFINITE in status (int8
// slices cannot carry it into the products).
__global__ void __launch_bounds__(256, 2) k_slice_rows(const double2* __restrict__ X, int Kc, int Kcp, int npad,
                                                       int np_out, int isB, int cj, const int* __restrict__ ex,
                                                       int8_t* __restrict__ out, int* __restrict__ status) {
  __shared__ double2 tile[64][33];
  __shared__ int rexp[32];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 64;
  const int tid = threadIdx.x;
  const int Kp = 2 * Kcp;
  const size_t rows = isB ? 2 * (size_t)np_out : (size_t)np_out;
  bool bad = false;
  for (int q = tid; q < 64 * 32; q += 256) {
    const int kk = q >> 5, r = q & 31;
    const int k = k0 + kk, row = r0 + r;
    const double2 v = (k < Kc && row < npad) ? X[(size_t)k * npad + row] : make_double2(0.0, 0.0);
    tile[kk][r] = v;
    bad |= l1g_nonfinite(v);
  }
  if (bad) atomicOr(status, L1G_STATUS_NONFINITE);
  if (tid < 32) rexp[tid] = (r0 + tid < np_out) ? ex[r0 + tid] : 0;
  __syncthreads();
  // one element per thread and pass, lanes along k: conflict-free tile
  // reads (stride 33) and byte stores coalesced along each row
  for (int idx = tid; idx < 32 * 64; idx += 256) {
    const int rr = idx >> 6, kk = idx & 63;
    const int row = r0 + rr, col = k0 + kk;
    if (row >= np_out || col >= Kcp) continue;
    const int e = rexp[rr];
    const double2 v = tile[kk][rr];
    double tr = digit_scale(v.x, e), ti = digit_scale(cj ? -v.y : v.y, e);  // cj: slice conj(X)
#pragma unroll
    for (int p = 0; p < S; p++) {
      const int8_t ar = (int8_t)digit7(tr), ai = (int8_t)digit7(ti);
      int8_t* base = out + (size_t)p * rows * Kp;
      if (!isB) {
        base[(size_t)row * Kp + col] = ar;
        base[(size_t)row * Kp + Kcp + col] = ai;
      } else {
        base[(2 * (size_t)row) * Kp + col] = ar;
        base[(2 * (size_t)row) * Kp + Kcp + col] = (int8_t)(-ai);
        base[(2 * (size_t)row + 1) * Kp + col] = ai;
        base[(2 * (size_t)row + 1) * Kp + Kcp + col] = ar;
      }
    }
  }
}

// 256 threads: warp 0 lane 0 issues the MMAs, warp 1 lane 0 the TMA loads;
// afterwards all 8 warps are the epilogue (warp w: TMEM lanes 32 (w%4).. =
// rows, column half w/4).  The HS values the epilogue adds to are loaded
// into registers when the CTA starts, so their latency hides behind the
// MMA main loop (the tiles of one launch own disjoint HS elements, written
// before the launch).
#define SPLIT_THREADS 256
template <int S>
__global__ void __launch_bounds__(SPLIT_THREADS, 1)
    k_split_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const int2* __restrict__ tiles, int nkb, int n, int nr, int mode, const int* __restrict__ exA,
                 const int* __restrict__ exB, double2* __restrict__ hs, int ld, int* __restrict__ status) {
  // mode bit 0: rectangular product (all i < n, j < nr) instead of the
  // lower triangle j <= i; bit 1: overwrite the output instead of adding
  // to it (no prefetch of the old values)
  const int rect = mode & 1, ovw = mode & 2;
  using C = Cfg<S>;
  constexpr int N = C::N, STAGES = C::STAGES;
  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t full[STAGES], empty[STAGES], accbar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int2 t = tiles[blockIdx.x];
  const int i0 = t.x * 128, j0 = t.y * C::JT;
  // this thread's epilogue share: row i, complex columns j0 + 8 c + q for
  // the NC chunks c of its column half; prefetch the old HS values
  constexpr int NCT = N / 16, NC = (NCT + 1) / 2;  // 16-column (8 complex) chunks: all, per half
  const int i = i0 + (warp & 3) * 32 + lane, cbase = (warp >> 2) * NC;
  // volatile loads: issued here, not sunk by the compiler to their use in
  // the epilogue, so the main loop hides their latency
  double2 old[NC][8];
#pragma unroll
  for (int c = 0; c < NC; c++)
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int j = j0 + (cbase + c) * 8 + q;
      old[c][q] = make_double2(0.0, 0.0);
      if (!ovw && cbase + c < NCT && i < n && j < nr && (rect || j <= i))
        asm volatile("ld.global.v2.f64 {%0, %1}, [%2];"
                     : "=d"(old[c][q].x), "=d"(old[c][q].y)
                     : "l"(hs + (size_t)j * ld + i));
    }

  if (warp == 0) {
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
    mbar_init(&accbar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (tid == 32) {
    // TMA producer (warp 1 lane 0): a full ring ahead of the MMAs
    int issued = 0;  // k blocks whose TMA was issued
    bool ok = true;
    for (int kb = 0; kb < nkb; kb++) {
      const int st = kb % STAGES;
      if (kb >= STAGES) {  // the MMAs of kb - STAGES have released the stage
        const uint32_t par = ((kb - STAGES) / STAGES) & 1;
        long long t0 = clock64();
        while (!mbar_try_wait(&empty[st], par)) {
          if (*(volatile int*)&abort_flag || clock64() - t0 > (1LL << 31)) {
            ok = false;
            break;
          }
        }
        if (!ok) break;
      }
      uint8_t* a = smem + st * C::STAGE;
      uint8_t* b = a + C::A_BYTES;
      mbar_expect_tx(&full[st], C::STAGE);
      tma_load_3d(a, &tmA, &full[st], kb * 64, i0, 0);
      tma_load_3d(b, &tmB, &full[st], kb * 64, 2 * j0, 0);
      issued = kb + 1;
    }
    if (!ok) atomicOr(status, L1G_STATUS_TIMEOUT);
    // the copies in flight land before the CTA may exit (the MMA issuer may
    // stop early; consumed stages return at once); every wait is bounded
    for (int kb = issued - STAGES > 0 ? issued - STAGES : 0; kb < issued; kb++)
      mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
  } else if (tid == 0) {
    // MMA issuer (warp 0 lane 0)
    bool ok = true;
    for (int kb = 0; kb < nkb; kb++) {
      const int st = kb % STAGES;
      if (!mbar_wait(&full[st], (kb / STAGES) & 1)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t a0 = smem_u32(smem + st * C::STAGE);
      const uint32_t b0 = a0 + C::A_BYTES;
      // B's S slices are one (S N)-row K-major tile and the level
      // accumulators lie N columns apart, so A slice p times B slices
      // q0..q0+cnt-1 is one MMA of width cnt N (at most 256 columns)
      // landing on levels p+q0..p+q0+cnt-1.
      constexpr int QC = (256 / N) < S ? (256 / N) : S;  // B slices per MMA
#pragma unroll
      for (int p = 0; p < S; p++)
#pragma unroll
        for (int q0 = 0; q0 < S - p; q0 += QC)
#pragma unroll
          for (int h = 0; h < 2; h++) {
            const int cnt = (S - p - q0) < QC ? (S - p - q0) : QC;
            const uint64_t ad = desc_sw64(a0 + p * 128 * 64 + h * 32);
            const uint64_t bd = desc_sw64(b0 + q0 * N * 64 + h * 32);
            // the first MMA into each level initialises it: level p+q0 first
            // appears with p = 0 (q0 = its index) at kb = 0, h = 0
            const uint32_t acc = (kb > 0 || h > 0 || p > 0) ? 1u : 0u;
            const uint32_t d = tmem + (uint32_t)((p + q0) * N);
            asm volatile(
                "{\n\t.reg .pred pa;\n\t"
                "setp.ne.b32 pa, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, pa;\n\t}" ::"r"(d),
                "l"(ad), "l"(bd), "r"(idesc_i8(128, cnt * N)), "r"(acc)
                : "memory");
          }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&empty[st]))
                   : "memory");
    }
    if (!ok) {
      atomicOr(status, L1G_STATUS_TIMEOUT);
      *(volatile int*)&abort_flag = 1;
    }
    // arrives once every MMA issued so far has completed, so TMEM is
    // quiescent when the epilogue (or the abort path) proceeds
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(&accbar))
                 : "memory");
  }
  __syncwarp();
  // epilogue: warp w owns TMEM lanes 32(w%4).. = rows i0+32(w%4).., column half w/4
  const bool acc_ok = __all_sync(0xffffffffu, mbar_wait(&accbar, 0));  // warp-uniform
  tc_fence_after();
  if (!acc_ok && lane == 0) atomicOr(status, L1G_STATUS_TIMEOUT);
  __syncthreads();
  bool bad = false;  // a written element is not finite
  if (acc_ok && !abort_flag) {
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const double sa = (i < n) ? pow2_exact(exA[i] - 12) : 0.0;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      const int cc = cbase + c;
      if (cc >= NCT) break;  // warp-uniform
      double v[16];
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = 0.0;
      // all S levels of these 16 columns in flight at once, one wait
      uint32_t r[S][16];
#pragma unroll
      for (int d = 0; d < S; d++)
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
            "[%16];"
            : "=r"(r[d][0]), "=r"(r[d][1]), "=r"(r[d][2]), "=r"(r[d][3]), "=r"(r[d][4]), "=r"(r[d][5]),
              "=r"(r[d][6]), "=r"(r[d][7]), "=r"(r[d][8]), "=r"(r[d][9]), "=r"(r[d][10]), "=r"(r[d][11]),
              "=r"(r[d][12]), "=r"(r[d][13]), "=r"(r[d][14]), "=r"(r[d][15])
            : "r"(trow + (uint32_t)(d * N + cc * 16)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      double w = 1.0;
#pragma unroll
      for (int d = 0; d < S; d++) {
#pragma unroll
        for (int q = 0; q < 16; q++) v[q] = fma(i2d_exact(r[d][q]), w, v[q]);
        w *= 0.0078125;  // 2^-7
      }
      if (i < n) {
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int j = j0 + cc * 8 + q;
          if (j < nr && (rect || j <= i)) {
            const double sc = sa * pow2_exact(exB[j]);
            double2 o = old[c][q];
            o.x = fma(v[2 * q], sc, o.x);
            o.y = fma(v[2 * q + 1], sc, o.y);
            hs[(size_t)j * ld + i] = o;
            bad |= l1g_nonfinite(o);
          }
        }
      }
    }
  }
  if (bad) atomicOr(status, L1G_STATUS_NONFINITE);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

}  // namespace split

// ---------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 l1g_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 3-D map over [S][rows][kp] int8 slice planes; a box is all S slices of
// box_rows rows and `inner` bytes of K (128, 64 or 32: the swizzle of
// that width)
static int l1g_tmap_3d(CUtensorMap* m, const void* base, uint64_t kp, uint64_t rows, uint64_t S, uint32_t box_rows,
                       uint32_t inner = 64) {
  auto enc = l1g_encode_fn();
  if (!enc) return LAPW1GPU_ERR_CUDA;
  cuuint64_t dims[3] = {kp, rows, S};
  cuuint64_t strides[2] = {kp, kp * rows};
  cuuint32_t box[3] = {inner, box_rows, (cuuint32_t)S};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   inner == 128  ? CU_TENSOR_MAP_SWIZZLE_128B
                   : inner == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                                 : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) l1g_note_error("cuTensorMapEncodeTiled", (long)r, __FILE__, __LINE__);
  return r == CUDA_SUCCESS ? LAPW1GPU_OK : LAPW1GPU_ERR_CUDA;
}

template <int S>
static int split_gemm_launch(lapw1gpu_context* c, lapw1gpu_kpoint* k, int set, int n, int npad, int Kc,
                             const double2* Lop, const double2* Rop, double2* hs, int ld, cudaStream_t s,
                             int* nlaunch, HnsPipe* hp, const cudaEvent_t* ev, int cjL, int phase, int ovw) {
  // phase 1: row exponents and slices only; 2: the products only (the
  // slices of this set are ready); 3: both.  ovw: write the products
  // instead of adding them to hs
  using Cf = split::Cfg<S>;
  const int Kcp = (Kc + 63) / 64 * 64;
  const int Kp = 2 * Kcp;
  const int np = (npad + 127) / 128 * 128;
  int8_t* A = (int8_t*)c->sbuf(set, "splitA", (size_t)S * np * Kp);
  int8_t* B = (int8_t*)c->sbuf(set, "splitB", (size_t)S * 2 * np * Kp);
  int* exA = (int*)c->sbuf(set, "splitExA", sizeof(int) * np);
  int* exB = (int*)c->sbuf(set, "splitExB", sizeof(int) * np);
  if (!A || !B || !exA || !exB) return LAPW1GPU_ERR_NOMEM;
  if (phase & 1) {
    // row exponents (0x80808080 bytes: a very negative start for atomicMax),
    // then the slices of every row and column of the padded operands
    if (cudaMemsetAsync(exA, 0x80, sizeof(int) * np, s) != cudaSuccess ||
        cudaMemsetAsync(exB, 0x80, sizeof(int) * np, s) != cudaSuccess)
      return LAPW1GPU_ERR_CUDA;
    const dim3 ge((npad + 127) / 128, (Kc + 63) / 64), gs(np / 32, Kcp / 64);
    split::k_rowexp<<<ge, 128, 0, s>>>(Lop, Kc, npad, exA);
    split::k_rowexp<<<ge, 128, 0, s>>>(Rop, Kc, npad, exB);
    split::k_slice_rows<S><<<gs, 256, 0, s>>>(Lop, Kc, Kcp, npad, np, 0, cjL, exA, A, c->d_status);
    split::k_slice_rows<S><<<gs, 256, 0, s>>>(Rop, Kc, Kcp, npad, np, 1, 0, exB, B, c->d_status);
    *nlaunch += 4;
  }
  if (!(phase & 2)) return l1g_launch_status(__FILE__, __LINE__);
  CUtensorMap ta, tb;
  if (l1g_tmap_3d(&ta, A, Kp, np, S, 128) || l1g_tmap_3d(&tb, B, Kp, 2 * (uint64_t)np, S, Cf::N))
    return LAPW1GPU_ERR_CUDA;
  // grouped order: W row tiles of L stay in L2 while every column tile of R
  // that meets them streams past once, so R is read from DRAM once per
  // group instead of once per row tile (W is a tunable, 16 by default).
  // With hp, one launch per column group (hp->groups), each followed by its
  // event unless its columns reach the LO block (recorded by the caller).
  const int W = c->split_group;
  const int nbi = (n + 127) / 128, nbj = (n + Cf::JT - 1) / Cf::JT;
  int G = 1;
  if (hp && hp->groups > 0 && hp->fixed) {
    G = hp->groups;  // the caller's boundaries, multiples of JT
  } else if (hp && hp->groups > 0) {
    G = std::min(hp->groups, nbj);
    hp->groups = G;
    for (int g = 0; g <= G; g++) hp->col[g] = std::min(n, (int)((long)nbj * g / G) * Cf::JT);
  }
  if (!c->smem((const void*)split::k_split_gemm<S>, Cf::SMEM)) return LAPW1GPU_ERR_CUDA;
  if (ev && cudaEventRecord(ev[0], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
  for (int g = 0; g < G; g++) {
    const int bj0 = hp && hp->groups > 0 ? std::min(nbj, hp->col[g] / Cf::JT) : 0;
    const int bj1 = hp && hp->groups > 0 ? (g == G - 1 ? nbj : std::min(nbj, hp->col[g + 1] / Cf::JT)) : nbj;
    int ntile = 0;
    const int2* dt = kp_tiles(k,
                              "split:" + std::to_string(n) + ":" + std::to_string(Cf::JT) + ":" + std::to_string(W) +
                                  ":" + std::to_string(bj0) + ":" + std::to_string(bj1),
                              &ntile, [&](std::vector<int2>& t) {
                                for (int g0 = 0; g0 < nbi; g0 += W)
                                  for (int bj = bj0; bj < bj1; bj++)
                                    for (int bi = g0; bi < std::min(nbi, g0 + W); bi++)
                                      if (bj * Cf::JT <= bi * 128 + 127) t.push_back(make_int2(bi, bj));
                              });
    if (!dt) return LAPW1GPU_ERR_NOMEM;
    split::k_split_gemm<S><<<(unsigned)ntile, SPLIT_THREADS, Cf::SMEM, s>>>(ta, tb, dt, Kp / 64, n, n, ovw ? 2 : 0,
                                                                             exA, exB, hs, ld, c->d_status);
    *nlaunch += 1;
    if (hp && hp->groups > 0 && hp->col[g + 1] <= k->nv) {
      if (cudaEventRecord(hp->ev[g], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
      hp->recorded[g] = true;
    }
  }
  if (ev && cudaEventRecord(ev[1], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
  return l1g_launch_status(__FILE__, __LINE__);
}

// Rectangular product out(i, j) += sum_k L(i, k) R(j, k), i < m, j < nr,
// every tile (no triangle), complex operands in k-major planes: L[k][npadL],
// R[k][npadR] (npadL >= m, npadR >= nr); out column-major with ld.
template <int S>
static int split_gemm_rect(lapw1gpu_context* c, lapw1gpu_kpoint* k, int set, int m, int nr, int Kc,
                           const double2* Lop, int npadL, const double2* Rop, int npadR, double2* out, int ld,
                           cudaStream_t s, int* nlaunch, int ovw, const char* tag) {
  using Cf = split::Cfg<S>;
  const int Kcp = (Kc + 63) / 64 * 64;
  const int Kp = 2 * Kcp;
  const int npL = (npadL + 127) / 128 * 128, npR = (npadR + 127) / 128 * 128;
  const std::string t(tag);
  int8_t* A = (int8_t*)c->sbuf(set, (t + "A").c_str(), (size_t)S * npL * Kp);
  int8_t* B = (int8_t*)c->sbuf(set, (t + "B").c_str(), (size_t)S * 2 * npR * Kp);
  int* exA = (int*)c->sbuf(set, (t + "ExA").c_str(), sizeof(int) * npL);
  int* exB = (int*)c->sbuf(set, (t + "ExB").c_str(), sizeof(int) * npR);
  if (!A || !B || !exA || !exB) return LAPW1GPU_ERR_NOMEM;
  if (cudaMemsetAsync(exA, 0x80, sizeof(int) * npL, s) != cudaSuccess ||
      cudaMemsetAsync(exB, 0x80, sizeof(int) * npR, s) != cudaSuccess)
    return LAPW1GPU_ERR_CUDA;
  split::k_rowexp<<<dim3((npadL + 127) / 128, (Kc + 63) / 64), 128, 0, s>>>(Lop, Kc, npadL, exA);
  split::k_rowexp<<<dim3((npadR + 127) / 128, (Kc + 63) / 64), 128, 0, s>>>(Rop, Kc, npadR, exB);
  split::k_slice_rows<S><<<dim3(npL / 32, Kcp / 64), 256, 0, s>>>(Lop, Kc, Kcp, npadL, npL, 0, 0, exA, A, c->d_status);
  split::k_slice_rows<S><<<dim3(npR / 32, Kcp / 64), 256, 0, s>>>(Rop, Kc, Kcp, npadR, npR, 1, 0, exB, B, c->d_status);
  *nlaunch += 4;
  CUtensorMap ta, tb;
  if (l1g_tmap_3d(&ta, A, Kp, npL, S, 128) || l1g_tmap_3d(&tb, B, Kp, 2 * (uint64_t)npR, S, Cf::N))
    return LAPW1GPU_ERR_CUDA;
  const int W = c->split_group;
  const int nbi = (m + 127) / 128, nbj = (nr + Cf::JT - 1) / Cf::JT;
  int ntile = 0;
  const int2* dt = kp_tiles(k,
                            "rect:" + std::to_string(m) + ":" + std::to_string(nr) + ":" + std::to_string(Cf::JT) +
                                ":" + std::to_string(W),
                            &ntile, [&](std::vector<int2>& t) {
                              for (int g0 = 0; g0 < nbi; g0 += W)
                                for (int bj = 0; bj < nbj; bj++)
                                  for (int bi = g0; bi < std::min(nbi, g0 + W); bi++) t.push_back(make_int2(bi, bj));
                            });
  if (!dt) return LAPW1GPU_ERR_NOMEM;
  if (!c->smem((const void*)split::k_split_gemm<S>, Cf::SMEM)) return LAPW1GPU_ERR_CUDA;
  split::k_split_gemm<S><<<(unsigned)ntile, SPLIT_THREADS, Cf::SMEM, s>>>(ta, tb, dt, Kp / 64, m, nr, ovw ? 3 : 1,
                                                                           exA, exB, out, ld, c->d_status);
  *nlaunch += 1;
  return l1g_launch_status(__FILE__, __LINE__);
}

// tag: the prefix of the scratch buffers (callers whose products differ
// much in size keep separate ones, so that growing one never reallocates
// a buffer that a captured batch uses)
static int split_rect_gemm(lapw1gpu_context* c, lapw1gpu_kpoint* k, int set, int m, int nr, int Kc,
                           const double2* Lop, int npadL, const double2* Rop, int npadR, double2* out, int ld,
                           int slices, cudaStream_t s, int* nlaunch, int ovw = 0, const char* tag = "rect") {
  switch (slices) {
    case 2: return split_gemm_rect<2>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    case 3: return split_gemm_rect<3>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    case 4: return split_gemm_rect<4>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    case 5: return split_gemm_rect<5>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    case 6: return split_gemm_rect<6>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    case 7: return split_gemm_rect<7>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    case 8: return split_gemm_rect<8>(c, k, set, m, nr, Kc, Lop, npadL, Rop, npadR, out, ld, s, nlaunch, ovw, tag);
    default: return LAPW1GPU_ERR_RANGE;
  }
}

// cjL: Lop holds conj(L) (sliced conjugated)
static int split_hns_gemm(lapw1gpu_context* c, lapw1gpu_kpoint* k, int set, int n, int npad, int Kc,
                          const double2* Lop, const double2* Rop, double2* hs, int ld, int slices, cudaStream_t s,
                          int* nlaunch, HnsPipe* hp, const cudaEvent_t* ev, int cjL = 0, int phase = 3,
                          int ovw = 0) {
  switch (slices) {
    case 2: return split_gemm_launch<2>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    case 3: return split_gemm_launch<3>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    case 4: return split_gemm_launch<4>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    case 5: return split_gemm_launch<5>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    case 6: return split_gemm_launch<6>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    case 7: return split_gemm_launch<7>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    case 8: return split_gemm_launch<8>(c, k, set, n, npad, Kc, Lop, Rop, hs, ld, s, nlaunch, hp, ev, cjL, phase, ovw);
    default: return LAPW1GPU_ERR_RANGE;
  }
}

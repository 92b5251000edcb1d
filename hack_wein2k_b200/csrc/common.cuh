// common.cuh -- device helpers shared by the lapw1 setup kernels.
//
// Complex numbers are double2 (x = re, y = im), the layout of Fortran
// COMPLEX*16, so HS/HSDIAG are written in the caller's format directly.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/lapw1gpu.h"

#define L1G_LOMAX LAPW1GPU_LOMAX
#define L1G_NLOAT LAPW1GPU_NLOAT
#define L1G_NSL2 LAPW1GPU_NSL2
#define L1G_MAXL 13  // LMAX of lapw1's param.inc: ltop <= 13

// device status word bits (lapw1gpu context keeps one int on the device)
#define L1G_STATUS_SPHBES 1     // SPHBES argument beyond its start table (sphbes.f:60-64)
#define L1G_STATUS_NONFINITE 2  // a written matrix element is not finite

// true when either component of v is Inf or NaN (all exponent bits set)
__device__ __forceinline__ bool l1g_nonfinite(double2 v) {
  return (((unsigned)(__double_as_longlong(v.x) >> 52) & 0x7ffu) == 0x7ffu) |
         (((unsigned)(__double_as_longlong(v.y) >> 52) & 0x7ffu) == 0x7ffu);
}
#define L1G_STATUS_RANGE 4      // a difference vector fell outside a table

__device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return cmk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return cmk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return cmk(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return cmk(a.x * s, a.y * s); }

// exp(2 pi i s) for a fractional phase s: sincospi avoids the rounding of
// 2*pi*s for large |s| (the reference's phases, hamilt.F:208-216, hns.F:171-174).
__device__ __forceinline__ double2 cexp2pi(double s) {
  double sn, cs;
  sincospi(2.0 * s, &sn, &cs);
  return cmk(cs, sn);
}

// Start index of SPHBES's downward recursion for j_0..j_n at x > 0.1
// (sphbes.f:55-59), before the cap at 98.
__host__ __device__ inline int l1g_sphbes_start(int n, double x) {
  double cufac = 4.2;
  if (x < (double)(n - 2)) cufac = 10.5 / ((double)n + 0.5 - x);
  int ns = (int)((double)(n + 5) + x * cufac);
  return (int)((double)ns + 15.0 / (1.0 + sqrt(x)));
}
// true when SPHBES refuses the argument (sphbes.f:60-64: the start index
// exceeds its table and x > 15); the host checks this before launching
// where it cannot read the device status word back
__host__ __device__ inline bool l1g_sphbes_refuses(int n, double x) {
  return x > 15.0 && l1g_sphbes_start(n, x) + 2 > 100;
}

// SPHBES (sphbes.f:47-142): fj[0..n] = j_l(x).  Returns 0, or a status bit.
__device__ inline int dev_sphbes(int n, double x, double* fj) {
  double* FJ = fj - 1;
  if (x > 0.1) {
    int ns = l1g_sphbes_start(n, x);
    if ((ns + 2) > 100) {
      if (x > 15.0) return L1G_STATUS_SPHBES;
      ns = 98;
    }
    double ffo = 0.0, ffn = 1.0e-25, ffp;
    int m = ns - 1;
    double xi = 1.0 / x;
    double fm = (double)(m + m) + 1.0;
    double sdr = fm * 1.0e-50;
    for (int guard = 0; guard < 200; guard++) {
      ffp = fm * xi * ffn - ffo;
      if (fabs(ffp) >= 1.0e25) {
        sdr = sdr * 1.0e-50;
        ffp = ffp * 1.0e-25;
        ffn = ffn * 1.0e-25;
      }
      sdr = sdr + (fm - 2.0) * ffp * ffp;
      ffo = ffn;
      ffn = ffp;
      if (m <= n) break;
      m = m - 1;
      fm = fm - 2.0;
    }
    FJ[m] = ffn;
    FJ[m + 1] = ffo;
    do {
      m = m - 1;
      fm = fm - 2.0;
      for (int guard = 0; guard < 64; guard++) {
        FJ[m] = fm * xi * FJ[m + 1] - FJ[m + 2];
        if (fabs(FJ[m]) >= 1.0e25) {
          for (int j = m + 1; j <= n + 1; j++) FJ[j] = FJ[j] * 1.0e-25;
          sdr = sdr * 1.0e-50;
          continue;
        }
        break;
      }
      sdr = sdr + (fm - 2.0) * FJ[m] * FJ[m];
    } while (m > 1);
    double ser = 1.0 / sqrt(sdr);
    for (m = 1; m <= n + 1; m++) FJ[m] = FJ[m] * ser;
  } else {
    double hfxsq = 0.5 * (x * x);
    double xl = 1.0, twm = 1.0, ta, xlp;
    int m = 0;
    do {
      m = m + 1;
      ta = xl;
      twm = twm + 2.0;
      xl = xl / twm;
      ta = ta - xl * hfxsq;
      xlp = xl / (twm + 2.0);
      FJ[m] = ta + 0.5 * xlp * hfxsq * hfxsq;
      xl = xl * x;
    } while (m <= n);
  }
  return 0;
}

// DVBES1 (dvbes1.f:32-49)
__device__ inline void dev_dvbes1(const double* fj, double* dj, double sm, double ri, int nt) {
  const double* FJ = fj - 1;
  double* DJ = dj - 1;
  double x = sm * ri;
  if (x > 1.0e-5) {
    double q2 = -1.0 / x, q3 = q2;
    DJ[1] = -FJ[2];
    int lm = 1;
    for (int l = 2; l <= nt; l++) {
      q3 = q3 + q2;
      DJ[l] = FJ[lm] + q3 * FJ[l];
      lm = lm + 1;
    }
  } else {
    DJ[1] = 0.0;
    DJ[2] = 1.0 / 3.0;
    for (int l = 3; l <= nt; l++) DJ[l] = 0.0;
  }
}

// ROTATE (rotate.f:22-28): out = ROTMAT * v, ROTMAT(3,3) in Fortran order
__device__ __forceinline__ void dev_rotate(const double* v, const double* rm, double* out) {
#pragma unroll
  for (int jc = 0; jc < 3; jc++) {
    double d = 0.0;
#pragma unroll
    for (int j = 0; j < 3; j++) d = d + v[j] * rm[j * 3 + jc];
    out[jc] = d;
  }
}

// YLM (ylm.f:162-263) for l <= LMAXT, y[l*l+l+m]
template <int LMAXT>
__device__ inline void dev_ylm(const double* v, int lmax, double2* y) {
  double2* Y = y - 1;
  const double pi = 3.141592653589793238462643;
  double yllr = 1.0 / sqrt(4.0 * pi);
  Y[1] = cmk(yllr, 0.0);
  if (lmax <= 0) return;
  double a, b, c, ab, abc, cosph, sinph, costh, sinth;
  double abmax = fmax(fabs(v[0]), fabs(v[1]));
  if (abmax > 0.0) {
    a = v[0] / abmax;
    b = v[1] / abmax;
    ab = sqrt(a * a + b * b);
    cosph = a / ab;
    sinph = b / ab;
  } else {
    cosph = 1.0;
    sinph = 0.0;
  }
  double abcmax = fmax(abmax, fabs(v[2]));
  if (abcmax > 0.0) {
    a = v[0] / abcmax;
    b = v[1] / abcmax;
    c = v[2] / abcmax;
    ab = a * a + b * b;
    abc = sqrt(ab + c * c);
    costh = c / abc;
    sinth = sqrt(ab) / abc;
  } else {
    costh = 1.0;
    sinth = 0.0;
  }
  Y[3] = cmk(sqrt(3.0) * yllr * costh, 0.0);
  double temp1 = -sqrt(1.5) * yllr * sinth;
  Y[4] = cmk(temp1 * cosph, temp1 * sinph);
  Y[2] = cmk(-Y[4].x, Y[4].y);
#pragma unroll
  for (int l = 2; l <= LMAXT; l++) {
    if (l > lmax) break;
    int index = l * l + 1;
    int index2 = index + 2 * l;
    double msign = (l & 1) ? -1.0 : 1.0;
    double yl1l1r = Y[index - 1].x, yl1l1i = Y[index - 1].y;
    double t1 = -sqrt((double)(2 * l + 1) / (double)(2 * l)) * sinth;
    Y[index2] = cmk(t1 * (cosph * yl1l1r - sinph * yl1l1i), t1 * (cosph * yl1l1i + sinph * yl1l1r));
    Y[index] = cmk(msign * Y[index2].x, -msign * Y[index2].y);
    index2--;
    index++;
    double t2 = sqrt((double)(2 * l + 1)) * costh;
    Y[index2] = cmk(t2 * yl1l1r, t2 * yl1l1i);
    Y[index] = cmk(-msign * Y[index2].x, msign * Y[index2].y);
    index2--;
    index++;
    int i4l2 = index2 - 4 * l + 2;
    int i2l = index2 - 2 * l;
    double d4ll1c = costh * sqrt((double)(4 * l * l - 1));
    double d2l13 = -sqrt((double)(2 * l + 1) / (double)(2 * l - 3));
#pragma unroll
    for (int m = l - 2; m >= 0; m--) {
      double tt1 = 1.0 / sqrt((double)((l + m) * (l - m)));
      double tt2 = d4ll1c * tt1;
      double tt3 = d2l13 * sqrt((double)((l + m - 1) * (l - m - 1))) * tt1;
      Y[index2] = cmk(tt2 * Y[i2l].x + tt3 * Y[i4l2].x, tt2 * Y[i2l].y + tt3 * Y[i4l2].y);
      Y[index] = cmk(msign * Y[index2].x, -msign * Y[index2].y);
      msign = -msign;
      index2--;
      index++;
      i4l2--;
      i2l--;
    }
  }
}

// Y_lm of the locally rotated k+G of one row for one atom
template <int LMAXT>
__device__ __forceinline__ void dev_ylm_row(double xk, double yk, double zk, const double* rotij,
                                            const double* rotloc, int lmax, double2* y) {
  double v[3] = {xk, yk, zk}, r1[3], r2[3];
  dev_rotate(v, rotij, r1);
  dev_rotate(r1, rotloc, r2);
  dev_ylm<LMAXT>(r2, lmax, y);
}

// split_tc.cuh -- split-precision (Ozaki int8 slices, tcgen05) contractions.
#pragma once
#define L1G_MAX_SLICES 8

static int split_hns_gemm(lapw1gpu_context* c, int n, int npad, int K, const double2* Lop, const double2* Rop,
                          double2* hs, int ld, int slices, cudaStream_t s, int* nlaunch) {
  (void)c; (void)n; (void)npad; (void)K; (void)Lop; (void)Rop; (void)hs; (void)ld; (void)slices; (void)s; (void)nlaunch;
  return LAPW1GPU_ERR_RANGE;
}

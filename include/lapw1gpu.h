/*
 * lapw1gpu.h -- C ABI of the B200 lapw1 Hamiltonian/overlap setup.
 *
 * The library replaces the matrix-setup segment of WIEN2k lapw1's CALKPT
 * (SRC_lapw1/calkpt.F:153-185):
 *
 *     CALL HAMILT(NT,NAT,NV,P,PE,DP,DPE,MULT,RMT,POS,V,VI,PEI,E,INS)
 *     CALL ZSWAP(HSROWS,HS,HSROWS+1,HSDIAG,1)
 *     if(.not.nohns) CALL HNS(NV,NAT,LNSMAX+1,POS,VI,RMT,MULT,LQIND,LQNS,
 *                             GFAC,ROTLOC,ROTIJ,VNS1,VNS2,VNS3)
 *     if(Nmod.ne.0)  CALL HORB(NV,NAT,LNSMAX+1,POS,VI,RMT,MULT,LQIND,LQNS,
 *                             PEI,ROTLOC,ROTIJ,HS)
 *
 * and leaves HS / HSDIAG in exactly the state that sequence leaves them
 * (complex build, sequential path):
 *   - HS(i,j), i>j   : conj-stored spherical H (hamilt.F:463) plus the HNS
 *                      'T'-transposed updates (hns.F:449-467) and HORB terms
 *   - HS(i,i)        : diagonal of H (after the ZSWAP, calkpt.F:164) plus
 *                      HNS/HORB diagonal terms
 *   - HS(i,j), i<j   : overlap S (hamilt.F:464)
 *   - HSDIAG(i)      : diagonal of S
 *
 * Every array is a plain host pointer.  Complex numbers are interleaved
 * (re, im) doubles, the layout of Fortran COMPLEX*16.  Array layouts are the
 * Fortran ones of the reference's modules, written here as C index order
 * (last C index fastest == first Fortran index).  Every entry point returns
 * a status code (LAPW1GPU_OK == 0) and never exits the process; the Fortran
 * shim maps a non-zero status to OUTERR + STOP (the reference's error path,
 * SRC_lapw1/outerr.f).
 */
#ifndef LAPW1GPU_H
#define LAPW1GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LAPW1GPU_LOMAX 3   /* param.inc LOMAX: highest l carrying local orbitals */
#define LAPW1GPU_NLOAT 3   /* param.inc nloat: local orbitals per (l, atom) */
#define LAPW1GPU_NSLMAX 5  /* param.inc NSLMAX: lmax_ns + 1 upper bound */
#define LAPW1GPU_NSL2 25   /* NSLMAX*NSLMAX: (l,m) pairs of the non-spherical block */
#define LAPW1GPU_NTNS 9    /* T blocks per atom type: see lapw1gpu_problem.tns */

/* status codes */
enum {
  LAPW1GPU_OK = 0,
  LAPW1GPU_ERR_ARG = 1,        /* inconsistent sizes or a NULL required array */
  LAPW1GPU_ERR_NOMEM = 2,      /* device allocation failed */
  LAPW1GPU_ERR_CUDA = 3,       /* a CUDA runtime call failed */
  LAPW1GPU_ERR_NONFINITE = 4,  /* a kernel met a non-finite intermediate */
  LAPW1GPU_ERR_TIMEOUT = 5,    /* a bounded device wait ran out */
  LAPW1GPU_ERR_NODEVICE = 6,   /* no usable sm_100 device */
  LAPW1GPU_ERR_RANGE = 7       /* a size exceeds a documented limit */
};

/* arithmetic of the muffin-tin contractions */
enum {
  LAPW1GPU_PREC_FP64 = 0,      /* every product in FP64 (the comparator path) */
  LAPW1GPU_PREC_SPLIT = 1      /* Ozaki int8 slices on tcgen05, exact int32 accumulation */
};

/*
 * One k-point's setup problem.  Field names follow the reference's module
 * variables; the comment gives the reference array each field carries.
 */
typedef struct lapw1gpu_problem {
  /* ---- sizes ---- */
  int n;        /* HSROWS = NV + NLO                     (modules.F:441-535) */
  int nv;       /* NV: plane waves                        (coors.f:165)        */
  int nlo;      /* NLO: local-orbital rows                (atpar.f:187-199)    */
  int nat;      /* NAT: inequivalent atoms                                     */
  int ndf;      /* NDF: all atoms, sum of MULT                                 */
  int ltop;     /* NT = lmax+1, 3 <= ltop <= ldl          (inilpw.f:346-350)   */
  int ldl;      /* leading dimension of the per-l arrays (LMAX=13 in lapw1)    */
  int lnsmax;   /* LNSMAX, 0..4: HNS uses (lnsmax+1)^2 (l,m) pairs             */
  int ins;      /* INS: 0 = warped interstitial (WARPIN), else USTPHX only     */
  int nohns;    /* 1 skips HNS (lapw1 -nohns, calkpt.F:169)                    */
  double vi;    /* VI = 1/unit-cell volume                                     */
  double bkzz[9]; /* row-major 3x3 B with Cartesian (k+G) = k + B.KZZ: the
                     matrix COORS builds XK/YK/ZK with (coors.f:47-55,81-83):
                     diag(PIA) for ORTHO lattices, BR2 otherwise            */

  /* ---- structure ---- */
  const int* mult;      /* MULT(NAT)                     [nat]            */
  const double* rmt;    /* RMT(NAT)                      [nat]            */
  const double* v;      /* V(NAT) = 4 pi VI RMT^3 / 3    [nat]            */
  const double* pos;    /* POS(3,NDF), fractional        [ndf][3]         */
  const double* rotij;  /* ROTIJ(3,3,NDF)                [ndf][3][3]      */
  const double* rotloc; /* ROTLOC(3,3,NAT)               [nat][3][3]      */

  /* ---- basis (COORS + LOPW output, fixes the row order) ---- */
  const int* kzz;       /* KZZ(3,HSROWS)                 [n][3]           */
  const double* xk;     /* XK(HSROWS): Cartesian k+G     [n]              */
  const double* yk;     /* YK(HSROWS)                    [n]              */
  const double* zk;     /* ZK(HSROWS)                    [n]              */
  const double* rk;     /* RK(HSROWS) = |k+G|            [n]              */

  /* ---- radial parameters (ATPAR output), [nat][ldl] = X(0:LMAX-1,NAT) ---- */
  const double* p;      /* U(R)      (HAMILT arg U   = P)    */
  const double* pe;     /* Udot(R)   (HAMILT arg UP  = PE)   */
  const double* dp;     /* U'(R)     (HAMILT arg DU  = DP)   */
  const double* dpe;    /* Udot'(R)  (HAMILT arg DUP = DPE)  */
  const double* pei;    /* |Udot|^2  (HAMILT arg CHN = PEI)  */
  const double* e;      /* E_l       (HAMILT arg E)          */
  const int* lapw;      /* LAPW(0:LMAX-1,NAT): 1 LAPW, 0 APW  [nat][ldl] */

  /* ---- local orbitals (modules loabc / lolog) ---- */
  const int* ilo;       /* ILO(0:LOMAX,NAT)                 [nat][4]        */
  const int* loor;      /* LOOR(0:LOMAX,NAT): 1 = LAPW-type LO [nat][4]     */
  const double* alo;    /* ALO(0:LOMAX,NLOAT,NAT)            [nat][3][4]    */
  const double* blo;    /* BLO(0:LOMAX,NLOAT,NAT)            [nat][3][4]    */
  const double* clo;    /* CLO(0:LOMAX,NLOAT,NAT)            [nat][3][4]    */
  const double* elo;    /* ELO(0:LOMAX,NLOAT,NAT)            [nat][3][4]    */
  const double* pi12lo; /* PI12LO(0:LOMAX,NAT)               [nat][4]       */
  const double* pe12lo; /* PE12LO(0:LOMAX,NAT)               [nat][4]       */
  const double* dplo;   /* DPLO(0:LOMAX,NAT)                 [nat][4]       */

  /* ---- interstitial warped potential (module out, SETWAR output) ---- */
  int warp1, warp2, warp3;  /* WARP1..3: half extents                       */
  const double* warp;       /* WARP(-W1:W1,-W2:W2,-W3:W3), complex
                               [2w3+1][2w2+1][2w1+1][2]                      */

  /* ---- non-spherical muffin-tin matrix elements (HNS) ----
   * tns[a][b][l0m0][lpmp] complex, a = atom type, lm = l*(l+1)+m.  These are
   * the sums that hns.F:317-380 forms from GNT x VNS before its loop 30:
   *   b=0 TUU   b=1 TDU   b=2 TUU21   (row block A2, hns.F:387-401)
   *   b=3 TUD   b=4 TDD   b=5 TUD21   (row block B2, hns.F:403-417)
   *   b=6 TUU12 b=7 TDU12 b=8 TUU22   (row block C2, hns.F:419-433)
   * lapw1gpu_tns_from_gaunt() builds them from the reference's GFAC/LQNS/VNS. */
  const double* tns;    /* [nat][9][25][25][2] */

  /* ---- orbital potential (HORB, module orb) ---- */
  int natorb;           /* NATORB; 0 skips HORB (calkpt.F:176)         */
  const int* iatom;     /* IATOM(NATORB): atom type of each U-atom     */
  const int* nlorb;     /* NLORB(NATORB)                               */
  const int* lorb;      /* LORB(3,NATORB)            [natorb][3]       */
  const double* vorb;   /* VORB(iat,l,m1,m2) complex [natorb][4][7][7][2],
                           index [iat][l][m1+3][m2+3]                  */
} lapw1gpu_problem;

/* timings of one setup, milliseconds of device time (CUDA events) */
typedef struct lapw1gpu_stats {
  double ms_total;      /* whole setup on the device                  */
  double ms_albl;       /* K-a: matching coefficients + operand build  */
  double ms_spherical;  /* K-b + K-c: PW x PW spherical + interstitial */
  double ms_lo;         /* K-b': local-orbital columns                 */
  double ms_hns;        /* K-ns: non-spherical contraction             */
  double ms_horb;       /* K-orb                                       */
  double ms_h2d;        /* host->device copies (host entry points)     */
  double ms_d2h;        /* device->host copy of HS/HSDIAG              */
  double flops_fp64_equiv; /* algorithmic FP64 flops of K-b + K-ns     */
  double kernel_launches;  /* kernels this library launched in the run */
  double ms_sph_main;   /* the spherical contraction kernel alone (k_spherical
                           or k_sph_tc), inside ms_spherical               */
  double ms_hns_main;   /* the HNS update alone (k_hns_gemm + ZGEMM panels, or
                           the tcgen05 slice products), inside ms_hns      */
  double ms_k_albl;     /* K-a: the matching-coefficient kernel k_albl alone  */
  double ms_table;      /* K-c: the Theta/WARP table kernel k_table alone     */
  double ms_sph_slice;  /* K-a, split path: the two spherical operand slicers
                           (phases x AL/BL cut into int8 slices)             */
  double ms_host;       /* batch: host time of enqueuing the graph launch   */
} lapw1gpu_stats;

typedef struct lapw1gpu_context lapw1gpu_context;

/* Context on one CUDA device: stream, events, cached device buffers.
 * Replaces nothing in the reference (lapw1 has no device); one context per
 * host thread and device. */
int lapw1gpu_init(int device, lapw1gpu_context** ctx);
int lapw1gpu_finalize(lapw1gpu_context* ctx);
/* select the muffin-tin contraction arithmetic (LAPW1GPU_PREC_*); with
 * LAPW1GPU_PREC_SPLIT both the spherical part and HNS use `slices` int8
 * slices (2..8; the spherical part runs on tensor cores for 4..7) */
int lapw1gpu_set_precision(lapw1gpu_context* ctx, int prec, int slices);
/* split precision with separate slice counts for the spherical part and
 * for HNS (the non-spherical part is one to two orders of magnitude
 * smaller, so it tolerates one slice fewer at the same eigenvalue error) */
int lapw1gpu_set_slices(lapw1gpu_context* ctx, int slices_sph, int slices_hns);
/* int8 slices (4..8 each, default 6 and 6) of the adjoint's products in
 * split precision (lapw1gpu_forces): the density matrices rho, rhoE and
 * the HNS projections Y = R^H (G c); the spherical pair sums are FP64
 * (lapw1gpu_set_force_projection moves the cross-block ones to int8
 * projections) */
int lapw1gpu_set_force_slices(lapw1gpu_context* ctx, int slices_density,
                              int slices_projection);
/* Spherical pair sums of the adjoint in split precision as projections:
 * slices = 0 keeps the FP64 pair kernel for every PW x PW pair; 4..8 forms
 * the pairs of two different blocks of block_rows PW rows (a multiple of
 * 32, at least 64) from int8 slice products of the rows' real-harmonic
 * expansion (addition theorem) with (G c)^T, block by block against the
 * running sum of the blocks before; the pairs inside a block stay on the
 * FP64 pair kernel.  slices = -1 (the default, with 1024-row blocks): 6
 * slices when the PW rows span at least 6 blocks, else the pair kernel. */
int lapw1gpu_set_force_projection(lapw1gpu_context* ctx, int slices,
                                  int block_rows);

/* One k-point's inputs resident in device memory (uploaded once; the
 * benchmark's resident-input path and the k-point batch driver use it). */
typedef struct lapw1gpu_kpoint lapw1gpu_kpoint;
int lapw1gpu_kpoint_upload(lapw1gpu_context* ctx, const lapw1gpu_problem* p,
                           lapw1gpu_kpoint** kp);
int lapw1gpu_kpoint_free(lapw1gpu_kpoint* kp);
/* Run the selected stages on a resident k-point into device memory:
 * d_hs is n x n complex column-major with leading dimension ldhs, d_hsdiag
 * n complex.  Stage bits: 1 HAMILT (+ZSWAP), 2 HNS, 4 HORB; 7 = all of
 * calkpt.F:153-185.  Asynchronous on the context's stream unless st != NULL
 * (then it synchronises and fills the timings). */
int lapw1gpu_kpoint_run(lapw1gpu_context* ctx, lapw1gpu_kpoint* kp, int stages,
                        double* d_hs, int ldhs, double* d_hsdiag,
                        lapw1gpu_stats* st);

/* Full drop-in for calkpt.F:153-185 (HAMILT, ZSWAP, HNS, HORB) with host
 * buffers: hs is HS(HSROWS,HSROWS) complex, column-major with leading
 * dimension ldhs >= n; hsdiag is HSDIAG(HSROWS).  The library writes every
 * element of the n x n block (INIT_MATRICES zeroing is not needed).
 * Synchronous: returns when hs/hsdiag hold the result. */
int lapw1gpu_setup(lapw1gpu_context* ctx, const lapw1gpu_problem* p,
                   double* hs, int ldhs, double* hsdiag, lapw1gpu_stats* st);
/* lapw1gpu_setup without the wait: returns once the setup's kernels and
 * the copies of HS/HSDIAG into the caller's buffers are queued.  The copies
 * run on the context's copy stream behind the kernels that produce each
 * column group, so later device work on the context's stream (the device
 * eigen-solve, lapw1gpu_forces of a resident k-point) overlaps them.
 * lapw1gpu_setup_wait ends it: it waits for the kernels and the copies and
 * returns the status lapw1gpu_setup would have returned (st optional).
 * Until then hs, hsdiag and the problem's host arrays stay valid and
 * unchanged, and no other lapw1gpu_setup* call is made on the context
 * (they return LAPW1GPU_ERR_ARG).  No counterpart in the reference (its
 * CALKPT is sequential). */
int lapw1gpu_setup_async(lapw1gpu_context* ctx, const lapw1gpu_problem* p,
                         double* hs, int ldhs, double* hsdiag);
int lapw1gpu_setup_wait(lapw1gpu_context* ctx, lapw1gpu_stats* st);

/* lapw1gpu_setup restricted to the given stages (parity tests of each
 * reference routine). */
int lapw1gpu_setup_stages(lapw1gpu_context* ctx, const lapw1gpu_problem* p,
                          int stages, double* hs, int ldhs, double* hsdiag,
                          lapw1gpu_stats* st);

/* the context's CUDA stream (cudaStream_t), for callers that order their
 * own work after an asynchronous lapw1gpu_kpoint_run */
void* lapw1gpu_stream(lapw1gpu_context* ctx);

/* Test hook of the bounded device waits.  No counterpart in the reference.
 * With on = 1, later runs of the split-precision spherical tensor-core
 * kernel make its MMA issuer wait on a barrier that nothing arrives at,
 * bounded to about half a millisecond: the kernel takes its timeout path
 * (status bit, copies in flight drained, TMEM freed) and the run returns
 * LAPW1GPU_ERR_TIMEOUT with the context still usable.  on = 0 (the
 * default) restores normal runs. */
int lapw1gpu_test_wait_timeout(lapw1gpu_context* ctx, int on);

/* Page-lock a caller buffer (typically HS, allocated once by INIT_MATRICES,
 * modules.F:526-535) for the context's lifetime, so that the host entry
 * points copy HS at full link speed and overlap those copies with the later
 * stages; without it the copies into pageable memory are staged by the
 * driver and serialise.  A buffer already page-locked by the caller is
 * accepted as is.  lapw1gpu_finalize (or lapw1gpu_host_unregister) undoes
 * it; the caller must not free the buffer before then.  No counterpart in
 * the reference. */
int lapw1gpu_host_register(lapw1gpu_context* ctx, void* ptr, size_t bytes);
int lapw1gpu_host_unregister(lapw1gpu_context* ctx, void* ptr);

/* kernels launched by the last setup, batch or forces call on the context
 * (a library product counts as one launch); no counterpart in the reference */
int lapw1gpu_last_launches(lapw1gpu_context* ctx);

/* device status word of the last run (L1G_STATUS_* bits), 0 if clean; after
 * an asynchronous lapw1gpu_kpoint_run it waits for that run first */
int lapw1gpu_last_status(lapw1gpu_context* ctx);

/* SECLR4's generalized eigen-solve (seclr4.F:149-345) on the device, from
 * the packed state the setup leaves: H x = e S x with H(i,j) = conj(HS(i,j))
 * and S(i,j) = conj(HS(j,i)) for i > j (ZHCGST factors S**T), real
 * diagonals from HS(i,i) and HSDIAG(i).  Eigenvalues in (el, eu], at most
 * nmax, ascending, into d_eig (device, nmax doubles); their S-orthonormal
 * eigenvectors into d_vec (device, n x nmax complex column-major, ldv >= n;
 * NULL: eigenvalues only); *nfound (host) their count.  d_hs/d_hsdiag are
 * read only.  The solver is the library's (cuSOLVER zhegvdx: Cholesky,
 * reduction, divide and conquer), where the reference calls ZPOTRF, ZHCGST,
 * ZHEEVX2 and ZTRSM.  A non-positive-definite S returns LAPW1GPU_ERR_NONFINITE.
 * Synchronous. */
int lapw1gpu_seclr4(lapw1gpu_context* ctx, const double* d_hs, int ldhs, const double* d_hsdiag, int n,
                    double el, double eu, int nmax, double* d_eig, double* d_vec, int ldv, int* nfound);

/* Build the nine HNS T blocks from the reference's gaunt lists: the sums of
 * hns.F:317-380 over LMSORT's grouping (lmsort.f:246-421: entries sorted by
 * (l0,m0,l',m',LM), a repeated tuple keeping its first gaunt factor).
 *   lqind[nat]                       LQIND(NAT)
 *   lqns  [nat][ngau][6]             LQNS(6,NGAU,NAT)
 *   gfac  complex [nat][ngau]        GFAC(NGAU,NAT)
 *   vns1/2/3 [nat][5][lmmx][5]       VNS1(0:NSLMAX-1,LMMX,0:NSLMAX-1,NAT)
 *   vnslo1/2/3 [nat][5][lmmx][4]     VNS1LO(LOMAX+1,LMMX,NSLMAX,NAT)
 *   loor  [nat][4]                   LOOR(0:LOMAX,NAT)
 * Output tns as in lapw1gpu_problem.tns.  Host-only, no device needed. */
int lapw1gpu_tns_from_gaunt(int nat, int lnsmax, int ngau, int lmmx,
                            const int* lqind, const int* lqns,
                            const double* gfac, const double* vns1,
                            const double* vns2, const double* vns3,
                            const double* vnslo1, const double* vnslo2,
                            const double* vnslo3, const int* loor,
                            double* tns);

/* HNS stage without any allocation.  No counterpart in the reference: it
 * exists for callers that cannot let this library allocate device memory,
 * such as a lapw1 whose device memory is already reserved by the eigen-solver
 * library that HS is handed to, or a host framework whose caching allocator
 * owns the GPU (a cudaMalloc here could fail or fragment their pool, and
 * cudaFree synchronises the device).  It adds the HNS update (hns.F:150-467,
 * the same result as stage 2 of lapw1gpu_setup_stages) into d_hs, a device
 * n x n complex column-major HS with leading dimension ldhs, on `stream`
 * (a cudaStream_t, NULL for the default stream), asynchronously.  All of its
 * intermediate buffers live in one 64 MiB device array inside the library
 * (held by every GPU that loads the library until the process exits);
 * problems needing more return LAPW1GPU_ERR_RANGE, and so do problems whose
 * RMT |k+G| lies beyond SPHBES's range (checked on the host, before any
 * device work, as the HNS stage reports it).  The problem's host arrays are
 * copied with cudaMemcpyAsync on `stream`.
 * d_status (optional, device int, NULL to skip): cleared on `stream`, then
 * given the L1G status bits of the call once the stream reaches its end
 * (2: a non-finite element in the updated HS; 0 clean).  Reading it after
 * the stream is the caller's way to learn what the HNS stage reports as
 * LAPW1GPU_ERR_NONFINITE.
 * The first call on a device looks up that array's device address and keeps
 * it for the process: make it before any stream capture, and make no call
 * on a device after cudaDeviceReset there.  Calls share the array, so calls
 * that overlap on the GPU race. */
int lapw1gpu_hns_noalloc(const lapw1gpu_problem* p, double* d_hs, int ldhs,
                         void* stream, int* d_status);

/* A k-point batch (a lapw1 k-list, lapw1.F:50-67 calls CALKPT per k) set
 * up in one launch: the stage sequences of all nk uploaded k-points are
 * captured once into a CUDA graph, the k-points spread over the context's
 * concurrent chains (each chain with its own scratch), and the graph is
 * replayed by later calls with the same arguments.  stages must include 1
 * (HS is built from scratch).  d_hs[i] / d_hsdiag[i]: device, k-point i's
 * HS (ldhs[i] >= n_i) and HSDIAG.  Synchronous; st (optional) gets
 * ms_total of the whole batch and the summed flops and launches. */
int lapw1gpu_setup_batch(lapw1gpu_context* ctx, lapw1gpu_kpoint* const* kps,
                         int nk, int stages, double* const* d_hs,
                         const int* ldhs, double* const* d_hsdiag,
                         lapw1gpu_stats* st);

/* Tunables of the context (tile and schedule parameters) and the
 * autotuner that picks them by timing candidates on a k-point. */
typedef struct {
  int hns_diag_b;   /* FP64 HNS: diagonal block of the blocked update (256..2048) */
  int split_group;  /* split HNS: row tiles per L2 rasterisation group           */
  int sph_tc;       /* split: spherical part on tcgen05 (1) or FP64 (0)          */
  int batch_sets;   /* concurrent k-point chains in a batch (1..4)               */
  int sph_kblock;   /* split: K bytes per k_sph_tc pipeline stage, 64 (four-deep
                       ring of 64-byte swizzled rows) or 128 (two stages of
                       128-byte rows; up to 5 slices, else 64 is used;
                       the default)                                           */
  double ms_best;   /* setup time of the tuned k-point with the choices, ms      */
} lapw1gpu_tuning;
int lapw1gpu_get_tuning(lapw1gpu_context* ctx, lapw1gpu_tuning* t);
int lapw1gpu_set_tuning(lapw1gpu_context* ctx, const lapw1gpu_tuning* t);
/* Time the candidates of every tunable of the current precision on kp
 * (stages 7 into d_hs/d_hsdiag) and keep the fastest; out (optional) gets
 * the choices.  No counterpart in the reference. */
int lapw1gpu_autotune(lapw1gpu_context* ctx, lapw1gpu_kpoint* kp, double* d_hs,
                      int ldhs, double* d_hsdiag, lapw1gpu_tuning* out);

/* Gradient of the band energy E = sum_b occ[b] eps[b] with respect to the
 * atom positions POS (lattice coordinates), for the eigenpairs of the H, S
 * that lapw1gpu_kpoint_run builds for kp (H c = eps S c as SECLR4 forms it).
 * d_c: device, complex, column-major n x nb (ldc >= n), S-normalized
 * eigenvectors; d_occ, d_eps: device, nb doubles each; d_grad: device,
 * ndf x 3 doubles, overwritten with dE/dPOS (Ry per lattice unit; Cartesian
 * forces follow as -(1/2pi) BKZZ dE/dPOS per atom).  Hellmann-Feynman for the
 * fixed basis: radial functions, rotations and the warped potential held
 * fixed.  No counterpart in lapw1 (it has no derivative code); the
 * reference's forces are lapw2's (SRC_lapw2/fomai1.f, l2main.F:630-634) on
 * another formulation.  Problems with HORB potentials (natorb > 0) return
 * LAPW1GPU_ERR_ARG.  Synchronous. */
int lapw1gpu_forces(lapw1gpu_context* ctx, lapw1gpu_kpoint* kp,
                    const double* d_c, int ldc, int nb, const double* d_occ,
                    const double* d_eps, double* d_grad);

/* lapw1gpu_forces for a k-point list (the k-points of a lapw1gpu_setup_batch
 * and their eigenvectors): kps[i], d_c[i] (ldc[i] >= n_i, nb columns),
 * d_eps[i] (nb eigenvalues) and d_grad[i] (ndf x 3) per k-point, one
 * occupation vector d_occ for all.  The k-points are queued back to back on
 * the context's stream with one synchronisation at the end; ms_total
 * (optional) gets the device time of the whole list.  Synchronous.  No
 * counterpart in lapw1. */
int lapw1gpu_forces_batch(lapw1gpu_context* ctx, lapw1gpu_kpoint* const* kps, int nk,
                          const double* const* d_c, const int* ldc, int nb, const double* d_occ,
                          const double* const* d_eps, double* const* d_grad, double* ms_total);

/* Device times of the last lapw1gpu_forces call on the context, in the
 * fields of lapw1gpu_stats: ms_total the whole call, ms_albl the operands
 * and the density matrices, ms_spherical the plane-wave pair sums with
 * ms_sph_main the pair kernel k_force_sph alone, ms_sph_slice the int8
 * products of the spherical projections with their operand slicing and
 * ms_table the projections' other kernels (both 0 without them), ms_lo the
 * step-function
 * sums and the local-orbital columns, ms_hns the non-spherical part,
 * kernel_launches its launches.  No counterpart in the reference. */
int lapw1gpu_forces_stats(lapw1gpu_context* ctx, lapw1gpu_stats* st);

/* version string of the library */
const char* lapw1gpu_version(void);
/* The CUDA call that made this thread's latest LAPW1GPU_ERR_CUDA ("file:line:
 * error name (code)"), or "" before any: a diagnostic for the caller's log.
 * No counterpart in the reference. */
const char* lapw1gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* LAPW1GPU_H */

// lapw1gpu.cu -- C ABI of the B200 lapw1 H/S setup (include/lapw1gpu.h).
//
// Host side: context (stream, events, grow-only device buffers), upload of
// one k-point's inputs, and the stage sequence of calkpt.F:153-185:
//   HAMILT  -> k_albl, k_phase, k_table, k_sph_coef, k_spherical, k_lo
//   ZSWAP   -> folded into the HAMILT writes (diag(HS) = H, HSDIAG = S)
//   HNS     -> k_hns_alm, k_hns_tmul, k_hns_lo_ops (operands), then
//              k_hns_gemm + library ZGEMM panels (FP64) or the
//              split-precision tcgen05 path, and k_hns_lo
//   HORB    -> k_horb_rows, k_horb_pairs per U-atom and l
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "kernels_fp64.cuh"
#include "forces.cuh"

// The last failing CUDA call of this thread, for lapw1gpu_last_error
static thread_local char g_last_error[192];
static void l1g_note_error(const char* what, long code, const char* file, int line) {
  const char* base = strrchr(file, '/');
  snprintf(g_last_error, sizeof(g_last_error), "%s:%d: %s (%ld)", base ? base + 1 : file, line, what, code);
}
// the launch status after kernel launches, noted when it is an error
static int l1g_launch_status(const char* file, int line) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return LAPW1GPU_OK;
  l1g_note_error(cudaGetErrorName(e), (long)e, file, line);
  return LAPW1GPU_ERR_CUDA;
}


#define L1G_VERSION "lapw1gpu 0.1 (sm_100a)"

namespace {

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace

#define L1G_MAX_SETS 4  // concurrent k-point chains in a batch (scratch sets)
#define L1G_MAX_GROUPS 16

// Column groups of HS: the spherical contraction and the HNS update run
// group by group, each group followed by an event, so that a caller can
// copy finished columns of HS while later groups run.  With fixed set, the
// caller chose the boundaries (multiples of every stage's tile width);
// otherwise (HNS only) the HNS stage picks them.  groups = 0: one pass.
struct HnsPipe {
  int groups = 0;
  bool fixed = false;
  int col[L1G_MAX_GROUPS + 1] = {};  // group g covers columns [col[g], col[g+1])
  cudaEvent_t ev[L1G_MAX_GROUPS] = {};   // HNS of group g done
  bool recorded[L1G_MAX_GROUPS] = {};
  cudaEvent_t sev[L1G_MAX_GROUPS] = {};  // S (upper triangle) of group g final
  bool srec[L1G_MAX_GROUPS] = {};
};

struct lapw1gpu_context {
  int device = 0;
  int nsm = 148;  // streaming multiprocessors (persistent grids)
  cudaStream_t stream = nullptr;
  cudaStream_t side[L1G_MAX_SETS] = {};  // streams of scratch sets 1.. in a batch
  cudaEvent_t ev[22] = {};  // 0-6 stages, 7-11 host copies, 12-15 main contraction kernels,
                            // 16-21 k_albl, k_table, the spherical slicers
  cudaEvent_t fork = nullptr, join[L1G_MAX_SETS] = {};
  cudaEvent_t fev[7] = {};  // the last forces call: start, density matrices, k_force_sph, LO columns, end;
                            // [6] the end of the spherical projections
  float fms[7] = {};        // its intervals (ms), read by lapw1gpu_forces_stats; [5] the projections,
                            // [6] their products (the split_rect_gemm calls)
  bool fproj_last = false;  // the last forces call formed spherical projections
  std::vector<cudaEvent_t> fpev;  // timed forces call: around each projection product
  int fpev_used = 0;
  // per scratch set: the stream that prepares the split HNS operands while
  // the spherical stage runs, and its fork/join events
  cudaStream_t aux[L1G_MAX_SETS] = {};
  cudaEvent_t auxf[L1G_MAX_SETS] = {}, auxj[L1G_MAX_SETS] = {};
  cudaEvent_t hns_ev[L1G_MAX_GROUPS] = {}, sph_ev[L1G_MAX_GROUPS] = {};
  int* d_status = nullptr;
  int last_status = 0;
  bool status_pending = false;  // an asynchronous run has not been read back
  // a setup queued by lapw1gpu_setup_async, ended by lapw1gpu_setup_wait
  struct lapw1gpu_kpoint* async_k = nullptr;  // its uploaded inputs (freed by the wait)
  int* h_async_status = nullptr;              // mapped host word: its status word
  int* h_async_status_dev = nullptr;          //   (the device view of it)
  int* h_status = nullptr;                    // mapped host word: the status of a synchronous call
  int* h_status_dev = nullptr;
  cudaEvent_t async_done = nullptr;           // its kernels and status copy (main stream)
  bool async_copies = false;                  // HS copies queued on the copy stream (ev[11] ends them)
  int async_nl = 0;
  bool async_pending = false;
  int prec = LAPW1GPU_PREC_FP64;
  int slices = 5;      // int8 slices of the spherical part (split precision)
  int slices_hns = 5;  // int8 slices of the HNS update
  int slices_frc = 6;  // int8 slices of the adjoint's density matrices
  int slices_prj = 6;  // and of its HNS projections
  int slices_fsp = -1;   // and of its spherical projections (0: the FP64 pair kernel for every pair;
                         // -1: L1G_FSP_SLICES slices when NV spans L1G_FSP_MIN_BLOCKS blocks)
  int fsp_block = 1024;  // PW rows per block of the spherical projections
  cublasHandle_t blas[L1G_MAX_SETS] = {};  // library ZGEMMs, one handle (and workspace) per scratch set
  cusolverDnHandle_t solver = nullptr;      // the eigen-solve (lapw1gpu_seclr4)
  // tunables (lapw1gpu_autotune)
  int hns_diag_b = 512;    // FP64 HNS: diagonal block of the blocked ZHER2M form
  int split_group = 16;    // split HNS: row tiles per rasterisation group
  int sph_tc = 1;          // split precision: spherical part on tcgen05 (1) or FP64 (0)
  int sph_kb = 128;        // k_sph_tc: bytes of K per pipeline stage (64: deep ring, 128: two stages)
  int batch_sets = 2;      // concurrent k-point chains in a batch
  int test_never_wait = 0; // test hook: the spherical tensor kernel's consumer wait runs out
  int last_launches = 0;   // kernels launched by the last call (a library product counts as one)
  std::map<std::string, DevBuf> bufs;
  std::map<std::string, std::pair<int2*, int>> tiles;  // tile lists per shape (kp_tiles)
  struct Graph {
    std::vector<uintptr_t> key;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
  };
  std::vector<Graph> graphs;  // captured batches
  std::vector<void*> host_pinned;        // caller buffers page-locked by lapw1gpu_host_register

  // raise a kernel's dynamic shared-memory limit (not a stream operation,
  // and kept out of captured sequences).  The limit belongs to the kernel
  // on the device, not to a context, so the record of what was set is
  // process-wide and the limit only ever grows: a second context (or a
  // second library user) asking for less must not lower it under a size
  // that another context's queued launches rely on.
  bool smem(const void* fn, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> raised;  // (device, kernel) -> limit set there
    static std::map<const void*, int> widest;                  // kernel -> largest limit set anywhere
    std::lock_guard<std::mutex> lock(mu);
    int& cur = raised[std::make_pair(device, fn)];
    if (cur >= bytes) return true;
    int& wide = widest[fn];
    const int want = std::max(bytes, wide);  // never below a limit set before, on any device
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, want);
    if (e != cudaSuccess) {
      l1g_note_error(cudaGetErrorName(e), (long)e, __FILE__, __LINE__);
      cudaGetLastError();
      return false;
    }
    cur = want;
    wide = want;
    return true;
  }

  // grow-only scratch buffer; returns nullptr on allocation failure
  void* buf(const std::string& name, size_t bytes) {
    DevBuf& b = bufs[name];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
      if (b.ptr) {
        cudaDeviceSynchronize();  // a captured batch or a queued run may still use it
        cudaFree(b.ptr);
        drop_graphs();
      }
      b.ptr = nullptr;
      b.bytes = 0;
      if (cudaMalloc(&b.ptr, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
      b.bytes = bytes;
    }
    return b.ptr;
  }
  // scratch of one set: buffers of concurrent k-point chains never alias
  void* sbuf(int set, const char* name, size_t bytes) {
    return set == 0 ? buf(name, bytes) : buf(std::string(name) + "#" + std::to_string(set), bytes);
  }
  cublasHandle_t handle(int set, cudaStream_t s) {
    if (!blas[set] && cublasCreate(&blas[set]) != CUBLAS_STATUS_SUCCESS) return nullptr;
    if (cublasSetStream(blas[set], s) != CUBLAS_STATUS_SUCCESS) return nullptr;
    return blas[set];
  }
  void drop_graphs() {
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
};


struct lapw1gpu_kpoint {
  lapw1gpu_context* ctx = nullptr;
  // host copies of sizes and small tables
  int n = 0, nv = 0, nlo = 0, nat = 0, ndf = 0, ltop = 0, ldl = 0, lnsmax = 0, ins = 0, nohns = 0;
  int nvpad = 0, npad = 0;
  double vi = 0.0;
  TabDesc tab{};
  std::vector<LoCol> locols;
  std::vector<LoRange> loranges;
  std::vector<int> mult, atype, afirst;
  // HORB description
  struct OrbItem {
    int a, lvor, iat;
  };
  std::vector<OrbItem> orbs;
  std::vector<double2> pots;  // [norb][49] pot(m1,m0) arrays
  // device inputs (one arena)
  void* arena = nullptr;
  size_t arena_bytes = 0;
  bool owns_arena = true;
  DevProb P{};
  const double2* d_warp = nullptr;
  const double2* d_tns = nullptr;
  const LoCol* d_locols = nullptr;
  const LoRange* d_loranges = nullptr;
  const double2* d_pots = nullptr;
};

// Device tile list for the shape named by `key` (sizes and tile parameters),
// built by `make` on first use and kept by the context: lists depend on the
// shape only, so k-points of equal shape share them and a list, once built,
// never changes under a queued run or a captured batch.
template <class F>
static const int2* kp_tiles(lapw1gpu_kpoint* k, const std::string& key, int* count, F make) {
  auto& tiles = k->ctx->tiles;
  auto it = tiles.find(key);
  if (it != tiles.end()) {
    *count = it->second.second;
    return it->second.first;
  }
  std::vector<int2> t;
  make(t);
  int2* d = nullptr;
  if (t.empty() || cudaMalloc(&d, sizeof(int2) * t.size()) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (cudaMemcpy(d, t.data(), sizeof(int2) * t.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  tiles[key] = std::make_pair(d, (int)t.size());
  *count = (int)t.size();
  return d;
}

#include "split_tc.cuh"
#include "sph_tc.cuh"

namespace {

#define CK(x)                                           \
  do {                                                  \
    cudaError_t _e = (x);                               \
    if (_e != cudaSuccess) {                            \
      l1g_note_error(cudaGetErrorName(_e), _e, __FILE__, __LINE__); \
      cudaGetLastError();                               \
      return LAPW1GPU_ERR_CUDA;                         \
    }                                                   \
  } while (0)

// one thread stores the device status word into a mapped host word
__global__ void k_status_out(const int* __restrict__ d, int* h) { *(volatile int*)h = *d; }

// The status word after the work queued on s: through the mapped host word
// (no copy engine), else by a copy.  Synchronises s; counts its launch in *nl.
static int read_status(lapw1gpu_context* c, cudaStream_t s, int* out, int* nl = nullptr) {
  if (c->h_status) {
    k_status_out<<<1, 1, 0, s>>>(c->d_status, c->h_status_dev);
    CK(cudaGetLastError());
    if (nl) ++*nl;
    CK(cudaStreamSynchronize(s));
    *out = *(volatile int*)c->h_status;
    return LAPW1GPU_OK;
  }
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *out = h;
  return LAPW1GPU_OK;
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// validation of the caller's problem (the checks the reference makes by
// array bounds and STOPs: param.inc limits, sizes consistent)
int validate(const lapw1gpu_problem* p) {
  if (!p) return LAPW1GPU_ERR_ARG;
  if (p->nv < 1 || p->nlo < 0 || p->n != p->nv + p->nlo || p->nat < 1 || p->ndf < p->nat) return LAPW1GPU_ERR_ARG;
  if (p->ltop < 3 || p->ltop > L1G_MAXL || p->ldl < p->ltop) return LAPW1GPU_ERR_RANGE;
  if (p->lnsmax < 0 || p->lnsmax > 4 || p->lnsmax + 1 > p->ltop) return LAPW1GPU_ERR_RANGE;
  if (!p->mult || !p->rmt || !p->v || !p->pos || !p->rotij || !p->rotloc || !p->kzz || !p->xk || !p->yk ||
      !p->zk || !p->rk || !p->p || !p->pe || !p->dp || !p->dpe || !p->pei || !p->e || !p->lapw || !p->ilo ||
      !p->loor || !p->alo || !p->blo || !p->clo || !p->elo || !p->pi12lo || !p->pe12lo || !p->dplo)
    return LAPW1GPU_ERR_ARG;
  if (p->ins == 0 && !p->warp) return LAPW1GPU_ERR_ARG;
  if (!p->nohns && !p->tns) return LAPW1GPU_ERR_ARG;
  int ndf = 0;
  for (int a = 0; a < p->nat; a++) {
    if (p->mult[a] < 1) return LAPW1GPU_ERR_ARG;
    ndf += p->mult[a];
  }
  if (ndf != p->ndf) return LAPW1GPU_ERR_ARG;
  long nlo = 0;
  for (int a = 0; a < p->nat; a++)
    for (int l = 0; l <= L1G_LOMAX; l++) {
      int il = p->ilo[a * (L1G_LOMAX + 1) + l];
      if (il < 0 || il > L1G_NLOAT) return LAPW1GPU_ERR_RANGE;
      nlo += (long)(2 * l + 1) * p->mult[a] * il;
    }
  if (nlo != p->nlo) return LAPW1GPU_ERR_ARG;
  if (p->natorb < 0) return LAPW1GPU_ERR_ARG;
  if (p->natorb > 0 && (!p->iatom || !p->nlorb || !p->lorb || !p->vorb)) return LAPW1GPU_ERR_ARG;
  for (int i = 0; i < p->natorb; i++) {
    if (p->iatom[i] < 1 || p->iatom[i] > p->nat) return LAPW1GPU_ERR_ARG;
    if (i > 0 && p->iatom[i] <= p->iatom[i - 1]) return LAPW1GPU_ERR_ARG;  // horb.F:100 walks them in order
    if (p->nlorb[i] < 0 || p->nlorb[i] > 3) return LAPW1GPU_ERR_RANGE;
    for (int q = 0; q < p->nlorb[i]; q++)
      if (p->lorb[i * 3 + q] < 0 || p->lorb[i * 3 + q] > 3 || p->lorb[i * 3 + q] >= p->ltop) return LAPW1GPU_ERR_RANGE;
  }
  return LAPW1GPU_OK;
}

}  // namespace

extern "C" {

const char* lapw1gpu_version(void) { return L1G_VERSION; }

const char* lapw1gpu_last_error(void) { return g_last_error; }

int lapw1gpu_init(int device, lapw1gpu_context** out) {
  if (!out) return LAPW1GPU_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return LAPW1GPU_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return LAPW1GPU_ERR_NODEVICE;
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return LAPW1GPU_ERR_NODEVICE;  // built for sm_100a only
  CK(cudaSetDevice(device));
  lapw1gpu_context* c = new lapw1gpu_context();
  c->device = device;
  c->nsm = prop.multiProcessorCount;
  // the main and chain streams at the highest priority, the auxiliary
  // (HNS operand) streams at the lowest: the block scheduler then places the
  // persistent spherical kernel's CTAs first and the operand kernels in the
  // gaps
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess) {
    delete c;
    return LAPW1GPU_ERR_CUDA;
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
  for (auto& e : c->fev) cudaEventCreate(&e);
  cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
  for (auto& e : c->hns_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto& e : c->sph_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (int i = 1; i < L1G_MAX_SETS; i++) {
    cudaStreamCreateWithPriority(&c->side[i], cudaStreamNonBlocking, prio_hi);
    cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming);
  }
  for (int i = 0; i < L1G_MAX_SETS; i++) {
    cudaStreamCreateWithPriority(&c->aux[i], cudaStreamNonBlocking, prio_lo);
    cudaEventCreateWithFlags(&c->auxf[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->auxj[i], cudaEventDisableTiming);
  }
  cudaEventCreateWithFlags(&c->async_done, cudaEventDisableTiming);
  // status words read back through mapped host memory (a one-thread kernel
  // stores them), not by copies, which would queue behind a running
  // lapw1gpu_setup_async's HS copies on the copy engines
  for (int** w : {&c->h_async_status, &c->h_status}) {
    if (cudaHostAlloc(w, sizeof(int), cudaHostAllocMapped) != cudaSuccess) {
      cudaGetLastError();
      *w = nullptr;
    }
  }
  if (c->h_async_status && cudaHostGetDevicePointer(&c->h_async_status_dev, c->h_async_status, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeHost(c->h_async_status);
    c->h_async_status = nullptr;
  }
  if (c->h_status && cudaHostGetDevicePointer(&c->h_status_dev, c->h_status, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeHost(c->h_status);
    c->h_status = nullptr;
  }
  if (cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return LAPW1GPU_ERR_NOMEM;
  }
  cudaMemset(c->d_status, 0, sizeof(int));
  *out = c;
  return LAPW1GPU_OK;
}

int lapw1gpu_finalize(lapw1gpu_context* c) {
  if (!c) return LAPW1GPU_ERR_ARG;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (void* h : c->host_pinned) cudaHostUnregister(h);
  c->drop_graphs();
  for (auto& h : c->blas)
    if (h) cublasDestroy(h);
  if (c->solver) cusolverDnDestroy(c->solver);
  for (auto& kv : c->bufs)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  for (auto& kv : c->tiles) cudaFree(kv.second.first);
  if (c->async_pending && c->async_k) lapw1gpu_kpoint_free(c->async_k);
  if (c->h_async_status) cudaFreeHost(c->h_async_status);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->async_done) cudaEventDestroy(c->async_done);
  if (c->d_status) cudaFree(c->d_status);
  for (auto& e : c->ev) cudaEventDestroy(e);
  for (auto& e : c->fev) cudaEventDestroy(e);
  for (auto& e : c->fpev) cudaEventDestroy(e);
  cudaEventDestroy(c->fork);
  for (auto& e : c->hns_ev) cudaEventDestroy(e);
  for (auto& e : c->sph_ev) cudaEventDestroy(e);
  for (int i = 1; i < L1G_MAX_SETS; i++) {
    cudaEventDestroy(c->join[i]);
    cudaStreamDestroy(c->side[i]);
  }
  for (int i = 0; i < L1G_MAX_SETS; i++) {
    cudaEventDestroy(c->auxf[i]);
    cudaEventDestroy(c->auxj[i]);
    cudaStreamDestroy(c->aux[i]);
  }
  cudaStreamDestroy(c->stream);
  delete c;
  return LAPW1GPU_OK;
}

int lapw1gpu_set_precision(lapw1gpu_context* c, int prec, int slices) {
  if (!c) return LAPW1GPU_ERR_ARG;
  if (prec != LAPW1GPU_PREC_FP64 && prec != LAPW1GPU_PREC_SPLIT) return LAPW1GPU_ERR_ARG;
  if (prec == LAPW1GPU_PREC_SPLIT && (slices < 2 || slices > L1G_MAX_SLICES)) return LAPW1GPU_ERR_RANGE;
  c->prec = prec;
  if (prec == LAPW1GPU_PREC_SPLIT) c->slices = c->slices_hns = slices;
  return LAPW1GPU_OK;
}

int lapw1gpu_set_force_slices(lapw1gpu_context* c, int slices_density, int slices_projection) {
  if (!c) return LAPW1GPU_ERR_ARG;
  if (slices_density < 4 || slices_density > L1G_MAX_SLICES || slices_projection < 4 ||
      slices_projection > L1G_MAX_SLICES)
    return LAPW1GPU_ERR_RANGE;
  c->slices_frc = slices_density;
  c->slices_prj = slices_projection;
  return LAPW1GPU_OK;
}

int lapw1gpu_set_force_projection(lapw1gpu_context* c, int slices, int block_rows) {
  if (!c) return LAPW1GPU_ERR_ARG;
  if ((slices > 0 && (slices < 4 || slices > L1G_MAX_SLICES)) || slices < -1 || block_rows < 64 ||
      block_rows % SPH_T)
    return LAPW1GPU_ERR_RANGE;
  c->slices_fsp = slices;
  c->fsp_block = block_rows;
  return LAPW1GPU_OK;
}

int lapw1gpu_set_slices(lapw1gpu_context* c, int slices_sph, int slices_hns) {
  if (!c) return LAPW1GPU_ERR_ARG;
  if (slices_sph < 2 || slices_sph > L1G_MAX_SLICES || slices_hns < 2 || slices_hns > L1G_MAX_SLICES)
    return LAPW1GPU_ERR_RANGE;
  c->slices = slices_sph;
  c->slices_hns = slices_hns;
  return LAPW1GPU_OK;
}

void* lapw1gpu_stream(lapw1gpu_context* c) { return c ? (void*)c->stream : nullptr; }

int lapw1gpu_last_launches(lapw1gpu_context* c) { return c ? c->last_launches : 0; }

int lapw1gpu_forces_stats(lapw1gpu_context* c, lapw1gpu_stats* st) {
  if (!c || !st) return LAPW1GPU_ERR_ARG;
  memset(st, 0, sizeof(*st));
  st->ms_albl = c->fms[0];      // operands and the density matrices
  st->ms_spherical = c->fms[1] + c->fms[2];
  st->ms_sph_main = c->fms[2] - c->fms[5];  // k_force_sph
  st->ms_sph_slice = c->fms[6];               // the products of the spherical projections
  st->ms_table = c->fms[5] - c->fms[6];       // and their other kernels (operand, prefix, bins)
  st->ms_lo = c->fms[3];        // the step-function sums and the LO columns
  st->ms_hns = c->fms[4];       // the HNS part
  st->ms_total = c->fms[0] + c->fms[1] + c->fms[2] + c->fms[3] + c->fms[4];
  st->kernel_launches = c->last_launches;
  return LAPW1GPU_OK;
}

int lapw1gpu_host_register(lapw1gpu_context* c, void* ptr, size_t bytes) {
  if (!c || !ptr || bytes == 0) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  if (std::find(c->host_pinned.begin(), c->host_pinned.end(), ptr) != c->host_pinned.end()) return LAPW1GPU_OK;
  const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {  // the caller pinned it already: nothing to undo later
    cudaGetLastError();
    return LAPW1GPU_OK;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? LAPW1GPU_ERR_NOMEM : LAPW1GPU_ERR_CUDA;
  }
  c->host_pinned.push_back(ptr);
  return LAPW1GPU_OK;
}

int lapw1gpu_host_unregister(lapw1gpu_context* c, void* ptr) {
  if (!c || !ptr) return LAPW1GPU_ERR_ARG;
  auto it = std::find(c->host_pinned.begin(), c->host_pinned.end(), ptr);
  if (it == c->host_pinned.end()) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  c->host_pinned.erase(it);
  CK(cudaHostUnregister(ptr));
  return LAPW1GPU_OK;
}

int lapw1gpu_test_wait_timeout(lapw1gpu_context* c, int on) {
  if (!c || (on != 0 && on != 1)) return LAPW1GPU_ERR_ARG;
  c->test_never_wait = on;
  return LAPW1GPU_OK;
}

int lapw1gpu_last_status(lapw1gpu_context* c) {
  if (!c) return 0;
  if (c->status_pending) {  // the last run was asynchronous: wait for it and read its status
    int hstat = 0;
    if (cudaSetDevice(c->device) == cudaSuccess && read_status(c, c->stream, &hstat) == LAPW1GPU_OK)
      c->last_status = hstat;
    c->status_pending = false;
  }
  return c->last_status;
}

}  // extern "C"

static int kpoint_upload_impl(lapw1gpu_context* ctx, const lapw1gpu_problem* p, lapw1gpu_kpoint** out,
                              bool borrow) {
  if (!ctx || !out) return LAPW1GPU_ERR_ARG;
  *out = nullptr;
  int rc = validate(p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  lapw1gpu_kpoint* k = new lapw1gpu_kpoint();
  k->ctx = ctx;
  k->n = p->n;
  k->nv = p->nv;
  k->nlo = p->nlo;
  k->nat = p->nat;
  k->ndf = p->ndf;
  k->ltop = p->ltop;
  k->ldl = p->ldl;
  k->lnsmax = p->lnsmax;
  k->ins = p->ins;
  k->nohns = p->nohns;
  k->vi = p->vi;
  k->nvpad = round_up(p->nv, 64);
  k->npad = round_up(p->n, 64);
  k->mult.assign(p->mult, p->mult + p->nat);
  k->afirst.resize(p->nat);
  k->atype.resize(p->ndf);
  for (int a = 0, q = 0; a < p->nat; a++) {
    k->afirst[a] = q;
    for (int e = 0; e < p->mult[a]; e++) k->atype[q++] = a;
  }
  // difference-vector box of the PW rows and the WARP extents
  int kmin[3] = {1 << 30, 1 << 30, 1 << 30}, kmax[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
  for (int i = 0; i < p->nv; i++)
    for (int c = 0; c < 3; c++) {
      kmin[c] = std::min(kmin[c], p->kzz[3 * i + c]);
      kmax[c] = std::max(kmax[c], p->kzz[3 * i + c]);
    }
  k->tab.d1 = kmax[0] - kmin[0];
  k->tab.d2 = kmax[1] - kmin[1];
  k->tab.d3 = kmax[2] - kmin[2];
  k->tab.w1 = p->warp1;
  k->tab.w2 = p->warp2;
  k->tab.w3 = p->warp3;
  for (int q = 0; q < 9; q++) k->tab.bk[q] = p->bkzz[q];
  // LO columns in the order of hamilt.F:495-791 and LOHNS ranges
  {
    int nnlo = 0;
    for (int jn = 0; jn < p->nat; jn++) {
      double clr = 1.0, cli = 0.0;
      for (int l = 0; l <= L1G_LOMAX; l++) {
        int nil = p->ilo[jn * (L1G_LOMAX + 1) + l];
        for (int jlo = 1; jlo <= nil; jlo++) {
          LoRange r;
          r.jn = jn;
          r.l = l;
          r.jlo = jlo;
          r.i1 = nnlo + 1;
          for (int jeqo = 1; jeqo <= p->mult[jn]; jeqo++)
            for (int mo1 = -l; mo1 <= l; mo1++) {
              nnlo++;
              LoCol cc;
              cc.jn = jn;
              cc.l = l;
              cc.jlo = jlo;
              cc.jeqo = jeqo;
              cc.mo1 = mo1;
              cc.nnlo = nnlo;
              cc.a0 = k->afirst[jn];
              cc.clr = clr;
              cc.cli = cli;
              k->locols.push_back(cc);
            }
          r.i2 = nnlo;
          k->loranges.push_back(r);
        }
        double t = clr;
        clr = -cli;
        cli = t;
      }
    }
  }
  // HORB items in the reference's order (horb.F:98-113): atom type, then
  // equivalent atom, then l; pot(m2,m1) = vorb(iat,lvor,m1,m2)
  for (int i = 0; i < p->natorb; i++) {
    int jn = p->iatom[i] - 1;
    int pot0 = (int)(k->pots.size() / 49);
    for (int q = 0; q < p->nlorb[i]; q++) {
      int lv = p->lorb[i * 3 + q];
      std::vector<double2> pot(49, make_double2(0, 0));
      for (int m1 = -lv; m1 <= lv; m1++)
        for (int m2 = -lv; m2 <= lv; m2++) {
          size_t o = (((size_t)i * 4 + lv) * 7 + (m1 + 3)) * 7 + (m2 + 3);
          pot[(m2 + 3) * 7 + (m1 + 3)] = make_double2(p->vorb[2 * o], p->vorb[2 * o + 1]);
        }
      k->pots.insert(k->pots.end(), pot.begin(), pot.end());
    }
    for (int e = 0; e < p->mult[jn]; e++)
      for (int q = 0; q < p->nlorb[i]; q++) {
        lapw1gpu_kpoint::OrbItem it{k->afirst[jn] + e, p->lorb[i * 3 + q], pot0 + q};
        k->orbs.push_back(it);
      }
  }
  // one arena for all device inputs
  struct Seg {
    const void* src;
    size_t bytes;
    size_t off;
  };
  std::vector<Seg> segs;
  size_t off = 0;
  auto add = [&](const void* src, size_t bytes) -> size_t {
    size_t o = off;
    segs.push_back({src, bytes, o});
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const int nat = p->nat, ndf = p->ndf, n = p->n, ldl = p->ldl;
  const int L4 = L1G_LOMAX + 1;
  size_t o_mult = add(p->mult, sizeof(int) * nat);
  size_t o_atype = add(k->atype.data(), sizeof(int) * ndf);
  size_t o_afirst = add(k->afirst.data(), sizeof(int) * nat);
  size_t o_rmt = add(p->rmt, sizeof(double) * nat);
  size_t o_v = add(p->v, sizeof(double) * nat);
  size_t o_pos = add(p->pos, sizeof(double) * 3 * ndf);
  size_t o_rotij = add(p->rotij, sizeof(double) * 9 * ndf);
  size_t o_rotloc = add(p->rotloc, sizeof(double) * 9 * nat);
  size_t o_kzz = add(p->kzz, sizeof(int) * 3 * n);
  size_t o_xk = add(p->xk, sizeof(double) * n);
  size_t o_yk = add(p->yk, sizeof(double) * n);
  size_t o_zk = add(p->zk, sizeof(double) * n);
  size_t o_rk = add(p->rk, sizeof(double) * n);
  size_t o_p = add(p->p, sizeof(double) * nat * ldl);
  size_t o_pe = add(p->pe, sizeof(double) * nat * ldl);
  size_t o_dp = add(p->dp, sizeof(double) * nat * ldl);
  size_t o_dpe = add(p->dpe, sizeof(double) * nat * ldl);
  size_t o_pei = add(p->pei, sizeof(double) * nat * ldl);
  size_t o_e = add(p->e, sizeof(double) * nat * ldl);
  size_t o_lapw = add(p->lapw, sizeof(int) * nat * ldl);
  size_t o_ilo = add(p->ilo, sizeof(int) * nat * L4);
  size_t o_loor = add(p->loor, sizeof(int) * nat * L4);
  size_t o_alo = add(p->alo, sizeof(double) * nat * L1G_NLOAT * L4);
  size_t o_blo = add(p->blo, sizeof(double) * nat * L1G_NLOAT * L4);
  size_t o_clo = add(p->clo, sizeof(double) * nat * L1G_NLOAT * L4);
  size_t o_elo = add(p->elo, sizeof(double) * nat * L1G_NLOAT * L4);
  size_t o_pi12 = add(p->pi12lo, sizeof(double) * nat * L4);
  size_t o_pe12 = add(p->pe12lo, sizeof(double) * nat * L4);
  size_t o_dplo = add(p->dplo, sizeof(double) * nat * L4);
  size_t nwarp = (size_t)(2 * p->warp1 + 1) * (2 * p->warp2 + 1) * (2 * p->warp3 + 1);
  size_t o_warp = add(p->ins == 0 ? (const void*)p->warp : nullptr, p->ins == 0 ? sizeof(double2) * nwarp : 16);
  size_t ntns = (size_t)nat * LAPW1GPU_NTNS * L1G_NSL2 * L1G_NSL2;
  size_t o_tns = add(p->nohns ? nullptr : (const void*)p->tns, p->nohns ? 16 : sizeof(double2) * ntns);
  size_t o_locol = add(k->locols.data(), sizeof(LoCol) * std::max<size_t>(1, k->locols.size()));
  size_t o_lor = add(k->loranges.data(), sizeof(LoRange) * std::max<size_t>(1, k->loranges.size()));
  size_t o_pots = add(k->pots.data(), sizeof(double2) * std::max<size_t>(1, k->pots.size()));
  if (borrow) {
    // one-shot host entry point: reuse the context's grow-only arena
    k->arena = ctx->buf("arena", off);
    k->owns_arena = false;
    if (!k->arena) {
      delete k;
      return LAPW1GPU_ERR_NOMEM;
    }
  } else if (cudaMalloc(&k->arena, off) != cudaSuccess) {
    cudaGetLastError();
    delete k;
    return LAPW1GPU_ERR_NOMEM;
  }
  k->arena_bytes = off;
  char* base = (char*)k->arena;
  int crc = LAPW1GPU_OK;
  for (auto& s : segs)
    if (s.src && s.bytes && crc == LAPW1GPU_OK)
      if (cudaMemcpyAsync(base + s.off, s.src, s.bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        crc = LAPW1GPU_ERR_CUDA;
  if (crc == LAPW1GPU_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) crc = LAPW1GPU_ERR_CUDA;
  if (crc != LAPW1GPU_OK) {
    cudaGetLastError();
    if (k->owns_arena) cudaFree(k->arena);
    delete k;
    return crc;
  }
  DevProb& P = k->P;
  P.n = n;
  P.nv = p->nv;
  P.nlo = p->nlo;
  P.nat = nat;
  P.ndf = ndf;
  P.ltop = p->ltop;
  P.ldl = ldl;
  P.lnsmax = p->lnsmax;
  P.ins = p->ins;
  P.nvpad = k->nvpad;
  P.npad = k->npad;
  P.vi = p->vi;
#define SEGP(T, o) reinterpret_cast<T>(base + (o))
  P.mult = SEGP(const int*, o_mult);
  P.atype = SEGP(const int*, o_atype);
  P.afirst = SEGP(const int*, o_afirst);
  P.rmt = SEGP(const double*, o_rmt);
  P.v = SEGP(const double*, o_v);
  P.pos = SEGP(const double*, o_pos);
  P.rotij = SEGP(const double*, o_rotij);
  P.rotloc = SEGP(const double*, o_rotloc);
  P.kzz = SEGP(const int*, o_kzz);
  P.xk = SEGP(const double*, o_xk);
  P.yk = SEGP(const double*, o_yk);
  P.zk = SEGP(const double*, o_zk);
  P.rk = SEGP(const double*, o_rk);
  P.p = SEGP(const double*, o_p);
  P.pe = SEGP(const double*, o_pe);
  P.dp = SEGP(const double*, o_dp);
  P.dpe = SEGP(const double*, o_dpe);
  P.pei = SEGP(const double*, o_pei);
  P.e = SEGP(const double*, o_e);
  P.lapw = SEGP(const int*, o_lapw);
  P.ilo = SEGP(const int*, o_ilo);
  P.loor = SEGP(const int*, o_loor);
  P.alo = SEGP(const double*, o_alo);
  P.blo = SEGP(const double*, o_blo);
  P.clo = SEGP(const double*, o_clo);
  P.elo = SEGP(const double*, o_elo);
  P.pi12lo = SEGP(const double*, o_pi12);
  P.pe12lo = SEGP(const double*, o_pe12);
  P.dplo = SEGP(const double*, o_dplo);
  k->d_warp = SEGP(const double2*, o_warp);
  k->d_tns = SEGP(const double2*, o_tns);
  k->d_locols = SEGP(const LoCol*, o_locol);
  k->d_loranges = SEGP(const LoRange*, o_lor);
  k->d_pots = SEGP(const double2*, o_pots);
#undef SEGP
  *out = k;
  return LAPW1GPU_OK;
}

extern "C" {

int lapw1gpu_kpoint_upload(lapw1gpu_context* ctx, const lapw1gpu_problem* p, lapw1gpu_kpoint** out) {
  return kpoint_upload_impl(ctx, p, out, false);
}

int lapw1gpu_kpoint_free(lapw1gpu_kpoint* k) {
  if (!k) return LAPW1GPU_ERR_ARG;
  cudaSetDevice(k->ctx->device);
  if (k->arena && k->owns_arena) {
    cudaDeviceSynchronize();
    cudaFree(k->arena);
  }
  // captured batches that name this k-point are stale
  lapw1gpu_context* c = k->ctx;
  for (auto it = c->graphs.begin(); it != c->graphs.end();) {
    if (std::find(it->key.begin(), it->key.end(), (uintptr_t)k) != it->key.end()) {
      cudaGraphExecDestroy(it->exec);
      it = c->graphs.erase(it);
    } else {
      ++it;
    }
  }
  delete k;
  return LAPW1GPU_OK;
}

// tile list of the lower triangle in T x T tiles, rows outer (a prefix of
// the list for a larger n covers a smaller one)
static const int2* tiles_tri(lapw1gpu_kpoint* k, const char* name, int n, int T, int* count) {
  return kp_tiles(k, std::string(name) + ":" + std::to_string(n) + ":" + std::to_string(T), count,
                  [&](std::vector<int2>& t) {
                    const int nb = (n + T - 1) / T;
                    for (int bi = 0; bi < nb; bi++)
                      for (int bj = 0; bj <= bi; bj++) t.push_back(make_int2(bi, bj));
                  });
}

// HNS operands: R = {ALM, BLM} per row, L = M conj(R) per atom (k_hns_tmul),
// LO-row terms (k_hns_lo_ops).  Without Lop (the adjoint, which needs R and
// CLM only) L is not formed.
static int launch_hns_ops(lapw1gpu_context* c, const DevProb& P, const double2* tns, const LoRange* lor, int nlor,
                          double2* Lop, double2* Rop, double2* Clo, double2* C2lo, cudaStream_t s, int* nl) {
  const int nsl2 = (P.lnsmax + 1) * (P.lnsmax + 1);
  k_hns_alm<<<dim3((P.npad + 127) / 128, P.ndf), 128, 0, s>>>(P, lor, nlor, Rop, Clo);
  if (!Lop) {
    *nl += 1;
    return l1g_launch_status(__FILE__, __LINE__);
  }
  if (c ? !c->smem((const void*)k_hns_tmul, TMUL_SMEM)
        : cudaFuncSetAttribute(k_hns_tmul, cudaFuncAttributeMaxDynamicSharedMemorySize, TMUL_SMEM) != cudaSuccess)
    return LAPW1GPU_ERR_CUDA;
  // two blocks per SM over the (atom, 64-column) items, contiguous ranges
  const int nitem = (P.npad + TMUL_I - 1) / TMUL_I * P.ndf;
  const int nblk = std::max(1, std::min(nitem, 2 * (c ? c->nsm : 148)));
  const int per = (nitem + nblk - 1) / nblk;
  k_hns_tmul<<<(nitem + per - 1) / per, 32 * TMUL_WARPS, TMUL_SMEM, s>>>(P.npad, nsl2, P.ndf, per, P.atype, tns, Rop,
                                                                       Lop);
  *nl += 2;
  if (P.nlo > 0) {
    k_hns_lo_ops<<<dim3((P.nlo + LOOPS_ROWS - 1) / LOOPS_ROWS, P.ndf), dim3(32, 8), 0, s>>>(P, tns, Lop, Rop, Clo,
                                                                                           C2lo, 0);
    *nl += 1;
  }
  return l1g_launch_status(__FILE__, __LINE__);
}

// The FP64 HNS update in the blocked form of ZHER2M (zher2m.f:69-80):
// diagonal blocks of B rows run in k_hns_gemm (64-row tiles, lower triangle
// only), the rows below each diagonal block in one library ZGEMM per block
// column.  B is a tunable (lapw1gpu_autotune), 512 by default.
static const int2* tiles_hns_diag(lapw1gpu_kpoint* k, int n, int B, int* count) {
  return kp_tiles(k, "hnsdiag:" + std::to_string(n) + ":" + std::to_string(B), count, [&](std::vector<int2>& t) {
    const int per = B / HNS_T;
    const int nt = (n + HNS_T - 1) / HNS_T;
    for (int b0 = 0; b0 < nt; b0 += per)
      for (int bi = b0; bi < std::min(nt, b0 + per); bi++)
        for (int bj = b0; bj <= bi; bj++) t.push_back(make_int2(bi, bj));
  });
}

// (hp: after the panels of each column group, its event; groups whose
// columns reach the LO block are left for the caller to record)
static int hns_panels_zgemm(cublasHandle_t h, int n, int nv, int npad, int K, int B, const double2* Lop,
                            const double2* Rop, double2* hs, int ld, cudaStream_t s, HnsPipe* hp) {
  if (!h) return LAPW1GPU_ERR_CUDA;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  if (hp && hp->groups > 0 && !hp->fixed) {  // groups of whole panels
    const int np = (n + B - 1) / B, G = std::min(hp->groups, np);
    hp->groups = G;
    for (int g = 0; g <= G; g++) hp->col[g] = std::min(n, (int)((long)np * g / G) * B);
  }
  int g = 0;
  for (int c0 = 0; c0 < n; c0 += B) {
    const int w = std::min(B, n - c0);
    const int r0 = c0 + w, m = n - r0;
    // HS(r0:n, c0:c0+w) += L(r0:n, :) R(c0:c0+w, :)^T ; L, R column-major npad x K
    if (m > 0 && cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, m, w, K, &one, (const cuDoubleComplex*)(Lop + r0), npad,
                             (const cuDoubleComplex*)(Rop + c0), npad, &one,
                             (cuDoubleComplex*)(hs + (size_t)c0 * ld + r0), ld) != CUBLAS_STATUS_SUCCESS)
      return LAPW1GPU_ERR_CUDA;
    if (hp && g < hp->groups && r0 >= hp->col[g + 1]) {
      if (hp->col[g + 1] <= nv && cudaEventRecord(hp->ev[g], s) == cudaSuccess) hp->recorded[g] = true;
      g++;
    }
  }
  return LAPW1GPU_OK;
}

}  // extern "C"

// Spherical part on tcgen05 (sph_tc.cuh): slice the per-l operands, then
// one CTA per (128 J, IT I) tile of the triangle; KB bytes of K per stage.
template <int S, int LS, int KB>
static int sph_tc_launch(lapw1gpu_context* c, lapw1gpu_kpoint* k, int set, const DevProb& P, const SphCoef* coef,
                         const double2* tab, double2* hs, int ld, double2* hsdiag, cudaStream_t s, int* nl,
                         const cudaEvent_t* ev, HnsPipe* sp) {
  using Cf = sphtc::Cfg<S, KB>;
  const int nv = k->nv, L = k->ltop, Kc = 2 * k->ndf;
  // Kp: whole 32-byte MMA steps; the tensor map's K extent is Kp, so the
  // last KB-byte TMA block reads zero fill past it
  const int Kcp = round_up(Kc, 16), Kp = 2 * Kcp;
  const int npA = round_up(nv, 128), npB = round_up(nv, Cf::IT);
  int8_t* A = (int8_t*)c->sbuf(set, "sphA", (size_t)S * L * npA * Kp);
  int8_t* B = (int8_t*)c->sbuf(set, "sphB", (size_t)S * L * 4 * npB * Kp);
  int* exA = (int*)c->sbuf(set, "sphExA", sizeof(int) * (size_t)L * npA);
  int* exB = (int*)c->sbuf(set, "sphExB", sizeof(int) * (size_t)L * 2 * npB);
  if (!A || !B || !exA || !exB) return LAPW1GPU_ERR_NOMEM;
  const int sl_smem = Kc * 33 * (int)sizeof(double2);
  if (sl_smem > 200 * 1024) return LAPW1GPU_ERR_RANGE;
  if (!c->smem((const void*)sphtc::k_sph_slice<S>, sl_smem)) return LAPW1GPU_ERR_CUDA;
  if (ev && cudaEventRecord(c->ev[20], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
  if (int rc = l1g_launch_status(__FILE__, __LINE__)) return rc;
  sphtc::k_sph_slice<S><<<dim3(npA / 32, L), 256, sl_smem, s>>>(P, coef, 0, Kcp, npA, A, exA, c->d_status);
  if (int rc = l1g_launch_status(__FILE__, __LINE__)) return rc;
  sphtc::k_sph_slice<S><<<dim3((2 * npB + 31) / 32, L), 256, sl_smem, s>>>(P, coef, 1, Kcp, 2 * npB, B, exB,
                                                                           c->d_status);
  if (int rc = l1g_launch_status(__FILE__, __LINE__)) return rc;
  if (ev && cudaEventRecord(c->ev[21], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
  *nl += 2;
  CUtensorMap ta, tb;
  if (l1g_tmap_3d(&ta, A, Kp, (uint64_t)L * npA, S, 128, KB) ||
      l1g_tmap_3d(&tb, B, Kp, (uint64_t)L * 4 * npB, S, Cf::N, KB))
    return LAPW1GPU_ERR_CUDA;
  int ntile = 0;
  // I tiles outer: the CTAs resident at one time share few I tiles (B
  // operand, streamed from DRAM once) and sweep the J tiles (A operand,
  // 11 l x NV rows x S slices ~ 50 MB at NV = 4600, L2-resident)
  const int2* dt = kp_tiles(k, "sphtc:" + std::to_string(nv) + ":" + std::to_string(Cf::IT), &ntile,
                            [&](std::vector<int2>& t) {
                              const int nbj = npA / 128, nbi = npB / Cf::IT;
                              for (int bi = 0; bi < nbi; bi++)
                                for (int bj = 0; bj < nbj; bj++)
                                  if (bj * 128 <= bi * Cf::IT + Cf::IT - 1) t.push_back(make_int2(bj, bi));
                            });
  if (!dt) return LAPW1GPU_ERR_NOMEM;
  if (!c->smem((const void*)sphtc::k_sph_tc<S, LS, KB>, Cf::SMEM)) return LAPW1GPU_ERR_CUDA;
  if (ev && cudaEventRecord(ev[0], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
  // tiles are ordered by the I tile (column of S); per I tile bi the J tiles
  // bj with bj 128 <= bi IT + IT - 1, so a column group is a contiguous range
  const int nbj = npA / 128, nbi = npB / Cf::IT;
  auto first_tile = [&](int bi) {  // tiles before I tile bi
    long t = 0;
    for (int b = 0; b < bi; b++) t += std::min(nbj, (b * Cf::IT + Cf::IT - 1) / 128 + 1);
    return t;
  };
  const int G = sp ? sp->groups : 1;
  for (int g = 0; g < G; g++) {
    const int b0 = sp ? std::min(nbi, sp->col[g] / Cf::IT) : 0;
    const int b1 = sp ? (g == G - 1 ? nbi : std::min(nbi, sp->col[g + 1] / Cf::IT)) : nbi;
    const long t0 = first_tile(b0), t1 = (g == G - 1) ? ntile : first_tile(b1);
    if (t1 > t0) {
      // persistent: one CTA per SM over the group's tiles
      const int grid = (int)std::min<long>(t1 - t0, c->nsm);
      const int nkb = (Kp + KB - 1) / KB, klast = (Kp - (nkb - 1) * KB) / 32;
      sphtc::k_sph_tc<S, LS, KB><<<grid, Cf::THREADS, Cf::SMEM, s>>>(ta, tb, P, dt + t0, (int)(t1 - t0), nkb, klast,
                                                                      npA, npB, exA, exB, tab, k->tab, hs, ld, hsdiag,
                                                                      c->d_status, c->test_never_wait);
      const cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) {
        char what[160];
        snprintf(what, sizeof(what), "%s launching k_sph_tc<%d,%d,%d> grid %d block %d smem %d", cudaGetErrorName(le),
                 S, LS, KB, grid, Cf::THREADS, Cf::SMEM);
        l1g_note_error(what, (long)le, __FILE__, __LINE__);
        return LAPW1GPU_ERR_CUDA;
      }
      *nl += 1;
    }
    if (sp && sp->col[g + 1] <= k->nv) {
      if (cudaEventRecord(sp->sev[g], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
      sp->srec[g] = true;
    }
  }
  if (ev && cudaEventRecord(ev[1], s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;
  return l1g_launch_status(__FILE__, __LINE__);
}

// Exactness of the level sums (|slice| <= 64; level d sums d+1 products of
// at most 4096 per k): the int32 pairs c_d 128 + c_(d+1) hold while
// S 4096 Kp 128 + (S+1) 4096 Kp < 2^31, and the int64 combination
// V = sum_d c_d 2^(7(S-1-d)) converts with one add while |V| < 2^51.
// Returns the level-sum form of k_sph_tc: 2 int64, 1 int32 pairs, 0 plain.
static int sph_level_mode(int S, int Kp) {
  const double pair = (double)S * 4096.0 * Kp * 128.0 + (double)(S + 1) * 4096.0 * Kp;
  if (pair >= 2147483647.0) return 0;
  double v = 0.0;
  for (int d = 0; d < S; d++) v += (double)(d + 1) * 4096.0 * Kp * std::ldexp(1.0, 7 * (S - 1 - d));
  return v < std::ldexp(1.0, 51) ? 2 : 1;
}

// true when the split-precision spherical path handles this slice count
static bool sph_tc_supported(int S) { return S >= 4 && S <= 7; }

static int sph_tc_dispatch(lapw1gpu_context* c, lapw1gpu_kpoint* k, int set, const DevProb& P, const SphCoef* coef,
                           const double2* tab, double2* hs, int ld, double2* hsdiag, cudaStream_t s, int* nl,
                           const cudaEvent_t* ev, HnsPipe* sp) {
  const int Kp = 2 * round_up(2 * k->ndf, 16);
  const int mode = sph_level_mode(c->slices, Kp);
  // 128-byte K blocks fit two stages up to 5 slices
  const bool kb128 = c->sph_kb == 128 && c->slices <= 5;
#define SPH_MODES(SS, KB)                                                                             \
  return mode == 2   ? sph_tc_launch<SS, 2, KB>(c, k, set, P, coef, tab, hs, ld, hsdiag, s, nl, ev, sp) \
         : mode == 1 ? sph_tc_launch<SS, 1, KB>(c, k, set, P, coef, tab, hs, ld, hsdiag, s, nl, ev, sp) \
                     : sph_tc_launch<SS, 0, KB>(c, k, set, P, coef, tab, hs, ld, hsdiag, s, nl, ev, sp);
  switch (c->slices) {
    case 4:
      if (kb128) SPH_MODES(4, 128)
      SPH_MODES(4, 64)
    case 5:
      if (kb128) SPH_MODES(5, 128)
      SPH_MODES(5, 64)
    case 6:
      SPH_MODES(6, 64)
    case 7:
      SPH_MODES(7, 64)
    default:
      return LAPW1GPU_ERR_RANGE;
  }
#undef SPH_MODES
}

// algorithmic FP64-equivalent flops of the contractions
static double alg_flops(const lapw1gpu_kpoint* k) {
  double nv = k->nv, n = k->n;
  // spherical: per pair and atom type 6 FMA per l, 4 FMA per equivalent
  // atom's phase product, 4 FMA to add PHASE * t into S and H
  double sph = 2.0 * (6.0 * k->ltop * k->nat + 4.0 * k->ndf + 4.0 * k->nat) * (nv * (nv + 1) / 2.0);
  int nsl2 = (k->lnsmax + 1) * (k->lnsmax + 1);
  double hns = k->nohns ? 0.0 : 8.0 * (2.0 * k->ndf * nsl2) * (n * (n + 1) / 2.0);
  return sph + hns;
}

// The stage sequence of one k-point on stream s with scratch set `set`.
// ev: events to record between stages (null in a batch).  Host-side work
// is limited to launches: every buffer and tile list already exists when
// the same k-point ran once before, so the sequence can be captured.
static int kpoint_run_impl(lapw1gpu_context* c, lapw1gpu_kpoint* k, int stages, double2* d_hs, int ldhs,
                           double2* d_hsdiag, cudaStream_t s, int set, const cudaEvent_t* ev, int* nlaunch,
                           HnsPipe* hp = nullptr) {
  DevProb P = k->P;
  const int n = k->n, nv = k->nv, ltop = k->ltop, ndf = k->ndf, nat = k->nat;
  P.al = (double*)c->sbuf(set, "al", sizeof(double) * (size_t)nat * ltop * k->nvpad);
  P.bl = (double*)c->sbuf(set, "bl", sizeof(double) * (size_t)nat * ltop * k->nvpad);
  P.phase = (double2*)c->sbuf(set, "phase", sizeof(double2) * (size_t)ndf * k->npad);
  if (!P.al || !P.bl || !P.phase) return LAPW1GPU_ERR_NOMEM;
  if (ev) {
    // kernel events start equal, so a kernel that does not run reads 0
    for (int q = 12; q < 22; q++) CK(cudaEventRecord(ev[q], s));
    CK(cudaEventRecord(ev[0], s));
  }
  int nl = 0;  // kernels launched by this run

  // ---- K-a: matching coefficients and phases (always needed) ----
  nl++;
  if (ev) CK(cudaEventRecord(ev[16], s));
  k_albl<<<dim3((k->nvpad + 127) / 128, nat), 128, 0, s>>>(P, c->d_status);
  if (ev) CK(cudaEventRecord(ev[17], s));
  nl++;
  k_phase<<<dim3((k->npad + 127) / 128, ndf), 128, 0, s>>>(P);
  CK(cudaGetLastError());
  if (ev) CK(cudaEventRecord(ev[1], s));

  // HNS operand buffers; in split precision the operands (ALM/BLM/CLM, L,
  // the LO terms, row exponents and int8 slices) are prepared on the set's
  // auxiliary stream while the spherical stage runs on s: they read AL/BL
  // and the phases only.  s joins it before the HNS products.
  const bool hns = (stages & 2) && !k->nohns;
  const bool hns_fork = hns && c->prec == LAPW1GPU_PREC_SPLIT;
  const int nsl2 = (k->lnsmax + 1) * (k->lnsmax + 1);
  const int Khns = ndf * 2 * nsl2;
  double2 *Lop = nullptr, *Rop = nullptr, *Clo = nullptr, *C2lo = nullptr;
  if (hns) {
    Lop = (double2*)c->sbuf(set, "hnsL", sizeof(double2) * (size_t)Khns * k->npad);
    Rop = (double2*)c->sbuf(set, "hnsR", sizeof(double2) * (size_t)Khns * k->npad);
    size_t nloc = (size_t)ndf * nsl2 * std::max(1, k->nlo);
    Clo = (double2*)c->sbuf(set, "hnsClo", sizeof(double2) * nloc);
    C2lo = (double2*)c->sbuf(set, "hnsC2lo", sizeof(double2) * nloc);
    if (!Lop || !Rop || !Clo || !C2lo) return LAPW1GPU_ERR_NOMEM;
  }
  if (hns_fork) {
    // on the set's auxiliary stream: the operands, their int8 slices and
    // the LO-LO block T = C2 CLM^T (tensor cores, added after the HNS products)
    cudaStream_t a = c->aux[set];
    CK(cudaEventRecord(c->auxf[set], s));
    CK(cudaStreamWaitEvent(a, c->auxf[set], 0));
    int rc = launch_hns_ops(c, P, k->d_tns, k->d_loranges, (int)k->loranges.size(), Lop, Rop, Clo, C2lo, a, &nl);
    if (!rc)
      rc = split_hns_gemm(c, k, set, n, k->npad, Khns, Lop, Rop, d_hs, ldhs, c->slices_hns, a, &nl, nullptr,
                          nullptr, 0, 1);
    if (!rc && k->nlo > 0) {
      double2* T = (double2*)c->sbuf(set, "hnsLoT", sizeof(double2) * (size_t)k->nlo * k->nlo);
      if (!T) return LAPW1GPU_ERR_NOMEM;
      rc = split_rect_gemm(c, k, set, k->nlo, k->nlo, ndf * nsl2, C2lo, k->nlo, Clo, k->nlo, T, k->nlo,
                           c->slices_hns, a, &nl, 1, "lorect");
    }
    if (rc) return rc;
    CK(cudaEventRecord(c->auxj[set], a));
  }

  bool sph_tc_used = false;  // the spherical stage ran on the tensor-core kernel
  if (stages & 1) {
    // ---- K-c table + K-b spherical ----
    size_t ntab = (size_t)(2 * k->tab.d1 + 1) * (2 * k->tab.d2 + 1) * (2 * k->tab.d3 + 1);
    double2* tab = (double2*)c->sbuf(set, "tab", sizeof(double2) * 2 * ntab);
    SphCoef* coef = (SphCoef*)c->sbuf(set, "coef", sizeof(SphCoef) * nat * ltop);
    if (!tab || !coef) return LAPW1GPU_ERR_NOMEM;
    nl++;
    if (ev) CK(cudaEventRecord(ev[18], s));
    k_table<<<(unsigned)((ntab + 127) / 128), 128, 0, s>>>(P, k->tab, k->d_warp, tab);
    if (int rc = l1g_launch_status(__FILE__, __LINE__)) return rc;
    if (ev) CK(cudaEventRecord(ev[19], s));
    nl++;
    k_sph_coef<<<nat, 32, 0, s>>>(P, coef);
    if (int rc = l1g_launch_status(__FILE__, __LINE__)) return rc;
    // column groups of the spherical contraction (the caller's boundaries)
    HnsPipe* sp = (hp && hp->fixed && hp->groups > 0) ? hp : nullptr;
    if (c->prec == LAPW1GPU_PREC_SPLIT && c->sph_tc && sph_tc_supported(c->slices)) {
      int rc = sph_tc_dispatch(c, k, set, P, coef, tab, d_hs, ldhs, d_hsdiag, s, &nl, ev ? ev + 12 : nullptr, sp);
      if (rc) return rc;
      sph_tc_used = true;
    } else {
      int ntiles = 0;
      const int2* tl = tiles_tri(k, "sph", nv, SPH_T, &ntiles);
      if (!tl) return LAPW1GPU_ERR_NOMEM;
      if (!c->smem((const void*)k_spherical, SPH_DYN_SMEM)) return LAPW1GPU_ERR_CUDA;
      if (ev) CK(cudaEventRecord(ev[12], s));
      // tiles are ordered by the I tile (column of S), bi (bi + 1) / 2 before tile row bi
      const int nbi = (nv + SPH_T - 1) / SPH_T;
      const int G = sp ? sp->groups : 1;
      for (int g = 0; g < G; g++) {
        const int b0 = sp ? std::min(nbi, sp->col[g] / SPH_T) : 0;
        const int b1 = sp ? (g == G - 1 ? nbi : std::min(nbi, sp->col[g + 1] / SPH_T)) : nbi;
        const long t0 = (long)b0 * (b0 + 1) / 2, t1 = (long)b1 * (b1 + 1) / 2;
        if (t1 > t0) {
          nl++;
          k_spherical<<<(unsigned)(t1 - t0), SPH_THREADS, SPH_DYN_SMEM, s>>>(P, tl + t0, coef, tab, k->tab, d_hs,
                                                                             ldhs, d_hsdiag);
        }
        if (sp && sp->col[g + 1] <= nv) {
          CK(cudaEventRecord(sp->sev[g], s));
          sp->srec[g] = true;
        }
      }
      if (ev) CK(cudaEventRecord(ev[13], s));
    }
    CK(cudaGetLastError());
    if (ev) CK(cudaEventRecord(ev[2], s));
    // ---- K-b': local-orbital columns ----
    if (k->nlo > 0) {
      nl++;
      k_lo<<<dim3((n + 127) / 128, k->nlo), 128, 0, s>>>(P, k->d_locols, d_hs, ldhs, d_hsdiag, c->d_status);
    }
    CK(cudaGetLastError());
    if (sp)  // groups whose columns reach the LO columns are final after k_lo
      for (int g = 0; g < sp->groups; g++)
        if (!sp->srec[g]) {
          CK(cudaEventRecord(sp->sev[g], s));
          sp->srec[g] = true;
        }
    if (ev) CK(cudaEventRecord(ev[3], s));
  } else if (ev) {
    CK(cudaEventRecord(ev[2], s));
    CK(cudaEventRecord(ev[3], s));
  }

  if (hns) {
    // ---- K-ns ----
    const int K = Khns;
    int rc = LAPW1GPU_OK;
    if (hns_fork) {
      CK(cudaStreamWaitEvent(s, c->auxj[set], 0));
      rc = split_hns_gemm(c, k, set, n, k->npad, K, Lop, Rop, d_hs, ldhs, c->slices_hns, s, &nl, hp,
                          ev ? ev + 14 : nullptr, 0, 2);
    } else {
      rc = launch_hns_ops(c, P, k->d_tns, k->d_loranges, (int)k->loranges.size(), Lop, Rop, Clo, C2lo, s, &nl);
      if (rc) return rc;
      int ntiles = 0;
      const int2* tl = tiles_hns_diag(k, n, c->hns_diag_b, &ntiles);
      if (!tl) return LAPW1GPU_ERR_NOMEM;
      nl++;
      if (ev) CK(cudaEventRecord(ev[14], s));
      k_hns_gemm<<<ntiles, 256, 0, s>>>(n, k->npad, K, tl, Lop, Rop, d_hs, ldhs);
      rc = hns_panels_zgemm(c->handle(set, s), n, nv, k->npad, K, c->hns_diag_b, Lop, Rop, d_hs, ldhs, s, hp);
      if (ev && !rc) CK(cudaEventRecord(ev[15], s));
    }
    if (rc) return rc;
    if (k->nlo > 0) {
      nl++;
      // T = C2 CLM^T (nlo x nlo, K = NDF 25): in split precision from the
      // auxiliary stream's tensor-core product, else by library ZGEMM; its
      // lower triangle into HS
      double2* T = (double2*)c->sbuf(set, "hnsLoT", sizeof(double2) * (size_t)k->nlo * k->nlo);
      if (!T) return LAPW1GPU_ERR_NOMEM;
      if (!hns_fork) {
        cublasHandle_t h = c->handle(set, s);
        if (!h) return LAPW1GPU_ERR_NOMEM;
        const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
        if (cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, k->nlo, k->nlo, ndf * nsl2, &one, (const cuDoubleComplex*)C2lo,
                        k->nlo, (const cuDoubleComplex*)Clo, k->nlo, &zero, (cuDoubleComplex*)T,
                        k->nlo) != CUBLAS_STATUS_SUCCESS)
          return LAPW1GPU_ERR_CUDA;
      }
      k_add_lower<<<dim3((k->nlo + 127) / 128, k->nlo), 128, 0, s>>>(nv, k->nlo, T, d_hs, ldhs, c->d_status);
    }
    CK(cudaGetLastError());
    if (hp)  // the groups whose columns reach the LO block end here
      for (int g = 0; g < hp->groups; g++)
        if (!hp->recorded[g]) {
          CK(cudaEventRecord(hp->ev[g], s));
          hp->recorded[g] = true;
        }
  }
  if (ev) CK(cudaEventRecord(ev[4], s));

  if ((stages & 4) && !k->orbs.empty()) {
    double2* alm = (double2*)c->sbuf(set, "orb_alm", sizeof(double2) * 7 * (size_t)n);
    double2* blm = (double2*)c->sbuf(set, "orb_blm", sizeof(double2) * 7 * (size_t)n);
    double2* clm = (double2*)c->sbuf(set, "orb_clm", sizeof(double2) * 7 * (size_t)n);
    if (!alm || !blm || !clm) return LAPW1GPU_ERR_NOMEM;
    for (auto& it : k->orbs) {
      const double2* pot = k->d_pots + (size_t)it.iat * 49;
      nl++;
      k_horb_rows<<<(n + 127) / 128, 128, 0, s>>>(P, it.a, it.lvor, pot, k->d_loranges, (int)k->loranges.size(), alm,
                                                  blm, clm);
      nl++;
      k_horb_pairs<<<dim3((n + 127) / 128, n), 128, 0, s>>>(P, it.a, it.lvor, pot, k->d_loranges,
                                                           (int)k->loranges.size(), alm, blm, clm, d_hs, ldhs);
    }
    CK(cudaGetLastError());
  }
  if (ev) CK(cudaEventRecord(ev[5], s));
  // Non-finite elements: the split path's writers (k_sph_tc, k_lo, the
  // split HNS epilogue, k_add_lower) check what they write; the scan of HS
  // and HSDIAG is needed when the spherical stage did not run (HS came from
  // the caller), ran on the FP64 kernel, or HORB added to it.
  const bool checked = sph_tc_used && !((stages & 4) && !k->orbs.empty());
  if (!checked) {
    nl++;
    k_check_finite<<<1184, 256, 0, s>>>(n, d_hs, ldhs, d_hsdiag, c->d_status);
    CK(cudaGetLastError());
  }
  if (ev) CK(cudaEventRecord(ev[6], s));
  *nlaunch += nl;
  return LAPW1GPU_OK;
}

// per-stage timings from the events kpoint_run_impl recorded (ev[0..6])
static void fill_stats(lapw1gpu_context* c, const lapw1gpu_kpoint* k, int nl, lapw1gpu_stats* st) {
  float t[6];
  for (int q = 0; q < 6; q++) cudaEventElapsedTime(&t[q], c->ev[q], c->ev[q + 1]);
  memset(st, 0, sizeof(*st));
  st->ms_albl = t[0];
  st->ms_spherical = t[1];
  st->ms_lo = t[2];
  st->ms_hns = t[3];
  st->ms_horb = t[4];
  float tot;
  cudaEventElapsedTime(&tot, c->ev[0], c->ev[6]);
  st->ms_total = tot;
  st->flops_fp64_equiv = alg_flops(k);
  st->kernel_launches = nl;
  // main contraction kernels: events 12-13 and 14-15 (absent stages read 0)
  float a = 0.f, b = 0.f;
  if (cudaEventQuery(c->ev[13]) == cudaSuccess && cudaEventElapsedTime(&a, c->ev[12], c->ev[13]) == cudaSuccess)
    st->ms_sph_main = a;
  if (cudaEventQuery(c->ev[15]) == cudaSuccess && cudaEventElapsedTime(&b, c->ev[14], c->ev[15]) == cudaSuccess)
    st->ms_hns_main = b;
  float ka = 0.f, kt = 0.f, ks = 0.f;
  if (cudaEventElapsedTime(&ka, c->ev[16], c->ev[17]) == cudaSuccess) st->ms_k_albl = ka;
  if (cudaEventElapsedTime(&kt, c->ev[18], c->ev[19]) == cudaSuccess) st->ms_table = kt;
  if (cudaEventElapsedTime(&ks, c->ev[20], c->ev[21]) == cudaSuccess) st->ms_sph_slice = ks;
  cudaGetLastError();
}

extern "C" {

int lapw1gpu_kpoint_run(lapw1gpu_context* c, lapw1gpu_kpoint* k, int stages, double* d_hs_, int ldhs,
                        double* d_hsdiag_, lapw1gpu_stats* st) {
  if (!c || !k || !d_hs_ || !d_hsdiag_ || ldhs < k->n || k->ctx != c) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
  int nl = 0;
  int rc = kpoint_run_impl(c, k, stages, reinterpret_cast<double2*>(d_hs_), ldhs, reinterpret_cast<double2*>(d_hsdiag_),
                           s, 0, st ? c->ev : nullptr, &nl);
  if (rc) return rc;
  c->last_launches = nl;
  c->status_pending = !st;
  if (st) {
    int hstat = 0;
    if (int rc2 = read_status(c, s, &hstat, &nl)) return rc2;
    c->last_launches = nl;
    c->last_status = hstat;
    fill_stats(c, k, nl, st);
    if (hstat & L1G_STATUS_TIMEOUT) return LAPW1GPU_ERR_TIMEOUT;
    if (hstat & L1G_STATUS_NONFINITE) return LAPW1GPU_ERR_NONFINITE;
    if (hstat) return LAPW1GPU_ERR_RANGE;
  }
  return LAPW1GPU_OK;
}

// ---- k-point batches: one captured graph per argument set ----
static int batch_enqueue(lapw1gpu_context* c, lapw1gpu_kpoint* const* kps, int nk, int stages, double* const* d_hs,
                         const int* ldhs, double* const* d_hsdiag, int* nl) {
  const int sets = std::max(1, std::min(c->batch_sets, L1G_MAX_SETS));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), c->stream));
  CK(cudaEventRecord(c->fork, c->stream));
  for (int q = 1; q < sets; q++) CK(cudaStreamWaitEvent(c->side[q], c->fork, 0));
  for (int i = 0; i < nk; i++) {
    const int set = i % sets;
    cudaStream_t s = set ? c->side[set] : c->stream;
    int rc = kpoint_run_impl(c, kps[i], stages, reinterpret_cast<double2*>(d_hs[i]), ldhs[i],
                             reinterpret_cast<double2*>(d_hsdiag[i]), s, set, nullptr, nl);
    if (rc) return rc;
  }
  for (int q = 1; q < sets; q++) {
    CK(cudaEventRecord(c->join[q], c->side[q]));
    CK(cudaStreamWaitEvent(c->stream, c->join[q], 0));
  }
  return LAPW1GPU_OK;
}

int lapw1gpu_setup_batch(lapw1gpu_context* c, lapw1gpu_kpoint* const* kps, int nk, int stages, double* const* d_hs,
                         const int* ldhs, double* const* d_hsdiag, lapw1gpu_stats* st) {
  if (!c || !kps || nk < 1 || !d_hs || !ldhs || !d_hsdiag || !(stages & 1)) return LAPW1GPU_ERR_ARG;
  for (int i = 0; i < nk; i++)
    if (!kps[i] || kps[i]->ctx != c || !d_hs[i] || !d_hsdiag[i] || ldhs[i] < kps[i]->n) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  std::vector<uintptr_t> key = {(uintptr_t)nk,         (uintptr_t)stages,        (uintptr_t)c->prec,
                                (uintptr_t)(c->slices * 16 + c->slices_hns), (uintptr_t)c->hns_diag_b,
                                (uintptr_t)c->split_group,
                                (uintptr_t)c->sph_tc,  (uintptr_t)c->sph_kb, (uintptr_t)c->batch_sets,
                                (uintptr_t)c->test_never_wait};
  for (int i = 0; i < nk; i++) {
    key.push_back((uintptr_t)kps[i]);
    key.push_back((uintptr_t)d_hs[i]);
    key.push_back((uintptr_t)ldhs[i]);
    key.push_back((uintptr_t)d_hsdiag[i]);
  }
  lapw1gpu_context::Graph* g = nullptr;
  for (auto& x : c->graphs)
    if (x.key == key) g = &x;
  if (!g) {
    // one eager pass sizes every scratch buffer and builds every tile list,
    // so that the capture below performs no allocation or host copy
    int nl = 0;
    int rc = batch_enqueue(c, kps, nk, stages, d_hs, ldhs, d_hsdiag, &nl);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    nl = 0;
    rc = batch_enqueue(c, kps, nk, stages, d_hs, ldhs, d_hsdiag, &nl);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc || e != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return rc ? rc : LAPW1GPU_ERR_CUDA;
    }
    cudaGraphExec_t exec = nullptr;
    // the kernel nodes keep the priorities of the streams they were captured
    // from (chains high, the HNS operand streams low), so that the
    // persistent spherical kernel's CTAs are placed before the side work, as
    // in eager runs; a graph uses them only when instantiated with this flag
    e = cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return LAPW1GPU_ERR_CUDA;
    }
    c->graphs.push_back({key, exec, nl});
    g = &c->graphs.back();
  }
  const auto th0 = std::chrono::steady_clock::now();
  CK(cudaEventRecord(c->ev[0], c->stream));
  CK(cudaGraphLaunch(g->exec, c->stream));
  CK(cudaEventRecord(c->ev[6], c->stream));
  const double host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - th0).count();
  int hstat = 0;
  int nl = g->launches;
  if (int rc2 = read_status(c, c->stream, &hstat, &nl)) return rc2;
  c->last_status = hstat;
  c->status_pending = false;
  c->last_launches = nl;
  if (st) {
    memset(st, 0, sizeof(*st));
    float tot = 0.f;
    cudaEventElapsedTime(&tot, c->ev[0], c->ev[6]);
    st->ms_total = tot;
    for (int i = 0; i < nk; i++) st->flops_fp64_equiv += alg_flops(kps[i]);
    st->kernel_launches = nl;
    st->ms_host = host_ms;
  }
  // a timed-out wait leaves elements unwritten, which later finite checks see
  if (hstat & L1G_STATUS_TIMEOUT) return LAPW1GPU_ERR_TIMEOUT;
  if (hstat & L1G_STATUS_NONFINITE) return LAPW1GPU_ERR_NONFINITE;
  if (hstat) return LAPW1GPU_ERR_RANGE;
  return LAPW1GPU_OK;
}

int lapw1gpu_get_tuning(lapw1gpu_context* c, lapw1gpu_tuning* t) {
  if (!c || !t) return LAPW1GPU_ERR_ARG;
  t->hns_diag_b = c->hns_diag_b;
  t->split_group = c->split_group;
  t->sph_tc = c->sph_tc;
  t->batch_sets = c->batch_sets;
  t->sph_kblock = c->sph_kb;
  t->ms_best = 0.0;
  return LAPW1GPU_OK;
}

int lapw1gpu_set_tuning(lapw1gpu_context* c, const lapw1gpu_tuning* t) {
  if (!c || !t) return LAPW1GPU_ERR_ARG;
  if (t->hns_diag_b < HNS_T || t->hns_diag_b % HNS_T || t->split_group < 1 || t->batch_sets < 1 ||
      t->batch_sets > L1G_MAX_SETS || (t->sph_tc != 0 && t->sph_tc != 1) ||
      (t->sph_kblock != 64 && t->sph_kblock != 128))
    return LAPW1GPU_ERR_RANGE;
  c->hns_diag_b = t->hns_diag_b;
  c->split_group = t->split_group;
  c->sph_tc = t->sph_tc;
  c->batch_sets = t->batch_sets;
  c->sph_kb = t->sph_kblock;
  return LAPW1GPU_OK;
}

// Autotuner: the candidates of a tunable are timed on kp with the others
// held, tunables one after another; the fastest is kept if it beats the
// value held before by more than 2%.  Each candidate's
// time is its best of three runs, the runs of the candidates interleaved
// (round r runs every candidate once) so that a drift of the clocks over
// the tuning favours none of them, and it is the time of the kernel the
// tunable shapes where there is one (the spherical tensor-core kernel for
// its K block, the HNS products for their L2 grouping), else of the whole
// stage sequence (CUDA events).
int lapw1gpu_autotune(lapw1gpu_context* c, lapw1gpu_kpoint* kp, double* d_hs, int ldhs, double* d_hsdiag,
                      lapw1gpu_tuning* out) {
  if (!c || !kp || !d_hs || !d_hsdiag || ldhs < kp->n || kp->ctx != c) return LAPW1GPU_ERR_ARG;
  enum { T_TOTAL, T_SPH, T_HNS };
  auto tune = [&](int* knob, const std::vector<int>& cand, int what) -> int {
    const int v0 = *knob;
    std::vector<double> t(cand.size(), 1e30);
    for (int r = 0; r < 3; r++)
      for (size_t q = 0; q < cand.size(); q++) {
        *knob = cand[q];
        lapw1gpu_stats st;
        int rc = lapw1gpu_kpoint_run(c, kp, 7, d_hs, ldhs, d_hsdiag, &st);
        if (rc) {
          *knob = v0;
          return rc;
        }
        const double m = what == T_SPH ? st.ms_sph_main : what == T_HNS ? st.ms_hns_main : st.ms_total;
        t[q] = std::min(t[q], m > 0.0 ? m : st.ms_total);
      }
    size_t b = 0;
    for (size_t q = 1; q < cand.size(); q++)
      if (t[q] < t[b]) b = q;
    // the value held before tuning stays unless another beats it by more
    // than 2% (short timings of about a second in all drift by a few %)
    for (size_t q = 0; q < cand.size(); q++)
      if (cand[q] == v0 && t[b] > 0.98 * t[q]) b = q;
    *knob = cand[b];
    return LAPW1GPU_OK;
  };
  int rc = LAPW1GPU_OK;
  if (c->prec == LAPW1GPU_PREC_FP64) {
    rc = tune(&c->hns_diag_b, {256, 512, 1024, 2048}, T_TOTAL);
  } else {
    if (sph_tc_supported(c->slices)) rc = tune(&c->sph_tc, {1, 0}, T_TOTAL);
    // the K block (and with it the ring depth) of k_sph_tc: 128-byte blocks
    // exist up to 5 slices
    if (!rc && c->sph_tc && c->slices <= 5) rc = tune(&c->sph_kb, {64, 128}, T_SPH);
    if (!rc) rc = tune(&c->split_group, {4, 8, 16, 32}, T_HNS);
  }
  if (rc) return rc;
  // the setup time with the final choices
  double total_best = 1e30;
  for (int r = 0; r < 2 && !rc; r++) {
    lapw1gpu_stats st;
    rc = lapw1gpu_kpoint_run(c, kp, 7, d_hs, ldhs, d_hsdiag, &st);
    if (!rc) total_best = std::min(total_best, st.ms_total);
  }
  if (rc) return rc;
  if (out) {
    lapw1gpu_get_tuning(c, out);
    out->ms_best = total_best;
  }
  return LAPW1GPU_OK;
}

// Column widths of one tile of the spherical and HNS contractions under
// the context's settings (group boundaries must be multiples of both).
static int sph_granule(const lapw1gpu_context* c) {
  if (c->prec == LAPW1GPU_PREC_SPLIT && c->sph_tc && sph_tc_supported(c->slices)) switch (c->slices) {
      case 4: return sphtc::Cfg<4>::IT;
      case 5: return sphtc::Cfg<5>::IT;
      case 6: return sphtc::Cfg<6>::IT;
      default: return sphtc::Cfg<7>::IT;
    }
  return SPH_T;
}
static int hns_granule(const lapw1gpu_context* c) {
  if (c->prec != LAPW1GPU_PREC_SPLIT) return c->hns_diag_b;
  switch (c->slices_hns) {
    case 2: return split::Cfg<2>::JT;
    case 3: return split::Cfg<3>::JT;
    case 4: return split::Cfg<4>::JT;
    case 5: return split::Cfg<5>::JT;
    case 6: return split::Cfg<6>::JT;
    case 7: return split::Cfg<7>::JT;
    default: return split::Cfg<8>::JT;
  }
}

// Host-buffer form.  When HAMILT runs together with HNS/HORB, the copy of
// S back to the host overlaps them: S (the strict upper triangle) and
// HSDIAG are final once HAMILT is done, and the later stages only touch the
// lower triangle and the diagonal, so a copy stream takes, per panel of
// columns [c0, c0+w), the rows above c0 as soon as HAMILT ends; the rest of
// each panel follows the last stage.
#define L1G_D2H_PANEL 256
// The host-buffer setup.  async: return once everything is queued, the
// copies of HS/HSDIAG left running on the copy stream and the status word
// copied into page-locked memory behind the kernels (lapw1gpu_setup_wait
// ends it); else wait for all of it.
static int setup_host_impl(lapw1gpu_context* c, const lapw1gpu_problem* p, int stages, double* hs_, int ldhs,
                           double* hsdiag_, lapw1gpu_stats* st, bool async) {
  if (!c || !p || !hs_ || !hsdiag_ || ldhs < p->n) return LAPW1GPU_ERR_ARG;
  if (c->async_pending) return LAPW1GPU_ERR_ARG;  // one queued setup at a time
  if (async && !c->h_async_status) return LAPW1GPU_ERR_NOMEM;
  CK(cudaSetDevice(c->device));
  double2* hs = reinterpret_cast<double2*>(hs_);
  double2* hsdiag = reinterpret_cast<double2*>(hsdiag_);
  cudaEvent_t e0 = c->ev[7], e1 = c->ev[8], e2 = c->ev[9], e3 = c->ev[10], ecp = c->ev[11];
  cudaStream_t s = c->stream, cs = c->side[1];
  CK(cudaEventRecord(e0, s));
  lapw1gpu_kpoint* k = nullptr;
  int rc = kpoint_upload_impl(c, p, &k, true);
  if (rc) return rc;
  const int n = p->n;
  const size_t z = sizeof(double2);
  double2* d_hs = (double2*)c->buf("hs", z * (size_t)n * n);
  double2* d_hd = (double2*)c->buf("hsdiag", z * (size_t)n);
  if (!d_hs || !d_hd) {
    lapw1gpu_kpoint_free(k);
    return LAPW1GPU_ERR_NOMEM;
  }
  // stages that only add (HNS/HORB alone) start from the caller's HS
  if (!(stages & 1)) {
    cudaMemcpy2DAsync(d_hs, z * n, hs, z * ldhs, z * n, n, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_hd, hsdiag, z * n, cudaMemcpyHostToDevice, s);
  }
  CK(cudaEventRecord(e1, s));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
  int nl = 0;
  const bool overlap = (stages & 1) && (stages & 6);
  // HNS in column groups, so that the lower triangle follows group by group
  // (not with HORB, which adds to every column after HNS)
  HnsPipe hp;
  const bool pipe = overlap && (stages & 2) && !k->nohns && !((stages & 4) && !k->orbs.empty());
  if (pipe) {
    // about 8 groups of columns, boundaries on a multiple of both tile widths
    const int a = sph_granule(c), b = hns_granule(c);
    int gcd = a, r = b;
    while (r) {
      const int t = gcd % r;
      gcd = r;
      r = t;
    }
    const long gran = (long)a / gcd * b;
    int G = 0;
    hp.col[0] = 0;
    for (int g = 1; g < 8; g++) {
      const int cb = (int)(((long)n * g / 8) / gran * gran);
      if (cb > hp.col[G] && cb < n) hp.col[++G] = cb;
    }
    hp.col[++G] = n;
    hp.groups = G;
    hp.fixed = true;
  }
  for (int g = 0; g < L1G_MAX_GROUPS; g++) {
    hp.ev[g] = c->hns_ev[g];
    hp.sev[g] = c->sph_ev[g];
  }
  rc = kpoint_run_impl(c, k, stages, d_hs, n, d_hd, s, 0, c->ev, &nl, pipe ? &hp : nullptr);
  c->last_launches = nl;
  if (rc == LAPW1GPU_OK) {
    CK(cudaEventRecord(e2, s));
    bool grouped = pipe && hp.groups > 0 && hp.col[hp.groups] == n;
    for (int g = 0; grouped && g < hp.groups; g++) grouped = hp.recorded[g] && hp.srec[g];
    if (grouped) {
      // S above each group's columns as soon as the group's spherical tiles
      // (and, for the last groups, the LO columns) are done, HSDIAG after
      // HAMILT, then the rest of each group's columns after its HNS update
      for (int g = 0; g < hp.groups; g++) {
        const int a = hp.col[g], w = hp.col[g + 1] - a;
        CK(cudaStreamWaitEvent(cs, hp.sev[g], 0));
        if (a > 0 && w > 0 &&
            cudaMemcpy2DAsync(hs + (size_t)a * ldhs, z * ldhs, d_hs + (size_t)a * n, z * n, z * a, w,
                              cudaMemcpyDeviceToHost, cs) != cudaSuccess)
          rc = LAPW1GPU_ERR_CUDA;
      }
      CK(cudaStreamWaitEvent(cs, c->ev[3], 0));
      if (cudaMemcpyAsync(hsdiag, d_hd, z * n, cudaMemcpyDeviceToHost, cs) != cudaSuccess) rc = LAPW1GPU_ERR_CUDA;
      for (int g = 0; g < hp.groups; g++) {
        const int a = hp.col[g], w = hp.col[g + 1] - a;
        if (w <= 0) continue;
        CK(cudaStreamWaitEvent(cs, hp.ev[g], 0));
        if (cudaMemcpy2DAsync(hs + (size_t)a * ldhs + a, z * ldhs, d_hs + (size_t)a * n + a, z * n, z * (n - a), w,
                              cudaMemcpyDeviceToHost, cs) != cudaSuccess)
          rc = LAPW1GPU_ERR_CUDA;
      }
      CK(cudaEventRecord(ecp, cs));
      if (!async) CK(cudaStreamWaitEvent(s, ecp, 0));
    } else if (overlap) {
      // c->ev[3] marks the end of HAMILT (+ LO columns) on s
      CK(cudaStreamWaitEvent(cs, c->ev[3], 0));
      for (int c0 = L1G_D2H_PANEL; c0 < n; c0 += L1G_D2H_PANEL) {
        const int w = std::min(L1G_D2H_PANEL, n - c0);
        if (cudaMemcpy2DAsync(hs + (size_t)c0 * ldhs, z * ldhs, d_hs + (size_t)c0 * n, z * n, z * c0, w,
                              cudaMemcpyDeviceToHost, cs) != cudaSuccess)
          rc = LAPW1GPU_ERR_CUDA;
      }
      if (cudaMemcpyAsync(hsdiag, d_hd, z * n, cudaMemcpyDeviceToHost, cs) != cudaSuccess) rc = LAPW1GPU_ERR_CUDA;
      CK(cudaEventRecord(ecp, cs));
    }
    if (!grouped && !overlap) {
      if (cudaMemcpy2DAsync(hs, z * ldhs, d_hs, z * n, z * n, n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaMemcpyAsync(hsdiag, d_hd, z * n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = LAPW1GPU_ERR_CUDA;
    } else if (!grouped) {
      for (int c0 = 0; c0 < n; c0 += L1G_D2H_PANEL) {
        const int w = std::min(L1G_D2H_PANEL, n - c0);
        // rows [c0, n) of the panel (the first panel: all rows)
        const int r0 = c0;
        if (cudaMemcpy2DAsync(hs + (size_t)c0 * ldhs + r0, z * ldhs, d_hs + (size_t)c0 * n + r0, z * n, z * (n - r0),
                              w, cudaMemcpyDeviceToHost, s) != cudaSuccess)
          rc = LAPW1GPU_ERR_CUDA;
      }
      if (!async) CK(cudaStreamWaitEvent(s, ecp, 0));
    }
    if (async && rc == LAPW1GPU_OK) {
      CK(cudaEventRecord(e3, s));
      k_status_out<<<1, 1, 0, s>>>(c->d_status, c->h_async_status_dev);
      CK(cudaGetLastError());
      CK(cudaEventRecord(c->async_done, s));
      c->async_k = k;
      c->async_copies = grouped || overlap;
      c->async_nl = nl + 1;
      c->async_pending = true;
      return LAPW1GPU_OK;
    }
  }
  CK(cudaEventRecord(e3, s));
  int hstat = 0;
  if (read_status(c, s, &hstat, &nl) != LAPW1GPU_OK) rc = rc ? rc : LAPW1GPU_ERR_CUDA;
  c->last_launches = nl;
  c->last_status = hstat;
  c->status_pending = false;
  if (st && rc == LAPW1GPU_OK) {
    fill_stats(c, k, nl, st);
    float a, b;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e2, e3);
    st->ms_h2d = a;
    st->ms_d2h = b;  // the copies not hidden behind HNS/HORB
  }
  lapw1gpu_kpoint_free(k);
  if (rc) return rc;
  // a timed-out wait leaves elements unwritten, which later finite checks see
  if (hstat & L1G_STATUS_TIMEOUT) return LAPW1GPU_ERR_TIMEOUT;
  if (hstat & L1G_STATUS_NONFINITE) return LAPW1GPU_ERR_NONFINITE;
  if (hstat) return LAPW1GPU_ERR_RANGE;
  return LAPW1GPU_OK;
}

int lapw1gpu_setup_stages(lapw1gpu_context* c, const lapw1gpu_problem* p, int stages, double* hs, int ldhs,
                          double* hsdiag, lapw1gpu_stats* st) {
  return setup_host_impl(c, p, stages, hs, ldhs, hsdiag, st, false);
}

int lapw1gpu_setup_async(lapw1gpu_context* c, const lapw1gpu_problem* p, double* hs, int ldhs, double* hsdiag) {
  return setup_host_impl(c, p, 7, hs, ldhs, hsdiag, nullptr, true);
}

int lapw1gpu_setup_wait(lapw1gpu_context* c, lapw1gpu_stats* st) {
  if (!c || !c->async_pending) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  int rc = LAPW1GPU_OK;
  if (cudaEventSynchronize(c->async_done) != cudaSuccess) rc = LAPW1GPU_ERR_CUDA;
  if (c->async_copies && cudaEventSynchronize(c->ev[11]) != cudaSuccess) rc = LAPW1GPU_ERR_CUDA;
  if (rc) cudaGetLastError();
  const int hstat = *c->h_async_status;
  c->last_status = hstat;
  c->status_pending = false;
  c->last_launches = c->async_nl;
  if (st && rc == LAPW1GPU_OK) {
    fill_stats(c, c->async_k, c->async_nl, st);
    float a = 0.f;
    cudaEventElapsedTime(&a, c->ev[7], c->ev[8]);
    st->ms_h2d = a;
    st->ms_d2h = 0.0;  // the copies run behind later work on the copy stream
  }
  lapw1gpu_kpoint_free(c->async_k);
  c->async_k = nullptr;
  c->async_pending = false;
  if (rc) return rc;
  // a timed-out wait leaves elements unwritten, which later finite checks see
  if (hstat & L1G_STATUS_TIMEOUT) return LAPW1GPU_ERR_TIMEOUT;
  if (hstat & L1G_STATUS_NONFINITE) return LAPW1GPU_ERR_NONFINITE;
  if (hstat) return LAPW1GPU_ERR_RANGE;
  return LAPW1GPU_OK;
}

// hns.F:317-380 sums over LMSORT's grouping of the gaunt list
// (lmsort.f:246-421): entries sorted by (l0,m0,l',m',LM) with a stable
// insertion sort; a repeated tuple keeps the first gaunt factor only.
int lapw1gpu_tns_from_gaunt(int nat, int lnsmax, int ngau, int lmmx, const int* lqind, const int* lqns,
                            const double* gfac, const double* vns1, const double* vns2, const double* vns3,
                            const double* vnslo1, const double* vnslo2, const double* vnslo3, const int* loor,
                            double* tns) {
  if (nat < 1 || lnsmax < 0 || lnsmax > 4 || ngau < 0 || lmmx < 1 || !lqind || !lqns || !gfac || !vns1 || !vns2 ||
      !vns3 || !vnslo1 || !vnslo2 || !vnslo3 || !loor || !tns)
    return LAPW1GPU_ERR_ARG;
  const int K = L1G_NSL2, NS = LAPW1GPU_NSLMAX, NL = L1G_LOMAX + 1;
  memset(tns, 0, sizeof(double) * 2 * (size_t)nat * LAPW1GPU_NTNS * K * K);
  struct Ent {
    int l0, m0, lp, mp, lmx;
    double gr, gi;
  };
  std::vector<Ent> e;
  for (int ja = 0; ja < nat; ja++) {
    const int nq = lqind[ja];
    if (nq < 0 || nq > ngau) return LAPW1GPU_ERR_RANGE;
    e.clear();
    for (int i = 0; i < nq; i++) {
      const int* q = lqns + ((size_t)ja * ngau + i) * 6;
      Ent x{q[2] - 1, q[5], q[0] - 1, q[4], q[3], gfac[((size_t)ja * ngau + i) * 2],
            gfac[((size_t)ja * ngau + i) * 2 + 1]};
      auto before = [](const Ent& a, const Ent& b) {
        if (a.l0 != b.l0) return a.l0 < b.l0;
        if (a.m0 != b.m0) return a.m0 < b.m0;
        if (a.lp != b.lp) return a.lp < b.lp;
        if (a.mp != b.mp) return a.mp < b.mp;
        return a.lmx < b.lmx;
      };
      auto it = std::upper_bound(e.begin(), e.end(), x, before);  // stable: after equal keys
      e.insert(it, x);
    }
    double* T = tns + (size_t)ja * LAPW1GPU_NTNS * K * K * 2;
    for (size_t i = 0; i < e.size(); i++) {
      const Ent& x = e[i];
      if (i > 0) {
        const Ent& y = e[i - 1];
        if (x.l0 == y.l0 && x.m0 == y.m0 && x.lp == y.lp && x.mp == y.mp && x.lmx == y.lmx) continue;
      }
      const int lmx = x.lmx - 1;
      if (x.l0 < 0 || x.lp < 0 || x.l0 > lnsmax || x.lp > lnsmax || lmx < 0 || lmx >= lmmx) continue;
      if (abs(x.m0) > x.l0 || abs(x.mp) > x.lp) return LAPW1GPU_ERR_ARG;
      const int a = x.l0 * (x.l0 + 1) + x.m0, b = x.lp * (x.lp + 1) + x.mp;
      auto v3 = [&](const double* arr, int i1, int i3) { return arr[(((size_t)ja * NS + i3) * lmmx + lmx) * NS + i1]; };
      auto vlo = [&](const double* arr, int i1, int i3) { return arr[(((size_t)ja * NS + i3) * lmmx + lmx) * NL + i1]; };
      auto addt = [&](int blk, double val) {
        T[(((size_t)blk * K + a) * K + b) * 2] += x.gr * val;
        T[(((size_t)blk * K + a) * K + b) * 2 + 1] += x.gi * val;
      };
      addt(0, v3(vns1, x.lp, x.l0));  // TUU  VNS1(LP,LMX,L0)
      addt(1, v3(vns3, x.l0, x.lp));  // TDU  VNS3(L0,LMX,LP)
      addt(3, v3(vns3, x.lp, x.l0));  // TUD  VNS3(LP,LMX,L0)
      addt(4, v3(vns2, x.lp, x.l0));  // TDD  VNS2(LP,LMX,L0)
      bool loorl0 = false;
      if (x.l0 <= L1G_LOMAX) {
        loorl0 = loor[ja * NL + x.l0] != 0;
        if (loorl0) {
          addt(6, vlo(vnslo1, x.l0, x.lp));  // TUU12 VNS1LO(L0+1,LMX,LP+1)
          addt(7, vlo(vnslo2, x.l0, x.lp));  // TDU12 VNS2LO(L0+1,LMX,LP+1)
        }
      }
      if (x.lp <= L1G_LOMAX && loor[ja * NL + x.lp]) {
        if (loorl0) addt(8, vlo(vnslo3, x.lp, x.l0));  // TUU22 VNS3LO(LP+1,LMX,L0+1)
        addt(2, vlo(vnslo1, x.lp, x.l0));              // TUU21 VNS1LO(LP+1,LMX,L0+1)
        addt(5, vlo(vnslo2, x.lp, x.l0));              // TUD21 VNS2LO(LP+1,LMX,L0+1)
      }
    }
  }
  return LAPW1GPU_OK;
}

int lapw1gpu_setup(lapw1gpu_context* c, const lapw1gpu_problem* p, double* hs, int ldhs, double* hsdiag,
                   lapw1gpu_stats* st) {
  return lapw1gpu_setup_stages(c, p, 7, hs, ldhs, hsdiag, st);
}

// The adjoint of one k-point queued on the context's stream (no host
// synchronisation): status bits go to c->d_status, which the caller clears.
// timed: record the interval events of lapw1gpu_forces_stats.
static int forces_enqueue(lapw1gpu_context* c, lapw1gpu_kpoint* k, const double* d_c_, int ldc, int nb,
                          const double* d_occ, const double* d_eps, double* d_grad, bool timed, int* nl_out) {
  const double2* C = reinterpret_cast<const double2*>(d_c_);
  cudaStream_t s = c->stream;
  DevProb P = k->P;
  const int n = k->n, nv = k->nv, ltop = k->ltop, ndf = k->ndf, nat = k->nat, nlo = k->nlo;
  P.al = (double*)c->buf("al", sizeof(double) * (size_t)nat * ltop * k->nvpad);
  P.bl = (double*)c->buf("bl", sizeof(double) * (size_t)nat * ltop * k->nvpad);
  P.phase = (double2*)c->buf("phase", sizeof(double2) * (size_t)ndf * k->npad);
  double2* Cf = (double2*)c->buf("frc_cf", sizeof(double2) * (size_t)n * nb);
  double2* Ce = (double2*)c->buf("frc_ce", sizeof(double2) * (size_t)n * nb);
  double2* rho = (double2*)c->buf("frc_rho", sizeof(double2) * (size_t)n * n);
  double2* rhoe = (double2*)c->buf("frc_rhoe", sizeof(double2) * (size_t)n * n);
  SphCoef* coef = (SphCoef*)c->buf("coef", sizeof(SphCoef) * nat * ltop);
  if (!P.al || !P.bl || !P.phase || !Cf || !Ce || !rho || !rhoe || !coef) return LAPW1GPU_ERR_NOMEM;
  cublasHandle_t h = c->handle(0, s);
  if (!h) return LAPW1GPU_ERR_CUDA;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  int nlf = 0;  // kernels launched (a library product counts as one)
  if (timed) CK(cudaEventRecord(c->fev[0], s));
  CK(cudaMemsetAsync(d_grad, 0, sizeof(double) * 3 * ndf, s));
  k_albl<<<dim3((k->nvpad + 127) / 128, nat), 128, 0, s>>>(P, c->d_status);
  k_phase<<<dim3((k->npad + 127) / 128, ndf), 128, 0, s>>>(P);
  k_sph_coef<<<nat, 32, 0, s>>>(P, coef);
  const bool split_rho = c->prec == LAPW1GPU_PREC_SPLIT;
  k_force_weight<<<dim3((n + 127) / 128, nb), 128, 0, s>>>(n, nb, C, ldc, d_occ, d_eps, split_rho ? 1 : 0, Cf, Ce);
  nlf += 4;  // k_albl, k_phase, k_sph_coef, k_force_weight
  CK(cudaGetLastError());
  // rho(J,I) = sum_b f_b c_b(J) conj(c_b(I)), column-major n x n, and rhoE:
  // Hermitian, and only J < I is read.  FP64: the library forms the upper
  // triangle alone (half the flops of a full product).  Split precision:
  // the int8 slice-product kernel of the HNS update forms the lower
  // triangle of C X^T with X = conj(Cf) (k_force_weight conjugated it), i.e.
  // conj(rho(J,I)) at (I, J) (rt = 1 below).
  int rt = 0;
  if (split_rho) {
    const double2* Cn = C;
    if (ldc != n) {  // the operand kernels take one row stride for both sides
      double2* Cc = (double2*)c->buf("frc_c", sizeof(double2) * (size_t)n * nb);
      if (!Cc) return LAPW1GPU_ERR_NOMEM;
      CK(cudaMemcpy2DAsync(Cc, sizeof(double2) * n, C, sizeof(double2) * ldc, sizeof(double2) * n, nb,
                           cudaMemcpyDeviceToDevice, s));
      Cn = Cc;
    }
    // written, not added (no zero fill): every lower-triangle element the
    // force kernels read is a product tile's element
    int nlr = 0;
    int rc = split_hns_gemm(c, k, 0, n, n, nb, Cn, Cf, rho, n, c->slices_frc, s, &nlr, nullptr, nullptr, 0, 3, 1);
    if (!rc)
      rc = split_hns_gemm(c, k, 0, n, n, nb, Cn, Ce, rhoe, n, c->slices_frc, s, &nlr, nullptr, nullptr, 0, 3, 1);
    if (rc) return rc;
    nlf += nlr;
    rt = 1;
  } else {
    const double rzero = 0.0;
    if (cublasZherkx(h, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, n, nb, &one, (const cuDoubleComplex*)Cf, n,
                     (const cuDoubleComplex*)C, ldc, &rzero, (cuDoubleComplex*)rho, n) != CUBLAS_STATUS_SUCCESS ||
        cublasZherkx(h, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, n, nb, &one, (const cuDoubleComplex*)Ce, n,
                     (const cuDoubleComplex*)C, ldc, &rzero, (cuDoubleComplex*)rhoe, n) != CUBLAS_STATUS_SUCCESS)
      return LAPW1GPU_ERR_CUDA;
    nlf += 2;
  }
  if (timed) CK(cudaEventRecord(c->fev[1], s));
  // G c (k_force_gscale) and, in split precision, its k-major copy (G c)^T:
  // the right operand of the spherical and of the HNS projections
  double2* GC = nullptr;
  double2* Gt = nullptr;
  auto make_gc = [&](bool with_gt) -> int {
    if (!GC) {
      GC = (double2*)c->buf("frc_gc", sizeof(double2) * (size_t)4 * nb * n);
      if (!GC) return LAPW1GPU_ERR_NOMEM;
      k_force_gscale<<<dim3((n + 127) / 128, nb), 128, 0, s>>>(n, nb, P.kzz, C, ldc, GC);
      nlf++;
    }
    if (with_gt && !Gt) {
      Gt = (double2*)c->buf("frc_gt", sizeof(double2) * (size_t)n * 4 * nb);
      if (!Gt) return LAPW1GPU_ERR_NOMEM;
      k_force_trans<<<dim3((n + 31) / 32, (4 * nb + 31) / 32), 256, 0, s>>>(GC, n, 4 * nb, n, 0, Gt, 4 * nb);
      nlf++;
    }
    return l1g_launch_status(__FILE__, __LINE__);
  };
  // split precision: the spherical pairs of two different row blocks as
  // projections (forces.cuh), the pairs inside a block on k_force_sph
  const int fB = c->fsp_block;
  const int fS = c->slices_fsp < 0 ? L1G_FSP_SLICES : c->slices_fsp;
  const bool fproj = split_rho && fS > 0 && nv > fB && (c->slices_fsp > 0 || nv >= L1G_FSP_MIN_BLOCKS * fB);
  if (timed) {
    c->fproj_last = fproj;
    c->fpev_used = 0;
  }
  int ntiles = 0;
  const int2* tl = nullptr;
  if (fproj) {
    tl = kp_tiles(k, "fsp_in:" + std::to_string(nv) + ":" + std::to_string(fB), &ntiles, [&](std::vector<int2>& t) {
      const int nt = (nv + SPH_T - 1) / SPH_T;
      for (int bi = 0; bi < nt; bi++)
        for (int bj = 0; bj <= bi; bj++)
          if ((bi * SPH_T) / fB == (bj * SPH_T) / fB) t.push_back(make_int2(bi, bj));
    });
  } else {
    tl = tiles_tri(k, "sph", nv, SPH_T, &ntiles);
  }
  if (!tl) return LAPW1GPU_ERR_NOMEM;
  const size_t nrow = (size_t)nat * ltop * k->nvpad;
  double2* rowJ = (double2*)c->buf("frc_rowj", sizeof(double2) * nrow);
  double2* rowI = (double2*)c->buf("frc_rowi", 2 * sizeof(double2) * nrow);
  if (!rowJ || !rowI) return LAPW1GPU_ERR_NOMEM;
  k_force_rows<<<dim3((k->nvpad + 127) / 128, nat * ltop), 128, 0, s>>>(P, coef, rowJ, rowI);
  nlf += 3;  // k_force_rows, k_force_sph, k_force_step
  const bool lt11 = ltop == FRC_LT;
  const void* fsph = lt11 ? (const void*)k_force_sph<FRC_LT, false> : (const void*)k_force_sph<SPH_LMAX, true>;
  const int fsmem = frc_smem_bytes(lt11 ? FRC_LT : SPH_LMAX);
  if (!c->smem(fsph, fsmem)) return LAPW1GPU_ERR_CUDA;
  const size_t nbox = (size_t)(2 * k->tab.d1 + 1) * (2 * k->tab.d2 + 1) * (2 * k->tab.d3 + 1);
  double* bins = (double*)c->buf("frc_bins", sizeof(double) * 2 * nbox);
  if (!bins) return LAPW1GPU_ERR_NOMEM;
  CK(cudaMemsetAsync(bins, 0, sizeof(double) * 2 * nbox, s));
  if (timed) CK(cudaEventRecord(c->fev[2], s));
  if (fproj) {
    const int L2 = ltop * ltop, Ks = ndf * 2 * L2, nblk = (nv + fB - 1) / fB;
    double2* Ls = (double2*)c->buf("frc_ls", sizeof(double2) * (size_t)nv * Ks);
    double2* Pre = (double2*)c->buf("frc_pre", sizeof(double2) * (size_t)Ks * 4 * nb);
    double2* Yp = (double2*)c->buf("frc_yp", sizeof(double2) * (size_t)Ks * 4 * nb);
    if (!Ls || !Pre || !Yp) return LAPW1GPU_ERR_NOMEM;
    if (int rc = make_gc(true)) return rc;
    k_force_rsph<<<nv, 256, 0, s>>>(P, Ls, Ks);
    nlf++;
    for (int pb = 0; pb < nblk; pb++) {
      const int r0 = pb * fB, kc = std::min(fB, nv - r0);
      int nly = 0;
      if (timed) {
        while ((int)c->fpev.size() < 2 * (pb + 1)) {
          cudaEvent_t e;
          CK(cudaEventCreate(&e));
          c->fpev.push_back(e);
        }
        CK(cudaEventRecord(c->fpev[2 * pb], s));
      }
      // block 0 is the first prefix; later blocks are contracted with it
      int rc = split_rect_gemm(c, k, 0, Ks, 4 * nb, kc, Ls + (size_t)r0 * Ks, Ks, Gt + (size_t)r0 * 4 * nb, 4 * nb,
                               pb == 0 ? Pre : Yp, Ks, fS, s, &nly, 1, "fsp");
      if (rc) return rc;
      if (timed) {
        CK(cudaEventRecord(c->fpev[2 * pb + 1], s));
        c->fpev_used = 2 * (pb + 1);
      }
      nlf += nly;
      if (pb > 0) {
        k_force_pre<<<dim3(ndf, (nb + FRC_PB - 1) / FRC_PB), 128, 0, s>>>(P, coef, Yp, Pre, Ks, nb, d_occ, d_eps,
                                                                          pb + 1 < nblk ? 1 : 0, d_grad);
        nlf++;
      }
    }
    int nto = 0;
    const int2* to = kp_tiles(k, "fsp_out:" + std::to_string(nv) + ":" + std::to_string(fB), &nto,
                              [&](std::vector<int2>& t) {
                                const int nt = (nv + SPH_T - 1) / SPH_T;
                                for (int bi = 0; bi < nt; bi++)
                                  for (int bj = 0; bj <= bi; bj++)
                                    if ((bi * SPH_T) / fB != (bj * SPH_T) / fB) t.push_back(make_int2(bi, bj));
                              });
    if (!to) return LAPW1GPU_ERR_NOMEM;
    k_force_bins<<<nto, FRC_THREADS, 0, s>>>(P, to, k->tab, rho, rhoe, n, rt, bins);
    nlf++;
    CK(cudaGetLastError());
    if (timed) CK(cudaEventRecord(c->fev[6], s));
  }
  if (lt11)
    k_force_sph<FRC_LT, false><<<ntiles, FRC_THREADS, fsmem, s>>>(P, tl, rowJ, rowI, k->tab, rho, rhoe, n, rt,
                                                                  d_grad, bins);
  else
    k_force_sph<SPH_LMAX, true><<<ntiles, FRC_THREADS, fsmem, s>>>(P, tl, rowJ, rowI, k->tab, rho, rhoe, n, rt,
                                                                   d_grad, bins);
  if (timed) CK(cudaEventRecord(c->fev[3], s));
  k_force_step<<<ndf, 256, 0, s>>>(P, k->tab, bins, d_grad);
  CK(cudaGetLastError());
  if (nlo > 0) {
    k_force_lo<<<dim3((n + 127) / 128, nlo), 128, 0, s>>>(P, k->d_locols, rho, rhoe, n, rt, d_grad);
    nlf++;
  }
  if (timed) CK(cudaEventRecord(c->fev[4], s));
  CK(cudaGetLastError());
  if (!k->nohns) {
    const int nsl2 = (k->lnsmax + 1) * (k->lnsmax + 1);
    const int K = ndf * 2 * nsl2, Kc = ndf * nsl2;
    double2* Rop = (double2*)c->buf("hnsR", sizeof(double2) * (size_t)K * k->npad);
    size_t nloc = (size_t)Kc * std::max(1, nlo);
    double2* Clo = (double2*)c->buf("hnsClo", sizeof(double2) * nloc);
    double2* Y = (double2*)c->buf("frc_y", sizeof(double2) * (size_t)4 * nb * K);
    double2* Z = (double2*)c->buf("frc_z", sizeof(double2) * (size_t)4 * nb * K);
    if (!Rop || !Clo || !Y || !Z) return LAPW1GPU_ERR_NOMEM;
    int nl = 0;
    // R and CLM only: the adjoint applies T to Y = R^H (G c), not L = M conj(R)
    int rc = launch_hns_ops(c, P, k->d_tns, k->d_loranges, (int)k->loranges.size(), nullptr, Rop, Clo, nullptr, s,
                            &nl);
    if (rc) return rc;
    nlf += nl;
    if ((rc = make_gc(split_rho))) return rc;
    // Y = R^H (G c): K x 4nb (rows of R beyond n unused); Yc = CLM^H (G c)
    // over the LO rows; Z = T (Y; Yc) per atom.  Split precision: Y and Yc
    // as int8 slice products, from k-major copies conj(R)^T, conj(CLM)^T
    // and (G c)^T
    if (split_rho) {
      double2* Lt = (double2*)c->buf("frc_rt", sizeof(double2) * (size_t)n * K);
      if (!Lt) return LAPW1GPU_ERR_NOMEM;
      k_force_trans<<<dim3((n + 31) / 32, (K + 31) / 32), 256, 0, s>>>(Rop, k->npad, K, n, 1, Lt, K);
      int nly = 0;
      rc = split_rect_gemm(c, k, 0, K, 4 * nb, n, Lt, K, Gt, 4 * nb, Y, K, c->slices_prj, s, &nly, 1);
      if (rc) return rc;
      nlf += nly + 1;
    } else if (cublasZgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, K, 4 * nb, n, &one, (const cuDoubleComplex*)Rop, k->npad,
                           (const cuDoubleComplex*)GC, n, &zero, (cuDoubleComplex*)Y, K) != CUBLAS_STATUS_SUCCESS) {
      return LAPW1GPU_ERR_CUDA;
    } else {
      nlf++;
    }
    double2* Yc = nullptr;
    double2* Zc = nullptr;
    if (nlo > 0) {
      Yc = (double2*)c->buf("frc_yc", sizeof(double2) * (size_t)4 * nb * Kc);
      Zc = (double2*)c->buf("frc_zc", sizeof(double2) * (size_t)4 * nb * Kc);
      if (!Yc || !Zc) return LAPW1GPU_ERR_NOMEM;
      if (split_rho) {  // the LO rows of (G c)^T follow its PW rows in Gt
        double2* Lc = (double2*)c->buf("frc_lc", sizeof(double2) * (size_t)nlo * Kc);
        if (!Lc) return LAPW1GPU_ERR_NOMEM;
        k_force_trans<<<dim3((nlo + 31) / 32, (Kc + 31) / 32), 256, 0, s>>>(Clo, nlo, Kc, nlo, 1, Lc, Kc);
        int nly = 0;
        rc = split_rect_gemm(c, k, 0, Kc, 4 * nb, nlo, Lc, Kc, Gt + (size_t)nv * 4 * nb, 4 * nb, Yc, Kc, c->slices_prj, s,
                             &nly, 1);
        if (rc) return rc;
        nlf += nly + 1;
      } else if (cublasZgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, Kc, 4 * nb, nlo, &one, (const cuDoubleComplex*)Clo, nlo,
                             (const cuDoubleComplex*)(GC + nv), n, &zero, (cuDoubleComplex*)Yc,
                             Kc) != CUBLAS_STATUS_SUCCESS) {
        return LAPW1GPU_ERR_CUDA;
      } else {
        nlf++;
      }
    }
    if (!c->smem((const void*)k_force_hns_z, FRC_ZSMEM)) return LAPW1GPU_ERR_CUDA;
    const dim3 zgrid((4 * nb + FRC_ZCOLS - 1) / FRC_ZCOLS, ndf);
    k_force_hns_z<<<zgrid, 256, FRC_ZSMEM, s>>>(0, nsl2, K, Kc, 4 * nb, P.atype, k->d_tns, Y, Yc, Z, nullptr);
    k_force_hns_reduce<<<ndf, 256, 0, s>>>(2 * nsl2, K, nb, Y, Z, d_occ, d_grad);
    nlf += 2;
    CK(cudaGetLastError());
    if (nlo > 0) {
      k_force_hns_z<<<zgrid, 256, FRC_ZSMEM, s>>>(1, nsl2, K, Kc, 4 * nb, P.atype, k->d_tns, Y, Yc, nullptr, Zc);
      k_force_hns_reduce<<<ndf, 256, 0, s>>>(nsl2, Kc, nb, Yc, Zc, d_occ, d_grad);
      nlf += 2;
      CK(cudaGetLastError());
    }
  }
  if (timed) CK(cudaEventRecord(c->fev[5], s));
  *nl_out += nlf;
  return LAPW1GPU_OK;
}

static int forces_check(lapw1gpu_context* c, lapw1gpu_kpoint* k, const double* d_c, int ldc, int nb,
                        const double* d_occ, const double* d_eps, const double* d_grad) {
  if (!c || !k || k->ctx != c || !d_c || !d_occ || !d_eps || !d_grad || nb < 1 || ldc < k->n)
    return LAPW1GPU_ERR_ARG;
  if (!k->orbs.empty()) return LAPW1GPU_ERR_ARG;
  return LAPW1GPU_OK;
}

// Band-energy gradient (forces.cuh): rho = C f C^H and rhoE = C f eps C^H by
// library ZGEMM, the PW x PW and LO parts by k_force_sph / k_force_lo, the
// HNS part through its factors (four ZGEMMs and a per-atom reduction).
int lapw1gpu_forces(lapw1gpu_context* c, lapw1gpu_kpoint* k, const double* d_c, int ldc, int nb, const double* d_occ,
                    const double* d_eps, double* d_grad) {
  int rc = forces_check(c, k, d_c, ldc, nb, d_occ, d_eps, d_grad);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
  int nl = 0;
  rc = forces_enqueue(c, k, d_c, ldc, nb, d_occ, d_eps, d_grad, true, &nl);
  if (rc) return rc;
  int hstat = 0;
  if (int rc2 = read_status(c, s, &hstat, &nl)) return rc2;
  c->last_status = hstat;
  c->status_pending = false;
  c->last_launches = nl;
  for (int q = 0; q < 5; q++) cudaEventElapsedTime(&c->fms[q], c->fev[q], c->fev[q + 1]);
  c->fms[5] = c->fms[6] = 0.f;
  if (c->fproj_last) {
    cudaEventElapsedTime(&c->fms[5], c->fev[2], c->fev[6]);
    for (int q = 0; q + 1 < c->fpev_used; q += 2) {
      float t = 0.f;
      cudaEventElapsedTime(&t, c->fpev[q], c->fpev[q + 1]);
      c->fms[6] += t;
    }
  }
  cudaGetLastError();
  return hstat ? LAPW1GPU_ERR_RANGE : LAPW1GPU_OK;
}

// The adjoint of a k-point list queued back to back on the context's stream
// (one host synchronisation and status read at the end), the companion of
// lapw1gpu_setup_batch.
int lapw1gpu_forces_batch(lapw1gpu_context* c, lapw1gpu_kpoint* const* kps, int nk, const double* const* d_c,
                          const int* ldc, int nb, const double* d_occ, const double* const* d_eps,
                          double* const* d_grad, double* ms_total) {
  if (!c || !kps || nk < 1 || !d_c || !ldc || !d_eps || !d_grad) return LAPW1GPU_ERR_ARG;
  for (int i = 0; i < nk; i++) {
    const int rc = forces_check(c, kps[i], d_c[i], ldc[i], nb, d_occ, d_eps[i], d_grad[i]);
    if (rc) return rc;
  }
  CK(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  CK(cudaEventRecord(c->ev[0], s));
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
  int nl = 0;
  for (int i = 0; i < nk; i++) {
    const int rc = forces_enqueue(c, kps[i], d_c[i], ldc[i], nb, d_occ, d_eps[i], d_grad[i], false, &nl);
    if (rc) return rc;
  }
  CK(cudaEventRecord(c->ev[6], s));
  int hstat = 0;
  if (int rc2 = read_status(c, s, &hstat, &nl)) return rc2;
  c->last_status = hstat;
  c->status_pending = false;
  c->last_launches = nl;
  if (ms_total) {
    float t = 0.f;
    cudaEventElapsedTime(&t, c->ev[0], c->ev[6]);
    *ms_total = t;
  }
  return hstat ? LAPW1GPU_ERR_RANGE : LAPW1GPU_OK;
}

}  // extern "C"

// SECLR4 on the device (seclr4.F:149-345): the generalized problem from the
// packed state, solved by the library (cuSOLVER zhegvdx: Cholesky of S,
// reduction, tridiagonal divide and conquer, eigenvalues in (el, eu]).
extern "C" int lapw1gpu_seclr4(lapw1gpu_context* c, const double* d_hs_, int ldhs, const double* d_hsdiag_, int n,
                               double el, double eu, int nmax, double* d_eig, double* d_vec_, int ldv, int* nfound) {
  if (!c || !d_hs_ || !d_hsdiag_ || n < 1 || ldhs < n || nmax < 1 || !d_eig || !nfound || (d_vec_ && ldv < n) ||
      !(el < eu))
    return LAPW1GPU_ERR_ARG;
  *nfound = 0;
  CK(cudaSetDevice(c->device));
  cudaStream_t s = c->stream;
  if (!c->solver && cusolverDnCreate(&c->solver) != CUSOLVER_STATUS_SUCCESS) return LAPW1GPU_ERR_CUDA;
  if (cusolverDnSetStream(c->solver, s) != CUSOLVER_STATUS_SUCCESS) return LAPW1GPU_ERR_CUDA;
  const size_t nn = (size_t)n * n;
  double2* H = (double2*)c->buf("sec_h", sizeof(double2) * nn);
  double2* S = (double2*)c->buf("sec_s", sizeof(double2) * nn);
  double* W = (double*)c->buf("sec_w", sizeof(double) * n);
  int* info = (int*)c->buf("sec_info", sizeof(int));
  if (!H || !S || !W || !info) return LAPW1GPU_ERR_NOMEM;
  k_unpack_seclr<<<dim3((n + 127) / 128, n), 128, 0, s>>>(n, reinterpret_cast<const double2*>(d_hs_), ldhs,
                                                         reinterpret_cast<const double2*>(d_hsdiag_), H, S);
  CK(cudaGetLastError());
  const cusolverEigMode_t jobz = d_vec_ ? CUSOLVER_EIG_MODE_VECTOR : CUSOLVER_EIG_MODE_NOVECTOR;
  int lwork = 0, meig = 0;
  if (cusolverDnZhegvdx_bufferSize(c->solver, CUSOLVER_EIG_TYPE_1, jobz, CUSOLVER_EIG_RANGE_V, CUBLAS_FILL_MODE_LOWER,
                                   n, (cuDoubleComplex*)H, n, (cuDoubleComplex*)S, n, el, eu, 0, 0, &meig, W,
                                   &lwork) != CUSOLVER_STATUS_SUCCESS)
    return LAPW1GPU_ERR_CUDA;
  double2* work = (double2*)c->buf("sec_work", sizeof(double2) * (size_t)std::max(1, lwork));
  if (!work) return LAPW1GPU_ERR_NOMEM;
  if (cusolverDnZhegvdx(c->solver, CUSOLVER_EIG_TYPE_1, jobz, CUSOLVER_EIG_RANGE_V, CUBLAS_FILL_MODE_LOWER, n,
                        (cuDoubleComplex*)H, n, (cuDoubleComplex*)S, n, el, eu, 0, 0, &meig, W,
                        (cuDoubleComplex*)work, lwork, info) != CUSOLVER_STATUS_SUCCESS)
    return LAPW1GPU_ERR_CUDA;
  int hinfo = 0;
  CK(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hinfo != 0) return hinfo > n ? LAPW1GPU_ERR_NONFINITE : LAPW1GPU_ERR_RANGE;  // S not positive definite / no convergence
  const int m = std::min(meig, nmax);
  if (m > 0) {
    CK(cudaMemcpyAsync(d_eig, W, sizeof(double) * m, cudaMemcpyDeviceToDevice, s));
    if (d_vec_)
      CK(cudaMemcpy2DAsync(d_vec_, sizeof(double2) * ldv, H, sizeof(double2) * n, sizeof(double2) * n, m,
                           cudaMemcpyDeviceToDevice, s));
    CK(cudaStreamSynchronize(s));
  }
  *nfound = m;
  c->last_launches = 1;
  return LAPW1GPU_OK;
}

// ---------------------------------------------------------------------
// HNS without device allocation.
//
// Some callers cannot let this library allocate device memory: a Fortran
// lapw1 whose device memory is already reserved by the eigen-solver library
// it hands HS to, or a host framework whose caching allocator owns the GPU,
// where a cudaMalloc here could fail for lack of memory or fragment their
// pool (and cudaFree synchronises the device under their stream work).
// This entry point computes the same HNS update as the HNS stage of
// lapw1gpu_setup_stages, with all of its intermediate buffers (the uploaded
// inputs, AL/BL, phases, the HNS operands, tile list, status word) carved
// from one file-scope device array of L1G_NOALLOC_BYTES.  Every GPU that
// loads the library holds that array until the process exits.
// ---------------------------------------------------------------------
#define L1G_NOALLOC_BYTES (64ull << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[L1G_NOALLOC_BYTES];
#define L1G_NOALLOC_MAXDEV 64
static void* g_noalloc_addr[L1G_NOALLOC_MAXDEV];  // device address of the array, per device

// bookkeeping tables of one problem, built on the device (one thread):
// atom type / first atom per type, the LOHNS ranges, the triangle tiles
__global__ void k_noalloc_tables(int nat, const int* __restrict__ mult, const int* __restrict__ ilo, int ntri,
                                 int* atype, int* afirst, LoRange* lor, int2* tiles) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int a = 0, q = 0; a < nat; a++) {
    afirst[a] = q;
    for (int e = 0; e < mult[a]; e++) atype[q++] = a;
  }
  int nr = 0;
  for (int jn = 0, nnlo = 0; jn < nat; jn++)
    for (int l = 0; l <= L1G_LOMAX; l++)
      for (int jlo = 1; jlo <= ilo[jn * (L1G_LOMAX + 1) + l]; jlo++) {
        LoRange r{jn, l, jlo, nnlo + 1, nnlo + (2 * l + 1) * mult[jn]};
        nnlo = r.i2;
        lor[nr++] = r;
      }
  for (int bi = 0, t = 0; bi < ntri; bi++)
    for (int bj = 0; bj <= bi; bj++) tiles[t++] = make_int2(bi, bj);
}

// true when SPHBES would refuse an argument RMT |k+G| of this problem's
// plane-wave rows (the check k_albl makes on the device, made here on the
// host because this entry point returns before its kernels run)
static bool sphbes_out_of_range(const lapw1gpu_problem* p) {
  for (int jn = 0; jn < p->nat; jn++)
    for (int i = 0; i < p->nv; i++)
      if (l1g_sphbes_refuses(p->ltop - 1, p->rmt[jn] * p->rk[i])) return true;
  return false;
}

extern "C" int lapw1gpu_hns_noalloc(const lapw1gpu_problem* p, double* d_hs_, int ldhs, void* stream,
                                    int* d_status_out) {
  int rc = validate(p);
  if (rc) return rc;
  if (!d_hs_ || ldhs < p->n) return LAPW1GPU_ERR_ARG;
  if (sphbes_out_of_range(p)) return LAPW1GPU_ERR_RANGE;  // as the HNS stage reports it
  if (p->nohns) {  // calkpt.F:169: nothing to add
    if (d_status_out) CK(cudaMemsetAsync(d_status_out, 0, sizeof(int), (cudaStream_t)stream));
    return LAPW1GPU_OK;
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= L1G_NOALLOC_MAXDEV) return LAPW1GPU_ERR_RANGE;
  // first call on this device: the array's device address (host code only
  // sees a host-side stand-in under its name)
  if (!g_noalloc_addr[dev]) {
    void* a = nullptr;
    CK(cudaGetSymbolAddress(&a, g_noalloc_scratch));
    g_noalloc_addr[dev] = a;
  }
  char* base = (char*)g_noalloc_addr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  double2* d_hs = reinterpret_cast<double2*>(d_hs_);

  // sizes of this problem (tables themselves are built on the device)
  const int n = p->n, nv = p->nv, nat = p->nat, ndf = p->ndf, ltop = p->ltop, ldl = p->ldl;
  const int nvpad = round_up(nv, 64), npad = round_up(n, 64);
  const int nsl2 = (p->lnsmax + 1) * (p->lnsmax + 1);
  const int K = ndf * 2 * nsl2;
  const int L4 = L1G_LOMAX + 1;
  int nlor = 0;
  for (int jn = 0; jn < nat; jn++)
    for (int l = 0; l <= L1G_LOMAX; l++) nlor += p->ilo[jn * L4 + l];
  const int ntri = (n + HNS_T - 1) / HNS_T;
  const int ntiles = ntri * (ntri + 1) / 2;

  // carve the array: inputs first, then the intermediates; the input copies
  // are issued as the regions are taken (no host-side bookkeeping storage)
  size_t off = 0;
  bool fits = true;
  auto take = [&](size_t bytes) -> char* {
    size_t o = off;
    off += (bytes + 255) / 256 * 256;
    if (off > L1G_NOALLOC_BYTES) fits = false;
    return base + o;
  };
  // first pass only sizes the layout; the copies run once it is known to fit
  struct Pending {
    char* dst;
    const void* src;
    size_t bytes;
  } pend[40];
  int npend = 0;
  auto in = [&](const void* src, size_t bytes) -> char* {
    char* d = take(bytes);
    pend[npend++] = {d, src, bytes};
    return d;
  };
  DevProb P{};
  P.n = n;
  P.nv = nv;
  P.nlo = p->nlo;
  P.nat = nat;
  P.ndf = ndf;
  P.ltop = ltop;
  P.ldl = ldl;
  P.lnsmax = p->lnsmax;
  P.ins = p->ins;
  P.nvpad = nvpad;
  P.npad = npad;
  P.vi = p->vi;
  P.mult = (const int*)in(p->mult, sizeof(int) * nat);
  int* d_atype = (int*)take(sizeof(int) * ndf);
  int* d_afirst = (int*)take(sizeof(int) * nat);
  P.atype = d_atype;
  P.afirst = d_afirst;
  P.rmt = (const double*)in(p->rmt, sizeof(double) * nat);
  P.v = (const double*)in(p->v, sizeof(double) * nat);
  P.pos = (const double*)in(p->pos, sizeof(double) * 3 * ndf);
  P.rotij = (const double*)in(p->rotij, sizeof(double) * 9 * ndf);
  P.rotloc = (const double*)in(p->rotloc, sizeof(double) * 9 * nat);
  P.kzz = (const int*)in(p->kzz, sizeof(int) * 3 * n);
  P.xk = (const double*)in(p->xk, sizeof(double) * n);
  P.yk = (const double*)in(p->yk, sizeof(double) * n);
  P.zk = (const double*)in(p->zk, sizeof(double) * n);
  P.rk = (const double*)in(p->rk, sizeof(double) * n);
  P.p = (const double*)in(p->p, sizeof(double) * nat * ldl);
  P.pe = (const double*)in(p->pe, sizeof(double) * nat * ldl);
  P.dp = (const double*)in(p->dp, sizeof(double) * nat * ldl);
  P.dpe = (const double*)in(p->dpe, sizeof(double) * nat * ldl);
  P.pei = (const double*)in(p->pei, sizeof(double) * nat * ldl);
  P.e = (const double*)in(p->e, sizeof(double) * nat * ldl);
  P.lapw = (const int*)in(p->lapw, sizeof(int) * nat * ldl);
  P.ilo = (const int*)in(p->ilo, sizeof(int) * nat * L4);
  P.loor = (const int*)in(p->loor, sizeof(int) * nat * L4);
  P.alo = (const double*)in(p->alo, sizeof(double) * nat * L1G_NLOAT * L4);
  P.blo = (const double*)in(p->blo, sizeof(double) * nat * L1G_NLOAT * L4);
  P.clo = (const double*)in(p->clo, sizeof(double) * nat * L1G_NLOAT * L4);
  P.elo = (const double*)in(p->elo, sizeof(double) * nat * L1G_NLOAT * L4);
  P.pi12lo = (const double*)in(p->pi12lo, sizeof(double) * nat * L4);
  P.pe12lo = (const double*)in(p->pe12lo, sizeof(double) * nat * L4);
  P.dplo = (const double*)in(p->dplo, sizeof(double) * nat * L4);
  const double2* d_tns = (const double2*)in(p->tns, sizeof(double2) * nat * LAPW1GPU_NTNS * L1G_NSL2 * L1G_NSL2);
  LoRange* d_lor = (LoRange*)take(sizeof(LoRange) * (nlor > 0 ? nlor : 1));
  int2* d_tiles = (int2*)take(sizeof(int2) * ntiles);
  P.al = (double*)take(sizeof(double) * (size_t)nat * ltop * nvpad);
  P.bl = (double*)take(sizeof(double) * (size_t)nat * ltop * nvpad);
  P.phase = (double2*)take(sizeof(double2) * (size_t)ndf * npad);
  double2* Lop = (double2*)take(sizeof(double2) * (size_t)K * npad);
  double2* Rop = (double2*)take(sizeof(double2) * (size_t)K * npad);
  const size_t nloc = (size_t)ndf * nsl2 * std::max(1, p->nlo);
  double2* Clo = (double2*)take(sizeof(double2) * nloc);
  double2* C2lo = (double2*)take(sizeof(double2) * nloc);
  int* d_status = (int*)take(sizeof(int));
  if (!fits) return LAPW1GPU_ERR_RANGE;  // beyond L1G_NOALLOC_BYTES
  if (d_status_out) d_status = d_status_out;  // the caller reads the bits after the stream

  for (int q = 0; q < npend; q++)
    if (pend[q].src && pend[q].bytes)
      CK(cudaMemcpyAsync(pend[q].dst, pend[q].src, pend[q].bytes, cudaMemcpyHostToDevice, s));
  // the array keeps the previous call's contents: the status word must start at 0
  CK(cudaMemsetAsync(d_status, 0, sizeof(int), s));
  k_noalloc_tables<<<1, 32, 0, s>>>(nat, P.mult, P.ilo, ntri, d_atype, d_afirst, d_lor, d_tiles);
  k_albl<<<dim3((nvpad + 127) / 128, nat), 128, 0, s>>>(P, d_status);
  k_phase<<<dim3((npad + 127) / 128, ndf), 128, 0, s>>>(P);
  int nops = 0;
  rc = launch_hns_ops(nullptr, P, d_tns, d_lor, nlor, Lop, Rop, Clo, C2lo, s, &nops);
  if (rc) return rc;
  k_hns_gemm<<<(unsigned)ntiles, 256, 0, s>>>(n, npad, K, d_tiles, Lop, Rop, d_hs, ldhs);
  if (p->nlo > 0)
    k_hns_lo<<<dim3((p->nlo + 127) / 128, p->nlo), 128, 0, s>>>(nv, p->nlo, ndf * nsl2, C2lo, Clo, d_hs, ldhs);
  // a non-finite element of the updated HS sets L1G_STATUS_NONFINITE, as
  // the HNS stage of the allocating entry points reports it
  if (d_status_out) k_check_finite<<<1184, 256, 0, s>>>(n, d_hs, ldhs, nullptr, d_status);
  CK(cudaGetLastError());
  return LAPW1GPU_OK;
}

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

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "kernels_fp64.cuh"
#include "forces.cuh"

#define L1G_VERSION "lapw1gpu 0.1 (sm_100a)"

namespace {

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace

struct lapw1gpu_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[12] = {};
  int* d_status = nullptr;
  int last_status = 0;
  int prec = LAPW1GPU_PREC_FP64;
  int slices = 6;
  bool sph_attr = false;
  cublasHandle_t blas = nullptr;  // library ZGEMM of the FP64 HNS panels
  std::map<std::string, DevBuf> bufs;
  std::map<std::string, std::pair<long, int>> tile_keys;  // tile lists already on the device: shape, count

  // grow-only scratch buffer; returns nullptr on allocation failure
  void* buf(const char* name, size_t bytes) {
    DevBuf& b = bufs[name];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
      if (b.ptr) cudaFree(b.ptr);
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
};

#include "split_tc.cuh"
#include "sph_tc.cuh"

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

namespace {

#define CK(x)                                 \
  do {                                        \
    cudaError_t _e = (x);                     \
    if (_e != cudaSuccess) {                  \
      cudaGetLastError();                     \
      return LAPW1GPU_ERR_CUDA;               \
    }                                         \
  } while (0)

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
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return LAPW1GPU_ERR_CUDA;
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
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
  cudaStreamSynchronize(c->stream);
  if (c->blas) cublasDestroy(c->blas);
  for (auto& kv : c->bufs)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  if (c->d_status) cudaFree(c->d_status);
  for (auto& e : c->ev) cudaEventDestroy(e);
  cudaStreamDestroy(c->stream);
  delete c;
  return LAPW1GPU_OK;
}

int lapw1gpu_set_precision(lapw1gpu_context* c, int prec, int slices) {
  if (!c) return LAPW1GPU_ERR_ARG;
  if (prec != LAPW1GPU_PREC_FP64 && prec != LAPW1GPU_PREC_SPLIT) return LAPW1GPU_ERR_ARG;
  if (prec == LAPW1GPU_PREC_SPLIT && (slices < 2 || slices > L1G_MAX_SLICES)) return LAPW1GPU_ERR_RANGE;
  c->prec = prec;
  if (prec == LAPW1GPU_PREC_SPLIT) c->slices = slices;
  return LAPW1GPU_OK;
}

void* lapw1gpu_stream(lapw1gpu_context* c) { return c ? (void*)c->stream : nullptr; }

int lapw1gpu_last_status(lapw1gpu_context* c) { return c ? c->last_status : 0; }

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
  if (k->arena && k->owns_arena) {
    cudaSetDevice(k->ctx->device);
    cudaStreamSynchronize(k->ctx->stream);
    cudaFree(k->arena);
  }
  delete k;
  return LAPW1GPU_OK;
}

// tile lists (device) for the triangle kernels, cached per shape in the context
static const int2* tiles_tri(lapw1gpu_context* c, const char* name, int n, int T, int* count) {
  const long key = (long)n * 4096 + T;
  auto it = c->tile_keys.find(name);
  if (it != c->tile_keys.end() && it->second.first == key) {  // uploaded by an earlier run
    *count = it->second.second;
    return (const int2*)c->bufs[name].ptr;
  }
  int nb = (n + T - 1) / T;
  std::vector<int2> t;
  for (int bi = 0; bi < nb; bi++)
    for (int bj = 0; bj <= bi; bj++) t.push_back(make_int2(bi, bj));
  *count = (int)t.size();
  c->tile_keys.erase(name);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return nullptr;  // earlier runs may still read it
  int2* d = (int2*)c->buf(name, sizeof(int2) * t.size());
  if (!d) return nullptr;
  if (cudaMemcpy(d, t.data(), sizeof(int2) * t.size(), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  c->tile_keys[name] = std::make_pair(key, *count);
  return d;
}

// HNS operands: R = {ALM, BLM} per row, L = M conj(R) per atom, LO-row terms
static int launch_hns_ops(const DevProb& P, const double2* tns, const LoRange* lor, int nlor, double2* Lop,
                          double2* Rop, double2* Clo, double2* C2lo, cudaStream_t s, int* nl) {
  const int nsl2 = (P.lnsmax + 1) * (P.lnsmax + 1);
  k_hns_alm<<<dim3((P.npad + 127) / 128, P.ndf), 128, 0, s>>>(P, lor, nlor, Rop, Clo);
  if (cudaFuncSetAttribute(k_hns_tmul, cudaFuncAttributeMaxDynamicSharedMemorySize, TMUL_SMEM) != cudaSuccess)
    return LAPW1GPU_ERR_CUDA;
  k_hns_tmul<<<dim3(P.npad / TMUL_I, P.ndf), 256, TMUL_SMEM, s>>>(P.npad, nsl2, P.atype, tns, Rop, Lop);
  *nl += 2;
  if (P.nlo > 0) {
    k_hns_lo_ops<<<dim3((P.nlo + 127) / 128, P.ndf), 128, 0, s>>>(P, tns, Lop, Rop, Clo, C2lo);
    *nl += 1;
  }
  return cudaGetLastError() == cudaSuccess ? LAPW1GPU_OK : LAPW1GPU_ERR_CUDA;
}

// Block width of the FP64 HNS update: diagonal blocks of HNS_DIAG_B rows run
// in k_hns_gemm (64-row tiles, lower triangle only), the rows below each
// diagonal block in one library ZGEMM per block column, as zher2m.f:69-80
// splits its update (ZGEMV on the diagonal block, ZGEMM below).
#define HNS_DIAG_B 512

static const int2* tiles_hns_diag(lapw1gpu_context* c, int n, int* count) {
  auto it = c->tile_keys.find("tiles_hns_diag");
  if (it != c->tile_keys.end() && it->second.first == n) {
    *count = it->second.second;
    return (const int2*)c->bufs["tiles_hns_diag"].ptr;
  }
  std::vector<int2> t;
  const int per = HNS_DIAG_B / HNS_T;
  const int nt = (n + HNS_T - 1) / HNS_T;
  for (int b0 = 0; b0 < nt; b0 += per)
    for (int bi = b0; bi < std::min(nt, b0 + per); bi++)
      for (int bj = b0; bj <= bi; bj++) t.push_back(make_int2(bi, bj));
  *count = (int)t.size();
  c->tile_keys.erase("tiles_hns_diag");
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return nullptr;  // earlier runs may still read it
  int2* d = (int2*)c->buf("tiles_hns_diag", sizeof(int2) * t.size());
  if (!d) return nullptr;
  if (cudaMemcpy(d, t.data(), sizeof(int2) * t.size(), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  c->tile_keys["tiles_hns_diag"] = std::make_pair((long)n, *count);
  return d;
}

static int hns_panels_zgemm(lapw1gpu_context* c, int n, int npad, int K, const double2* Lop, const double2* Rop,
                            double2* hs, int ld, cudaStream_t s) {
  if (!c->blas) {
    if (cublasCreate(&c->blas) != CUBLAS_STATUS_SUCCESS) return LAPW1GPU_ERR_CUDA;
  }
  if (cublasSetStream(c->blas, s) != CUBLAS_STATUS_SUCCESS) return LAPW1GPU_ERR_CUDA;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  for (int c0 = 0; c0 < n; c0 += HNS_DIAG_B) {
    const int w = std::min(HNS_DIAG_B, n - c0);
    const int r0 = c0 + w, m = n - r0;
    if (m <= 0) continue;
    // HS(r0:n, c0:c0+w) += L(r0:n, :) R(c0:c0+w, :)^T ; L, R column-major npad x K
    if (cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, m, w, K, &one, (const cuDoubleComplex*)(Lop + r0), npad,
                    (const cuDoubleComplex*)(Rop + c0), npad, &one, (cuDoubleComplex*)(hs + (size_t)c0 * ld + r0),
                    ld) != CUBLAS_STATUS_SUCCESS)
      return LAPW1GPU_ERR_CUDA;
  }
  return LAPW1GPU_OK;
}

}  // extern "C"

// Spherical part on tcgen05 (sph_tc.cuh): slice the per-l operands, then
// one CTA per (128 J, IT I) tile of the triangle.
template <int S, bool PAIR>
static int sph_tc_launch(lapw1gpu_context* c, const lapw1gpu_kpoint* k, const DevProb& P, const SphCoef* coef,
                         const double2* tab, double2* hs, int ld, double2* hsdiag, cudaStream_t s, int* nl) {
  using Cf = sphtc::Cfg<S>;
  const int nv = k->nv, L = k->ltop, Kc = 2 * k->ndf;
  const int Kcp = round_up(Kc, 32), Kp = 2 * Kcp;
  const int npA = round_up(nv, 128), npB = round_up(nv, Cf::IT);
  int8_t* A = (int8_t*)c->buf("sphA", (size_t)S * L * npA * Kp);
  int8_t* B = (int8_t*)c->buf("sphB", (size_t)S * L * 4 * npB * Kp);
  int* exA = (int*)c->buf("sphExA", sizeof(int) * (size_t)L * npA);
  int* exB = (int*)c->buf("sphExB", sizeof(int) * (size_t)L * 2 * npB);
  if (!A || !B || !exA || !exB) return LAPW1GPU_ERR_NOMEM;
  const int sl_smem = Kc * 33 * (int)sizeof(double2);
  if (sl_smem > 200 * 1024) return LAPW1GPU_ERR_RANGE;
  if (cudaFuncSetAttribute(sphtc::k_sph_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, sl_smem) != cudaSuccess)
    return LAPW1GPU_ERR_CUDA;
  sphtc::k_sph_slice<<<dim3(npA / 32, L), 256, sl_smem, s>>>(P, coef, 0, Kcp, npA, S, A, exA);
  sphtc::k_sph_slice<<<dim3((2 * npB + 31) / 32, L), 256, sl_smem, s>>>(P, coef, 1, Kcp, 2 * npB, S, B, exB);
  *nl += 2;
  CUtensorMap ta, tb;
  if (l1g_tmap_3d(&ta, A, Kp, (uint64_t)L * npA, S, 128) || l1g_tmap_3d(&tb, B, Kp, (uint64_t)L * 4 * npB, S, Cf::N))
    return LAPW1GPU_ERR_CUDA;
  const long key = (long)nv * 1024 + Cf::IT;
  int ntile = 0;
  int2* dt = nullptr;
  auto it = c->tile_keys.find("tiles_sphtc");
  if (it != c->tile_keys.end() && it->second.first == key) {
    ntile = it->second.second;
    dt = (int2*)c->bufs["tiles_sphtc"].ptr;
  } else {
    std::vector<int2> t;
    const int nbj = npA / 128, nbi = npB / Cf::IT;
    for (int bj = 0; bj < nbj; bj++)
      for (int bi = 0; bi < nbi; bi++)
        if (bj * 128 <= bi * Cf::IT + Cf::IT - 1) t.push_back(make_int2(bj, bi));
    c->tile_keys.erase("tiles_sphtc");
    if (cudaStreamSynchronize(s) != cudaSuccess) return LAPW1GPU_ERR_CUDA;  // earlier runs may still read it
    dt = (int2*)c->buf("tiles_sphtc", sizeof(int2) * t.size());
    if (!dt) return LAPW1GPU_ERR_NOMEM;
    if (cudaMemcpy(dt, t.data(), sizeof(int2) * t.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return LAPW1GPU_ERR_CUDA;
    ntile = (int)t.size();
    c->tile_keys["tiles_sphtc"] = std::make_pair(key, ntile);
  }
  if (cudaFuncSetAttribute(sphtc::k_sph_tc<S, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cf::SMEM) !=
      cudaSuccess)
    return LAPW1GPU_ERR_CUDA;
  sphtc::k_sph_tc<S, PAIR><<<ntile, Cf::THREADS, Cf::SMEM, s>>>(ta, tb, P, dt, Kp / 64, npA, npB, exA, exB, tab,
                                                                k->tab, hs, ld, hsdiag, c->d_status);
  *nl += 1;
  return cudaGetLastError() == cudaSuccess ? LAPW1GPU_OK : LAPW1GPU_ERR_CUDA;
}

// Pairing two levels in int32 before the conversion is exact while
// (d+1) 4096 Kp 128 + (d+2) 4096 Kp < 2^31 for every level d < S-1
// (|slice| <= 64, level d sums d+1 products per k).
static bool sph_pair_ok(int S, int Kp) {
  const double worst = (double)S * 4096.0 * Kp * 128.0 + (double)(S + 1) * 4096.0 * Kp;
  return worst < 2147483647.0;
}

// true when the split-precision spherical path handles this slice count
static bool sph_tc_supported(int S) { return false && S >= 4 && S <= 7; }

static int sph_tc_dispatch(lapw1gpu_context* c, const lapw1gpu_kpoint* k, const DevProb& P, const SphCoef* coef,
                           const double2* tab, double2* hs, int ld, double2* hsdiag, cudaStream_t s, int* nl) {
  const int Kp = 2 * round_up(2 * k->ndf, 32);
  const bool pair = sph_pair_ok(c->slices, Kp);
#define SPH_CASE(SS)                                                                   \
  case SS:                                                                             \
    return pair ? sph_tc_launch<SS, true>(c, k, P, coef, tab, hs, ld, hsdiag, s, nl)   \
                : sph_tc_launch<SS, false>(c, k, P, coef, tab, hs, ld, hsdiag, s, nl);
  switch (c->slices) {
    SPH_CASE(4)
    SPH_CASE(5)
    SPH_CASE(6)
    SPH_CASE(7)
    default:
      return LAPW1GPU_ERR_RANGE;
  }
#undef SPH_CASE
}

extern "C" {

// algorithmic FP64-equivalent flops of the contractions (see DESIGN.md roofline)
static double alg_flops(const lapw1gpu_kpoint* k) {
  double nv = k->nv, n = k->n;
  // spherical: per pair and atom type 6 FMA per l, 4 FMA per equivalent
  // atom's phase product, 4 FMA to add PHASE * t into S and H
  double sph = 2.0 * (6.0 * k->ltop * k->nat + 4.0 * k->ndf + 4.0 * k->nat) * (nv * (nv + 1) / 2.0);
  int nsl2 = (k->lnsmax + 1) * (k->lnsmax + 1);
  double hns = k->nohns ? 0.0 : 8.0 * (2.0 * k->ndf * nsl2) * (n * (n + 1) / 2.0);
  return sph + hns;
}

int lapw1gpu_kpoint_run(lapw1gpu_context* c, lapw1gpu_kpoint* k, int stages, double* d_hs_, int ldhs,
                        double* d_hsdiag_, lapw1gpu_stats* st) {
  if (!c || !k || !d_hs_ || !d_hsdiag_ || ldhs < k->n || k->ctx != c) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  double2* d_hs = reinterpret_cast<double2*>(d_hs_);
  double2* d_hsdiag = reinterpret_cast<double2*>(d_hsdiag_);
  cudaStream_t s = c->stream;
  DevProb P = k->P;
  const int n = k->n, nv = k->nv, ltop = k->ltop, ndf = k->ndf, nat = k->nat;
  P.al = (double*)c->buf("al", sizeof(double) * (size_t)nat * ltop * k->nvpad);
  P.bl = (double*)c->buf("bl", sizeof(double) * (size_t)nat * ltop * k->nvpad);
  P.phase = (double2*)c->buf("phase", sizeof(double2) * (size_t)ndf * k->npad);
  if (!P.al || !P.bl || !P.phase) return LAPW1GPU_ERR_NOMEM;
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
  if (st) CK(cudaEventRecord(c->ev[0], s));
  int nl = 0;  // kernels launched by this run

  // ---- K-a: matching coefficients and phases (always needed) ----
  nl++;
  k_albl<<<dim3((k->nvpad + 127) / 128, nat), 128, 0, s>>>(P, c->d_status);
  nl++;
  k_phase<<<dim3((k->npad + 127) / 128, ndf), 128, 0, s>>>(P);
  CK(cudaGetLastError());
  if (st) CK(cudaEventRecord(c->ev[1], s));

  if (stages & 1) {
    // ---- K-c table + K-b spherical ----
    size_t ntab = (size_t)(2 * k->tab.d1 + 1) * (2 * k->tab.d2 + 1) * (2 * k->tab.d3 + 1);
    double2* tab = (double2*)c->buf("tab", sizeof(double2) * 2 * ntab);
    SphCoef* coef = (SphCoef*)c->buf("coef", sizeof(SphCoef) * nat * ltop);
    if (!tab || !coef) return LAPW1GPU_ERR_NOMEM;
    nl++;
    k_table<<<(unsigned)((ntab + 127) / 128), 128, 0, s>>>(P, k->tab, k->d_warp, tab);
    nl++;
    k_sph_coef<<<nat, 32, 0, s>>>(P, coef);
    int ntiles = 0;
    const int2* tl = tiles_tri(c, "tiles_sph", nv, SPH_T, &ntiles);
    if (!tl) return LAPW1GPU_ERR_NOMEM;
    if (c->prec == LAPW1GPU_PREC_SPLIT && sph_tc_supported(c->slices)) {
      int rc = sph_tc_dispatch(c, k, P, coef, tab, d_hs, ldhs, d_hsdiag, s, &nl);
      if (rc) return rc;
    } else {
      if (!c->sph_attr) {  // function attributes are per device: once per context
        CK(cudaFuncSetAttribute(k_spherical, cudaFuncAttributeMaxDynamicSharedMemorySize, SPH_DYN_SMEM));
        c->sph_attr = true;
      }
      nl++;
      k_spherical<<<ntiles, SPH_THREADS, SPH_DYN_SMEM, s>>>(P, tl, coef, tab, k->tab, d_hs, ldhs, d_hsdiag);
    }
    CK(cudaGetLastError());
    if (st) CK(cudaEventRecord(c->ev[2], s));
    // ---- K-b': local-orbital columns ----
    if (k->nlo > 0) nl++;
    if (k->nlo > 0) k_lo<<<dim3((n + 127) / 128, k->nlo), 128, 0, s>>>(P, k->d_locols, d_hs, ldhs, d_hsdiag);
    CK(cudaGetLastError());
    if (st) CK(cudaEventRecord(c->ev[3], s));
  } else if (st) {
    CK(cudaEventRecord(c->ev[2], s));
    CK(cudaEventRecord(c->ev[3], s));
  }

  if ((stages & 2) && !k->nohns) {
    // ---- K-ns ----
    const int nsl2 = (k->lnsmax + 1) * (k->lnsmax + 1);
    const int K = ndf * 2 * nsl2;
    double2* Lop = (double2*)c->buf("hnsL", sizeof(double2) * (size_t)K * k->npad);
    double2* Rop = (double2*)c->buf("hnsR", sizeof(double2) * (size_t)K * k->npad);
    size_t nloc = (size_t)ndf * nsl2 * std::max(1, k->nlo);
    double2* Clo = (double2*)c->buf("hnsClo", sizeof(double2) * nloc);
    double2* C2lo = (double2*)c->buf("hnsC2lo", sizeof(double2) * nloc);
    if (!Lop || !Rop || !Clo || !C2lo) return LAPW1GPU_ERR_NOMEM;
    int rc = launch_hns_ops(P, k->d_tns, k->d_loranges, (int)k->loranges.size(), Lop, Rop, Clo, C2lo, s, &nl);
    if (rc) return rc;
    if (c->prec == LAPW1GPU_PREC_SPLIT)
      rc = split_hns_gemm(c, n, k->npad, K, Lop, Rop, d_hs, ldhs, c->slices, s, &nl);
    else {
      // the blocked form of ZHER2M (zher2m.f:69-80): diagonal blocks of the
      // lower triangle by k_hns_gemm, the panels below them by ZGEMM
      int ntiles = 0;
      const int2* tl = tiles_hns_diag(c, n, &ntiles);
      if (!tl) return LAPW1GPU_ERR_NOMEM;
      nl++;
      k_hns_gemm<<<ntiles, 256, 0, s>>>(n, k->npad, K, tl, Lop, Rop, d_hs, ldhs);
      rc = hns_panels_zgemm(c, n, k->npad, K, Lop, Rop, d_hs, ldhs, s);
    }
    if (rc) return rc;
    if (k->nlo > 0) {
      nl++;
      k_hns_lo<<<dim3((k->nlo + 127) / 128, k->nlo), 128, 0, s>>>(nv, k->nlo, ndf * nsl2, C2lo, Clo, d_hs, ldhs);
    }
    CK(cudaGetLastError());
  }
  if (st) CK(cudaEventRecord(c->ev[4], s));

  if ((stages & 4) && !k->orbs.empty()) {
    double2* alm = (double2*)c->buf("orb_alm", sizeof(double2) * 7 * (size_t)n);
    double2* blm = (double2*)c->buf("orb_blm", sizeof(double2) * 7 * (size_t)n);
    double2* clm = (double2*)c->buf("orb_clm", sizeof(double2) * 7 * (size_t)n);
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
  if (st) CK(cudaEventRecord(c->ev[5], s));
  nl++;
  k_check_finite<<<296, 256, 0, s>>>(n, d_hs, ldhs, d_hsdiag, c->d_status);
  CK(cudaGetLastError());
  if (st) {
    CK(cudaEventRecord(c->ev[6], s));
    int hstat = 0;
    CK(cudaMemcpyAsync(&hstat, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c->last_status = hstat;
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
    if (hstat & L1G_STATUS_NONFINITE) return LAPW1GPU_ERR_NONFINITE;
    if (hstat) return LAPW1GPU_ERR_RANGE;
  }
  return LAPW1GPU_OK;
}

int lapw1gpu_setup_stages(lapw1gpu_context* c, const lapw1gpu_problem* p, int stages, double* hs, int ldhs,
                          double* hsdiag, lapw1gpu_stats* st) {
  if (!c || !p || !hs || !hsdiag || ldhs < p->n) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
  cudaEvent_t e0 = c->ev[7], e1 = c->ev[8], e2 = c->ev[9], e3 = c->ev[10];
  cudaEventRecord(e0, c->stream);
  lapw1gpu_kpoint* k = nullptr;
  int rc = kpoint_upload_impl(c, p, &k, true);
  if (rc) return rc;
  const int n = p->n;
  double2* d_hs = (double2*)c->buf("hs", sizeof(double2) * (size_t)n * n);
  double2* d_hd = (double2*)c->buf("hsdiag", sizeof(double2) * (size_t)n);
  if (!d_hs || !d_hd) {
    lapw1gpu_kpoint_free(k);
    return LAPW1GPU_ERR_NOMEM;
  }
  // stages that only add (HNS/HORB alone) start from the caller's HS
  if (!(stages & 1)) {
    cudaMemcpy2DAsync(d_hs, sizeof(double2) * n, hs, sizeof(double2) * ldhs, sizeof(double2) * n, n,
                      cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(d_hd, hsdiag, sizeof(double2) * n, cudaMemcpyHostToDevice, c->stream);
  }
  cudaEventRecord(e1, c->stream);
  lapw1gpu_stats st2;
  rc = lapw1gpu_kpoint_run(c, k, stages, (double*)d_hs, n, (double*)d_hd, &st2);
  cudaEventRecord(e2, c->stream);
  if (rc == LAPW1GPU_OK) {
    if (cudaMemcpy2DAsync(hs, sizeof(double2) * ldhs, d_hs, sizeof(double2) * n, sizeof(double2) * n, n,
                          cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaMemcpyAsync(hsdiag, d_hd, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      rc = LAPW1GPU_ERR_CUDA;
  }
  cudaEventRecord(e3, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = LAPW1GPU_ERR_CUDA;
  if (st) {
    *st = st2;
    float a, b;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e2, e3);
    st->ms_h2d = a;
    st->ms_d2h = b;
  }
  lapw1gpu_kpoint_free(k);
  return rc;
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

// Band-energy gradient (forces.cuh): rho = C f C^H and rhoE = C f eps C^H by
// library ZGEMM, the PW x PW and LO parts by k_force_sph / k_force_lo, the
// HNS part through its factors (four ZGEMMs and a per-atom reduction).
int lapw1gpu_forces(lapw1gpu_context* c, lapw1gpu_kpoint* k, const double* d_c_, int ldc, int nb, const double* d_occ,
                    const double* d_eps, double* d_grad) {
  if (!c || !k || k->ctx != c || !d_c_ || !d_occ || !d_eps || !d_grad || nb < 1 || ldc < k->n)
    return LAPW1GPU_ERR_ARG;
  if (!k->orbs.empty()) return LAPW1GPU_ERR_ARG;
  CK(cudaSetDevice(c->device));
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
  if (!c->blas && cublasCreate(&c->blas) != CUBLAS_STATUS_SUCCESS) return LAPW1GPU_ERR_CUDA;
  if (cublasSetStream(c->blas, s) != CUBLAS_STATUS_SUCCESS) return LAPW1GPU_ERR_CUDA;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  CK(cudaMemsetAsync(c->d_status, 0, sizeof(int), s));
  CK(cudaMemsetAsync(d_grad, 0, sizeof(double) * 3 * ndf, s));
  k_albl<<<dim3((k->nvpad + 127) / 128, nat), 128, 0, s>>>(P, c->d_status);
  k_phase<<<dim3((k->npad + 127) / 128, ndf), 128, 0, s>>>(P);
  k_sph_coef<<<nat, 32, 0, s>>>(P, coef);
  k_force_weight<<<dim3((n + 127) / 128, nb), 128, 0, s>>>(n, nb, C, ldc, d_occ, d_eps, Cf, Ce);
  CK(cudaGetLastError());
  // rho(J,I) = sum_b f_b c_b(J) conj(c_b(I)): column-major n x n
  if (cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_C, n, n, nb, &one, (const cuDoubleComplex*)Cf, n,
                  (const cuDoubleComplex*)C, ldc, &zero, (cuDoubleComplex*)rho, n) != CUBLAS_STATUS_SUCCESS ||
      cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_C, n, n, nb, &one, (const cuDoubleComplex*)Ce, n,
                  (const cuDoubleComplex*)C, ldc, &zero, (cuDoubleComplex*)rhoe, n) != CUBLAS_STATUS_SUCCESS)
    return LAPW1GPU_ERR_CUDA;
  int ntiles = 0;
  const int2* tl = tiles_tri(c, "tiles_sph", nv, SPH_T, &ntiles);
  if (!tl) return LAPW1GPU_ERR_NOMEM;
  CK(cudaFuncSetAttribute(k_force_sph, cudaFuncAttributeMaxDynamicSharedMemorySize, SPH_DYN_SMEM));
  k_force_sph<<<ntiles, SPH_THREADS, SPH_DYN_SMEM, s>>>(P, tl, coef, k->tab, rho, rhoe, n, d_grad);
  CK(cudaGetLastError());
  if (nlo > 0) k_force_lo<<<dim3((n + 127) / 128, nlo), 128, 0, s>>>(P, k->d_locols, rho, rhoe, n, d_grad);
  CK(cudaGetLastError());
  if (!k->nohns) {
    const int nsl2 = (k->lnsmax + 1) * (k->lnsmax + 1);
    const int K = ndf * 2 * nsl2, Kc = ndf * nsl2;
    double2* Lop = (double2*)c->buf("hnsL", sizeof(double2) * (size_t)K * k->npad);
    double2* Rop = (double2*)c->buf("hnsR", sizeof(double2) * (size_t)K * k->npad);
    size_t nloc = (size_t)Kc * std::max(1, nlo);
    double2* Clo = (double2*)c->buf("hnsClo", sizeof(double2) * nloc);
    double2* C2lo = (double2*)c->buf("hnsC2lo", sizeof(double2) * nloc);
    double2* GC = (double2*)c->buf("frc_gc", sizeof(double2) * (size_t)4 * nb * n);
    double2* Y = (double2*)c->buf("frc_y", sizeof(double2) * (size_t)4 * nb * K);
    double2* Z = (double2*)c->buf("frc_z", sizeof(double2) * (size_t)4 * nb * K);
    if (!Lop || !Rop || !Clo || !C2lo || !GC || !Y || !Z) return LAPW1GPU_ERR_NOMEM;
    int nl = 0;
    int rc = launch_hns_ops(P, k->d_tns, k->d_loranges, (int)k->loranges.size(), Lop, Rop, Clo, C2lo, s, &nl);
    if (rc) return rc;
    k_force_gscale<<<dim3((n + 127) / 128, nb), 128, 0, s>>>(n, nb, P.kzz, C, ldc, GC);
    CK(cudaGetLastError());
    // Y = R^H (G c), Z = L^T (G c): K x 4nb, rows of R and L beyond n unused
    if (cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, K, 4 * nb, n, &one, (const cuDoubleComplex*)Rop, k->npad,
                    (const cuDoubleComplex*)GC, n, &zero, (cuDoubleComplex*)Y, K) != CUBLAS_STATUS_SUCCESS ||
        cublasZgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, K, 4 * nb, n, &one, (const cuDoubleComplex*)Lop, k->npad,
                    (const cuDoubleComplex*)GC, n, &zero, (cuDoubleComplex*)Z, K) != CUBLAS_STATUS_SUCCESS)
      return LAPW1GPU_ERR_CUDA;
    k_force_hns_reduce<<<ndf, 256, 0, s>>>(2 * nsl2, K, nb, Y, Z, d_occ, d_grad);
    CK(cudaGetLastError());
    if (nlo > 0) {
      // CLM rows: Yc = CLM^H (G c) over the LO rows, Zc = T_C (Y; Yc)
      double2* Yc = (double2*)c->buf("frc_yc", sizeof(double2) * (size_t)4 * nb * Kc);
      double2* Zc = (double2*)c->buf("frc_zc", sizeof(double2) * (size_t)4 * nb * Kc);
      if (!Yc || !Zc) return LAPW1GPU_ERR_NOMEM;
      if (cublasZgemm(c->blas, CUBLAS_OP_C, CUBLAS_OP_N, Kc, 4 * nb, nlo, &one, (const cuDoubleComplex*)Clo, nlo,
                      (const cuDoubleComplex*)(GC + nv), n, &zero, (cuDoubleComplex*)Yc, Kc) != CUBLAS_STATUS_SUCCESS)
        return LAPW1GPU_ERR_CUDA;
      k_force_hns_zc<<<dim3(4 * nb, ndf), 32, 0, s>>>(nsl2, K, Kc, P.atype, k->d_tns, Y, Yc, Zc);
      k_force_hns_reduce<<<ndf, 256, 0, s>>>(nsl2, Kc, nb, Yc, Zc, d_occ, d_grad);
      CK(cudaGetLastError());
    }
  }
  int hstat = 0;
  CK(cudaMemcpyAsync(&hstat, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  c->last_status = hstat;
  return hstat ? LAPW1GPU_ERR_RANGE : LAPW1GPU_OK;
}

}  // extern "C"

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

extern "C" int lapw1gpu_hns_noalloc(const lapw1gpu_problem* p, double* d_hs_, int ldhs, void* stream) {
  int rc = validate(p);
  if (rc) return rc;
  if (!d_hs_ || ldhs < p->n) return LAPW1GPU_ERR_ARG;
  if (p->nohns) return LAPW1GPU_OK;  // calkpt.F:169: nothing to add
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

  for (int q = 0; q < npend; q++)
    if (pend[q].src && pend[q].bytes)
      CK(cudaMemcpyAsync(pend[q].dst, pend[q].src, pend[q].bytes, cudaMemcpyHostToDevice, s));
  // the array keeps the previous call's contents: the status word must start at 0
  CK(cudaMemsetAsync(d_status, 0, sizeof(int), s));
  k_noalloc_tables<<<1, 32, 0, s>>>(nat, P.mult, P.ilo, ntri, d_atype, d_afirst, d_lor, d_tiles);
  k_albl<<<dim3((nvpad + 127) / 128, nat), 128, 0, s>>>(P, d_status);
  k_phase<<<dim3((npad + 127) / 128, ndf), 128, 0, s>>>(P);
  int nops = 0;
  rc = launch_hns_ops(P, d_tns, d_lor, nlor, Lop, Rop, Clo, C2lo, s, &nops);
  if (rc) return rc;
  k_hns_gemm<<<(unsigned)ntiles, 256, 0, s>>>(n, npad, K, d_tiles, Lop, Rop, d_hs, ldhs);
  if (p->nlo > 0)
    k_hns_lo<<<dim3((p->nlo + 127) / 128, p->nlo), 128, 0, s>>>(nv, p->nlo, ndf * nsl2, C2lo, Clo, d_hs, ldhs);
  CK(cudaGetLastError());
  return LAPW1GPU_OK;
}

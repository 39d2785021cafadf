// C ABI of the sm_100a DGFS collision operators (single translation unit).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/dgfs_sm100.h"
#include "fft_reg.cuh"
#include "cluster_slab.cuh"
#include "vhs_kernels.cuh"
#include "dg_kernels.cuh"
#include "vss_kernels.cuh"

using namespace dgfs;

// NVTX range over an entry point (host side: the launches it issues), for
// nsys / ncu --nvtx; free when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define DGFS_CUDA(call)                                                      \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return fail(DGFS_ERR_CUDA, std::string(#call) + ": " +                 \
                                     cudaGetErrorString(e_));                \
  } while (0)

extern "C" const char* dgfs_last_error_string(void) { return g_err.c_str(); }
extern "C" const char* dgfs_version(void) { return "dgfs_sm100 0.1 (sm_100a)"; }

// ---------------------------------------------------------------------------
// twiddle tables (uploaded once per device)
// ---------------------------------------------------------------------------
// Host-to-device copies from pageable memory (cudaMemcpy, cudaMemcpyToSymbol)
// and cudaMemset run on the legacy default stream, and the copies may still
// be in flight when the call returns.  The handles' kernels run on the
// caller's and the handles' own streams, which may be non-blocking and then
// do not wait for the legacy stream: every create (and every upload of
// constant tables) ends by waiting for that stream, so a kernel launched
// right after it reads complete tables.
static int settle_uploads() {
  DGFS_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  return DGFS_OK;
}

static std::mutex g_tw_mu;
static bool g_tw_done[64];

static int ensure_twiddles() {
  int dev = 0;
  DGFS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(DGFS_ERR_INVALID, "device id out of range");
  std::lock_guard<std::mutex> lk(g_tw_mu);
  if (g_tw_done[dev]) return DGFS_OK;
  std::vector<double2> t64(kTwTotal);
  std::vector<float2> t32(kTwTotal);
  for (int i = 0; i < kNumTw; ++i) {
    const int nt = tw_size(i), off = tw_offset(nt);
    for (int k = 0; k < nt; ++k) {
      // exp(-2 pi i k / nt), argument reduced to the first half-turn
      const long double ang = 2.0L * 3.141592653589793238462643383279502884L *
                              (long double)k / (long double)nt;
      const double c = (double)std::cos(ang), s = -(double)std::sin(ang);
      t64[off + k] = make_double2(c, s);
      t32[off + k] = make_float2((float)c, (float)s);
    }
  }
  DGFS_CUDA(cudaMemcpyToSymbol(c_tw64, t64.data(), sizeof(double2) * kTwTotal));
  DGFS_CUDA(cudaMemcpyToSymbol(c_tw32, t32.data(), sizeof(float2) * kTwTotal));
  if (int rc = settle_uploads()) return rc;
  g_tw_done[dev] = true;
  return DGFS_OK;
}

// ---------------------------------------------------------------------------
// cluster launch helper
// ---------------------------------------------------------------------------
template <typename K, typename A>
static int launch_cluster(K kernel, dim3 grid, dim3 block, int cluster,
                          size_t smem, cudaStream_t st, const A& args) {
  DGFS_CUDA(cudaFuncSetAttribute(kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  if (cluster > 8)
    DGFS_CUDA(cudaFuncSetAttribute(
        kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  DGFS_CUDA(cudaLaunchKernelEx(&cfg, kernel, args));
  return DGFS_OK;
}

template <typename K, typename A, typename B>
static int launch_cluster2(K kernel, dim3 grid, dim3 block, int cluster,
                           size_t smem, cudaStream_t st, const A& args,
                           const B& args2) {
  DGFS_CUDA(cudaFuncSetAttribute(kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  if (cluster > 8)
    DGFS_CUDA(cudaFuncSetAttribute(
        kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  DGFS_CUDA(cudaLaunchKernelEx(&cfg, kernel, args, args2));
  return DGFS_OK;
}

template <typename K, typename A>
static int launch_plain(K kernel, dim3 grid, dim3 block, size_t smem,
                        cudaStream_t st, const A& args) {
  if (smem > 48 * 1024)
    DGFS_CUDA(cudaFuncSetAttribute(
        kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kernel<<<grid, block, smem, st>>>(args);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

// ---------------------------------------------------------------------------
// VHS handle
// ---------------------------------------------------------------------------
struct dgfs_vhs_s {
  int N = 0, Nrho = 0, M = 0, Mu = 0, n = 0;
  int precision = DGFS_PREC_FP64;
  int max_evals = 0;
  double prefac = 0, cw = 0;
  int device = 0;
  int project = 0;
  double Ginv[25] = {};
  int c32 = 0;  // cluster size of the FP32 terms kernel (autotuner choice)
  // constant tables
  double* c0 = nullptr;      // [N]
  double* b2 = nullptr;      // [n]
  double* b1w64 = nullptr;   // [Nrho][n]
  float* b1w32 = nullptr;    // [Nrho][n] (FP32 mode)
  void* ph = nullptr;        // [Nrho][Mu][3][N] precision R
  double* kappa = nullptr;   // [Nrho][Mu][3]
  float* mult = nullptr;     // [Mu]
  float2* nyq32 = nullptr;   // [Nrho][Mu][3] exp(i N kappa_a) (FP32 mode)
  // scratch
  float2* rho = nullptr;     // [E][Nrho][Mu][3][N][N] Nyquist-plane transforms
  float2* Fny = nullptr;     // [E][3][N][N] Nyquist planes of F_g
  void* Fg = nullptr;        // [E][n] complex R
  void* H = nullptr;         // [E][Nrho][n] complex R
  double* ReLf = nullptr;    // [E][n]
  double2* mhat = nullptr;   // [E][3][N]
  double* moments = nullptr; // [E][5]
  void* uv = nullptr;        // [E][Nrho][Mu][2][3][N] R
  double2* hh = nullptr;     // [E][Nrho][Mu][3][N]
  double2* GM = nullptr;     // [E][n]
  int* err = nullptr;        // device error flag of the bounded waits
  CUtensorMap fg_map;        // FP32: TMA map of Fg, box P x N x (N+2)
  bool fg_map_ok = false;
  // optional per-kernel timing (events recorded between the launches)
  bool profile = false;
  cudaEvent_t ev[6] = {};
  cudaEvent_t evg[2] = {};
  int ev_used = 0;
  // FP32 mode, three streams: the caller's runs prologue, Nyquist planes and
  // epilogue; `aux` (lowest priority) the tables and the FP64 Maxwellian-gain
  // kernel; `hi` (highest priority) the FP32 terms kernel, so the block
  // scheduler fills SMs with terms CTAs first and the gain kernel takes the
  // SMs the terms kernel's last wave leaves idle
  cudaStream_t aux = nullptr, hi = nullptr;
  cudaEvent_t fork0 = nullptr, tab = nullptr, fork1 = nullptr;
  cudaEvent_t join_hi = nullptr, join_aux = nullptr;
};

// FP64-kernel and FP32-terms cluster sizes per N (shared memory per CTA
// must hold three padded slabs of N^3/C complex elements).
static int c64_of(int N) {
  switch (N) {
    case 8: return 1;
    case 16: return 2;
    case 24: return 4;
    case 32: return 8;
    case 48: return 16;  // FP64 sums in global memory (vhs_terms_fp64g_kernel)
    default: return 0;
  }
}
static int c32_of(int N) {
  switch (N) {
    case 8: return 1;
    case 16: return 1;
    case 24: return 3;
    case 32: return 4;
    case 48: return 16;
    default: return 0;
  }
}
template <int N> struct VhsClusters;
// c64: FP64 terms kernel; c32: FP32 terms kernel (default); cpro / cepi:
// prologue / epilogue (FP64, one slab per CTA up to N=32).  At N=32 an 8-CTA prologue
// cluster needs 75 KB per CTA and a 16-CTA epilogue cluster 34 KB, so two
// (four) CTAs share an SM and a 24-point batch runs in one wave of each.
template <> struct VhsClusters<8> { static constexpr int c64 = 1, c32 = 1, cpro = 1, cepi = 1; };
template <> struct VhsClusters<16> { static constexpr int c64 = 2, c32 = 1, cpro = 2, cepi = 2; };
template <> struct VhsClusters<24> { static constexpr int c64 = 4, c32 = 3, cpro = 4, cepi = 4; };
template <> struct VhsClusters<32> { static constexpr int c64 = 8, c32 = 4, cpro = 8, cepi = 16; };
// N=48: 16-CTA clusters of 3 planes; the FP64 terms kernel keeps its running
// sums in global memory (three FP64 slabs would need 331 KB per CTA)
template <> struct VhsClusters<48> { static constexpr int c64 = 16, c32 = 16, cpro = 16, cepi = 16; };

static size_t slab_bytes(int N, int C, size_t elem) {
  return (size_t)(N / C) * N * (N + 1) * elem;
}

static void free_handle(dgfs_vhs_s* h) {
  void* ptrs[] = {h->c0, h->b2, h->b1w64, h->b1w32, h->ph, h->kappa, h->mult,
                  h->Fg, h->H, h->ReLf, h->mhat, h->moments, h->uv, h->hh,
                  h->GM, h->nyq32, h->rho, h->Fny, h->err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : h->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : h->evg)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : {h->fork0, h->tab, h->fork1, h->join_hi, h->join_aux})
    if (e) cudaEventDestroy(e);
  if (h->aux) cudaStreamDestroy(h->aux);
  if (h->hi) cudaStreamDestroy(h->hi);
  delete h;
}

template <typename T>
static int upload(T** dst, const std::vector<T>& v) {
  DGFS_CUDA(cudaMalloc((void**)dst, sizeof(T) * v.size()));
  DGFS_CUDA(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(),
                       cudaMemcpyHostToDevice));
  return DGFS_OK;
}

extern "C" int dgfs_vhs_create(const dgfs_vhs_desc* d, dgfs_vhs_handle* out) {
  if (!d || !out) return fail(DGFS_ERR_INVALID, "null descriptor or handle");
  *out = nullptr;
  if (d->N <= 0 || d->Nrho <= 0 || d->M <= 0 || d->max_evals <= 0)
    return fail(DGFS_ERR_INVALID, "N, Nrho, M and max_evals must be positive");
  if (!d->qz || !d->qw || !d->sz || !d->c0)
    return fail(DGFS_ERR_INVALID, "qz, qw, sz and c0 are required");
  if (d->precision != DGFS_PREC_FP64 && d->precision != DGFS_PREC_FP32)
    return fail(DGFS_ERR_INVALID, "unknown precision");
  if (c32_of(d->N) == 0)
    return fail(DGFS_ERR_UNSUPPORTED,
                "velocity grid N=" + std::to_string(d->N) +
                    " is not compiled in (supported: 8, 16, 24, 32, 48)");
  if (d->precision == DGFS_PREC_FP64 && c64_of(d->N) == 0)
    return fail(DGFS_ERR_UNSUPPORTED,
                "velocity grid N=" + std::to_string(d->N) +
                    " is compiled for the FP32 mode only");
  if (int rc = ensure_twiddles()) return rc;

  const int N = d->N, n = N * N * N, Nrho = d->Nrho, M = d->M;
  const bool fp32 = d->precision == DGFS_PREC_FP32;

  // unique directions: merge exact antipodal pairs (identical h, weight 2)
  std::vector<int> uq;
  std::vector<float> mult;
  std::vector<char> used(M, 0);
  for (int q = 0; q < M; ++q) {
    if (used[q]) continue;
    used[q] = 1;
    float m = 1.f;
    for (int r = q + 1; r < M; ++r) {
      if (!used[r] && d->sz[3 * r] == -d->sz[3 * q] &&
          d->sz[3 * r + 1] == -d->sz[3 * q + 1] &&
          d->sz[3 * r + 2] == -d->sz[3 * q + 2]) {
        used[r] = 1;
        m = 2.f;
        break;
      }
    }
    uq.push_back(q);
    mult.push_back(m);
  }
  const int Mu = (int)uq.size();

  auto* h = new dgfs_vhs_s();
  h->N = N; h->n = n; h->Nrho = Nrho; h->M = M; h->Mu = Mu;
  h->precision = d->precision;
  h->max_evals = d->max_evals;
  h->prefac = d->prefac;
  h->cw = d->cw;
  cudaGetDevice(&h->device);

  // l-vectors in FFT order, x slowest (std/scattering.py:116-128)
  std::vector<double> l0(N);
  for (int i = 0; i < N; ++i) l0[i] = (i < N / 2) ? i : i - N;
  auto sinc = [&](double s) {
    return std::sin(s + d->sinc_eps) / (s + d->sinc_eps);
  };
  // b1 (weighted), b2 (vhs-gll.mako:69-99); W_p = sf*qw_p*sw/n (:188-193)
  std::vector<double> b1w((size_t)Nrho * n), b2(n, 0.0);
  for (int ix = 0; ix < N; ++ix)
    for (int iy = 0; iy < N; ++iy)
      for (int iz = 0; iz < N; ++iz) {
        const size_t l = ((size_t)ix * N + iy) * N + iz;
        const double cS = std::sqrt(l0[ix] * l0[ix] + l0[iy] * l0[iy] +
                                    l0[iz] * l0[iz]);
        double bsum = 0.0;
        for (int p = 0; p < Nrho; ++p) {
          const double qz = d->qz[p];
          const double b1 = std::pow(qz, d->gamma + 2.) * 4 * M_PI *
                            sinc(M_PI / d->L * qz / 2. * cS);
          b1w[(size_t)p * n + l] =
              (d->sphere_factor * d->qw[p] * d->sw / n) * b1;
          bsum += d->qw[p] * std::pow(qz, d->gamma + 2.) * 16 * M_PI * M_PI *
                  sinc(M_PI / d->L * qz * cS);
        }
        b2[l] = bsum;
      }
  // phase tables exp(i kappa_a rep(l)) and kappa
  std::vector<double> kappa((size_t)Nrho * Mu * 3);
  std::vector<double2> ph64((size_t)Nrho * Mu * 3 * N);
  for (int p = 0; p < Nrho; ++p)
    for (int u = 0; u < Mu; ++u)
      for (int a = 0; a < 3; ++a) {
        const double k = M_PI / d->L * d->qz[p] / 2. * d->sz[3 * uq[u] + a];
        kappa[((size_t)p * Mu + u) * 3 + a] = k;
        for (int l = 0; l < N; ++l)
          ph64[(((size_t)p * Mu + u) * 3 + a) * N + l] =
              make_double2(std::cos(k * l0[l]), std::sin(k * l0[l]));
      }
  std::vector<double> c0(d->c0, d->c0 + N);

  int rc = DGFS_OK;
  if ((rc = upload(&h->c0, c0)) || (rc = upload(&h->b2, b2)) ||
      (rc = upload(&h->b1w64, b1w)) || (rc = upload(&h->kappa, kappa)) ||
      (rc = upload(&h->mult, mult))) {
    free_handle(h);
    return rc;
  }
  if (fp32) {
    std::vector<float> b1w32(b1w.begin(), b1w.end());
    // FP32 phase tables carry sqrt(multiplicity) on the x axis
    std::vector<float2> ph32(ph64.size());
    for (size_t i = 0; i < ph64.size(); ++i) {
      const size_t u = (i / (3 * N)) % Mu, ax = (i / N) % 3;
      const double sc = ax == 0 ? std::sqrt((double)mult[u]) : 1.0;
      ph32[i] = make_float2((float)(sc * ph64[i].x), (float)(sc * ph64[i].y));
    }
    // Nyquist rotation factors exp(i N kappa_a), unit modulus
    std::vector<float2> nyq(kappa.size());
    for (size_t i = 0; i < kappa.size(); ++i)
      nyq[i] = make_float2((float)std::cos(N * kappa[i]),
                           (float)std::sin(N * kappa[i]));
    float2* p32 = nullptr;
    if ((rc = upload(&h->b1w32, b1w32)) || (rc = upload(&p32, ph32)) ||
        (rc = upload(&h->nyq32, nyq))) {
      free_handle(h);
      return rc;
    }
    h->ph = p32;
  } else {
    double2* p64 = nullptr;
    if ((rc = upload(&p64, ph64))) { free_handle(h); return rc; }
    h->ph = p64;
  }

  const size_t E = (size_t)d->max_evals;
  const size_t ce = fp32 ? sizeof(float2) : sizeof(double2);
  cudaError_t ce_ = cudaSuccess;
  auto alloc = [&](void** p, size_t bytes) {
    if (ce_ == cudaSuccess) ce_ = cudaMalloc(p, bytes);
  };
  alloc((void**)&h->err, sizeof(int));
  if (ce_ == cudaSuccess) ce_ = cudaMemset(h->err, 0, sizeof(int));
  alloc(&h->Fg, E * n * ce);
  alloc(&h->H, E * Nrho * n * ce);
  alloc((void**)&h->ReLf, E * n * sizeof(double));
  if (fp32) {
    alloc((void**)&h->mhat, E * 3 * N * sizeof(double2));
    alloc((void**)&h->moments, E * 5 * sizeof(double));
    alloc(&h->uv, E * Nrho * Mu * 6 * N * sizeof(float2));
    alloc((void**)&h->hh, E * Nrho * Mu * 3 * N * sizeof(double2));
    alloc((void**)&h->GM, E * n * sizeof(double2));
    alloc((void**)&h->rho, E * Nrho * Mu * 3 * N * N * sizeof(float2));
    alloc((void**)&h->Fny, E * 3 * N * N * sizeof(float2));
  }
  if (ce_ != cudaSuccess) {
    free_handle(h);
    return fail(DGFS_ERR_CUDA,
                std::string("scratch allocation: ") + cudaGetErrorString(ce_));
  }
  if (fp32) {
    // TMA map of F_g for the TMA terms variant at the default cluster size
    // (P = N / c32 planes per CTA): dims (lz, ly, lx, eval), 8-byte elements
    // (one complex float), box (N+2, N, P, 1): the two elements past each
    // row are out of bounds and arrive as zeros (the row padding)
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault,
                                &q) == cudaSuccess && fn &&
        q == cudaDriverEntryPointSuccess) {
      const cuuint64_t dims[4] = {(cuuint64_t)N, (cuuint64_t)N, (cuuint64_t)N,
                                  (cuuint64_t)E};
      const cuuint64_t strides[3] = {(cuuint64_t)N * 8, (cuuint64_t)N * N * 8,
                                     (cuuint64_t)n * 8};
      const cuuint32_t box[4] = {(cuuint32_t)(N + 2), (cuuint32_t)N,
                                 (cuuint32_t)(N / c32_of(N)), 1u};
      const cuuint32_t estr[4] = {1, 1, 1, 1};
      const CUresult r = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn)(
          &h->fg_map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, h->Fg, dims, strides,
          box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      h->fg_map_ok = r == CUDA_SUCCESS;
    }
  }
  if (fp32) {
    int lo_prio = 0, hi_prio = 0;
    cudaError_t e1 = cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    if (e1 == cudaSuccess)
      e1 = cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, lo_prio);
    if (e1 == cudaSuccess)
      e1 = cudaStreamCreateWithPriority(&h->hi, cudaStreamNonBlocking, hi_prio);
    for (cudaEvent_t* ev : {&h->fork0, &h->tab, &h->fork1, &h->join_hi, &h->join_aux})
      if (e1 == cudaSuccess)
        e1 = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e1 != cudaSuccess) {
      free_handle(h);
      return fail(DGFS_ERR_CUDA, std::string("stream/event creation: ") +
                                     cudaGetErrorString(e1));
    }
  }
  if (int rc_s = settle_uploads()) { free_handle(h); return rc_s; }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_vhs_destroy(dgfs_vhs_handle h) {
  if (!h) return DGFS_OK;
  free_handle(h);
  return DGFS_OK;
}

extern "C" const double* dgfs_vhs_last_moments(dgfs_vhs_handle h) {
  return h ? h->moments : nullptr;
}

extern "C" int dgfs_vhs_device_error(dgfs_vhs_handle h, int32_t* out) {
  if (!h || !out) return fail(DGFS_ERR_INVALID, "null argument");
  int v = 0;
  DGFS_CUDA(cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (v) DGFS_CUDA(cudaMemset(h->err, 0, sizeof(int)));
  *out = v;
  return DGFS_OK;
}

// FP32 terms kernel at cluster size C (each C must divide N and fit three
// slabs in shared memory).
template <int N, int C, bool TMA = false>
static int launch_terms32_c(const VhsTermsArgs& a, int nevals, int Nrho,
                            cudaStream_t st, const CUtensorMap* map = nullptr) {
  using G = Geo<N, C>;
  // three slabs (with TMA the transform slab has rows of N+2 elements and
  // 128 bytes of alignment slack), two table slots, the staged plane
  // transforms of one term (and the TMA mbarrier)
  const size_t smem = (TMA ? (size_t)G::P * N * (N + 2) * sizeof(float2) + 128
                           : slab_bytes(N, C, sizeof(float2))) +
                      2 * slab_bytes(N, C, sizeof(float2)) +
                      2 * (9 * N + 4) * sizeof(float2) +
                      (size_t)((TermsRyStaged<C>::value ? N * N : 0) +
                               2 * G::P * N) * sizeof(float2) +
                      (TMA ? sizeof(uint64_t) : 0);
  if (TMA && !map) return fail(DGFS_ERR_UNSUPPORTED, "no TMA map for this handle");
  CUtensorMap none;
  std::memset(&none, 0, sizeof(none));
  return launch_cluster2(vhs_terms_fp32_kernel<N, C, TMA>,
                         dim3(C, (Nrho + 1) / 2, nevals), dim3(G::NT), C, smem,
                         st, a, map ? *map : none);
}

// Split-pencil terms kernel (two threads per pencil), same shared memory.
template <int N, int C>
static int launch_terms32s_c(const VhsTermsArgs& a, int nevals, int Nrho,
                             cudaStream_t st) {
  using G = Geo<N, C>;
  const size_t smem = 3 * slab_bytes(N, C, sizeof(float2)) +
                      2 * (9 * N + 4) * sizeof(float2) +
                      (size_t)((TermsRyStaged<C>::value ? N * N : 0) +
                               2 * G::P * N) * sizeof(float2);
  return launch_cluster(vhs_terms_fp32s_kernel<N, C>,
                        dim3(C, (Nrho + 1) / 2, nevals), dim3(GeoS<N, C>::NT), C,
                        smem, st, a);
}

// Variant codes: the cluster size C for the one-thread-per-pencil kernel,
// 100 + C for the split-pencil kernel, 500 + C for the one-thread kernel
// whose F_g slab and plane transforms arrive by TMA and bulk copies.
template <int N> struct Terms32Variants;
template <> struct Terms32Variants<8> { static constexpr int v[3] = {1, 2, 501}; };
template <> struct Terms32Variants<16> { static constexpr int v[3] = {1, 2, 501}; };
template <> struct Terms32Variants<24> { static constexpr int v[4] = {3, 4, 6, 503}; };
template <> struct Terms32Variants<32> { static constexpr int v[5] = {4, 8, 104, 108, 504}; };
template <> struct Terms32Variants<48> { static constexpr int v[3] = {16, 116, 516}; };

template <int N>
static int launch_terms32(int c, const VhsTermsArgs& a, int nevals, int Nrho,
                          cudaStream_t st, const CUtensorMap* map = nullptr) {
  if constexpr (N == 8 || N == 16) {
    if (c == 1) return launch_terms32_c<N, 1>(a, nevals, Nrho, st);
    if (c == 2) return launch_terms32_c<N, 2>(a, nevals, Nrho, st);
    if (c == 501) return launch_terms32_c<N, 1, true>(a, nevals, Nrho, st, map);
  } else if constexpr (N == 24) {
    if (c == 503) return launch_terms32_c<N, 3, true>(a, nevals, Nrho, st, map);
    if (c == 3) return launch_terms32_c<N, 3>(a, nevals, Nrho, st);
    if (c == 4) return launch_terms32_c<N, 4>(a, nevals, Nrho, st);
    if (c == 6) return launch_terms32_c<N, 6>(a, nevals, Nrho, st);
  } else if constexpr (N == 32) {
    if (c == 4) return launch_terms32_c<N, 4>(a, nevals, Nrho, st);
    if (c == 8) return launch_terms32_c<N, 8>(a, nevals, Nrho, st);
    if (c == 104) return launch_terms32s_c<N, 4>(a, nevals, Nrho, st);
    if (c == 108) return launch_terms32s_c<N, 8>(a, nevals, Nrho, st);
    if (c == 504) return launch_terms32_c<N, 4, true>(a, nevals, Nrho, st, map);
  } else if constexpr (N == 48) {
    if (c == 16) return launch_terms32_c<N, 16>(a, nevals, Nrho, st);
    if (c == 116) return launch_terms32s_c<N, 16>(a, nevals, Nrho, st);
    if (c == 516) return launch_terms32_c<N, 16, true>(a, nevals, Nrho, st, map);
  }
  return fail(DGFS_ERR_UNSUPPORTED, "terms kernel cluster size not compiled in");
}

// One component of the bilinear form: the pipeline transforms
// alpha f + beta g and adds prefac (cg Re G - cl f Re Lf) (dgfs_vhs_eval2).
struct VhsBilin {
  const void* g;
  double alpha, beta, cg, cl;
};

template <int N>
static int vhs_run(dgfs_vhs_s* h, const void* f, int f_double, void* Q,
                   int q_double, const int32_t* src_slots, int src_base,
                   const int32_t* dst_slots, int dst_base, int nevals,
                   cudaStream_t st, const VhsBilin* bl = nullptr,
                   const void* const* f_list = nullptr,
                   void* const* q_list = nullptr) {
  constexpr int C64 = VhsClusters<N>::c64 > 0 ? VhsClusters<N>::c64 : 1;
  constexpr bool HAS64 = VhsClusters<N>::c64 > 0;
  constexpr int C32 = VhsClusters<N>::c32;
  constexpr int CPRO = VhsClusters<N>::cpro;
  constexpr int CEPI = VhsClusters<N>::cepi;
  using G64 = Geo<N, C64>;
  using GPRO = Geo<N, CPRO>;
  using GEPI = Geo<N, CEPI>;
  using G32 = Geo<N, C32>;
  const bool fp32 = h->precision == DGFS_PREC_FP32;
  int rc;
  int evi = 0;
  auto mark = [&]() {
    if (h->profile) cudaEventRecord(h->ev[evi++], st);
  };
  mark();
  // prologue
  {
    VhsPrologueArgs a{};
    a.f = f; a.f_list = f_list; a.f_double = f_double;
    a.src_slots = src_slots; a.src_base = src_base;
    a.c0 = h->c0; a.b2 = h->b2; a.cw = h->cw; a.split = fp32 ? 1 : 0;
    a.Fg = h->Fg; a.ReLf = h->ReLf; a.mhat = h->mhat; a.moments = h->moments;
    a.Fny = h->Fny;
    if (bl) { a.g = bl->g; a.alpha = bl->alpha; a.beta = bl->beta; }
    const size_t smem = prologue_smem<N, CPRO>();
    if ((rc = launch_cluster(vhs_prologue_kernel<N, CPRO>, dim3(CPRO, nevals),
                             dim3(GPRO::NT), CPRO, smem, st, a)))
      return rc;
  }
  mark();
  if (fp32) {
    // aux: tables (needs the prologue's Maxwellian spectra)
    DGFS_CUDA(cudaEventRecord(h->fork0, st));
    DGFS_CUDA(cudaStreamWaitEvent(h->aux, h->fork0, 0));
    VhsTablesArgs t{};
    t.mhat = h->mhat; t.mult = h->mult; t.kappa = h->kappa; t.uv = h->uv;
    t.hh = h->hh;
    t.Mu = h->Mu; t.Nrho = h->Nrho; t.nevals = nevals; t.uv_double = 0;
    const int total = nevals * h->Nrho * h->Mu * 3;
    if ((rc = launch_plain(vhs_tables_kernel<N>, dim3((total + 95) / 96),
                           dim3(96), 0, h->aux, t)))
      return rc;
    DGFS_CUDA(cudaEventRecord(h->tab, h->aux));
    // caller's stream: Nyquist-plane transforms, concurrently with the tables
    VhsTermsArgs a{};
    a.Fg = h->Fg; a.ph = h->ph; a.uv = h->uv; a.mult = h->mult;
    a.b1w = h->b1w32; a.H = h->H; a.Mu = h->Mu; a.Nrho = h->Nrho;
    a.nyq = h->nyq32; a.rho = h->rho; a.Fny = h->Fny; a.err = h->err;
    const size_t psmem = (size_t)(9 * N * (N + 1) + 2 * (3 * N + 3)) * sizeof(float2);
    if ((rc = launch_plain(vhs_nyq_planes_kernel<N>,
                           dim3((h->Mu + 1) / 2, h->Nrho, nevals), dim3(6 * N),
                           psmem, st, a)))
      return rc;
    DGFS_CUDA(cudaStreamWaitEvent(st, h->tab, 0));
    mark();
    // hi: terms
    DGFS_CUDA(cudaEventRecord(h->fork1, st));
    DGFS_CUDA(cudaStreamWaitEvent(h->hi, h->fork1, 0));
    if (h->profile) cudaEventRecord(h->ev[evi++], h->hi);
    // default: the TMA variant at the default cluster size, when its map
    // could be made
    const int c = h->c32 ? h->c32 : (h->fg_map_ok ? 500 + C32 : C32);
    if ((rc = launch_terms32<N>(c, a, nevals, h->Nrho, h->hi,
                                h->fg_map_ok ? &h->fg_map : nullptr)))
      return rc;
    if (h->profile) cudaEventRecord(h->ev[evi++], h->hi);
    DGFS_CUDA(cudaEventRecord(h->join_hi, h->hi));
    // aux (after the tables, and not before the terms kernel is launched, so
    // that it does not take SMs from the Nyquist-plane kernel): Maxwellian
    // gain, behind the terms kernel on the SMs its clusters leave free
    DGFS_CUDA(cudaStreamWaitEvent(h->aux, h->fork1, 0));
    VhsGainArgs g{};
    g.hh = h->hh; g.mult = h->mult; g.b1w = h->b1w64; g.GM = h->GM;
    g.Mu = h->Mu; g.Nrho = h->Nrho;
    const size_t per_p = (size_t)h->Mu * (2 * N + 1) * sizeof(double2);
    g.pch = (int)std::max<size_t>(1, std::min<size_t>(h->Nrho, (104 * 1024) / per_p));
    const size_t smem = per_p * g.pch;
    if (h->profile) cudaEventRecord(h->evg[0], h->aux);
    if ((rc = launch_plain(vhs_maxwell_gain_kernel<N>, dim3(N, nevals),
                           dim3(GainGeo<N>::NT), smem, h->aux, g)))
      return rc;
    if (h->profile) cudaEventRecord(h->evg[1], h->aux);
    DGFS_CUDA(cudaEventRecord(h->join_aux, h->aux));
    DGFS_CUDA(cudaStreamWaitEvent(st, h->join_hi, 0));
    DGFS_CUDA(cudaStreamWaitEvent(st, h->join_aux, 0));
  } else {
    mark(); mark();  // no tables / Maxwellian-gain stages in FP64 mode
    if constexpr (HAS64) {
      VhsTermsArgs a{};
      a.Fg = h->Fg; a.ph = h->ph; a.uv = nullptr; a.mult = h->mult;
      a.b1w = h->b1w64; a.H = h->H; a.Mu = h->Mu; a.Nrho = h->Nrho;
      constexpr size_t kSmemMax = 232448;  // 227 KB per CTA
      constexpr size_t smem3 = 3 * (size_t)G64::SLAB * sizeof(double2) +
                               9 * N * sizeof(double2);
      if constexpr (smem3 <= kSmemMax) {
        if ((rc = launch_cluster(vhs_terms_kernel<double, N, C64, false>,
                                 dim3(C64, h->Nrho, nevals), dim3(G64::NT), C64,
                                 smem3, st, a)))
          return rc;
      } else {
        constexpr size_t smem2 = 2 * (size_t)G64::SLAB * sizeof(double2) +
                                 3 * N * sizeof(double2);
        static_assert(smem2 <= kSmemMax, "FP64 terms slabs exceed shared memory");
        if ((rc = launch_cluster(vhs_terms_fp64g_kernel<N, C64>,
                                 dim3(C64, h->Nrho, nevals), dim3(G64::NT), C64,
                                 smem2, st, a)))
          return rc;
      }
    } else {
      return fail(DGFS_ERR_UNSUPPORTED, "no FP64 terms kernel at this N");
    }
    mark();
  }
  // epilogue
  {
    VhsEpilogueArgs a{};
    a.H = h->H; a.h_double = fp32 ? 0 : 1; a.GM = fp32 ? h->GM : nullptr;
    a.ReLf = h->ReLf; a.f = f; a.f_list = f_list; a.f_double = f_double;
    a.src_slots = src_slots; a.src_base = src_base;
    a.Q = Q; a.q_list = q_list; a.q_double = q_double;
    a.dst_slots = dst_slots; a.dst_base = dst_base;
    a.prefac = h->prefac;
    a.Nrho = fp32 ? (h->Nrho + 1) / 2 : h->Nrho;  // FP32: packed radial pairs
    a.project = h->project; a.c0 = h->c0; a.cw = h->cw;
    for (int i = 0; i < 25; ++i) a.Ginv[i] = h->Ginv[i];
    if (bl) { a.bilinear = 1; a.cg = bl->cg; a.cl = bl->cl; }
    const size_t smem = epilogue_smem<N, CEPI>();
    if ((rc = launch_cluster(vhs_epilogue_kernel<N, CEPI>, dim3(CEPI, nevals),
                             dim3(GEPI::NT), CEPI, smem, st, a)))
      return rc;
  }
  mark();
  h->ev_used = evi;
  return DGFS_OK;
}

static int vhs_eval_impl(dgfs_vhs_handle h, const void* f, int32_t f_dtype,
                         void* Q, int32_t q_dtype, const int32_t* src_slots,
                         int32_t src_base, const int32_t* dst_slots,
                         int32_t dst_base, int32_t nevals, void* stream,
                         const VhsBilin* bl, const void* const* f_list = nullptr,
                         void* const* q_list = nullptr);

extern "C" int dgfs_vhs_eval(dgfs_vhs_handle h, const void* f, int32_t f_dtype,
                             void* Q, int32_t q_dtype,
                             const int32_t* src_slots, int32_t src_base,
                             const int32_t* dst_slots, int32_t dst_base,
                             int32_t nevals, void* stream) {
  NvtxRange nvtx_range("dgfs_vhs_eval");
  return vhs_eval_impl(h, f, f_dtype, Q, q_dtype, src_slots, src_base,
                       dst_slots, dst_base, nevals, stream, nullptr);
}

// Bilinear Q(f, g) of `vhs` (std/scattering.py:346-429): gain
// B(f, g) = sum_pq FFT(IFFT(cos a F) IFFT(cos a G) + IFFT(sin a F) IFFT(sin a G))
// (weighted by b1), loss f Re IFFT(b2 G).  B is symmetric and bilinear with
// B(h, h) the gain of Q(h, h), so it is evaluated by polarisation through
// the Q(h, h) pipeline, whose kernels are unchanged:
//   FP64: B(f, g) = (B(f+g, f+g) - B(f-g, f-g)) / 4, and by linearity
//         Re IFFT(b2 G) = (Lf(f+g) - Lf(f-g)) / 2  (two passes);
//   FP32: B(f, g) = (B(f+g, f+g) - B(f, f) - B(g, g)) / 2, loss from the g
//         pass (three passes: every transformed input stays close to a
//         Maxwellian, which the split of the FP32 mode needs; f - g is
//         not).
// Each pass adds prefac (cg Re G_h - cl f Re Lf_h) into Q.
extern "C" int dgfs_vhs_eval2(dgfs_vhs_handle h, const void* f, const void* g,
                              int32_t f_dtype, void* Q, int32_t q_dtype,
                              const int32_t* src_slots, int32_t src_base,
                              const int32_t* dst_slots, int32_t dst_base,
                              int32_t nevals, void* stream) {
  NvtxRange nvtx_range("dgfs_vhs_eval2");
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (!g) return fail(DGFS_ERR_INVALID, "null g");
  const bool fp32 = h->precision == DGFS_PREC_FP32;
  const VhsBilin p64[2] = {{g, 1.0, 1.0, 0.25, 0.5},
                           {g, 1.0, -1.0, -0.25, -0.5}};
  const VhsBilin p32[3] = {{g, 1.0, 1.0, 0.5, 0.0},
                           {g, 1.0, 0.0, -0.5, 0.0},
                           {g, 0.0, 1.0, -0.5, 1.0}};
  const VhsBilin* parts = fp32 ? p32 : p64;
  const int np = fp32 ? 3 : 2;
  for (int i = 0; i < np; ++i)
    if (int rc = vhs_eval_impl(h, f, f_dtype, Q, q_dtype, src_slots, src_base,
                               dst_slots, dst_base, nevals, stream, parts + i))
      return rc;
  return DGFS_OK;
}

extern "C" int dgfs_vhs_fs2(dgfs_vhs_handle h, const void* f, const void* g,
                            void* Q, int32_t dtype, int32_t Ne, int32_t elem,
                            int32_t modein, int32_t modeout, void* stream) {
  if (Ne <= 0 || elem < 0 || elem >= Ne || modein < 0 || modeout < 0)
    return fail(DGFS_ERR_INVALID, "bad Ne/elem/mode");
  return dgfs_vhs_eval2(h, f, g, dtype, Q, dtype, nullptr, modein * Ne + elem,
                        nullptr, modeout * Ne + elem, 1, stream);
}

// Q(f, f) for a list of (array, slot) pairs: f_list and q_list are device
// arrays of nevals pointers, evaluation i reading slot src(i) of f_list[i]
// and adding into slot dst(i) of q_list[i] -- points of several problems
// that share one operator (same grid, rules and parameters) in one launch
// sequence.
extern "C" int dgfs_vhs_eval_multi(dgfs_vhs_handle h, const void* const* f_list,
                                   int32_t f_dtype, void* const* q_list,
                                   int32_t q_dtype, const int32_t* src_slots,
                                   int32_t src_base, const int32_t* dst_slots,
                                   int32_t dst_base, int32_t nevals,
                                   void* stream) {
  NvtxRange nvtx_range("dgfs_vhs_eval_multi");
  if (!f_list || !q_list) return fail(DGFS_ERR_INVALID, "null array lists");
  return vhs_eval_impl(h, nullptr, f_dtype, nullptr, q_dtype, src_slots,
                       src_base, dst_slots, dst_base, nevals, stream, nullptr,
                       f_list, q_list);
}

static int vhs_eval_impl(dgfs_vhs_handle h, const void* f, int32_t f_dtype,
                         void* Q, int32_t q_dtype, const int32_t* src_slots,
                         int32_t src_base, const int32_t* dst_slots,
                         int32_t dst_base, int32_t nevals, void* stream,
                         const VhsBilin* bl, const void* const* f_list,
                         void* const* q_list) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (nevals < 0) return fail(DGFS_ERR_INVALID, "negative nevals");
  if (nevals == 0) return DGFS_OK;
  if ((!f && !f_list) || (!Q && !q_list)) return fail(DGFS_ERR_INVALID, "null f or Q");
  if ((f_dtype != DGFS_F32 && f_dtype != DGFS_F64) ||
      (q_dtype != DGFS_F32 && q_dtype != DGFS_F64))
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  if (src_base < 0 || dst_base < 0)
    return fail(DGFS_ERR_INVALID, "negative slot base");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int off = 0; off < nevals; off += h->max_evals) {
    const int cnt = std::min(h->max_evals, nevals - off);
    const int32_t* ss = src_slots ? src_slots + off : nullptr;
    const int32_t* ds = dst_slots ? dst_slots + off : nullptr;
    const void* const* fl = f_list ? f_list + off : nullptr;
    void* const* ql = q_list ? q_list + off : nullptr;
    int rc;
    switch (h->N) {
      case 8: rc = vhs_run<8>(h, f, f_dtype, Q, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, bl, fl, ql); break;
      case 16: rc = vhs_run<16>(h, f, f_dtype, Q, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, bl, fl, ql); break;
      case 24: rc = vhs_run<24>(h, f, f_dtype, Q, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, bl, fl, ql); break;
      case 32: rc = vhs_run<32>(h, f, f_dtype, Q, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, bl, fl, ql); break;
      case 48: rc = vhs_run<48>(h, f, f_dtype, Q, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, bl, fl, ql); break;
      default: return fail(DGFS_ERR_UNSUPPORTED, "N not compiled in");
    }
    if (rc) return rc;
  }
  return DGFS_OK;
}

extern "C" int dgfs_vhs_fs(dgfs_vhs_handle h, const void* f, void* Q,
                           int32_t dtype, int32_t Ne, int32_t elem,
                           int32_t modein, int32_t modeout, void* stream) {
  if (Ne <= 0 || elem < 0 || elem >= Ne || modein < 0 || modeout < 0)
    return fail(DGFS_ERR_INVALID, "bad Ne/elem/mode");
  return dgfs_vhs_eval(h, f, dtype, Q, dtype, nullptr, modein * Ne + elem,
                       nullptr, modeout * Ne + elem, 1, stream);
}

// ---------------------------------------------------------------------------
// profiling helpers
// ---------------------------------------------------------------------------
extern "C" int dgfs_vhs_profile(dgfs_vhs_handle h, int32_t enable) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (enable && !h->ev[0]) {
    for (auto& e : h->ev) DGFS_CUDA(cudaEventCreate(&e));
    for (auto& e : h->evg) DGFS_CUDA(cudaEventCreate(&e));
  }
  h->profile = enable != 0;
  return DGFS_OK;
}

extern "C" int dgfs_vhs_stage_ms(dgfs_vhs_handle h, double* out5) {
  if (!h || !out5) return fail(DGFS_ERR_INVALID, "null argument");
  if (!h->profile || h->ev_used != 6)
    return fail(DGFS_ERR_INVALID, "profiling was not enabled for the last call");
  DGFS_CUDA(cudaEventSynchronize(h->ev[5]));
  for (int i = 0; i < 5; ++i) {
    float ms = 0.f;
    DGFS_CUDA(cudaEventElapsedTime(&ms, h->ev[i], h->ev[i + 1]));
    out5[i] = ms;
  }
  if (h->precision == DGFS_PREC_FP32) {
    // the gain kernel runs on the forked stream: report its own span, and
    // the terms stage as the span from the fork point to the terms end
    float ms = 0.f;
    DGFS_CUDA(cudaEventElapsedTime(&ms, h->evg[0], h->evg[1]));
    out5[3] += out5[2];
    out5[2] = ms;
  }
  return DGFS_OK;
}

// FP32 fused multiply-add throughput of the current GPU (TFLOP/s), measured
// with independent FMA chains on every SM; the roofline denominator of the
// FFT-bound kernels.
__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters) {
  float a0 = threadIdx.x * 1e-3f, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
  float a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const float b = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c);
      a3 = fmaf(a3, b, c); a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c);
      a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[0] = s;  // keep the chains alive
}

extern "C" int dgfs_fma_peak(double* tflops, void* stream) {
  if (!tflops) return fail(DGFS_ERR_INVALID, "null output");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  DGFS_CUDA(cudaGetDevice(&dev));
  DGFS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  float* out = nullptr;
  DGFS_CUDA(cudaMalloc(&out, sizeof(float)));
  const int iters = 4096, blocks = sms * 8, threads = 256;
  cudaEvent_t e0, e1;
  DGFS_CUDA(cudaEventCreate(&e0));
  DGFS_CUDA(cudaEventCreate(&e1));
  fma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters / 8);  // warm-up
  DGFS_CUDA(cudaEventRecord(e0, st));
  fma_peak_kernel<<<blocks, threads, 0, st>>>(out, iters);
  DGFS_CUDA(cudaEventRecord(e1, st));
  DGFS_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  DGFS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return DGFS_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free VHS evaluation.
//
// For callers that cannot allocate device memory -- services whose device
// memory is a fixed pool carved out at start-up, plugins loaded into a
// process that forbids cudaMalloc once it is serving, and time loops that
// cannot afford cudaMalloc's implicit device synchronisation.  All scratch of the FP64
// evaluation (tables and per-evaluation buffers) lives in one file-scope
// device array of kNoallocBytes; every GPU that loads this library holds it
// until the process exits.  The array is shared by every call: two calls
// whose kernels overlap on the GPU (different streams, no ordering) race on
// it.  Nothing in it needs to start at zero: each call rebuilds the tables
// and every buffer is fully written before it is read.
// ---------------------------------------------------------------------------
static constexpr size_t kNoallocBytes = size_t(16) << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

static constexpr int kNoallocMaxNrho = 48;
static constexpr int kNoallocMaxMu = 96;

struct NoallocTableArgs {
  double* b1w;       // [Nrho][n]
  double* b2;        // [n]
  double2* ph;       // [Nrho][Mu][3][N]
  float* mult_out;   // [Mu]
  double L, gamma, sw, sphere_factor, sinc_eps;
  int Nrho, Mu;
  double qz[kNoallocMaxNrho];
  double qw[kNoallocMaxNrho];
  double sz[kNoallocMaxMu * 3];  // unique directions
  float mult[kNoallocMaxMu];     // their multiplicities
};

// b1 (weighted), b2 and the 1-D phase tables of vhs-gll.mako:43-99, built on
// the device from the descriptor values carried in the kernel parameters.
template <int N>
__global__ void noalloc_tables_kernel(NoallocTableArgs a) {
  constexpr int n = N * N * N;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  auto rep = [](int i) { return (double)((i < N / 2) ? i : i - N); };
  if (gid < n) {
    const int ix = gid / (N * N), iy = (gid / N) % N, iz = gid % N;
    const double cS = sqrt(rep(ix) * rep(ix) + rep(iy) * rep(iy) +
                           rep(iz) * rep(iz));
    double bsum = 0.0;
    for (int p = 0; p < a.Nrho; ++p) {
      const double qz = a.qz[p];
      const double s1 = M_PI / a.L * qz / 2. * cS + a.sinc_eps;
      const double s2 = M_PI / a.L * qz * cS + a.sinc_eps;
      const double b1 = pow(qz, a.gamma + 2.) * 4 * M_PI * (sin(s1) / s1);
      a.b1w[(size_t)p * n + gid] = (a.sphere_factor * a.qw[p] * a.sw / n) * b1;
      bsum += a.qw[p] * pow(qz, a.gamma + 2.) * 16 * M_PI * M_PI * (sin(s2) / s2);
    }
    a.b2[gid] = bsum;
  }
  if (gid < a.Mu) a.mult_out[gid] = a.mult[gid];
  const int nph = a.Nrho * a.Mu * 3 * N;
  if (gid < nph) {
    const int l = gid % N, ax = (gid / N) % 3, u = (gid / (3 * N)) % a.Mu,
              p = gid / (3 * N * a.Mu);
    const double k = M_PI / a.L * a.qz[p] / 2. * a.sz[3 * u + ax];
    double s, c;
    sincos(k * rep(l), &s, &c);
    a.ph[gid] = make_double2(c, s);
  }
}

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_ptr[64];  // device address per device id

// Per-device set-up, done by the first call on each device: upload the FFT
// twiddles from static host buffers and resolve the device address of the
// scratch array (its name is only a host-side stand-in in host code).
static int noalloc_setup(unsigned char** out) {
  int dev = 0;
  DGFS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(DGFS_ERR_INVALID, "device id out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    static double2 t64[kTwTotal];
    static float2 t32[kTwTotal];
    std::lock_guard<std::mutex> lk2(g_tw_mu);
    if (!g_tw_done[dev]) {
      for (int i = 0; i < kNumTw; ++i) {
        const int nt = tw_size(i), off = tw_offset(nt);
        for (int k = 0; k < nt; ++k) {
          const long double ang = 2.0L * 3.141592653589793238462643383279502884L *
                                  (long double)k / (long double)nt;
          const double c = (double)std::cos(ang), s = -(double)std::sin(ang);
          t64[off + k] = make_double2(c, s);
          t32[off + k] = make_float2((float)c, (float)s);
        }
      }
      DGFS_CUDA(cudaMemcpyToSymbol(c_tw64, t64, sizeof(t64)));
      DGFS_CUDA(cudaMemcpyToSymbol(c_tw32, t32, sizeof(t32)));
      if (int rc = settle_uploads()) return rc;
      g_tw_done[dev] = true;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(DGFS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                     cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return DGFS_OK;
}

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

extern "C" int dgfs_vhs_eval_noalloc(const dgfs_vhs_desc* d, const double* f,
                                     double* Q, const int32_t* src_slots,
                                     int32_t src_base, const int32_t* dst_slots,
                                     int32_t dst_base, int32_t nevals,
                                     void* stream) {
  if (!d) return fail(DGFS_ERR_INVALID, "null descriptor");
  if (nevals < 0 || src_base < 0 || dst_base < 0)
    return fail(DGFS_ERR_INVALID, "negative nevals or slot base");
  if (d->precision != DGFS_PREC_FP64)
    return fail(DGFS_ERR_UNSUPPORTED, "the allocation-free path is FP64 only");
  if (d->N != 8 && d->N != 16 && d->N != 32)
    return fail(DGFS_ERR_UNSUPPORTED, "N must be 8, 16 or 32");
  if (d->Nrho <= 0 || d->Nrho > kNoallocMaxNrho || d->M <= 0 ||
      !d->qz || !d->qw || !d->sz)
    return fail(DGFS_ERR_INVALID, "bad Nrho, M or rule arrays");
  if (nevals == 0) return DGFS_OK;
  if (!f || !Q) return fail(DGFS_ERR_INVALID, "null f or Q");

  NoallocTableArgs ta{};
  float* mult = ta.mult;
  bool used[4 * kNoallocMaxMu] = {};
  if (d->M > 4 * kNoallocMaxMu)
    return fail(DGFS_ERR_CAPACITY, "M exceeds the allocation-free maximum");
  int Mu = 0;
  for (int q = 0; q < d->M; ++q) {
    if (used[q]) continue;
    used[q] = true;
    float m = 1.f;
    for (int r = q + 1; r < d->M; ++r)
      if (!used[r] && d->sz[3 * r] == -d->sz[3 * q] &&
          d->sz[3 * r + 1] == -d->sz[3 * q + 1] &&
          d->sz[3 * r + 2] == -d->sz[3 * q + 2]) {
        used[r] = true;
        m = 2.f;
        break;
      }
    if (Mu >= kNoallocMaxMu)
      return fail(DGFS_ERR_CAPACITY, "too many sphere directions");
    for (int a = 0; a < 3; ++a) ta.sz[3 * Mu + a] = d->sz[3 * q + a];
    mult[Mu++] = m;
  }
  const int N = d->N, n = N * N * N, Nrho = d->Nrho;
  // layout of the scratch array: tables, then per-evaluation buffers
  const size_t b_b1w = align256(sizeof(double) * Nrho * n);
  const size_t b_b2 = align256(sizeof(double) * n);
  const size_t b_ph = align256(sizeof(double2) * Nrho * Mu * 3 * N);
  const size_t b_mult = align256(sizeof(float) * Mu);
  const size_t tables = b_b1w + b_b2 + b_ph + b_mult;
  const size_t per_eval = align256(sizeof(double2) * n) +
                          align256(sizeof(double2) * Nrho * n) +
                          align256(sizeof(double) * n);
  if (tables + per_eval > kNoallocBytes)
    return fail(DGFS_ERR_CAPACITY,
                "N=" + std::to_string(N) + ", Nrho=" + std::to_string(Nrho) +
                    " needs " + std::to_string(tables + per_eval) +
                    " bytes of scratch; the allocation-free maximum is " +
                    std::to_string(kNoallocBytes));
  const int E = (int)std::min<size_t>((kNoallocBytes - tables) / per_eval, 1024);

  unsigned char* base = nullptr;
  if (int rc = noalloc_setup(&base)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // a handle that only points into the scratch array (nothing allocated)
  dgfs_vhs_s h;
  h.N = N; h.n = n; h.Nrho = Nrho; h.M = d->M; h.Mu = Mu;
  h.precision = DGFS_PREC_FP64; h.max_evals = E;
  h.prefac = d->prefac; h.cw = d->cw;
  unsigned char* p = base;
  h.b1w64 = reinterpret_cast<double*>(p); p += b_b1w;
  h.b2 = reinterpret_cast<double*>(p); p += b_b2;
  h.ph = p; p += b_ph;
  h.mult = reinterpret_cast<float*>(p); p += b_mult;
  h.Fg = p; p += align256(sizeof(double2) * n) * E;
  h.H = p; p += align256(sizeof(double2) * Nrho * n) * E;
  h.ReLf = reinterpret_cast<double*>(p);
  // (the per-eval buffers above are contiguous [E][...] blocks: every
  // per-eval size is already a multiple of 256 bytes for N >= 8)

  ta.b1w = h.b1w64; ta.b2 = h.b2; ta.ph = static_cast<double2*>(h.ph);
  ta.mult_out = h.mult;
  ta.L = d->L; ta.gamma = d->gamma; ta.sw = d->sw;
  ta.sphere_factor = d->sphere_factor; ta.sinc_eps = d->sinc_eps;
  ta.Nrho = Nrho; ta.Mu = Mu;
  for (int i = 0; i < Nrho; ++i) { ta.qz[i] = d->qz[i]; ta.qw[i] = d->qw[i]; }
  const int work = std::max(std::max(n, Nrho * Mu * 3 * N), Mu);
  int rc = DGFS_OK;
  switch (N) {
    case 8: rc = launch_plain(noalloc_tables_kernel<8>, dim3((work + 255) / 256), dim3(256), 0, st, ta); break;
    case 16: rc = launch_plain(noalloc_tables_kernel<16>, dim3((work + 255) / 256), dim3(256), 0, st, ta); break;
    default: rc = launch_plain(noalloc_tables_kernel<32>, dim3((work + 255) / 256), dim3(256), 0, st, ta); break;
  }
  if (rc) return rc;
  for (int off = 0; off < nevals; off += E) {
    const int cnt = std::min(E, nevals - off);
    const int32_t* ss = src_slots ? src_slots + off : nullptr;
    const int32_t* ds = dst_slots ? dst_slots + off : nullptr;
    switch (N) {
      case 8: rc = vhs_run<8>(&h, f, 1, Q, 1, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      case 16: rc = vhs_run<16>(&h, f, 1, Q, 1, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      default: rc = vhs_run<32>(&h, f, 1, Q, 1, ss, src_base + off, ds, dst_base + off, cnt, st); break;
    }
    if (rc) break;
  }
  // the stack handle owns nothing: detach before it goes out of scope
  h.c0 = h.b2 = h.b1w64 = h.ReLf = nullptr;
  h.b1w32 = nullptr; h.ph = h.Fg = h.H = nullptr; h.mult = nullptr;
  return rc;
}

// ---------------------------------------------------------------------------
// DG right-hand side, stage updates, moments, residual
// ---------------------------------------------------------------------------
struct dgfs_dg_s {
  DgAdvectArgs base{};
  int Nqr = 0;
  double cw = 0;
  double* c0 = nullptr;
  double* invjac = nullptr;
  double* f0[2] = {nullptr, nullptr};
  double* nden = nullptr;
  double* im = nullptr;
  double* part = nullptr;  // residual partials
  double* part_h = nullptr;
  double* wpart = nullptr;  // wall-density partials [2][kWallCh][2]
  double* lim = nullptr;    // limiter tables: wavg [K] | wdr [K] | dx [K][Ne] | h [Ne]
  double* mpart = nullptr;  // penalty-moment partials [mpts][kPmCh][<= 14]
  int mpts = 0;
};

static void free_dg(dgfs_dg_s* h) {
  void* ptrs[] = {h->c0, h->invjac, h->f0[0], h->f0[1], h->nden, h->im, h->part,
                  h->wpart, h->mpart, h->lim};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->part_h) cudaFreeHost(h->part_h);
  delete h;
}

extern "C" int dgfs_dg_create(const dgfs_dg_desc* d, dgfs_dg_handle* out) {
  if (!d || !out) return fail(DGFS_ERR_INVALID, "null descriptor or handle");
  *out = nullptr;
  if (d->K < 1 || d->K > kDgMaxK || d->Ne < 1 || d->N < 2 || d->Nqr < 1)
    return fail(DGFS_ERR_INVALID, "need 1 <= K <= 8, Ne >= 1, N >= 2, Nqr >= 1");
  if (!d->trL || !d->trR || !d->D || !d->gLD || !d->gRD || !d->invjac ||
      !d->c0 || !d->im)
    return fail(DGFS_ERR_INVALID, "missing operator arrays");
  for (int s = 0; s < 2; ++s) {
    if (d->bc_kind[s] < kBcCopy || d->bc_kind[s] > kBcWallExpr)
      return fail(DGFS_ERR_INVALID, "unknown boundary kind");
    if ((d->bc_kind[s] == kBcWall || d->bc_kind[s] == kBcInlet) && !d->bc_f0[s])
      return fail(DGFS_ERR_INVALID, "wall/inlet boundary needs its Maxwellian");
  }
  const int K = d->K, Ne = d->Ne, N = d->N, Nv = N * N * N;
  auto* h = new dgfs_dg_s();
  DgAdvectArgs& a = h->base;
  a.K = K; a.Ne = Ne; a.Nv = Nv; a.N = N;
  for (int k = 0; k < K; ++k) {
    a.trL[k] = d->trL[k]; a.trR[k] = d->trR[k];
    a.gLD[k] = d->gLD[k]; a.gRD[k] = d->gRD[k];
    for (int m = 0; m < K; ++m) a.D[k * K + m] = d->D[k * K + m];
  }
  for (int s = 0; s < 2; ++s) {
    a.bc[s] = d->bc_kind[s];
    a.bc_ux[s] = d->bc_ux[s];
    a.nl[s] = s == 0 ? -1.0 : 1.0;
    a.ws[s][0] = a.ws[s][1] = a.ws[s][2] = 0.0;
    a.ws[s][3] = a.ws[s][4] = 1.0;
  }
  h->Nqr = d->Nqr;
  h->cw = d->cw;
  int rc = DGFS_OK;
  std::vector<double> c0(d->c0, d->c0 + N), ij(d->invjac, d->invjac + Ne),
      im(d->im, d->im + (size_t)K * d->Nqr);
  if ((rc = upload(&h->c0, c0)) || (rc = upload(&h->invjac, ij)) ||
      (rc = upload(&h->im, im))) {
    free_dg(h);
    return rc;
  }
  for (int s = 0; s < 2; ++s)
    if (d->bc_f0[s]) {
      std::vector<double> f0(d->bc_f0[s], d->bc_f0[s] + Nv);
      if ((rc = upload(&h->f0[s], f0))) { free_dg(h); return rc; }
    }
  cudaError_t e1 = cudaMalloc(&h->nden, 2 * sizeof(double));
  if (e1 == cudaSuccess) e1 = cudaMalloc(&h->part, 2 * 1024 * sizeof(double));
  if (e1 == cudaSuccess) e1 = cudaMallocHost(&h->part_h, 2 * 1024 * sizeof(double));
  if (e1 == cudaSuccess) e1 = cudaMalloc(&h->wpart, 2 * kWallCh * 2 * sizeof(double));
  h->mpts = std::max(K, d->Nqr) * Ne;
  if (e1 == cudaSuccess)
    e1 = cudaMalloc(&h->mpart, (size_t)h->mpts * kPmCh * kPmMaxNa * sizeof(double));
  if (e1 != cudaSuccess) {
    free_dg(h);
    return fail(DGFS_ERR_CUDA, std::string("allocation: ") + cudaGetErrorString(e1));
  }
  a.c0 = h->c0; a.invjac = h->invjac;
  a.f0[0] = h->f0[0]; a.f0[1] = h->f0[1];
  a.nden = h->nden;
  if (int rc_s = settle_uploads()) { free_dg(h); return rc_s; }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_dg_destroy(dgfs_dg_handle h) {
  if (h) free_dg(h);
  return DGFS_OK;
}

extern "C" int dgfs_dg_advect(dgfs_dg_handle h, const void* u, void* ux,
                              int32_t dtype, void* stream) {
  NvtxRange nvtx_range("dgfs_dg_advect");
  if (!h || !u || !ux) return fail(DGFS_ERR_INVALID, "null argument");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  if (u == ux) return fail(DGFS_ERR_INVALID, "u and ux must not alias");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DgAdvectArgs a = h->base;
  a.u = u; a.ux = ux; a.f_double = dtype == DGFS_F64;
  dg_wall_partial_kernel<<<dim3(kWallCh, 2), 256, 0, st>>>(a, h->cw, h->wpart);
  dg_wall_final_kernel<<<1, 32, 0, st>>>(a, h->wpart, h->nden);
  DGFS_CUDA(cudaGetLastError());
  const dim3 grid((a.Nv + 255) / 256), block(256);
  switch (a.K) {
    case 1: dg_advect_kernel<1><<<grid, block, 0, st>>>(a); break;
    case 2: dg_advect_kernel<2><<<grid, block, 0, st>>>(a); break;
    case 3: dg_advect_kernel<3><<<grid, block, 0, st>>>(a); break;
    case 4: dg_advect_kernel<4><<<grid, block, 0, st>>>(a); break;
    case 5: dg_advect_kernel<5><<<grid, block, 0, st>>>(a); break;
    case 6: dg_advect_kernel<6><<<grid, block, 0, st>>>(a); break;
    case 7: dg_advect_kernel<7><<<grid, block, 0, st>>>(a); break;
    default: dg_advect_kernel<8><<<grid, block, 0, st>>>(a); break;
  }
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_dg_set_wall_state(dgfs_dg_handle h, int32_t side,
                                      double ux, double uy, double uz,
                                      double T, double mass) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (side < 0 || side > 1) return fail(DGFS_ERR_INVALID, "side must be 0 or 1");
  if (h->base.bc[side] != kBcWallExpr)
    return fail(DGFS_ERR_INVALID, "boundary is not a dgfs-wall-expr-diffuse wall");
  if (!(T > 0) || !(mass > 0))
    return fail(DGFS_ERR_INVALID, "wall temperature and mass must be > 0");
  double* w = h->base.ws[side];
  w[0] = ux; w[1] = uy; w[2] = uz; w[3] = T; w[4] = mass;
  return DGFS_OK;
}

extern "C" int dgfs_dg_wall_density(dgfs_dg_handle h, double* out2) {
  if (!h || !out2) return fail(DGFS_ERR_INVALID, "null argument");
  DGFS_CUDA(cudaMemcpy(out2, h->nden, 2 * sizeof(double), cudaMemcpyDeviceToHost));
  return DGFS_OK;
}

extern "C" int dgfs_dg_moments(dgfs_dg_handle h, const void* coeff,
                               int32_t dtype, double* out, void* stream) {
  if (!h || !coeff || !out) return fail(DGFS_ERR_INVALID, "null argument");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  MomentArgs m{};
  m.coeff = coeff; m.f_double = dtype == DGFS_F64;
  m.K = h->base.K; m.Ne = h->base.Ne; m.Nv = h->base.Nv; m.N = h->base.N;
  m.Nqr = h->Nqr; m.im = h->im; m.c0 = h->c0; m.cw = h->cw; m.out = out;
  std_moments_kernel<<<dim3(h->Nqr, h->base.Ne), 256, 0,
                       static_cast<cudaStream_t>(stream)>>>(m);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_dg_moments_bi(dgfs_dg_handle h, const void* const* coeffs,
                                  int32_t nspcs, const double* masses,
                                  int32_t dtype, double* out, void* stream) {
  if (!h || !coeffs || !masses || !out) return fail(DGFS_ERR_INVALID, "null argument");
  if (nspcs < 1 || nspcs > kMaxSpecies)
    return fail(DGFS_ERR_INVALID, "need 1 <= nspcs <= 4");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  BiMomentArgs m{};
  for (int p = 0; p < nspcs; ++p) {
    if (!coeffs[p]) return fail(DGFS_ERR_INVALID, "null species solution");
    if (!(masses[p] > 0)) return fail(DGFS_ERR_INVALID, "species mass must be > 0");
    m.coeff[p] = coeffs[p];
    m.mass[p] = masses[p];
  }
  m.f_double = dtype == DGFS_F64; m.nspcs = nspcs;
  m.K = h->base.K; m.Ne = h->base.Ne; m.Nv = h->base.Nv; m.N = h->base.N;
  m.Nqr = h->Nqr; m.im = h->im; m.c0 = h->c0; m.cw = h->cw; m.out = out;
  auto st = static_cast<cudaStream_t>(stream);
  bi_moments_pass1_kernel<<<dim3(h->Nqr, h->base.Ne, nspcs), 256, 0, st>>>(m);
  DGFS_CUDA(cudaGetLastError());
  bi_moments_pass2_kernel<<<dim3(h->Nqr, h->base.Ne), 256, 0, st>>>(m);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_axnpby(void* x0, int64_t n, int32_t dtype, double a0,
                           int32_t nterms, const void* const* xs,
                           const double* as, void* stream) {
  if (!x0 || n < 0 || nterms < 1 || nterms > kAxMax || !xs || !as)
    return fail(DGFS_ERR_INVALID, "bad axnpby arguments (1..4 terms)");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  AxnpbyArgs a{};
  a.x0 = x0; a.a0 = a0; a.nterms = nterms; a.f_double = dtype == DGFS_F64;
  a.n = (size_t)n;
  for (int i = 0; i < nterms; ++i) {
    if (!xs[i]) return fail(DGFS_ERR_INVALID, "null axnpby operand");
    a.x[i] = xs[i];
    a.a[i] = as[i];
  }
  if (n == 0) return DGFS_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t want = ((size_t)n + 255) / 256;
  const unsigned blocks = (unsigned)std::min<size_t>(want, (size_t)sms * 16);
  axnpby_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_dg_residual(dgfs_dg_handle h, const void* x, const void* y,
                                int64_t n, int32_t dtype, double* out2,
                                void* stream) {
  if (!h || !x || !y || !out2 || n < 0)
    return fail(DGFS_ERR_INVALID, "bad residual arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = 512;
  residual_kernel<<<blocks, 512, 0, st>>>(x, y, dtype == DGFS_F64, (size_t)n,
                                          h->part);
  DGFS_CUDA(cudaGetLastError());
  DGFS_CUDA(cudaMemcpyAsync(h->part_h, h->part, 2 * blocks * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  DGFS_CUDA(cudaStreamSynchronize(st));
  double a = 0, b = 0;
  for (int i = 0; i < blocks; ++i) { a += h->part_h[2 * i]; b += h->part_h[2 * i + 1]; }
  out2[0] = a;
  out2[1] = b;
  return DGFS_OK;
}

// ---------------------------------------------------------------------------
// VSS binary-mixture operator
// ---------------------------------------------------------------------------
struct VssPair {
  double2* b = nullptr;    // [Nrho][M][n]
  double2* c = nullptr;    // [n]
  double2* ph = nullptr;   // [Nrho][M][2][3][N]
  float2* b32 = nullptr;   // FP32 mode: FP32 copies of b and ph
  float2* ph32 = nullptr;
  double prefac = 0;
};

struct dgfs_vss_s {
  int N = 0, Nrho = 0, M = 0, nspcs = 0, n = 0, max_evals = 0;
  int precision = DGFS_PREC_FP64;
  double* w = nullptr;     // [Nrho] w_r s_w / n
  VssPair pair[16];
  double2* F[2] = {nullptr, nullptr};  // [E][n] spectra of the two inputs
  // FP32 mode scratch (Maxwellian split): per input slot s (the two inputs
  // of a pair, or every species of dgfs_vss_eval_species) F_g, spectra and
  // moments; per partner q of a species (slice q) the loss, tables, FP64
  // Maxwellian gain and the FP32 terms
  double* c0 = nullptr;                // [N]
  double* b2dummy = nullptr;           // [n] unused real loss kernel
  float2* Fg[4] = {};                  // [E][n]
  double2* mhat[4] = {};               // [E][3][N]
  double* mom[4] = {};                 // [E][5]
  double* ReLf = nullptr;              // [nspcs][E][n]
  float2* uv = nullptr;                // [nspcs][E][T][2][3][N]
  double2* hh = nullptr;               // [nspcs][E][T][3][N]
  double2* GM = nullptr;               // [nspcs][E][n]
  float2* H = nullptr;                 // [nspcs][E][Nrho][n]
  double cw = 0;
  // the FP64 Maxwellian gain of dgfs_vss_eval_species runs on `aux` (low
  // priority) beside the FP32 terms kernel
  cudaStream_t aux = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

static void free_vss(dgfs_vss_s* h) {
  for (auto& p : h->pair) {
    if (p.b) cudaFree(p.b);
    if (p.c) cudaFree(p.c);
    if (p.ph) cudaFree(p.ph);
    if (p.b32) cudaFree(p.b32);
    if (p.ph32) cudaFree(p.ph32);
  }
  void* ptrs[] = {h->w, h->F[0], h->F[1], h->c0, h->b2dummy, h->ReLf, h->uv,
                  h->hh, h->GM, h->H};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (int s = 0; s < 4; ++s)
    for (void* q : {(void*)h->Fg[s], (void*)h->mhat[s], (void*)h->mom[s]})
      if (q) cudaFree(q);
  if (h->fork) cudaEventDestroy(h->fork);
  if (h->join) cudaEventDestroy(h->join);
  if (h->aux) cudaStreamDestroy(h->aux);
  delete h;
}

// FP32 copies of a pair's weights and phases
__global__ void vss_to_fp32_kernel(const double2* in, float2* out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

template <int N> struct VssClusters;
template <> struct VssClusters<8> { static constexpr int c = 1; };
template <> struct VssClusters<16> { static constexpr int c = 2; };
template <> struct VssClusters<24> { static constexpr int c = 6; };
template <> struct VssClusters<32> { static constexpr int c = 16; };
// FP32 terms kernel: five FP32 slabs per CTA
template <int N> struct VssClusters32;
template <> struct VssClusters32<8> { static constexpr int c = 1; };
template <> struct VssClusters32<16> { static constexpr int c = 2; };
template <> struct VssClusters32<24> { static constexpr int c = 3; };
template <> struct VssClusters32<32> { static constexpr int c = 8; };

template <int N>
static int vss_setup_pair(dgfs_vss_s* h, const dgfs_vss_desc* d, int p, int q,
                          cudaStream_t st) {
  const int Nrho = d->Nrho, M = d->M, Mpre = d->Mpre, n = N * N * N;
  const int pq = p * d->nspcs + q;
  VssPair& P = h->pair[pq];
  P.prefac = d->prefac[pq];
  const double mp = d->masses[p], mq = d->masses[q];
  const double eta = d->eta[pq], gam = d->gamma[pq];
  const double swpre = 4 * M_PI / Mpre;
  std::vector<double> Bmk((size_t)M * Mpre), srho(Nrho), fb(Nrho), fc(Nrho);
  for (int m = 0; m < M; ++m)
    for (int k = 0; k < Mpre; ++k)
      Bmk[(size_t)m * Mpre + k] = std::pow(
          1 + d->sz[3 * m] * d->szpre[3 * k] + d->sz[3 * m + 1] * d->szpre[3 * k + 1] +
              d->sz[3 * m + 2] * d->szpre[3 * k + 2],
          eta);
  for (int r = 0; r < Nrho; ++r) {
    srho[r] = M_PI / d->L * d->qz[r];
    fb[r] = swpre * std::pow(d->qz[r], gam + 2);
    fc[r] = d->qw[r] * d->sw * fb[r];
  }
  std::vector<double2> ph((size_t)Nrho * M * 6 * N);
  for (int r = 0; r < Nrho; ++r)
    for (int m = 0; m < M; ++m)
      for (int ax = 0; ax < 3; ++ax)
        for (int l = 0; l < N; ++l) {
          const double rl = (l < N / 2) ? l : l - N;
          const double a = srho[r] * d->sz[3 * m + ax] * rl;
          const size_t base = ((size_t)r * M + m) * 6 * N;
          const double a1 = a * (mq / (mp + mq)), a2 = -a * (mp / (mp + mq));
          ph[base + ax * N + l] = make_double2(std::cos(a1), std::sin(a1));
          ph[base + (3 + ax) * N + l] = make_double2(std::cos(a2), std::sin(a2));
        }
  double *dB = nullptr, *ds = nullptr, *dfb = nullptr, *dfc = nullptr, *dspre = nullptr;
  double2* cpart = nullptr;
  std::vector<double> spre(d->szpre, d->szpre + 3 * Mpre);
  int rc = DGFS_OK;
  if ((rc = upload(&dB, Bmk)) || (rc = upload(&ds, srho)) || (rc = upload(&dfb, fb)) ||
      (rc = upload(&dfc, fc)) || (rc = upload(&dspre, spre)) || (rc = upload(&P.ph, ph)))
    return rc;
  cudaError_t e1 = cudaMalloc(&P.b, sizeof(double2) * (size_t)Nrho * M * n);
  if (e1 == cudaSuccess) e1 = cudaMalloc(&P.c, sizeof(double2) * n);
  if (e1 == cudaSuccess) e1 = cudaMalloc(&cpart, sizeof(double2) * (size_t)Nrho * n);
  if (e1 != cudaSuccess)
    return fail(DGFS_ERR_CUDA, std::string("allocation: ") + cudaGetErrorString(e1));
  VssSetupArgs a{};
  a.Bmk = dB; a.spre = dspre; a.srho = ds; a.fac_b = dfb; a.fac_c = dfc;
  a.mpq = mq / (mp + mq); a.M = M; a.Mpre = Mpre; a.Nrho = Nrho;
  a.b = P.b; a.cpart = cpart;
  const size_t smem = (2 * kVssKChunk + 4 * kVssKChunk * N) * sizeof(double2) +
                      (size_t)M * kVssKChunk * sizeof(double);
  if ((rc = launch_plain(vss_setup_kernel<N>, dim3(N, Nrho),
                         dim3(vss_setup_threads<N>()), smem, st, a)))
    return rc;
  vss_sum_c_kernel<<<(n + 255) / 256, 256, 0, st>>>(cpart, Nrho, (size_t)n, P.c);
  DGFS_CUDA(cudaGetLastError());
  DGFS_CUDA(cudaStreamSynchronize(st));
  cudaFree(dB); cudaFree(ds); cudaFree(dfb); cudaFree(dfc); cudaFree(dspre);
  cudaFree(cpart);
  return DGFS_OK;
}

extern "C" int dgfs_vss_create(const dgfs_vss_desc* d, dgfs_vss_handle* out) {
  if (!d || !out) return fail(DGFS_ERR_INVALID, "null descriptor or handle");
  *out = nullptr;
  if (d->nspcs < 1 || d->nspcs > 4 || d->Nrho <= 0 || d->M <= 0 || d->M > 16 ||
      d->Mpre <= 0 || d->max_evals <= 0)
    return fail(DGFS_ERR_INVALID, "need 1 <= nspcs <= 4, 1 <= M <= 16, Nrho, Mpre, max_evals > 0");
  if (!d->qz || !d->qw || !d->sz || !d->szpre || !d->masses || !d->gamma ||
      !d->eta || !d->prefac)
    return fail(DGFS_ERR_INVALID, "missing descriptor arrays");
  if (d->N != 8 && d->N != 16 && d->N != 24 && d->N != 32)
    return fail(DGFS_ERR_UNSUPPORTED, "VSS: N must be 8, 16, 24 or 32");
  if (int rc = ensure_twiddles()) return rc;
  if (d->precision != DGFS_PREC_FP64 && d->precision != DGFS_PREC_FP32)
    return fail(DGFS_ERR_INVALID, "unknown precision");
  auto* h = new dgfs_vss_s();
  h->N = d->N; h->n = d->N * d->N * d->N; h->Nrho = d->Nrho; h->M = d->M;
  h->nspcs = d->nspcs; h->max_evals = d->max_evals;
  h->precision = d->precision;
  std::vector<double> w(d->Nrho);
  for (int r = 0; r < d->Nrho; ++r) w[r] = d->qw[r] * d->sw / h->n;
  int rc = upload(&h->w, w);
  for (int p = 0; p < d->nspcs && !rc; ++p)
    for (int q = 0; q < d->nspcs && !rc; ++q) {
      switch (d->N) {
        case 8: rc = vss_setup_pair<8>(h, d, p, q, 0); break;
        case 16: rc = vss_setup_pair<16>(h, d, p, q, 0); break;
        case 24: rc = vss_setup_pair<24>(h, d, p, q, 0); break;
        default: rc = vss_setup_pair<32>(h, d, p, q, 0); break;
      }
    }
  if (!rc) {
    cudaError_t e1 = cudaMalloc(&h->F[0], sizeof(double2) * (size_t)h->max_evals * h->n);
    if (e1 == cudaSuccess)
      e1 = cudaMalloc(&h->F[1], sizeof(double2) * (size_t)h->max_evals * h->n);
    if (e1 != cudaSuccess)
      rc = fail(DGFS_ERR_CUDA, std::string("allocation: ") + cudaGetErrorString(e1));
  }
  if (!rc && h->precision == DGFS_PREC_FP32) {
    const size_t E = h->max_evals, n = h->n, N = h->N, T = (size_t)h->Nrho * h->M;
    cudaError_t e1 = cudaSuccess;
    auto A = [&](auto** q, size_t cnt) {
      if (e1 == cudaSuccess) e1 = cudaMalloc((void**)q, cnt * sizeof(**q));
    };
    const size_t ns = h->nspcs;
    for (int s2 = 0; s2 < std::max(2, h->nspcs); ++s2) {
      A(&h->Fg[s2], E * n); A(&h->mhat[s2], E * 3 * N); A(&h->mom[s2], E * 5);
    }
    A(&h->ReLf, ns * E * n); A(&h->uv, ns * E * T * 6 * N);
    A(&h->hh, ns * E * T * 3 * N); A(&h->GM, ns * E * n);
    A(&h->H, ns * E * h->Nrho * n); A(&h->b2dummy, n);
    if (e1 == cudaSuccess) {
      int lo = 0, hi = 0;
      e1 = cudaDeviceGetStreamPriorityRange(&lo, &hi);
      if (e1 == cudaSuccess)
        e1 = cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, lo);
      if (e1 == cudaSuccess) e1 = cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming);
      if (e1 == cudaSuccess) e1 = cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming);
    }
    for (int pq = 0; pq < h->nspcs * h->nspcs; ++pq) {
      A(&h->pair[pq].b32, T * n); A(&h->pair[pq].ph32, T * 6 * N);
    }
    if (e1 == cudaSuccess) {
      for (int pq = 0; pq < h->nspcs * h->nspcs; ++pq) {
        vss_to_fp32_kernel<<<(unsigned)((T * n + 255) / 256), 256>>>(
            h->pair[pq].b, h->pair[pq].b32, T * n);
        vss_to_fp32_kernel<<<(unsigned)((T * 6 * N + 255) / 256), 256>>>(
            h->pair[pq].ph, h->pair[pq].ph32, T * 6 * N);
      }
      e1 = cudaDeviceSynchronize();
    }
    std::vector<double> c0(N);
    for (size_t i = 0; i < N; ++i) c0[i] = -d->L + d->L / N + i * (2.0 * d->L / N);
    h->cw = std::pow(2.0 * d->L / N, 3);
    if (e1 == cudaSuccess) rc = upload(&h->c0, c0);
    else rc = fail(DGFS_ERR_CUDA, std::string("FP32 scratch: ") + cudaGetErrorString(e1));
  }
  if (rc) { free_vss(h); return rc; }
  if (int rc_s = settle_uploads()) { free_vss(h); return rc_s; }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_vss_destroy(dgfs_vss_handle h) {
  if (h) free_vss(h);
  return DGFS_OK;
}

template <int N>
static int vss_run(dgfs_vss_s* h, int p, int q, const void* fp, const void* fq,
                   int f_double, void* Q, int q_double, const int32_t* ss,
                   int sb, const int32_t* ds, int db, int nevals,
                   cudaStream_t st) {
  constexpr int C = VssClusters<N>::c;
  using G = Geo<N, C>;
  int rc;
  const VssPair& P = h->pair[p * h->nspcs + q];
  if (h->precision == DGFS_PREC_FP32) {
    constexpr int CPRO = VhsClusters<N>::cpro;
    constexpr int CEPI = VhsClusters<N>::cepi;
    constexpr int C3 = VssClusters32<N>::c;
    using GPRO = Geo<N, CPRO>;
    using GEPI = Geo<N, CEPI>;
    using G3 = Geo<N, C3>;
    const int T = h->Nrho * h->M;
    // prologues: F_g, Maxwellian spectra of f_p and f_q; the f_q pass also
    // leaves the loss Re IFFT(c G) (complex loss kernel)
    for (int s2 = 0; s2 < 2; ++s2) {
      VhsPrologueArgs a{};
      a.f = s2 == 0 ? fp : fq; a.f_double = f_double; a.src_slots = ss; a.src_base = sb;
      a.c0 = h->c0; a.b2 = h->b2dummy; a.b2c = P.c; a.cw = h->cw; a.split = 1;
      a.Fg = h->Fg[s2]; a.ReLf = h->ReLf; a.mhat = h->mhat[s2]; a.moments = h->mom[s2];
      a.Fny = nullptr;
      const size_t smem = prologue_smem<N, CPRO>();
      if ((rc = launch_cluster(vhs_prologue_kernel<N, CPRO>, dim3(CPRO, nevals),
                               dim3(GPRO::NT), CPRO, smem, st, a)))
        return rc;
    }
    VssTablesArgs ta{};
    ta.mhat_p = h->mhat[0]; ta.mhat_q = h->mhat[1]; ta.ph = P.ph; ta.uv = h->uv;
    ta.hh = h->hh; ta.T = T; ta.nevals = nevals;
    if ((rc = launch_plain(vss_tables_kernel<N>, dim3((nevals * T * 3 + 127) / 128),
                           dim3(128), 0, st, ta)))
      return rc;
    VssGainArgs ga{};
    ga.hh = h->hh; ga.b = P.b; ga.w = h->w; ga.GM = h->GM; ga.Nrho = h->Nrho; ga.M = h->M;
    if ((rc = launch_plain(vss_maxwell_gain_kernel<N>,
                           dim3((h->n + 255) / 256, nevals), dim3(256), 0, st, ga)))
      return rc;
    VssTerms32Args tt{};
    tt.pr[0] = {h->Fg[0], h->Fg[1], P.ph32, h->uv, P.b32, h->H};
    tt.w = h->w; tt.Nrho = h->Nrho; tt.M = h->M; tt.nevals = nevals;
    const size_t smem3 = 5 * slab_bytes(N, C3, sizeof(float2)) + 24 * N * sizeof(float2);
    if ((rc = launch_cluster(vss_terms32_kernel<N, C3>, dim3(C3, h->Nrho, nevals),
                             dim3(G3::NT), C3, smem3, st, tt)))
      return rc;
    VhsEpilogueArgs ea{};
    ea.H = h->H; ea.h_double = 0; ea.GM = h->GM; ea.ReLf = h->ReLf; ea.f = fp;
    ea.f_double = f_double; ea.src_slots = ss; ea.src_base = sb; ea.Q = Q;
    ea.q_double = q_double; ea.dst_slots = ds; ea.dst_base = db;
    ea.prefac = P.prefac; ea.Nrho = h->Nrho; ea.project = 0; ea.c0 = h->c0; ea.cw = h->cw;
    const size_t smemE = epilogue_smem<N, CEPI>();
    return launch_cluster(vhs_epilogue_kernel<N, CEPI>, dim3(CEPI, nevals),
                          dim3(GEPI::NT), CEPI, smemE, st, ea);
  }
  for (int s = 0; s < 2; ++s) {
    Fft3Args fa{};
    fa.f = s == 0 ? fp : fq; fa.f_double = f_double; fa.slots = ss; fa.base = sb;
    fa.out = h->F[s];
    if ((rc = launch_cluster(fft3_forward_kernel<N, C>, dim3(C, nevals),
                             dim3(G::NT), C, slab_bytes(N, C, sizeof(double2)),
                             st, fa)))
      return rc;
  }
  VssPairArgs a{};
  a.Fp = h->F[0]; a.Fq = h->F[1]; a.b = P.b; a.c = P.c; a.ph = P.ph; a.w = h->w;
  a.fp = fp; a.f_double = f_double; a.src_slots = ss; a.src_base = sb;
  a.Q = Q; a.q_double = q_double; a.dst_slots = ds; a.dst_base = db;
  a.prefac = P.prefac; a.Nrho = h->Nrho; a.M = h->M;
  const size_t smem = 4 * slab_bytes(N, C, sizeof(double2)) + 6 * N * sizeof(double2);
  return launch_cluster(vss_pair_kernel<N, C>, dim3(C, nevals), dim3(G::NT), C,
                        smem, st, a);
}

extern "C" int dgfs_vss_eval(dgfs_vss_handle h, int32_t p, int32_t q,
                             const void* fp, const void* fq, int32_t f_dtype,
                             void* Q, int32_t q_dtype, const int32_t* src_slots,
                             int32_t src_base, const int32_t* dst_slots,
                             int32_t dst_base, int32_t nevals, void* stream);

// All pairs (p, q), q < nspcs, of one species p in FP32 mode:
//   Q_p[dst] += sum_q Q_pq(f_p[src], f_q[src])
// with one prologue per input species q (its F_g, Maxwellian spectra and
// the loss of the pair, Re IFFT(c_pq F_q)), the 1-D tables per pair, the
// FP64 Maxwellian gain per pair on the low-priority stream beside one FP32
// terms launch over every pair, and one epilogue that sums the pairs'
// spectra with their prefactors before a single inverse transform
// (Re IFFT is linear: sum_q pref_pq Re IFFT(Ghat_pq) = Re IFFT(sum ...)).
template <int N>
static int vss_run_species(dgfs_vss_s* h, int p, const void* const* f,
                           int f_double, void* Qp, int q_double,
                           const int32_t* ss, int sb, const int32_t* ds,
                           int db, int nevals, cudaStream_t st,
                           const void* const* fl = nullptr, size_t fl_stride = 0,
                           void* const* ql = nullptr) {
  constexpr int CPRO = VhsClusters<N>::cpro;
  constexpr int CEPI = VhsClusters<N>::cepi;
  constexpr int C3 = VssClusters32<N>::c;
  using GPRO = Geo<N, CPRO>;
  using GEPI = Geo<N, CEPI>;
  using G3 = Geo<N, C3>;
  const int ns = h->nspcs, T = h->Nrho * h->M;
  const size_t E = h->max_evals, n = h->n;
  auto ReLf = [&](int q) { return h->ReLf + q * E * n; };
  auto uv = [&](int q) { return h->uv + q * E * T * 6 * N; };
  auto hh = [&](int q) { return h->hh + q * E * T * 3 * N; };
  auto GM = [&](int q) { return h->GM + q * E * n; };
  auto H = [&](int q) { return h->H + q * E * h->Nrho * n; };
  int rc;
  for (int q = 0; q < ns; ++q) {
    const VssPair& P = h->pair[p * ns + q];
    VhsPrologueArgs a{};
    a.f = fl ? nullptr : f[q]; a.f_list = fl ? fl + q * fl_stride : nullptr;
    a.f_double = f_double; a.src_slots = ss; a.src_base = sb;
    a.c0 = h->c0; a.b2 = h->b2dummy; a.b2c = P.c; a.cw = h->cw; a.split = 1;
    a.Fg = h->Fg[q]; a.ReLf = ReLf(q); a.mhat = h->mhat[q]; a.moments = h->mom[q];
    if ((rc = launch_cluster(vhs_prologue_kernel<N, CPRO>, dim3(CPRO, nevals),
                             dim3(GPRO::NT), CPRO, prologue_smem<N, CPRO>(), st,
                             a)))
      return rc;
  }
  for (int q = 0; q < ns; ++q) {
    VssTablesArgs ta{};
    ta.mhat_p = h->mhat[p]; ta.mhat_q = h->mhat[q];
    ta.ph = h->pair[p * ns + q].ph; ta.uv = uv(q); ta.hh = hh(q);
    ta.T = T; ta.nevals = nevals;
    if ((rc = launch_plain(vss_tables_kernel<N>, dim3((nevals * T * 3 + 127) / 128),
                           dim3(128), 0, st, ta)))
      return rc;
  }
  DGFS_CUDA(cudaEventRecord(h->fork, st));
  DGFS_CUDA(cudaStreamWaitEvent(h->aux, h->fork, 0));
  VssTerms32Args tt{};
  for (int q = 0; q < ns; ++q) {
    const VssPair& P = h->pair[p * ns + q];
    tt.pr[q] = {h->Fg[p], h->Fg[q], P.ph32, uv(q), P.b32, H(q)};
  }
  tt.w = h->w; tt.Nrho = h->Nrho; tt.M = h->M; tt.nevals = nevals;
  const size_t smem3 = 5 * slab_bytes(N, C3, sizeof(float2)) + 24 * N * sizeof(float2);
  if ((rc = launch_cluster(vss_terms32_kernel<N, C3>, dim3(C3, h->Nrho, nevals * ns),
                           dim3(G3::NT), C3, smem3, st, tt)))
    return rc;
  for (int q = 0; q < ns; ++q) {
    VssGainArgs ga{};
    ga.hh = hh(q); ga.b = h->pair[p * ns + q].b; ga.w = h->w; ga.GM = GM(q);
    ga.Nrho = h->Nrho; ga.M = h->M;
    if ((rc = launch_plain(vss_maxwell_gain_kernel<N>,
                           dim3((h->n + 255) / 256, nevals), dim3(256), 0,
                           h->aux, ga)))
      return rc;
  }
  DGFS_CUDA(cudaEventRecord(h->join, h->aux));
  DGFS_CUDA(cudaStreamWaitEvent(st, h->join, 0));
  VhsEpilogueArgs ea{};
  ea.f = fl ? nullptr : f[p]; ea.f_list = fl ? fl + p * fl_stride : nullptr;
  ea.f_double = f_double; ea.src_slots = ss; ea.src_base = sb;
  ea.Q = Qp; ea.q_list = ql; ea.q_double = q_double;
  ea.dst_slots = ds; ea.dst_base = db;
  ea.Nrho = h->Nrho; ea.project = 0; ea.c0 = h->c0; ea.cw = h->cw;
  ea.nt = ns;
  for (int q = 0; q < ns; ++q) {
    ea.Ht[q] = H(q); ea.GMt[q] = GM(q); ea.ReLft[q] = ReLf(q);
    ea.pref[q] = h->pair[p * ns + q].prefac;
  }
  return launch_cluster(vhs_epilogue_kernel<N, CEPI>, dim3(CEPI, nevals),
                        dim3(GEPI::NT), CEPI, epilogue_smem<N, CEPI>(), st, ea);
}

extern "C" int dgfs_vss_eval_species(dgfs_vss_handle h, int32_t p,
                                     const void* const* f, int32_t f_dtype,
                                     void* Qp, int32_t q_dtype,
                                     const int32_t* src_slots, int32_t src_base,
                                     const int32_t* dst_slots, int32_t dst_base,
                                     int32_t nevals, void* stream) {
  NvtxRange nvtx_range("dgfs_vss_eval_species");
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (p < 0 || p >= h->nspcs) return fail(DGFS_ERR_INVALID, "species out of range");
  if (!f || !Qp) return fail(DGFS_ERR_INVALID, "null f list or Q");
  for (int q = 0; q < h->nspcs; ++q)
    if (!f[q]) return fail(DGFS_ERR_INVALID, "null f in the species list");
  if (nevals < 0 || src_base < 0 || dst_base < 0)
    return fail(DGFS_ERR_INVALID, "negative nevals or slot base");
  if ((f_dtype != DGFS_F32 && f_dtype != DGFS_F64) ||
      (q_dtype != DGFS_F32 && q_dtype != DGFS_F64))
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  if (nevals == 0) return DGFS_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->precision != DGFS_PREC_FP32) {
    // the FP64 mode (the reference's) evaluates the pairs one by one
    for (int q = 0; q < h->nspcs; ++q)
      if (int rc = dgfs_vss_eval(h, p, q, f[p], f[q], f_dtype, Qp, q_dtype,
                                 src_slots, src_base, dst_slots, dst_base,
                                 nevals, stream))
        return rc;
    return DGFS_OK;
  }
  for (int off = 0; off < nevals; off += h->max_evals) {
    const int cnt = std::min(h->max_evals, nevals - off);
    const int32_t* ss = src_slots ? src_slots + off : nullptr;
    const int32_t* ds = dst_slots ? dst_slots + off : nullptr;
    int rc;
    switch (h->N) {
      case 8: rc = vss_run_species<8>(h, p, f, f_dtype, Qp, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      case 16: rc = vss_run_species<16>(h, p, f, f_dtype, Qp, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      case 24: rc = vss_run_species<24>(h, p, f, f_dtype, Qp, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      default: rc = vss_run_species<32>(h, p, f, f_dtype, Qp, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st); break;
    }
    if (rc) return rc;
  }
  return DGFS_OK;
}

// Every pair of species p for a list of points of several mixtures that
// share one operator (FP32 mode): f_lists is a device array [nspcs][nevals]
// of input arrays (evaluation i of species q reads slot src(i) of
// f_lists[q * nevals + i]), q_list a device array [nevals] of output arrays.
extern "C" int dgfs_vss_eval_species_multi(dgfs_vss_handle h, int32_t p,
                                           const void* const* f_lists,
                                           int32_t f_dtype,
                                           void* const* q_list, int32_t q_dtype,
                                           const int32_t* src_slots,
                                           int32_t src_base,
                                           const int32_t* dst_slots,
                                           int32_t dst_base, int32_t nevals,
                                           void* stream) {
  NvtxRange nvtx_range("dgfs_vss_eval_species_multi");
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (h->precision != DGFS_PREC_FP32)
    return fail(DGFS_ERR_UNSUPPORTED, "array lists need the FP32 mode");
  if (p < 0 || p >= h->nspcs) return fail(DGFS_ERR_INVALID, "species out of range");
  if (!f_lists || !q_list) return fail(DGFS_ERR_INVALID, "null array lists");
  if (nevals < 0 || src_base < 0 || dst_base < 0)
    return fail(DGFS_ERR_INVALID, "negative nevals or slot base");
  if ((f_dtype != DGFS_F32 && f_dtype != DGFS_F64) ||
      (q_dtype != DGFS_F32 && q_dtype != DGFS_F64))
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const void* none[4] = {};
  for (int off = 0; off < nevals; off += h->max_evals) {
    const int cnt = std::min(h->max_evals, nevals - off);
    const int32_t* ss = src_slots ? src_slots + off : nullptr;
    const int32_t* ds = dst_slots ? dst_slots + off : nullptr;
    const void* const* fl = f_lists + off;
    void* const* ql = q_list + off;
    int rc;
    switch (h->N) {
      case 8: rc = vss_run_species<8>(h, p, none, f_dtype, nullptr, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, fl, nevals, ql); break;
      case 16: rc = vss_run_species<16>(h, p, none, f_dtype, nullptr, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, fl, nevals, ql); break;
      case 24: rc = vss_run_species<24>(h, p, none, f_dtype, nullptr, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, fl, nevals, ql); break;
      default: rc = vss_run_species<32>(h, p, none, f_dtype, nullptr, q_dtype, ss, src_base + off, ds, dst_base + off, cnt, st, fl, nevals, ql); break;
    }
    if (rc) return rc;
  }
  return DGFS_OK;
}

extern "C" int dgfs_vss_eval(dgfs_vss_handle h, int32_t p, int32_t q,
                             const void* f_p, const void* f_q, int32_t f_dtype,
                             void* Q_p, int32_t q_dtype,
                             const int32_t* src_slots, int32_t src_base,
                             const int32_t* dst_slots, int32_t dst_base,
                             int32_t nevals, void* stream) {
  NvtxRange nvtx_range("dgfs_vss_eval");
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (p < 0 || q < 0 || p >= h->nspcs || q >= h->nspcs)
    return fail(DGFS_ERR_INVALID, "species index out of range");
  if (nevals < 0 || src_base < 0 || dst_base < 0)
    return fail(DGFS_ERR_INVALID, "negative nevals or slot base");
  if (nevals == 0) return DGFS_OK;
  if (!f_p || !f_q || !Q_p) return fail(DGFS_ERR_INVALID, "null array");
  if ((f_dtype != DGFS_F32 && f_dtype != DGFS_F64) ||
      (q_dtype != DGFS_F32 && q_dtype != DGFS_F64))
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int off = 0; off < nevals; off += h->max_evals) {
    const int cnt = std::min(h->max_evals, nevals - off);
    const int32_t* ss = src_slots ? src_slots + off : nullptr;
    const int32_t* ds = dst_slots ? dst_slots + off : nullptr;
    int rc;
    switch (h->N) {
      case 8: rc = vss_run<8>(h, p, q, f_p, f_q, f_dtype == DGFS_F64, Q_p, q_dtype == DGFS_F64, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      case 16: rc = vss_run<16>(h, p, q, f_p, f_q, f_dtype == DGFS_F64, Q_p, q_dtype == DGFS_F64, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      case 24: rc = vss_run<24>(h, p, q, f_p, f_q, f_dtype == DGFS_F64, Q_p, q_dtype == DGFS_F64, ss, src_base + off, ds, dst_base + off, cnt, st); break;
      default: rc = vss_run<32>(h, p, q, f_p, f_q, f_dtype == DGFS_F64, Q_p, q_dtype == DGFS_F64, ss, src_base + off, ds, dst_base + off, cnt, st); break;
    }
    if (rc) return rc;
  }
  return DGFS_OK;
}

// Conservation projection of Q (no counterpart in the reference): after it,
// sum_v Q phi_j cw = 0 for phi = (1, cx, cy, cz, |c|^2) to FP64 rounding.
extern "C" int dgfs_vhs_set_projection(dgfs_vhs_handle h, int32_t enable) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (enable) {
    // G_jk = sum_v phi_j phi_k cw, inverted by Gauss-Jordan in long double
    const int N = h->N;
    std::vector<double> c0(N);
    DGFS_CUDA(cudaMemcpy(c0.data(), h->c0, N * sizeof(double),
                         cudaMemcpyDeviceToHost));
    long double G[5][10] = {};
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j)
        for (int k = 0; k < N; ++k) {
          const long double cx = c0[i], cy = c0[j], cz = c0[k];
          const long double ph[5] = {1, cx, cy, cz, cx * cx + cy * cy + cz * cz};
          for (int r = 0; r < 5; ++r)
            for (int s = 0; s < 5; ++s) G[r][s] += ph[r] * ph[s] * h->cw;
        }
    for (int r = 0; r < 5; ++r) G[r][5 + r] = 1;
    for (int col = 0; col < 5; ++col) {
      int piv = col;
      for (int r = col + 1; r < 5; ++r)
        if (fabsl(G[r][col]) > fabsl(G[piv][col])) piv = r;
      if (fabsl(G[piv][col]) < 1e-300L)
        return fail(DGFS_ERR_INVALID, "singular moment Gram matrix");
      for (int s = 0; s < 10; ++s) std::swap(G[col][s], G[piv][s]);
      const long double d = G[col][col];
      for (int s = 0; s < 10; ++s) G[col][s] /= d;
      for (int r = 0; r < 5; ++r)
        if (r != col) {
          const long double f = G[r][col];
          for (int s = 0; s < 10; ++s) G[r][s] -= f * G[col][s];
        }
    }
    for (int r = 0; r < 5; ++r)
      for (int s = 0; s < 5; ++s) h->Ginv[r * 5 + s] = (double)G[r][5 + s];
  }
  h->project = enable ? 1 : 0;
  return DGFS_OK;
}

// ---------------------------------------------------------------------------
// Penalty model (IMEX) entry points
// ---------------------------------------------------------------------------
// Linear slope limiter: tables (host, FP64) then in-place application.
extern "C" int dgfs_dg_set_limiter(dgfs_dg_handle h, const double* wavg,
                                   const double* wdr, const double* dx,
                                   const double* hs) {
  if (!h || !wavg || !wdr || !dx || !hs) return fail(DGFS_ERR_INVALID, "null argument");
  const int K = h->base.K, Ne = h->base.Ne;
  std::vector<double> t;
  t.insert(t.end(), wavg, wavg + K);
  t.insert(t.end(), wdr, wdr + K);
  t.insert(t.end(), dx, dx + (size_t)K * Ne);
  t.insert(t.end(), hs, hs + Ne);
  if (h->lim) {
    cudaFree(h->lim);
    h->lim = nullptr;
  }
  return upload(&h->lim, t);
}

extern "C" int dgfs_std_esbgk_relax(dgfs_dg_handle h, const void* f, void* Q,
                                    int32_t dtype, int32_t npts, double prefac,
                                    double omega, double Pr, void* stream) {
  if (!h || !f || !Q || npts < 0) return fail(DGFS_ERR_INVALID, "bad arguments");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  if (!(Pr > 0)) return fail(DGFS_ERR_INVALID, "Pr must be > 0");
  if (npts == 0) return DGFS_OK;
  StdEsArgs a{};
  a.f = f; a.Q = Q; a.f_double = dtype == DGFS_F64;
  a.N = h->base.N; a.Nv = h->base.Nv; a.c0 = h->c0; a.cw = h->cw;
  a.prefac = prefac; a.omega = omega; a.Pr = Pr;
  std_esbgk_relax_kernel<<<npts, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_dg_limit_positivity(dgfs_dg_handle h, void* u,
                                        int32_t dtype, void* stream) {
  if (!h || !u) return fail(DGFS_ERR_INVALID, "null argument");
  if (!h->lim) return fail(DGFS_ERR_INVALID, "limiter tables not set");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  DgLimitArgs a{};
  a.u = u; a.f_double = dtype == DGFS_F64; a.K = h->base.K; a.Ne = h->base.Ne;
  a.Nv = h->base.Nv; a.wavg = h->lim;
  dg_limit_pos_kernel<<<(a.Nv + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_dg_set_upwind(dgfs_dg_handle h, const double* Dpos,
                                  const double* Dneg, int32_t swap) {
  if (!h || !Dpos || !Dneg) return fail(DGFS_ERR_INVALID, "null argument");
  DgAdvectArgs& a = h->base;
  if (swap && (a.bc[0] == kBcWall || a.bc[1] == kBcWall ||
               a.bc[0] == kBcWallExpr || a.bc[1] == kBcWallExpr))
    return fail(DGFS_ERR_UNSUPPORTED, "swapped (periodic) traces with a wall boundary");
  const int K = a.K;
  for (int i = 0; i < K * K; ++i) {
    a.D[i] = Dpos[i];
    a.D2[i] = Dneg[i];
  }
  a.upwind = 1;
  a.swap = swap ? 1 : 0;
  return DGFS_OK;
}

extern "C" int dgfs_dg_set_entropy_stable(dgfs_dg_handle h, const double* Dr) {
  if (!h || !Dr) return fail(DGFS_ERR_INVALID, "null argument");
  DgAdvectArgs& a = h->base;
  for (int i = 0; i < a.K * a.K; ++i) a.D[i] = Dr[i];
  a.upwind = 2;
  a.swap = 0;
  return DGFS_OK;
}

extern "C" int dgfs_dg_limit(dgfs_dg_handle h, void* u, int32_t dtype,
                             void* stream) {
  if (!h || !u) return fail(DGFS_ERR_INVALID, "null argument");
  if (!h->lim) return fail(DGFS_ERR_INVALID, "limiter tables not set");
  if (dtype != DGFS_F32 && dtype != DGFS_F64)
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  const int K = h->base.K, Ne = h->base.Ne;
  DgLimitArgs a{};
  a.u = u; a.f_double = dtype == DGFS_F64; a.K = K; a.Ne = Ne; a.Nv = h->base.Nv;
  a.wavg = h->lim; a.wdr = h->lim + K; a.dx = h->lim + 2 * K;
  a.h = h->lim + 2 * K + (size_t)K * Ne; a.invjac = h->invjac; a.tol = 1e-6;
  dg_limit_kernel<<<(a.Nv + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

// Penalty-model moments: NA = 5 (BGK), 11 (ES-BGK) or 14 (Shakov) per
// point, in chunks of the handle's partial-sum capacity.
static int penalty_moments_n(dgfs_dg_s* h, const void* f, int32_t dtype,
                             int32_t npts, int32_t na, double* U,
                             cudaStream_t st) {
  if (!h || !f || !U || npts < 0) return fail(DGFS_ERR_INVALID, "bad arguments");
  if (na != 5 && na != 11 && na != 14)
    return fail(DGFS_ERR_INVALID, "moments per point must be 5, 11 or 14");
  const size_t elem = dtype == DGFS_F64 ? sizeof(double) : sizeof(float);
  for (int off = 0; off < npts; off += h->mpts) {
    const int cnt = std::min(h->mpts, npts - off);
    PenaltyMomentArgs a{};
    a.f = static_cast<const char*>(f) + (size_t)off * h->base.Nv * elem;
    a.f_double = dtype == DGFS_F64; a.Nv = h->base.Nv; a.N = h->base.N;
    a.c0 = h->c0; a.cw = h->cw; a.U = U + (size_t)off * na;
    const dim3 grid(kPmCh, cnt);
    if (na == 5) penalty_moments_part_kernel<5><<<grid, 256, 0, st>>>(a, h->mpart);
    else if (na == 11) penalty_moments_part_kernel<11><<<grid, 256, 0, st>>>(a, h->mpart);
    else penalty_moments_part_kernel<14><<<grid, 256, 0, st>>>(a, h->mpart);
    penalty_moments_final_kernel<<<(cnt * na + 127) / 128, 128, 0, st>>>(
        h->mpart, a.U, cnt, na);
  }
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_penalty_moments(dgfs_dg_handle h, const void* f,
                                    int32_t dtype, int32_t npts, double* U,
                                    void* stream) {
  return penalty_moments_n(h, f, dtype, npts, 5, U, static_cast<cudaStream_t>(stream));
}

extern "C" int dgfs_penalty_moments_n(dgfs_dg_handle h, const void* f,
                                      int32_t dtype, int32_t npts, int32_t nalph,
                                      double* U, void* stream) {
  return penalty_moments_n(h, f, dtype, npts, nalph, U,
                           static_cast<cudaStream_t>(stream));
}

static int penalty_kind_ok(int32_t kind) {
  return kind == kPenBGK || kind == kPenESBGK || kind == kPenShakov;
}

extern "C" int dgfs_penalty_model_implicit(dgfs_dg_handle h, int32_t kind,
                                           const double* U, const void* rhs,
                                           void* f, void* P, void* M,
                                           int32_t dtype, int32_t npts,
                                           double adiv, double cdt,
                                           double prefac, double omega,
                                           double Pr, void* stream) {
  if (!h || !U || !rhs || !f || npts < 0) return fail(DGFS_ERR_INVALID, "bad arguments");
  if (!penalty_kind_ok(kind)) return fail(DGFS_ERR_INVALID, "unknown penalty model");
  PenaltyImplicitArgs a{};
  a.U = U; a.rhs = rhs; a.f = f; a.P = P; a.Mout = M;
  a.f_double = dtype == DGFS_F64; a.Nv = h->base.Nv; a.N = h->base.N;
  a.c0 = h->c0; a.adiv = adiv; a.cdt = cdt; a.prefac = prefac; a.omega = omega;
  a.Pr = Pr;
  a.total = (size_t)npts * h->base.Nv;
  if (a.total == 0) return DGFS_OK;
  const dim3 pgrid((h->base.Nv + 256 * kPenaltyEpt - 1) / (256 * kPenaltyEpt), npts);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (kind == kPenBGK) penalty_implicit_kernel<kPenBGK><<<pgrid, 256, 0, st>>>(a);
  else if (kind == kPenESBGK) penalty_implicit_kernel<kPenESBGK><<<pgrid, 256, 0, st>>>(a);
  else penalty_implicit_kernel<kPenShakov><<<pgrid, 256, 0, st>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_penalty_implicit(dgfs_dg_handle h, const double* U,
                                     const void* rhs, void* f, void* P,
                                     void* M, int32_t dtype, int32_t npts,
                                     double adiv, double cdt, double prefac,
                                     double omega, void* stream) {
  return dgfs_penalty_model_implicit(h, kPenBGK, U, rhs, f, P, M, dtype, npts,
                                     adiv, cdt, prefac, omega, 1.0, stream);
}

extern "C" int dgfs_penalty_model_collide(dgfs_dg_handle h, int32_t kind,
                                          const double* U, const void* f,
                                          void* P, void* M, int32_t dtype,
                                          int32_t npts, double prefac,
                                          double omega, double Pr,
                                          void* stream) {
  if (!h || !U || !f || !P || npts < 0) return fail(DGFS_ERR_INVALID, "bad arguments");
  if (!penalty_kind_ok(kind)) return fail(DGFS_ERR_INVALID, "unknown penalty model");
  PenaltyImplicitArgs a{};
  a.U = U; a.f = const_cast<void*>(f); a.P = P; a.Mout = M;
  a.f_double = dtype == DGFS_F64; a.Nv = h->base.Nv; a.N = h->base.N;
  a.c0 = h->c0; a.prefac = prefac; a.omega = omega; a.Pr = Pr;
  a.total = (size_t)npts * h->base.Nv;
  if (a.total == 0) return DGFS_OK;
  const dim3 pgrid((h->base.Nv + 256 * kPenaltyEpt - 1) / (256 * kPenaltyEpt), npts);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (kind == kPenBGK) penalty_collide_kernel<kPenBGK><<<pgrid, 256, 0, st>>>(a);
  else if (kind == kPenESBGK) penalty_collide_kernel<kPenESBGK><<<pgrid, 256, 0, st>>>(a);
  else penalty_collide_kernel<kPenShakov><<<pgrid, 256, 0, st>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

extern "C" int dgfs_penalty_collide(dgfs_dg_handle h, const double* U,
                                    const void* f, void* P, void* M,
                                    int32_t dtype, int32_t npts, double prefac,
                                    double omega, void* stream) {
  return dgfs_penalty_model_collide(h, kPenBGK, U, f, P, M, dtype, npts,
                                    prefac, omega, 1.0, stream);
}

extern "C" int dgfs_penalty_model_relax(dgfs_dg_handle h, int32_t kind,
                                        double* U, int32_t npts, double adiv,
                                        double cdt, double prefac, double omega,
                                        double Pr, void* stream) {
  if (!h || !U || npts < 0) return fail(DGFS_ERR_INVALID, "bad arguments");
  if (!penalty_kind_ok(kind)) return fail(DGFS_ERR_INVALID, "unknown penalty model");
  if (kind == kPenBGK || npts == 0) return DGFS_OK;  // nothing to relax
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned grid = (unsigned)((npts + 127) / 128);
  if (kind == kPenESBGK)
    penalty_relax_kernel<kPenESBGK><<<grid, 128, 0, st>>>(U, npts, adiv, cdt, prefac, omega, Pr);
  else
    penalty_relax_kernel<kPenShakov><<<grid, 128, 0, st>>>(U, npts, adiv, cdt, prefac, omega, Pr);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

// Variants of the FP32 terms kernel (cluster sizes) for the autotuner.
extern "C" int dgfs_vhs_variants(int32_t N, int32_t* out, int32_t max) {
  if (!out || max <= 0) return fail(DGFS_ERR_INVALID, "bad output buffer");
  const int* v = nullptr;
  int n = 0;
  switch (N) {
    case 8: v = Terms32Variants<8>::v; n = 3; break;
    case 16: v = Terms32Variants<16>::v; n = 3; break;
    case 24: v = Terms32Variants<24>::v; n = 4; break;
    case 32: v = Terms32Variants<32>::v; n = 5; break;
    case 48: v = Terms32Variants<48>::v; n = 3; break;
    default: return fail(DGFS_ERR_UNSUPPORTED, "N not compiled in");
  }
  for (int i = 0; i < n && i < max; ++i) out[i] = v[i];
  return std::min(n, (int)max);
}

extern "C" int dgfs_vhs_set_variant(dgfs_vhs_handle h, int32_t cluster) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  int buf[8];
  const int n = dgfs_vhs_variants(h->N, buf, 8);
  if (n < 0) return n;
  for (int i = 0; i < n; ++i)
    if (buf[i] == cluster) { h->c32 = cluster; return DGFS_OK; }
  if (cluster == 0) { h->c32 = 0; return DGFS_OK; }
  return fail(DGFS_ERR_INVALID, "cluster size not a variant for this N");
}

// ---------------------------------------------------------------------------
// FNO surrogate of Q(f,f)
// ---------------------------------------------------------------------------
#include "fno_kernels.cuh"

struct dgfs_fno_s {
  int N = 0, K = 0, maxB = 0;
  long n = 0;
  double cw = 0, sQ = 1, Ginv[25] = {};
  fno::Layout L{};
  double* c0 = nullptr;
  float* p32 = nullptr;              // master parameters
  __nv_bfloat16* p16 = nullptr;      // BF16 copy read by the kernels
  float* grad = nullptr;
  float* am = nullptr;
  float* av = nullptr;
  float2 *tF = nullptr, *tG = nullptr, *tFs = nullptr, *tGs = nullptr;
  __nv_bfloat16* x0 = nullptr;
  __nv_bfloat16* v[5] = {};
  __nv_bfloat16* y[4] = {};
  float2* Vh[4] = {};
  float2 *Uh = nullptr, *T1 = nullptr, *T2 = nullptr;
  __nv_bfloat16* U = nullptr;        // spectral-path output (BF16)
  float* out = nullptr;
  double* qs = nullptr;
  double* fpart = nullptr;           // [maxB][FCH][6] partial sums
  float *dout = nullptr, *dz = nullptr, *aw = nullptr, *dvA = nullptr,
        *dvB = nullptr, *dy = nullptr, *part = nullptr;
  float2 *gUh = nullptr, *gVh = nullptr;
  double* loss = nullptr;
  int* err = nullptr;                // device error flag (bounded waits)
  int use_tc = 1;                    // dense layers on tcgen05 tensor cores
  int use_fused = 1;                 // eval: fused spectral passes
  float2 *Yp = nullptr, *Sp = nullptr;  // eval: yz spectra, x-mixed spectra
  std::vector<void*> owned;
};

static constexpr int kFnoWgradGrid = 296;

static void fno_free(dgfs_fno_s* h) {
  for (void* p : h->owned)
    if (p) cudaFree(p);
  delete h;
}

template <typename T>
static cudaError_t fno_alloc(dgfs_fno_s* h, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e == cudaSuccess) h->owned.push_back((void*)*p);
  return e;
}

extern "C" int dgfs_fno_create(const dgfs_fno_desc* d, dgfs_fno_handle* out) {
  if (!d || !out) return fail(DGFS_ERR_INVALID, "null argument");
  *out = nullptr;
  if (d->N != 16 && d->N != 32)
    return fail(DGFS_ERR_UNSUPPORTED, "FNO velocity grid must be N=16 or N=32");
  if ((d->N == 16 && d->modes != 8) || (d->N == 32 && d->modes != 12))
    return fail(DGFS_ERR_UNSUPPORTED,
                "FNO modes per axis: 8 at N=16, 12 at N=32 are compiled in");
  if (d->max_batch < 1 || d->max_batch > 32)
    return fail(DGFS_ERR_INVALID, "FNO max_batch must be in [1, 32]");
  if (!(d->L > 0) || !(d->q_scale > 0))
    return fail(DGFS_ERR_INVALID, "FNO needs L > 0 and q_scale > 0");
  // the fused evaluation kernels use the register FFTs' twiddle tables
  if (int rc = ensure_twiddles()) return rc;
  auto* h = new dgfs_fno_s();
  h->N = d->N; h->K = d->modes; h->maxB = d->max_batch;
  h->n = (long)h->N * h->N * h->N;
  h->sQ = d->q_scale;
  h->L.init(h->K);
  const int N = h->N, K = h->K;
  const long n = h->n, B = h->maxB;
  std::vector<double> c0(N);
  for (int i = 0; i < N; ++i) c0[i] = -d->L + d->L / N + i * (2.0 * d->L / N);
  h->cw = std::pow(2.0 * d->L / N, 3);
  // Gram matrix of (1, c, |c|^2) under cw, inverted in long double
  {
    long double G[5][10] = {};
    for (int ix = 0; ix < N; ++ix)
      for (int iy = 0; iy < N; ++iy)
        for (int iz = 0; iz < N; ++iz) {
          const long double cx = c0[ix], cy = c0[iy], cz = c0[iz];
          const long double ph[5] = {1, cx, cy, cz, cx * cx + cy * cy + cz * cz};
          for (int r = 0; r < 5; ++r)
            for (int s = 0; s < 5; ++s) G[r][s] += ph[r] * ph[s] * h->cw;
        }
    for (int r = 0; r < 5; ++r) G[r][5 + r] = 1;
    for (int c = 0; c < 5; ++c) {
      int pv = c;
      for (int r = c + 1; r < 5; ++r)
        if (fabsl(G[r][c]) > fabsl(G[pv][c])) pv = r;
      for (int s = 0; s < 10; ++s) std::swap(G[c][s], G[pv][s]);
      const long double inv = 1.0L / G[c][c];
      for (int s = 0; s < 10; ++s) G[c][s] *= inv;
      for (int r = 0; r < 5; ++r)
        if (r != c) {
          const long double f = G[r][c];
          for (int s = 0; s < 10; ++s) G[r][s] -= f * G[c][s];
        }
    }
    for (int r = 0; r < 5; ++r)
      for (int s = 0; s < 5; ++s) h->Ginv[r * 5 + s] = (double)G[r][5 + s];
  }
  // DFT tables: modes k = 0..K/2-1, -K/2..-1
  std::vector<float2> tF(K * N), tG(N * K), tFs(K * N), tGs(N * K);
  for (int kk = 0; kk < K; ++kk) {
    const int k = kk < K / 2 ? kk : kk - K;
    for (int x = 0; x < N; ++x) {
      const double a = -2.0 * M_PI * (double)k * x / N;
      const double c = std::cos(a), s = std::sin(a);
      tF[kk * N + x] = make_float2((float)c, (float)s);
      tFs[kk * N + x] = make_float2((float)(c / N), (float)(s / N));
      tG[x * K + kk] = make_float2((float)(c / N), (float)(-s / N));
      tGs[x * K + kk] = make_float2((float)c, (float)(-s));
    }
  }
  cudaError_t e = cudaSuccess;
  auto A = [&](auto** p, size_t cnt) {
    if (e == cudaSuccess) e = fno_alloc(h, p, cnt);
  };
  A(&h->c0, N);
  A(&h->p32, h->L.total); A(&h->p16, h->L.total); A(&h->grad, h->L.total);
  A(&h->am, h->L.total); A(&h->av, h->L.total);
  A(&h->tF, K * N); A(&h->tG, K * N); A(&h->tFs, K * N); A(&h->tGs, K * N);
  A(&h->x0, B * n * fno::CIN);
  for (int l = 0; l < 5; ++l) A(&h->v[l], B * n * fno::WD);
  for (int l = 0; l < 4; ++l) A(&h->y[l], B * n * fno::WD);
  const long nm = (long)K * K * K;
  for (int l = 0; l < 4; ++l) A(&h->Vh[l], B * nm * fno::WD);
  A(&h->Uh, B * nm * fno::WD);
  A(&h->gUh, B * nm * fno::WD);
  A(&h->gVh, B * nm * fno::WD);
  A(&h->Yp, B * N * K * K * fno::WD);
  A(&h->Sp, B * N * K * K * fno::WD);
  A(&h->T1, B * K * N * N * fno::WD);
  A(&h->T2, B * K * K * N * fno::WD);
  A(&h->U, B * n * fno::WD);
  A(&h->out, B * n);
  A(&h->qs, B);
  A(&h->fpart, B * fno::FCH * 6);
  A(&h->dout, B * n);
  A(&h->dz, B * n * fno::PJ);
  A(&h->aw, B * n * fno::PJ);
  A(&h->dvA, B * n * fno::WD);
  A(&h->dvB, B * n * fno::WD);
  A(&h->dy, B * n * fno::WD);
  A(&h->part, (size_t)kFnoWgradGrid * fno::WD * fno::PJ);
  A(&h->loss, B);
  A(&h->err, 1);
  if (e == cudaSuccess) e = cudaMemcpy(h->c0, c0.data(), N * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->tF, tF.data(), K * N * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->tG, tG.data(), K * N * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->tFs, tFs.data(), K * N * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->tGs, tGs.data(), K * N * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(h->p32, 0, h->L.total * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(h->p16, 0, h->L.total * sizeof(__nv_bfloat16));
  if (e == cudaSuccess) e = cudaMemset(h->err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(h->am, 0, h->L.total * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(h->av, 0, h->L.total * sizeof(float));
  if (e != cudaSuccess) {
    fno_free(h);
    return fail(DGFS_ERR_CUDA, std::string("FNO allocation: ") + cudaGetErrorString(e));
  }
  if (int rc_s = settle_uploads()) { fno_free(h); return rc_s; }
  *out = h;
  return DGFS_OK;
}

extern "C" int dgfs_fno_destroy(dgfs_fno_handle h) {
  if (h) fno_free(h);
  return DGFS_OK;
}

extern "C" int64_t dgfs_fno_num_params(dgfs_fno_handle h) {
  return h ? (int64_t)h->L.total : 0;
}

extern "C" int dgfs_fno_set_params(dgfs_fno_handle h, const float* host) {
  if (!h || !host) return fail(DGFS_ERR_INVALID, "null argument");
  DGFS_CUDA(cudaMemcpy(h->p32, host, h->L.total * sizeof(float), cudaMemcpyHostToDevice));
  fno::fno_to_bf16_kernel<<<(unsigned)((h->L.total + 255) / 256), 256>>>(h->p32, h->p16, h->L.total);
  DGFS_CUDA(cudaGetLastError());
  DGFS_CUDA(cudaMemset(h->am, 0, h->L.total * sizeof(float)));
  DGFS_CUDA(cudaMemset(h->av, 0, h->L.total * sizeof(float)));
  DGFS_CUDA(cudaDeviceSynchronize());
  return DGFS_OK;
}

extern "C" int dgfs_fno_get_params(dgfs_fno_handle h, float* host) {
  if (!h || !host) return fail(DGFS_ERR_INVALID, "null argument");
  DGFS_CUDA(cudaDeviceSynchronize());
  DGFS_CUDA(cudaMemcpy(host, h->p32, h->L.total * sizeof(float), cudaMemcpyDeviceToHost));
  return DGFS_OK;
}

extern "C" int dgfs_fno_get_grads(dgfs_fno_handle h, float* host) {
  if (!h || !host) return fail(DGFS_ERR_INVALID, "null argument");
  DGFS_CUDA(cudaDeviceSynchronize());
  DGFS_CUDA(cudaMemcpy(host, h->grad, h->L.total * sizeof(float), cudaMemcpyDeviceToHost));
  return DGFS_OK;
}

template <int LIN, int LOUT, int IN, int OUT>
static int fno_dft(const void* in, void* out, const float2* table, long outer,
                   int inner, cudaStream_t st) {
  const long tot = outer * (inner / 2);
  fno::fno_dft_kernel<LIN, LOUT, IN, OUT>
      <<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(in, out, table, outer, inner);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

// forward DFT of a real field [B][n][WD] (IN: 0 BF16, 1 FP32) into [B][K^3][WD]:
// one pass per axis (the y and z passes read 32 complex values per pencil,
// which keeps every thread busy; a fused y/z kernel idles 60% of its
// threads in the y pass and measured slower)
template <int N, int K, int IN>
static int fno_dft3(dgfs_fno_s* h, const void* in, const float2* tab, float2* out,
                    int B, cudaStream_t st) {
  constexpr int WD = fno::WD;
  int rc;
  if ((rc = fno_dft<N, K, IN, 0>(in, h->T1, tab, B, N * N * WD, st))) return rc;
  if ((rc = fno_dft<N, K, 2, 0>(h->T1, h->T2, tab, (long)B * K, N * WD, st))) return rc;
  return fno_dft<N, K, 2, 0>(h->T2, out, tab, (long)B * K * K, WD, st);
}

// expand [B][K^3][WD] complex to the real part on the grid: fused z/y
// passes, then the x pass (OUT: 2 FP32 add, 3 BF16 store)
template <int N, int K, int OUT>
static int fno_idft3(dgfs_fno_s* h, const float2* in, const float2* tab, void* out,
                     int B, cudaStream_t st) {
  constexpr int WD = fno::WD;
  const size_t smem = (size_t)(K * K * fno::DCG + K * N * fno::DCG + N * K) * sizeof(float2);
  if (smem > 48 * 1024)
    DGFS_CUDA(cudaFuncSetAttribute(fno::fno_dft_zy_inv_kernel<N, K>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  fno::fno_dft_zy_inv_kernel<N, K><<<dim3(WD / fno::DCG, K, B), 256, smem, st>>>(
      in, h->T1, tab);
  DGFS_CUDA(cudaGetLastError());
  return fno_dft<K, N, 2, OUT>(h->T1, out, tab, B, N * N * WD, st);
}

// Dense layer / projection on the tensor cores: persistent 128-row tiles.
template <int NC, int EPI>
static int fno_tc(dgfs_fno_s* h, const fno::TcArgs& a, cudaStream_t st) {
  const long ntiles = (a.R + 127) / 128;
  // NC=128: pad shared memory so that at most 3 CTAs share an SM (3 x 128 of
  // the 512 TMEM columns); NC=32: 16 CTAs x 32 columns fit
  const size_t pad = NC == 128 ? 40 * 1024 : 0;
  const int per_sm = NC == 128 ? 3 : 8;
  const unsigned grid = (unsigned)std::min<long>(ntiles, 148L * per_sm);
  if (pad)
    DGFS_CUDA(cudaFuncSetAttribute(fno::fno_tc_kernel<NC, EPI>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)pad));
  fno::fno_tc_kernel<NC, EPI><<<grid, 128, pad, st>>>(a);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

template <int N, int K>
static int fno_forward(dgfs_fno_s* h, const void* f, int f_double,
                       const int32_t* src_slots, int src_base, int B,
                       cudaStream_t st, bool store_y = true) {
  using namespace fno;
  const long R = (long)B * h->n;
  const long nm = (long)K * K * K;
  int rc;
  FeatArgs fa{};
  fa.f = f; fa.f_double = f_double; fa.src_slots = src_slots; fa.src_base = src_base;
  fa.c0 = h->c0; fa.cw = h->cw; fa.N = N; fa.w16 = h->p16; fa.L = h->L;
  fa.x0 = h->x0; fa.v0 = h->v[0]; fa.qs = h->qs; fa.part = h->fpart;
  const dim3 fg(FCH, B);
  fno_features_kernel<0><<<fg, 256, 0, st>>>(fa);
  fno_features_kernel<1><<<fg, 256, 0, st>>>(fa);
  fno_features_kernel<2><<<fg, 256, 0, st>>>(fa);
  DGFS_CUDA(cudaGetLastError());
  for (int l = 0; l < 4; ++l) {
    if ((rc = fno_dft3<N, K, 0>(h, h->v[l], h->tF, h->Vh[l], B, st))) return rc;
    fno_mix_kernel<0><<<(unsigned)nm, dim3(32, 8), 0, st>>>(
        h->Vh[l], nullptr, h->p16 + h->L.W[l], h->Uh, nullptr, B, (int)nm);
    DGFS_CUDA(cudaGetLastError());
    if ((rc = fno_idft3<N, K, 3>(h, h->Uh, h->tG, h->U, B, st))) return rc;
    if (h->use_tc) {
      TcArgs ta{};
      ta.x = h->v[l]; ta.w16 = h->p16; ta.offW = h->L.D[l]; ta.offb = h->L.d[l];
      ta.U = h->U; ta.y = store_y ? h->y[l] : nullptr; ta.v = h->v[l + 1];
      ta.R = R; ta.act = l < 3 ? 1 : 0; ta.err = h->err;
      if ((rc = fno_tc<WD, 0>(h, ta, st))) return rc;
    } else {
      fno_dense_fwd_kernel<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(
          h->v[l], h->p16, h->L.D[l], h->L.d[l], h->U, h->y[l], h->v[l + 1], R,
          l < 3 ? 1 : 0);
      DGFS_CUDA(cudaGetLastError());
    }
  }
  if (h->use_tc) {
    TcArgs ta{};
    ta.x = h->v[4]; ta.w16 = h->p16; ta.offW = h->L.Q1; ta.offb = h->L.q1;
    ta.offq2 = h->L.q2; ta.offq2b = h->L.q2b; ta.out = h->out; ta.R = R;
    ta.err = h->err;
    if ((rc = fno_tc<PJ, 1>(h, ta, st))) return rc;
  } else {
    fno_proj_fwd_kernel<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(
        h->v[4], h->p16, h->L, h->out, R);
    DGFS_CUDA(cudaGetLastError());
  }
  return DGFS_OK;
}

// Inference forward with the fused spectral passes (see fno_kernels.cuh):
// per layer one x-mix launch and one yz-inverse + dense launch, and one
// yz-forward launch for the next layer's spectra.
template <int N, int K>
static int fno_forward_fused(dgfs_fno_s* h, const void* f, int f_double,
                             const int32_t* src_slots, int src_base, int B,
                             cudaStream_t st) {
  using namespace fno;
  const long R = (long)B * h->n;
  FeatArgs fa{};
  fa.f = f; fa.f_double = f_double; fa.src_slots = src_slots; fa.src_base = src_base;
  fa.c0 = h->c0; fa.cw = h->cw; fa.N = N; fa.w16 = h->p16; fa.L = h->L;
  fa.x0 = h->x0; fa.v0 = h->v[0]; fa.qs = h->qs; fa.part = h->fpart;
  const dim3 fg(FCH, B);
  fno_features_kernel<0><<<fg, 256, 0, st>>>(fa);
  fno_features_kernel<1><<<fg, 256, 0, st>>>(fa);
  fno_features_kernel<2><<<fg, 256, 0, st>>>(fa);
  DGFS_CUDA(cudaGetLastError());
  const int fsm = N * K * WD * (int)sizeof(float2);
  const int xsm = 2 * K * K * WD * (int)sizeof(float2);
  const int ism = YzInvGeo<N, K>::SMEM;
  DGFS_CUDA(cudaFuncSetAttribute(fno_yzfwd_kernel<N, K>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, fsm));
  DGFS_CUDA(cudaFuncSetAttribute(fno_xmix_kernel<N, K>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, xsm));
  DGFS_CUDA(cudaFuncSetAttribute(fno_yzinv_dense_kernel<N, K>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, ism));
  const dim3 pg(N, B);
  fno_yzfwd_kernel<N, K><<<pg, 256, fsm, st>>>(h->v[0], h->Yp);
  DGFS_CUDA(cudaGetLastError());
  for (int l = 0; l < 4; ++l) {
    fno_xmix_kernel<N, K><<<dim3(K * K, (B + K - 1) / K), K * 32, xsm, st>>>(
        h->Yp, h->p16 + h->L.W[l], h->Sp, B);
    YzInvArgs ya{};
    ya.S = h->Sp; ya.v = h->v[l]; ya.w16 = h->p16; ya.offD = h->L.D[l];
    ya.offd = h->L.d[l]; ya.vout = h->v[l + 1]; ya.act = l < 3 ? 1 : 0;
    ya.err = h->err;
    fno_yzinv_dense_kernel<N, K><<<dim3(N * YzInvGeo<N, K>::ZP, B),
                                   YzInvGeo<N, K>::NT, ism, st>>>(ya);
    if (l < 3) fno_yzfwd_kernel<N, K><<<pg, 256, fsm, st>>>(h->v[l + 1], h->Yp);
    DGFS_CUDA(cudaGetLastError());
  }
  TcArgs ta{};
  ta.x = h->v[4]; ta.w16 = h->p16; ta.offW = h->L.Q1; ta.offb = h->L.q1;
  ta.offq2 = h->L.q2; ta.offq2b = h->L.q2b; ta.out = h->out; ta.R = R;
  ta.err = h->err;
  return fno_tc<PJ, 1>(h, ta, st);
}

template <int KA, int KB>
static int fno_wgrad(dgfs_fno_s* h, const __nv_bfloat16* A, const float* Bm,
                     long R, long off, cudaStream_t st) {
  constexpr int RI = KA < 4 ? KA : 4;
  constexpr int NTH = (KA / RI) * (KB / 4);
  fno::fno_wgrad_kernel<KA, KB><<<kFnoWgradGrid, NTH, 0, st>>>(A, Bm, R, h->part);
  DGFS_CUDA(cudaGetLastError());
  fno::fno_reduce_kernel<<<(KA * KB + 255) / 256, 256, 0, st>>>(
      h->part, kFnoWgradGrid, KA * KB, h->grad + off);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

template <int KB>
static int fno_colsum(dgfs_fno_s* h, const float* Bm, long R, long off,
                      cudaStream_t st) {
  fno::fno_colsum_kernel<KB><<<kFnoWgradGrid, 256, 0, st>>>(Bm, R, h->part);
  DGFS_CUDA(cudaGetLastError());
  fno::fno_reduce_kernel<<<(KB + 255) / 256, 256, 0, st>>>(h->part, kFnoWgradGrid,
                                                           KB, h->grad + off);
  DGFS_CUDA(cudaGetLastError());
  return DGFS_OK;
}

// gradients of the loss (dout already set) w.r.t. every parameter
template <int N, int K>
static int fno_backward(dgfs_fno_s* h, int B, cudaStream_t st) {
  using namespace fno;
  const long R = (long)B * h->n;
  const long nm = (long)K * K * K;
  const unsigned gR = (unsigned)((R + 255) / 256);
  int rc;
  // projection
  fno_proj_bwd_kernel<<<gR, 256, 0, st>>>(h->v[4], h->p16, h->L, h->dout, h->dz,
                                          h->aw, h->dvA, R);
  DGFS_CUDA(cudaGetLastError());
  if ((rc = fno_wgrad<WD, PJ>(h, h->v[4], h->dz, R, h->L.Q1, st))) return rc;
  if ((rc = fno_colsum<PJ>(h, h->dz, R, h->L.q1, st))) return rc;
  if ((rc = fno_colsum<PJ>(h, h->aw, R, h->L.q2, st))) return rc;
  if ((rc = fno_colsum<1>(h, h->dout, R, h->L.q2b, st))) return rc;
  float* dv = h->dvA;     // gradient w.r.t. v_{l+1}
  float* dvn = h->dvB;
  for (int l = 3; l >= 0; --l) {
    const float* dyl = dv;
    if (l < 3) {
      fno_gelu_bwd_kernel<<<(unsigned)((R * WD + 255) / 256), 256, 0, st>>>(
          dv, h->y[l], h->dy, R * WD);
      DGFS_CUDA(cudaGetLastError());
      dyl = h->dy;
    }
    if ((rc = fno_wgrad<WD, WD>(h, h->v[l], dyl, R, h->L.D[l], st))) return rc;
    if ((rc = fno_colsum<WD>(h, dyl, R, h->L.d[l], st))) return rc;
    fno_dense_bwd_kernel<<<gR, 256, 0, st>>>(dyl, h->p16, h->L.D[l], dvn, R);
    DGFS_CUDA(cudaGetLastError());
    // spectral path: gUh = B^H dy, gW, gVh = gUh W^H, dv += Re(A^H gVh)
    if ((rc = fno_dft3<N, K, 1>(h, dyl, h->tFs, h->gUh, B, st))) return rc;
    fno_mix_kernel<2><<<(unsigned)nm, dim3(32, 8), 0, st>>>(
        h->Vh[l], h->gUh, nullptr, nullptr, h->grad + h->L.W[l], B, (int)nm);
    DGFS_CUDA(cudaGetLastError());
    fno_mix_kernel<1><<<(unsigned)nm, dim3(32, 8), 0, st>>>(
        h->gUh, nullptr, h->p16 + h->L.W[l], h->gVh, nullptr, B, (int)nm);
    DGFS_CUDA(cudaGetLastError());
    if ((rc = fno_idft3<N, K, 2>(h, h->gVh, h->tGs, dvn, B, st))) return rc;
    std::swap(dv, dvn);
  }
  // lift
  if ((rc = fno_wgrad<CIN, WD>(h, h->x0, dv, R, h->L.P, st))) return rc;
  return fno_colsum<WD>(h, dv, R, h->L.p, st);
}

template <int N, int K>
static int fno_eval_t(dgfs_fno_s* h, const void* f, int f_double, void* Q,
                      int q_double, const int32_t* src_slots, int src_base,
                      const int32_t* dst_slots, int dst_base, int nevals,
                      cudaStream_t st) {
  for (int off = 0; off < nevals; off += h->maxB) {
    const int B = std::min(h->maxB, nevals - off);
    int rc;
    const int32_t* ss = src_slots ? src_slots + off : nullptr;
    if ((rc = (h->use_fused && h->use_tc)
                  ? fno_forward_fused<N, K>(h, f, f_double, ss, src_base + off, B, st)
                  : fno_forward<N, K>(h, f, f_double, ss, src_base + off, B, st, false)))
      return rc;
    fno::OutArgs oa{};
    oa.out = h->out; oa.qs = h->qs; oa.sQ = h->sQ; oa.c0 = h->c0; oa.cw = h->cw;
    oa.N = N;
    for (int i = 0; i < 25; ++i) oa.Ginv[i] = h->Ginv[i];
    oa.Q = Q; oa.q_double = q_double;
    oa.dst_slots = dst_slots ? dst_slots + off : nullptr; oa.dst_base = dst_base + off;
    oa.part = h->fpart;
    fno::fno_output_kernel<0><<<dim3(fno::FCH, B), 256, 0, st>>>(oa);
    fno::fno_output_kernel<1><<<dim3(fno::FCH, B), 256, 0, st>>>(oa);
    DGFS_CUDA(cudaGetLastError());
  }
  return DGFS_OK;
}

extern "C" int dgfs_fno_eval(dgfs_fno_handle h, const void* f, int32_t f_dtype,
                             void* Q, int32_t q_dtype, const int32_t* src_slots,
                             int32_t src_base, const int32_t* dst_slots,
                             int32_t dst_base, int32_t nevals, void* stream) {
  NvtxRange nvtx_range("dgfs_fno_eval");
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  if (nevals < 0 || src_base < 0 || dst_base < 0)
    return fail(DGFS_ERR_INVALID, "negative count or slot base");
  if (nevals == 0) return DGFS_OK;
  if (!f || !Q) return fail(DGFS_ERR_INVALID, "null f or Q");
  if ((f_dtype != DGFS_F32 && f_dtype != DGFS_F64) ||
      (q_dtype != DGFS_F32 && q_dtype != DGFS_F64))
    return fail(DGFS_ERR_INVALID, "dtype must be DGFS_F32 or DGFS_F64");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int fd = f_dtype == DGFS_F64, qd = q_dtype == DGFS_F64;
  if (h->N == 16)
    return fno_eval_t<16, 8>(h, f, fd, Q, qd, src_slots, src_base, dst_slots,
                             dst_base, nevals, st);
  return fno_eval_t<32, 12>(h, f, fd, Q, qd, src_slots, src_base, dst_slots,
                            dst_base, nevals, st);
}

template <int N, int K>
static int fno_train_t(dgfs_fno_s* h, const double* f, const double* Qt, int B,
                       float lr, int step, int update, cudaStream_t st) {
  int rc;
  if ((rc = fno_forward<N, K>(h, f, 1, nullptr, 0, B, st))) return rc;
  fno::fno_loss_kernel<512><<<B, 512, 0, st>>>(h->out, Qt, h->qs, h->sQ, h->n,
                                                B, h->dout, h->loss);
  DGFS_CUDA(cudaGetLastError());
  if ((rc = fno_backward<N, K>(h, B, st))) return rc;
  if (update) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - std::pow(b1, (float)step);
    const float bc2 = 1.f - std::pow(b2, (float)step);
    fno::fno_adam_kernel<<<(unsigned)((h->L.total + 255) / 256), 256, 0, st>>>(
        h->p32, h->p16, h->grad, h->am, h->av, h->L.total, lr, b1, b2, 1e-8f,
        bc1, bc2);
    DGFS_CUDA(cudaGetLastError());
  }
  return DGFS_OK;
}

extern "C" int dgfs_fno_train_step(dgfs_fno_handle h, const double* f,
                                   const double* Qt, int32_t B, float lr,
                                   int32_t step, int32_t update, void* stream) {
  if (!h || !f || !Qt) return fail(DGFS_ERR_INVALID, "null argument");
  if (B < 1 || B > h->maxB) return fail(DGFS_ERR_CAPACITY, "batch exceeds max_batch");
  if (update && step < 1) return fail(DGFS_ERR_INVALID, "Adam step counts from 1");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->N == 16) return fno_train_t<16, 8>(h, f, Qt, B, lr, step, update, st);
  return fno_train_t<32, 12>(h, f, Qt, B, lr, step, update, st);
}

extern "C" int dgfs_fno_last_loss(dgfs_fno_handle h, double* host, int32_t B) {
  if (!h || !host) return fail(DGFS_ERR_INVALID, "null argument");
  if (B < 1 || B > h->maxB) return fail(DGFS_ERR_INVALID, "bad batch size");
  DGFS_CUDA(cudaDeviceSynchronize());
  DGFS_CUDA(cudaMemcpy(host, h->loss, B * sizeof(double), cudaMemcpyDeviceToHost));
  return DGFS_OK;
}

extern "C" int dgfs_fno_set_tensor_cores(dgfs_fno_handle h, int32_t enable) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  h->use_tc = enable ? 1 : 0;
  return DGFS_OK;
}

extern "C" int dgfs_fno_set_fused(dgfs_fno_handle h, int32_t enable) {
  if (!h) return fail(DGFS_ERR_INVALID, "null handle");
  h->use_fused = enable ? 1 : 0;
  return DGFS_OK;
}

extern "C" int dgfs_fno_error(dgfs_fno_handle h, int32_t* out) {
  if (!h || !out) return fail(DGFS_ERR_INVALID, "null argument");
  DGFS_CUDA(cudaDeviceSynchronize());
  int v = 0;
  DGFS_CUDA(cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost));
  DGFS_CUDA(cudaMemset(h->err, 0, sizeof(int)));
  *out = v;
  return DGFS_OK;
}

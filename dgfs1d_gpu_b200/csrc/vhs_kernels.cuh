// Fused fast-spectral VHS collision operator Q(f,f) for a batch of spatial
// points ("evals").  Reference: DGFSVHSGLLScatteringModelStd.fs
// (dgfs1D/std/scattering.py:251-313) and its kernels in
// dgfs1D/std/kernels/scattering/vhs-gll.mako.
//
// Per eval the reference computes (cuFFT conventions, F = FFT(f)/n):
//   t3_pq = IFFT(cos a_pq F), t4_pq = IFFT(sin a_pq F),
//   a_pq(l) = (pi/L)(rho_p/2) sigma_q . l
//   Ghat  = sum_p (sf w_p s_w / n) b1_p sum_q FFT(t3^2 + t4^2)
//   Q    += prefac * (Re IFFT(Ghat) - f * Re IFFT(b2 F))
// The kernels below restructure this without changing its value:
//   * linearity: sum_q FFT(h_pq) = FFT(sum_q h_pq) (one forward FFT per p);
//   * antipodal pairs sigma_q' = -sigma_q give identical h, so only one of
//     each pair is transformed, with multiplicity 2;
//   * a_pq is linear in l, so exp(i a) is the product of three 1-D phase
//     tables and is never stored;
//   * in the FP32 mode, f = M + g with M the separable local Maxwellian: the
//     M-parts of t3, t4, h and FFT(h) are products of 1-D transforms computed
//     in FP64, and only the small remainder g runs through FP32 3-D FFTs.
//
// Kernels (one stage = prologue, [tables, maxwell_gain], terms, epilogue):
//   prologue   (cluster per eval, FP64): F, moments, Maxwellian spectra,
//              F_g = F - M_hat, Re IFFT(b2 F)
//   tables     (FP64): per (eval,p,q) 1-D u_a, v_a and FFT(u_a v_a)
//   maxwell_gain (FP64): Ghat_M = sum_p W_p b1_p sum_q m_q prod_a FFT(u_a v_a)
//   terms      (cluster per (eval,p), precision R): H_p = W_p b1_p FFT(S_p)
//   epilogue   (cluster per eval, FP64): Ghat = Ghat_M + sum_p H_p,
//              Q += prefac (Re IFFT(Ghat) - f Re IFFT(b2 F))
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cuda.h>

#include "cluster_slab.cuh"
#include "fft_reg.cuh"

namespace dgfs {

struct VhsPrologueArgs {
  const void* f;              // input distribution (float or double)
  const void* const* f_list;  // or, if set, one input array per evaluation
                              // (device array [nevals]; slots index into it)
  int f_double;               // 1: f is double
  const void* g;              // optional second input (same dtype as f): the
                              // transformed input is then alpha f + beta g
  double alpha, beta;
  const int32_t* src_slots;   // device slot list or null
  int src_base;               // slot(i) = src_slots ? src_slots[i] : src_base+i
  const double* c0;           // [N] velocity grid (x, y and z)
  const double* b2;           // [n] loss kernel b2(l)
  const double2* b2c;         // [n] complex loss kernel (used instead of b2
                              // when set: the VSS c_pq)
  double cw;                  // velocity cell volume
  int split;                  // 1: Maxwellian split (FP32 mode)
  void* Fg;                   // out [nevals][n] complex (float2 if split else double2)
  double* ReLf;               // out [nevals][n] Re IFFT(b2 F)
  double2* mhat;              // out [nevals][3][N] Maxwellian 1-D spectra (split)
  double* moments;            // out [nevals][5] rho, ux, uy, uz, T (split)
                              // Fg, mhat and moments may be null (split):
                              // the launch then only writes the loss
  float2* Fny;                // out (split) [nevals][3][N][N] Nyquist planes of
                              // F_g: [0][ly][lz] at lx=N/2, [1][lx][lz] at
                              // ly=N/2, [2][lx][ly] at lz=N/2
};

struct VhsTermsArgs {
  const void* Fg;             // [nevals][n] complex, precision R
  const void* ph;             // [Nrho][Mu][3][N] exp(i kappa_a rep(l)), precision R
  const void* uv;             // [nevals][Nrho][Mu][2][3][N] u_a, v_a (split)
  const float* mult;          // [Mu] multiplicity of each transformed direction
  const void* b1w;            // [Nrho][n] W_p b1_p(l), precision R
  void* H;                    // out [nevals][Nrho][n] complex, precision R
                              // (FP32: [nevals][ceil(Nrho/2)][n], packed pairs)
  const void* nyq;            // FP32: [Nrho][Mu][3] exp(i N kappa_a)
  const void* Fny;            // FP32: [nevals][3][N][N] Nyquist planes of F_g
  void* rho;                  // FP32: [nevals][Nrho][Mu][3][N][N] plane transforms
  int Mu;
  int Nrho;
  int* err;                   // device error flag (a bounded wait gave up)
};

struct VhsTablesArgs {
  const double2* mhat;        // [nevals][3][N]
  const float* mult;          // [Mu] (FP32 tables carry sqrt(mult) on axis x)
  const double* kappa;        // [Nrho][Mu][3] kappa_a = (pi/L)(rho_p/2) sigma_qa
  void* uv;                   // out [nevals][Nrho][Mu][2][3][N] precision R
  double2* hh;                // out [nevals][Nrho][Mu][3][N] FFT(u_a v_a)
  int Mu;
  int Nrho;
  int nevals;
  int uv_double;              // 1: uv stored as double2
};

struct VhsGainArgs {
  const double2* hh;          // [nevals][Nrho][Mu][3][N]
  const float* mult;          // [Mu]
  const double* b1w;          // [Nrho][n] W_p b1_p(l)
  double2* GM;                // out [nevals][n]
  int Mu;
  int Nrho;
  int pch;                    // radial points staged per shared-memory chunk
};

struct VhsEpilogueArgs {
  const void* H;              // [nevals][Nrho][n] precision R
  int h_double;
  const double2* GM;          // [nevals][n] or null
  const double* ReLf;         // [nevals][n]
  const void* f;              // input distribution
  const void* const* f_list;  // or one input array per evaluation
  int f_double;
  const int32_t* src_slots;
  int src_base;
  void* Q;                    // output distribution (+=)
  void* const* q_list;        // or one output array per evaluation
  int q_double;
  const int32_t* dst_slots;
  int dst_base;
  double prefac;
  int Nrho;
  // conservation projection (no reference counterpart): Q <- Q - sum_k
  // lambda_k phi_k with phi = (1, cx, cy, cz, |c|^2) and G lambda = moments
  // of Q, G_jk = sum_v phi_j phi_k cw; Ginv = G^{-1} (row-major)
  int project;
  const double* c0;           // [N]
  double cw;
  double Ginv[25];
  // bilinear component (polarisation of the gain, see dgfs_vhs_eval2):
  // Q += prefac (cg Re G - cl f Re Lf) instead of prefac (Re G - f Re Lf)
  int bilinear;
  double cg, cl;
  // several pair operators into one output (the VSS species sum): when
  // nt > 0, Ghat = sum_t pref[t] (GMt[t] + sum_p Ht[t][p]) and the loss is
  // f sum_t pref[t] ReLft[t] (FP32 H); H, GM, ReLf and prefac are unused
  int nt;
  const void* Ht[4];
  const double2* GMt[4];
  const double* ReLft[4];
  double pref[4];
};

__device__ __forceinline__ int slot_of(const int32_t* slots, int base, int i) {
  return slots ? slots[i] : base + i;
}
__device__ __forceinline__ double load_real(const void* p, int is_double,
                                            size_t idx) {
  return is_double ? static_cast<const double*>(p)[idx]
                   : (double)static_cast<const float*>(p)[idx];
}

// ---------------------------------------------------------------------------
// Prologue: one cluster (C CTAs, FP64) per eval.  Up to N=32 one slab per CTA
// serves both transforms (the exchange of the inverse transform waits for
// every CTA to have read its slab), which keeps a 24-point batch in one wave.
// ---------------------------------------------------------------------------
// Whether the prologue and epilogue keep one slab per CTA (exchange after a
// cluster barrier) or a separate receive slab.  One slab pays off where it
// lets more CTAs share an SM (N <= 32); at N=48 registers allow one CTA per
// SM either way and the second slab saves the barrier.
template <int N> struct OneSlab { static constexpr bool value = N <= 32; };

// Shared memory: the slab(s), the moment partials [5][NT] + [5] and the 1-D
// Maxwellian factors [3N] (doubles; with two slabs they borrow the receive
// slab, which peers write only two cluster barriers later), the Maxwellian
// spectra [3][N] (complex) and the moments [8].
template <int N, int C>
constexpr size_t prologue_smem() {
  // ... + the N twiddles of the 1-D spectra (double2)
  return OneSlab<N>::value
             ? (size_t)Geo<N, C>::SLAB * sizeof(double2) +
                   (size_t)(6 * Geo<N, C>::NT + 8 + 3 * N) * sizeof(double) +
                   (size_t)3 * N * sizeof(double2) + 8 * sizeof(double) +
                   (size_t)N * sizeof(double2)
             : (size_t)2 * Geo<N, C>::SLAB * sizeof(double2) +
                   (size_t)3 * N * sizeof(double2) + 8 * sizeof(double) +
                   (size_t)N * sizeof(double2);
}
template <int N, int C>
constexpr size_t epilogue_smem() {
  return (size_t)(OneSlab<N>::value ? 1 : 2) * Geo<N, C>::SLAB * sizeof(double2);
}

template <int N, int C>
__global__ void __launch_bounds__(Geo<N, C>::NT)
vhs_prologue_kernel(VhsPrologueArgs a) {
  using G = Geo<N, C>;
  using T = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr bool OS = OneSlab<N>::value;
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Rb = OS ? A : A + G::SLAB;                             // Y-slab receive
  double* red = OS ? reinterpret_cast<double*>(A + G::SLAB)  // [6 NT + 8 + 3N]
                   : reinterpret_cast<double*>(Rb);
  T* mh = OS ? reinterpret_cast<T*>(red + 6 * G::NT + 8 + 3 * N)
             : A + 2 * G::SLAB;                              // [3][N]
  double* mom = reinterpret_cast<double*>(mh + 3 * N);      // [8]
  T* tws = reinterpret_cast<T*>(mom + 8);                   // [N] twiddles

  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int e = blockIdx.y;
  const int yl = t / N, z = t % N, y = rank * G::P + yl;
  const size_t fbase = (size_t)slot_of(a.src_slots, a.src_base, e) * G::n;
  const void* fin = a.f_list ? a.f_list[e] : a.f;

  T v[N];
#pragma unroll
  for (int x = 0; x < N; ++x) {
    const size_t idx = fbase + ((size_t)x * N + y) * N + z;
    v[x].x = a.g ? a.alpha * load_real(fin, a.f_double, idx) +
                       a.beta * load_real(a.g, a.f_double, idx)
                 : load_real(fin, a.f_double, idx);
    v[x].y = 0.0;
  }

  if (a.split) {
    // moments of f on the grid (sum f, sum f c, sum f |c|^2); deterministic
    // two-level reduction: per-thread partials -> CTA -> cluster.
    double s[5] = {0, 0, 0, 0, 0};
    const double cy = a.c0[y], cz = a.c0[z];
#pragma unroll
    for (int x = 0; x < N; ++x) {
      const double cx = a.c0[x], fv = v[x].x;
      s[0] += fv;
      s[1] += fv * cx;
      s[2] += fv * cy;
      s[3] += fv * cz;
      s[4] += fv * (cx * cx + cy * cy + cz * cz);
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) red[k * G::NT + t] = s[k];
    // the spectra's twiddles into shared memory (read below with a
    // different index on every lane, which constant memory serialises)
    for (int i = t; i < N; i += G::NT) tws[i] = c_tw64[tw_offset(N) + i];
    __syncthreads();
    // this CTA's partial of moment k = t / 8: eight lanes each sum a strided
    // eighth of the thread partials, then a three-step xor tree inside the
    // eight-lane group (a fixed order: every run adds the same operands)
    if (t < 40) {
      const int k = t >> 3, sub = t & 7;
      double acc = 0;
      for (int i = sub; i < G::NT; i += 8) acc += red[k * G::NT + i];
      const unsigned grp = t < 32 ? 0xFFFFFFFFu : 0xFFu;  // lanes in this branch
      acc += __shfl_xor_sync(grp, acc, 4, 8);
      acc += __shfl_xor_sync(grp, acc, 2, 8);
      acc += __shfl_xor_sync(grp, acc, 1, 8);
      if (sub == 0) red[5 * G::NT + k] = acc;
    }
    cluster_sync_all();
    if (t < 5) {
      double acc = 0;
      for (int c = 0; c < C; ++c)
        acc += peer_ptr(red, (unsigned)c)[5 * G::NT + t];
      mom[t] = acc;
    }
    __syncthreads();
    if (t == 0) {
      double rho = mom[0] * a.cw, ux = 0, uy = 0, uz = 0, Tm = 1;
      if (rho > 1e-300) {
        ux = mom[1] * a.cw / rho; uy = mom[2] * a.cw / rho; uz = mom[3] * a.cw / rho;
        Tm = (2.0 / 3.0) * (mom[4] * a.cw / rho - (ux * ux + uy * uy + uz * uz));
        if (!(Tm > 1e-6)) { rho = 0; Tm = 1; }  // no useful Maxwellian
      } else {
        rho = 0;
      }
      mom[0] = rho; mom[1] = ux; mom[2] = uy; mom[3] = uz; mom[4] = Tm;
      if (rank == 0 && a.moments)
        for (int k = 0; k < 5; ++k) a.moments[(size_t)e * 5 + k] = mom[k];
    }
    __syncthreads();
    // 1-D Maxwellian factors (3N values, each computed once; past the moment
    // partials, which peers read only below offset 5 NT + 5) and their
    // spectra (direct DFT, table twiddles)
    double* mv = red + 6 * G::NT + 8;
    for (int i = t; i < 3 * N; i += G::NT) {
      const int ax = i / N, j = i % N;
      const double rho = mom[0], Tm = mom[4], u = mom[1 + ax];
      const double amp = (ax == 0) ? rho / pow(M_PI * Tm, 1.5) : 1.0;
      const double d = a.c0[j] - u;
      mv[i] = amp * exp(-d * d / Tm);
    }
    __syncthreads();
    for (int i = t; i < 3 * N; i += G::NT) {
      const int ax = i / N, k = i % N;
      double re = 0, im = 0;
#pragma unroll 8
      for (int j = 0; j < N; ++j) {
        const double2 w = tws[(j * k) % N];
        const double m = mv[ax * N + j];
        re += m * w.x;
        im += m * w.y;
      }
      mh[ax * N + k] = make_double2(re / N, im / N);
    }
    // (visibility of mh is ensured by the barriers below)
  }

  // forward x-pass and exchange into X-slabs
  fft<double, N, -1>(v);
  push_pencils_to_xslab<double, N, C>(A, t, rank, v);
  cluster_sync_all();
  {
    T w[N];
    slab_col_load_fft<double, N, C, -1>(A, t, w);
    const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
    for (int k = 0; k < N; ++k) A[base + k * G::ROW] = w[k];
  }
  __syncthreads();
  slab_row_pass<double, N, C, -1>(A, t);
  __syncthreads();

  // F = FFT(f)/n; write F (FP64) or F_g = F - mhat (FP32); then A <- b2 F
  const double inv_n = 1.0 / (double)G::n;
  const size_t gbase = (size_t)e * G::n + (size_t)rank * G::P * N * N;
#pragma unroll 4
  for (int j = t; j < G::P * N * N; j += G::NT) {
    const int si = slab_index<N, C>(j);
    T Fv = A[si];
    Fv.x *= inv_n;
    Fv.y *= inv_n;
    if (a.split) {
      const int lx = rank * G::P + j / (N * N), ly = (j / N) % N, lz = j % N;
      const T mm = cmul(cmul(mh[lx], mh[N + ly]), mh[2 * N + lz]);
      float2 g;
      g.x = (float)(Fv.x - mm.x);
      g.y = (float)(Fv.y - mm.y);
      if (a.Fg) static_cast<float2*>(a.Fg)[gbase + j] = g;
      if (a.Fny) {
        float2* ny = a.Fny + (size_t)e * 3 * N * N;
        if (lx == N / 2) ny[ly * N + lz] = g;
        if (ly == N / 2) ny[N * N + lx * N + lz] = g;
        if (lz == N / 2) ny[2 * N * N + lx * N + ly] = g;
      }
    } else {
      static_cast<double2*>(a.Fg)[gbase + j] = Fv;
    }
    if (a.b2c) {
      Fv = cmul(Fv, a.b2c[(size_t)rank * G::P * N * N + j]);
    } else {
      const double b = a.b2[(size_t)rank * G::P * N * N + j];
      Fv.x *= b;
      Fv.y *= b;
    }
    A[si] = Fv;
  }
  if (a.split && rank == 0)
    if (a.mhat)
      for (int i = t; i < 3 * N; i += G::NT) a.mhat[(size_t)e * 3 * N + i] = mh[i];
  __syncthreads();
  // loss: Re IFFT(b2 F); the Y-slab exchange reuses the slab once every CTA
  // of the cluster has read its own
  slab_row_pass<double, N, C, +1>(A, t);
  __syncthreads();
  {
    T w[N];
    slab_col_load_fft<double, N, C, +1>(A, t, w);
    if (OS) cluster_sync_all();
    push_cols_to_yslab<double, N, C>(Rb, t, rank, w);
  }
  cluster_sync_all();
  yslab_load_pencil<double, N, C>(Rb, t, v);
  fft<double, N, +1>(v);
#pragma unroll
  for (int x = 0; x < N; ++x)
    a.ReLf[(size_t)e * G::n + ((size_t)x * N + y) * N + z] = v[x].x;
}

// ---------------------------------------------------------------------------
// Tables: per (eval, p, q, axis) u_a = IFFT(e^{+i k l} mhat_a),
// v_a = IFFT(e^{-i k l} mhat_a), hh_a = FFT(u_a v_a)  (FP64, one thread each).
// ---------------------------------------------------------------------------
template <int N>
__global__ void vhs_tables_kernel(VhsTablesArgs a) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = a.nevals * a.Nrho * a.Mu * 3;
  if (gid >= total) return;
  const int ax = gid % 3;
  const int q = (gid / 3) % a.Mu;
  const int p = (gid / (3 * a.Mu)) % a.Nrho;
  const int e = gid / (3 * a.Mu * a.Nrho);
  const double kap = a.kappa[((size_t)p * a.Mu + q) * 3 + ax];
  const double2* mh = a.mhat + (size_t)e * 3 * N + ax * N;
  double2 u[N], w[N];
#pragma unroll
  for (int l = 0; l < N; ++l) {
    const int rl = (l < N / 2) ? l : l - N;
    double s, c;
    sincos(kap * (double)rl, &s, &c);
    const double2 m = mh[l];
    u[l] = cmul(m, make_double2(c, s));
    w[l] = cmul(m, make_double2(c, -s));
  }
  fft<double, N, +1>(u);
  fft<double, N, +1>(w);
  const size_t tb = (((size_t)e * a.Nrho + p) * a.Mu + q);
  if (a.uv_double) {
    double2* uv = static_cast<double2*>(a.uv) + tb * 6 * N;
#pragma unroll
    for (int l = 0; l < N; ++l) {
      uv[ax * N + l] = u[l];
      uv[(3 + ax) * N + l] = w[l];
    }
  } else {
    float2* uv = static_cast<float2*>(a.uv) + tb * 6 * N;
    const double sc = (ax == 0) ? sqrt((double)a.mult[q]) : 1.0;
#pragma unroll
    for (int l = 0; l < N; ++l) {
      uv[ax * N + l] = make_float2((float)(sc * u[l].x), (float)(sc * u[l].y));
      uv[(3 + ax) * N + l] = make_float2((float)(sc * w[l].x), (float)(sc * w[l].y));
    }
  }
#pragma unroll
  for (int l = 0; l < N; ++l) u[l] = cmul(u[l], w[l]);
  fft<double, N, -1>(u);
  double2* hh = a.hh + tb * 3 * N + ax * N;
#pragma unroll
  for (int l = 0; l < N; ++l) hh[l] = u[l];
}

// ---------------------------------------------------------------------------
// Maxwellian gain: Ghat_M(l) = sum_p W_p b1_p(l) sum_q m_q hx(lx) hy(ly) hz(lz)
// grid (N [lx], nevals), block N*NYB threads: thread (ly0 = t/N, lz = t%N)
// owns the points (lx, ly0 + NYB*k, lz), k < KY.  The 1-D factors of a chunk
// of a.pch radial points are staged in shared memory at once (m_q folded into
// hx), hx*hy is formed once per (p, q, ly) in place of the y table, and the
// b1 weights of the next p are loaded while the current one is summed.
// ---------------------------------------------------------------------------
template <int N>
struct GainGeo {
  static constexpr int NYB = 256 / N;                 // ly rows per pass
  static constexpr int NT = N * NYB;                  // threads
  static constexpr int KY = (N + NYB - 1) / NYB;      // points per thread
};

template <int N>
__global__ void __launch_bounds__(GainGeo<N>::NT)
vhs_maxwell_gain_kernel(VhsGainArgs a) {
  using GG = GainGeo<N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Mu = a.Mu;
  double2* hyz = reinterpret_cast<double2*>(smem_raw);   // [pch][Mu][2][N]
  double2* hxs = hyz + (size_t)a.pch * Mu * 2 * N;       // [pch][Mu]
  const int lx = blockIdx.x, e = blockIdx.y;
  const int t = threadIdx.x, ly0 = t / N, lz = t % N;
  const size_t nn = (size_t)N * N;
  const double* b1 = a.b1w + (size_t)lx * nn + lz;
  double2 Gs[GG::KY];
  double wk[GG::KY];
#pragma unroll
  for (int k = 0; k < GG::KY; ++k) {
    Gs[k] = make_double2(0, 0);
    const int ly = ly0 + GG::NYB * k;
    wk[k] = ly < N ? b1[(size_t)ly * N] : 0.0;  // p = 0
  }
  for (int pc = 0; pc < a.Nrho; pc += a.pch) {
    const int np = min(a.pch, a.Nrho - pc);
    __syncthreads();
    // the y and z tables of the chunk: asynchronous 16-byte copies, all in
    // flight at once (a load-store loop would expose one L2 round trip per
    // element per thread)
    {
      const uint32_t h0 = (uint32_t)__cvta_generic_to_shared(hyz);
      for (int i = t; i < np * Mu * 2 * N; i += GG::NT) {
        const int pq = i / (2 * N), r = i % (2 * N);
        const int pp = pc + pq / Mu, q = pq % Mu;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n"
                     :: "r"(h0 + 16u * (uint32_t)i),
                        "l"(a.hh + (((size_t)e * a.Nrho + pp) * Mu + q) * 3 * N + N + r)
                     : "memory");
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    for (int i = t; i < np * Mu; i += GG::NT) {
      const int pp = pc + i / Mu, q = i % Mu;
      const double2 h = a.hh[(((size_t)e * a.Nrho + pp) * Mu + q) * 3 * N + lx];
      const double m = (double)a.mult[q];
      hxs[i] = make_double2(m * h.x, m * h.y);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // fold hx (with m_q) into the y table once per (p, q, ly): hxy = hx hy
    for (int i = t; i < np * Mu * N; i += GG::NT) {
      const int pq = i / N, ly = i % N;
      double2* y = hyz + (size_t)pq * 2 * N + ly;
      *y = cmul(hxs[pq], *y);
    }
    __syncthreads();
    for (int j = 0; j < np; ++j) {
      const int p = pc + j;
      double wn[GG::KY];
#pragma unroll
      for (int k = 0; k < GG::KY; ++k) {
        const int ly = ly0 + GG::NYB * k;
        wn[k] = (p + 1 < a.Nrho && ly < N)
                    ? b1[(size_t)(p + 1) * N * nn + (size_t)ly * N] : 0.0;
      }
      double2 acc[GG::KY];
#pragma unroll
      for (int k = 0; k < GG::KY; ++k) acc[k] = make_double2(0, 0);
      const double2* hj = hyz + (size_t)j * Mu * 2 * N;
      for (int q = 0; q < Mu; ++q) {
        const double2 hz = hj[q * 2 * N + N + lz];
#pragma unroll
        for (int k = 0; k < GG::KY; ++k) {
          const int ly = min(ly0 + GG::NYB * k, N - 1);
          const double2 hxy = hj[q * 2 * N + ly];
          acc[k].x += hxy.x * hz.x - hxy.y * hz.y;
          acc[k].y += hxy.x * hz.y + hxy.y * hz.x;
        }
      }
#pragma unroll
      for (int k = 0; k < GG::KY; ++k) {
        Gs[k].x += wk[k] * acc[k].x;
        Gs[k].y += wk[k] * acc[k].y;
        wk[k] = wn[k];
      }
    }
  }
  double2* out = a.GM + (size_t)e * N * nn + (size_t)lx * nn + lz;
#pragma unroll
  for (int k = 0; k < GG::KY; ++k) {
    const int ly = ly0 + GG::NYB * k;
    if (ly < N) out[(size_t)ly * N] = Gs[k];
  }
}

// ---------------------------------------------------------------------------
// Terms: one cluster per (eval, p).  Precision R; SPLIT selects the
// Maxwellian-split combine.  FP32 keeps the running S_p in registers and the
// F slab resident in shared memory; FP64 keeps S_p in shared memory and
// streams F rows from global memory.
// ---------------------------------------------------------------------------
template <typename R, int N, int C, bool SPLIT>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
vhs_terms_kernel(VhsTermsArgs a) {
  using G = Geo<N, C>;
  using T = c2_t<R>;
  constexpr bool S_REG = (sizeof(R) == 4);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Rb = A + G::SLAB;
  T* F = Rb + G::SLAB;              // S_REG: resident F slab; else S slab
  T* tab = F + G::SLAB;             // [3][N] phase + [6][N] u,v
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int p = blockIdx.y, e = blockIdx.z;
  const T* Fg = static_cast<const T*>(a.Fg) + (size_t)e * G::n;
  const T* ph = static_cast<const T*>(a.ph);
  const T* uvg = static_cast<const T*>(a.uv);

  T S[S_REG ? N : 1];
  if constexpr (S_REG) {
#pragma unroll
    for (int x = 0; x < N; ++x) S[x] = T{0, 0};
    for (int j = t; j < G::P * N * N; j += G::NT)
      F[slab_index<N, C>(j)] = Fg[(size_t)rank * G::P * N * N + j];
  } else {
    const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
    for (int x = 0; x < N; ++x) F[base + x * G::ROW] = T{0, 0};
  }

  const int yl = t / N, zz = t % N, yy = rank * G::P + yl;
  bool first = true;
  for (int q = 0; q < a.Mu; ++q) {
    __syncthreads();  // previous term's table readers are done
    for (int i = t; i < 3 * N; i += G::NT)
      tab[i] = ph[((size_t)p * a.Mu + q) * 3 * N + i];
    if constexpr (SPLIT) {
      for (int i = t; i < 6 * N; i += G::NT)
        tab[3 * N + i] =
            uvg[((((size_t)e * a.Nrho) + p) * a.Mu + q) * 6 * N + i];
    }
    __syncthreads();
    const R mq = (R)a.mult[q];
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      // z-pass: multiplier cos/sin of a(l), inverse FFT along z
      {
        const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
        const T bxy = cmul(tab[lx], tab[N + ly]);
        T v[N];
        if constexpr (S_REG) {
          const int base = pl * G::PLANE + ly * G::ROW;
#pragma unroll
          for (int k = 0; k < N; ++k) v[k] = F[base + k];
        } else {
          const T* row = Fg + ((size_t)lx * N + ly) * N;
#pragma unroll
          for (int k = 0; k < N; ++k) v[k] = row[k];
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const T ph3 = cmul(bxy, tab[2 * N + k]);
          const R m = s == 0 ? ph3.x : ph3.y;
          v[k].x *= m;
          v[k].y *= m;
        }
        fft<R, N, +1>(v);
        const int base = pl * G::PLANE + ly * G::ROW;
#pragma unroll
        for (int k = 0; k < N; ++k) A[base + k] = v[k];
      }
      __syncthreads();
      {
        T v[N];
        slab_col_load_fft<R, N, C, +1>(A, t, v);
        if (!first) cluster_wait();  // receive buffers are free
        push_cols_to_yslab<R, N, C>(Rb, t, rank, v);
      }
      first = false;
      cluster_arrive();
      cluster_wait();
      T v[N];
      yslab_load_pencil<R, N, C>(Rb, t, v);
      cluster_arrive();  // done reading the receive buffer
      fft<R, N, +1>(v);
      T sv[N];
      if constexpr (!S_REG) {
        const int base = yl * G::PLANE + zz;
#pragma unroll
        for (int x = 0; x < N; ++x) sv[x] = F[base + x * G::ROW];
      }
      if constexpr (SPLIT) {
        const T* ut = tab + 3 * N;
        const T* vt = tab + 6 * N;
        const T uyz = cmul(ut[N + yy], ut[2 * N + zz]);
        const T vyz = cmul(vt[N + yy], vt[2 * N + zz]);
#pragma unroll
        for (int x = 0; x < N; ++x) {
          const T um = cmul(ut[x], uyz), vm = cmul(vt[x], vyz);
          T XM;
          if (s == 0) { XM.x = R(0.5) * (um.x + vm.x); XM.y = R(0.5) * (um.y + vm.y); }
          else        { XM.x = R(0.5) * (um.y - vm.y); XM.y = R(-0.5) * (um.x - vm.x); }
          // h_rest = 2 XM X + X^2 = X (2 XM + X)
          T w; w.x = R(2) * XM.x + v[x].x; w.y = R(2) * XM.y + v[x].y;
          const T h = cmul(v[x], w);
          if constexpr (S_REG) { S[x].x += mq * h.x; S[x].y += mq * h.y; }
          else { sv[x].x += mq * h.x; sv[x].y += mq * h.y; }
        }
      } else {
#pragma unroll
        for (int x = 0; x < N; ++x) {
          const T h = cmul(v[x], v[x]);
          if constexpr (S_REG) { S[x].x += mq * h.x; S[x].y += mq * h.y; }
          else { sv[x].x += mq * h.x; sv[x].y += mq * h.y; }
        }
      }
      if constexpr (!S_REG) {
        const int base = yl * G::PLANE + zz;
#pragma unroll
        for (int x = 0; x < N; ++x) F[base + x * G::ROW] = sv[x];
      }
    }
  }

  // forward FFT of S_p: x-pass, exchange into X-slabs, y-pass, z-pass
  T v[N];
  if constexpr (S_REG) {
#pragma unroll
    for (int x = 0; x < N; ++x) v[x] = S[x];
  } else {
    const int base = yl * G::PLANE + zz;
#pragma unroll
    for (int x = 0; x < N; ++x) v[x] = F[base + x * G::ROW];
  }
  fft<R, N, -1>(v);
  if (!first) cluster_wait();
  push_pencils_to_xslab<R, N, C>(A, t, rank, v);
  cluster_arrive();
  cluster_wait();
  {
    T w[N];
    slab_col_load_fft<R, N, C, -1>(A, t, w);
    const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
    for (int k = 0; k < N; ++k) A[base + k * G::ROW] = w[k];
  }
  __syncthreads();
  slab_row_pass<R, N, C, -1>(A, t);
  __syncthreads();
  const R* b1w = static_cast<const R*>(a.b1w) + (size_t)p * G::n +
                 (size_t)rank * G::P * N * N;
  T* H = static_cast<T*>(a.H) + ((size_t)e * a.Nrho + p) * G::n +
         (size_t)rank * G::P * N * N;
  for (int j = t; j < G::P * N * N; j += G::NT) {
    T hv = A[slab_index<N, C>(j)];
    const R w = b1w[j];
    hv.x *= w;
    hv.y *= w;
    H[j] = hv;
  }
}

// ---------------------------------------------------------------------------
// FP64 terms for grids whose three FP64 slabs do not fit in shared memory
// (N = 48: 16-CTA clusters of three planes; the transform slab A and the
// receive slab take 225.8 KB of the 227 KB).  Same algorithm as
// vhs_terms_kernel<double, N, C, false>, but each thread's running sum
// S_p(x, y, z) over the sphere directions lives in global memory at
// Sg[x * NT + t] (coalesced across the CTA) inside this CTA's own block of H,
// which the CTA reads back once before the final transform and overwrites
// with the output only after the cluster barrier that follows.
// ---------------------------------------------------------------------------
template <int N, int C>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
vhs_terms_fp64g_kernel(VhsTermsArgs a) {
  using G = Geo<N, C>;
  using R = double;
  using T = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Rb = A + G::SLAB;
  T* tab = Rb + G::SLAB;            // [3][N] phase
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int p = blockIdx.y, e = blockIdx.z;
  const T* Fg = static_cast<const T*>(a.Fg) + (size_t)e * G::n;
  const T* ph = static_cast<const T*>(a.ph);
  T* H = static_cast<T*>(a.H) + ((size_t)e * a.Nrho + p) * G::n +
         (size_t)rank * G::P * N * N;
  T* Sg = H;                        // running sums, then the output block
  for (int x = 0; x < N; ++x) Sg[(size_t)x * G::NT + t] = T{0, 0};

  bool first = true;
  for (int q = 0; q < a.Mu; ++q) {
    __syncthreads();  // previous term's table readers are done
    for (int i = t; i < 3 * N; i += G::NT)
      tab[i] = ph[((size_t)p * a.Mu + q) * 3 * N + i];
    __syncthreads();
    const R mq = a.mult[q];
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      // z-pass: multiplier cos/sin of a(l), inverse FFT along z
      {
        const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
        const T bxy = cmul(tab[lx], tab[N + ly]);
        T v[N];
        const T* row = Fg + ((size_t)lx * N + ly) * N;
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = row[k];
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const T ph3 = cmul(bxy, tab[2 * N + k]);
          const R m = s == 0 ? ph3.x : ph3.y;
          v[k].x *= m;
          v[k].y *= m;
        }
        fft<R, N, +1>(v);
        const int base = pl * G::PLANE + ly * G::ROW;
#pragma unroll
        for (int k = 0; k < N; ++k) A[base + k] = v[k];
      }
      __syncthreads();
      {
        T v[N];
        slab_col_load_fft<R, N, C, +1>(A, t, v);
        if (!first) cluster_wait();  // receive buffers are free
        push_cols_to_yslab<R, N, C>(Rb, t, rank, v);
      }
      first = false;
      cluster_arrive();
      cluster_wait();
      T v[N];
      yslab_load_pencil<R, N, C>(Rb, t, v);
      cluster_arrive();  // done reading the receive buffer
      fft<R, N, +1>(v);
#pragma unroll
      for (int x = 0; x < N; ++x) {
        const T h = cmul(v[x], v[x]);
        T sv = Sg[(size_t)x * G::NT + t];
        sv.x += mq * h.x;
        sv.y += mq * h.y;
        Sg[(size_t)x * G::NT + t] = sv;
      }
    }
  }

  // forward FFT of S_p: x-pass, exchange into X-slabs, y-pass, z-pass
  T v[N];
#pragma unroll
  for (int x = 0; x < N; ++x) v[x] = Sg[(size_t)x * G::NT + t];
  fft<R, N, -1>(v);
  if (!first) cluster_wait();
  push_pencils_to_xslab<R, N, C>(A, t, rank, v);
  cluster_arrive();
  cluster_wait();
  {
    T w[N];
    slab_col_load_fft<R, N, C, -1>(A, t, w);
    const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
    for (int k = 0; k < N; ++k) A[base + k * G::ROW] = w[k];
  }
  __syncthreads();
  slab_row_pass<R, N, C, -1>(A, t);
  __syncthreads();
  const R* b1w = static_cast<const R*>(a.b1w) + (size_t)p * G::n +
                 (size_t)rank * G::P * N * N;
  for (int j = t; j < G::P * N * N; j += G::NT) {
    T hv = A[slab_index<N, C>(j)];
    const R w = b1w[j];
    hv.x *= w;
    hv.y *= w;
    H[j] = hv;
  }
}

// ---------------------------------------------------------------------------
// Terms, FP32 Maxwellian-split path with packed real transforms.
//
// g = f - M is real, so F_g is Hermitian.  With the phase a(l) = kappa.l the
// reference forms t3 = IFFT(cos a F_g) and t4 = IFFT(sin a F_g); off the
// Nyquist planes (any l_a = -N/2) cos a F_g is Hermitian and sin a F_g
// anti-Hermitian, so t3 = C and t4 = i s with C, s real, and ONE complex
// inverse transform z = IFFT((cos a + sin a) F_g) = C + i s yields both.
// On the Nyquist planes the mirror l' of l is not -l, and each product splits
// exactly into a Hermitian and an anti-Hermitian part.  With
// a(l') = -a(l) - theta_S(l), theta_S = N sum_{a in S} kappa_a over the set S
// of Nyquist axes of l, f_S = exp(i theta_S) and E = exp(i a):
//   main  multiplier m  = Re(E (1 + f_S)(1 - i)/2)  -> z  = C + i s
//   plane multiplier mc = Re(E (1 - f_S)(1 - i)/2)  -> zc = s_R + i c_I
// so that t3 = C + i c_I and t4 = i s + s_R exactly.  mc vanishes off the
// Nyquist planes, so zc is a sum of three plane-extruded 2-D transforms
//   zc(x,y,z) = (-1)^x rx(y,z) + (-1)^y ry(x,z) + (-1)^z rz(x,y)
// (vhs_nyq_planes_kernel).  With the Maxwellian parts t3_M = (u_M + v_M)/2,
// t4_M = (u_M - v_M)/(2i) (u_M, v_M: separable products of the FP64 1-D
// tables), the g-dependent real part of t3^2 + t4^2 is
//   C (A.x + C) + s (B.x - s) + s_R (B.y + s_R) - c_I (A.y + c_I),
//   A = u_M + v_M, B = u_M - v_M
// (only Re of the gain survives: b1 is real and even, and the epilogue takes
// the real part of the final inverse transform).
//
// Two radial points p0, p1 share one cluster: their real sums S_p0, S_p1 are
// packed as S = S_p0 + i S_p1 and forward-transformed together; since both
// spectra are Hermitian, Re IFFT((b1_p0 - i b1_p1) FFT(S)) =
// IFFT(b1_p0 FFT(S_p0) + b1_p1 FFT(S_p1)), so the epilogue sums the packed
// spectra H = (b1_p0 - i b1_p1) FFT(S) unchanged.
//
// Pipeline per transform k (term (p, q) = (p0 + k / Mu, k % Mu)):
//   y-pass(k) -> exchange(k) into receive buffer k%2 -> arrive
//   -> [load F_g slab, z-pass(k+1)]  (overlaps the exchange latency)
//   -> wait -> x-pass(k) + combine into S
// Two receive buffers make one cluster barrier per transform sufficient: a
// CTA stores into buffer k%2 of a peer only after the barrier of transform
// k-1, which that peer joined after reading its buffer k%2 for transform k-2.
// The multiplicity m_q is folded into the tables as sqrt(m_q) (on the x-phase
// and on u_x, v_x), and so into zc.
// ---------------------------------------------------------------------------
// Asynchronous copy of this CTA's F_g slab (global, dense) into the padded
// X-slab A: 8-byte cp.async per complex element, one commit group.
template <int N, int C>
__device__ __forceinline__ void fp32_issue_slab_copy(float2* A,
                                                     const float2* Fg, int t) {
  using G = Geo<N, C>;
  const uint32_t a0 = smem_u32(A);
  constexpr int TOT = G::P * N * N;
#pragma unroll 4
  for (int j = t; j < TOT; j += G::NT) {
    const uint32_t dst = a0 + (uint32_t)slab_index<N, C>(j) * 8u;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
                 :: "r"(dst), "l"(Fg + j) : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n"
               :: "r"(dst), "l"(src) : "memory");
}

// (1 + f)(1 - i)/2 and (1 - f)(1 - i)/2
__device__ __forceinline__ float2 nyq_main(float2 f) {
  const float ux = 1.f + f.x, uy = f.y;
  return make_float2(0.5f * (ux + uy), 0.5f * (uy - ux));
}
__device__ __forceinline__ float2 nyq_plane(float2 f) {
  const float ux = 1.f - f.x, uy = -f.y;
  return make_float2(0.5f * (ux + uy), 0.5f * (uy - ux));
}

// z-pass of the packed transform: multiply this thread's z-pencil
// (lx, ly) by m(l) and inverse-transform it along z.
// tb: [ph x,y,z (3N) | u (3N) | v (3N) | nu x,y,z (3)]
template <int N, int C, int ROW = N + 1>
__device__ __forceinline__ void fp32_zpass(float2* A, const float2* tb, int t,
                                           unsigned rank) {
  using G = Geo<N, C>;
  constexpr int PLANE = N * ROW;
  const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
  const float2 bxy = cmul(tb[lx], tb[N + ly]);
  const float2* nu = tb + 9 * N;
  float2 fxy = make_float2(1.f, 0.f);
  if (lx == N / 2) fxy = nu[0];
  if (ly == N / 2) fxy = cmul(fxy, nu[1]);
  const float2 gb = cmul(nyq_main(fxy), bxy);
  const float2 gbz = cmul(nyq_main(cmul(fxy, nu[2])), bxy);
  const int base = pl * PLANE + ly * ROW;
  float2 v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    const float2 bz = tb[2 * N + k];
    const float2 g = (k == N / 2) ? gbz : gb;
    const float m = g.x * bz.x - g.y * bz.y;
    const float2 f = A[base + k];
    v[k] = make_float2(f.x * m, f.y * m);
  }
  fft<float, N, +1>(v);
#pragma unroll
  for (int k = 0; k < N; ++k) A[base + k] = v[k];
}

// Plane transforms rx, ry, rz of two directions q of one (eval e, radial p).
// grid (ceil(Mu/2), Nrho, nevals), block 6N: thread t = half*3N + plane*N +
// row.  The three Nyquist planes of F_g (written compactly by the prologue)
// are staged in shared memory with coalesced loads.
template <int N>
__global__ void __launch_bounds__(6 * N)
vhs_nyq_planes_kernel(VhsTermsArgs a) {
  constexpr int ROW = N + 1, H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* Fp = reinterpret_cast<float2*>(smem_raw);  // [3][N][ROW]
  float2* pl = Fp + 3 * N * ROW;                      // [2][3][N][ROW]
  float2* tph = pl + 2 * 3 * N * ROW;                 // [2][3N + 3]
  const int q0 = 2 * blockIdx.x, p = blockIdx.y, e = blockIdx.z;
  const int t = threadIdx.x, half = t / (3 * N), tt = t % (3 * N);
  const int P = tt / N, i = tt % N;
  const int Mu = a.Mu;
  const float2* Fny = static_cast<const float2*>(a.Fny) + (size_t)e * 3 * N * N;
#pragma unroll 4
  for (int j = t; j < 3 * N * N; j += 6 * N)
    Fp[(j / N) * ROW + j % N] = Fny[j];
  for (int j = t; j < 2 * (3 * N + 3); j += 6 * N) {
    const int hq = j / (3 * N + 3), r = j % (3 * N + 3), q = q0 + hq;
    if (q < Mu) {
      const size_t pq = (size_t)p * Mu + q;
      tph[j] = r < 3 * N ? static_cast<const float2*>(a.ph)[pq * 3 * N + r]
                         : static_cast<const float2*>(a.nyq)[pq * 3 + r - 3 * N];
    }
  }
  __syncthreads();
  const int q = q0 + half;
  float2* pl_h = pl + half * 3 * N * ROW;
  const float2* tb = tph + half * (3 * N + 3);
  float2 v[N];
  if (q < Mu) {
    const float2 nx = tb[3 * N], ny = tb[3 * N + 1], nz = tb[3 * N + 2];
    // rows: P=0 (lx=H, ly=i, lz=k); P=1 (lx=i, ly=H, lz=k), lx=H excluded;
    //       P=2 (lx=i, ly=k, lz=H), lx=H and ly=H excluded.
    // E = rowc * tk[k]; f = f_row off k=H, f_rowH at k=H.
    float2 rowc, f_row, f_rowH;
    const float2* tk;
    if (P == 0) {
      rowc = cmul(tb[H], tb[N + i]);
      f_row = (i == H) ? cmul(nx, ny) : nx;
      f_rowH = cmul(f_row, nz);
      tk = tb + 2 * N;
    } else if (P == 1) {
      rowc = cmul(tb[i], tb[N + H]);
      f_row = ny;
      f_rowH = cmul(ny, nz);
      tk = tb + 2 * N;
    } else {
      rowc = cmul(tb[i], tb[2 * N + H]);
      f_row = nz;
      f_rowH = nz;
      tk = tb + N;
    }
    if (P >= 1 && i == H) rowc = make_float2(0.f, 0.f);
    const float2 g = cmul(nyq_plane(f_row), rowc);
    const float2 gH = (P == 2) ? make_float2(0.f, 0.f)
                               : cmul(nyq_plane(f_rowH), rowc);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const float2 gk = (k == H) ? gH : g;
      const float2 b = tk[k];
      const float m = gk.x * b.x - gk.y * b.y;
      const float2 F = Fp[(P * N + i) * ROW + k];
      v[k] = make_float2(F.x * m, F.y * m);
    }
    fft<float, N, +1>(v);
#pragma unroll
    for (int k = 0; k < N; ++k) pl_h[(P * N + i) * ROW + k] = v[k];
  }
  __syncthreads();
  if (q < Mu) {
    // columns: transform pl[P][.][i] along the rows
#pragma unroll
    for (int r = 0; r < N; ++r) v[r] = pl_h[(P * N + r) * ROW + i];
    fft<float, N, +1>(v);
    float2* rho = static_cast<float2*>(a.rho) +
                  ((((size_t)e * a.Nrho + p) * Mu + q) * 3 + P) * N * N;
#pragma unroll
    for (int r = 0; r < N; ++r) rho[(size_t)r * N + i] = v[r];
  }
}

// Whether the terms kernel stages r_y (N*N complex) in shared memory.  With
// 8 or more CTAs per cluster it reads r_y through L1 instead, which leaves
// room for two CTAs per SM.
template <int C> struct TermsRyStaged { static constexpr bool value = C < 8; };

// Stage this CTA's share of the plane transforms of one term into smem:
// rY = ry[x][z] (all; only if staged), rX = rx[y][z] (own y),
// rZ = rz[x][y] (own y) as [x][yl].
template <int N, int C>
__device__ __forceinline__ void fp32_issue_rho_copy(float2* rbuf,
                                                    const float2* rho, int t,
                                                    unsigned rank) {
  using G = Geo<N, C>;
  constexpr int P = G::P;
  constexpr bool RYS = TermsRyStaged<C>::value;
  const uint32_t s0 = smem_u32(rbuf);
  // ry: N*N complex = N*N/2 chunks of 16 B
  if (RYS)
    for (int c = t; c < N * N / 2; c += G::NT)
      cp_async16(s0 + 16u * c, rho + N * N + 2 * c);
  // rx rows y in [rank P, rank P + P): P*N complex
  const uint32_t sx = s0 + (RYS ? 8u * N * N : 0u);
  const float2* rx = rho + (size_t)rank * P * N;
  for (int c = t; c < P * N / 2; c += G::NT) cp_async16(sx + 16u * c, rx + 2 * c);
  // rz[x][rank P .. rank P + P): N segments of P complex, copied element by
  // element (8 bytes) because P may be odd (N=48 with 16 planes: P=3), which
  // leaves the segments only 8-byte aligned
  const uint32_t szz = sx + 8u * P * N;
  const float2* rz = rho + 2 * N * N + rank * P;
  for (int c = t; c < N * P; c += G::NT) {
    const int x = c / P, j = c % P;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
                 :: "r"(szz + 8u * c), "l"(rz + (size_t)x * N + j) : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// TMA selects how the F_g slab (once per transform) and the staged plane
// transforms of a term reach shared memory:
//   false: 8-byte cp.async per element into rows padded to N+1 elements;
//   true:  one tiled TMA load of the CTA's P x N x (N+2) box of F_g (the two
//          elements past the end of each row lie outside the tensor and are
//          filled with zeros, which gives padded rows whose starts are
//          16-byte aligned), and 1-D bulk copies of r_y and r_x, all
//          completing on one mbarrier (bounded wait, error flag a.err); r_z
//          (P-element pieces) stays on cp.async.  Rows of N+2 elements give
//          the z-pass two-way bank conflicts, which N+1 avoids.
template <int N, int C, bool TMA = false>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
vhs_terms_fp32_kernel(VhsTermsArgs a, const __grid_constant__ CUtensorMap tmap) {
  using G = Geo<N, C>;
  using T = float2;
  constexpr int TB = 9 * N + 4;  // ring slot: ph | u | v | nu (+1 pad)
  constexpr int RA = TMA ? N + 2 : G::ROW;   // row pitch of the A slab
  constexpr int PA = N * RA;                 // its plane pitch
  constexpr int SA = G::P * PA;              // its size
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA writes need a 128-byte aligned destination: the launch adds 128
  // bytes of slack and A starts at the next 128-byte boundary
  T* A = reinterpret_cast<T*>(
      TMA ? smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u) : smem_raw);
  T* R0 = A + SA;               // receive buffer b at R0 + b*SLAB
  T* tab = R0 + 2 * G::SLAB;    // [2][TB]
  constexpr bool RYS = TermsRyStaged<C>::value;
  T* rbuf = tab + 2 * TB;       // (ry [N*N]) | rx [P*N] | rz [N*P]
  const T* rX = rbuf + (RYS ? N * N : 0);
  const T* rZ = rX + G::P * N;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(rbuf + (RYS ? N * N : 0) +
                                               2 * G::P * N);
  static_assert(((N + 2) * 8) % 16 == 0, "TMA rows must be 16-byte multiples");
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int pair = blockIdx.y, e = blockIdx.z;
  const int Mu = a.Mu;
  const int p0 = 2 * pair;
  const int npass = (p0 + 1 < a.Nrho ? 2 : 1) * Mu;
  const T* Fg = static_cast<const T*>(a.Fg) + (size_t)e * G::n +
                (size_t)rank * G::P * N * N;
  const T* phb = static_cast<const T*>(a.ph);
  const T* uvb = static_cast<const T*>(a.uv);
  const T* nyb = static_cast<const T*>(a.nyq);
  const T* rhob = static_cast<const T*>(a.rho);
  // term k -> (p, q) = (p0 + k / Mu, k % Mu); tables index p*Mu + q
  auto term = [&](int k) { return (p0 + k / Mu) * Mu + k % Mu; };
  auto load_tables = [&](int k) {
    T* dst = tab + (k & 1) * TB;
    const int pq = term(k);
    const T* ph = phb + (size_t)pq * 3 * N;
    const T* uv = uvb + ((size_t)e * a.Nrho * Mu + pq) * 6 * N;
    for (int i = t; i < 3 * N; i += G::NT) dst[i] = ph[i];
    for (int i = t; i < 6 * N; i += G::NT) dst[3 * N + i] = uv[i];
    if (t < 3) dst[9 * N + t] = nyb[(size_t)pq * 3 + t];
  };
  // TMA: thread 0 issues the copies of one stage (the slab of the next
  // transform if `slab`, the r_y and r_x of term k if k >= 0) on mbar;
  // every thread then waits for phase `ph` (bounded) before using them
  constexpr uint32_t SLAB_BYTES = (uint32_t)(G::P * N * (N + 2) * sizeof(T));
  constexpr uint32_t RY_BYTES = RYS ? (uint32_t)(N * N * sizeof(T)) : 0u;
  constexpr uint32_t RX_BYTES = (uint32_t)(G::P * N * sizeof(T));
  uint32_t tphase = 0;
  bool tma_ok = true;
  auto tma_issue = [&](bool slab, int k) {
    if (t != 0) return;
    const uint32_t mb = smem_u32(mbar);
    const uint32_t bytes = (slab ? SLAB_BYTES : 0u) + (k >= 0 ? RY_BYTES + RX_BYTES : 0u);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
                 :: "r"(mb), "r"(bytes) : "memory");
    if (slab)
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
          :: "r"(smem_u32(A)), "l"(&tmap), "r"(0), "r"(0), "r"((int)(rank * G::P)),
             "r"(e), "r"(mb) : "memory");
    if (k >= 0) {
      const T* rho = rhob + ((size_t)e * a.Nrho * Mu + term(k)) * 3 * N * N;
      if (RYS)
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
            " [%0], [%1], %2, [%3];\n"
            :: "r"(smem_u32(rbuf)), "l"(rho + N * N), "r"(RY_BYTES), "r"(mb)
            : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
          " [%0], [%1], %2, [%3];\n"
          :: "r"(smem_u32(rbuf + (RYS ? N * N : 0))),
             "l"(rho + (size_t)rank * G::P * N), "r"(RX_BYTES), "r"(mb)
          : "memory");
    }
  };
  auto tma_wait = [&]() {
    const uint32_t mb = smem_u32(mbar);
    uint32_t done = 0;
    uint64_t t0 = 0;
    for (int it = 0; !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t}\n"
          : "=r"(done) : "r"(mb), "r"(tphase) : "memory");
      if (done) break;
      if (it == 0) t0 = global_ns();
      else if (global_ns() - t0 > 200000000ull) { tma_ok = false; break; }
    }
    tphase ^= 1u;
  };
  // r_z pieces (P elements per x) by 8-byte cp.async, one commit group
  auto issue_rz = [&](int k) {
    const uint32_t szz = smem_u32(rbuf + (RYS ? N * N : 0) + G::P * N);
    const T* rz = rhob + ((size_t)e * a.Nrho * Mu + term(k)) * 3 * N * N +
                  2 * N * N + rank * G::P;
    for (int c = t; c < N * G::P; c += G::NT) {
      const int x = c / G::P, j = c % G::P;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
                   :: "r"(szz + 8u * c), "l"(rz + (size_t)x * N + j) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  auto rho_of = [&](int k) {
    return rhob + ((size_t)e * a.Nrho * Mu + term(k)) * 3 * N * N;
  };
  load_tables(0);
  uint32_t rbase[C];
#pragma unroll
  for (int c = 0; c < C; ++c) rbase[c] = mapa_u32(smem_u32(R0), (uint32_t)c);

  const int yl = t / N, zz = t % N, yy = rank * G::P + yl;
  const float sy = (yy & 1) ? -1.f : 1.f, sz = (zz & 1) ? -1.f : 1.f;
  T S[N];
#pragma unroll
  for (int x = 0; x < N; ++x) S[x] = make_float2(0.f, 0.f);

  if constexpr (TMA) {
    if (t == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n"
                   :: "r"(smem_u32(mbar)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    tma_issue(true, -1);
    tma_wait();
    __syncthreads();
  } else {
    fp32_issue_slab_copy<N, C>(A, Fg, t);
    cp_async_wait_all();
    __syncthreads();
  }
  fp32_zpass<N, C, RA>(A, tab, t, rank);
  __syncthreads();
#pragma unroll 1
  for (int k = 0; k < npass; ++k) {
    T v[N];
    {
      const int base = (t / N) * PA + (t % N);
#pragma unroll
      for (int y = 0; y < N; ++y) v[y] = A[base + y * RA];
    }
    __syncthreads();  // every thread has read A and used rbuf: refill both
    if constexpr (TMA) {
      tma_issue(k + 1 < npass, k);
      issue_rz(k);
      if (k + 1 < npass) load_tables(k + 1);
    } else {
      fp32_issue_rho_copy<N, C>(rbuf, rho_of(k), t, rank);
      if (k + 1 < npass) {
        load_tables(k + 1);
        fp32_issue_slab_copy<N, C>(A, Fg, t);
      }
    }
    fft<float, N, +1>(v);
    {
      const int lx = rank * G::P + t / N, z = t % N;
      const uint32_t off = (uint32_t)((k & 1) * G::SLAB + lx * G::ROW + z) * 8u;
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int j = 0; j < G::P; ++j)
          st_cluster(rbase[c] + off + (uint32_t)(j * G::PLANE) * 8u,
                     v[c * G::P + j]);
    }
    cluster_arrive();
    cp_async_wait_all();
    if constexpr (TMA) tma_wait();
    __syncthreads();
    if (k + 1 < npass) {
      fp32_zpass<N, C, RA>(A, tab + ((k + 1) & 1) * TB, t, rank);
      __syncthreads();
    }
    cluster_wait();
    {
      const T* Rk = R0 + (k & 1) * G::SLAB;
      const int base = yl * G::PLANE + zz;
#pragma unroll
      for (int x = 0; x < N; ++x) v[x] = Rk[base + x * G::ROW];
    }
    fft<float, N, +1>(v);
    const T* tb = tab + (k & 1) * TB;
    const T* ut = tb + 3 * N;
    const T* vt = tb + 6 * N;
    const T uyz = cmul(ut[N + yy], ut[2 * N + zz]);
    const T vyz = cmul(vt[N + yy], vt[2 * N + zz]);
    const T rx = rX[yl * N + zz];
    const T* rY = RYS ? rbuf : rho_of(k) + N * N;
    const bool hi = k >= Mu;
#pragma unroll
    for (int x = 0; x < N; ++x) {
      const T um = cmul(ut[x], uyz), vm = cmul(vt[x], vyz);
      const float Ax = um.x + vm.x, Ay = um.y + vm.y;
      const float Bx = um.x - vm.x, By = um.y - vm.y;
      const T ry = rY[x * N + zz], rz = rZ[x * G::P + yl];
      const float xs = (x & 1) ? -1.f : 1.f;
      const float sR = xs * rx.x + sy * ry.x + sz * rz.x;
      const float cI = xs * rx.y + sy * ry.y + sz * rz.y;
      const float Cm = v[x].x, sm = v[x].y;
      const float h = Cm * (Ax + Cm) + sm * (Bx - sm) + sR * (By + sR) -
                      cI * (Ay + cI);
      if (hi) S[x].y += h;
      else S[x].x += h;
    }
  }

  // forward FFT of S = S_p0 + i S_p1: x-pass, exchange into X-slabs,
  // y-pass, z-pass
  fft<float, N, -1>(S);
  {
    const uint32_t a0 = smem_u32(A);
    const uint32_t off = (uint32_t)(yy * RA + zz) * 8u;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const uint32_t ab = mapa_u32(a0, (uint32_t)c) + off;
#pragma unroll
      for (int j = 0; j < G::P; ++j)
        st_cluster(ab + (uint32_t)(j * PA) * 8u, S[c * G::P + j]);
    }
  }
  cluster_arrive();
  cluster_wait();
  {
    T w[N];
    const int base = (t / N) * PA + (t % N);
#pragma unroll
    for (int k = 0; k < N; ++k) w[k] = A[base + k * RA];
    fft<float, N, -1>(w);
#pragma unroll
    for (int k = 0; k < N; ++k) A[base + k * RA] = w[k];
  }
  __syncthreads();
  {
    T w[N];
    const int base = (t / N) * PA + (t % N) * RA;
#pragma unroll
    for (int k = 0; k < N; ++k) w[k] = A[base + k];
    fft<float, N, -1>(w);
#pragma unroll
    for (int k = 0; k < N; ++k) A[base + k] = w[k];
  }
  __syncthreads();
  const size_t off = (size_t)rank * G::P * N * N;
  const float* b1a = static_cast<const float*>(a.b1w) + (size_t)p0 * G::n + off;
  const float* b1b = (p0 + 1 < a.Nrho) ? b1a + G::n : nullptr;
  const int npairs = (a.Nrho + 1) / 2;
  T* H = static_cast<T*>(a.H) + ((size_t)e * npairs + pair) * G::n + off;
  if (TMA && !tma_ok && a.err && t == 0) atomicExch(a.err, 1);
  for (int j = t; j < G::P * N * N; j += G::NT) {
    const T hv = A[(j / (N * N)) * PA + ((j / N) % N) * RA + (j % N)];
    const float w0 = b1a[j], w1 = b1b ? b1b[j] : 0.f;
    H[j] = make_float2(hv.x * w0 + hv.y * w1, hv.y * w0 - hv.x * w1);
  }
}

// ---------------------------------------------------------------------------
// Split-pencil variant of the FP32 terms kernel: two threads (adjacent lanes
// h = 0, 1) share every pencil, each holding N/2 values, so a CTA runs twice
// the warps for the same shared memory (registers per thread roughly halve).
// An N-point transform is one radix-2 step across the pair (register
// exchange by shuffles) around N/2-point register transforms:
//   DIT (input samples 2m+h, output X[h N/2 + m]):  E/O transforms, then
//       X[k] = E[k] + W^k O[k], X[k + N/2] = E[k] - W^k O[k];
//   DIF (input x[h N/2 + m], output X[2m + h]):  a = x[m] + x[m + N/2],
//       b = (x[m] - x[m + N/2]) W^m, then the N/2-point transforms.
// Same algorithm, data layout and pipeline as vhs_terms_fp32_kernel.
// ---------------------------------------------------------------------------
template <int N, int SIGN>
__device__ __forceinline__ void fft_pair_dit(float2* v, int h) {
  constexpr int H = N / 2;
  fft<float, H, SIGN>(v);
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const float2 w = h ? twiddle_mul<float, N, SIGN>(v[k], k) : v[k];
    float2 o;
    o.x = __shfl_xor_sync(0xffffffffu, w.x, 1);
    o.y = __shfl_xor_sync(0xffffffffu, w.y, 1);
    // h = 0 holds E, receives W O;  h = 1 holds W O, receives E
    v[k] = h ? make_float2(o.x - w.x, o.y - w.y) : make_float2(w.x + o.x, w.y + o.y);
  }
}

template <int N, int SIGN>
__device__ __forceinline__ void fft_pair_dif(float2* v, int h) {
  constexpr int H = N / 2;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    float2 o;
    o.x = __shfl_xor_sync(0xffffffffu, v[k].x, 1);
    o.y = __shfl_xor_sync(0xffffffffu, v[k].y, 1);
    // h = 0 holds x[k], receives x[k + H];  h = 1 the reverse
    const float2 a = make_float2(v[k].x + o.x, v[k].y + o.y);
    const float2 b = make_float2(o.x - v[k].x, o.y - v[k].y);
    v[k] = h ? twiddle_mul<float, N, SIGN>(b, k) : a;
  }
  fft<float, H, SIGN>(v);
}

template <int N, int C>
struct GeoS {
  using G = Geo<N, C>;
  static constexpr int NT = 2 * G::NT;  // two threads per pencil
};

template <int N, int C>
__device__ __forceinline__ void fp32s_zpass(float2* A, const float2* tb, int pp,
                                            int h, unsigned rank) {
  using G = Geo<N, C>;
  constexpr int H = N / 2;
  const int pl = pp / N, ly = pp % N, lx = rank * G::P + pl;
  const float2 bxy = cmul(tb[lx], tb[N + ly]);
  const float2* nu = tb + 9 * N;
  float2 fxy = make_float2(1.f, 0.f);
  if (lx == N / 2) fxy = nu[0];
  if (ly == N / 2) fxy = cmul(fxy, nu[1]);
  const float2 gb = cmul(nyq_main(fxy), bxy);
  const float2 gbz = cmul(nyq_main(cmul(fxy, nu[2])), bxy);
  const int base = pl * G::PLANE + ly * G::ROW;
  float2 v[H];
#pragma unroll
  for (int m = 0; m < H; ++m) {
    const int k = 2 * m + h;
    const float2 bz = tb[2 * N + k];
    const float2 g = (k == N / 2) ? gbz : gb;
    const float mm = g.x * bz.x - g.y * bz.y;
    const float2 f = A[base + k];
    v[m] = make_float2(f.x * mm, f.y * mm);
  }
  fft_pair_dit<N, +1>(v, h);
#pragma unroll
  for (int m = 0; m < H; ++m) A[base + h * H + m] = v[m];
}

template <int N, int C>
__global__ void __launch_bounds__(GeoS<N, C>::NT,
                                  (512 / GeoS<N, C>::NT) > 0 ? 512 / GeoS<N, C>::NT : 1)
vhs_terms_fp32s_kernel(VhsTermsArgs a) {
  using G = Geo<N, C>;
  using T = float2;
  constexpr int H = N / 2;
  constexpr int NT = GeoS<N, C>::NT;
  constexpr int TB = 9 * N + 4;
  constexpr bool RYS = TermsRyStaged<C>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);
  T* R0 = A + G::SLAB;
  T* tab = R0 + 2 * G::SLAB;
  T* rbuf = tab + 2 * TB;
  const T* rX = rbuf + (RYS ? N * N : 0);
  const T* rZ = rX + G::P * N;
  const int t = threadIdx.x, pp = t >> 1, h = t & 1;
  const unsigned rank = cluster_rank();
  const int pair = blockIdx.y, e = blockIdx.z;
  const int Mu = a.Mu;
  const int p0 = 2 * pair;
  const int npass = (p0 + 1 < a.Nrho ? 2 : 1) * Mu;
  const T* Fg = static_cast<const T*>(a.Fg) + (size_t)e * G::n +
                (size_t)rank * G::P * N * N;
  const T* phb = static_cast<const T*>(a.ph);
  const T* uvb = static_cast<const T*>(a.uv);
  const T* nyb = static_cast<const T*>(a.nyq);
  const T* rhob = static_cast<const T*>(a.rho);
  auto term = [&](int k) { return (p0 + k / Mu) * Mu + k % Mu; };
  auto load_tables = [&](int k) {
    T* dst = tab + (k & 1) * TB;
    const int pq = term(k);
    const T* ph = phb + (size_t)pq * 3 * N;
    const T* uv = uvb + ((size_t)e * a.Nrho * Mu + pq) * 6 * N;
    for (int i = t; i < 3 * N; i += NT) dst[i] = ph[i];
    for (int i = t; i < 6 * N; i += NT) dst[3 * N + i] = uv[i];
    if (t < 3) dst[9 * N + t] = nyb[(size_t)pq * 3 + t];
  };
  auto rho_of = [&](int k) {
    return rhob + ((size_t)e * a.Nrho * Mu + term(k)) * 3 * N * N;
  };
  // the copy helpers stride by the one-thread-per-pencil count; thread
  // pairs split the work by running them on the even threads' indices
  auto slab_copy = [&]() {
    const uint32_t a0 = smem_u32(A);
    constexpr int TOT = G::P * N * N;
#pragma unroll 4
    for (int j = t; j < TOT; j += NT) {
      const uint32_t dst = a0 + (uint32_t)slab_index<N, C>(j) * 8u;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
                   :: "r"(dst), "l"(Fg + j) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  auto rho_copy = [&](const T* rho) {
    constexpr int P = G::P;
    const uint32_t s0 = smem_u32(rbuf);
    if (RYS)
      for (int c = t; c < N * N / 2; c += NT) cp_async16(s0 + 16u * c, rho + N * N + 2 * c);
    const uint32_t sx = s0 + (RYS ? 8u * N * N : 0u);
    const T* rx = rho + (size_t)rank * P * N;
    for (int c = t; c < P * N / 2; c += NT) cp_async16(sx + 16u * c, rx + 2 * c);
    const uint32_t szz = sx + 8u * P * N;
    const T* rz = rho + 2 * N * N + rank * P;
    for (int c = t; c < N * P; c += NT) {
      const int x = c / P, j = c % P;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n"
                   :: "r"(szz + 8u * c), "l"(rz + (size_t)x * N + j) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  load_tables(0);
  uint32_t rbase[C];
#pragma unroll
  for (int c = 0; c < C; ++c) rbase[c] = mapa_u32(smem_u32(R0), (uint32_t)c);

  const int yl = pp / N, zz = pp % N, yy = rank * G::P + yl;
  const float sy = (yy & 1) ? -1.f : 1.f, sz = (zz & 1) ? -1.f : 1.f;
  T S[H];   // x = h*H + m
#pragma unroll
  for (int m = 0; m < H; ++m) S[m] = make_float2(0.f, 0.f);

  slab_copy();
  cp_async_wait_all();
  __syncthreads();
  fp32s_zpass<N, C>(A, tab, pp, h, rank);
  __syncthreads();
#pragma unroll 1
  for (int k = 0; k < npass; ++k) {
    T v[H];
    {
      const int base = (pp / N) * G::PLANE + (pp % N);
#pragma unroll
      for (int m = 0; m < H; ++m) v[m] = A[base + (2 * m + h) * G::ROW];
    }
    __syncthreads();
    rho_copy(rho_of(k));
    if (k + 1 < npass) {
      load_tables(k + 1);
      slab_copy();
    }
    fft_pair_dit<N, +1>(v, h);
    {
      const int lx = rank * G::P + pp / N, z = pp % N;
      const uint32_t off = (uint32_t)((k & 1) * G::SLAB + lx * G::ROW + z) * 8u;
#pragma unroll
      for (int m = 0; m < H; ++m) {
        const int y = h * H + m, c = y / G::P, j = y % G::P;
        st_cluster(rbase[c] + off + (uint32_t)(j * G::PLANE) * 8u, v[m]);
      }
    }
    cluster_arrive();
    cp_async_wait_all();
    __syncthreads();
    if (k + 1 < npass) {
      fp32s_zpass<N, C>(A, tab + ((k + 1) & 1) * TB, pp, h, rank);
      __syncthreads();
    }
    cluster_wait();
    {
      const T* Rk = R0 + (k & 1) * G::SLAB;
      const int base = yl * G::PLANE + zz;
#pragma unroll
      for (int m = 0; m < H; ++m) v[m] = Rk[base + (2 * m + h) * G::ROW];
    }
    fft_pair_dit<N, +1>(v, h);
    const T* tb = tab + (k & 1) * TB;
    const T* ut = tb + 3 * N;
    const T* vt = tb + 6 * N;
    const T uyz = cmul(ut[N + yy], ut[2 * N + zz]);
    const T vyz = cmul(vt[N + yy], vt[2 * N + zz]);
    const T rx = rX[yl * N + zz];
    const T* rY = RYS ? rbuf : rho_of(k) + N * N;
    const bool hi = k >= Mu;
#pragma unroll
    for (int m = 0; m < H; ++m) {
      const int x = h * H + m;
      const T um = cmul(ut[x], uyz), vm = cmul(vt[x], vyz);
      const float Ax = um.x + vm.x, Ay = um.y + vm.y;
      const float Bx = um.x - vm.x, By = um.y - vm.y;
      const T ry = rY[x * N + zz], rz = rZ[x * G::P + yl];
      const float xs = (m & 1) ? -1.f : 1.f;   // (-1)^x, H even
      const float sR = xs * rx.x + sy * ry.x + sz * rz.x;
      const float cI = xs * rx.y + sy * ry.y + sz * rz.y;
      const float Cm = v[m].x, sm = v[m].y;
      const float hh = Cm * (Ax + Cm) + sm * (Bx - sm) + sR * (By + sR) -
                       cI * (Ay + cI);
      if (hi) S[m].y += hh;
      else S[m].x += hh;
    }
  }

  // forward FFT of S = S_p0 + i S_p1: x pass (DIF: outputs lx = 2m + h),
  // exchange into X-slabs, y pass, z pass
  fft_pair_dif<N, -1>(S, h);
  {
    const uint32_t a0 = smem_u32(A);
    const uint32_t off = (uint32_t)(yy * G::ROW + zz) * 8u;
#pragma unroll
    for (int m = 0; m < H; ++m) {
      const int lx = 2 * m + h, c = lx / G::P, j = lx % G::P;
      st_cluster(mapa_u32(a0, (uint32_t)c) + off + (uint32_t)(j * G::PLANE) * 8u, S[m]);
    }
  }
  cluster_arrive();
  cluster_wait();
  {
    T w[H];
    const int base = (pp / N) * G::PLANE + (pp % N);
#pragma unroll
    for (int m = 0; m < H; ++m) w[m] = A[base + (2 * m + h) * G::ROW];
    fft_pair_dit<N, -1>(w, h);
    __syncthreads();   // all column reads done before the in-place writes
#pragma unroll
    for (int m = 0; m < H; ++m) A[base + (h * H + m) * G::ROW] = w[m];
  }
  __syncthreads();
  {
    T w[H];
    const int base = (pp / N) * G::PLANE + (pp % N) * G::ROW;
#pragma unroll
    for (int m = 0; m < H; ++m) w[m] = A[base + 2 * m + h];
    fft_pair_dit<N, -1>(w, h);
    __syncthreads();
#pragma unroll
    for (int m = 0; m < H; ++m) A[base + h * H + m] = w[m];
  }
  __syncthreads();
  const size_t off = (size_t)rank * G::P * N * N;
  const float* b1a = static_cast<const float*>(a.b1w) + (size_t)p0 * G::n + off;
  const float* b1b = (p0 + 1 < a.Nrho) ? b1a + G::n : nullptr;
  const int npairs = (a.Nrho + 1) / 2;
  T* Hout = static_cast<T*>(a.H) + ((size_t)e * npairs + pair) * G::n + off;
  for (int j = t; j < G::P * N * N; j += NT) {
    const T hv = A[slab_index<N, C>(j)];
    const float w0 = b1a[j], w1 = b1b ? b1b[j] : 0.f;
    Hout[j] = make_float2(hv.x * w0 + hv.y * w1, hv.y * w0 - hv.x * w1);
  }
}

// ---------------------------------------------------------------------------
// Epilogue: one cluster (FP64) per eval.
// ---------------------------------------------------------------------------
template <int N, int C>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
vhs_epilogue_kernel(VhsEpilogueArgs a) {
  using G = Geo<N, C>;
  using T = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr bool OS = OneSlab<N>::value;
  T* A = reinterpret_cast<T*>(smem_raw);
  T* Rb = OS ? A : A + G::SLAB;  // Y-slab receive
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int e = blockIdx.y;
  const size_t off = (size_t)rank * G::P * N * N;
  // Ghat = Ghat_M + sum_p H_p over this CTA's slab: elements in pairs,
  // UNR pairs per thread in flight per p so that the loads overlap
  constexpr int TOT2 = G::P * N * N / 2;
  constexpr int UNR = 8;
  for (int b0 = t; b0 < TOT2 && a.nt > 0; b0 += G::NT * UNR) {
    T acc[UNR][2];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      acc[u][0] = T{0, 0};
      acc[u][1] = T{0, 0};
    }
    for (int it = 0; it < a.nt; ++it) {
      const double w = a.pref[it];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int j2 = b0 + u * G::NT;
        if (j2 < TOT2) {
          T g0 = a.GMt[it][(size_t)e * G::n + off + 2 * j2];
          T g1 = a.GMt[it][(size_t)e * G::n + off + 2 * j2 + 1];
          for (int p = 0; p < a.Nrho; ++p) {
            const float4 h = reinterpret_cast<const float4*>(
                static_cast<const float2*>(a.Ht[it]) +
                ((size_t)e * a.Nrho + p) * G::n + off)[j2];
            g0.x += (double)h.x; g0.y += (double)h.y;
            g1.x += (double)h.z; g1.y += (double)h.w;
          }
          acc[u][0].x += w * g0.x; acc[u][0].y += w * g0.y;
          acc[u][1].x += w * g1.x; acc[u][1].y += w * g1.y;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int j2 = b0 + u * G::NT;
      if (j2 < TOT2) {
        const int si = slab_index<N, C>(2 * j2);
        A[si] = acc[u][0];
        A[si + 1] = acc[u][1];
      }
    }
  }
  // FP64 spectra (FP64 mode: one per radial point): UNR pairs per thread,
  // two radial points' loads in flight per step
  for (int b0 = t; b0 < TOT2 && a.nt == 0 && a.h_double; b0 += G::NT * UNR) {
    T acc[UNR][2];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int j2 = b0 + u * G::NT;
      if (a.GM && j2 < TOT2) {
        acc[u][0] = a.GM[(size_t)e * G::n + off + 2 * j2];
        acc[u][1] = a.GM[(size_t)e * G::n + off + 2 * j2 + 1];
      } else {
        acc[u][0] = T{0, 0};
        acc[u][1] = T{0, 0};
      }
    }
#pragma unroll 2
    for (int p = 0; p < a.Nrho; ++p) {
      const size_t hb = ((size_t)e * a.Nrho + p) * G::n + off;
      const double2* Hp = static_cast<const double2*>(a.H) + hb;
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        const int j2 = b0 + u * G::NT;
        if (j2 < TOT2) {
          const double2 h0 = Hp[2 * j2], h1 = Hp[2 * j2 + 1];
          acc[u][0].x += h0.x; acc[u][0].y += h0.y;
          acc[u][1].x += h1.x; acc[u][1].y += h1.y;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      const int j2 = b0 + u * G::NT;
      if (j2 < TOT2) {
        const int si = slab_index<N, C>(2 * j2);
        A[si] = acc[u][0];
        A[si + 1] = acc[u][1];
      }
    }
  }
  // packed FP32 spectra (FP32 mode: one per radial pair, eight at Nrho=16):
  // UNR32 pairs per thread with eight radial pairs' loads in flight per step,
  // so that a thread's whole share of a step's loads overlaps
  constexpr int UNR32 = 4;
  for (int b0 = t; b0 < TOT2 && a.nt == 0 && !a.h_double; b0 += G::NT * UNR32) {
    T acc[UNR32][2];
#pragma unroll
    for (int u = 0; u < UNR32; ++u) {
      const int j2 = b0 + u * G::NT;
      if (a.GM && j2 < TOT2) {
        acc[u][0] = a.GM[(size_t)e * G::n + off + 2 * j2];
        acc[u][1] = a.GM[(size_t)e * G::n + off + 2 * j2 + 1];
      } else {
        acc[u][0] = T{0, 0};
        acc[u][1] = T{0, 0};
      }
    }
#pragma unroll 8
    for (int p = 0; p < a.Nrho; ++p) {
      const size_t hb = ((size_t)e * a.Nrho + p) * G::n + off;
      const float4* Hp =
          reinterpret_cast<const float4*>(static_cast<const float2*>(a.H) + hb);
#pragma unroll
      for (int u = 0; u < UNR32; ++u) {
        const int j2 = b0 + u * G::NT;
        if (j2 < TOT2) {
          const float4 h = Hp[j2];
          acc[u][0].x += (double)h.x; acc[u][0].y += (double)h.y;
          acc[u][1].x += (double)h.z; acc[u][1].y += (double)h.w;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UNR32; ++u) {
      const int j2 = b0 + u * G::NT;
      if (j2 < TOT2) {
        const int si = slab_index<N, C>(2 * j2);
        A[si] = acc[u][0];
        A[si + 1] = acc[u][1];
      }
    }
  }
  __syncthreads();
  slab_row_pass<double, N, C, +1>(A, t);
  __syncthreads();
  {
    T w[N];
    slab_col_load_fft<double, N, C, +1>(A, t, w);
    if (OS) cluster_sync_all();  // every CTA has read its slab: exchange into it
    push_cols_to_yslab<double, N, C>(Rb, t, rank, w);
  }
  cluster_sync_all();
  T v[N];
  yslab_load_pencil<double, N, C>(Rb, t, v);
  fft<double, N, +1>(v);
  const int yl = t / N, z = t % N, y = rank * G::P + yl;
  const size_t fb = (size_t)slot_of(a.src_slots, a.src_base, e) * G::n;
  const size_t qb = (size_t)slot_of(a.dst_slots, a.dst_base, e) * G::n;
  const void* fin = a.f_list ? a.f_list[e] : a.f;
  void* qout = a.q_list ? a.q_list[e] : a.Q;
#pragma unroll
  for (int x = 0; x < N; ++x) {
    const size_t idx = ((size_t)x * N + y) * N + z;
    const double fv = load_real(fin, a.f_double, fb + idx);
    if (a.nt > 0) {
      double lf = 0;
      for (int it = 0; it < a.nt; ++it)
        lf += a.pref[it] * a.ReLft[it][(size_t)e * G::n + idx];
      v[x].y = v[x].x - fv * lf;
      continue;
    }
    const double lf = a.ReLf[(size_t)e * G::n + idx];
    v[x].y = a.bilinear ? a.prefac * (a.cg * v[x].x - a.cl * fv * lf)
                        : a.prefac * (v[x].x - fv * lf);
  }
  double lam[5] = {0, 0, 0, 0, 0};
  if (a.project) {
    // moments of this point's Q (FP64): thread -> CTA -> cluster, in a
    // fixed order so every CTA derives the same multipliers
    double* red = reinterpret_cast<double*>(A);  // A is free again
    const double cy = a.c0[y], cz = a.c0[z];
    double m[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int x = 0; x < N; ++x) {
      const double cx = a.c0[x], q = v[x].y * a.cw;
      m[0] += q; m[1] += q * cx; m[2] += q * cy; m[3] += q * cz;
      m[4] += q * (cx * cx + cy * cy + cz * cz);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 5; ++k) red[k * G::NT + t] = m[k];
    __syncthreads();
    if (t < 5) {
      double acc = 0;
      for (int i = 0; i < G::NT; ++i) acc += red[t * G::NT + i];
      red[5 * G::NT + t] = acc;
    }
    cluster_sync_all();
    double tot[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double acc = 0;
      for (int c = 0; c < C; ++c) acc += peer_ptr(red, (unsigned)c)[5 * G::NT + k];
      tot[k] = acc;
    }
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      double l = 0;
#pragma unroll
      for (int k = 0; k < 5; ++k) l += a.Ginv[j * 5 + k] * tot[k];
      lam[j] = l;
    }
    cluster_sync_all();  // peers have read this CTA's partial sums
  }
#pragma unroll
  for (int x = 0; x < N; ++x) {
    const size_t idx = ((size_t)x * N + y) * N + z;
    double qv = v[x].y;
    if (a.project) {
      const double cx = a.c0[x], cy = a.c0[y], cz = a.c0[z];
      qv -= lam[0] + lam[1] * cx + lam[2] * cy + lam[3] * cz +
            lam[4] * (cx * cx + cy * cy + cz * cz);
    }
    if (a.q_double) static_cast<double*>(qout)[qb + idx] += qv;
    else static_cast<float*>(qout)[qb + idx] += (float)qv;
  }
}

}  // namespace dgfs

// Fused fast-spectral VSS collision operator of a binary mixture, one
// species pair (p, q) per call.  Reference: DGFSBiVSSScatteringModel
// (dgfs1D/bi/scattering.py:47-321) and dgfs1D/bi/kernels/scattering/vss.mako.
//
// Per point the reference computes, with F = FFT(f_p)/n, G = FFT(f_q)/n and
// a_rm(l) = (pi/L) rho_r sigma_m . l:
//   t1 = e^{+i a m_q/(m_p+m_q)} F,  t2 = e^{-i a m_p/(m_p+m_q)} G,
//   Qhat = sum_{r,m} (w_r s_w / n) b_{pq,rm}(l) FFT(IFFT(t1) IFFT(t2)),
//   Q_p += prefac_pq (Re IFFT(Qhat) - f_p Re IFFT(c_pq G)).
// The weights b_{pq,rm} depend on both r and m, so every term needs its own
// forward transform (3 transforms per term).  Here one thread-block cluster
// evaluates one point completely: per term the two inverse transforms and
// the forward transform exchange through distributed shared memory, the
// spectral accumulator stays in shared memory, and the final inverse
// transform, the loss and the output run in the same kernel.  FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cluster_slab.cuh"
#include "fft_reg.cuh"

namespace dgfs {

// F = FFT(f)/n for a batch of slots (one cluster per slot, FP64).
struct Fft3Args {
  const void* f;
  int f_double;
  const int32_t* slots;
  int base;
  double2* out;        // [nevals][n]
};

template <int N, int C>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
fft3_forward_kernel(Fft3Args a) {
  using G = Geo<N, C>;
  using T = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int e = blockIdx.y;
  const int yl = t / N, z = t % N, y = rank * G::P + yl;
  const int slot = a.slots ? a.slots[e] : a.base + e;
  const size_t fb = (size_t)slot * G::n;
  T v[N];
#pragma unroll
  for (int x = 0; x < N; ++x) {
    v[x].x = a.f_double ? static_cast<const double*>(a.f)[fb + ((size_t)x * N + y) * N + z]
                        : (double)static_cast<const float*>(a.f)[fb + ((size_t)x * N + y) * N + z];
    v[x].y = 0.0;
  }
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
  const double inv_n = 1.0 / (double)G::n;
  T* out = a.out + (size_t)e * G::n + (size_t)rank * G::P * N * N;
  for (int j = t; j < G::P * N * N; j += G::NT) {
    T w = A[slab_index<N, C>(j)];
    w.x *= inv_n;
    w.y *= inv_n;
    out[j] = w;
  }
  cluster_sync_all();  // no CTA leaves while peers may still write into it
}

// Weights of one pair (vss.mako:51-93, launch loop bi/scattering.py:185-204):
//   b_rm(l) = sum_k B_mk fac_b(r) e^{-i mpq s_r sigma'_k . l}
//   c(l)   += sum_r sum_m sum_k B_mk fac_c(r) e^{-i s_r sigma'_k . l}
// with B_mk = (1 + sigma_m . sigma'_k)^eta, s_r = (pi/L) rho_r.  The phases
// are products of per-axis factors; k is processed in chunks so that the
// factor tables of a chunk fit in shared memory.
struct VssSetupArgs {
  const double* Bmk;         // [M][Mpre]
  const double* spre;        // [Mpre][3]
  const double* srho;        // [Nrho] s_r = (pi/L) rho_r
  const double* fac_b;       // [Nrho]
  const double* fac_c;       // [Nrho]
  double mpq;
  int M, Mpre, Nrho;
  double2* b;                // out [Nrho][M][n]
  double2* cpart;            // out [Nrho][n]: the r-th term of c
};

constexpr int kVssKChunk = 16;

template <int N>
__host__ __device__ constexpr int vss_setup_threads() { return N * N < 1024 ? N * N : 1024; }

template <int N>
__global__ void __launch_bounds__(vss_setup_threads<N>())
vss_setup_kernel(VssSetupArgs a) {
  constexpr int n = N * N * N;
  constexpr int NTH = vss_setup_threads<N>();
  const int lx = blockIdx.x, r = blockIdx.y;
  const int t = threadIdx.x;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // per chunk: x factor [K] (b, c), y/z factors [K][N] (b, c), B [M][K]
  double2* xb = reinterpret_cast<double2*>(smem_raw);
  double2* xc = xb + kVssKChunk;
  double2* yb = xc + kVssKChunk;
  double2* yc = yb + kVssKChunk * N;
  double2* zb = yc + kVssKChunk * N;
  double2* zc = zb + kVssKChunk * N;
  double* Bs = reinterpret_cast<double*>(zc + kVssKChunk * N);
  auto rep = [](int i) { return (double)((i < N / 2) ? i : i - N); };
  constexpr int PTS = (N * N + NTH - 1) / NTH;
  double2 accb[PTS][16];  // M <= 16
  double2 accc[PTS];
#pragma unroll
  for (int k = 0; k < PTS; ++k) {
    accc[k] = make_double2(0, 0);
#pragma unroll
    for (int m = 0; m < 16; ++m) accb[k][m] = make_double2(0, 0);
  }
  const double s = a.srho[r];
  for (int k0 = 0; k0 < a.Mpre; k0 += kVssKChunk) {
    const int kc = min(kVssKChunk, a.Mpre - k0);
    __syncthreads();
    for (int i = t; i < kc * (2 * N + 1); i += blockDim.x) {
      const int k = i / (2 * N + 1), j = i % (2 * N + 1);
      const double* sp = a.spre + 3 * (k0 + k);
      double sn, cs;
      if (j == 0) {
        const double ph = s * sp[0] * rep(lx);
        sincos(a.mpq * ph, &sn, &cs); xb[k] = make_double2(cs, -sn);
        sincos(ph, &sn, &cs); xc[k] = make_double2(cs, -sn);
      } else if (j <= N) {
        const int l = j - 1;
        const double ph = s * sp[1] * rep(l);
        sincos(a.mpq * ph, &sn, &cs); yb[k * N + l] = make_double2(cs, -sn);
        sincos(ph, &sn, &cs); yc[k * N + l] = make_double2(cs, -sn);
      } else {
        const int l = j - 1 - N;
        const double ph = s * sp[2] * rep(l);
        sincos(a.mpq * ph, &sn, &cs); zb[k * N + l] = make_double2(cs, -sn);
        sincos(ph, &sn, &cs); zc[k * N + l] = make_double2(cs, -sn);
      }
    }
    for (int i = t; i < a.M * kc; i += blockDim.x)
      Bs[i] = a.Bmk[(i / kc) * a.Mpre + k0 + i % kc];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PTS; ++p) {
      const int pt = min(t + p * NTH, N * N - 1);
      const int ly = pt / N, lz = pt % N;
      for (int k = 0; k < kc; ++k) {
        const double2 eb = cmul(cmul(xb[k], yb[k * N + ly]), zb[k * N + lz]);
        const double2 ec = cmul(cmul(xc[k], yc[k * N + ly]), zc[k * N + lz]);
        double bsum = 0;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
          if (m < a.M) {
            const double B = Bs[m * kc + k];
            accb[p][m].x += B * eb.x;
            accb[p][m].y += B * eb.y;
            bsum += B;
          }
        }
        accc[p].x += bsum * ec.x;
        accc[p].y += bsum * ec.y;
      }
    }
  }
#pragma unroll
  for (int p = 0; p < PTS; ++p) {
    const int pt = t + p * NTH;
    if (pt < N * N) {
      const size_t l = (size_t)lx * N * N + pt;
#pragma unroll
      for (int m = 0; m < 16; ++m)
        if (m < a.M) {
          double2 v = accb[p][m];
          v.x *= a.fac_b[r];
          v.y *= a.fac_b[r];
          a.b[((size_t)r * a.M + m) * n + l] = v;
        }
      a.cpart[(size_t)r * n + l] =
          make_double2(a.fac_c[r] * accc[p].x, a.fac_c[r] * accc[p].y);
    }
  }
}

// c(l) = sum_r cpart[r][l], in ascending r.
__global__ void vss_sum_c_kernel(const double2* cpart, int Nrho, size_t n,
                                 double2* c) {
  const size_t l = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  double2 s = make_double2(0, 0);
  for (int r = 0; r < Nrho; ++r) {
    s.x += cpart[(size_t)r * n + l].x;
    s.y += cpart[(size_t)r * n + l].y;
  }
  c[l] = s;
}

struct VssPairArgs {
  const double2* Fp;       // [nevals][n]  FFT(f_p)/n
  const double2* Fq;       // [nevals][n]  FFT(f_q)/n
  const double2* b;        // [Nrho][M][n]
  const double2* c;        // [n]
  const double2* ph;       // [Nrho][M][2][3][N]: e^{+i a mq'}, e^{-i a mp'} factors
  const double* w;         // [Nrho] w_r s_w / n
  const void* fp;          // f_p (for the loss product)
  int f_double;
  const int32_t* src_slots;
  int src_base;
  void* Q;                 // Q_p output (+=)
  int q_double;
  const int32_t* dst_slots;
  int dst_base;
  double prefac;
  int Nrho, M;
};

template <int N, int C>
__device__ __forceinline__ void vss_zpass_inverse(double2* A, const double2* Frow0,
                                                  const double2* tb, int t,
                                                  unsigned rank) {
  using G = Geo<N, C>;
  const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
  const double2 bxy = cmul(tb[lx], tb[N + ly]);
  const double2* row = Frow0 + ((size_t)lx * N + ly) * N;
  double2 v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = cmul(row[k], cmul(bxy, tb[2 * N + k]));
  fft<double, N, +1>(v);
  const int base = pl * G::PLANE + ly * G::ROW;
#pragma unroll
  for (int k = 0; k < N; ++k) A[base + k] = v[k];
}

template <int N, int C>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
vss_pair_kernel(VssPairArgs a) {
  using G = Geo<N, C>;
  using T = double2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);   // X-slab work buffer
  T* Rb = A + G::SLAB;                     // Y-slab receive buffer
  T* U = Rb + G::SLAB;                     // Y-slab: u pencils / loss
  T* Qh = U + G::SLAB;                     // X-slab spectral accumulator
  T* tab = Qh + G::SLAB;                   // [2][3][N] phase factors
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int e = blockIdx.y;
  const int yl = t / N, zz = t % N;
  const int ybase = yl * G::PLANE + zz;    // thread's pencil in a Y-slab
  const T* Fp = a.Fp + (size_t)e * G::n;
  const T* Fq = a.Fq + (size_t)e * G::n;
  bool pending = false;  // an arrive is outstanding (receive buffer in use)

  // exchange this thread's y-pass column into the owners' receive buffers
  auto exchange_cols = [&](const T* v) {
    if (pending) cluster_wait();
    push_cols_to_yslab<double, N, C>(Rb, t, rank, v);
    cluster_arrive();
    cluster_wait();
  };
  auto release_receive = [&]() {
    cluster_arrive();
    pending = true;
  };
  // inverse 3-D FFT of F * tables; result pencil (x) left in v
  auto inverse = [&](const T* F, const T* tb, T* v) {
    vss_zpass_inverse<N, C>(A, F, tb, t, rank);
    __syncthreads();
    slab_col_load_fft<double, N, C, +1>(A, t, v);
    exchange_cols(v);
    yslab_load_pencil<double, N, C>(Rb, t, v);
    release_receive();
    fft<double, N, +1>(v);
  };

  for (int j = t; j < G::SLAB; j += G::NT) Qh[j] = T{0, 0};
  const int T_terms = a.Nrho * a.M;
#pragma unroll 1
  for (int term = 0; term < T_terms; ++term) {
    const int r = term / a.M;
    __syncthreads();
    for (int i = t; i < 6 * N; i += G::NT) tab[i] = a.ph[(size_t)term * 6 * N + i];
    __syncthreads();
    T v[N];
    inverse(Fp, tab, v);                       // u = IFFT(e^{+i a mq'} F)
#pragma unroll
    for (int x = 0; x < N; ++x) U[ybase + x * G::ROW] = v[x];
    inverse(Fq, tab + 3 * N, v);               // v = IFFT(e^{-i a mp'} G)
#pragma unroll
    for (int x = 0; x < N; ++x) v[x] = cmul(U[ybase + x * G::ROW], v[x]);
    fft<double, N, -1>(v);                     // forward: x pass
    if (pending) cluster_wait();
    push_pencils_to_xslab<double, N, C>(A, t, rank, v);
    cluster_arrive();
    cluster_wait();
    pending = false;
    {
      T w[N];
      slab_col_load_fft<double, N, C, -1>(A, t, w);
      const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
      for (int k = 0; k < N; ++k) A[base + k * G::ROW] = w[k];
    }
    __syncthreads();
    {
      // z pass (rows) and accumulation W_r b_rm (*) FFT(h) into Qhat
      const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
      const int base = pl * G::PLANE + ly * G::ROW;
      T w[N];
#pragma unroll
      for (int k = 0; k < N; ++k) w[k] = A[base + k];
      fft<double, N, -1>(w);
      const T* brow = a.b + (size_t)term * G::n + ((size_t)lx * N + ly) * N;
      const double wr = a.w[r];
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const T bb = brow[k];
        const T pr = cmul(w[k], bb);
        Qh[base + k].x += wr * pr.x;
        Qh[base + k].y += wr * pr.y;
      }
    }
  }

  // loss: Re IFFT(c (*) G) -> U (real parts), then the gain IFFT(Qhat)
  {
    __syncthreads();
    const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
    const T* row = Fq + ((size_t)lx * N + ly) * N;
    const T* crow = a.c + ((size_t)lx * N + ly) * N;
    T w[N];
#pragma unroll
    for (int k = 0; k < N; ++k) w[k] = cmul(crow[k], row[k]);
    fft<double, N, +1>(w);
    const int base = pl * G::PLANE + ly * G::ROW;
#pragma unroll
    for (int k = 0; k < N; ++k) A[base + k] = w[k];
  }
  __syncthreads();
  T v[N];
  slab_col_load_fft<double, N, C, +1>(A, t, v);
  exchange_cols(v);
  yslab_load_pencil<double, N, C>(Rb, t, v);
  release_receive();
  fft<double, N, +1>(v);
#pragma unroll
  for (int x = 0; x < N; ++x) U[ybase + x * G::ROW] = v[x];
  slab_row_pass<double, N, C, +1>(Qh, t);
  __syncthreads();
  slab_col_load_fft<double, N, C, +1>(Qh, t, v);
  exchange_cols(v);
  yslab_load_pencil<double, N, C>(Rb, t, v);
  release_receive();
  fft<double, N, +1>(v);
  const int y = rank * G::P + yl;
  const size_t fb = (size_t)(a.src_slots ? a.src_slots[e] : a.src_base + e) * G::n;
  const size_t qb = (size_t)(a.dst_slots ? a.dst_slots[e] : a.dst_base + e) * G::n;
#pragma unroll
  for (int x = 0; x < N; ++x) {
    const size_t idx = ((size_t)x * N + y) * N + zz;
    const double fv = a.f_double ? static_cast<const double*>(a.fp)[fb + idx]
                                 : (double)static_cast<const float*>(a.fp)[fb + idx];
    const double qv = a.prefac * (v[x].x - fv * U[ybase + x * G::ROW].x);
    if (a.q_double) static_cast<double*>(a.Q)[qb + idx] += qv;
    else static_cast<float*>(a.Q)[qb + idx] += (float)qv;
  }
  if (pending) cluster_wait();
}

// ---------------------------------------------------------------------------
// FP32 mode (no counterpart in the reference, which is FP64 only): the
// Maxwellian split of the VHS operator carried over to a pair.  With
// f_p = M_p + g_p, f_q = M_q + g_q (M from FP64 moments, separable),
//   IFFT(t1) = u_M + X_u,  IFFT(t2) = v_M + X_v,
//   u_M = prod_a IFFT1(e^{+i a_a mq'} mhat_p,a),  v_M likewise with q, -mp',
//   X_u = IFFT3(e^{+i a mq'} F_gp),  X_v = IFFT3(e^{-i a mp'} F_gq)  (FP32),
// and the product splits into u_M v_M, whose 3-D transform is the product of
// the 1-D FP64 transforms H_a = FFT1(u_M,a v_M,a) (vss_maxwell_gain_kernel),
// and the remainder u_M X_v + X_u (v_M + X_v), transformed in FP32
// (vss_terms32_kernel, one cluster per (pair, point, radial point), summed
// over the directions in shared memory).  The radial sum, the final transform
// and the loss f_p Re IFFT(c G) run in FP64 (prologue and epilogue kernels
// of the VHS operator, with the complex loss kernel c).
// ---------------------------------------------------------------------------
struct VssTablesArgs {
  const double2* mhat_p;   // [E][3][N]
  const double2* mhat_q;   // [E][3][N]
  const double2* ph;       // [T][2][3][N]
  float2* uv;              // out [E][T][2][3][N]: u_M,a and v_M,a (FP32)
  double2* hh;             // out [E][T][3][N]: FFT1(u_M,a v_M,a)
  int T, nevals;
};

template <int N>
__global__ void vss_tables_kernel(VssTablesArgs a) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= a.nevals * a.T * 3) return;
  const int ax = gid % 3, term = (gid / 3) % a.T, e = gid / (3 * a.T);
  const double2* mp = a.mhat_p + (size_t)e * 3 * N + ax * N;
  const double2* mq = a.mhat_q + (size_t)e * 3 * N + ax * N;
  const double2* pu = a.ph + ((size_t)term * 6 + ax) * N;
  const double2* pv = a.ph + ((size_t)term * 6 + 3 + ax) * N;
  double2 u[N], v[N];
#pragma unroll
  for (int l = 0; l < N; ++l) {
    u[l] = cmul(mp[l], pu[l]);
    v[l] = cmul(mq[l], pv[l]);
  }
  fft<double, N, +1>(u);
  fft<double, N, +1>(v);
  float2* uv = a.uv + ((size_t)e * a.T + term) * 6 * N;
#pragma unroll
  for (int l = 0; l < N; ++l) {
    uv[ax * N + l] = make_float2((float)u[l].x, (float)u[l].y);
    uv[(3 + ax) * N + l] = make_float2((float)v[l].x, (float)v[l].y);
    u[l] = cmul(u[l], v[l]);
  }
  fft<double, N, -1>(u);
  double2* hh = a.hh + (((size_t)e * a.T + term) * 3 + ax) * N;
#pragma unroll
  for (int l = 0; l < N; ++l) hh[l] = u[l];
}

// GM[e][l] = sum_r w_r sum_m b_rm(l) prod_a H_a,rm(l_a)   (FP64)
// grid (ceil(n/256), E), one thread per wavenumber l.
struct VssGainArgs {
  const double2* hh;       // [E][T][3][N]
  const double2* b;        // [T][n]
  const double* w;         // [Nrho]
  double2* GM;             // out [E][n]
  int Nrho, M;
};

template <int N>
__global__ void __launch_bounds__(256) vss_maxwell_gain_kernel(VssGainArgs a) {
  constexpr int n = N * N * N;
  const int l = blockIdx.x * 256 + threadIdx.x, e = blockIdx.y;
  if (l >= n) return;
  const int lx = l / (N * N), ly = (l / N) % N, lz = l % N;
  const int T = a.Nrho * a.M;
  const double2* hh = a.hh + (size_t)e * T * 3 * N;
  double2 G = make_double2(0, 0);
  for (int r = 0; r < a.Nrho; ++r) {
    double2 acc = make_double2(0, 0);
    for (int m = 0; m < a.M; ++m) {
      const int term = r * a.M + m;
      const double2* h = hh + (size_t)term * 3 * N;
      const double2 x = cmul(cmul(h[lx], h[N + ly]), h[2 * N + lz]);
      const double2 p = cmul(x, a.b[(size_t)term * n + l]);
      acc.x += p.x;
      acc.y += p.y;
    }
    G.x += a.w[r] * acc.x;
    G.y += a.w[r] * acc.y;
  }
  a.GM[(size_t)e * n + l] = G;
}

// Pointers of one species pair; a launch covers npair pairs, grid z =
// npair * nevals (pair major).
struct VssTerms32Pair {
  const float2* Fgp;       // [E][n] F_gp
  const float2* Fgq;       // [E][n] F_gq
  const float2* ph;        // [T][2][3][N] FP32 phase factors
  const float2* uv;        // [E][T][2][3][N] u_M,a, v_M,a
  const float2* b;         // [T][n] FP32 weights
  float2* H;               // out [E][Nrho][n]
};
struct VssTerms32Args {
  VssTerms32Pair pr[16];
  const double* w;         // [Nrho]
  int Nrho, M, nevals;
};

// z-pass of an inverse transform: rows of F (global, FP32) times the phase.
template <int N, int C>
__device__ __forceinline__ void vss32_zpass(float2* A, const float2* F,
                                            const float2* tb, int t,
                                            unsigned rank) {
  using G = Geo<N, C>;
  const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
  const float2 bxy = cmul(tb[lx], tb[N + ly]);
  const float2* row = F + ((size_t)lx * N + ly) * N;
  float2 v[N];
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = cmul(row[k], cmul(bxy, tb[2 * N + k]));
  fft<float, N, +1>(v);
  const int base = pl * G::PLANE + ly * G::ROW;
#pragma unroll
  for (int k = 0; k < N; ++k) A[base + k] = v[k];
}

// One cluster per (pair, point, radial point r); per direction m three
// transforms, each with one cluster barrier (arrive after the stores into
// the peers, wait before reading):
//   T1 = IFFT3(phi_p F_gp) -> receive buffer R0 -> X_u (registers)
//   T2 = IFFT3(phi_q F_gq) -> R1 -> X_v, combined with X_u into h
//   T3 = FFT3(h) -> X-slab B -> b_rm (*) FFT(h) added into Qhat (shared)
// The z-pass of T2 runs while T1's stores land, and the z-pass of T1 of the
// next direction while T2's do.  Five slabs: A (z/y passes of T1 and T2),
// B (T3), R0, R1, Qhat; the direction tables sit in a two-slot ring.
template <int N, int C>
__global__ void __launch_bounds__(Geo<N, C>::NT, 1)
vss_terms32_kernel(VssTerms32Args a) {
  using G = Geo<N, C>;
  using T = float2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);   // X-slab work buffer (inverse)
  T* B = A + G::SLAB;                      // X-slab receive (forward)
  T* R0 = B + G::SLAB;                     // Y-slab receive buffers R0, R1
  T* Qh = R0 + 2 * G::SLAB;                // X-slab spectral accumulator
  T* tab = Qh + G::SLAB;                   // [2][12N]: phases p, q | u_M | v_M
  const int t = threadIdx.x;
  const unsigned rank = cluster_rank();
  const int r = blockIdx.y, e = blockIdx.z % a.nevals;
  const VssTerms32Pair& P = a.pr[blockIdx.z / a.nevals];
  const int yl = t / N, zz = t % N, yy = rank * G::P + yl;
  const T* Fp = P.Fgp + (size_t)e * G::n;
  const T* Fq = P.Fgq + (size_t)e * G::n;
  const int Tt = a.Nrho * a.M;
  auto load_tables = [&](int m) {
    T* dst = tab + (m & 1) * 12 * N;
    const int term = r * a.M + m;
    for (int i = t; i < 6 * N; i += G::NT) {
      dst[i] = P.ph[(size_t)term * 6 * N + i];
      dst[6 * N + i] = P.uv[((size_t)e * Tt + term) * 6 * N + i];
    }
  };
  uint32_t rb[C], bb[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    rb[c] = mapa_u32(smem_u32(R0), (uint32_t)c);
    bb[c] = mapa_u32(smem_u32(B), (uint32_t)c);
  }
  // y-pass stores of an inverse transform into the peers' receive buffer buf
  auto push_y = [&](int buf, const T* v) {
    const int lx = rank * G::P + t / N, z = t % N;
    const uint32_t off = (uint32_t)(buf * G::SLAB + lx * G::ROW + z) * 8u;
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int j = 0; j < G::P; ++j)
        st_cluster(rb[c] + off + (uint32_t)(j * G::PLANE) * 8u, v[c * G::P + j]);
  };
  auto col_load = [&](const T* S, T* v) {
    const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = S[base + k * G::ROW];
  };
  for (int j = t; j < G::SLAB; j += G::NT) Qh[j] = T{0.f, 0.f};
  load_tables(0);
  __syncthreads();
  vss32_zpass<N, C>(A, Fp, tab, t, rank);
  __syncthreads();
#pragma unroll 1
  for (int m = 0; m < a.M; ++m) {
    const T* tb = tab + (m & 1) * 12 * N;
    const int term = r * a.M + m;
    T v[N], Xu[N];
    // T1: y-pass, stores into R0; the z-pass of T2 overlaps them
    col_load(A, v);
    __syncthreads();                 // A read; ring slot (m+1)&1 free
    if (m + 1 < a.M) load_tables(m + 1);
    fft<float, N, +1>(v);
    push_y(0, v);
    cluster_arrive();
    vss32_zpass<N, C>(A, Fq, tb + 3 * N, t, rank);
    __syncthreads();
    cluster_wait();
    {
      const T* R = R0 + yl * G::PLANE + zz;
#pragma unroll
      for (int x = 0; x < N; ++x) Xu[x] = R[x * G::ROW];
    }
    fft<float, N, +1>(Xu);
    // T2: y-pass, stores into R1; the z-pass of T1 of the next direction
    // overlaps them
    col_load(A, v);
    __syncthreads();                 // A read; the tables of m+1 are stored
    fft<float, N, +1>(v);
    push_y(1, v);
    cluster_arrive();
    if (m + 1 < a.M) vss32_zpass<N, C>(A, Fp, tab + ((m + 1) & 1) * 12 * N, t, rank);
    cluster_wait();
    {
      const T* R = R0 + G::SLAB + yl * G::PLANE + zz;
#pragma unroll
      for (int x = 0; x < N; ++x) v[x] = R[x * G::ROW];
    }
    fft<float, N, +1>(v);            // X_v
    {
      const T* ut = tb + 6 * N;
      const T* vt = tb + 9 * N;
      const T uyz = cmul(ut[N + yy], ut[2 * N + zz]);
      const T vyz = cmul(vt[N + yy], vt[2 * N + zz]);
#pragma unroll
      for (int x = 0; x < N; ++x) {
        const T uM = cmul(ut[x], uyz), vM = cmul(vt[x], vyz);
        const T Xv = v[x];
        const T a1 = cmul(uM, Xv);
        const T a2 = cmul(Xu[x], make_float2(vM.x + Xv.x, vM.y + Xv.y));
        v[x] = make_float2(a1.x + a2.x, a1.y + a2.y);
      }
    }
    // T3: forward x-pass, stores into the peers' B, then y- and z-passes
    // on B and the weighted accumulation into Qhat
    fft<float, N, -1>(v);
    {
      const uint32_t off = (uint32_t)(yy * G::ROW + zz) * 8u;
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int j = 0; j < G::P; ++j)
          st_cluster(bb[c] + off + (uint32_t)(j * G::PLANE) * 8u, v[c * G::P + j]);
    }
    cluster_arrive();
    cluster_wait();
    {
      T w2[N];
      col_load(B, w2);
      fft<float, N, -1>(w2);
      const int base = (t / N) * G::PLANE + (t % N);
#pragma unroll
      for (int k = 0; k < N; ++k) B[base + k * G::ROW] = w2[k];
    }
    __syncthreads();
    {
      const int pl = t / N, ly = t % N, lx = rank * G::P + pl;
      const int base = pl * G::PLANE + ly * G::ROW;
      T w2[N];
#pragma unroll
      for (int k = 0; k < N; ++k) w2[k] = B[base + k];
      fft<float, N, -1>(w2);
      const T* brow = P.b + (size_t)term * G::n + ((size_t)lx * N + ly) * N;
#pragma unroll
      for (int k = 0; k < N; ++k) {
        const T pr = cmul(w2[k], brow[k]);
        Qh[base + k].x += pr.x;
        Qh[base + k].y += pr.y;
      }
    }
  }
  __syncthreads();
  const float wr = (float)a.w[r];
  T* H = P.H + ((size_t)e * a.Nrho + r) * G::n + (size_t)rank * G::P * N * N;
  for (int j = t; j < G::P * N * N; j += G::NT) {
    const T q = Qh[slab_index<N, C>(j)];
    H[j] = make_float2(wr * q.x, wr * q.y);
  }
}

}  // namespace dgfs

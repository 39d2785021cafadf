// Fourier-neural-operator surrogate of Q(f,f): forward, backward and Adam.
//
// Network (width WD = 32, projection width PJ = 128, GELU in the tanh form):
//   features  x0 = [f/rho, g, g r, g r^2],  g = (f - M)/(rho sigma),
//             r = |c - u|/sqrt(T), sigma = rms((f - M)/rho) per sample
//             (M: local Maxwellian; g r^k let the lift form the local loss
//             frequency times g, which no convolution can)
//   lift      v0 = x0 P + p                          (4 -> 32)
//   layer l   y_l = v_l D_l + d_l + Re IDFT(W_l . DFT(v_l)),  l = 0..3
//             v_{l+1} = GELU(y_l) (l < 3),  v_4 = y_3
//   project   out = GELU(v_4 Q1 + q1) q2 + q2b       (32 -> 128 -> 1)
//   Q = rho^2 sigma sQ out (Q is nearly linear in f - M near equilibrium, so
//   the target Q/(rho^2 sigma sQ) and the features are O(1)), then the FP64
//   conservation projection.
// DFT is the truncated separable transform onto K modes per axis
// (k = 0..K/2-1, -K/2..-1): A = F_x (x) F_y (x) F_z, F[k][x] = e^{-2 pi i k x/N};
// IDFT applies conj(F)^T / N per axis.  W_l[m] is a 32x32 complex matrix per
// retained mode m.  Activations are stored in BF16 (features, v_l, y_l), the
// weights are read from a BF16 copy of the FP32 master parameters, and every
// sum accumulates in FP32 (moments, projection and loss norms in FP64).
//
// Layouts: point-major, channels innermost: v[b][pt][c], pt = (x*N + y)*N + z.
// Spectral data: [b][kx][ky][kz][c] complex FP32.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dgfs {
namespace fno {

constexpr int WD = 32;   // width
constexpr int PJ = 128;  // projection width
constexpr int CIN = 4;   // input features

// GELU in the tanh form, GELU(x) = x/2 (1 + tanh(c (x + a x^3))),
// c = sqrt(2/pi), a = 0.044715 (Hendrycks & Gimpel), with the hardware tanh
// approximation (tanh.approx.f32, relative error below 2^-10.9): one MUFU and
// five FP32 operations.  GELU is the hot scalar of the projection (128 per
// grid point) and of the dense layers' epilogues.
__device__ __forceinline__ float tanh_fast(float u) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(u));
  return r;
}
__device__ __forceinline__ float gelu(float x) {
  const float h = 0.5f * x;
  return fmaf(h, tanh_fast(x * fmaf(0.0356774081f, x * x, 0.7978845608f)), h);
}
__device__ __forceinline__ float gelu_d(float x) {
  const float x2 = x * x;
  const float t = tanh_fast(x * fmaf(0.0356774081f, x2, 0.7978845608f));
  return 0.5f * (1.f + t) +
         0.5f * x * (1.f - t * t) * fmaf(0.1070322244f, x2, 0.7978845608f);
}
__device__ __forceinline__ float bf(const __nv_bfloat16 v) {
  return __bfloat162float(v);
}
__device__ __forceinline__ __nv_bfloat16 tobf(float v) {
  return __float2bfloat16_rn(v);
}

// Parameter offsets (in floats) of the flat parameter vector.
struct Layout {
  int K;           // modes per axis
  long P, p;       // lift [CIN][WD], [WD]
  long W[4];       // spectral [K^3][WD][WD] complex (2 floats)
  long D[4], d[4]; // dense [WD][WD], [WD]
  long Q1, q1, q2, q2b;
  long total;
  __host__ __device__ void init(int K_) {
    K = K_;
    long o = 0;
    P = o; o += CIN * WD;
    p = o; o += WD;
    for (int l = 0; l < 4; ++l) {
      W[l] = o; o += 2L * K * K * K * WD * WD;
      D[l] = o; o += WD * WD;
      d[l] = o; o += WD;
    }
    Q1 = o; o += WD * PJ;
    q1 = o; o += PJ;
    q2 = o; o += PJ;
    q2b = o; o += 1;
    total = o;
  }
};

// ---------------------------------------------------------------------------
// Features + lift: one CTA per sample.  FP64 moments of f, the Maxwellian,
// x0 = [f/rho, g, g r, g r^2] (BF16) and v0 = x0 P + p (BF16).
// ---------------------------------------------------------------------------
struct FeatArgs {
  const void* f; int f_double; const int32_t* src_slots; int src_base;
  const double* c0; double cw; int N;
  const __nv_bfloat16* w16;  // BF16 parameters
  Layout L;
  __nv_bfloat16* x0;  // [B][n][CIN]
  __nv_bfloat16* v0;  // [B][n][WD]
  double* qs;         // out [B] rho^2 sigma (output scale without sQ)
  double* part;       // scratch [B][FCH][6] partial sums
};

template <int NT>
__device__ __forceinline__ void block_sum5(double* s, double* red) {
  // s[5] per thread -> totals in red[0..4] (all threads see them after return)
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double v = s[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[8 + w * 5 + k] = v;
  }
  __syncthreads();
  if (t < 5) {
    double v = 0;
    for (int i = 0; i < NT / 32; ++i) v += red[8 + i * 5 + t];
    red[t] = v;
  }
  __syncthreads();
}

// Features in three grid-wide passes over f, grid (CH chunks, B samples):
//   pass 0: per-chunk partial moments  (sum f, f c, f |c|^2)      -> part[b][ch][0..4]
//   pass 1: per-chunk partial sum g^2 (g = (f - M)/rho)            -> part[b][ch][5]
//   pass 2: features x0 and lift v0; qs[b] = rho^2 sigma
// Every CTA re-reduces the CH partials of its sample in a fixed order, so all
// CTAs see identical rho, u, T, sigma.
constexpr int FCH = 64;  // chunks per sample
static_assert(CIN == 4, "the feature pass packs four BF16 values");

// Totals of the FCH partial records [FCH][6] of one sample, by one warp:
// lane l adds chunks l and l + 32, then an xor-shuffle tree.  Every step adds
// the same two operands on both lanes of a pair, so all lanes (and all CTAs
// reading the same partials) end with bitwise identical totals.
static_assert(FCH == 64, "reduce_parts assumes 64 chunks");
__device__ __forceinline__ void reduce_parts(const double* P, double* m) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = P[lane * 6 + k] + P[(lane + 32) * 6 + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    m[k] = v;
  }
}

__device__ __forceinline__ void feat_load(const FeatArgs& a, int b, long i,
                                          double& fv, double& cx, double& cy,
                                          double& cz) {
  const int N = a.N;
  const long n = (long)N * N * N;
  const long fb = (long)(a.src_slots ? a.src_slots[b] : a.src_base + b) * n;
  const int x = (int)(i / (N * N)), y = (int)((i / N) % N), z = (int)(i % N);
  fv = a.f_double ? static_cast<const double*>(a.f)[fb + i]
                  : (double)static_cast<const float*>(a.f)[fb + i];
  cx = a.c0[x]; cy = a.c0[y]; cz = a.c0[z];
}

struct FeatState { double rho, ux, uy, uz, T, amp, irho; };

// State of one sample from the totals m of its partial records.
__device__ __forceinline__ FeatState feat_state(const FeatArgs& a,
                                                const double* m) {
  FeatState s;
  double rho = m[0] * a.cw;
  s.ux = m[1] * a.cw / rho; s.uy = m[2] * a.cw / rho; s.uz = m[3] * a.cw / rho;
  double T = (2.0 / 3.0) * (m[4] * a.cw / rho - (s.ux * s.ux + s.uy * s.uy + s.uz * s.uz));
  if (!(rho > 1e-300)) rho = 1.0;
  if (!(T > 1e-6)) T = 1.0;
  s.rho = rho; s.T = T;
  s.amp = rho / pow(M_PI * T, 1.5);
  s.irho = 1.0 / rho;
  return s;
}

template <int PASS>
__global__ void __launch_bounds__(256) fno_features_kernel(FeatArgs a) {
  __shared__ double red[8 + 5 * 8];
  __shared__ float wl[CIN * WD + WD];
  __shared__ FeatState st;
  __shared__ double sig_s;
  const int ch = blockIdx.x, b = blockIdx.y, t = threadIdx.x, N = a.N;
  const long n = (long)N * N * N, len = n / FCH, i0 = ch * len;
  if (PASS >= 1) {
    if (t < 32) {
      double m[6];
      reduce_parts(a.part + (long)b * FCH * 6, m);
      if (t == 0) {
        st = feat_state(a, m);
        if (PASS == 2) sig_s = fmax(sqrt(m[5] / (double)n), 1e-300);
      }
    }
    if (PASS == 2)
      for (int i = t; i < CIN * WD + WD; i += 256) wl[i] = bf(a.w16[a.L.P + i]);
    __syncthreads();
  }
  if (PASS == 0) {
    double s[5] = {0, 0, 0, 0, 0};
    for (long i = i0 + t; i < i0 + len; i += 256) {
      double fv, cx, cy, cz;
      feat_load(a, b, i, fv, cx, cy, cz);
      s[0] += fv; s[1] += fv * cx; s[2] += fv * cy; s[3] += fv * cz;
      s[4] += fv * (cx * cx + cy * cy + cz * cz);
    }
    block_sum5<256>(s, red);
    if (t < 5) a.part[((long)b * FCH + ch) * 6 + t] = red[t];
  } else if (PASS == 1) {
    const FeatState S = st;
    double s[5] = {0, 0, 0, 0, 0};
    for (long i = i0 + t; i < i0 + len; i += 256) {
      double fv, cx, cy, cz;
      feat_load(a, b, i, fv, cx, cy, cz);
      const double dx = cx - S.ux, dy = cy - S.uy, dz = cz - S.uz;
      const double g = (fv - S.amp * exp(-(dx * dx + dy * dy + dz * dz) / S.T)) * S.irho;
      s[0] += g * g;
    }
    block_sum5<256>(s, red);
    if (t == 0) a.part[((long)b * FCH + ch) * 6 + 5] = red[0];
  } else {
    const FeatState S = st;
    const double isig = 1.0 / sig_s;
    if (ch == 0 && t == 0) a.qs[b] = S.rho * S.rho * sig_s;
    for (long i = i0 + t; i < i0 + len; i += 256) {
      double fv, cx, cy, cz;
      feat_load(a, b, i, fv, cx, cy, cz);
      const double dx = cx - S.ux, dy = cy - S.uy, dz = cz - S.uz;
      const double r2 = (dx * dx + dy * dy + dz * dz) / S.T;
      const double g = (fv - S.amp * exp(-r2)) * S.irho * isig, r = sqrt(r2);
      const __nv_bfloat16 h[CIN] = {tobf((float)(fv * S.irho)), tobf((float)g),
                                    tobf((float)(g * r)), tobf((float)(g * r2))};
      const long pt = (long)b * n + i;
      float xf[CIN];
      uint2 xs;
      reinterpret_cast<__nv_bfloat16*>(&xs)[0] = h[0];
      reinterpret_cast<__nv_bfloat16*>(&xs)[1] = h[1];
      reinterpret_cast<__nv_bfloat16*>(&xs)[2] = h[2];
      reinterpret_cast<__nv_bfloat16*>(&xs)[3] = h[3];
      *reinterpret_cast<uint2*>(a.x0 + pt * CIN) = xs;
#pragma unroll
      for (int k = 0; k < CIN; ++k) xf[k] = bf(h[k]);
      uint4* v = reinterpret_cast<uint4*>(a.v0 + pt * WD);
#pragma unroll
      for (int q = 0; q < WD / 8; ++q) {
        uint4 pk;
        __nv_bfloat162* p2 = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int o = q * 8 + 2 * e;
          float y0 = wl[CIN * WD + o], y1 = wl[CIN * WD + o + 1];
#pragma unroll
          for (int k = 0; k < CIN; ++k) {
            y0 += xf[k] * wl[k * WD + o];
            y1 += xf[k] * wl[k * WD + o + 1];
          }
          p2[e] = __floats2bfloat162_rn(y0, y1);
        }
        v[q] = pk;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Truncated DFT along one axis: in [outer][LIN][inner] -> out [outer][LOUT][inner],
// out[k] = sum_j T[k][j] in[j] with a complex table T [LOUT][LIN].
// IN: 0 BF16 real, 1 FP32 real, 2 complex FP32.
// OUT: 0 complex FP32, 1 Re -> FP32 store, 2 Re -> FP32 accumulate,
//      3 Re -> BF16 store.
// One thread per two adjacent (outer, inner) pencils (inner is even):
// consecutive threads take consecutive inner pairs, so loads and stores are
// coalesced and every table entry read from shared memory serves two pencils.
// ---------------------------------------------------------------------------
template <int LIN, int LOUT, int IN, int OUT>
__global__ void __launch_bounds__(256)
fno_dft_kernel(const void* in, void* out, const float2* table, long outer,
               int inner) {
  __shared__ float2 tb[LOUT * LIN];
  for (int i = threadIdx.x; i < LOUT * LIN; i += blockDim.x) tb[i] = table[i];
  __syncthreads();
  const int half = inner / 2;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= outer * half) return;
  const long o = gid / half;
  const int i = 2 * (int)(gid % half);
  float2 x0[LIN], x1[LIN];
#pragma unroll
  for (int j = 0; j < LIN; ++j) {
    const long idx = (o * LIN + j) * inner + i;
    if (IN == 0) {
      const float2 v = __bfloat1622float2(
          *reinterpret_cast<const __nv_bfloat162*>(static_cast<const __nv_bfloat16*>(in) + idx));
      x0[j] = make_float2(v.x, 0.f);
      x1[j] = make_float2(v.y, 0.f);
    } else if (IN == 1) {
      const float2 v = *reinterpret_cast<const float2*>(static_cast<const float*>(in) + idx);
      x0[j] = make_float2(v.x, 0.f);
      x1[j] = make_float2(v.y, 0.f);
    } else {
      const float4 v = *reinterpret_cast<const float4*>(static_cast<const float2*>(in) + idx);
      x0[j] = make_float2(v.x, v.y);
      x1[j] = make_float2(v.z, v.w);
    }
  }
#pragma unroll 2
  for (int k = 0; k < LOUT; ++k) {
    float r0 = 0.f, i0 = 0.f, r1 = 0.f, i1 = 0.f;
#pragma unroll
    for (int j = 0; j < LIN; ++j) {
      const float2 w = tb[k * LIN + j];
      if (IN == 2) {
        r0 += w.x * x0[j].x - w.y * x0[j].y;
        r1 += w.x * x1[j].x - w.y * x1[j].y;
        if (OUT == 0) {
          i0 += w.x * x0[j].y + w.y * x0[j].x;
          i1 += w.x * x1[j].y + w.y * x1[j].x;
        }
      } else {
        r0 += w.x * x0[j].x;
        r1 += w.x * x1[j].x;
        if (OUT == 0) {
          i0 += w.y * x0[j].x;
          i1 += w.y * x1[j].x;
        }
      }
    }
    const long idx = (o * LOUT + k) * inner + i;
    if (OUT == 0) {
      *reinterpret_cast<float4*>(static_cast<float2*>(out) + idx) = make_float4(r0, i0, r1, i1);
    } else if (OUT == 1) {
      *reinterpret_cast<float2*>(static_cast<float*>(out) + idx) = make_float2(r0, r1);
    } else if (OUT == 2) {
      float2* q = reinterpret_cast<float2*>(static_cast<float*>(out) + idx);
      const float2 c = *q;
      *q = make_float2(c.x + r0, c.y + r1);
    } else {
      *reinterpret_cast<__nv_bfloat162*>(static_cast<__nv_bfloat16*>(out) + idx) =
          __floats2bfloat162_rn(r0, r1);
    }
  }
}

// ---------------------------------------------------------------------------
// Fused inverse z and y passes.  One CTA per (sample b, x-mode kx, group of
// DCG channels); the (ky, z) intermediate of the group stays in shared
// memory between the two passes:
//   in U [B][K][K][K][WD] -> out T1 [B][K][N][N][WD],
//   out[y][z] = sum_ky sum_kz G[y][ky] G[z][kz] in[ky][kz],  G: [N][K].
// ---------------------------------------------------------------------------
constexpr int DCG = 8;  // channels per CTA

template <int N, int K>
__global__ void __launch_bounds__(256)
fno_dft_zy_inv_kernel(const float2* in, float2* out, const float2* table) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* S1 = reinterpret_cast<float2*>(smem_raw);  // [K][K][DCG]
  float2* S2 = S1 + K * K * DCG;                      // [K][N][DCG]
  float2* tb = S2 + K * N * DCG;                      // [N][K]
  const int cg = blockIdx.x, kx = blockIdx.y, b = blockIdx.z, t = threadIdx.x;
  for (int i = t; i < N * K; i += 256) tb[i] = table[i];
  const long ibase = ((long)b * K + kx) * K * K * WD + cg * DCG;
  for (int e = t; e < K * K * DCG; e += 256) {
    const int c = e % DCG, kk = e / DCG;
    S1[e] = in[ibase + (long)kk * WD + c];
  }
  __syncthreads();
  // z expand: thread per (ky, c)
  for (int w = t; w < K * DCG; w += 256) {
    const int ky = w / DCG, c = w % DCG;
    float2 x[K];
#pragma unroll
    for (int kz = 0; kz < K; ++kz) x[kz] = S1[(ky * K + kz) * DCG + c];
#pragma unroll 4
    for (int z = 0; z < N; ++z) {
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int kz = 0; kz < K; ++kz) {
        const float2 g = tb[z * K + kz];
        re += g.x * x[kz].x - g.y * x[kz].y;
        im += g.x * x[kz].y + g.y * x[kz].x;
      }
      S2[(ky * N + z) * DCG + c] = make_float2(re, im);
    }
  }
  __syncthreads();
  // y expand: thread per (z, c)
  const long obase = ((long)b * K + kx) * N * N * WD + cg * DCG;
  for (int w = t; w < N * DCG; w += 256) {
    const int z = w / DCG, c = w % DCG;
    float2 x[K];
#pragma unroll
    for (int ky = 0; ky < K; ++ky) x[ky] = S2[(ky * N + z) * DCG + c];
#pragma unroll 4
    for (int y = 0; y < N; ++y) {
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int ky = 0; ky < K; ++ky) {
        const float2 g = tb[y * K + ky];
        re += g.x * x[ky].x - g.y * x[ky].y;
        im += g.x * x[ky].y + g.y * x[ky].x;
      }
      out[obase + ((long)y * N + z) * WD + c] = make_float2(re, im);
    }
  }
}

// ---------------------------------------------------------------------------
// Per-mode channel mixing, one CTA per mode m, block (32, 8).
//   MODE 0 (forward):      out[b][i'] = sum_i in[b][i] W[i][i']
//   MODE 1 (data grad):    out[b][i]  = sum_o g[b][o] conj(W[i][o])
//   MODE 2 (weight grad):  gW[i][o]   = sum_b conj(V[b][i]) g[b][o]
// W: BF16 complex [K^3][WD][WD] (re, im interleaved); in/out [B][K^3][WD].
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(256)
fno_mix_kernel(const float2* in, const float2* in2, const __nv_bfloat16* W,
               float2* out, float* gW, int B, int nm) {
  __shared__ float2 ws[WD * WD];
  __shared__ float2 xs[32 * WD];   // up to 32 samples
  __shared__ float2 gs[32 * WD];
  const int m = blockIdx.x, tx = threadIdx.x, ty = threadIdx.y;
  const int t = ty * 32 + tx;
  if (MODE != 2) {
    const __nv_bfloat162* wm =
        reinterpret_cast<const __nv_bfloat162*>(W) + (long)m * WD * WD;
    for (int i = t; i < WD * WD; i += 256) ws[i] = __bfloat1622float2(wm[i]);
  }
  for (int i = t; i < B * WD; i += 256) {
    const int b = i / WD, c = i % WD;
    xs[i] = in[((long)b * nm + m) * WD + c];
    if (MODE == 2) gs[i] = in2[((long)b * nm + m) * WD + c];
  }
  __syncthreads();
  if (MODE == 0 || MODE == 1) {
    for (int b = ty; b < B; b += 8) {
      float re = 0.f, im = 0.f;
#pragma unroll 8
      for (int i = 0; i < WD; ++i) {
        const float2 x = xs[b * WD + i];
        if (MODE == 0) {
          const float2 w = ws[i * WD + tx];
          re += x.x * w.x - x.y * w.y;
          im += x.x * w.y + x.y * w.x;
        } else {
          const float2 w = ws[tx * WD + i];  // conj(W[tx][i])
          re += x.x * w.x + x.y * w.y;
          im += x.y * w.x - x.x * w.y;
        }
      }
      out[((long)b * nm + m) * WD + tx] = make_float2(re, im);
    }
  } else {
    for (int i = ty; i < WD; i += 8) {
      float re = 0.f, im = 0.f;
      for (int b = 0; b < B; ++b) {
        const float2 v = xs[b * WD + i], g = gs[b * WD + tx];
        re += v.x * g.x + v.y * g.y;
        im += v.x * g.y - v.y * g.x;
      }
      float* o = gW + 2 * (((long)m * WD + i) * WD + tx);
      o[0] = re;
      o[1] = im;
    }
  }
}

// ---------------------------------------------------------------------------
// Dense layer, forward: y = x D + d + U; v = GELU(y) (or y for the last layer).
// One thread per point; D staged in shared memory (FP32).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
fno_dense_fwd_kernel(const __nv_bfloat16* x, const __nv_bfloat16* w16, long offD,
                     long offd, const __nv_bfloat16* U, __nv_bfloat16* y,
                     __nv_bfloat16* v, long R, int act) {
  __shared__ float Ds[WD * WD + WD];
  for (int i = threadIdx.x; i < WD * WD; i += blockDim.x) Ds[i] = bf(w16[offD + i]);
  for (int i = threadIdx.x; i < WD; i += blockDim.x) Ds[WD * WD + i] = bf(w16[offd + i]);
  __syncthreads();
  const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  float xi[WD];
  const uint4* xp = reinterpret_cast<const uint4*>(x + r * WD);
#pragma unroll
  for (int q = 0; q < WD / 8; ++q) {
    const uint4 u = xp[q];
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 f = __bfloat1622float2(h[k]);
      xi[q * 8 + 2 * k] = f.x;
      xi[q * 8 + 2 * k + 1] = f.y;
    }
  }
  const __nv_bfloat16* Ur = U + r * WD;
#pragma unroll 4
  for (int o = 0; o < WD; o += 2) {
    float a0 = Ds[WD * WD + o] + bf(Ur[o]), a1 = Ds[WD * WD + o + 1] + bf(Ur[o + 1]);
#pragma unroll
    for (int i = 0; i < WD; ++i) {
      a0 += xi[i] * Ds[i * WD + o];
      a1 += xi[i] * Ds[i * WD + o + 1];
    }
    const __nv_bfloat162 yy = __floats2bfloat162_rn(a0, a1);
    *reinterpret_cast<__nv_bfloat162*>(y + r * WD + o) = yy;
    const float2 yf = __bfloat1622float2(yy);
    *reinterpret_cast<__nv_bfloat162*>(v + r * WD + o) =
        act ? __floats2bfloat162_rn(gelu(yf.x), gelu(yf.y)) : yy;
  }
}

// Dense layer, data gradient: dx = dy D^T (FP32 in/out).
__global__ void __launch_bounds__(256)
fno_dense_bwd_kernel(const float* dy, const __nv_bfloat16* w16, long offD,
                     float* dx, long R) {
  __shared__ float Ds[WD * WD];
  for (int i = threadIdx.x; i < WD * WD; i += blockDim.x) Ds[i] = bf(w16[offD + i]);
  __syncthreads();
  const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  float g[WD];
  const float4* gp = reinterpret_cast<const float4*>(dy + r * WD);
#pragma unroll
  for (int q = 0; q < WD / 4; ++q) {
    const float4 u = gp[q];
    g[4 * q] = u.x; g[4 * q + 1] = u.y; g[4 * q + 2] = u.z; g[4 * q + 3] = u.w;
  }
  float4* op = reinterpret_cast<float4*>(dx + r * WD);
#pragma unroll 2
  for (int i = 0; i < WD; i += 4) {
    float a[4] = {0, 0, 0, 0};
#pragma unroll
    for (int o = 0; o < WD; ++o) {
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] += g[o] * Ds[(i + k) * WD + o];
    }
    op[i / 4] = make_float4(a[0], a[1], a[2], a[3]);
  }
}

// dy = dv * GELU'(y)
__global__ void fno_gelu_bwd_kernel(const float* dv, const __nv_bfloat16* y,
                                    float* dy, long total) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) dy[i] = dv[i] * gelu_d(bf(y[i]));
}

// ---------------------------------------------------------------------------
// Projection, forward: out = sum_j q2[j] GELU(x Q1[:, j] + q1[j]) + q2b.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
fno_proj_fwd_kernel(const __nv_bfloat16* x, const __nv_bfloat16* w16, Layout L,
                    float* out, long R) {
  __shared__ float Qs[WD * PJ + 3 * PJ + 1];
  for (int i = threadIdx.x; i < WD * PJ; i += blockDim.x) Qs[i] = bf(w16[L.Q1 + i]);
  for (int i = threadIdx.x; i < PJ; i += blockDim.x) {
    Qs[WD * PJ + i] = bf(w16[L.q1 + i]);
    Qs[WD * PJ + PJ + i] = bf(w16[L.q2 + i]);
  }
  if (threadIdx.x == 0) Qs[WD * PJ + 2 * PJ] = bf(w16[L.q2b]);
  __syncthreads();
  const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  float xi[WD];
  const uint4* xp = reinterpret_cast<const uint4*>(x + r * WD);
#pragma unroll
  for (int q = 0; q < WD / 8; ++q) {
    const uint4 u = xp[q];
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 f = __bfloat1622float2(h[k]);
      xi[q * 8 + 2 * k] = f.x;
      xi[q * 8 + 2 * k + 1] = f.y;
    }
  }
  float acc = Qs[WD * PJ + 2 * PJ];
#pragma unroll 2
  for (int j = 0; j < PJ; ++j) {
    float z = Qs[WD * PJ + j];
#pragma unroll
    for (int i = 0; i < WD; ++i) z += xi[i] * Qs[i * PJ + j];
    acc += Qs[WD * PJ + PJ + j] * gelu(z);
  }
  out[r] = acc;
}

// Projection, backward: dz = dout q2 GELU'(z), aw = dout GELU(z) (for dq2),
// dx = dz Q1^T.
__global__ void __launch_bounds__(256)
fno_proj_bwd_kernel(const __nv_bfloat16* x, const __nv_bfloat16* w16, Layout L,
                    const float* dout, float* dz, float* aw, float* dx, long R) {
  __shared__ float Qs[WD * PJ + 2 * PJ];
  for (int i = threadIdx.x; i < WD * PJ; i += blockDim.x) Qs[i] = bf(w16[L.Q1 + i]);
  for (int i = threadIdx.x; i < PJ; i += blockDim.x) {
    Qs[WD * PJ + i] = bf(w16[L.q1 + i]);
    Qs[WD * PJ + PJ + i] = bf(w16[L.q2 + i]);
  }
  __syncthreads();
  const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  float xi[WD], gx[WD];
  const uint4* xp = reinterpret_cast<const uint4*>(x + r * WD);
#pragma unroll
  for (int q = 0; q < WD / 8; ++q) {
    const uint4 u = xp[q];
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 f = __bfloat1622float2(h[k]);
      xi[q * 8 + 2 * k] = f.x;
      xi[q * 8 + 2 * k + 1] = f.y;
    }
  }
#pragma unroll
  for (int i = 0; i < WD; ++i) gx[i] = 0.f;
  const float go = dout[r];
#pragma unroll 2
  for (int j = 0; j < PJ; ++j) {
    float z = Qs[WD * PJ + j];
#pragma unroll
    for (int i = 0; i < WD; ++i) z += xi[i] * Qs[i * PJ + j];
    const float g = go * Qs[WD * PJ + PJ + j] * gelu_d(z);
    dz[r * PJ + j] = g;
    aw[r * PJ + j] = go * gelu(z);
#pragma unroll
    for (int i = 0; i < WD; ++i) gx[i] += g * Qs[i * PJ + j];
  }
  float4* op = reinterpret_cast<float4*>(dx + r * WD);
#pragma unroll
  for (int i = 0; i < WD; i += 4) op[i / 4] = make_float4(gx[i], gx[i + 1], gx[i + 2], gx[i + 3]);
}

// ---------------------------------------------------------------------------
// Weight gradient G[i][j] = sum_r A[r][i] Bm[r][j] (A: BF16 [R][KA], Bm: FP32
// [R][KB]).  Persistent CTAs over 64-row tiles; thread owns an RI x 4 block;
// per-CTA partials [gridDim][KA][KB], summed by fno_reduce_kernel in a fixed
// order (deterministic).
// ---------------------------------------------------------------------------
template <int KA, int KB>
__global__ void fno_wgrad_kernel(const __nv_bfloat16* A, const float* Bm, long R,
                                 float* partial) {
  constexpr int RI = KA < 4 ? KA : 4;
  constexpr int NTH = (KA / RI) * (KB / 4);
  constexpr int TR = 64;
  __shared__ __align__(16) float As[TR * KA];
  __shared__ __align__(16) float Bs[TR * KB];
  const int t = threadIdx.x;
  const int i0 = (t / (KB / 4)) * RI, j0 = (t % (KB / 4)) * 4;
  float acc[RI][4];
#pragma unroll
  for (int a = 0; a < RI; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = 0.f;
  for (long r0 = (long)blockIdx.x * TR; r0 < R; r0 += (long)gridDim.x * TR) {
    const int nr = (int)min((long)TR, R - r0);
    __syncthreads();
    for (int k = t; k < TR * KA; k += NTH)
      As[k] = (k / KA < nr) ? bf(A[r0 * KA + k]) : 0.f;
    for (int k = t; k < TR * KB; k += NTH)
      Bs[k] = (k / KB < nr) ? Bm[r0 * KB + k] : 0.f;
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < TR; ++r) {
      float av[RI];
#pragma unroll
      for (int a = 0; a < RI; ++a) av[a] = As[r * KA + i0 + a];
      const float4 bv = *reinterpret_cast<const float4*>(&Bs[r * KB + j0]);
#pragma unroll
      for (int a = 0; a < RI; ++a) {
        acc[a][0] += av[a] * bv.x; acc[a][1] += av[a] * bv.y;
        acc[a][2] += av[a] * bv.z; acc[a][3] += av[a] * bv.w;
      }
    }
  }
  float* P = partial + (long)blockIdx.x * KA * KB;
#pragma unroll
  for (int a = 0; a < RI; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) P[(i0 + a) * KB + j0 + c] = acc[a][c];
}

// Column sums S[j] = sum_r Bm[r][j] (bias gradients); partials per CTA.
template <int KB>
__global__ void __launch_bounds__(256)
fno_colsum_kernel(const float* Bm, long R, float* partial) {
  constexpr int RPT = 256 / KB;  // rows per pass
  __shared__ float red[256];
  const int t = threadIdx.x, j = t % KB, rr = t / KB;
  float s = 0.f;
  for (long r = (long)blockIdx.x * RPT + rr; r < R; r += (long)gridDim.x * RPT)
    s += Bm[r * KB + j];
  red[t] = s;
  __syncthreads();
  if (t < KB) {
    float v = 0.f;
    for (int k = 0; k < RPT; ++k) v += red[k * KB + t];
    partial[(long)blockIdx.x * KB + t] = v;
  }
}

// out[i] = sum_g partial[g][i] (fixed order)
__global__ void fno_reduce_kernel(const float* partial, int G, int n, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int g = 0; g < G; ++g) s += partial[(long)g * n + i];
  out[i] = s;
}

// ---------------------------------------------------------------------------
// Output: Q[dst] += P(rho^2 sigma sQ out) with the FP64 conservation projection P
// (5 moments, Gram inverse Ginv).  One CTA per sample.
// ---------------------------------------------------------------------------
struct OutArgs {
  const float* out; const double* qs; double sQ;
  const double* c0; double cw; int N; double Ginv[25];
  void* Q; int q_double; const int32_t* dst_slots; int dst_base;
  double* part;  // scratch [B][FCH][6]
};

// Two grid-wide passes, grid (FCH chunks, B samples): partial moments of the
// raw output (FP64), then every CTA reduces them in a fixed order, forms the
// multipliers and writes its chunk.
template <int PASS>
__global__ void __launch_bounds__(256) fno_output_kernel(OutArgs a) {
  __shared__ double red[8 + 5 * 8];
  __shared__ double lam_s[5];
  const int ch = blockIdx.x, b = blockIdx.y, t = threadIdx.x, N = a.N;
  const long n = (long)N * N * N, len = n / FCH, i0 = ch * len;
  const double sc = a.qs[b] * a.sQ;
  const float* o = a.out + (long)b * n;
  if (PASS == 0) {
    double s[5] = {0, 0, 0, 0, 0};
    for (long i = i0 + t; i < i0 + len; i += 256) {
      const int x = (int)(i / (N * N)), y = (int)((i / N) % N), z = (int)(i % N);
      const double q = sc * o[i] * a.cw;
      const double cx = a.c0[x], cy = a.c0[y], cz = a.c0[z];
      s[0] += q; s[1] += q * cx; s[2] += q * cy; s[3] += q * cz;
      s[4] += q * (cx * cx + cy * cy + cz * cz);
    }
    block_sum5<256>(s, red);
    if (t < 5) a.part[((long)b * FCH + ch) * 6 + t] = red[t];
    return;
  }
  if (t < 32) {
    double m[6];
    reduce_parts(a.part + (long)b * FCH * 6, m);
    if (t < 5) {
      double l = 0;
#pragma unroll
      for (int k = 0; k < 5; ++k) l += a.Ginv[t * 5 + k] * m[k];
      lam_s[t] = l;
    }
  }
  __syncthreads();
  const double l0 = lam_s[0], l1 = lam_s[1], l2 = lam_s[2], l3 = lam_s[3],
               l4 = lam_s[4];
  const long qb = (long)(a.dst_slots ? a.dst_slots[b] : a.dst_base + b) * n;
  for (long i = i0 + t; i < i0 + len; i += 256) {
    const int x = (int)(i / (N * N)), y = (int)((i / N) % N), z = (int)(i % N);
    const double cx = a.c0[x], cy = a.c0[y], cz = a.c0[z];
    const double q = sc * o[i] - (l0 + l1 * cx + l2 * cy + l3 * cz +
                                  l4 * (cx * cx + cy * cy + cz * cz));
    if (a.q_double) static_cast<double*>(a.Q)[qb + i] += q;
    else static_cast<float*>(a.Q)[qb + i] += (float)q;
  }
}

// ---------------------------------------------------------------------------
// Loss: per sample, t = Q/(rho^2 sigma sQ); L_b = |out - t|^2 / |t|^2;
// dout = (2/B) (out - t)/|t|^2.  One CTA per sample.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT)
fno_loss_kernel(const float* out, const double* Qt, const double* qs, double sQ,
                long n, int B, float* dout, double* loss) {
  __shared__ double red[8 + 5 * (NT / 32)];
  const int b = blockIdx.x, t = threadIdx.x;
  const double isc = 1.0 / (qs[b] * sQ);
  const float* o = out + (long)b * n;
  const double* q = Qt + (long)b * n;
  double s[5] = {0, 0, 0, 0, 0};
  for (long i = t; i < n; i += NT) {
    const double tv = q[i] * isc, e = (double)o[i] - tv;
    s[0] += e * e;
    s[1] += tv * tv;
  }
  block_sum5<NT>(s, red);
  const double tn = red[1] > 0 ? red[1] : 1.0;
  if (t == 0) loss[b] = red[0] / tn;
  const double g = 2.0 / (B * tn);
  for (long i = t; i < n; i += NT) {
    const double tv = q[i] * isc;
    dout[(long)b * n + i] = (float)(g * ((double)o[i] - tv));
  }
}

// ---------------------------------------------------------------------------
// Dense layers on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// One CTA (4 warps) computes 128-row tiles of D[128 x NC] = A[128 x 32] B,
// A = BF16 activations (row-major [R][32], i.e. K-major), B = BF16 weights
// W[32][NC] staged once per CTA as B^T (K-major).  Operands sit in shared
// memory in the canonical no-swizzle K-major layout: 8x8 core matrices of
// 128 contiguous bytes, core (row group g, K chunk c) at (g*4 + c)*128, so the
// leading-dimension offset (next K chunk) is 128 B and the stride-dimension
// offset (next 8 rows) 512 B.  One elected thread issues two
// tcgen05.mma.kind::f16 (K = 16 each) into a TMEM accumulator (FP32, NC
// columns, lane = row), commits to an mbarrier, and every thread reads its
// row back with tcgen05.ld for the fused epilogue:
//   EPI 0 (dense):      y = D + d + U;  v = GELU(y) (act) or y;  y stored if asked
//   EPI 1 (projection): out = sum_j q2[j] GELU(D_j + q1[j]) + q2b
// The mbarrier wait is bounded: on timeout the CTA records an error code
// and stops issuing work (still freeing its TMEM).
// ---------------------------------------------------------------------------
struct TcArgs {
  const __nv_bfloat16* x;   // [R][32]
  const __nv_bfloat16* w16; // parameters (BF16)
  long offW, offb;          // weight [32][NC], bias [NC]
  long offq2, offq2b;       // projection only
  const __nv_bfloat16* U;   // dense: [R][32] spectral part (BF16)
  __nv_bfloat16* y;         // dense: pre-activation out (may be null)
  __nv_bfloat16* v;         // dense: activation out
  float* out;               // projection: [R]
  long R;
  int act;
  int* err;
};

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}

template <int NC, int EPI>
__global__ void __launch_bounds__(128) fno_tc_kernel(TcArgs a) {
  static_assert(NC == 32 || NC == 128, "NC");
  __shared__ __align__(1024) uint8_t sA[128 * 64];
  __shared__ __align__(1024) uint8_t sB[NC * 64];
  __shared__ float ep[3 * NC + 1];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int abort_flag;
  const int t = threadIdx.x, warp = t >> 5;
  // weights as B^T [NC][32] in core-matrix layout; epilogue vectors
  for (int e = t; e < NC * WD; e += 128) {
    const int j = e / WD, k = e % WD;
    const __nv_bfloat16 w = a.w16[a.offW + (long)k * NC + j];
    *reinterpret_cast<__nv_bfloat16*>(
        sB + ((j >> 3) * 4 + (k >> 3)) * 128 + (j & 7) * 16 + (k & 7) * 2) = w;
  }
  for (int j = t; j < NC; j += 128) {
    ep[j] = bf(a.w16[a.offb + j]);
    if (EPI == 1) ep[NC + j] = bf(a.w16[a.offq2 + j]);
  }
  if (EPI == 1 && t == 0) ep[2 * NC] = bf(a.w16[a.offq2b]);
  if (t == 0) {
    abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc_smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(tc_smem_u32(&tslot)), "r"(NC));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tslot;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                         ((uint32_t)(NC >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  const uint32_t aS = tc_smem_u32(sA), bS = tc_smem_u32(sB);
  const uint32_t mb = tc_smem_u32(&mbar);
  const long ntiles = (a.R + 127) / 128;
  uint32_t phase = 0;
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long row = tile * 128 + t;
    // A row -> 4 core-matrix rows of 16 B
    uint4 q[4] = {};
    if (row < a.R) {
      const uint4* src = reinterpret_cast<const uint4*>(a.x + row * WD);
#pragma unroll
      for (int c = 0; c < 4; ++c) q[c] = src[c];
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
      *reinterpret_cast<uint4*>(sA + ((t >> 3) * 4 + c) * 128 + (t & 7) * 16) = q[c];
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        const uint64_t ad = tc_desc(aS + s2 * 256), bd = tc_desc(bS + s2 * 256);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(s2), "r"(0u), "r"(0u),
              "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                   ::"r"(mb) : "memory");
    }
    // bounded wait for the MMA's completion
    {
      uint32_t done = 0;
      for (int it = 0; it < (1 << 22) && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done) : "r"(mb), "r"(phase) : "memory");
      }
      if (!done) abort_flag = 1;
    }
    phase ^= 1u;
    __syncthreads();
    if (abort_flag) {
      if (t == 0) atomicExch(a.err, 1);
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    if (EPI == 0) {
      uint32_t r[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, "
          "%8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, "
          "%23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
            "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
            "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
            "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
            "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]),
            "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
          : "r"(lane_addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (row < a.R) {
        const uint4* Ur = reinterpret_cast<const uint4*>(a.U + row * WD);
        uint4 ub[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) ub[c] = Ur[c];
        uint4 yo[4], vo[4];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const __nv_bfloat162* u2 = reinterpret_cast<const __nv_bfloat162*>(&ub[c >> 1]) + (c & 1) * 2;
          const float2 ua = __bfloat1622float2(u2[0]), ub2 = __bfloat1622float2(u2[1]);
          const float4 u = make_float4(ua.x, ua.y, ub2.x, ub2.y);
          const float y0 = __uint_as_float(r[4 * c]) + ep[4 * c] + u.x;
          const float y1 = __uint_as_float(r[4 * c + 1]) + ep[4 * c + 1] + u.y;
          const float y2 = __uint_as_float(r[4 * c + 2]) + ep[4 * c + 2] + u.z;
          const float y3 = __uint_as_float(r[4 * c + 3]) + ep[4 * c + 3] + u.w;
          const __nv_bfloat162 ya = __floats2bfloat162_rn(y0, y1);
          const __nv_bfloat162 yb = __floats2bfloat162_rn(y2, y3);
          __nv_bfloat162 va = ya, vb = yb;
          if (a.act) {
            const float2 fa = __bfloat1622float2(ya), fb = __bfloat1622float2(yb);
            va = __floats2bfloat162_rn(gelu(fa.x), gelu(fa.y));
            vb = __floats2bfloat162_rn(gelu(fb.x), gelu(fb.y));
          }
          reinterpret_cast<__nv_bfloat162*>(&yo[c >> 1])[(c & 1) * 2] = ya;
          reinterpret_cast<__nv_bfloat162*>(&yo[c >> 1])[(c & 1) * 2 + 1] = yb;
          reinterpret_cast<__nv_bfloat162*>(&vo[c >> 1])[(c & 1) * 2] = va;
          reinterpret_cast<__nv_bfloat162*>(&vo[c >> 1])[(c & 1) * 2 + 1] = vb;
        }
        uint4* vd = reinterpret_cast<uint4*>(a.v + row * WD);
#pragma unroll
        for (int c = 0; c < 4; ++c) vd[c] = vo[c];
        if (a.y) {
          uint4* yd = reinterpret_cast<uint4*>(a.y + row * WD);
#pragma unroll
          for (int c = 0; c < 4; ++c) yd[c] = yo[c];
        }
      }
    } else {
      float o = ep[2 * NC];
#pragma unroll 1
      for (int cc = 0; cc < NC / 32; ++cc) {
        uint32_t r[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, "
            "%8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, "
            "%23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
              "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]),
              "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(lane_addr + (uint32_t)(cc * 32)));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int jj = cc * 32 + j;
          o += ep[NC + jj] * gelu(__uint_as_float(r[j]) + ep[jj]);
        }
      }
      if (row < a.R) a.out[row] = o;
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n"
                 ::"r"(tmem), "r"(NC));
}

// ---------------------------------------------------------------------------
// Evaluation path with fused spectral passes (inference; training keeps the
// per-axis passes above, whose intermediates its backward pass reuses).
// With Y[b][x][ky][kz][c] = the yz spectra of v_l (complex FP32):
//   fno_xmix_kernel        one CTA per (ky, kz): FFT over x, keep K modes, mix
//                          with W_l, inverse FFT over x (1/N)
//                          -> S[b][x][ky][kz][c]
//   fno_yzinv_dense_kernel one CTA per z-slab of a (b, x) plane: U = Re IDFT_yz(S) (BF16),
//                          y_l = v_l D_l + d_l + U on tcgen05,
//                          v_{l+1} = GELU(y_l) (or y_l for the last layer)
//   fno_yzfwd_kernel       one CTA per plane: Y = DFT_yz(v_{l+1})
// Every truncated transform is a zero-padded N-point register FFT (modes
// k = 0..K/2-1 sit in bins 0..K/2-1, k = -K/2..-1 in bins N-K/2..N-1); two
// real pencils share one complex FFT.  Same values as the per-axis DFT passes
// up to FP32 rounding; U, y_l and v_{l+1} are rounded to BF16 at the same
// points.
// ---------------------------------------------------------------------------
template <int N, int K>
__host__ __device__ constexpr int fbin(int kk) {
  return kk < K / 2 ? kk : N - K + kk;
}


// Grid (K*K, ceil(B / K)): blockIdx.x = ky K + kz, blockIdx.y = chunk of K
// samples (one per warp in the transforms; thread (kx, o) in the mix).  Two
// CTAs share an SM, so one's loads overlap the other's transforms; the W
// column is loaded after the forward transforms so that the two register sets
// are not live together.
template <int N, int K>
__global__ void __launch_bounds__(K * 32)
fno_xmix_kernel(const float2* __restrict__ Y, const __nv_bfloat16* __restrict__ W,
                float2* __restrict__ S, int B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* Vs = reinterpret_cast<float2*>(smem_raw);  // [K samples][K][WD]
  float2* Us = Vs + K * K * WD;                       // [K samples][K][WD]
  const int kyz = blockIdx.x, ky = kyz / K, kz = kyz % K;
  const int b0 = blockIdx.y * K, nb = min(K, B - b0);
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const long xs = (long)K * K * WD;  // stride between x planes
  if (w < nb) {  // forward FFT over x, one warp per sample, lane = channel
    const float2* src = Y + ((long)(b0 + w) * N * K * K + kyz) * WD + lane;
    float2 v[N];
#pragma unroll
    for (int x = 0; x < N; ++x) v[x] = src[x * xs];
    fft<float, N, -1>(v);
#pragma unroll
    for (int kk = 0; kk < K; ++kk) Vs[(w * K + kk) * WD + lane] = v[fbin<N, K>(kk)];
  }
  __syncthreads();
  {  // mix: thread (kx = w, o = lane) with the column W[m][.][o] in registers,
     // m = (kx K + ky) K + kz
    float2 wc[WD];
    const long m = ((long)w * K + ky) * K + kz;
    const __nv_bfloat162* wm = reinterpret_cast<const __nv_bfloat162*>(W) + m * WD * WD;
#pragma unroll
    for (int i = 0; i < WD; ++i) wc[i] = __bfloat1622float2(wm[i * WD + lane]);
    // two samples per pass, two input channels per 16-byte load (the second
    // sample's row stays inside Vs when nb is odd: s + 1 < K)
    for (int s = 0; s < nb; s += 2) {
      const float4* v0 = reinterpret_cast<const float4*>(Vs + (s * K + w) * WD);
      const float4* v1 = reinterpret_cast<const float4*>(Vs + ((s + 1) * K + w) * WD);
      float r0 = 0.f, i0 = 0.f, r1 = 0.f, i1 = 0.f;
#pragma unroll
      for (int q = 0; q < WD / 2; ++q) {
        const float4 a = v0[q], c = v1[q];
        const float2 wa = wc[2 * q], wb = wc[2 * q + 1];
        r0 = fmaf(a.x, wa.x, r0); r0 = fmaf(-a.y, wa.y, r0);
        i0 = fmaf(a.x, wa.y, i0); i0 = fmaf(a.y, wa.x, i0);
        r0 = fmaf(a.z, wb.x, r0); r0 = fmaf(-a.w, wb.y, r0);
        i0 = fmaf(a.z, wb.y, i0); i0 = fmaf(a.w, wb.x, i0);
        r1 = fmaf(c.x, wa.x, r1); r1 = fmaf(-c.y, wa.y, r1);
        i1 = fmaf(c.x, wa.y, i1); i1 = fmaf(c.y, wa.x, i1);
        r1 = fmaf(c.z, wb.x, r1); r1 = fmaf(-c.w, wb.y, r1);
        i1 = fmaf(c.z, wb.y, i1); i1 = fmaf(c.w, wb.x, i1);
      }
      Us[(s * K + w) * WD + lane] = make_float2(r0, i0);
      if (s + 1 < nb) Us[((s + 1) * K + w) * WD + lane] = make_float2(r1, i1);
    }
  }
  __syncthreads();
  if (w < nb) {  // inverse FFT over x
    float2 v[N];
#pragma unroll
    for (int j = 0; j < N; ++j) v[j] = make_float2(0.f, 0.f);
#pragma unroll
    for (int kk = 0; kk < K; ++kk) v[fbin<N, K>(kk)] = Us[(w * K + kk) * WD + lane];
    fft<float, N, +1>(v);
    float2* dst = S + ((long)(b0 + w) * N * K * K + kyz) * WD + lane;
    constexpr float inv = 1.f / N;
#pragma unroll
    for (int x = 0; x < N; ++x) dst[x * xs] = make_float2(v[x].x * inv, v[x].y * inv);
  }
}

// yz spectra of one (b, x) plane of a BF16 field [B][N][N][N][WD].
template <int N, int K>
__global__ void __launch_bounds__(256)
fno_yzfwd_kernel(const __nv_bfloat16* __restrict__ v, float2* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* T2 = reinterpret_cast<float2*>(smem_raw);  // [N y][K kz][WD]
  const int x = blockIdx.x, b = blockIdx.y, t = threadIdx.x;
  const long plane = (long)b * N + x;
  const __nv_bfloat16* vp = v + plane * N * N * WD;
  // z pass: pencil (y, channel pair cp); the two channels are the real and
  // imaginary parts of one FFT, separated by Hermitian symmetry
  for (int p = t; p < N * (WD / 2); p += 256) {
    const int y = p / (WD / 2), cp = p % (WD / 2);
    float2 c[N];
#pragma unroll
    for (int z = 0; z < N; ++z)
      c[z] = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(
          vp + ((long)y * N + z) * WD + 2 * cp));
    fft<float, N, -1>(c);
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
      const int k = fbin<N, K>(kk), nk = (N - k) % N;
      const float2 C = c[k], Cn = c[nk];
      // channel 2cp: (C + conj Cn)/2; channel 2cp+1: (C - conj Cn)/(2i)
      *reinterpret_cast<float4*>(T2 + (y * K + kk) * WD + 2 * cp) =
          make_float4(0.5f * (C.x + Cn.x), 0.5f * (C.y - Cn.y),
                      0.5f * (C.y + Cn.y), -0.5f * (C.x - Cn.x));
    }
  }
  __syncthreads();
  // y pass: pencil (kz, channel)
  for (int p = t; p < K * WD; p += 256) {
    const int kk = p / WD, ch = p % WD;
    float2 c[N];
#pragma unroll
    for (int y = 0; y < N; ++y) c[y] = T2[(y * K + kk) * WD + ch];
    fft<float, N, -1>(c);
    float2* dst = Y + (plane * K * K + kk) * WD + ch;
#pragma unroll
    for (int ky = 0; ky < K; ++ky) dst[(long)ky * K * WD] = c[fbin<N, K>(ky)];
  }
}

struct YzInvArgs {
  const float2* S;           // [B][N][K][K][WD]
  const __nv_bfloat16* v;    // v_l [B][N^3][WD]
  const __nv_bfloat16* w16;  // BF16 parameters
  long offD, offd;           // D_l [WD][WD], d_l [WD]
  __nv_bfloat16* vout;       // v_{l+1} [B][N^3][WD]
  int act;                   // GELU (layers 0..2) or identity (last layer)
  int* err;                  // device error flag
};

// One CTA of fno_yzinv_dense_kernel takes a z-slab of a (b, x) plane: all y
// and NZ = N/ZP consecutive z values; its rows (points) are r = y NZ + zl.
// Two slabs per plane keep the shared memory under half an SM, so two CTAs
// share an SM and one's loads overlap the other's transforms.
template <int N, int K>
struct YzInvGeo {
  static constexpr int ZP = 2;                    // z-slabs per plane
  static constexpr int NZ = N / ZP;               // z values per CTA
  static constexpr int ROWS = N * NZ;             // points per CTA
  static constexpr int TILES = ROWS / 128;        // 128-row MMA tiles
  static constexpr int NT = 256;                  // threads
  static constexpr int NCOL = TILES * WD;         // TMEM columns
  static constexpr int A_BYTES = ROWS * WD * 2;   // BF16 rows (then U)
  static constexpr int T_BYTES = K * NZ * WD * 8; // [K][NZ][WD] complex
  static constexpr int SMEM = A_BYTES + T_BYTES + WD * WD * 2 + WD * 4 + 64;
  static_assert(ROWS % 128 == 0, "slab must be whole 128-row tiles");
  static_assert(NCOL >= 32 && (NCOL & (NCOL - 1)) == 0, "TMEM allocation");
  static_assert(NT % 128 == 0, "epilogue warps cover the four TMEM lane quadrants");
};

// kz -> z inverse of one (ky, channel) pencil, keeping the slab's z values.
template <int N, int K, int Z0, int NZ>
__device__ __forceinline__ void yzinv_zpass(const float2* src, float2* T, int ky,
                                            int ch) {
  constexpr float inv = 1.f / N;
  float2 c[N];
#pragma unroll
  for (int j = 0; j < N; ++j) c[j] = make_float2(0.f, 0.f);
#pragma unroll
  for (int kz = 0; kz < K; ++kz) c[fbin<N, K>(kz)] = src[kz * WD];
  fft<float, N, +1>(c);
#pragma unroll
  for (int zl = 0; zl < NZ; ++zl)
    T[(ky * NZ + zl) * WD + ch] = make_float2(c[Z0 + zl].x * inv, c[Z0 + zl].y * inv);
}

// Grid (N ZP, B): blockIdx.x = x ZP + slab.  The rows' BF16 activations load
// asynchronously while the CUDA cores run the kz -> z pass; the dense MMAs
// are issued next, and U overwrites their A operand only after the MMA
// completion barrier; the epilogue adds U to the accumulator.
template <int N, int K>
__global__ void __launch_bounds__(YzInvGeo<N, K>::NT, 2)
fno_yzinv_dense_kernel(YzInvArgs a) {
  using G = YzInvGeo<N, K>;
  constexpr int NT = G::NT, NZ = G::NZ;
  // (the no-swizzle operand layout needs 16-byte alignment only)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint8_t* sA = smem_raw;
  __nv_bfloat16* Us = reinterpret_cast<__nv_bfloat16*>(smem_raw);  // [ROWS][WD]
  float2* T = reinterpret_cast<float2*>(smem_raw + G::A_BYTES);     // [K][NZ][WD]
  uint8_t* sB = smem_raw + G::A_BYTES + G::T_BYTES;
  float* ep = reinterpret_cast<float*>(sB + WD * WD * 2);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(ep + WD);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  int* abort_flag = reinterpret_cast<int*>(tslot + 1);
  const int x = blockIdx.x / G::ZP, zh = blockIdx.x % G::ZP, z0 = zh * NZ;
  const int b = blockIdx.y, t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const long plane = (long)b * N + x;
  // A operand: the slab's rows as 128-row tiles in the canonical no-swizzle
  // K-major layout (core (row group g, K chunk c) at g*512 + c*128)
  {
    const uint32_t a0 = tc_smem_u32(sA);
    const __nv_bfloat16* vp = a.v + plane * N * N * WD;
    for (int c = t; c < G::ROWS * 4; c += NT) {
      const int r = c >> 2, q = c & 3, tile = r >> 7, rr = r & 127;
      const int y = r / NZ, zl = r % NZ;
      cp_async16(a0 + (uint32_t)(tile * 8192 + ((rr >> 3) * 4 + q) * 128 + (rr & 7) * 16),
                 vp + ((long)y * N + z0 + zl) * WD + q * 8);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int e = t; e < WD * WD; e += NT) {  // D^T [o][i]
    const int j = e / WD, k = e % WD;
    *reinterpret_cast<__nv_bfloat16*>(sB + ((j >> 3) * 4 + (k >> 3)) * 128 +
                                      (j & 7) * 16 + (k & 7) * 2) =
        a.w16[a.offD + (long)k * WD + j];
  }
  if (t < WD) ep[t] = bf(a.w16[a.offd + t]);
  if (t == 0) {
    *abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc_smem_u32(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                 ::"r"(tc_smem_u32(tslot)), "r"(G::NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  // kz -> z: pencil (ky, channel), while the A operand loads
  for (int p = t; p < K * WD; p += NT) {
    const int ky = p / WD, ch = p % WD;
    const float2* src = a.S + (plane * K + ky) * K * WD + ch;
    if (zh == 0) yzinv_zpass<N, K, 0, NZ>(src, T, ky, ch);
    else yzinv_zpass<N, K, NZ, NZ>(src, T, ky, ch);
  }
  cp_async_wait_all();
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t mb = tc_smem_u32(mbar);
  if (t == 0) {
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) |
                           ((uint32_t)(WD >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    const uint32_t aS = tc_smem_u32(sA), bS = tc_smem_u32(sB);
    for (int tile = 0; tile < G::TILES; ++tile) {
#pragma unroll
      for (int s2 = 0; s2 < 2; ++s2) {
        const uint64_t ad = tc_desc(aS + tile * 8192 + s2 * 256);
        const uint64_t bd = tc_desc(bS + s2 * 256);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            ::"r"(tmem + (uint32_t)(tile * WD)), "l"(ad), "l"(bd), "r"(idesc), "r"(s2),
              "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                 ::"r"(mb) : "memory");
  }
  // the MMAs have read the A operand before U overwrites it (bounded wait)
  {
    uint32_t done = 0;
    for (int it = 0; it < (1 << 22) && !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t}\n"
          : "=r"(done) : "r"(mb), "r"(0u) : "memory");
    }
    if (!done) *abort_flag = 1;
  }
  __syncthreads();
  const bool ok = *abort_flag == 0;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  // ky -> y, real part: pencil (zl, channel pair); c = sym(a) + i sym(b) with
  // sym(a)(k) = (a(k) + conj a(-k))/2, so that IFFT(c) = Re IFFT(a) + i Re IFFT(b)
  if (ok) {
    constexpr float inv = 1.f / N;
    for (int p = t; p < NZ * (WD / 2); p += NT) {
      const int zl = p / (WD / 2), cp = p % (WD / 2);
      float2 c[N];
#pragma unroll
      for (int j = 0; j < N; ++j) c[j] = make_float2(0.f, 0.f);
#pragma unroll
      for (int ky = 0; ky < K; ++ky) {
        const float4 ab = *reinterpret_cast<const float4*>(T + (ky * NZ + zl) * WD + 2 * cp);
        const int k = fbin<N, K>(ky), nk = (N - k) % N;
        c[k].x += 0.5f * (ab.x - ab.w);
        c[k].y += 0.5f * (ab.y + ab.z);
        c[nk].x += 0.5f * (ab.x + ab.w);
        c[nk].y += 0.5f * (ab.z - ab.y);
      }
      fft<float, N, +1>(c);
#pragma unroll
      for (int y = 0; y < N; ++y)
        *reinterpret_cast<__nv_bfloat162*>(Us + (long)(y * NZ + zl) * WD + 2 * cp) =
            __floats2bfloat162_rn(c[y].x * inv, c[y].y * inv);
    }
  }
  __syncthreads();
  // epilogue: warp w reads TMEM lane quadrant w % 4 of tiles w/4, w/4 + NT/128, ...
  if (ok) {
    const int q = warp & 3;
    for (int tile = warp >> 2; tile < G::TILES; tile += NT / 128) {
      const int r = tile * 128 + q * 32 + lane;
      const long pt = (long)(r / NZ) * N + z0 + r % NZ;
      uint32_t rg[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, "
          "%8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, "
          "%23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
          : "=r"(rg[0]), "=r"(rg[1]), "=r"(rg[2]), "=r"(rg[3]), "=r"(rg[4]), "=r"(rg[5]),
            "=r"(rg[6]), "=r"(rg[7]), "=r"(rg[8]), "=r"(rg[9]), "=r"(rg[10]), "=r"(rg[11]),
            "=r"(rg[12]), "=r"(rg[13]), "=r"(rg[14]), "=r"(rg[15]), "=r"(rg[16]),
            "=r"(rg[17]), "=r"(rg[18]), "=r"(rg[19]), "=r"(rg[20]), "=r"(rg[21]),
            "=r"(rg[22]), "=r"(rg[23]), "=r"(rg[24]), "=r"(rg[25]), "=r"(rg[26]),
            "=r"(rg[27]), "=r"(rg[28]), "=r"(rg[29]), "=r"(rg[30]), "=r"(rg[31])
          : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(tile * WD)));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      const uint4* Ur = reinterpret_cast<const uint4*>(Us + (long)r * WD);
      uint4 vo[4];
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4) {
        const uint4 u = Ur[c4];
        const __nv_bfloat162* u2 = reinterpret_cast<const __nv_bfloat162*>(&u);
        __nv_bfloat162* o2 = reinterpret_cast<__nv_bfloat162*>(&vo[c4]);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const int j = c4 * 8 + 2 * h;
          const float2 uf = __bfloat1622float2(u2[h]);
          const __nv_bfloat162 yy = __floats2bfloat162_rn(
              __uint_as_float(rg[j]) + ep[j] + uf.x,
              __uint_as_float(rg[j + 1]) + ep[j + 1] + uf.y);
          if (a.act) {
            const float2 yf = __bfloat1622float2(yy);
            o2[h] = __floats2bfloat162_rn(gelu(yf.x), gelu(yf.y));
          } else {
            o2[h] = yy;
          }
        }
      }
      uint4* vd = reinterpret_cast<uint4*>(a.vout + (plane * N * N + pt) * WD);
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4) vd[c4] = vo[c4];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n"
                 ::"r"(tmem), "r"(G::NCOL));
  if (!ok && t == 0) atomicExch(a.err, 1);
}

// Adam on the FP32 master parameters; refreshes the BF16 copy.
__global__ void fno_adam_kernel(float* p, __nv_bfloat16* p16, const float* g,
                                float* m, float* v, long n, float lr, float b1,
                                float b2, float eps, float bc1, float bc2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  p[i] = pi;
  p16[i] = tobf(pi);
}

__global__ void fno_to_bf16_kernel(const float* p, __nv_bfloat16* p16, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p16[i] = tobf(p[i]);
}

}  // namespace fno
}  // namespace dgfs

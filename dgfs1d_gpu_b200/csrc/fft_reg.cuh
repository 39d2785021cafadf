// In-register fast Fourier transforms of short lengths (N = 2^a 3^b <= 64).
//
// One thread holds one pencil of N complex values in registers; every loop is
// unrolled at compile time so that all indices -- and therefore all twiddle
// factors -- are constants.  Twiddles live in __constant__ memory (filled from
// the host in double precision by dgfs_twiddle_upload) and are read as
// constant-bank operands; the trivial ones (1, -1, +-i) are folded away.
//
// Conventions follow cuFFT: SIGN = -1 is CUFFT_FORWARD (e^{-2 pi i jk/N}),
// SIGN = +1 is CUFFT_INVERSE (e^{+2 pi i jk/N}); neither is normalised.
#pragma once
#include <cuda_runtime.h>

namespace dgfs {

template <typename R> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename R> using c2_t = typename C2<R>::type;

template <typename T> __device__ __forceinline__ T cmul(T a, T b) {
  T r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename T> __device__ __forceinline__ T cadd(T a, T b) {
  T r; r.x = a.x + b.x; r.y = a.y + b.y; return r;
}
template <typename T> __device__ __forceinline__ T csub(T a, T b) {
  T r; r.x = a.x - b.x; r.y = a.y - b.y; return r;
}
// multiply by s*i (s = +-1)
template <int S, typename T> __device__ __forceinline__ T cmul_i(T a) {
  T r;
  if (S > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

// Twiddle tables: forward twiddles exp(-2 pi i k / NT) for each supported NT,
// concatenated.  Offsets are compile-time.
constexpr int kNumTw = 9;
__host__ __device__ constexpr int tw_size(int i) {
  return i == 0 ? 4 : i == 1 ? 6 : i == 2 ? 8 : i == 3 ? 12 : i == 4 ? 16
       : i == 5 ? 24 : i == 6 ? 32 : i == 7 ? 48 : 64;
}
__host__ __device__ constexpr int tw_offset(int nt) {
  int off = 0;
  for (int i = 0; i < kNumTw; ++i) {
    if (tw_size(i) == nt) return off;
    off += tw_size(i);
  }
  return -1;
}
constexpr int kTwTotal = tw_offset(64) + 64;

// Defined here: the library is a single translation unit.
__constant__ double2 c_tw64[kTwTotal];
__constant__ float2 c_tw32[kTwTotal];

template <typename R> struct TwTab;
template <> struct TwTab<double> {
  static __device__ __forceinline__ double2 get(int i) { return c_tw64[i]; }
};
template <> struct TwTab<float> {
  static __device__ __forceinline__ float2 get(int i) { return c_tw32[i]; }
};

// y * exp(SIGN * 2 pi i e / NT); e is a compile-time constant after unrolling.
template <typename R, int NT, int SIGN>
__device__ __forceinline__ c2_t<R> twiddle_mul(c2_t<R> y, int e) {
  e = ((e % NT) + NT) % NT;
  if (e == 0) return y;
  if (2 * e == NT) { y.x = -y.x; y.y = -y.y; return y; }
  if (4 * e == NT) return cmul_i<SIGN>(y);       // exp(SIGN i pi/2) = SIGN*i
  if (4 * e == 3 * NT) return cmul_i<-SIGN>(y);  // exp(SIGN 3i pi/2)
  constexpr int off = tw_offset(NT);
  static_assert(off >= 0, "no twiddle table for this length");
  c2_t<R> w = TwTab<R>::get(off + e);
  if (SIGN > 0) w.y = -w.y;
  return cmul(y, w);
}

template <int N> struct Radix {
  static constexpr int value = (N % 4 == 0 && N != 8) ? 4 : (N % 2 == 0 ? 2 : 3);
};
template <> struct Radix<8> { static constexpr int value = 8; };

// small DFT kernels on y[0..R)
template <typename T, int SIGN>
__device__ __forceinline__ void dft2(T* y) {
  T a = y[0], b = y[1];
  y[0] = cadd(a, b); y[1] = csub(a, b);
}
template <typename T, int SIGN>
__device__ __forceinline__ void dft4(T* y) {
  T t0 = cadd(y[0], y[2]), t1 = csub(y[0], y[2]);
  T t2 = cadd(y[1], y[3]), t3 = cmul_i<SIGN>(csub(y[1], y[3]));
  y[0] = cadd(t0, t2); y[2] = csub(t0, t2);
  y[1] = cadd(t1, t3); y[3] = csub(t1, t3);
}
template <typename R, int SIGN>
__device__ __forceinline__ void dft3(c2_t<R>* y) {
  using T = c2_t<R>;
  const R h = R(0.86602540378443864676);  // sqrt(3)/2
  T s = cadd(y[1], y[2]), d = csub(y[1], y[2]);
  T a = y[0];
  y[0] = cadd(a, s);
  T m; m.x = a.x - R(0.5) * s.x; m.y = a.y - R(0.5) * s.y;
  T di; di.x = h * d.x; di.y = h * d.y;
  di = cmul_i<SIGN>(di);
  y[1] = cadd(m, di); y[2] = csub(m, di);
}
template <typename R, int SIGN>
__device__ __forceinline__ void dft8(c2_t<R>* y) {
  using T = c2_t<R>;
  // radix-2 x radix-4 split: even/odd
  T e[4] = {y[0], y[2], y[4], y[6]};
  T o[4] = {y[1], y[3], y[5], y[7]};
  dft4<T, SIGN>(e);
  dft4<T, SIGN>(o);
  const R r2 = R(0.70710678118654752440);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    T w = o[k];
    if (k == 1) {  // exp(SIGN i pi/4) = (1 + SIGN i)/sqrt2
      T t; t.x = r2 * (w.x - SIGN * w.y); t.y = r2 * (w.y + SIGN * w.x); w = t;
    } else if (k == 2) {
      w = cmul_i<SIGN>(w);
    } else if (k == 3) {  // exp(SIGN 3i pi/4) = (-1 + SIGN i)/sqrt2
      T t; t.x = r2 * (-w.x - SIGN * w.y); t.y = r2 * (-w.y + SIGN * w.x); w = t;
    }
    y[k] = cadd(e[k], w);
    y[k + 4] = csub(e[k], w);
  }
}

// In-place DFT of x[OFF + k*STR], k in [0, N), twiddles from the NT table.
template <typename R, int N, int SIGN, int NT, int STR, int OFF>
struct RegFFT {
  static __device__ __forceinline__ void run(c2_t<R>* x) {
    using T = c2_t<R>;
    constexpr int RR = Radix<N>::value;
    constexpr int Q = N / RR;
    if constexpr (Q > 1) {
#pragma unroll
      for (int r = 0; r < RR; ++r) {
        // decimated sub-sequence x[OFF + (r + RR*m)*STR], m < Q
        switch (r) {
          case 0: RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 0 * STR>::run(x); break;
          case 1: RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 1 * STR>::run(x); break;
          case 2: if constexpr (RR > 2) RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 2 * STR>::run(x); break;
          case 3: if constexpr (RR > 3) RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 3 * STR>::run(x); break;
          case 4: if constexpr (RR > 4) RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 4 * STR>::run(x); break;
          case 5: if constexpr (RR > 5) RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 5 * STR>::run(x); break;
          case 6: if constexpr (RR > 6) RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 6 * STR>::run(x); break;
          case 7: if constexpr (RR > 7) RegFFT<R, Q, SIGN, NT, STR * RR, OFF + 7 * STR>::run(x); break;
        }
      }
    }
    T t[N];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      T y[RR];
#pragma unroll
      for (int r = 0; r < RR; ++r) {
        y[r] = x[OFF + (r + RR * k) * STR];
        y[r] = twiddle_mul<R, NT, SIGN>(y[r], r * k * (NT / N));
      }
      if constexpr (RR == 2) dft2<T, SIGN>(y);
      else if constexpr (RR == 3) dft3<R, SIGN>(y);
      else if constexpr (RR == 4) dft4<T, SIGN>(y);
      else dft8<R, SIGN>(y);
#pragma unroll
      for (int j = 0; j < RR; ++j) t[k + j * Q] = y[j];
    }
#pragma unroll
    for (int k = 0; k < N; ++k) x[OFF + k * STR] = t[k];
  }
};

// Convenience: full-length transform of a register array v[N].
template <typename R, int N, int SIGN>
__device__ __forceinline__ void fft(c2_t<R>* v) {
  RegFFT<R, N, SIGN, N, 1, 0>::run(v);
}

}  // namespace dgfs

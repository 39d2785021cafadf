// Nodal DG advection right-hand side, boundary conditions, stage updates
// (axnpby) and FP64 bulk moments of the single-species solver.
//
// Reference: the rhs() closure of dgfs1D/std/std.py:281-366 with the kernels
// of dgfs1D/std/kernels/std.mako (extract/transfer/insert, flux, mul_by_adv,
// totalFlux, mul_by_invjac), the diffuse-wall / inlet / periodic boundary
// kernels of dgfs1D/std/kernels/bcs/*.mako, axnpby of dgfs1D/axnpby.py:10-58
// and the moments of dgfs1D/std/moments.py:11-70.  The reference runs about
// fifteen small kernels and two host reductions per right-hand side; here
// one reduction kernel (wall densities) and one fused kernel produce it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dgfs {

constexpr int kDgMaxK = 8;

// boundary kinds
constexpr int kBcCopy = 0;     // dgfs-periodic / dgfs-cyclic on one rank: ghost = interior
constexpr int kBcWall = 1;     // dgfs-wall-diffuse
constexpr int kBcInlet = 2;    // dgfs-inlet, dgfs-inlet-nondim (incoming test (c_x - u_x) n)
constexpr int kBcVanish = 3;   // dgfs-vanish
constexpr int kBcWallExpr = 4; // dgfs-wall-expr-diffuse (wall state set per call)

struct DgAdvectArgs {
  const void* u;            // (K, Ne, Nv) in
  void* ux;                 // (K, Ne, Nv) out: advection + flux terms
  int f_double;
  int K, Ne, Nv, N;
  const double* c0;         // [N] velocity grid; c_x of v = c0[v / (N*N)]
  const double* invjac;     // [Ne]
  const double* f0[2];      // [Nv] boundary Maxwellians (left, right)
  const double* nden;       // [2] wall densities (from dg_wall_final_kernel)
  int bc[2];                // boundary kinds (left, right)
  double bc_ux[2];          // wall x-velocities
  double nl[2];             // outward normals (-1, +1)
  double ws[2][5];          // kBcWallExpr: ux, uy, uz, T, mass of the wall
  double trL[kDgMaxK];      // left-face trace weights  (row 0 of Bqf^T)
  double trR[kDgMaxK];      // right-face trace weights (row Nqf-1 of Bqf^T)
  double D[kDgMaxK * kDgMaxK];  // derivOp (K x K): ux = D u
  double gLD[kDgMaxK], gRD[kDgMaxK];
  // volume term: upwind = 0: -c_x D u; 1: upwind summation-by-parts
  // (dgfsABUstd1D), D applied where c_x > 0 and D2 where c_x < 0;
  // 2: entropy-stable two-point form (dgfsABE2std1D),
  // -2 c_x sum_l D[k][l] aveL(u_k, u_l) with the logarithmic mean aveL.
  // swap: the ghosts take the trace at the opposite end of the domain
  // (one-rank dgfs-cyclic right boundary of dgfsABUstd1D)
  double D2[kDgMaxK * kDgMaxK];
  int upwind;
  int swap;
};

// Logarithmic mean (a + b) / 2 / (log(xi) / (2 f)), xi = |a / b|,
// f = (xi - 1)/(xi + 1), with the series 1 + u/3 + u^2/5 + u^3/7 (u = f^2)
// for u < 1e-2 and the 1e-20 guards of aveL in astd/kernels/limiters.mako:163-170.
__device__ __forceinline__ double log_mean(double a, double b) {
  const double xi = fabs(a / (b + 1e-20));
  const double f = (xi - 1) / (xi + 1);
  const double u = f * f;
  return 0.5 * (a + b) /
         (u < 1e-2 ? (1 + u / 3 + u * u / 5 + u * u * u / 7)
                   : log(xi + 1e-20) / 2. / (f + 1e-20));
}

__device__ __forceinline__ double ld(const void* p, int dbl, size_t i) {
  return dbl ? static_cast<const double*>(p)[i]
             : (double)static_cast<const float*>(p)[i];
}
__device__ __forceinline__ void st(void* p, int dbl, size_t i, double v) {
  if (dbl) static_cast<double*>(p)[i] = v;
  else static_cast<float*>(p)[i] = (float)v;
}

// Linear slope limiter of dgfsABstd1D (``[time-integrator] limiter = 1``,
// abstd.py:403-415 with limitLin of astd/kernels/limiters.mako:17-76), in
// place, one thread per velocity point walking the interior elements.  The
// cell averages (row 0 of the cell-average operator) and the linear slopes
// (row 0 of the differentiated linear projection, times invjac) come from the
// unlimited solution: a window of three averages is formed before an element
// is written.  An element is limited when its end values differ from the
// minmod-limited linear reconstruction by more than tol; it then becomes
// avg + dx_k minmod(slope, (avg_R - avg)/h, (avg - avg_L)/h).
struct DgLimitArgs {
  void* u;
  int f_double;
  int K, Ne, Nv;
  const double* wavg;   // [K]
  const double* wdr;    // [K]
  const double* invjac; // [Ne]
  const double* dx;     // [K][Ne] node position minus element centre
  const double* h;      // [Ne] element length
  double tol;
};

__device__ __forceinline__ double minmod3(double a, double b, double c) {
  const int sa = (a > 0) - (a < 0), sb = (b > 0) - (b < 0), sc = (c > 0) - (c < 0);
  const int m = (sa + sb + sc) / 3;
  return (m == 1 || m == -1) ? m * fmin(fmin(fabs(a), fabs(b)), fabs(c)) : 0.;
}

__global__ void __launch_bounds__(256) dg_limit_kernel(DgLimitArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.Nv || a.Ne < 3) return;
  const int K = a.K, Ne = a.Ne;
  auto U = [&](int k, int e) {
    return ld(a.u, a.f_double, ((size_t)k * Ne + e) * a.Nv + v);
  };
  auto avg = [&](int e) {
    double s = 0;
    for (int k = 0; k < K; ++k) s += a.wavg[k] * U(k, e);
    return s;
  };
  double aL = avg(0), ac = avg(1);
  for (int e = 1; e < Ne - 1; ++e) {
    const double aR = avg(e + 1);
    const double u0 = U(0, e), uK = U(K - 1, e);
    const bool lim =
        fabs(ac - minmod3(ac - u0, aR - ac, ac - aL) - u0) +
            fabs(ac + minmod3(uK - ac, aR - ac, ac - aL) - uK) > a.tol;
    if (lim) {
      double sl = 0;
      for (int k = 0; k < K; ++k) sl += a.wdr[k] * U(k, e);
      sl *= a.invjac[e];
      const double he = a.h[e];
      const double m = minmod3(sl, (aR - ac) / he, (ac - aL) / he);
      for (int k = 0; k < K; ++k)
        st(a.u, a.f_double, ((size_t)k * Ne + e) * a.Nv + v,
           ac + a.dx[k * Ne + e] * m);
    }
    aL = ac;
    ac = aR;
  }
}

// Positivity limiter of dgfsABUstd1D (abstdu.py:432-441, limitPos of
// astd/kernels/limiters.mako:198-227), in place, every element: with the cell
// average a and the smallest nodal value m, u_k <- a + theta (u_k - a),
// theta = min(1, |(a - 1e-13) / (a - m)|), the ratio rounded to single
// precision as the reference's fabsf rounds it.
__global__ void __launch_bounds__(256) dg_limit_pos_kernel(DgLimitArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.Nv) return;
  const int K = a.K, Ne = a.Ne;
  for (int e = 0; e < Ne; ++e) {
    double avg = 0, m = 1e10;
    for (int k = 0; k < K; ++k) {
      const double x = ld(a.u, a.f_double, ((size_t)k * Ne + e) * a.Nv + v);
      avg += a.wavg[k] * x;
      m = fmin(m, x);
    }
    const float ratio = (float)((avg - 1e-13) / (avg - m));
    const double theta = fmin(1.0, (double)fabsf(ratio));
    for (int k = 0; k < K; ++k) {
      const size_t i = ((size_t)k * Ne + e) * a.Nv + v;
      st(a.u, a.f_double, i, avg + theta * (ld(a.u, a.f_double, i) - avg));
    }
  }
}

// Unnormalised wall Maxwellian exp(-m |c - u_w|^2 / T_w) of a wall whose
// state is set per call (dgfs-wall-expr-diffuse.mako, bi: with the mass m).
__device__ __forceinline__ double wall_expr_maxwellian(const DgAdvectArgs& a,
                                                      int side, int v) {
  const int N = a.N;
  const double* w = a.ws[side];
  const double dx = a.c0[v / (N * N)] - w[0], dy = a.c0[(v / N) % N] - w[1],
               dz = a.c0[v % N] - w[2];
  return exp(-w[4] * (dx * dx + dy * dy + dz * dz) / w[3]);
}

// Wall densities n_w = -sum_{out} (c-u_w).n f cw / sum_{in} (c-u_w).n f0 cw
// (updateBC of dgfs-wall-diffuse.mako with the two gpuarray.sum of
// std/bc.py:63-76), in a deterministic order.
// Grid (kWallCh chunks of the velocity grid, 2 sides): partial sums
// [2][kWallCh][2]; then one thread per side adds them in a fixed order (one
// CTA per side would leave the reduction latency-bound on two SMs).
constexpr int kWallCh = 32;
__global__ void __launch_bounds__(256) dg_wall_partial_kernel(DgAdvectArgs a,
                                                              double cw,
                                                              double* part) {
  const int ch = blockIdx.x, side = blockIdx.y, t = threadIdx.x;
  __shared__ double rn[256], rd[256];
  double sn = 0, sd = 0;
  const int kind = a.bc[side];
  if (kind == kBcWall || kind == kBcWallExpr) {
    const int e = side == 0 ? 0 : a.Ne - 1;
    const double* tw = side == 0 ? a.trL : a.trR;
    const double nl = a.nl[side];
    const double ux = kind == kBcWall ? a.bc_ux[side] : a.ws[side][0];
    const int len = (a.Nv + kWallCh - 1) / kWallCh;
    const int v1 = min(a.Nv, (ch + 1) * len);
    for (int v = ch * len + t; v < v1; v += 256) {
      double ul = 0;
      for (int k = 0; k < a.K; ++k)
        ul += tw[k] * ld(a.u, a.f_double, ((size_t)k * a.Ne + e) * a.Nv + v);
      const double fac = (a.c0[v / (a.N * a.N)] - ux) * nl;
      if (fac >= 0.) sn += fac * ul * cw;
      else sd += fac * (kind == kBcWall ? a.f0[side][v] : wall_expr_maxwellian(a, side, v)) * cw;
    }
  }
  rn[t] = sn;
  rd[t] = sd;
  __syncthreads();
  for (int s2 = 128; s2 > 0; s2 >>= 1) {
    if (t < s2) { rn[t] += rn[t + s2]; rd[t] += rd[t + s2]; }
    __syncthreads();
  }
  if (t == 0) {
    part[(side * kWallCh + ch) * 2] = rn[0];
    part[(side * kWallCh + ch) * 2 + 1] = rd[0];
  }
}

__global__ void dg_wall_final_kernel(DgAdvectArgs a, const double* part,
                                     double* nden) {
  const int side = threadIdx.x;
  if (side >= 2) return;
  double rn = 0, rd = 0;
  for (int c = 0; c < kWallCh; ++c) {
    rn += part[(side * kWallCh + c) * 2];
    rd += part[(side * kWallCh + c) * 2 + 1];
  }
  nden[side] = (a.bc[side] == kBcWall || a.bc[side] == kBcWallExpr) ? -(rn / rd) : 0.0;
}

__device__ __forceinline__ double dg_ghost(const DgAdvectArgs& a, int side,
                                           int v, double cx, double ul) {
  const int kind = a.bc[side];
  if (kind == kBcWall) {
    const double fac = (cx - a.bc_ux[side]) * a.nl[side];
    return fac < 0 ? a.f0[side][v] * a.nden[side] : ul;
  }
  if (kind == kBcInlet) {
    const double fac = (cx - a.bc_ux[side]) * a.nl[side];
    return fac < 0 ? a.f0[side][v] : ul;
  }
  if (kind == kBcWallExpr) {
    const double fac = (cx - a.ws[side][0]) * a.nl[side];
    return fac < 0 ? wall_expr_maxwellian(a, side, v) * a.nden[side] : ul;
  }
  if (kind == kBcVanish) {
    const double fac = cx * a.nl[side];
    return fac >= 0 ? 0.0 : ul;
  }
  return ul;
}

// ux[k][e][v] = ((D u)[k] * (-c) - jL[e+1] gRD[k] + jR[e] gLD[k]) * invjac[e]
// with jL = 0.5|c|(uL-uR) + 0.5c(uR-uL), jR = 0.5|c|(uL-uR) + 0.5c(uL-uR)
// at each face (uL: state on its left, uR: on its right).  One thread per
// velocity point walks the elements.
template <int K>
__global__ void __launch_bounds__(256) dg_advect_kernel(DgAdvectArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.Nv) return;
  const int Ne = a.Ne, Nv = a.Nv;
  const double cx = a.c0[v / (a.N * a.N)];
  const double ac = 0.5 * fabs(cx), hc = 0.5 * cx;
  double ue[K], un[K];
#pragma unroll
  for (int k = 0; k < K; ++k) ue[k] = ld(a.u, a.f_double, ((size_t)k * Ne) * Nv + v);
  auto tl = [&](const double* w) {
    double s = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) s += a.trL[k] * w[k];
    return s;
  };
  auto tr = [&](const double* w) {
    double s = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) s += a.trR[k] * w[k];
    return s;
  };
  // the volume operator of this velocity (upwind: split by the sign of c_x)
  const double* Dv = (a.upwind == 1 && cx < 0) ? a.D2 : a.D;
  // traces at the two ends of the domain, for the swapped (periodic) ghosts
  double uEnd0 = 0, uEnd1 = 0;
  if (a.swap) {
    double ul[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
      ul[k] = ld(a.u, a.f_double, ((size_t)k * Ne + Ne - 1) * Nv + v);
    uEnd1 = tr(ul);
    uEnd0 = tl(ue);
  }
  // face 0: ghost on the left, element 0 on the right
  double uRf = tl(ue);
  double uLf = dg_ghost(a, 0, v, cx, a.swap ? uEnd1 : uRf);
  double jR = ac * (uLf - uRf) + hc * (uLf - uRf);
  for (int e = 0; e < Ne; ++e) {
    // face e+1
    const double uL1 = tr(ue);
    double uR1;
    if (e + 1 < Ne) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        un[k] = ld(a.u, a.f_double, ((size_t)k * Ne + e + 1) * Nv + v);
      uR1 = tl(un);
    } else {
      uR1 = dg_ghost(a, 1, v, cx, a.swap ? uEnd0 : uL1);
    }
    const double jd = ac * (uL1 - uR1);
    const double jL1 = jd + hc * (uR1 - uL1);
    const double ij = a.invjac[e];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double r;
      if (a.upwind == 2) {
        r = 0;
#pragma unroll
        for (int m = 0; m < K; ++m)
          r += -2 * Dv[k * K + m] * cx * log_mean(ue[k], ue[m]);
      } else {
        double d = 0;
#pragma unroll
        for (int m = 0; m < K; ++m) d += Dv[k * K + m] * ue[m];
        r = d * (-cx);
      }
      r += -jL1 * a.gRD[k] + jR * a.gLD[k];
      st(a.ux, a.f_double, ((size_t)k * Ne + e) * Nv + v, r * ij);
    }
    jR = jd + hc * (uL1 - uR1);  // jR of face e+1 for element e+1
#pragma unroll
    for (int k = 0; k < K; ++k) ue[k] = un[k];
  }
}

// x0 <- a0 x0 + sum_i a_i x_i, with the a0 == 0 (x0 not read) and a0 == 1
// branches of axnpby.py:10-44.
constexpr int kAxMax = 4;
struct AxnpbyArgs {
  void* x0;
  const void* x[kAxMax];
  double a[kAxMax];
  double a0;
  int nterms;
  int f_double;
  size_t n;
};

__global__ void axnpby_kernel(AxnpbyArgs a) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
       i += (size_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < a.nterms; ++j) {
      const double v = ld(a.x[j], a.f_double, i);
      s = (j == 0) ? a.a[0] * v : s + a.a[j] * v;
    }
    double r;
    if (a.a0 == 0.0) r = s;
    else if (a.a0 == 1.0) r = ld(a.x0, a.f_double, i) + s;
    else r = a.a0 * ld(a.x0, a.f_double, i) + s;
    st(a.x0, a.f_double, i, r);
  }
}

// Bulk moments at the reconstruction points (FP64), two passes per block:
// rho, U (then peculiar velocities), T, Q, P.  One block per (r, e).
struct MomentArgs {
  const void* coeff;        // (K, Ne, Nv)
  int f_double;
  int K, Ne, Nv, N, Nqr;
  const double* im;         // [K][Nqr] interpolation to reconstruction points
  const double* c0;         // [N]
  double cw;
  double* out;              // [Nqr][Ne][10] nondimensional
};

__global__ void __launch_bounds__(256) std_moments_kernel(MomentArgs a) {
  const int r = blockIdx.x, e = blockIdx.y;
  const int t = threadIdx.x;
  __shared__ double red[8][256];
  __shared__ double bulk[4];
  const int NN = a.N * a.N;
  auto sol = [&](int v) {
    double s = 0;
    for (int k = 0; k < a.K; ++k)
      s += a.im[k * a.Nqr + r] * ld(a.coeff, a.f_double, ((size_t)k * a.Ne + e) * a.Nv + v);
    return s;
  };
  double s0 = 0, s1 = 0, s2 = 0;
  for (int v = t; v < a.Nv; v += blockDim.x) {
    const double f = sol(v);
    s0 += f;
    s1 += f * a.c0[v / NN];
    s2 += f * a.c0[(v / a.N) % a.N];
  }
  red[0][t] = s0; red[1][t] = s1; red[2][t] = s2;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s)
      for (int i = 0; i < 3; ++i) red[i][t] += red[i][t + s];
    __syncthreads();
  }
  if (t == 0) {
    const double rho = red[0][0] * a.cw;
    bulk[0] = rho;
    bulk[1] = red[1][0] * a.cw / rho;
    bulk[2] = red[2][0] * a.cw / rho;
  }
  __syncthreads();
  const double ux = bulk[1], uy = bulk[2];
  double m[6] = {0, 0, 0, 0, 0, 0};  // |c|^2, |c|^2 cx, |c|^2 cy, cxcx, cycy, cxcy
  for (int v = t; v < a.Nv; v += blockDim.x) {
    const double f = sol(v);
    const double cx = a.c0[v / NN] - ux, cy = a.c0[(v / a.N) % a.N] - uy,
                 cz = a.c0[v % a.N];
    const double c2 = cx * cx + cy * cy + cz * cz;
    m[0] += f * c2;
    m[1] += f * c2 * cx;
    m[2] += f * c2 * cy;
    m[3] += f * cx * cx;
    m[4] += f * cy * cy;
    m[5] += f * cx * cy;
  }
  __syncthreads();
  for (int i = 0; i < 6; ++i) red[i][t] = m[i];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s)
      for (int i = 0; i < 6; ++i) red[i][t] += red[i][t + s];
    __syncthreads();
  }
  if (t == 0) {
    double* o = a.out + ((size_t)r * a.Ne + e) * 10;
    const double rho = bulk[0];
    o[0] = rho;
    o[1] = ux;
    o[2] = uy;
    o[3] = red[0][0] * (2. / 3. * a.cw) / rho;
    o[4] = red[1][0] * a.cw;
    o[5] = red[2][0] * a.cw;
    o[6] = 2 * red[3][0] * a.cw;
    o[7] = 2 * red[4][0] * a.cw;
    o[8] = 2 * red[5][0] * a.cw;
    o[9] = 0;
  }
}

// Moments of a multi-species solution (dgfs1D/bi/moments.py:11-113), FP64,
// nondimensional, [Nqr][Ne][nspcs][5] = rho, ux, uy, T, qx per species.
// Species temperatures use the species' own velocity, heat fluxes the
// mass-weighted mixture velocity; u_z is taken as zero in both, as there.
// A species whose density summed over all points is below 1e-10 keeps its
// density, gets zero velocity and temperature and is left out of the
// mixture velocity (bi/moments.py:43-45).  Two launches: pass 1 per (r, e,
// species) writes rho, ux, uy; pass 2 per (r, e) reads every point's
// densities for the global test, then writes T and qx.
constexpr int kMaxSpecies = 4;
constexpr double kMinSpeciesDensity = 1e-10;

struct BiMomentArgs {
  const void* coeff[kMaxSpecies];   // (K, Ne, Nv) per species
  double mass[kMaxSpecies];         // nondimensional molecular masses
  int f_double, nspcs;
  int K, Ne, Nv, N, Nqr;
  const double* im;                 // [K][Nqr]
  const double* c0;                 // [N]
  double cw;
  double* out;                      // [Nqr][Ne][nspcs][5]
};

__device__ __forceinline__ double bi_sol(const BiMomentArgs& a, int p, int r,
                                         int e, int v) {
  double s = 0;
  for (int k = 0; k < a.K; ++k)
    s += a.im[k * a.Nqr + r] *
         ld(a.coeff[p], a.f_double, ((size_t)k * a.Ne + e) * a.Nv + v);
  return s;
}

// Tree sum of n per-thread values over a 256-thread block; result in red[i][0].
__device__ __forceinline__ void block_sum256(double (*red)[256], int n) {
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int i = 0; i < n; ++i) red[i][threadIdx.x] += red[i][threadIdx.x + s];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) bi_moments_pass1_kernel(BiMomentArgs a) {
  const int r = blockIdx.x, e = blockIdx.y, p = blockIdx.z, t = threadIdx.x;
  __shared__ double red[3][256];
  const int NN = a.N * a.N;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int v = t; v < a.Nv; v += 256) {
    const double f = bi_sol(a, p, r, e, v);
    s0 += f;
    s1 += f * a.c0[v / NN];
    s2 += f * a.c0[(v / a.N) % a.N];
  }
  red[0][t] = s0; red[1][t] = s1; red[2][t] = s2;
  block_sum256(red, 3);
  if (t == 0) {
    const double mcw = a.mass[p] * a.cw;
    const double rho = red[0][0] * mcw;
    double* o = a.out + (((size_t)r * a.Ne + e) * a.nspcs + p) * 5;
    o[0] = rho;
    o[1] = red[1][0] * mcw / rho;
    o[2] = red[2][0] * mcw / rho;
    o[3] = 0;
    o[4] = 0;
  }
}

__global__ void __launch_bounds__(256) bi_moments_pass2_kernel(BiMomentArgs a) {
  const int r = blockIdx.x, e = blockIdx.y, t = threadIdx.x;
  __shared__ double red[2 * kMaxSpecies][256];
  __shared__ int keep[kMaxSpecies];
  __shared__ double ut[2];
  const int npts = a.Nqr * a.Ne, ns = a.nspcs;
  // global densities per species (each block sums in the same order)
  for (int p = 0; p < ns; ++p) {
    double s = 0;
    for (int i = t; i < npts; i += 256) s += a.out[((size_t)i * ns + p) * 5];
    red[p][t] = s;
  }
  block_sum256(red, ns);
  if (t == 0) {
    const double* o = a.out + ((size_t)r * a.Ne + e) * ns * 5;
    double rho = 0, mx = 0, my = 0;
    for (int p = 0; p < ns; ++p) {
      keep[p] = !(red[p][0] < kMinSpeciesDensity);
      if (keep[p]) {
        rho += o[p * 5];
        mx += o[p * 5] * o[p * 5 + 1];
        my += o[p * 5] * o[p * 5 + 2];
      }
    }
    ut[0] = mx / rho;
    ut[1] = my / rho;
  }
  __syncthreads();
  const int NN = a.N * a.N;
  double* o = a.out + ((size_t)r * a.Ne + e) * ns * 5;
  for (int p = 0; p < ns; ++p) {
    const double ux = keep[p] ? o[p * 5 + 1] : 0.0, uy = keep[p] ? o[p * 5 + 2] : 0.0;
    double sT = 0, sq = 0;
    for (int v = t; v < a.Nv; v += 256) {
      const double f = bi_sol(a, p, r, e, v);
      const double cx = a.c0[v / NN], cy = a.c0[(v / a.N) % a.N], cz = a.c0[v % a.N];
      const double px = cx - ux, py = cy - uy;
      sT += f * (px * px + py * py + cz * cz);
      const double qx = cx - ut[0], qy = cy - ut[1];
      sq += f * (qx * qx + qy * qy + cz * cz) * qx;
    }
    red[2 * p][t] = sT;
    red[2 * p + 1][t] = sq;
  }
  block_sum256(red, 2 * ns);
  if (t == 0) {
    for (int p = 0; p < ns; ++p) {
      const double m = a.mass[p], mcw = m * a.cw;
      if (keep[p]) {
        o[p * 5 + 3] = red[2 * p][0] * (2.0 / 3.0 * mcw * m) / o[p * 5];
      } else {
        o[p * 5 + 1] = 0;
        o[p * 5 + 2] = 0;
        o[p * 5 + 3] = 0;
      }
      o[p * 5 + 4] = m * red[2 * p + 1][0] * mcw;
    }
  }
}

// Explicit ES-BGK relaxation of dgfsStd1D (esbgk-direct-gll, the fs of
// std/scattering.py:1540-1637 with std/kernels/scattering/esbgk-direct-gll.mako):
// per point rho = sum f cw, u = sum f c / sum f, T = sum f |c-u|^2 cw/(1.5 rho);
// the covariance S_ij = sum (c-u)_i (c-u)_j ((1-1/Pr) f + (1/Pr) f_M) cw / rho
// with the grid Maxwellian f_M = rho/(pi T)^1.5 exp(-|c-u|^2/T); then
// Q += prefac rho / T^(omega-1) (f_ES - f), f_ES = rho/((2 pi)^1.5 sqrt(det S))
// exp(-(c-u)^T S^-1 (c-u) / 2).  One block per point (FP64 sums).
struct StdEsArgs {
  const void* f;
  void* Q;
  int f_double;
  int N, Nv;
  const double* c0;
  double cw, prefac, omega, Pr;
};

__global__ void __launch_bounds__(256) std_esbgk_relax_kernel(StdEsArgs a) {
  const int pt = blockIdx.x, t = threadIdx.x;
  __shared__ double red[6][256];
  __shared__ double pv[12];  // rho, ux, uy, uz, T, det, A[6]
  const int N = a.N, NN = N * N, Nv = a.Nv;
  const size_t base = (size_t)pt * Nv;
  auto fv = [&](int v) { return ld(a.f, a.f_double, base + v); };
  auto cxyz = [&](int v, double& x, double& y, double& z) {
    x = a.c0[v / NN]; y = a.c0[(v / N) % N]; z = a.c0[v % N];
  };
  // rho, u
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  for (int v = t; v < Nv; v += 256) {
    double x, y, z;
    cxyz(v, x, y, z);
    const double f = fv(v);
    s0 += f; s1 += f * x; s2 += f * y; s3 += f * z;
  }
  red[0][t] = s0; red[1][t] = s1; red[2][t] = s2; red[3][t] = s3;
  block_sum256(red, 4);
  if (t == 0) {
    pv[1] = red[1][0] / red[0][0];
    pv[2] = red[2][0] / red[0][0];
    pv[3] = red[3][0] / red[0][0];
    pv[0] = red[0][0] * a.cw;
  }
  __syncthreads();
  const double rho = pv[0], ux = pv[1], uy = pv[2], uz = pv[3];
  // T
  double s4 = 0;
  for (int v = t; v < Nv; v += 256) {
    double x, y, z;
    cxyz(v, x, y, z);
    s4 += fv(v) * ((x - ux) * (x - ux) + (y - uy) * (y - uy) + (z - uz) * (z - uz));
  }
  __syncthreads();
  red[0][t] = s4;
  block_sum256(red, 1);
  if (t == 0) pv[4] = red[0][0] * (a.cw / (1.5 * rho));
  __syncthreads();
  const double T = pv[4];
  // covariance of (1 - 1/Pr) f + (1/Pr) f_M
  const double wf = 1. - 1. / a.Pr, wm = 1. / a.Pr;
  const double nm = rho / pow(M_PI * T, 1.5);
  double m[6] = {0, 0, 0, 0, 0, 0};  // xx, yy, zz, xy, yz, zx
  for (int v = t; v < Nv; v += 256) {
    double x, y, z;
    cxyz(v, x, y, z);
    const double dx = x - ux, dy = y - uy, dz = z - uz;
    const double fm = nm * exp(-(dx * dx + dy * dy + dz * dz) / T);
    const double w = wf * fv(v) + wm * fm;
    m[0] += dx * dx * w; m[1] += dy * dy * w; m[2] += dz * dz * w;
    m[3] += dx * dy * w; m[4] += dy * dz * w; m[5] += dz * dx * w;
  }
  __syncthreads();
  for (int i = 0; i < 6; ++i) red[i][t] = m[i];
  block_sum256(red, 6);
  if (t == 0) {
    const double k = a.cw / rho;
    const double m4 = red[0][0] * k, m5 = red[1][0] * k, m6 = red[2][0] * k,
                 m7 = red[3][0] * k, m8 = red[4][0] * k, m9 = red[5][0] * k;
    const double det = -m6 * m7 * m7 + 2 * m7 * m8 * m9 - m4 * m8 * m8 -
                       m5 * m9 * m9 + m4 * m5 * m6;
    pv[5] = det;
    pv[6] = (m5 * m6 - m8 * m8) / det;   // 11
    pv[7] = (m4 * m6 - m9 * m9) / det;   // 22
    pv[8] = (m4 * m5 - m7 * m7) / det;   // 33
    pv[9] = (m8 * m9 - m6 * m7) / det;   // 12
    pv[10] = (m7 * m9 - m4 * m8) / det;  // 23
    pv[11] = (m7 * m8 - m9 * m5) / det;  // 31
  }
  __syncthreads();
  const double* A = pv + 6;
  const double ne = rho / (pow(2 * M_PI, 1.5) * sqrt(pv[5]));
  const double nu = a.prefac * (rho / pow(T, a.omega - 1.));
  for (int v = t; v < Nv; v += 256) {
    double x, y, z;
    cxyz(v, x, y, z);
    const double dx = x - ux, dy = y - uy, dz = z - uz;
    const double q = A[0] * (dx * dx) + A[1] * (dy * dy) + A[2] * (dz * dz) +
                     2 * A[3] * (dx * dy) + 2 * A[4] * (dy * dz) + 2 * A[5] * (dz * dx);
    const double fes = ne * exp(-q / 2.);
    const double r = ld(a.Q, a.f_double, base + v) + nu * (fes - fv(v));
    st(a.Q, a.f_double, base + v, r);
  }
}

// sum (x - y)^2 and sum y^2 in FP64 (residual of std/residual.py:15-29)
__global__ void __launch_bounds__(512) residual_kernel(const void* x,
                                                       const void* y, int dbl,
                                                       size_t n, double* out) {
  __shared__ double r0[512], r1[512];
  const int t = threadIdx.x;
  double a = 0, b = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + t; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double xv = ld(x, dbl, i), yv = ld(y, dbl, i), d = xv - yv;
    a += d * d;
    b += yv * yv;
  }
  r0[t] = a;
  r1[t] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) { r0[t] += r0[t + s]; r1[t] += r1[t + s]; }
    __syncthreads();
  }
  if (t == 0) {
    out[2 * blockIdx.x] = r0[0];
    out[2 * blockIdx.x + 1] = r1[0];
  }
}

}  // namespace dgfs

namespace dgfs {

// ---------------------------------------------------------------------------
// Penalty (BGK-type) model of the penalised IMEX schemes (FP64).
// Reference: dgfs1D/astd/scattering.py:44-284 with the kernels of
// dgfs1D/astd/kernels/scattering/bgk-direct-gll.mako (moments by a cuBLAS
// gemm there, cmaxwellian, collide, updateDistribution{q}_BDF / _LM).
// Moments per point: U = (rho, rho ux, rho uy, rho uz, E) with
// E = sum f |c|^2 cw;  T = (E - |rho u|^2 / rho) / (1.5 rho);
// nu = prefac rho T^(1-omega).
// ---------------------------------------------------------------------------
struct PenaltyMomentArgs {
  const void* f;          // [npts][Nv]
  int f_double;
  int Nv, N;
  const double* c0;
  double cw;
  double* U;              // [npts][5]
};


// The same moments over many CTAs: grid (kPmCh chunks, npts), partial sums
// [npts][kPmCh][NA], then a fixed-order sum per (point, moment).  NA = 5
// (BGK), 11 (ES-BGK: + c_x^2, c_y^2, c_z^2, c_x c_y, c_y c_z, c_z c_x) or
// 14 (Shakov: + |c|^2 c), the rows of astd/scattering.py:155-162, 306-316,
// 375-388.
constexpr int kPmCh = 16;
constexpr int kPmMaxNa = 14;
template <int NA>
__global__ void __launch_bounds__(256)
penalty_moments_part_kernel(PenaltyMomentArgs a, double* part) {
  const int ch = blockIdx.x, p = blockIdx.y, t = threadIdx.x;
  __shared__ double red[NA][256];
  const int NN = a.N * a.N;
  const int len = (a.Nv + kPmCh - 1) / kPmCh, v1 = min(a.Nv, (ch + 1) * len);
  double s[NA];
#pragma unroll
  for (int k = 0; k < NA; ++k) s[k] = 0;
  for (int v = ch * len + t; v < v1; v += 256) {
    const double fv = ld(a.f, a.f_double, (size_t)p * a.Nv + v) * a.cw;
    const double cx = a.c0[v / NN], cy = a.c0[(v / a.N) % a.N], cz = a.c0[v % a.N];
    const double c2 = cx * cx + cy * cy + cz * cz;
    s[0] += fv;
    s[1] += fv * cx;
    s[2] += fv * cy;
    s[3] += fv * cz;
    s[4] += fv * c2;
    if (NA > 5) {
      s[5] += fv * cx * cx;
      s[6] += fv * cy * cy;
      s[7] += fv * cz * cz;
      s[8] += fv * cx * cy;
      s[9] += fv * cy * cz;
      s[10] += fv * cz * cx;
    }
    if (NA > 11) {
      s[11] += fv * c2 * cx;
      s[12] += fv * c2 * cy;
      s[13] += fv * c2 * cz;
    }
  }
#pragma unroll
  for (int k = 0; k < NA; ++k) red[k][t] = s[k];
  __syncthreads();
  for (int st2 = 128; st2 > 0; st2 >>= 1) {
    if (t < st2)
      for (int k = 0; k < NA; ++k) red[k][t] += red[k][t + st2];
    __syncthreads();
  }
  if (t < NA) part[((size_t)p * kPmCh + ch) * NA + t] = red[t][0];
}

__global__ void penalty_moments_final_kernel(const double* part, double* U,
                                             int npts, int na) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts * na) return;
  const int p = i / na, k = i % na;
  double s = 0;
  for (int c = 0; c < kPmCh; ++c) s += part[((size_t)p * kPmCh + c) * na + k];
  U[i] = s;
}

struct PenaltyImplicitArgs {
  const double* U;        // [npts][NA] moments at the new level
  const void* rhs;        // [npts][Nv] explicit combination
  void* f;                // out [npts][Nv] new distribution
  void* P;                // out (or null) nu (M - f)
  void* Mout;             // out (or null) the Maxwellian
  int f_double;
  int Nv, N;
  const double* c0;
  double adiv;            // denominator constant (a_q for BDF, 1 for LM)
  double cdt;             // implicit weight times dt (b dt, c0 dt)
  double prefac, omega;
  double Pr;              // Prandtl number (ES-BGK, Shakov)
  size_t total;           // npts * Nv
};

// Penalty models: 0 BGK (Maxwellian), 1 ES-BGK (anisotropic Gaussian),
// 2 Shakov (Maxwellian times the heat-flux polynomial).  U holds each point's
// NA = 5 / 11 / 14 raw moments (see penalty_moments_part_kernel).
constexpr int kPenBGK = 0, kPenESBGK = 1, kPenShakov = 2;
template <int KIND> struct PenaltyNa;
template <> struct PenaltyNa<kPenBGK> { static constexpr int value = 5; };
template <> struct PenaltyNa<kPenESBGK> { static constexpr int value = 11; };
template <> struct PenaltyNa<kPenShakov> { static constexpr int value = 14; };

// Per-point state, formed once per CTA: u, T, nu = prefac rho T^(1-omega)
// (the powers once per point, not per velocity) and the Gaussian's
// parameters: amp and, for ES-BGK, the inverse of the temperature tensor
// T_ij = T/Pr delta_ij + 2 (1 - 1/Pr)(P_ij/rho - u_i u_j)
// (esbgk-direct-gll.mako:157-254); for Shakov, the peculiar heat flux
// scaled by 2 (1 - Pr)/(5 rho T^2) (shakov-direct-gll.mako:193-278).
struct PenaltyPoint {
  double ux, uy, uz, T, amp, nu;
  double Ai[6];  // ES-BGK: inverse tensor xx, yy, zz, xy, yz, zx
  double qc[3];  // Shakov: scaled heat flux
};
template <int KIND>
__device__ __forceinline__ PenaltyPoint penalty_point(const double* U,
                                                      double prefac,
                                                      double omega, double Pr) {
  PenaltyPoint s;
  const double rho = U[0];
  const double T = (U[4] - (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rho) /
                   (1.5 * rho);
  s.ux = U[1] / rho; s.uy = U[2] / rho; s.uz = U[3] / rho;
  s.T = T;
  s.nu = prefac * rho * pow(T, 1. - omega);
  s.amp = rho / pow(M_PI * T, 1.5);
  if (KIND == kPenESBGK) {
    const double lam = 1. / Pr, mu = 2. * (1. - 1. / Pr);
    const double a = lam * T + mu * (U[5] / rho - s.ux * s.ux);
    const double b = lam * T + mu * (U[6] / rho - s.uy * s.uy);
    const double c = lam * T + mu * (U[7] / rho - s.uz * s.uz);
    const double d = mu * (U[8] / rho - s.ux * s.uy);
    const double e = mu * (U[9] / rho - s.uy * s.uz);
    const double f = mu * (U[10] / rho - s.uz * s.ux);
    const double det = -c * d * d + 2 * d * e * f - a * e * e - b * f * f + a * b * c;
    s.Ai[0] = (b * c - e * e) / det;
    s.Ai[1] = (a * c - f * f) / det;
    s.Ai[2] = (a * b - d * d) / det;
    s.Ai[3] = (e * f - c * d) / det;
    s.Ai[4] = (d * f - a * e) / det;
    s.Ai[5] = (d * e - f * b) / det;
    s.amp = rho / (pow(M_PI, 1.5) * sqrt(det));
  } else if (KIND == kPenShakov) {
    const double u2 = s.ux * s.ux + s.uy * s.uy + s.uz * s.uz;
    const double u[3] = {s.ux, s.uy, s.uz};
    const int row[3][3] = {{5, 8, 10}, {8, 6, 9}, {10, 9, 7}};
    const double sc = 2. * (1. - Pr) / 5. / (rho * T * T);
#pragma unroll
    for (int i = 0; i < 3; ++i)
      s.qc[i] = sc * (U[11 + i] - 2. * (U[row[i][0]] * s.ux + U[row[i][1]] * s.uy +
                                       U[row[i][2]] * s.uz) +
                      rho * u[i] * u2 - 1.5 * u[i] * rho * T);
  }
  return s;
}

constexpr int kPenaltyEpt = 8;  // velocities per thread
template <int KIND>
__device__ __forceinline__ double penalty_gaussian(const PenaltyPoint& s,
                                                   const double* c0, int N,
                                                   int v) {
  const int NN = N * N;
  const double dx = c0[v / NN] - s.ux;
  const double dy = c0[(v / N) % N] - s.uy;
  const double dz = c0[v % N] - s.uz;
  const double d2 = dx * dx + dy * dy + dz * dz;
  if (KIND == kPenESBGK) {
    const double q = s.Ai[0] * dx * dx + s.Ai[1] * dy * dy + s.Ai[2] * dz * dz +
                     2. * (s.Ai[3] * dx * dy + s.Ai[4] * dy * dz + s.Ai[5] * dz * dx);
    return s.amp * exp(-q);
  }
  const double M = s.amp * exp(-d2 / s.T);
  if (KIND == kPenShakov)
    return M * (1. + (s.qc[0] * dx + s.qc[1] * dy + s.qc[2] * dz) *
                         (2. * d2 / s.T - 5.));
  return M;
}

// f = (rhs + cdt nu G) / (adiv + cdt nu), optionally P = nu (G - f) and G;
// grid (chunks of the velocity grid, npts).
template <int KIND>
__global__ void __launch_bounds__(256) penalty_implicit_kernel(PenaltyImplicitArgs a) {
  __shared__ PenaltyPoint sp;
  constexpr int NA = PenaltyNa<KIND>::value;
  const size_t p = blockIdx.y;
  if (threadIdx.x == 0) sp = penalty_point<KIND>(a.U + p * NA, a.prefac, a.omega, a.Pr);
  __syncthreads();
  const PenaltyPoint s = sp;
  const int v0 = blockIdx.x * 256 * kPenaltyEpt + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kPenaltyEpt; ++r) {
    const int v = v0 + r * 256;
    if (v >= a.Nv) break;
    const size_t i = p * a.Nv + v;
    const double M = penalty_gaussian<KIND>(s, a.c0, a.N, v);
    const double rr = ld(a.rhs, a.f_double, i);
    const double fn = (rr + a.cdt * s.nu * M) / (a.adiv + a.cdt * s.nu);
    st(a.f, a.f_double, i, fn);
    if (a.P) st(a.P, a.f_double, i, s.nu * (M - fn));
    if (a.Mout) st(a.Mout, a.f_double, i, M);
  }
}

// P = nu (G(U) - f) for the current f and its moments U (collide).
template <int KIND>
__global__ void __launch_bounds__(256) penalty_collide_kernel(PenaltyImplicitArgs a) {
  __shared__ PenaltyPoint sp;
  constexpr int NA = PenaltyNa<KIND>::value;
  const size_t p = blockIdx.y;
  if (threadIdx.x == 0) sp = penalty_point<KIND>(a.U + p * NA, a.prefac, a.omega, a.Pr);
  __syncthreads();
  const PenaltyPoint s = sp;
  const int v0 = blockIdx.x * 256 * kPenaltyEpt + threadIdx.x;
#pragma unroll
  for (int r = 0; r < kPenaltyEpt; ++r) {
    const int v = v0 + r * 256;
    if (v >= a.Nv) break;
    const size_t i = p * a.Nv + v;
    const double M = penalty_gaussian<KIND>(s, a.c0, a.N, v);
    st(a.P, a.f_double, i, s.nu * (M - ld(a.f, a.f_double, i)));
    if (a.Mout) st(a.Mout, a.f_double, i, M);
  }
}

// Implicit relaxation of the non-conserved moments after the linear
// combination of a BDF / IMEX-LM moment update (updateMom{q}_BDF and _LM of
// esbgk-direct-gll.mako :16-81, :480-540 and shakov-direct-gll.mako :18-120,
// :549-645, with adiv = a_q, cdt = b dt for BDF and adiv = 1, cdt = c_0 dt
// for LM): with nu = prefac rho T^(1-omega) from the updated conserved
// moments, the stresses relax as (adiv U + k tau)/(adiv + k), tau_ii =
// rho T/2 + (rho u_i)^2/rho, tau_ij = (rho u_i)(rho u_j)/rho, k = cdt nu/Pr
// (ES-BGK) or cdt nu (Shakov); the Shakov heat flux as (adiv U + cdt nu
// tau_q)/(adiv + Pr cdt nu) with the relaxed stresses.  One thread per point.
template <int KIND>
__global__ void penalty_relax_kernel(double* Uall, int npts, double adiv,
                                     double cdt, double prefac, double omega,
                                     double Pr) {
  constexpr int NA = PenaltyNa<KIND>::value;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npts) return;
  double* U = Uall + (size_t)p * NA;
  const double rho = U[0];
  const double T = (U[4] - (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / rho) /
                   (1.5 * rho);
  const double nu = prefac * rho * pow(T, 1. - omega);
  const double k = KIND == kPenESBGK ? cdt / Pr * nu : cdt * nu;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double tau = 0.5 * rho * T + U[1 + i] * U[1 + i] / rho;
    U[5 + i] = (adiv * U[5 + i] + k * tau) / (adiv + k);
  }
  const int oi[3] = {1, 2, 3}, oj[3] = {2, 3, 1};
#pragma unroll
  for (int n = 0; n < 3; ++n) {
    const double tau = U[oi[n]] * U[oj[n]] / rho;
    U[8 + n] = (adiv * U[8 + n] + k * tau) / (adiv + k);
  }
  if (KIND == kPenShakov) {
    const int row[3][3] = {{5, 8, 10}, {8, 6, 9}, {10, 9, 7}};
    const double m2 = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / (rho * rho);
    const double kq = cdt * nu;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double ru = U[1 + i];
      const double tq = (1. - Pr) * (-2. * (U[row[i][0]] * U[1] + U[row[i][1]] * U[2] +
                                            U[row[i][2]] * U[3]) / rho +
                                     ru * m2 - 1.5 * ru * T) +
                        (ru * m2 + 2.5 * ru * T);
      U[11 + i] = (adiv * U[11 + i] + kq * tq) / (adiv + Pr * kq);
    }
  }
}

}  // namespace dgfs

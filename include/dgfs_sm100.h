/*
 * dgfs_sm100 -- C ABI of the B200 (sm_100a) fast-spectral Boltzmann
 * collision operators of DGFS.
 *
 * Plain pointers and sizes only.  Every call returns 0 on success or a
 * negative DGFS_ERR_* code; dgfs_last_error_string() describes the last
 * failure on the calling thread.  Device pointers are CUDA device addresses
 * on the current device; `stream` is a cudaStream_t (NULL = legacy default
 * stream).  Evaluation calls launch work asynchronously, allocate nothing and
 * never synchronise the host.  A handle owns its scratch: calls on one
 * handle must be ordered (same stream, or externally synchronised).
 *
 * Layout (as in the reference): a distribution array holds `slots` of n =
 * N^3 values, slot s at offset s*n, velocity index v = (i*N + j)*N + k with
 * i <-> c_x slowest.  The reference addresses slot (mode*Ne + elem)
 * (dgfs1D/std/kernels/scattering/vhs-gll.mako:408).
 */
#ifndef DGFS_SM100_H
#define DGFS_SM100_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGFS_OK 0
#define DGFS_ERR_INVALID (-1)      /* bad argument or descriptor */
#define DGFS_ERR_UNSUPPORTED (-2)  /* shape/precision not compiled in */
#define DGFS_ERR_CUDA (-3)         /* CUDA runtime or launch failure */
#define DGFS_ERR_CAPACITY (-4)     /* size beyond a fixed maximum */

#define DGFS_F32 0                 /* float arrays */
#define DGFS_F64 1                 /* double arrays */

#define DGFS_PREC_FP64 0           /* all arithmetic in FP64 */
#define DGFS_PREC_FP32 1           /* FP32 3-D FFTs on f - M (local
                                      Maxwellian M handled in FP64) */

typedef struct dgfs_vhs_s* dgfs_vhs_handle;

/*
 * Single-species VHS/HS fast-spectral model, `vhs-gll` and `vhs` in the
 * reference (dgfs1D/std/scattering.py:51-313, 317-429).  The descriptor
 * carries what DGFSVHSGLLScatteringModelStd.perform_precomputation reads
 * from the velocity mesh (std/scattering.py:106-191): grid size N, radial
 * Gauss rule qz/qw (Nrho points on [0, R]), spherical rule sz (M x 3) with
 * weight sw, the factor 2 of computeQG for a half-sphere rule
 * (vhs-gll.mako:192; 1 for a full-sphere rule), gamma = 2(1-omega), the
 * collision prefactor, the sinc regulariser (1e-15 double, 1e-6 float), the
 * cell volume cw and the 1-D velocity grid c0[N].
 */
typedef struct {
  int32_t N;
  int32_t Nrho;
  int32_t M;
  double L;
  const double* qz;        /* [Nrho] host */
  const double* qw;        /* [Nrho] host */
  const double* sz;        /* [M*3] host, row-major */
  double sw;
  double sphere_factor;
  double gamma;
  double prefac;
  double sinc_eps;
  double cw;
  const double* c0;        /* [N] host */
  int32_t precision;       /* DGFS_PREC_* */
  int32_t max_evals;       /* evaluations per launch batch (scratch size) */
} dgfs_vhs_desc;

/* Replaces DGFSVHSGLLScatteringModelStd.__init__/perform_precomputation
 * (std/scattering.py:51-246): builds tables, allocates scratch. */
int dgfs_vhs_create(const dgfs_vhs_desc* desc, dgfs_vhs_handle* out);

/* Batched Q(f,f):  for i in [0, nevals):
 *     Q[dst(i)] += prefac * (gain(f[src(i)]) - f[src(i)] * loss(f[src(i)]))
 * with src(i) = src_slots ? src_slots[i] : src_base + i (device int32
 * array), likewise dst.  One call replaces nevals calls of
 * DGFSVHSGLLScatteringModelStd.fs (std/scattering.py:251-313). */
int dgfs_vhs_eval(dgfs_vhs_handle h, const void* f, int32_t f_dtype, void* Q,
                  int32_t q_dtype, const int32_t* src_slots, int32_t src_base,
                  const int32_t* dst_slots, int32_t dst_base, int32_t nevals,
                  void* stream);

/* Q(f, f) for points of several problems that share this handle's operator
 * (same grid, rules and parameters) in one launch sequence: f_list and
 * q_list are DEVICE arrays of nevals pointers; evaluation i reads slot
 * src(i) of f_list[i] and adds into slot dst(i) of q_list[i].  No reference
 * counterpart (the reference evaluates one point per call). */
int dgfs_vhs_eval_multi(dgfs_vhs_handle h, const void* const* f_list,
                        int32_t f_dtype, void* const* q_list, int32_t q_dtype,
                        const int32_t* src_slots, int32_t src_base,
                        const int32_t* dst_slots, int32_t dst_base,
                        int32_t nevals, void* stream);

/* Reference-shaped single evaluation: fs(d_f, d_g, d_Q, elem, modein,
 * modeout) of std/scattering.py:251 (d_g unused there as here):
 * src = modein*Ne + elem, dst = modeout*Ne + elem. */
int dgfs_vhs_fs(dgfs_vhs_handle h, const void* f, void* Q, int32_t dtype,
                int32_t Ne, int32_t elem, int32_t modein, int32_t modeout,
                void* stream);

/* Bilinear Q(f, g), `vhs` in the reference (DGFSVHSScatteringModelStd.fs,
 * std/scattering.py:346-429 with cosMul/sinMul/cplxMul/cplxMulAdd of
 * vhs-gll.mako:260-397):  for i in [0, nevals):
 *     Q[dst(i)] += prefac * (gain(f[src(i)], g[src(i)])
 *                            - f[src(i)] * Re IFFT(b2 FFT(g[src(i)])/n))
 * with the gain sum_pq FFT(IFFT(cos a F) IFFT(cos a G) + IFFT(sin a F)
 * IFFT(sin a G)) weighted by b1 as in Q(f, f).  f and g are read at the same
 * slot of two arrays of dtype f_dtype.  Evaluated by polarisation of the
 * symmetric gain through the Q(h, h) pipeline: two passes in the FP64 mode,
 * three in the FP32 mode (so twice / three times the cost of dgfs_vhs_eval).
 * With g == f it equals dgfs_vhs_eval up to rounding. */
int dgfs_vhs_eval2(dgfs_vhs_handle h, const void* f, const void* g,
                   int32_t f_dtype, void* Q, int32_t q_dtype,
                   const int32_t* src_slots, int32_t src_base,
                   const int32_t* dst_slots, int32_t dst_base, int32_t nevals,
                   void* stream);

/* Reference-shaped bilinear evaluation: fs(d_arr_in1, d_arr_in2, d_arr_out,
 * elem, modein, modeout) of std/scattering.py:346: f = d_arr_in1 and
 * g = d_arr_in2, both read at slot modein*Ne + elem; dst = modeout*Ne + elem. */
int dgfs_vhs_fs2(dgfs_vhs_handle h, const void* f, const void* g, void* Q,
                 int32_t dtype, int32_t Ne, int32_t elem, int32_t modein,
                 int32_t modeout, void* stream);

/* Conservation projection (no counterpart in the reference, which has no
 * projection): when enabled, every evaluation subtracts from its increment
 * the minimal-L2 combination of (1, cx, cy, cz, |c|^2) that makes the five
 * discrete moments sum_v Q phi cw vanish (FP64 multipliers, Gram matrix
 * inverted at enable time).  Off by default. */
int dgfs_vhs_set_projection(dgfs_vhs_handle h, int32_t enable);

/* Autotuning (no reference counterpart): the FP32 terms kernel comes in
 * several thread-block-cluster sizes per N.  dgfs_vhs_variants writes the
 * compiled cluster sizes for N into out (up to max) and returns their count;
 * dgfs_vhs_set_variant selects one for a handle (0 = built-in default). */
int dgfs_vhs_variants(int32_t N, int32_t* out, int32_t max);
int dgfs_vhs_set_variant(dgfs_vhs_handle h, int32_t cluster);

/* Device error flag of the handle's kernels (no reference counterpart):
 * nonzero when a bounded wait (the TMA copies of the TMA terms variant)
 * gave up, which leaves that evaluation's Q invalid.  Waits for the device,
 * writes the flag to *out and clears it. */
int dgfs_vhs_device_error(dgfs_vhs_handle h, int32_t* out);

/* Per-eval local moments (rho, ux, uy, uz, T) of the last FP32 evaluation
 * batch, device pointer owned by the handle ([max_evals][5] doubles). */
const double* dgfs_vhs_last_moments(dgfs_vhs_handle h);

int dgfs_vhs_destroy(dgfs_vhs_handle h);

/* Profiling (no reference counterpart: the reference times whole runs with
 * timeit, std/std.py:394-423).  When enabled, dgfs_vhs_eval records CUDA
 * events on its stream between its five kernels; dgfs_vhs_stage_ms waits
 * for the last call and returns the durations in ms of: prologue, tables,
 * Maxwellian gain, terms, epilogue (zero for stages the mode skips). */
int dgfs_vhs_profile(dgfs_vhs_handle h, int32_t enable);
int dgfs_vhs_stage_ms(dgfs_vhs_handle h, double* out5);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (the
 * roofline denominator of the CUDA-core FFT kernels). */
int dgfs_fma_peak(double* tflops, void* stream);

/*
 * Binary-mixture VSS model, `vss` in the reference (dgfs1D/bi/scattering.py:
 * 47-321, dgfs1D/bi/kernels/scattering/vss.mako).  Mirrors what
 * DGFSBiVSSScatteringModel.load_parameters/perform_precomputation read: the
 * full-sphere rule sz (M <= 16 points, weight sw = 4 pi / M), the
 * pre-integration rule szpre (Mpre points), nondimensional masses, and per
 * ordered pair pq = p*nspcs + q: gamma = 2(1-omega), eta = alpha - 1 and the
 * prefactor (bi/scattering.py:66-89).  The weights b_pq and c_pq
 * (precompute_bc_pq, vss.mako:51-93) are built on the GPU at create.
 */
typedef struct dgfs_vss_s* dgfs_vss_handle;
typedef struct {
  int32_t N;
  int32_t Nrho;
  int32_t M;
  int32_t Mpre;
  int32_t nspcs;           /* 1..4 */
  double L;
  const double* qz;        /* [Nrho] host */
  const double* qw;        /* [Nrho] host */
  const double* sz;        /* [M*3] host */
  double sw;
  const double* szpre;     /* [Mpre*3] host */
  const double* masses;    /* [nspcs] host, nondimensional */
  const double* gamma;     /* [nspcs*nspcs] host */
  const double* eta;       /* [nspcs*nspcs] host */
  const double* prefac;    /* [nspcs*nspcs] host */
  int32_t max_evals;
  int32_t precision;       /* DGFS_PREC_FP64 (reference) or DGFS_PREC_FP32:
                              FP32 transforms of f - M with the Maxwellian
                              parts and the radial sum, final transform and
                              loss in FP64 (no counterpart in the reference,
                              which is FP64 only) */
} dgfs_vss_desc;

int dgfs_vss_create(const dgfs_vss_desc* desc, dgfs_vss_handle* out);
int dgfs_vss_destroy(dgfs_vss_handle h);

/* Q_p[dst(i)] += Q_pq(f_p[src(i)], f_q[src(i)]) for i < nevals: the batched
 * form of DGFSBiVSSScatteringModel.fs('pq', d_f1, d_f2, d_Q, elem, upt,
 * uptout) (bi/scattering.py:263-321). */
int dgfs_vss_eval(dgfs_vss_handle h, int32_t p, int32_t q, const void* f_p,
                  const void* f_q, int32_t f_dtype, void* Q_p, int32_t q_dtype,
                  const int32_t* src_slots, int32_t src_base,
                  const int32_t* dst_slots, int32_t dst_base, int32_t nevals,
                  void* stream);

/* Every pair of one species in one call (the species loop of the
 * reference's mixture right-hand side, bi/bi.py:336-342, which calls fs once
 * per partner q):  Q_p[dst(i)] += sum_q Q_pq(f_p[src(i)], f_q[src(i)]).
 * f is a host array of nspcs device pointers (f[q] holds species q).  In
 * the FP32 mode one launch per stage covers every pair (prologues once per
 * input species, the FP64 Maxwellian gain beside the FP32 terms kernel, one
 * epilogue summing the pairs); in the FP64 mode the pairs run one by one. */
int dgfs_vss_eval_species(dgfs_vss_handle h, int32_t p, const void* const* f,
                          int32_t f_dtype, void* Q_p, int32_t q_dtype,
                          const int32_t* src_slots, int32_t src_base,
                          const int32_t* dst_slots, int32_t dst_base,
                          int32_t nevals, void* stream);

/* dgfs_vss_eval_species for points of several mixtures that share this
 * handle's operator (FP32 mode only): f_lists is a DEVICE array
 * [nspcs][nevals] of input arrays (evaluation i of species q reads slot
 * src(i) of f_lists[q*nevals + i]), q_list a DEVICE array [nevals] of the
 * species-p output arrays.  No reference counterpart. */
int dgfs_vss_eval_species_multi(dgfs_vss_handle h, int32_t p,
                                const void* const* f_lists, int32_t f_dtype,
                                void* const* q_list, int32_t q_dtype,
                                const int32_t* src_slots, int32_t src_base,
                                const int32_t* dst_slots, int32_t dst_base,
                                int32_t nevals, void* stream);

/*
 * Nodal DG advection right-hand side of the single-species solver.
 * Replaces the kernels of the rhs() closure in dgfs1D/std/std.py:281-345:
 * bwdTransFace + extract_left/right + transfer/insert BC (std.mako:4-89),
 * the boundary kernels updateBC/applyBC (std/kernels/bcs/*.mako with the two
 * host sums of std/bc.py:73-74), flux (std.mako:115-152), deriv (gimmik),
 * mul_by_adv, totalFlux and mul_by_invjac (std.mako:92-190).  trL/trR are
 * rows 0 and Nqf-1 of Bqf^T, D the derivative operator (ux = D u), gLD/gRD
 * the lifting vectors, im the K x Nqr interpolation to the moment points.
 * Boundary kinds: 0 dgfs-periodic / dgfs-cyclic (one rank: ghost = interior
 * trace), 1 dgfs-wall-diffuse, 2 dgfs-inlet / dgfs-inlet-nondim (incoming
 * where (c_x - bc_ux) n < 0; bc_ux = 0 for dgfs-inlet), 3 dgfs-vanish,
 * 4 dgfs-wall-expr-diffuse (state set by dgfs_dg_set_wall_state);
 * bc_f0 the wall/inlet Maxwellian (kinds 1 and 2).
 * (std/bc.py:25-327, std/kernels/bcs/*.mako, bi/bc.py)
 */
typedef struct dgfs_dg_s* dgfs_dg_handle;
typedef struct {
  int32_t K;
  int32_t Ne;
  int32_t N;
  int32_t Nqr;
  const double* trL;       /* [K] host */
  const double* trR;       /* [K] host */
  const double* D;         /* [K*K] host, row-major */
  const double* gLD;       /* [K] host */
  const double* gRD;       /* [K] host */
  const double* invjac;    /* [Ne] host */
  const double* c0;        /* [N] host */
  const double* im;        /* [K*Nqr] host */
  double cw;
  int32_t bc_kind[2];      /* left, right */
  const double* bc_f0[2];  /* [N^3] host, or null for kind 0 */
  double bc_ux[2];         /* wall x-velocities (nondimensional) */
} dgfs_dg_desc;

int dgfs_dg_create(const dgfs_dg_desc* desc, dgfs_dg_handle* out);
int dgfs_dg_destroy(dgfs_dg_handle h);

/* ux = advection + upwind flux lifting of u (shape (K, Ne, N^3), the
 * solution coefficients), scaled by the inverse Jacobian -- the state of
 * d_ux in std.py:346 before the collision loop.  Also records the wall
 * densities of this call (dgfs_dg_wall_density). */
int dgfs_dg_advect(dgfs_dg_handle h, const void* u, void* ux, int32_t dtype,
                   void* stream);
int dgfs_dg_wall_density(dgfs_dg_handle h, double* out2);

/* State of a dgfs-wall-expr-diffuse wall for the following dgfs_dg_advect
 * calls: nondimensional velocity, temperature, and the species mass in the
 * exponent of its Maxwellian exp(-mass |c - u|^2 / T) (1 for one species).
 * Replaces the ux/uy/uz/T expressions of t rendered into
 * dgfs-wall-expr-diffuse.mako (std/bc.py:136-199, bi/bc.py:122-205): the
 * caller evaluates them at the stage time.  Host-side only; a CUDA graph
 * keeps the state it was captured with. */
int dgfs_dg_set_wall_state(dgfs_dg_handle h, int32_t side, double ux,
                           double uy, double uz, double T, double mass);

/* Bulk moments (FP64) at the Nqr reconstruction points of each element,
 * nondimensional, out[(r*Ne + e)*10 + i] for i = rho, Ux, Uy, T, Qx, Qy,
 * Pxx, Pyy, Pxy, (0) -- std/moments.py:11-60 before its dimensional scaling.
 * `out` is a device pointer. */
int dgfs_dg_moments(dgfs_dg_handle h, const void* coeff, int32_t dtype,
                    double* out, void* stream);

/* Moments of a mixture of nspcs <= 4 species sharing the grid of h
 * (replaces DGFSMomWriterBi._compute_moments_1D, bi/moments.py:11-113,
 * before its dimensional scaling): coeffs[p] is species p's solution
 * (K, Ne, N^3), masses[p] its nondimensional mass (host array); out (device)
 * receives out[((r*Ne + e)*nspcs + p)*5 + i] for i = rho, Ux, Uy, T, Qx.
 * T uses the species velocity, Qx the mixture velocity; a species whose
 * density summed over all points is below 1e-10 keeps rho, has zero U and T
 * and is left out of the mixture velocity, as in the reference. */
int dgfs_dg_moments_bi(dgfs_dg_handle h, const void* const* coeffs,
                       int32_t nspcs, const double* masses, int32_t dtype,
                       double* out, void* stream);

/* Residual sums (|x-y|^2, |y|^2) in FP64 (std/residual.py:15-29); waits for
 * the stream and writes the two sums to host memory out2. */
int dgfs_dg_residual(dgfs_dg_handle h, const void* x, const void* y, int64_t n,
                     int32_t dtype, double* out2, void* stream);

/* Linear slope limiter of dgfsABstd1D ([time-integrator] limiter = 1;
 * abstd.py:403-415, astd/kernels/limiters.mako:17-76), applied in place to a
 * (K, Ne, N^3) solution.  Tables: wavg[K] and wdr[K] are row 0 of the basis'
 * cell-average operator and of its differentiated linear projection
 * (basis.py:289-301), dx[K][Ne] the node positions minus the element centre,
 * hs[Ne] the element lengths. */
int dgfs_dg_set_limiter(dgfs_dg_handle h, const double* wavg, const double* wdr,
                        const double* dx, const double* hs);
int dgfs_dg_limit(dgfs_dg_handle h, void* u, int32_t dtype, void* stream);

/* Positivity limiter of dgfsABUstd1D (abstdu.py:432-441, limitPos of
 * astd/kernels/limiters.mako:198-227), in place on every element: u_k <-
 * a + theta (u_k - a), a the cell average, theta = min(1, |(a - 1e-13) /
 * (a - min_k u_k)|) rounded to single precision as there.  Needs the tables
 * of dgfs_dg_set_limiter. */
int dgfs_dg_limit_positivity(dgfs_dg_handle h, void* u, int32_t dtype,
                             void* stream);

/* Switch h's advection to the upwind summation-by-parts volume term of
 * dgfsABUstd1D (abstdu.py:355-383, upwind.mako): Dpos (K x K, row-major,
 * applied as ux = -c_x Dpos u) where c_x > 0 -- the reference's Dm^T -- and
 * Dneg (Dp^T) where c_x < 0; the face fluxes are unchanged.  swap != 0 gives
 * the ghost at each end the trace at the other end (abstdu.py:330-331, a
 * one-rank dgfs-cyclic right boundary); not with wall boundaries. */
int dgfs_dg_set_upwind(dgfs_dg_handle h, const double* Dpos, const double* Dneg,
                       int32_t swap);

/* Explicit ES-BGK relaxation of dgfsStd1D (esbgk-direct-gll, the fs of
 * std/scattering.py:1540-1637 with std/kernels/scattering/esbgk-direct-gll.mako)
 * on npts consecutive points of f (N^3 each, the grid of h): Q += prefac rho /
 * T^(omega-1) (f_ES - f), f_ES the Gaussian whose covariance is the discrete
 * second moment of (1-1/Pr) f + (1/Pr) f_M (f_M the grid Maxwellian of the
 * point), normalised by rho.  f and Q have the same dtype. */
int dgfs_std_esbgk_relax(dgfs_dg_handle h, const void* f, void* Q, int32_t dtype,
                         int32_t npts, double prefac, double omega, double Pr,
                         void* stream);

/* Switch h's advection to the entropy-stable volume term of dgfsABE2std1D
 * (abstde2.py:363-367, eDeriv of astd/kernels/limiters.mako:162-195):
 * ux_k = -2 c_x sum_l Dr[k][l] aveL(u_k, u_l), aveL the logarithmic mean, Dr
 * (K x K, row-major) the basis' derivMat; the face fluxes are unchanged. */
int dgfs_dg_set_entropy_stable(dgfs_dg_handle h, const double* Dr);

/*
 * Penalty (BGK-type) model of the penalised IMEX schemes, FP64 arithmetic
 * (dgfs1D/astd/scattering.py:44-284, astd/kernels/scattering/
 * bgk-direct-gll.mako).  Points are the npts = K*Ne slots of f; U holds five
 * moments per point: rho, rho ux, rho uy, rho uz, E = sum f |c|^2 cw, with
 * T = (E - |rho u|^2/rho)/(1.5 rho) and nu = prefac rho T^(1-omega).
 */
/* U = moments of f (replaces the cuBLAS gemm of astd/scattering.py:155-162). */
int dgfs_penalty_moments(dgfs_dg_handle h, const void* f, int32_t dtype,
                         int32_t npts, double* U, void* stream);
/* Closed-form implicit stage (updateDistribution{q}_BDF / _LM):
 * f = (rhs + cdt nu M(U)) / (adiv + cdt nu); optionally P = nu (M - f) and
 * the Maxwellian M (null to skip). */
int dgfs_penalty_implicit(dgfs_dg_handle h, const double* U, const void* rhs,
                          void* f, void* P, void* M, int32_t dtype,
                          int32_t npts, double adiv, double cdt, double prefac,
                          double omega, void* stream);
/* P = nu (M(U) - f) (collide, bgk-direct-gll.mako:157-181); M optional. */
int dgfs_penalty_collide(dgfs_dg_handle h, const double* U, const void* f,
                         void* P, void* M, int32_t dtype, int32_t npts,
                         double prefac, double omega, void* stream);

/*
 * ES-BGK and Shakov penalty models (astd/scattering.py:280-400,
 * astd/kernels/scattering/esbgk-direct-gll.mako, shakov-direct-gll.mako;
 * the boltz-* variants use the same kernels).  kind: 0 BGK (5 moments per
 * point), 1 ES-BGK (11: + sum f c_i c_j cw), 2 Shakov (14: + sum f |c|^2 c
 * cw), in the row order of the reference's moment matrices.  The Gaussian is
 * built from the moments inside the kernels (momentNorm + cmaxwellian).
 */
/* U[npts][nalph] = moments of f, nalph = 5, 11 or 14. */
int dgfs_penalty_moments_n(dgfs_dg_handle h, const void* f, int32_t dtype,
                           int32_t npts, int32_t nalph, double* U,
                           void* stream);
/* After the linear combination of a BDF / IMEX-LM moment update: the
 * implicit relaxation of the stresses (and the Shakov heat flux) towards the
 * model's targets (updateMom{q}_BDF: adiv = a_q, cdt = b dt; updateMom{q}_LM:
 * adiv = 1, cdt = c_0 dt).  A no-op for BGK. */
int dgfs_penalty_model_relax(dgfs_dg_handle h, int32_t kind, double* U,
                             int32_t npts, double adiv, double cdt,
                             double prefac, double omega, double Pr,
                             void* stream);
/* dgfs_penalty_implicit / _collide with the model's Gaussian G(U). */
int dgfs_penalty_model_implicit(dgfs_dg_handle h, int32_t kind,
                                const double* U, const void* rhs, void* f,
                                void* P, void* M, int32_t dtype, int32_t npts,
                                double adiv, double cdt, double prefac,
                                double omega, double Pr, void* stream);
int dgfs_penalty_model_collide(dgfs_dg_handle h, int32_t kind,
                               const double* U, const void* f, void* P,
                               void* M, int32_t dtype, int32_t npts,
                               double prefac, double omega, double Pr,
                               void* stream);

/* x0 <- a0 x0 + sum_i as[i] xs[i] over n elements, 1..4 terms, with the
 * a0 == 0 (x0 not read) and a0 == 1 branches of dgfs1D/axnpby.py:10-44. */
int dgfs_axnpby(void* x0, int64_t n, int32_t dtype, double a0, int32_t nterms,
                const void* const* xs, const double* as, void* stream);

/* Allocation-free Q(f,f) in FP64, for callers that cannot allocate device
 * memory: services whose device memory is a fixed pool carved out at
 * start-up (a cudaMalloc would fail or eat into the pool), plugins loaded
 * into a host process that forbids cudaMalloc once it is serving, and time
 * loops that cannot afford cudaMalloc's implicit device synchronisation.
 * No counterpart in the reference.  Same
 * semantics as creating a DGFS_PREC_FP64 handle from `desc` and calling
 * dgfs_vhs_eval with double f and Q, but no handle is created and nothing is
 * allocated: tables and scratch live in one static 16 MiB device array that
 * the library holds on every GPU that loads it.  Limits: N in {8, 16, 32},
 * Nrho <= 48, at most 96 sphere directions after merging antipodal pairs,
 * and the tables plus one evaluation must fit in 16 MiB (N=32 with
 * Nrho <= 16 does); larger shapes return DGFS_ERR_CAPACITY.  The first call
 * on a device sets it up (twiddle upload, symbol lookup) -- make that call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU race. */
int dgfs_vhs_eval_noalloc(const dgfs_vhs_desc* desc, const double* f,
                          double* Q, const int32_t* src_slots,
                          int32_t src_base, const int32_t* dst_slots,
                          int32_t dst_base, int32_t nevals, void* stream);

/* ---------------------------------------------------------------------------
 * Fourier-neural-operator surrogate of Q(f,f).  No counterpart in the
 * reference (a new learned component): 4 Fourier layers of width 32 with
 * `modes` retained modes per velocity axis (8 at N=16, 12 at N=32), GELU,
 * a 32 -> 128 -> 1 projection; input features f/rho, g, g r, g r^2 with
 * g = (f - M)/(rho sigma), sigma = rms((f - M)/rho), r = |c - u|/sqrt(T)
 * (M the local Maxwellian from FP64 moments), output
 * Q = rho^2 sigma q_scale * net(f),
 * followed by the FP64 conservation projection.  BF16 weights and
 * activations, FP32 accumulation.  Parameters are a flat FP32 vector
 * (dgfs_fno_num_params floats) set by the caller.
 * ------------------------------------------------------------------------- */
typedef struct dgfs_fno_s* dgfs_fno_handle;
typedef struct {
  int32_t N;          /* velocity grid points per axis: 16 or 32 */
  int32_t modes;      /* retained modes per axis: 8 (N=16) or 12 (N=32) */
  int32_t max_batch;  /* samples per launch, 1..32 (activation buffers) */
  double L;           /* velocity box half-width, grid c = linspace(-L+L/N, L-L/N, N) */
  double q_scale;     /* output scale: Q = rho^2 sigma q_scale net(f) */
} dgfs_fno_desc;

int dgfs_fno_create(const dgfs_fno_desc* desc, dgfs_fno_handle* out);
int dgfs_fno_destroy(dgfs_fno_handle h);
int64_t dgfs_fno_num_params(dgfs_fno_handle h);
/* Host FP32 parameter vector in / out (synchronous; set also resets Adam). */
int dgfs_fno_set_params(dgfs_fno_handle h, const float* host);
int dgfs_fno_get_params(dgfs_fno_handle h, float* host);
/* Gradients of the last dgfs_fno_train_step (synchronous copy). */
int dgfs_fno_get_grads(dgfs_fno_handle h, float* host);
/* Q[dst(i)] += surrogate Q(f[src(i)]), i < nevals; same slot conventions as
 * dgfs_vhs_eval (the drop-in replacement of that call). */
int dgfs_fno_eval(dgfs_fno_handle h, const void* f, int32_t f_dtype, void* Q,
                  int32_t q_dtype, const int32_t* src_slots, int32_t src_base,
                  const int32_t* dst_slots, int32_t dst_base, int32_t nevals,
                  void* stream);
/* One training step on B (f, Q) pairs (FP64, [B][N^3] each): forward, loss
 * mean_b |net - t|^2 / |t|^2 with t = Q/(rho^2 sigma q_scale), backward, and
 * (update != 0) one Adam step (beta 0.9/0.999, eps 1e-8, bias-corrected with
 * `step` >= 1). */
int dgfs_fno_train_step(dgfs_fno_handle h, const double* f, const double* Qt,
                        int32_t B, float lr, int32_t step, int32_t update,
                        void* stream);
/* Per-sample losses of the last training step (synchronous copy). */
int dgfs_fno_last_loss(dgfs_fno_handle h, double* host, int32_t B);
/* Dense layers and projection on the tcgen05 tensor cores (default, 1) or on
 * the CUDA cores (0; the reference implementation the tensor-core kernels
 * are tested against). */
int dgfs_fno_set_tensor_cores(dgfs_fno_handle h, int32_t enable);
/* Evaluation with the fused spectral kernels (default, 1: per layer an x-mix
 * launch and a yz-inverse + tensor-core dense launch, yz spectra by register
 * FFTs) or with the per-axis DFT passes that training uses (0).  The fused
 * path needs the tensor cores; with them disabled eval uses the passes. */
int dgfs_fno_set_fused(dgfs_fno_handle h, int32_t enable);
/* Device error flag of the tensor-core kernels (1: an MMA completion wait
 * timed out and the kernel stopped); synchronous, resets the flag. */
int dgfs_fno_error(dgfs_fno_handle h, int32_t* out);

/* Library identification and error reporting. */
const char* dgfs_version(void);
const char* dgfs_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif /* DGFS_SM100_H */

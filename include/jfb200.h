/*
 * jfb200.h — C ABI of the B200-native pseudo-spectral Galerkin Couette step.
 *
 * Plain C: device pointers, sizes and a CUDA stream handle (passed as void*,
 * the value of a cudaStream_t; NULL = legacy default stream).  Every entry
 * point returns an int status (JFB_OK == 0); jfb_last_error() returns a
 * thread-local description of the last failure.  No C++ exceptions cross
 * this boundary and no torch types appear in it.
 *
 * Each declaration cites the fnauman/jaxfun interface it replaces
 * (file:line within that project).  Complex arrays are interleaved
 * (re, im) float64 pairs (numpy/jax complex128 memory layout), C-ordered.
 */
#ifndef JFB200_H
#define JFB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define JFB_OK 0
#define JFB_ERR_ARG 1        /* invalid argument / unsupported shape         */
#define JFB_ERR_CUDA 2       /* a CUDA runtime call failed                   */
#define JFB_ERR_SINGULAR 3   /* zero or non-finite pivot (diamatrix.py:461)  */
#define JFB_ERR_NONFINITE 4  /* non-finite value detected in the state       */
#define JFB_ERR_STATE 5      /* call sequence error (e.g. no state set)      */
#define JFB_ERR_DEVICE 6     /* a bounded device-side wait gave up           */

/* ---- library ------------------------------------------------------------ */
int jfb_version(void);
const char* jfb_last_error(void);

/* ---- jaxfun.la DIA matrices --------------------------------------------- */

/* DiaMatrix.matvec(x, axis) / DiaMatrix.rmatvec(x, axis)
 * (src/jaxfun/la/diamatrix.py:227-283, 285-348).
 * Column-aligned DIA storage: data[d * n_cols + j] = A[j - offsets[d], j]
 * (diamatrix.py:100-123).  x is viewed as (outer, m, inner) with the
 * contracted axis in the middle; y as (outer, n, inner), where for
 * transpose == 0 (matvec) m = n_cols, n = n_rows and for transpose == 1
 * (rmatvec, x @ A) m = n_rows, n = n_cols.  is_complex selects interleaved
 * complex128 x / y; data is always real float64.  offsets is a host array. */
int jfb_dia_matvec(const double* data, const int64_t* offsets, int64_t n_diags,
                   int64_t n_rows, int64_t n_cols, const double* x, double* y,
                   int64_t outer, int64_t inner, int is_complex, int transpose,
                   void* stream);

/* Batched banded LU without pivoting (src/jaxfun/la/diamatrix.py:394-504,
 * kernel 1936-1973; batched use in tpmatrix.py:1105-1149).
 * band has shape (n_batch, p + q + 1, n) with band[b, p + off, j] =
 * A_b[j - off, j]; it is factored in place (multipliers in the sub-diagonal
 * rows, U in the rest).  Returns JFB_ERR_SINGULAR if any pivot is zero or
 * non-finite (diamatrix.py:461-471); synchronises the stream to check. */
int jfb_banded_lu_factor(double* band, int64_t n_batch, int64_t p, int64_t q,
                         int64_t n, void* stream);

/* Allocation-free variant of jfb_banded_lu_factor (no counterpart in the
 * reference).  For callers that cannot allocate device memory: an XLA custom
 * call or another framework's operator whose device memory belongs to that
 * framework's allocator, or a process whose caching pool already holds all
 * of the GPU's memory.  It factors the same batch in place with the same
 * arithmetic but keeps the per-matrix pivot status in a fixed device array of
 * the library (256 KiB per GPU, held until exit), so it calls no allocator.
 * n_batch must not exceed JFB_NOALLOC_LU_MAX_BATCH (else JFB_ERR_ARG).  On a
 * zero or non-finite pivot it returns JFB_ERR_SINGULAR and, if
 * first_singular is non-NULL, the lowest singular matrix index there (-1 when
 * none).  Synchronises `stream` (it reads that index back to the host).  The
 * first call on a device looks up the array's device address and keeps it
 * for the life of the process, so make that call before any stream capture,
 * and do not keep using the library on a device after cudaDeviceReset.  All
 * calls share the array: calls that overlap on the GPU (different streams or
 * threads) race. */
#define JFB_NOALLOC_LU_MAX_BATCH 65536
int jfb_banded_lu_factor_noalloc(double* band, int64_t n_batch, int64_t p, int64_t q,
                                 int64_t n, int32_t* first_singular, void* stream);

/* TPMatricesWavenumberSolver.solve / solve_many / *_with_runtime_args
 * (src/jaxfun/la/tpmatrix.py:1550-1677, batched recurrence 686-799).
 * L: (n_F, n_L, n_P) unit-lower sub-diagonals with L_offsets (< 0);
 * U: (n_F, n_U, n_P) with U_offsets (>= 0, containing 0).  Offsets are host
 * arrays.  rhs / out are (n_rhs, outer, n_P, inner) with n_F = outer*inner:
 * the polynomial axis sits between the Fourier axes exactly as in the
 * reference tensor (Fourier index flattened C-order, tpmatrix.py:1335-1357).
 * rhs and out may alias. */
int jfb_wavenumber_solve(const double* L, const int64_t* L_offsets, int64_t n_L,
                         const double* U, const int64_t* U_offsets, int64_t n_U,
                         int64_t n_P, int64_t outer, int64_t inner, int64_t n_rhs,
                         const double* rhs, double* out, int is_complex,
                         void* stream);

/* ---- KMM plane-Couette / channel step ----------------------------------- */

#define JFB_FAMILY_CHEBYSHEV 0
#define JFB_PRECISION_FP64 0
#define JFB_PRECISION_MIXED 1
/* nonlinear term (channelflow_kmm.py:754-770): rotational -(u x omega) or the
 * gradient form u . grad u (the reference's default) */
#define JFB_NONLINEAR_ROTATIONAL 0
#define JFB_NONLINEAR_GRADIENT 1
/* time integrators of KMM.step (channelflow_kmm.py:937-1192): SBDF3 with an
 * IMEXRK3 startup (sbdf3.py:15-62), the three-stage IMEXRK3 every step
 * (imex_rk.py:96-125, channelflow_kmm.py:872-935), the two-stage ARS
 * IMEXRK222 (imex_rk.py:175-198, integrators/coupled.py:13-44), CNAB2 with a
 * fixed step (channelflow_kmm.py:1071-1121, cnab2.py:185-240; a state's
 * history_steps holds the reference's have_old, 0 or 1) */
#define JFB_INTEGRATOR_SBDF3 0
#define JFB_INTEGRATOR_IMEXRK3 1
#define JFB_INTEGRATOR_IMEXRK222 2
#define JFB_INTEGRATOR_CNAB2 3

/* Constructor arguments of KMM / PlaneCouetteFluctuationJax
 * (examples/channelflow_kmm.py:107-230, examples/pcf_fluctuations_jax.py:35-75)
 * restricted to the hot path: Chebyshev or Legendre family, x unpadded, the
 * rotational or gradient nonlinear form, the time integrators above (MHD
 * plans: SBDF3, Chebyshev, rotational; the adjoint: also FP64).
 * u_wall = 0 gives the plain KMM channel (no base flow). */
typedef struct jfb_kmm_config {
  int32_t nx, ny, nz;     /* N = (wall-normal orthogonal size, Fourier y, z) */
  int32_t family;         /* JFB_FAMILY_CHEBYSHEV or JFB_FAMILY_LEGENDRE    */
  double x_lo, x_hi;      /* wall-normal domain                             */
  double ly, lz;          /* periodic lengths of the y and z axes           */
  double pad_y, pad_z;    /* dealiasing padding factors (1.5 = 3/2 rule)    */
  double nu;              /* kinematic viscosity                            */
  double dt;              /* fixed time step                                */
  double u_wall;          /* base flow U_b(x) = u_wall * x                  */
  int32_t precision;      /* JFB_PRECISION_FP64 or JFB_PRECISION_MIXED      */
  int32_t nonlinear_form; /* JFB_NONLINEAR_ROTATIONAL or _GRADIENT          */
  int32_t time_integrator; /* JFB_INTEGRATOR_* (0: SBDF3)                   */
} jfb_kmm_config;

/* Device pointers to a KMMState in the reference layout
 * (examples/channelflow_kmm.py:50-101): u0 (nx-4, ny, nz) complex128 in the
 * biharmonic basis; u1, u2, g (nx-2, ny, nz) complex128 in the Dirichlet
 * basis; history levels as (Nu | u0, Ng | g) complex plus (Nv00 | v00,
 * Nw00 | w00) float64 vectors of length nx-2. */
typedef struct jfb_kmm_state {
  void* u0;
  void* u1;
  void* u2;
  void* g;
  void* nonlinear_old[4];
  void* nonlinear_older[4];
  void* solution_old[4];
  void* solution_older[4];
  double history_steps;
} jfb_kmm_state;

typedef struct jfb_kmm_info {
  int64_t n_pencils;          /* stored (ky, kz >= 0) spectral pencils      */
  int64_t device_bytes;       /* device memory held by the plan             */
  int64_t launches_per_step;  /* kernels launched per steady SBDF3 step     */
  int64_t algorithmic_bytes;  /* stage-model HBM bytes per steady step      */
  int32_t my, mz;             /* padded quadrature counts                   */
} jfb_kmm_info;

typedef struct jfb_kmm_plan jfb_kmm_plan;

/* KMM.__init__ + _build_operators + lu_factor of Su/Sg/S00 and the three
 * IMEXRK3 startup factor sets (channelflow_kmm.py:107-444).  Allocates the
 * plan's device memory on the current device. */
int jfb_kmm_create(const jfb_kmm_config* cfg, jfb_kmm_plan** plan);
int jfb_kmm_destroy(jfb_kmm_plan* plan);
int jfb_kmm_get_info(const jfb_kmm_plan* plan, jfb_kmm_info* info);

/* Load / store the full KMMState (all history levels).  The plan keeps the
 * real-field (Hermitian, kz >= 0) half of every spectrum; set_state reads the
 * kz < nz/2 columns, get_state writes the full spectrum back using
 * c(-ky, -kz) = conj(c(ky, kz)). */
int jfb_kmm_set_state(jfb_kmm_plan* plan, const jfb_kmm_state* state,
                      void* stream);
int jfb_kmm_get_state(jfb_kmm_plan* plan, const jfb_kmm_state* state,
                      void* stream);

/* KMM.solve(state, steps) (channelflow_kmm.py:1231-1247): the IMEXRK3
 * startup steps while history_steps < 2 (_step_sbdf3, :937-1014), then
 * steady SBDF3 steps (_step_sbdf3_steady, :1016-1064), replayed from a CUDA
 * graph.  steps == 1 is KMM.step. */
int jfb_kmm_advance(jfb_kmm_plan* plan, int64_t steps, void* stream);

/* KMM.convection(state) (channelflow_kmm.py:772-782) of the loaded state:
 * writes the three dealiased TD coefficient fields H (nx-2, ny, nz) complex. */
int jfb_kmm_convection(jfb_kmm_plan* plan, void* h0, void* h1, void* h2,
                       void* stream);

/* KMM.state_from_physical (channelflow_kmm.py:677-683) as used by
 * PlaneCouetteFluctuationJax.initial_state (pcf_fluctuations_jax.py:77-97):
 * u0, u1, u2 are real float64 samples (nx, ny, nz) on the Gauss-Chebyshev x
 * nodes and the uniform y, z grids; loads TB/TD.forward of them (Nyquist
 * masked), g = i ky u2 - i kz u1, and a zero history (history_steps = 0). */
int jfb_kmm_state_from_physical(jfb_kmm_plan* plan, const double* u0,
                                const double* u1, const double* u2, void* stream);

/* PlaneCouetteFluctuationJax.diagnostics (pcf_fluctuations_jax.py:131-161) of
 * the loaded state, written to the device array out[8] = (Epert, Etot, divL2,
 * u_top, u_bot, wall_shear_top, wall_shear_bot, mean_shear).  Deterministic
 * fixed-order reduction. */
int jfb_kmm_diagnostics(jfb_kmm_plan* plan, double* out, void* stream);

/* The non-finite-state guard of the production runner
 * (production/oracles.py:3257-3261, `_tree_all_finite(candidate_state)` ->
 * FloatingPointError("nonfinite solver state ...")).  The step kernels set a
 * bit of a device status word of the plan when a solved coefficient (u0, g,
 * the mean flow, A) is NaN or infinite, the diagnostics when one of their
 * values is, and the tensor-core pencil stage when its bounded wait for a
 * bulk copy gave up.  This call synchronises `stream`, returns the word in
 * *flags (may be NULL), clears it, and returns JFB_ERR_NONFINITE if a
 * non-finite value was seen, JFB_ERR_DEVICE if a wait timed out, else
 * JFB_OK.  Cheap enough to call after every advance. */
int jfb_kmm_check(jfb_kmm_plan* plan, int32_t* flags, void* stream);

/* Measurement entry point (no reference counterpart; the reference's
 * production/benchmark.py:282-354 times blocks of KMM.solve with host
 * clocks): advances `steps` steady steps with the same kernels as
 * jfb_kmm_advance, launched without the graph and bracketed by CUDA events
 * on `stream`.  Before each step, if flush_buf is non-NULL, flush_bytes of it
 * are overwritten (an L2 flush outside the timed events).  Returns the summed
 * device time of each kernel slot (kernel_ms[4]: pencil stage, y backward,
 * z cross, y forward; when the plan fuses the periodic-axis transforms into
 * one launch, jfb_kmm_info.launches_per_step == 2, slot 1 holds that launch
 * and slots 2-3 are zero) and of the whole steps (step_ms).
 * IMEXRK3 startup steps still pending are run first and not timed. */
int jfb_kmm_timed_steps(jfb_kmm_plan* plan, int64_t steps, void* flush_buf,
                        int64_t flush_bytes, double* kernel_ms, double* step_ms,
                        void* stream);

/* perturbation_gain + jax.value_and_grad of it (examples/
 * pcf_minimal_seed_jax.py:111-150): runs `steps` steps from `init` (its
 * u0, u1, u2, g; history_steps must be 0, history pointers are ignored) and
 * writes gain = E(T) / E(0) (perturbation energies) to *gain_out (host).  If
 * grad is non-NULL, writes d gain / d init in jax.grad's convention (the
 * directional derivative along d is Re sum(grad * d) over the leaves) to
 * grad->u0, u1, u2, g (full-spectrum reference layout; the Hermitian
 * representative) and zeros to any history pointers given.  The gradient is
 * the hand-written discrete adjoint of the FP64 step (transposed transforms,
 * transposed banded solves, linearised rotational product) over a reverse
 * sweep that recomputes `checkpoint` steps at a time from stored states.
 * FP64 flow plans only.  The plan's loaded state is consumed. */
int jfb_kmm_gain_gradient(jfb_kmm_plan* plan, const jfb_kmm_state* init, int64_t steps,
                          int64_t checkpoint, double* gain_out, const jfb_kmm_state* grad,
                          void* stream);

/* jax.grad(perturbation_energy)(state) (pcf_minimal_seed_jax.py:125-137
 * uses it for the fixed-energy tangent): writes the gradient of
 * E = sum_f int |u_f|^2 with respect to u0, u1, u2 (jax.grad convention,
 * full-spectrum layout) and zeros to grad->g if given.  Loads `state`. */
int jfb_kmm_energy_gradient(jfb_kmm_plan* plan, const jfb_kmm_state* state,
                            const jfb_kmm_state* grad, void* stream);

/* ---- kernel variants and the autotuner --------------------------------- */

/* Kernel choices of a flow plan (no counterpart in the reference, whose XLA
 * compiler picks its own kernels): pencil 1 = the FP64 tensor-core pencil
 * stage (folded operators, needs nx <= 65), 0 = one warp per pencil;
 * transforms 1 = the fused plane transforms (one launch per step, padded
 * sizes 64 or 96), 0 = three launches; tc_velocity 1 = the mixed form's
 * velocity products on tcgen05 (split BF16, FP32 accumulation); pdl 1 =
 * programmatic dependent launch between the step kernels; replicas = copies
 * of the folded operators the CTAs spread their L2 reads over (1-16). */
typedef struct jfb_kmm_variant {
  int32_t pencil;
  int32_t transforms;
  int32_t tc_velocity;
  int32_t pdl;
  int32_t replicas;
} jfb_kmm_variant;

/* The plan's current variant (cur) and, field by field, the largest value
 * it accepts (avail); either may be NULL. */
int jfb_kmm_get_variant(const jfb_kmm_plan* plan, jfb_kmm_variant* cur, jfb_kmm_variant* avail);
/* Selects a variant (JFB_ERR_ARG if the plan cannot run it); drops the
 * captured step graphs. */
int jfb_kmm_set_variant(jfb_kmm_plan* plan, const jfb_kmm_variant* v);
/* Times every variant the plan accepts (replicas 4, 8, 16) on copies of the
 * loaded state: `steps` CUDA-graph steps each after five warm-up steps,
 * CUDA events on `stream`; selects the fastest, returns it in *best and its
 * time per step in *best_ms, and leaves the loaded state unchanged.  Only
 * choices with the same arithmetic are compared: tc_velocity (a different
 * accumulation precision) keeps its current value.  Allocates a temporary
 * copy of the state; flow plans only. */
int jfb_kmm_autotune(jfb_kmm_plan* plan, int64_t steps, jfb_kmm_variant* best, double* best_ms,
                     void* stream);

/* ---- plane-Couette MHD (vector potential, conducting walls) ------------- */

/* Device pointers to an MHDState (examples/pcf_mhd_jax.py:34-66): the flow
 * KMMState and the vector potential A in the Dirichlet basis, three
 * (nx-2, ny, nz) complex128 components per level, with its SBDF3 history
 * (the mass rows of the EMF and the two previous A levels). */
typedef struct jfb_mhd_state {
  jfb_kmm_state flow;
  void* A[3];
  void* nonlinear_A_old[3];
  void* nonlinear_A_older[3];
  void* A_old[3];
  void* A_older[3];
} jfb_mhd_state;

/* Magnetic parameters.  PlaneCouetteMHDJax (pcf_mhd_jax.py:76-115):
 * eta = U_wall / Rm, omega = 0, b0 = 0.  PlaneCouetteMRIShearpyJax
 * (pcf_mhd_mri_shearpy_jax.py:36-97, 149-176): eta = 1 / Rm, the rotation
 * rate omega (Coriolis term -2 omega e_z x u in the momentum nonlinear term)
 * and the imposed uniform field b0 (added to B in the Lorentz force and the
 * EMF); its base flow U_b = -shear_rate x is jfb_kmm_config.u_wall =
 * -shear_rate with nu = 1 / Re. */
typedef struct jfb_mhd_params {
  double eta;    /* magnetic diffusivity                     */
  double omega;  /* rotation rate of the frame               */
  double b0[3];  /* imposed uniform magnetic field (x, y, z) */
} jfb_mhd_params;

/* PlaneCouetteMHDJax.__init__ + _build_A_operators (pcf_mhd_jax.py:76-143):
 * the flow plan of jfb_kmm_create plus the A systems MA - gamma eta LA
 * (steady SBDF3 and the three IMEXRK3 startup stages).  FP64 only
 * (JFB_ERR_ARG for JFB_PRECISION_MIXED).  All other jfb_kmm_* entry points
 * accept the plan; jfb_kmm_advance / jfb_kmm_timed_steps then advance the
 * coupled flow + A system (_step_sbdf3_mhd, pcf_mhd_jax.py:563-715; Lorentz
 * force in the momentum nonlinear term, EMF in the A equation) and
 * jfb_kmm_convection returns H with the Lorentz force. */
int jfb_mhd_create(const jfb_kmm_config* cfg, const jfb_mhd_params* params,
                   jfb_kmm_plan** plan);

/* Load / store the full MHDState; the flow part as jfb_kmm_set_state /
 * jfb_kmm_get_state.  NULL A-history pointers load zeros (get: skipped). */
int jfb_mhd_set_state(jfb_kmm_plan* plan, const jfb_mhd_state* state, void* stream);
int jfb_mhd_get_state(jfb_kmm_plan* plan, const jfb_mhd_state* state, void* stream);

/* _A_state_from_physical (pcf_mhd_jax.py:210-215): TD.forward (Nyquist
 * masked) of real float64 samples (nx, ny, nz) of the three components of A,
 * written to a0, a1, a2 ((nx-2, ny, nz) complex128).  The loaded state is
 * unchanged. */
int jfb_mhd_potential_from_physical(jfb_kmm_plan* plan, const double* ax, const double* ay,
                                    const double* az, void* a0, void* a1, void* a2,
                                    void* stream);

/* _mhd_convection (pcf_mhd_jax.py:339-357) of the loaded state: H (the TD
 * forward of -(u_t x omega_t) - J x B) and HA (the TD forward of
 * (u + U_b e_y) x B), six (nx-2, ny, nz) complex128 fields. */
int jfb_mhd_convection(jfb_kmm_plan* plan, void* h0, void* h1, void* h2, void* ha0,
                       void* ha1, void* ha2, void* stream);

/* PlaneCouetteMHDJax.diagnostics (pcf_mhd_jax.py:776-790) of the loaded
 * state: device array out[10] = the eight values of jfb_kmm_diagnostics,
 * then divB_L2 and Emag. */
int jfb_mhd_diagnostics(jfb_kmm_plan* plan, double* out, void* stream);

/* ---- tensor-product spaces ------------------------------------------------ */

#define JFB_BASIS_ORTHOGONAL 0  /* T_k / P_k of the family                   */
#define JFB_BASIS_DIRICHLET 1   /* P_k - P_{k+2} (Composite, u(+-1) = 0)      */
#define JFB_BASIS_BIHARMONIC 2  /* u(+-1) = u'(+-1) = 0 (Composite)           */
#define JFB_FAMILY_LEGENDRE 1   /* family of a tensor-product space x axis    */

/* TensorProduct(orthogonal-family x axis, Fourier[, Fourier])
 * (src/jaxfun/galerkin/tensorproductspace.py:104-293): n[0] Gauss points of
 * the family (Gauss-Chebyshev, Chebyshev.py:159-180, or Gauss-Legendre,
 * Legendre.py:136-147) on [x_lo, x_hi], n[1] (and n[2]) Fourier modes on
 * periods l[0] (l[1]), padding factors pad[] for the padded backward /
 * forward (get_dealiased: max(N, int(pad N)) points).  The wall-normal
 * transforms are dense Vandermonde contractions (orthogonal.py:121-145,
 * 240-331) with the Shen stencil folded in. */
typedef struct jfb_tps_config {
  int32_t ndim;   /* 2: (x, y), 3: (x, y, z) */
  int32_t basis;  /* JFB_BASIS_*             */
  int32_t n[3];
  double x_lo, x_hi;
  double l[2];
  double pad[2];
  int32_t family; /* JFB_FAMILY_CHEBYSHEV or JFB_FAMILY_LEGENDRE */
} jfb_tps_config;

typedef struct jfb_tps jfb_tps;
int jfb_tps_create(const jfb_tps_config* cfg, jfb_tps** tps);
int jfb_tps_destroy(jfb_tps* tps);
/* out4 = (basis dofs nb, quadrature points N, padded counts m1, m2). */
int jfb_tps_get_sizes(const jfb_tps* tps, int32_t* out4);

/* TensorProductSpace.backward (tensorproductspace.py:253-293, 553-594):
 * coeffs (nb, n1[, n2]) complex128 -> phys (N, m1[, m2]) complex128, m = n
 * unpadded or the padded counts when padded != 0 (Fourier.py:128-150). */
int jfb_tps_backward(jfb_tps* tps, const void* coeffs, void* phys, int padded, void* stream);

/* kind 0: TensorProductSpace.forward (tensorproductspace.py:529-551; the L2
 * projection along x, Fourier.forward scaled 1/M and truncated, Nyquist kept);
 * kind 1: scalar_product (per-axis scalar products, Fourier weight 2 pi / df).
 * phys (N, m1[, m2]) -> coeffs (nb, n1[, n2]). */
int jfb_tps_forward(jfb_tps* tps, const void* phys, void* coeffs, int padded, int kind,
                    void* stream);

/* Galerkin x-matrix (phi_i, phi_j^(order))_w, order 0 or 2, dense row-major
 * nb x nb on the host (the 1-D mass / stiffness of inner.py, domain-scaled). */
int jfb_tps_galerkin(const jfb_tps* tps, int order, double* out);

/* TensorProductSpace.backward_primitive(c, k) (tensorproductspace.py:553-594):
 * the mixed derivative d^k0/dx^k0 d^k1/dy^k1 [d^k2/dz^k2] of the field on the
 * (padded) mesh; coeffs (nb, n1[, n2]) -> phys as jfb_tps_backward.  Along x
 * the derivative is taken on the orthogonal coefficients (chebder / legder,
 * domain-scaled); along Fourier axes (i m df)^k with the Nyquist mode zeroed
 * for odd k (Fourier.py:210-223).  k: ndim non-negative orders. */
int jfb_tps_backward_primitive(jfb_tps* tps, const void* coeffs, void* phys, const int32_t* k,
                               int padded, void* stream);

/* TensorProductSpace.to_orthogonal (tensorproductspace.py:596-616):
 * coeffs (nb, n1[, n2]) -> orthogonal coefficients (N, n1[, n2]) (c @ S). */
int jfb_tps_to_orthogonal(jfb_tps* tps, const void* coeffs, void* orth, void* stream);

/* TensorProductSpace.differentiate_orthogonal_coeffs(c, k)
 * (tensorproductspace.py:638-682): orthogonal coefficients (N, n1[, n2]) ->
 * the coefficients of the k-th mixed derivative, same shape. */
int jfb_tps_differentiate_orthogonal(jfb_tps* tps, const void* orth, void* out, const int32_t* k,
                                     void* stream);

/* TensorProductSpace.project_from_orthogonal (tensorproductspace.py:706-728;
 * composite.py:292-298 per axis): Galerkin projection of orthogonal
 * coefficients (N, n1[, n2]) into this space (nb, n1[, n2]): mass-weight,
 * stencil, mass solve; Fourier axes are identities. */
int jfb_tps_project_from_orthogonal(jfb_tps* tps, const void* orth, void* coeffs, void* stream);

/* TensorProductSpace.scalar_product_from_orthogonal (tensorproductspace.py:
 * 730-754; composite.py:300-305): scalar products of the field given by
 * orthogonal coefficients (N, n1[, n2]) -> (nb, n1[, n2]); Fourier axes
 * multiply by their mass 2 pi / df. */
int jfb_tps_scalar_product_from_orthogonal(jfb_tps* tps, const void* orth, void* out,
                                           void* stream);

/* The 2-D Helmholtz solve -lap u + alpha u = f of la/solvers.py:22-61 as one
 * launch: orthogonal-Chebyshev x Fourier coefficients f_hat (N, n1) ->
 * backward of tc, scalar products of td divided by fourier_mass, the
 * per-wavenumber banded solve with the no-pivot LU factors (L, U) of
 * TPMatricesWavenumberSolver (tpmatrix.py:1550-1677; DIA data (n1, n_diag,
 * N - 2), L offsets < 0, U offsets >= 0 with 0), backward of td -> u (N, n1)
 * complex128.  tc: 2-D, JFB_BASIS_ORTHOGONAL; td: 2-D, JFB_BASIS_DIRICHLET,
 * same sizes.  One cluster of 8 CTAs holds the whole problem in distributed
 * shared memory (per CTA 16 (2 N c + N q + 2 n1 ceil(N/8)) + 8 N (N - 2)
 * bytes, c = ceil(n1/8), q = c rounded up to 1 mod 4): JFB_ERR_ARG when that
 * exceeds a CTA's shared memory (use the separate transforms and
 * jfb_wavenumber_solve then).  U_inv (optional, N - 2 <= 128): the inverse of
 * each mode's U, (n1, N - 2, N - 2) with entry (r, c) at c (N - 2) + r; with
 * it and L offsets among {-2, -4} the solve is two short recurrences and a
 * product (no dependent column chain); NULL: column-oriented substitution. */
int jfb_helmholtz2d_solve(const jfb_tps* tc, const jfb_tps* td, const double* L,
                          const int64_t* L_offsets, int64_t n_L, const double* U,
                          const int64_t* U_offsets, int64_t n_U, const double* U_inv,
                          double fourier_mass, const void* f_hat, void* u, void* stream);

/* ---- ensembles ------------------------------------------------------------ */

/* Independent members (flow or MHD plans, any sizes; no reference counterpart:
 * the reference runs members one solver at a time, pcf_mhd_mri_shearpy_jax.py
 * / pcf_mhd_jax.py:563-715 per member) advanced together, one CUDA graph per
 * steady step.  When every member is an MHD plan on the tensor-core pencil
 * stage with warp-FFT y transforms of one length (up to 64 members of any
 * wall-normal size), the step is FIVE launches, one per stage over all
 * members' tiles (a work list; JFB200_ENSEMBLE=streams disables it);
 * otherwise every member's step runs on its own stream.  Both forms give
 * bitwise the results of the members' own plans.  Members keep their own
 * states (jfb_kmm_set_state / jfb_mhd_set_state, get_state); all must share
 * the step phase and history count when advanced.  Destroy the ensemble
 * before its members. */
typedef struct jfb_ensemble jfb_ensemble;
int jfb_ensemble_create(jfb_kmm_plan* const* plans, int32_t n, jfb_ensemble** ensemble);
int jfb_ensemble_advance(jfb_ensemble* ensemble, int64_t steps, void* stream);
/* *batched = 1 for the five-launch form; *launches_per_step = kernels per
 * steady step of the whole ensemble (either may be NULL). */
int jfb_ensemble_info(const jfb_ensemble* ensemble, int32_t* batched, int64_t* launches_per_step);
int jfb_ensemble_destroy(jfb_ensemble* ensemble);

#ifdef __cplusplus
}
#endif

#endif /* JFB200_H */

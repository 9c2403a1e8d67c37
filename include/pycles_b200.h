/*
 * pycles_b200 -- C ABI of the B200 (sm_100a) PyCLES hot path.
 *
 * Every entry point takes plain pointers and sizes (device pointers unless
 * stated otherwise), a CUDA stream as `void*` (NULL = legacy default
 * stream), is stream-ordered, never synchronises the host, allocates no
 * device memory, and returns a pb_status.  Fields use the reference layout:
 * flat ghosted [i][j][k] arrays, k contiguous, length npg each, as held in
 * PrognosticVariables.values / DiagnosticVariables.values
 * (PrognosticVariables.pyx:78-79, DiagnosticVariables.pyx).
 *
 * Numerical failures detected on the device (pv* table range, secant
 * iteration cap, non-finite temperatures) are OR-ed into a device error
 * word that pb_get_error() reads; they do not make a call return non-zero.
 */
#ifndef PYCLES_B200_H
#define PYCLES_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum pb_status {
  PB_OK = 0,
  PB_ERR_ARG = 1,          /* invalid shape, null pointer, bad enum      */
  PB_ERR_CUDA = 2,         /* a CUDA runtime call or launch failed       */
  PB_ERR_UNSUPPORTED = 3,  /* valid for the reference, not built here    */
  PB_ERR_WORKSPACE = 4     /* workspace missing or too small             */
};

/* Arithmetic form of the advection / FFT paths. */
enum pb_precision {
  PB_FP64 = 0,             /* plain form: the reference method in FP64  */
  PB_FP32 = 1              /* fluxes in FP32, divergence accumulated in FP64 */
};

/*
 * Grid geometry.  Field for field (types and order) the reference's
 * struct DimStruct (Csrc/grid.h:2-24), so a Cython caller can pass
 * &Grid.dims directly.  One rank holds the whole domain: nl == n,
 * nlg == n + 2*gw, indx_lo == 0.
 */
typedef struct pb_dims {
  long dims;
  long n[3];
  long ng[3];
  long nl[3];
  long nlg[3];
  long npd;
  long npl;
  long npg;
  long gw;
  long indx_lo[3];
  long indx_lo_g[3];
  long nbuffer[3];
  long ghosted_stride[3];
  double dx[3];
  double dxi[3];
} pb_dims;

/*
 * Saturation vapour pressure table on the device: the reference's
 * LookupStruct (Csrc/lookup.h:4-13) with y in device memory.
 * x_min = min(T), dx = T[1]-T[0], dxi = 1/dx as init_table computes them.
 */
typedef struct pb_table {
  const double* y;
  long n;
  double x_min;
  double dx;
  double dxi;
} pb_table;

/*
 * Learned saturation-adjustment seed: a 3->64->64->1 SiLU MLP with BF16
 * weights (device pointers), inputs (p0, s, qt) mapped affinely to [-1,1]
 * by in_lo/in_hi; the seed is T = T_1 + out_mean + out_scale * y with T_1
 * the secant's first point (the network learns the correction to it).
 * Weight layouts: w1 [64][3], w2 [64][64], w3 [64] (row = output unit),
 * biases FP32.  seed_y: the seed's state between pb_thermo_sa calls, a
 * device float[npg] owned by the caller and zeroed before the first call
 * (the network's output y per cell); seed_refresh: whether pb_thermo_sa
 * re-evaluates the network into seed_y before its kernel (a caller may
 * refresh once per time step rather than once per RK stage: y moves ~1e-4 K
 * within a step, the network's own error is ~1e-2 K).  Both are unused by
 * pb_mlp_forward / pb_mlp_grad.
 */
typedef struct pb_mlp {
  const void* w1;   /* bf16 [64*3]  */
  const float* b1;  /* [64]         */
  const void* w2;   /* bf16 [64*64] */
  const float* b2;  /* [64]         */
  const void* w3;   /* bf16 [64]    */
  const float* b3;  /* [1]          */
  float in_lo[3];
  float in_hi[3];
  float out_mean;
  float out_scale;
  float* seed_y;    /* [npg], see above */
  int seed_refresh; /* pb_thermo_sa: nonzero = refresh seed_y first */
} pb_mlp;

/* ------------------------------------------------------------------------
 * Advection
 * --------------------------------------------------------------------- */

/*
 * ScalarAdvection.update (ScalarAdvection.pyx:69-123) without the
 * sedimentation branch: for every scalar and every direction d, the face
 * fluxes of compute_advective_fluxes_a (Csrc/scalar_advection.h:689-730;
 * WENO5 :319-394, WENO7 :396-480) and their divergence
 * scalar_flux_divergence (Csrc/flux_divergence.h:4-32), subtracted from the
 * scalar's tendency over the interior, d = 0, 1, 2 in that order.
 *   scalars, tendencies : HOST arrays of nscalars device pointers.
 *   flux (nullable)     : nscalars*3*npg doubles, [scalar][d][ijk] as
 *                         ScalarAdvection.flux (:55); written on the faces
 *                         the divergence reads (interior cells in the other
 *                         two directions, faces gw-1 .. nlg-gw-1 along d).
 *   order               : 5 or 7 (needs gw >= 3 resp. gw >= 4).
 */
int pb_scalar_advection(const pb_dims* dims, const double* rho0, const double* rho0_half,
                        const double* alpha0, const double* alpha0_half, const double* u,
                        const double* v, const double* w, int nscalars,
                        const double* const* scalars, double* const* tendencies, double* flux,
                        int order, int precision, void* stream);

/*
 * The precision form's scalar advection (as pb_scalar_advection with
 * PB_FP32, no flux output) fused with the scalars' SSP-RK3 stage
 * (TimeStepping.update_third, TimeStepping.pyx:131-151) for a step driver
 * that owns the whole stage (no counterpart in the reference).  The
 * tendencies are taken to hold nothing but the advection: the x pass stores
 * its term, the y pass adds, the z pass applies the stage; they are left
 * holding the x and y terms.  New interior values go to new_values[i]
 * (arrays other than scalars[i]), the stage-0 copies to copies[i]; ghosts
 * are left for the ghost fill that follows the stage.  HOST arrays of
 * device pointers, as for pb_scalar_advection.
 */
int pb_scalar_advection_rk3(const pb_dims* dims, const double* rho0, const double* rho0_half,
                            const double* alpha0, const double* alpha0_half, const double* u,
                            const double* v, const double* w, int nscalars,
                            const double* const* scalars, double* const* tendencies,
                            double* const* new_values, double* const* copies, double dt, int rk_step,
                            int order, void* stream);

/*
 * MomentumAdvection.update (MomentumAdvection.pyx:41-69): for advected
 * component a and advecting direction d (a, d = 0..2 in that order),
 * compute_advective_tendencies_m (Csrc/momentum_advection.h:13-93; WENO5
 * Csrc/momentum_advection_weno.h:113-245, WENO7 :247-400) including its
 * momentum_flux_divergence (Csrc/flux_divergence.h:34-60).  The reference
 * mallocs a flux array per call; this path needs none.
 */
int pb_momentum_advection(const pb_dims* dims, const double* rho0, const double* rho0_half,
                          const double* alpha0, const double* alpha0_half, const double* u,
                          const double* v, const double* w, double* ut, double* vt, double* wt,
                          int order, int precision, void* stream);

/*
 * The precision form's momentum advection (as pb_momentum_advection with
 * PB_FP32) fused with the SSP-RK3 stage of u, v, w (TimeStepping.update_third,
 * TimeStepping.pyx:131-151) for a step driver that owns the whole stage (no
 * counterpart in the reference; PB_FP32 arithmetic).  The u and v
 * tendencies are taken to hold nothing but the advection (they are neither
 * read nor written); wt holds the w tendency accumulated before the call
 * (the thermodynamics' buoyancy) and is only read (the caller clears it
 * before the next stage's accumulation).  The new
 * interior values go to u_new, v_new, w_new (arrays other than u, v, w:
 * neighbouring cells are still being read), the stage-0 copies to
 * u_copy.. at rk_step 0; ghosts of the new arrays are left for the ghost
 * fill that follows the stage.
 */
int pb_momentum_advection_rk3(const pb_dims* dims, const double* rho0, const double* rho0_half,
                              const double* alpha0, const double* alpha0_half, const double* u,
                              const double* v, const double* w, double* wt, double* u_new,
                              double* v_new, double* w_new, double* u_copy, double* v_copy,
                              double* w_copy, double dt, int rk_step, int order, void* stream);

/* ------------------------------------------------------------------------
 * Thermodynamics
 * --------------------------------------------------------------------- */

/*
 * ThermodynamicsSA.update (ThermodynamicsSA.pyx:176-213): clip_qt
 * (Csrc/thermodynamics_sa.h:213-219) when clip_qt != 0, eos_update
 * (:68-96, per-cell eos_c secant :17-66 and alpha_c), buoyancy_update_sa
 * (:98-132, adds to w_tend), bvf_sa (:134-182), thetali_update (:185-211).
 * Latent heat: latent_heat_variable, lambda = 1 (Microphysics.pxd:65-75).
 *   mlp (nullable)        : learned seed for the secant's second point
 *                           (no counterpart in the reference; precision
 *                           PB_FP32 only; mlp->seed_y required).  First,
 *                           if mlp->seed_refresh, the network refreshes
 *                           seed_y = MLP(p0, s, qt) for every cell with
 *                           ql > 0 on entry (saturated at the previous
 *                           call); then each saturated cell
 *                           starts its secant from T_2 = T_1 + out_mean +
 *                           out_scale * seed_y, clamped to the bracket
 *                           [T_1 + (T_2r - T_1)/16, T_2r] of the root (T_1
 *                           the first point :22-24, T_2r the reference's
 *                           second point :39).  The refresh sets seed_y to
 *                           NaN for the cells it does not evaluate: those
 *                           (saturated since the last refresh) start from
 *                           T_2r.  The secant's stopping test decides every
 *                           result.
 *   secant_iters (nullable): device long long[2]; receives
 *                           {sum of secant iterations, saturated cells}.
 *   max_iter              : secant iteration cap (the reference has none);
 *                           reaching it sets PB_ERR_SECANT_CAP in the error word.
 *   precision             : PB_FP64 (plain form: correctly rounded exp/log,
 *                           no FMA contraction, the reference's roundings) or
 *                           PB_FP32 (precision form: FP64 arithmetic with
 *                           CUDA's exp/log and FMA, optional learned seed).
 */
int pb_thermo_sa(const pb_dims* dims, const double* p0_half, const double* alpha0_half,
                 const pb_table* table, const double* s, double* qt, double* T, double* qv,
                 double* ql, double* qi, double* alpha, double* buoyancy, double* theta_rho,
                 double* bvf, double* thetali, double* w_tend, int clip_qt, const pb_mlp* mlp,
                 long long* secant_iters, int max_iter, int precision, void* stream);

/*
 * ThermodynamicsDry.update (ThermodynamicsDry.pyx:105-120): eos_update
 * (Csrc/thermodynamics_dry.h:12-37), buoyancy_update (:39-73, adds to
 * w_tend), bvf_dry (:75-110).  pd is RS.p0_half as the reference passes it.
 * precision as for pb_thermo_sa (without a seed).
 */
int pb_thermo_dry(const pb_dims* dims, const double* p0_half, const double* alpha0_half,
                  const double* s, double* T, double* alpha, double* buoyancy, double* theta,
                  double* bvf, double* w_tend, int precision, void* stream);

/*
 * ThermodynamicsSA.eos (ThermodynamicsSA.pyx:169-174) for n points: eos_c
 * (Csrc/thermodynamics_sa.h:17-66, FP64 plain form) on (p0[i], s[i], qt[i])
 * -> T[i], ql[i], qi[i] (ql, qi nullable), T_first[i] = the secant's first
 * point T_1 (:22-24; nullable), iters[i] = secant iterations (nullable; 0
 * for unsaturated points).  seed (nullable) replaces the secant's second
 * point.
 */
int pb_eos_sa(const pb_table* table, const double* p0, const double* s, const double* qt,
              const double* seed, double* T, double* ql, double* qi, double* T_first, int* iters,
              long long n, int max_iter, void* stream);

/* ------------------------------------------------------------------------
 * Learned seed (no counterpart in the reference).  BF16 tensor-core
 * (mma.sync m16n8k16, FP32 accumulation) forward and backward passes of the
 * 3 -> 64 -> 64 -> 1 SiLU MLP of pb_mlp.  Packed FP32 parameter vector
 * (PB_MLP_NPARAM = 4481): W1[64][3], b1[64], W2[64][64], b2[64], w3[64], b3.
 * --------------------------------------------------------------------- */
#define PB_MLP_NPARAM 4481

/*
 * T_seed[i] = T_1 + out_mean + out_scale * MLP(normalised p0[i], s[i], qt[i]),
 * T_1 the secant's first point (Csrc/thermodynamics_sa.h:22-24, evaluated
 * with the precision form's arithmetic): the seed pb_thermo_sa uses.
 */
int pb_mlp_forward(const pb_mlp* mlp, const double* p0, const double* s, const double* qt,
                   double* T_seed, long long n, void* stream);

/*
 * The learned seed's refresh on the 5th-generation tensor cores (tcgen05,
 * FP32 accumulators in tensor memory): net->seed_y[cell] = the network's
 * output y for every cell with ql > 0, NaN elsewhere -- what pb_thermo_sa
 * runs before its kernel when net->seed_refresh is set.  p0_half per level;
 * s, qt, ql ghosted fields.  No counterpart in the reference.
 */
int pb_mlp_refresh_seed(const pb_mlp* net, const pb_dims* dims, const double* p0_half, const double* s,
                        const double* qt, const double* ql, void* stream);

/*
 * Adds the gradient of sum_i 0.5 (MLP(x_i) - target_i)^2 to grad[PB_MLP_NPARAM]
 * and the loss sum to *loss (both FP32, device, accumulated).  x: n x 3
 * inputs already normalised to [-1, 1]; target: n normalised outputs.
 * workspace: device scratch of at least pb_mlp_grad_workspace_bytes(n)
 * bytes, 16-byte aligned (PB_ERR_WORKSPACE otherwise), for the per-block
 * partial sums.  The result is deterministic: the partials are added in a
 * fixed order (no floating-point atomics), so the same inputs give the same
 * gradient bit for bit.  No counterpart in the reference.
 */
long long pb_mlp_grad_workspace_bytes(long long n);
int pb_mlp_grad(const pb_mlp* mlp, const float* x, const float* target, long long n, float* grad,
                float* loss, void* workspace, long long workspace_bytes, void* stream);

/*
 * One Adam step on the FP32 master parameters (grad scaled by grad_scale),
 * then refreshes the BF16 weights and FP32 biases the kernels read.
 */
int pb_mlp_adam(float* params, float* m, float* v, const float* grad, int step, float lr, float beta1,
                float beta2, float eps, float grad_scale, void* w1, float* b1, void* w2, float* b2,
                void* w3, float* b3, void* stream);

/* ------------------------------------------------------------------------
 * Time stepping and boundary conditions
 * --------------------------------------------------------------------- */

/*
 * TimeStepping.update_third (TimeStepping.pyx:131-151) over n values
 * (nv*npg, ghosts included): SSP-RK3 stage rk_step (0, 1, 2), tendencies
 * zeroed afterwards.  value_copy is TimeStepping.value_copies[0].
 */
int pb_rk3_update(double* values, double* tendencies, double* value_copy, long long n, double dt,
                  int rk_step, void* stream);

/*
 * pb_rk3_update with the new values written to values_out (which may be
 * values itself): the out-of-place form used with
 * pb_momentum_advection_rk3, whose new velocities go to a second buffer.
 */
int pb_rk3_update_to(const double* values, double* values_out, double* tendencies, double* value_copy,
                     long long n, double dt, int rk_step, void* stream);

/*
 * PrognosticVariables.update_all_bcs (PrognosticVariables.pyx:183-233) on
 * one periodic-x,y rank, and DiagnosticVariables.communicate_variable
 * (DiagnosticVariables.pyx:65-112) when nv == 1: x and y ghost planes from
 * the opposite interior planes (build_buffer / buffer_to_values,
 * Csrc/prognostic_variables.h:11-203), z ghosts by set_bcs (:205-270) with
 * bc_factor 1 (sym), -1 (asym) or 2.  values holds nv fields spaced npg;
 * bc_factor is a HOST array of nv doubles.
 */
int pb_update_all_bcs(const pb_dims* dims, double* values, const double* bc_factor, int nv,
                      void* stream);

/* ------------------------------------------------------------------------
 * Pressure
 * --------------------------------------------------------------------- */

/* Bytes of device scratch pb_pressure_solve needs for this grid. */
long long pb_pressure_workspace_bytes(const pb_dims* dims);

/*
 * PressureFFTParallel.initialize (PressureFFTParallel.pyx:27-62): fills the
 * grid constants of the workspace -- the modified wave numbers of
 * compute_modified_wave_numbers (:64-98), evaluated on the host with the C
 * library cos exactly as the reference evaluates them, and the FFT twiddle
 * factors.  Synchronous; call once per workspace before pb_pressure_solve.
 */
int pb_pressure_init(const pb_dims* dims, void* workspace, long long workspace_bytes);

/*
 * PressureSolver.update (PressureSolver.pyx:38-80) up to, not including,
 * its final PV.update_all_bcs: w -= HorizontalMean(w) (ParallelMPI.pyx:
 * 196-241, remove_mean_u3 :113-136), divergence = second_order_divergence
 * (:138-175), PressureFFTParallel.solve (PressureFFTParallel.pyx:150-219:
 * horizontal FFT, per-(kx,ky) tridiagonal solve with modified wave numbers
 * :64-98 and the matrix of :100-148, mode (0,0) zeroed, inverse FFT, real
 * part; SparseSolvers.TDMA :24-44), the sym ghost fill of the pressure
 * (DiagnosticVariables.communicate_variable) and
 * second_order_pressure_correction (:83-110).
 *   workspace : >= pb_pressure_workspace_bytes(dims) bytes, 256-byte aligned,
 *               initialised by pb_pressure_init.
 *   n[0], n[1] : powers of two up to 4096 (Stockham radix-8 FFTs), other
 *                sizes up to 1024 (direct DFT); PB_ERR_UNSUPPORTED otherwise.
 *   precision  : PB_FP64 -- the reference method in FP64 (refine_sweeps
 *                ignored).  PB_FP32 -- the precision form: FFTs in FP32,
 *                tridiagonal solves in FP64, then refine_sweeps (0..8)
 *                iterative-refinement sweeps p += solve(div - A p) with the
 *                residual evaluated in FP64 (no counterpart in the reference).
 */
int pb_pressure_solve(const pb_dims* dims, const double* rho0, const double* rho0_half,
                      const double* alpha0, const double* alpha0_half, double* u, double* v,
                      double* w, double* divergence, double* dynamic_pressure, void* workspace,
                      long long workspace_bytes, int precision, int refine_sweeps, void* stream);

/* ------------------------------------------------------------------------
 * Pressure solve of a domain split across GPUs (x-slabs: full y and z)
 *
 * The reference decomposes the domain over MPI ranks and transposes the
 * spectral data between pencils with MPI_Alltoallv (ParallelMPI.pyx:542-1068,
 * PressureFFTParallel.pyx:150-219) around the same mathematics as the
 * single-rank solve.  Here the solve is cut into phases; between them the
 * caller exchanges data between GPUs (all-to-all, halo exchange):
 *   divergence (x-slab) -> [x-slab to z-slab] -> fft_forward (z-slab: every
 *   column, a range of levels) -> [z-slab to row slab] -> fft_columns (every
 *   level, a range of rows j) -> [back] -> fft_inverse -> [back to x-slab]
 *   -> ghost fill + x-halo exchange of the pressure -> correct.
 * Dense arrays are the interior cells [i][j][k] (k fastest) of the slab.
 * The spectral arithmetic is the single-GPU solve's (the same kernels).
 * ------------------------------------------------------------------------ */

/* Byte offset of the spectral array W[k][j][m] (n2 levels of n1 rows of
 * n0/2 + 1 complex values) in a workspace of pb_pressure_workspace_bytes(dims),
 * for a caller that moves it between GPUs; -1 for invalid dims. */
long long pb_pressure_spectral_offset(const pb_dims* dims);

/* Per-level sums of `field` over this grid's interior columns, i outer and j
 * inner as HorizontalMean adds them (ParallelMPI.pyx:219-226), unscaled:
 * sums[nlg2].  A sharded mean adds the GPUs' sums, then scales by
 * 1/(n0 n1) of the whole domain (ParallelMPI.pyx:229-236). */
int pb_horizontal_sums(const pb_dims* dims, const double* field, double* sums, void* stream);

/* PressureSolver.update's divergence (PressureSolver.pyx:113-175) on the
 * cells of this slab: w - mean[k] (remove_mean_u3; mean has nlg2 values),
 * then second_order_divergence, written to `divergence` (ghosts zero) and,
 * when div_dense is not NULL, to a dense interior array.  The x-ghost planes
 * of u must hold the neighbouring slab's values. */
int pb_pressure_divergence(const pb_dims* dims, const double* rho0, const double* rho0_half,
                           const double* alpha0, const double* alpha0_half, const double* u,
                           const double* v, const double* w, const double* mean, double* divergence,
                           double* div_dense, int precision, void* stream);

/* The precision form's refinement residual div - A p on the cells of this
 * slab into a dense interior array (the pressure's ghosts filled, x-ghost
 * planes from the neighbours).  No counterpart in the reference. */
int pb_pressure_residual(const pb_dims* dims, const double* rho0, const double* rho0_half,
                         const double* pressure, const double* divergence, double* resid_dense,
                         void* stream);

/* Forward x- and y-FFT (PressureFFTParallel.pyx:168-180) of the levels of a
 * z-slab (dims: the whole horizontal plane, the slab's levels; indx_lo of x
 * and y zero) from a dense right-hand side into the spectral array of a
 * workspace that pb_pressure_init made for these dims: W[k][j][m], m =
 * 0 .. n0/2 (the Hermitian half), complex FP64 (PB_FP64) or FP32. */
int pb_pressure_fft_forward(const pb_dims* slab, void* workspace, long long workspace_bytes,
                            const double* src_dense, int precision, void* stream);

/* The Thomas solves (SparseSolvers.pyx:24-44, PressureFFTParallel.pyx:
 * 181-205) of the (kx, ky) columns of a slab of rows j0 .. j0 + rows->n[1]
 * - 1 over every level: spec W[k][j - j0][m] (complex, the precision's
 * type) and scratch (doubles, the same count) of the caller; wave numbers
 * from the z-slab's workspace (slab, slab_workspace); rho0, rho0_half over
 * the whole column. */
int pb_pressure_fft_columns(const pb_dims* rows, const double* rho0, const double* rho0_half,
                            const pb_dims* slab, const void* slab_workspace, void* spec, double* scratch,
                            int j0, int precision, void* stream);

/* Inverse y- and x-FFT (PressureFFTParallel.pyx:206-219) of a z-slab's
 * spectral array into a dense pressure. */
int pb_pressure_fft_inverse(const pb_dims* slab, void* workspace, long long workspace_bytes,
                            double* dst_dense, int precision, void* stream);

/* second_order_pressure_correction with remove_mean_u3 on every cell
 * (PressureSolver.pyx:83-136) of this slab; the pressure's ghosts filled. */
int pb_pressure_correct(const pb_dims* dims, const double* pressure, double* u, double* v, double* w,
                        const double* mean, void* stream);

/*
 * pb_pressure_solve for callers that cannot allocate device memory.  No
 * counterpart in the reference.  Same inputs, outputs and results as
 * pb_pressure_solve (FP64), but its scratch lives in a fixed file-scope
 * device array inside the library instead of a caller workspace, for code
 * that may not call cudaMalloc (a loop that cannot afford the device-wide
 * synchronisation an allocation may bring, an allocator policy that forbids
 * late device allocations, a host binding without a device allocator).
 *   Limit : pb_pressure_workspace_bytes(dims) must not exceed
 *           PB_PRESSURE_NOALLOC_MAX_BYTES (64 MiB, e.g. 128 x 128 x 160);
 *           larger grids return PB_ERR_WORKSPACE.  Every GPU that loads the
 *           library holds the 64 MiB until the process exits.
 *   Set-up: the first call on a device, and the first call after the grid
 *           changes, takes the array's device address (cudaGetSymbolAddress)
 *           and fills the grid constants synchronously; a grid change first
 *           waits for the whole device, so solves of the previous grid still
 *           queued on any stream finish with their own constants -- make
 *           that first call before any stream capture.
 *   Races : all calls on a device share the array (it keeps the last call's
 *           contents; nothing needs clearing, every word read is written
 *           first in the same call), so calls that may overlap on the GPU
 *           must be ordered by the caller.  Host threads are serialised by a
 *           lock held from the set-up until the call's kernels are enqueued.
 */
#define PB_PRESSURE_NOALLOC_MAX_BYTES (64ll << 20)
int pb_pressure_solve_noalloc(const pb_dims* dims, const double* rho0, const double* rho0_half,
                              const double* alpha0, const double* alpha0_half, double* u, double* v,
                              double* w, double* divergence, double* dynamic_pressure, void* stream);

/* ------------------------------------------------------------------------
 * Surface fluxes (lowest model level)
 * --------------------------------------------------------------------- */

/* Surface schemes, as SurfaceFactory (Surface.pyx:39-74) picks them by case. */
enum pb_surface_scheme {
  PB_SURFACE_NONE = 0,             /* SurfaceNone (Surface.pyx:203-213)             */
  PB_SURFACE_SULLIVAN_PATTON = 1,  /* SurfaceSullivanPatton (Surface.pyx:216-294)   */
  PB_SURFACE_BOMEX = 2,            /* SurfaceBomex (Surface.pyx:297-377)            */
  PB_SURFACE_DYCOMS_RF01 = 3       /* SurfaceDYCOMS_RF01 (Surface.pyx:474-561)      */
};

/*
 * The scheme's constants (the attributes its __init__/initialize set).
 *   theta_flux : SullivanPatton 0.24, Bomex 8.0e-3 (K m/s)
 *   z0         : roughness length (SullivanPatton 0.1 m)
 *   gustiness  : minimum wind speed of compute_windspeed (SullivanPatton
 *                0.001 m/s, Bomex and DYCOMS_RF01 0)
 *   ustar      : Bomex's fixed friction velocity ustar_ (0.28 m/s)
 *   cm, ft, fq : DYCOMS_RF01's bulk drag coefficient (0.0011), sensible and
 *                latent heat fluxes (15, 115 W/m^2)
 *   u0, v0     : the reference state's Galilean shift (Ref.u0, Ref.v0)
 */
typedef struct pb_surface {
  int scheme;
  double theta_flux;
  double z0;
  double gustiness;
  double ustar;
  double cm, ft, fq;
  double u0, v0;
} pb_surface;

/*
 * The surface arrays of SurfaceBase (Surface.pyx:84-94), device, nlg0*nlg1
 * doubles each, indexed i*nlg1 + j, owned by the caller and zeroed at
 * set-up as SurfaceBase.initialize does (Bomex also sets qt_flux to
 * 5.2e-5, Surface.pyx:305).  windspeed holds compute_windspeed's output;
 * scratch is PB_SURFACE_SCRATCH doubles for the horizontal mean of the
 * lowest-level temperature.
 */
#define PB_SURFACE_SCRATCH 512
typedef struct pb_surface_fields {
  double* u_flux;
  double* v_flux;
  double* qt_flux;
  double* s_flux;
  double* obukhov_length;
  double* friction_velocity;
  double* shf;
  double* lhf;
  double* b_flux;
  double* windspeed;
  double* scratch;
} pb_surface_fields;

/*
 * Surface<scheme>.update followed by SurfaceBase.update (Surface.pyx:116-
 * 178): wind speed at the lowest level (compute_windspeed,
 * Csrc/surface.h:157-185), friction velocity (SullivanPatton: the
 * Monin-Obukhov secant compute_ustar, Csrc/surface.h:34-93; Bomex: fixed;
 * DYCOMS_RF01: sqrt(cm) * wind speed), entropy and moisture fluxes, momentum
 * fluxes, then sensible / latent / buoyancy fluxes, Obukhov length and the
 * tendencies of the first interior level: u, v, s, and qt for the moist
 * schemes, += flux * alpha0_half[gw] / alpha0[gw-1] / dz.
 *   T, qt, qv, ql: DiagnosticVariables temperature, qv, ql and the
 *                  prognostic qt (qt, qv, ql, qt_tend NULL for
 *                  SullivanPatton, which is dry).
 * FP64 in both arithmetic forms: the work is one horizontal plane.
 * compute_ustar returns its first fixed-point iterate from the neutral guess
 * (`ustar` is assigned before its secant loop, Csrc/surface.h:52,73, and the
 * loop's result is not used); this computes that value and runs no loop.
 * PB_SURFACE_NONE returns PB_OK without work.
 */
int pb_surface_update(const pb_dims* dims, const pb_surface* surface, const double* p0_half,
                      const double* alpha0, const double* alpha0_half, const double* rho0_half,
                      const double* u, const double* v, const double* T, const double* qt, const double* qv,
                      const double* ql, double* u_tend, double* v_tend, double* s_tend, double* qt_tend,
                      const pb_surface_fields* fields, void* stream);

/* ------------------------------------------------------------------------
 * Subgrid scale and diffusion
 * --------------------------------------------------------------------- */

/* SGS schemes (SGS.pyx:35-44) and the Smagorinsky length scale (:101-145). */
enum pb_sgs_scheme {
  PB_SGS_UNIFORM = 1,       /* UniformViscosity (SGS.pyx:57-97)              */
  PB_SGS_SMAGORINSKY = 2    /* Smagorinsky (SGS.pyx:101-149)                 */
};
enum pb_sgs_length {
  PB_SGS_LENGTH_GRID = 0,   /* smagorinsky_update (Csrc/sgs.h:4-18)          */
  PB_SGS_LENGTH_WALL = 1,   /* smagorinsky_update_wall (Csrc/sgs.h:21-54)    */
  PB_SGS_LENGTH_ILES = 2    /* smagorinsky_update_iles (Csrc/sgs.h:56-89)    */
};
/* cs, prt: Smagorinsky constant and turbulent Prandtl number (defaults
 * 0.17, 1/3); viscosity, diffusivity: UniformViscosity's constants. */
typedef struct pb_sgs {
  int scheme;
  int length;
  double cs, prt;
  double viscosity, diffusivity;
} pb_sgs;

/*
 * Kinematics.update (Kinematics.pyx:42-58) followed by SGS.update
 * (SGS.pyx:48-53): the strain-rate magnitude of compute_strain_rate_mag
 * (Csrc/kinematics.h:72-131, from the velocity gradients :6-34 and strain
 * rates :37-69, formed in registers, not stored), then the eddy viscosity
 * and diffusivity over all cells.  The velocity gradients and the nine
 * strain-rate components the reference stores are not materialised.
 * sgs == NULL: Kinematics.update alone (the strain-rate magnitude; the
 * viscosity, diffusivity, buoyancy_frequency and zl_half are not used).
 *   buoyancy_frequency: DiagnosticVariables 'buoyancy_frequency' (Smagorinsky)
 *   zl_half           : Grid.zl_half, nlg2 doubles (wall / ILES length scale)
 * Where the reference's strain-magnitude stencil leaves the computed strain
 * field (the (x,x) pair on the plane i = 1 reads before the array, the (y,y)
 * pair on j = 1 wraps into the previous row), the term is 0; no interior
 * tendency reads those planes' viscosity when gw >= 3.
 */
int pb_kinematics_sgs(const pb_dims* dims, const pb_sgs* sgs, const double* u, const double* v,
                      const double* w, const double* buoyancy_frequency, const double* zl_half,
                      double* strain_rate_mag, double* viscosity, double* diffusivity, void* stream);

/*
 * ScalarDiffusion.update (ScalarDiffusion.pyx:112-150): for every scalar and
 * direction the second-order diffusive flux (Csrc/scalar_diffusion.h:6-57,
 * formed in registers) and its divergence (scalar_flux_divergence,
 * Csrc/flux_divergence.h:4-32) subtracted from the scalar's tendency over
 * the interior; factors (HOST, nscalars doubles, NULL = all 1) as the
 * reference's flux_factor.  qt_index >= 0 adds the qt-diffusion entropy
 * source (compute_qt_diffusion_s_source, Csrc/scalar_diffusion.h:70-113;
 * namelist diffusion.qt_entropy_source) to the tendency of scalar s_index,
 * with p0_half, qv (DV) and T (DV).  scalars / tendencies: HOST arrays of
 * device pointers.  Needs gw >= 2.
 */
int pb_scalar_diffusion(const pb_dims* dims, const double* rho0, const double* rho0_half,
                        const double* alpha0_half, const double* diffusivity, int nscalars,
                        const double* const* scalars, double* const* tendencies, const double* factors,
                        int qt_index, int s_index, const double* p0_half, const double* qv, const double* T,
                        void* stream);

/*
 * MomentumDiffusion.update (MomentumDiffusion.pyx:52-78): the nine stress
 * fluxes (compute_diffusive_flux_m, Csrc/momentum_diffusion.h:5-96, formed
 * in registers from the velocities and the viscosity) and their divergence
 * (momentum_flux_divergence, Csrc/flux_divergence.h:34-60) into the u, v, w
 * tendencies, then the entropy source S^2 nu / T into s_tend
 * (compute_entropy_source, :98-118).  strain_rate_mag as pb_kinematics_sgs
 * leaves it.  Needs gw >= 2.
 */
int pb_momentum_diffusion(const pb_dims* dims, const double* rho0, const double* rho0_half,
                          const double* alpha0, const double* alpha0_half, const double* u, const double* v,
                          const double* w, const double* viscosity, const double* strain_rate_mag,
                          const double* T, double* ut, double* vt, double* wt, double* s_tend, void* stream);

/* ------------------------------------------------------------------------
 * Case forcing
 * --------------------------------------------------------------------- */

/* Forcing schemes, as Forcing.__init__ (Forcing.pyx:29-67) picks them by case. */
enum pb_forcing_scheme {
  PB_FORCING_NONE = 0,
  PB_FORCING_SULLIVAN_PATTON = 1,  /* ForcingSullivanPatton (Forcing.pyx:256-300): Coriolis */
  PB_FORCING_BOMEX = 2,            /* ForcingBomex (:102-254): pressure gradient, sources, subsidence */
  PB_FORCING_DYCOMS_RF01 = 3       /* ForcingDyCOMS_RF01 (:346-460): subsidence, Coriolis */
};

/*
 * The scheme's per-level profiles (device, nlg2 doubles each, as the
 * scheme's initialize sets them from Grid.zl_half and p0_half) and
 * constants.  dtdt, dqtdt: Bomex's large-scale temperature and qt
 * tendencies; subsidence: the large-scale vertical velocity (Bomex,
 * DYCOMS_RF01); u0, v0: the Galilean shift.
 */
typedef struct pb_forcing {
  int scheme;
  double coriolis_param;
  double u0, v0;
  const double* ug;
  const double* vg;
  const double* dtdt;
  const double* dqtdt;
  const double* subsidence;
} pb_forcing;

/*
 * Forcing.update for the scheme, in its order: Bomex -- large_scale_p_gradient
 * (Forcing.pyx:1982-2011) with umean, vmean the horizontal means of u and v
 * (pb_horizontal_stat), the entropy and qt sources (s_tendency_c,
 * Csrc/entropies.h:17-21), then apply_subsidence (:2013-2039) of s, qt, u,
 * v; DYCOMS_RF01 -- apply_subsidence of s, qt, u, v, then coriolis_force
 * (:1954-1980); SullivanPatton -- coriolis_force.  As in the reference the
 * subsidence also reaches the tendencies of the top ghost levels.
 * PB_FORCING_NONE returns PB_OK without work.
 */
int pb_forcing_update(const pb_dims* dims, const pb_forcing* forcing, const double* p0_half,
                      const double* umean, const double* vmean, const double* u, const double* v,
                      const double* s, const double* qt, const double* ql, const double* T, double* ut,
                      double* vt, double* s_tend, double* qt_tend, void* stream);

/* ------------------------------------------------------------------------
 * DYCOMS radiation
 * --------------------------------------------------------------------- */

/* RadiationDyCOMS_RF01's constants (Radiation.pyx:231-240): f0 (namelist
 * radiation.dycoms_f0, default 70), f1 = 22, kap = 85, alpha_z = 1,
 * divergence = 3.75e-6. */
typedef struct pb_dycoms_radiation_params {
  double f0, f1, kap, alpha_z, divergence;
} pb_dycoms_radiation_params;

/*
 * RadiationDyCOMS_RF01.update (Radiation.pyx:252-353) on one rank: per
 * interior column the level of the 8 g/kg qt isoline zi, the flux F of
 * Stevens et al. 2005 eq. 3 on the n2+1 faces, the heating rate
 * -(F[k+1] - F[k]) dzi / rho0_half[k] (indexed without the ghost offset,
 * as the reference does) into heating_rate (interior cells), then
 * s_tend += heating / T and dTdt_rad = heating / cpm(qt).  z: Grid.z
 * (nlg2 face heights).  A column with no level above 8 g/kg takes zi above
 * the domain (the reference reuses the previous pencil's zi there).
 */
int pb_dycoms_radiation(const pb_dims* dims, const pb_dycoms_radiation_params* params,
                        const double* rho0_half, const double* z, const double* ql, const double* qt,
                        const double* T, double* s_tend, double* heating_rate, double* dTdt_rad, void* stream);

/* ------------------------------------------------------------------------
 * Horizontal statistics
 * --------------------------------------------------------------------- */

/* The reductions of ParallelMPI (ParallelMPI.pyx:196-540), one rank. */
enum pb_stat_kind {
  PB_STAT_MEAN = 0,                      /* HorizontalMean :196-241                      */
  PB_STAT_MEAN_SQUARES = 1,              /* HorizontalMeanofSquares :243-289 (v1 v2)     */
  PB_STAT_MEAN_CUBES = 2,                /* HorizontalMeanofCubes :291-325 (v1 v2 v3)    */
  PB_STAT_MAX = 3,                       /* HorizontalMaximum :327-357                   */
  PB_STAT_MIN = 4,                       /* HorizontalMinimum :359-389                   */
  PB_STAT_MEAN_SURFACE = 5,              /* HorizontalMeanSurface :391-428 (one plane)   */
  PB_STAT_MEAN_CONDITIONAL = 6,          /* HorizontalMeanConditional :430-483           */
  PB_STAT_MEAN_SQUARES_CONDITIONAL = 7   /* HorizontalMeanofSquaresConditional :485-540  */
};

/* Bytes of device scratch pb_horizontal_stat needs for this grid. */
long long pb_stat_workspace_bytes(const pb_dims* dims);

/*
 * One horizontal statistic over the interior columns, per level: out[k],
 * k = 0 .. nlg2-1 (device, nlg2 doubles), as the reference's loops and
 * normalisation give it: the means times 1/(n0 n1); the conditional means
 * divided by max(sum of the mask, 1); the maximum / minimum starting from
 * -9e12 / 9e12.  PB_STAT_MEAN_SURFACE reduces one nlg0*nlg1 plane (indexed
 * i*nlg1 + j) to out[0] and needs no workspace.  v2, v3, mask: NULL where
 * the kind does not use them.  The sums use a fixed partition and order
 * (deterministic; not the reference's sequential order, so sums agree to
 * rounding).
 */
int pb_horizontal_stat(const pb_dims* dims, int kind, const double* v1, const double* v2, const double* v3,
                       const double* mask, double* out, void* workspace, long long workspace_bytes,
                       void* stream);

/* ------------------------------------------------------------------------
 * Errors
 * --------------------------------------------------------------------- */

/* Reads (synchronously) and returns the device error word of the current device. */
int pb_get_error(unsigned int* word);
/* Clears the device error word of the current device (stream-ordered). */
int pb_clear_error(void* stream);
/* Human-readable status text. */
const char* pb_status_string(int status);

/*
 * Number of kernels this library has launched in this process (host-side
 * counter, incremented at every launch).  Instrumentation with no
 * counterpart in the reference.
 */
long long pb_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* PYCLES_B200_H */

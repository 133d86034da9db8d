/*
 * turbid_gpu.h -- C ABI of libturbid_gpu.so, the B200 (sm_100a) implementation
 * of TURBID's flat-bottom Fourier-Chebyshev RK3 substep.
 *
 * Plain C types only: host pointers for state exchange, device pointers (as
 * double* or float*) for the field-container primitives, an opaque context.
 * Every entry point returns a tg_status (0 = success); tg_last_error() gives
 * a message in the reference's "Class::Method > text" style.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the yueliangyi/TURBID source tree).
 *
 * Device layouts used by the primitives:
 *   physical field   [dim][Nz][Ny][Nx]      real, x fastest (as the reference)
 *   spectral field   [dim][Nz][M]           complex (re,im) pairs, m fastest,
 *                                            m = iy + Nyc*ix ("z-slab" layout)
 *   host state (tg_upload_state / tg_download_state) uses the reference's
 *   restart layout ccube(Nz, Nyc, Nxh*dim): [dim][Nxh][Nyc][Nz], z fastest.
 *
 * Threading: one host thread per context; all work is ordered on the
 * context's CUDA stream; entry points are not reentrant on one context.
 */
#ifndef TURBID_GPU_H_
#define TURBID_GPU_H_

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TG_API __attribute__((visibility("default")))
#else
#define TG_API
#endif

typedef int tg_status;
#define TG_OK            0
#define TG_ERR_CUDA      1   /* a CUDA runtime call or kernel launch failed      */
#define TG_ERR_SHAPE     2   /* unsupported or inconsistent grid / buffer sizes  */
#define TG_ERR_ARG       3   /* invalid argument (null pointer, bad stage, ...)  */
#define TG_ERR_NAN       4   /* non-finite value detected in the features        */
#define TG_ERR_SETUP     5   /* operator construction failed (eigen-solver)      */
#define TG_ERR_NOMEM     6   /* device allocation failed                         */
#define TG_ERR_STATE     7   /* call out of order (e.g. step before upload)      */
#define TG_ERR_TIMEOUT   8   /* a bounded device wait gave up                    */

#define TG_PREC_FP64   0     /* all arithmetic in FP64 (parity mode)             */
#define TG_PREC_MIXED  1     /* transforms and nonlinear products in FP32,
                                z-operators and Helmholtz solves in FP64         */

#define TG_NFEATURE 50       /* Phase::featureglobal_ (src/phase.cc:16-17)       */

/* One case = the .ini parameters the hot path reads
 * (src/configure.h:51-118; read by the Configuration::Load methods). */
typedef struct tg_case {
  int    nx, ny, nz;                 /* [Domain] grid_point_number              */
  double lx, ly;                     /* [Domain] dimensionless_length (lz == 2) */
  int    nphase;                     /* [System] total_phase_number (1 or 2)    */
  int    mapping;                    /* [Space Stepper] 0 None,1 TwoEndTangent,
                                        2 TwoEndSin, 3 OneEndTangent            */
  double mapping_coef;
  double slope; int slope_direction; /* [Domain] top_bottom_slope, direction    */
  double dt;                         /* [Time Stepper] marching_time_step       */
  int    output_based_on_step;
  double reynolds, froude, averaged_concentration, specific_gravity;
  int    affected_by_scalar;
  double bc_u[5], bc_v[5], bc_w[5], bc_p[5];  /* vertical_type_u1/u2/u3/p      */
  int    force_type;                 /* 0 None 1 Constant 2 Oscillatory
                                        3 Pulsatile 4 Damping                   */
  int    force_direction[2];
  double force_amplitude[4];
  double schmidt, settling, erosion_rate, critical_shear;
  int    scalar_bc;                  /* 0 ZeroFlux, 1 ErosionDeposition         */
  int    precision;                  /* TG_PREC_FP64 or TG_PREC_MIXED           */
} tg_case;

typedef struct tg_ctx tg_ctx;

TG_API const char* tg_last_error(void);
TG_API int tg_version(void);
/* Number of kernels this library has launched so far in the process
 * (no reference counterpart; measurement support). */
TG_API long long tg_launch_count(void);

/* Replaces System::System + DomainDecomposition::Configure (src/system.cc:19-64,
 * src/base.cc:202-342), Domain::Configure (src/domain.cc:292-347),
 * ChebyshevSpaceStepper::Configure (src/stepper_space_chebyshev.cc:101-250) and
 * the decompositions built in FlatCarrierPhase::Configure /
 * FlatScalarPhase::Configure (src/phase_carrier_flat.cc:178-246,
 * src/phase_scalar_flat.cc:176-221, src/cmdz2_decomposition.cc:19-227).
 * Operators are built on the host (own eigen-solver); allocates device memory. */
TG_API tg_status tg_create(const tg_case* c, tg_ctx** out);
TG_API tg_status tg_destroy(tg_ctx* ctx);
/* dims = {nx, ny, nz, nxh, nyc, M} */
TG_API tg_status tg_get_dims(const tg_ctx* ctx, int dims[6]);
/* Order all later work of the context on the caller's CUDA stream
 * (cudaStream_t passed as void*, used verbatim: NULL is the legacy default
 * stream).  The library's own stream, created by tg_create, is released. */
TG_API tg_status tg_set_stream(tg_ctx* ctx, void* stream);
TG_API tg_status tg_synchronize(tg_ctx* ctx);

/* Replaces the matrices of CmDz2DecompositionCplx::Construct
 * (src/cmdz2_decomposition.cc:19-227) with caller-supplied ones.
 * which: 0 u, 1 v, 2 w, 3 p, 4 scalar.  Each matrix is nz*nz row-major FP64;
 * E/Einv are the full matrices with the identity corners; lam has nz entries
 * (rows 0 and nz-1 ignored); fbb/ftb/fbf/ftf are the four fix rows. */
TG_API tg_status tg_set_decomposition(tg_ctx* ctx, int which, const double* E,
                               const double* Einv, const double* lam,
                               const double* fbb, const double* ftb,
                               const double* fbf, const double* ftf);
/* Reads back the operators built by tg_create (same layouts). */
TG_API tg_status tg_get_decomposition(const tg_ctx* ctx, int which, double* E,
                               double* Einv, double* lam, double* fbb,
                               double* ftb, double* fbf, double* ftf);
/* Host-only (no GPU needed): the operators tg_create builds, for a grid of
 * nz Chebyshev points.  tg_operators_host replaces ChebyshevSpaceStepper::
 * Configure (src/stepper_space_chebyshev.cc:101-250); tg_decomposition_host
 * replaces CmDz2DecompositionCplx::Construct (src/cmdz2_decomposition.cc:19-227)
 * for bc = {a_bottom, b_bottom, a_top, b_top}; outputs as in
 * tg_get_decomposition. */
TG_API tg_status tg_operators_host(int nz, int mapping, double mapping_coef, double* D1, double* D2);
TG_API tg_status tg_decomposition_host(int nz, int mapping, double mapping_coef, const double* bc,
                                double* E, double* Einv, double* lam, double* fbb,
                                double* ftb, double* fbf, double* ftf);
/* D1, D2 (nz*nz row-major) of ChebyshevSpaceStepper::Configure. */
TG_API tg_status tg_get_operators(const tg_ctx* ctx, double* D1, double* D2);

/* Replaces FlatCarrierVariable::Load / FlatScalarVariable::Load and the
 * remainder of Variable::Configure (src/variable_carrier_flat.cc:262-421,
 * src/variable_scalar_flat.cc). Host arrays in the restart layout: uvw is
 * 3*Nxh*Nyc*Nz complex, p and phi Nxh*Nyc*Nz complex (phi may be NULL when
 * nphase == 1).  Resets the RK3 registers and boundary history like a fresh
 * Configure; sets step/time from start_step. */
TG_API tg_status tg_upload_state(tg_ctx* ctx, const double* uvw, const double* p,
                          const double* phi, int start_step);
/* Replaces FlatCarrierVariable::Save / FlatScalarVariable::Save
 * (src/variable_carrier_flat.cc:143-246): device -> host, same layout. */
TG_API tg_status tg_download_state(tg_ctx* ctx, double* uvw, double* p, double* phi);

/* Time bookkeeping of TimeStepper (src/stepper_time.h:56-91): the phases read
 * time, dt, step and the alternation flag from here.  A dt different from the
 * current one (the adaptive branch, TimeStepper::Update2,
 * src/stepper_time.cc:117-208) also re-assembles the velocity and scalar
 * solves as FlatCarrierPhase::Update / FlatScalarPhase::Update do
 * (src/phase_carrier_flat.cc:248-262, src/phase_scalar_flat.cc:225-238). */
TG_API tg_status tg_set_time(tg_ctx* ctx, int step, double time, double dt, int alternation);
TG_API tg_status tg_get_time(const tg_ctx* ctx, int* step, double* time, double* dt,
                      int* alternation, int* isforward, double* cfl);

/* Phase plugin methods (src/phase.h:25-114). */
TG_API tg_status tg_carrier_predict(tg_ctx* ctx, int stage);  /* phase_carrier_flat.cc:272-559 */
TG_API tg_status tg_carrier_correct(tg_ctx* ctx, int stage);  /* phase_carrier_flat.cc:566-709 */
TG_API tg_status tg_scalar_predict(tg_ctx* ctx, int stage);   /* phase_scalar_flat.cc:245-284  */
TG_API tg_status tg_scalar_correct(tg_ctx* ctx, int stage);   /* phase_scalar_flat.cc:291-533  */

/* nsteps passes of the FlatChannelSolver::Execute loop body
 * (src/solver_channel_flat.cc:199-293): TimeStepper::Update with the previous
 * CFL feature, three stages of both phases, alternation flip.  Stops early when
 * the CFL guard of TimeStepper::Update (src/stepper_time.cc:72-113) clears
 * isForward.  maxstep / maxcfl as in [Time Stepper]; *done receives the number
 * of steps taken (may be NULL).  When features is non-NULL it receives the
 * 50-entry feature vector after the last step (one 400-byte device->host read). */
TG_API tg_status tg_run_steps(tg_ctx* ctx, int nsteps, int maxstep, double maxcfl,
                       double* features, int* done);
/* tg_run_steps records each of the two step variants (the nonlinear forms
 * alternate) once as a CUDA graph and replays it when the step's kernel
 * arguments do not change from step to step (fixed dt, flat bed, no profiling,
 * a stream other than the legacy default stream); enable = 0 issues every
 * kernel separately.  Results are identical either way.  Default: enabled.
 * (No reference counterpart; execution control.) */
TG_API tg_status tg_set_graphs(tg_ctx* ctx, int enable);
/* Row-tiling autotuner of the z-operator GEMMs (no reference counterpart: the
 * reference's Armadillo products have no launch shape).  Times each distinct
 * row tiling (output rows per CTA) of the dense and the folded product kernel
 * on this grid and GPU, and applies the fastest to every operator of the
 * context; results do not depend on the tiling.  cache_path (may be NULL): a
 * JSON object {"<Nx>x<Ny>x<Nz>:<precision>:sm<cc>x<SMs>": [dense, folded]} of
 * the two preferences (most 8-row m-tiles per CTA, 1-16 and 1-6); an entry for
 * this case is applied without timing, a missing one is timed and added (the
 * file is rewritten whole and renamed into place).  tiling (may be NULL)
 * receives {m-tiles, row tiles} of the dense kernel then of the folded one.
 * Call between steps: it waits for the context's streams, and the recorded
 * step graphs are dropped. */
TG_API tg_status tg_autotune(tg_ctx* ctx, const char* cache_path, int* tiling);
/* tg_run_steps for n independent cases (each context on its own stream, e.g.
 * an ensemble of uneven grids and parameters): every case's step is enqueued
 * before any case's previous features are awaited, so the cases run
 * concurrently on the GPU.  done[i] (may be NULL) receives the steps case i
 * took.  (No reference counterpart: the reference runs one case per job.) */
TG_API tg_status tg_run_ensemble(tg_ctx** ctxs, int n, int nsteps, int maxstep, double maxcfl,
                                 int* done);

/* FlatChannelPostprocessor::Execute (src/postprocessor_channel_flat.cc:195-236)
 * for the current state: swirling strength lambda_ci (largest |Im| of the
 * eigenvalues of the velocity-gradient tensor du_i/dx_j) at every physical
 * point, FP64, into vortex[nz][ny][nx] (host; the reference's real cube
 * layout, x fastest).  Allocates its work buffers on the first call. */
TG_API tg_status tg_swirling_strength(tg_ctx* ctx, double* vortex);

/* Phase::GetFeatureGlobal (src/phase.h:57): 50 doubles, device -> host. */
TG_API tg_status tg_features(tg_ctx* ctx, double* out);

/* Kernel-class timing (no reference counterpart; measurement support):
 * tg_profile_begin starts recording CUDA events around every instrumented
 * launch on the context's stream; tg_profile_end synchronizes and returns per
 * class the summed device milliseconds, algorithmic bytes and flops and the
 * launch count.  Classes: 0 z-operator GEMM (FP64 DMMA), 1 forward x pass,
 * 2 forward y pass, 3 backward y pass, 4 backward x pass, 5 elementwise,
 * 6 positivity filter, 7 feature reduction, 8 backward x pass fused with the
 * advective products (three gradient fields per output), 9 int8-slice
 * z-operator products (slicing and tensor-core product).  The algorithmic flops of a z-operator are
 * those of the dense product, 4 Nz^2 M per component (the reference's count);
 * tg_profile_executed returns, for the window that tg_profile_end closed, the
 * flops the kernels executed (half of those for folded or split operators). */
#define TG_PROF_NCAT 10
TG_API tg_status tg_profile_begin(tg_ctx* ctx);
TG_API tg_status tg_profile_end(tg_ctx* ctx, int ncat, double* ms, double* bytes,
                                double* flops, int* count);
TG_API tg_status tg_profile_executed(const tg_ctx* ctx, int ncat, double* flops);

/* Field-container primitives on device buffers (layouts above). */
/* RealCplxCube::DftForward (src/cube_real_cplx.cc:525-539): pruned x r2c,
 * y c2c, scaled 1/(NxNy).  phys: dim physical fields; spec: dim spectral. */
TG_API tg_status tg_dft_forward_f64(tg_ctx* ctx, const double* phys, double* spec, int dim);
TG_API tg_status tg_dft_forward_f32(tg_ctx* ctx, const float* phys, double* spec, int dim);
/* Allocation-free variant of tg_dft_forward_f64 (no counterpart in the
 * reference).  For callers that must not allocate device memory: a host code
 * that reserves and manages all device memory itself (a solver sized to fill
 * HBM with its own fields, or one that runs under a fixed memory budget),
 * where a cudaMalloc would fail or take memory the caller has promised
 * elsewhere.  It needs no tg_ctx (tg_create allocates): phys and spec are the
 * caller's device buffers in the layouts above, stream is a cudaStream_t
 * (NULL = legacy default stream).  The x->y intermediate lives in a 16 MiB
 * device array inside the library (every GPU that loads the library holds it
 * until exit), so nx and ny must be powers of two in [8, 1024]; larger grids
 * are rejected with TG_ERR_SHAPE.  The first call on each device sets up the
 * static twiddle and index tables on that device (make it with the device
 * current); that set-up copies the tables with cudaMemcpyToSymbol, so make the
 * first call on each device before any stream capture begins.  Nothing has to
 * start at zero: each call writes every scratch element before reading it.
 * All calls share the one scratch array: calls whose work overlaps on the GPU
 * (other streams or other host threads) race; order them on one stream.
 * A device reset after the first call is followed by the set-up again on the
 * next call.  Results agree with tg_dft_forward_f64's to rounding (about 1e-13
 * relative L2): the same pruned transform, evaluated here with radix-4 and
 * radix-2 passes where the context path uses radix-16 passes. */
TG_API tg_status tg_dft_forward_f64_noalloc(int nx, int ny, int nz, const double* phys,
                                            double* spec, int dim, void* stream);
/* The same transforms over any number of z planes (physical planes of Ny x Nx
 * in, spectral planes of M out, or back): the local x and y passes of one
 * rank's z-slab in a slab/column decomposition over several GPUs, as P3DFFT
 * does them before its z exchange (build/ftran.F90:50-263,
 * build/btran.F90:48-257).  fp32 != 0: FP32 physical planes. */
TG_API tg_status tg_dft_forward_planes(tg_ctx* ctx, const void* phys, double* spec, int planes, int fp32);
TG_API tg_status tg_dft_backward_planes(tg_ctx* ctx, const double* spec, void* phys, int planes, int fp32);
/* RealCplxCube::DftBackward (src/cube_real_cplx.cc:542-555): zero-fill, unscaled. */
TG_API tg_status tg_dft_backward_f64(tg_ctx* ctx, const double* spec, double* phys, int dim);
TG_API tg_status tg_dft_backward_f32(tg_ctx* ctx, const double* spec, float* phys, int dim);
/* RealCplxCube::Multiply(cmat, RealCplxCube&) (src/cube_real_cplx.cc:461-471):
 * out = A * in along z for dim components; A is nz*nz row-major FP64 host
 * memory (copied to the device on each call). */
TG_API tg_status tg_multiply(tg_ctx* ctx, const double* A_host, const double* in,
                      double* out, int dim);
/* RealCplxCube::Multiply (src/cube_real_cplx.cc:461-471) through the
 * int8-slice tensor-core product that the mixed precision mode uses for its
 * dense Helmholtz solves: A and in split into 5 exact int8 slices over the
 * interior rows (z = 1 .. nz-2), the slice products exact in int32 on the
 * tcgen05 tensor cores, combined in FP64, the two boundary rows added in FP64.
 * Relative error about 1e-9 of the FP64 product; nz <= 258.  Same arguments
 * as tg_multiply. */
TG_API tg_status tg_multiply_islice(tg_ctx* ctx, const double* A_host, const double* in, double* out, int dim);
/* z-solver of the dense Helmholtz solves (u, v and the scalar) in mixed
 * precision (no reference counterpart; execution control):
 * TG_ZSOLVER_DMMA = FP64 tensor-core products, TG_ZSOLVER_ISLICE = the
 * int8-slice product of tg_multiply_islice (default in mixed precision).
 * FP64 precision always uses TG_ZSOLVER_DMMA.  Recorded step graphs are
 * dropped. */
#define TG_ZSOLVER_DMMA   0
#define TG_ZSOLVER_ISLICE 1
TG_API tg_status tg_set_zsolver(tg_ctx* ctx, int solver);
/* 1 in *flag when a bounded device wait of an int8-slice product gave up
 * since the context was created (the product's output is then invalid).
 * tg_run_steps checks the same flag with every step's features and stops
 * with TG_ERR_TIMEOUT when it is set. */
TG_API tg_status tg_zsolver_error(tg_ctx* ctx, int* flag);
/* Failure-path check of the int8-slice product (no reference counterpart):
 * runs one product whose operator copies are withheld, so that its bounded
 * wait for them gives up; the kernel drains, frees its tensor memory, sets
 * the flag and returns.  Returns TG_ERR_TIMEOUT when that path worked (the
 * flag is cleared again; the context stays usable), TG_OK if the wait did
 * not give up. */
TG_API tg_status tg_islice_selftest(tg_ctx* ctx);
/* CmDz2 solve of FlatCarrierPhase::Helmholtz / FlatScalarPhase::Helmholtz
 * (src/phase_carrier_flat.cc:861-994, src/phase_scalar_flat.cc:635-667) for
 * one spectral component: which as in tg_set_decomposition, stage 0..2;
 * rhs is not modified (the reference modifies its target in place). */
TG_API tg_status tg_helmholtz(tg_ctx* ctx, int which, int stage, const double* rhs,
                       double* out);

#ifdef __cplusplus
}
#endif
#endif /* TURBID_GPU_H_ */

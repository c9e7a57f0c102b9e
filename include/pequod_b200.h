/*
 * pequod_b200.h -- C ABI of the B200-native PEQUOD QG time-step hot path.
 *
 * The reference (PEQUOD, Fortran 2003 + MPI) has no C or FFI plugin API; its
 * swap point for the elliptic solver is the module alias in qg3p_aux.F90:10-17
 *     use qg_helmholtz, only : solve_helmholtz => helm, helmholtz_solver_cache => helm_cache
 * and the advection routines are qg_aux's public list (qg3p_aux.F90:33-43),
 * called positionally from qg3.F90:598-807,952.  Every entry point below is
 * the C side of a bind(C) interface that replaces one of those Fortran
 * routines.
 *
 * Conventions
 *  - Arrays are Fortran column-major, i (first index) fastest, REAL(8).
 *    sdata-shaped arrays are (ii, jj, L); "reference layout" arrays in
 *    pq_get_field / pq_set_field are the reference's own shapes:
 *      full data (ii+2, jj+2, L), FLUX_II (ii+3, jj+2, L),
 *      FLUX_JJ (ii+2, jj+3, L), residuals (ii, jj, L)
 *    (qg3p_base.F90:1322-1323, 2808-2818; qg3.F90:84).
 *  - ptr_kind: PQ_PTR_HOST (pointer into host memory, copied) or
 *    PQ_PTR_DEVICE (dense device array on the context's device).
 *  - Every call returns PQ_OK (0) or a PQ_ERR_* code and never aborts the
 *    process (the reference calls mpi_abort, qg3p_base.F90:383-403);
 *    pq_last_error() gives the message.
 *  - One context per caller thread; calls on different contexts are
 *    independent.  A context's device state persists between calls.
 *  - All quantities are in the reference's non-dimensional units
 *    (qg3.F90:152-168): grid spacing 1, t_scale = l_scale / u_scale.
 */
#ifndef PEQUOD_B200_H
#define PEQUOD_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PQ_API __attribute__((visibility("default")))
#else
#define PQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define PQ_OK 0
#define PQ_ERR_ARG 1         /* invalid argument / unsupported size */
#define PQ_ERR_CUDA 2        /* CUDA runtime error */
#define PQ_ERR_NAN 3         /* NaN psiC or energy (the reference aborts) */
#define PQ_ERR_NOMEM 4       /* device allocation failed */
#define PQ_ERR_UNSUPPORTED 5 /* feature not available in this build */
#define PQ_ERR_STATE 6       /* call out of order (e.g. step before init) */
#define PQ_ERR_BUDGET 7      /* request exceeds the server's HBM budget */
#define PQ_ERR_NOTFOUND 8    /* unknown request id */

#define PQ_PTR_HOST 0
#define PQ_PTR_DEVICE 1

#define PQ_SCHEME_CABARET 0  /* config.h: #define CABARET, CABARET_LIMITER */
#define PQ_SCHEME_LEAPFROG 1 /* config.h: #undef CABARET (centred + RAW filter) */

#define PQ_PREC_FP64 0       /* plain form: FP64 throughout */
#define PQ_PREC_MIXED 1      /* FP32 storage/transforms, FP64 barotropic solve, projection and reductions */

/* Velocity boundary conditions, qg3p_diagnostics.F90:57-58. */
#define PQ_BC_PARTIAL_SLIP 1
#define PQ_BC_NO_SLIP 2
#define PQ_BC_FREE_SLIP 3

#define PQ_MAX_LAYERS 8

/* Fields of the model state, for pq_get_field / pq_set_field. */
#define PQ_F_PSI 0       /* psi%data       (ii+2, jj+2, L) */
#define PQ_F_ZETA 1      /* zeta%data      (ii+2, jj+2, L) */
#define PQ_F_REL 2       /* rel%data       (ii+2, jj+2, L) */
#define PQ_F_ZETA_OLD 3  /* zeta_old       (ii+2, jj+2, L) */
#define PQ_F_UI 4        /* ui%data        (ii+3, jj+2, L) */
#define PQ_F_UJ 5        /* uj%data        (ii+2, jj+3, L) */
#define PQ_F_UIMO 6      /* uimo%data      (ii+3, jj+2, L) */
#define PQ_F_UJMO 7      /* ujmo%data      (ii+2, jj+3, L) */
#define PQ_F_ZETA_FI 8   /* zeta_fi%data   (ii+3, jj+2, L) */
#define PQ_F_ZETA_FJ 9   /* zeta_fj%data   (ii+2, jj+3, L) */
#define PQ_F_RES 10      /* res            (ii, jj, L) */
#define PQ_F_RES_BETA 11 /* res_beta       (ii, jj, L) */
#define PQ_F_CORR 12     /* hcache%corr    (ii, jj, L), read only */
/* Leapfrog second time level (qg3.F90 psi(2), zeta(2), rel(2), zeta_old(2)). */
#define PQ_F_PSI2 13
#define PQ_F_ZETA2 14
#define PQ_F_REL2 15
#define PQ_F_ZETA_OLD2 16

/* Model description in non-dimensional units.  Matrices are column-major
 * with leading dimension `layers` (the Fortran strat%modes_to_z layout). */
typedef struct pq_model_desc {
    int ii, jj, layers;   /* nodes including the boundary; ii - 1 = 2^p, p >= 2 */
    int periodic_j;       /* 0: closed basin; 1: zonal channel periodic in j, walls at
                             i = 1 and ii: the momentum-corrected inversion
                             (qg3p_aux.F90:233-379, 524-575) and periodic stencils,
                             CABARET or leapfrog, with checkpoints, the time
                             average and the quad covariances */
    int scheme;           /* PQ_SCHEME_* */
    int limiter;          /* CABARET_LIMITER (1 = on) */
    int bc_type;          /* PQ_BC_* */
    int precision;        /* PQ_PREC_* */
    int adapt_dt;         /* cabaret_adapt_dt each step */
    double alpha;         /* partial-slip parameter l_scale / alpha_dim */
    double dt;            /* time step */
    double viscosity;     /* lateral viscosity */
    double visc_bot;      /* bottom drag */
    double target_cfl, max_dt, max_dt_increase;  /* adaptive time step */
    double ra_nu, ra_alpha;                      /* leapfrog RAW filter */
    double beta[PQ_MAX_LAYERS];   /* beta per layer */
    double h[PQ_MAX_LAYERS];      /* layer thicknesses */
    double s1[PQ_MAX_LAYERS];     /* strat%s1 (s1[0] unused) */
    double s2[PQ_MAX_LAYERS];     /* strat%s2 (s2[L-1] unused) */
    double ss[PQ_MAX_LAYERS];     /* strat%ss, ss[0] = 0 (barotropic) */
    double m2z[PQ_MAX_LAYERS * PQ_MAX_LAYERS];  /* strat%modes_to_z */
    double z2m[PQ_MAX_LAYERS * PQ_MAX_LAYERS];  /* strat%z_to_modes */
    const double* force_wind;     /* (ii, jj) layer-1 wind forcing, or NULL */
} pq_model_desc;

/* Physical (cgs) description of a wind-driven double gyre; converted to a
 * pq_model_desc by pq_setup_double_gyre the way qg3.F90:150-307 does. */
typedef struct pq_physical {
    int ii, jj, layers;
    double basinscale;      /* cm: (ii - 1) * dx (qg3p_params.F90:47) */
    double dt;              /* s */
    double f0;              /* s^-1 */
    double beta;            /* cm^-1 s^-1 */
    double H[PQ_MAX_LAYERS];       /* cm */
    double gprime[PQ_MAX_LAYERS];  /* cm s^-2, interfaces 1..L-1 */
    double tau;             /* cm^2 s^-2: wind stress / rho */
    double wind_asym, wind_tilt, wind_shift;
    double visc;            /* cm^2 s^-1 */
    double visc_bot;        /* s^-1 */
    double alpha;           /* cm; >= 1e100 selects free slip */
    int partial_slip;       /* 0: no slip */
    int scheme, limiter, precision, adapt_dt;
    double target_cfl, max_dt, max_dt_increase;  /* max_dt in s */
    double u_scale;         /* cm s^-1 (qg3p_params.F90:105) */
} pq_physical;

typedef struct pq_ctx pq_ctx;

/* ---- set-up (host) ------------------------------------------------------ */

/* Stratification from layer thicknesses and s1(2:L), s2(1:L-1) in cgs
 * (allocate_stratification_parameters + s_conversion_matrices,
 * qg3p_diagnostics.F90:210-236, 372-422): fills h, s1, s2, ss, m2z, z2m of
 * `d` scaled by l_scale. */
PQ_API int pq_stratification(pq_model_desc* d, int layers, const double* H, const double* s1_in,
                      const double* s2_in, double l_scale);

/* Non-dimensionalisation, stratification, wind forcing and beta of
 * qg3.F90:150-307.  wind_out: caller buffer of ii*jj doubles that d->force_wind
 * will point to. */
PQ_API int pq_setup_double_gyre(const pq_physical* p, pq_model_desc* d, double* wind_out, double* t_scale_out);

/* Seeded synthetic initial PV: amplitude * (N(0,1) white noise smoothed by a
 * separable Gaussian of standard deviation sigma cells), sdata (ii, jj, L). */
PQ_API int pq_make_ic(int ii, int jj, int layers, uint64_t seed, double amplitude, double sigma, double* out);

/* ---- context ------------------------------------------------------------ */

/* helm_cache + helmholtz_cache allocation (qg3p_aux.F90:152-193,
 * qg3p_helmholtz.F90:292-386) plus the device model state. */
PQ_API int pq_create(pq_ctx** out, const pq_model_desc* d, int device);
PQ_API void pq_destroy(pq_ctx* ctx);
PQ_API const char* pq_last_error(const pq_ctx* ctx);
PQ_API size_t pq_device_bytes(const pq_ctx* ctx);

/* ---- drop-in elliptic entry points --------------------------------------- */

/* helm(helm_c, zeta), qg3p_helmholtz.F90:614-769: zeta (ii, jj, L) holds the
 * right-hand side on entry and the solution on exit, with helm's in-place
 * semantics (boundary entries untouched except row ii and column 1, which
 * are zeroed).  The layers of the context are the modes, ss = d->ss. */
PQ_API int pq_helm(pq_ctx* ctx, double* zeta, int ptr_kind);

/* pv_inversion(strat, vbc, zeta, hcache, psi), qg3p_aux.F90:452-479:
 * zeta sdata (ii, jj, L) in, psi sdata (ii, jj, L) out.  Returns PQ_ERR_NAN
 * where the reference aborts on a NaN psiC. */
PQ_API int pq_pv_inversion(pq_ctx* ctx, const double* zeta_sdata, double* psi_sdata, int ptr_kind);

/* ---- Dirichlet boundary conditions (qg_laplace_bc) -----------------------
 * The public routines of qg3p_laplace_bc.F90:14-36 on the context's grid,
 * as device kernels.  field / rhs: (ii, jj, layers) column-major, layers
 * 1..L of the context (1 for the reference's *_layer variants).  bc: nbc
 * values, nbc = 1 (one value for every layer, *_layers_single) or
 * nbc = layers (one per layer, *_layers_multiple).  Closed basin: bc is
 * the value on all four walls and bc_d must be NULL.  Channel (periodic_j):
 * bc is the wall i = 1 (bc_b) and bc_d the wall i = ii (NULL: the same as
 * bc), the *_periodic_* variants.  Host arrays are copied in and out and
 * the call returns when done; device arrays are updated in place,
 * asynchronously on pq_stream(ctx).  Results equal the reference's to the
 * bit (each node subtracts or takes its values in the reference's order).
 *
 * add_laplace_bc_rhs (:55-190): rhs(i, j) -= bc on the nodes next to each
 * wall (i = 2, ii-1 and, closed basin, j = 2, jj-1; a corner of that ring
 * twice). */
PQ_API int pq_add_laplace_bc_rhs(pq_ctx* ctx, double* rhs, int layers, const double* bc, const double* bc_d,
                                 int nbc, int ptr_kind);
/* apply_dirichlet_bc (:193-374): the boundary nodes take the wall values. */
PQ_API int pq_apply_dirichlet_bc(pq_ctx* ctx, double* field, int layers, const double* bc, const double* bc_d,
                                 int nbc, int ptr_kind);
/* laplace_bc_rhs (:42-51): rhs (ii, jj) = 0, then add_laplace_bc_rhs with
 * one value. */
PQ_API int pq_laplace_bc_rhs(pq_ctx* ctx, double bc, double* rhs, int ptr_kind);

/* ---- model state and time stepping -------------------------------------- */

/* START_PERTURB initialisation, qg3.F90:365-404 and :450-459: zeta sdata
 * (ii, jj, L) initial PV; Dirichlet 0, inversion, rel and boundary PV, zeroed
 * CABARET fields, zeta_old = zeta, tweights 0.5.  For the leapfrog scheme
 * zeta_ic holds both time levels, (ii, jj, L, 2), and the forward-Euler start
 * (:463-497) follows. */
PQ_API int pq_init_perturb(pq_ctx* ctx, const double* zeta_ic, int ptr_kind);

/* nsteps iterations of the CABARET timestep_loop body (qg3.F90:590-957):
 * adapt_dt, predictor, beta, pv_inversion, rel, boundary PV, forcing, cell
 * boundaries, extrapolator, flux, corrector, zeta_old = zeta.  Runs as
 * captured CUDA graphs on the context's stream. */
PQ_API int pq_step(pq_ctx* ctx, int nsteps);

/* One CABARET step with the time step and time weights the caller gives, as
 * the reference's loop passes dt, tweight_a and tweight_u to every cabaret_*
 * routine (qg3.F90:598-807, qg3p_aux.F90:993-1642): a host driver that
 * chooses dt itself.  The values must satisfy cabaret_adapt_dt's checks
 * (dt > 0, tweight_a >= 0, 0 <= tweight_u <= 1, qg3p_aux.F90:982-988); the
 * step recomputes the predictor with this dt.  With adapt_dt set, the
 * device still adapts dt at the end of the step (pq_get_scalars). */
PQ_API int pq_cabaret_step(pq_ctx* ctx, double dt, double tweight_a, double tweight_u);

/* pq_step without the final wait: enqueues the steps on the context's stream
 * and returns.  pq_check waits for the stream and reports a NaN psiC or
 * energy (PQ_ERR_NAN) raised by the device since initialisation. */
PQ_API int pq_step_async(pq_ctx* ctx, int nsteps);
PQ_API int pq_check(pq_ctx* ctx);

/* One step with the prognostic state exchanged through caller buffers, the
 * way a host-side driver that owns its arrays would call the solver: if
 * zeta_in is not NULL it replaces zeta (sdata (ii, jj, L)) before the step;
 * if psi_out is not NULL it receives the step's psi (sdata).  Asynchronous:
 * host buffers should be pinned; pq_check or pq_sync completes the copies.
 * With both host buffers given, the copies are pipelined: the input and
 * output transfers run on the context's own copy streams through device
 * staging buffers, overlapping the kernels of the neighbouring calls'
 * steps.  The buffers must stay valid, and zeta_in unchanged, until
 * pq_sync / pq_check; successive calls may reuse the same buffers (psi_out
 * then holds the last step's psi).  The first copy of a sequence follows
 * the work already on pq_stream(ctx); pq_join(ctx) makes work enqueued on
 * that stream afterwards follow the sequence's copies, without a host wait. */
PQ_API int pq_step_exchange(pq_ctx* ctx, const double* zeta_in, double* psi_out, int ptr_kind);
PQ_API int pq_join(pq_ctx* ctx);

/* energy(strat, psi, ekin, epot), qg3p_diagnostics.F90:778-863, on the
 * current psi.  ekin: L doubles. */
PQ_API int pq_energy(pq_ctx* ctx, double* ekin, double* epot);

/* cabaret_cfl, qg3p_aux.F90:920-942, of the last step's face velocities. */
PQ_API int pq_cfl(pq_ctx* ctx, double* cfl);

/* Copy a state field (PQ_F_*) out of / into the context, reference layout,
 * host memory. */
PQ_API int pq_get_field(pq_ctx* ctx, int field, double* out);
PQ_API int pq_set_field(pq_ctx* ctx, int field, const double* in);

/* dt, tweight_a, tweight_u the last step ran with, and model_time
 * (non-dimensional): the reference's state after a step (it adapts dt at the
 * start of the next one, qg3.F90 timestep loop). */
PQ_API int pq_get_scalars(pq_ctx* ctx, double* out4);

/* ---- checkpoint dump and pickup ------------------------------------------
 * The reference's checkpoint files, byte for byte: Fortran unformatted stream
 * records (4-byte byte count, REAL(8) data column-major, byte count;
 * qg3p_io.F90:574-760), native byte order.
 *   s_path     qg<L>_<ii>_s.d: model_time_day, total_time_day, L x psi sdata,
 *              L x zeta sdata (qg3.F90:836-856); leapfrog records hold both
 *              time levels.
 *   supp_path  qg<L>_<ii>_s_supp.d (CABARET only, qg3.F90:858-881):
 *              model_time_day, total_time_day, dt, L x ui, L x uj,
 *              L x zeta_fi, L x zeta_fj (interior faces), L x res,
 *              L x res_beta.
 * pq_write_checkpoint writes the current state; model_time_day =
 * model_time * t_scale / 86400 and total_time_day = start_time_day +
 * model_time_day (qg3.F90:661, 844-845).  supp_path may be NULL to write the
 * _s file alone (the reference writes _s_supp every k_cp dumps).
 * pq_read_checkpoint is START_PICKUP (read_parallel_checkpoint,
 * qg3p_io.F90:202-314, then qg3.F90:316-363 and :448-497): CABARET takes dt
 * from the file, sets uimo / ujmo to the face velocities of psi, advances
 * zeta half a step with the stored fluxes, zeta_old = zeta, model_time =
 * dt / 2; leapfrog sets rel from psi on both levels, zeta_old = zeta,
 * model_time = 0 and skips the forward-Euler start.  The file times must
 * agree (PQ_ERR_ARG "Input times do not match", as the reference aborts);
 * total_time_day receives the checkpoint's total time (the new run's
 * start_time_day) and may be NULL.  A channel (periodic_j) saves rows
 * 2..jj+1 and j faces 2..jj+2 (it is its own j neighbour: fa_j_min = 1,
 * fa_j_max = jj + 2, qg3p_base.F90:893-918) and its pickup fills psi's
 * periodic halo rows first (qg3.F90:324-339). */
PQ_API int pq_write_checkpoint(pq_ctx* ctx, const char* s_path, const char* supp_path, double t_scale,
                               double start_time_day);
PQ_API int pq_read_checkpoint(pq_ctx* ctx, const char* s_path, const char* supp_path, double* total_time_day);

/* ---- time-averaged streamfunction ----------------------------------------
 * psi_av (qg3.F90:93, 502-503, 672-680, 725): while on, every step whose
 * model time (after the CABARET step's first half increment, after the
 * leapfrog sub-step) exceeds `threshold` = max_spin - start_time
 * (non-dimensional) adds dt * psi (the step's inversion result, every node)
 * to the sum and dt to diagnostic_time.  The sum is added to inside the fused
 * CABARET kernel.  pq_average(ctx, 1, threshold) allocates (first time) and
 * clears the sum, as initialisation does (pq_init_perturb and
 * pq_read_checkpoint clear it too); pq_average(ctx, 0, 0) frees it.  Call it
 * between steps, not while a stream capture is in progress.
 * pq_get_average: psi_av / diagnostic_time as sdata (ii, jj, L), the field
 * the reference writes to qg<L>_<ii>_s_av.d (:886-899), and diagnostic_time
 * (either pointer may be NULL; PQ_ERR_STATE before any step was averaged).
 * pq_write_average writes that file: model_time_day, total_time_day, L x
 * the averaged sdata, in the checkpoint's record format. */
PQ_API int pq_average(pq_ctx* ctx, int enable, double threshold);
/* enable = 2 also accumulates the 23 quad eddy covariances (qg3.F90:683-721,
 * the reference's `quad` option) in one extra kernel per CABARET step or
 * leapfrog sub-step (on the level just inverted):
 * products of the zonal / meridional velocities (0 where the reference
 * never writes them, rel / alpha, 0 or NaN on the walls by the velocity
 * boundary condition), interface velocities, thickness, rel, zeta and psi,
 * each times dt.  pq_get_quad copies accumulator q (0..22, the order of
 * PQ_QUAD_NAMES) times 1 / diagnostic_time as (ii, jj, layers of q);
 * pq_write_quad writes the qg<L>_<ii>_quad_av.d file (qg3.F90:903-929).
 * The reference leaves ut, vt, rt and tt uninitialised; here all start at 0.
 * Closed basin or channel (no j walls: v is central across the periodic
 * seam). */
#define PQ_QUAD_NAMES "uu vv uu_i vv_i uv ur vr rr pr uz vz zz zr pp pz ut vt rt tt sc_ub sc_vb sc_bb sc_bb_i"
PQ_API int pq_get_quad(pq_ctx* ctx, int q, double* out);
PQ_API int pq_write_quad(pq_ctx* ctx, const char* path, double t_scale, double start_time_day);
PQ_API int pq_get_average(pq_ctx* ctx, double* psi_av, double* diagnostic_time);
PQ_API int pq_write_average(pq_ctx* ctx, const char* path, double t_scale, double start_time_day);

/* Block until the context's queued device work is complete. */
PQ_API int pq_sync(pq_ctx* ctx);

/* The CUDA stream the context's work is ordered on (a cudaStream_t). */
PQ_API void* pq_stream(pq_ctx* ctx);

/* Per-kernel CUDA-event timing of steps launched outside CUDA graphs (an odd
 * single step, or every step of pq_step_async(ctx, 1)).  pq_kernel_times
 * waits for the stream and returns, for the four kernels of a step
 * (forward DST, tridiagonal, inverse DST + back-projection, fused CABARET),
 * the summed milliseconds and launch counts since the last call. */
PQ_API int pq_kernel_timing(pq_ctx* ctx, int enable);
PQ_API int pq_kernel_times(pq_ctx* ctx, double* ms4, long* launches4);

/* ---- energy for callers that cannot allocate device memory --------------
 * No counterpart in the reference: its energy() (qg3p_diagnostics.F90:778-
 * 863) runs on host arrays.  pq_energy_noalloc computes the same ekin / epot
 * as pq_energy on a psi array the caller already owns on the device, without
 * a context and without allocating anything.  It is for host drivers that
 * cannot let a library allocate device memory: one whose device memory is
 * reserved up front (an HBM budget, or a caching allocator that owns the
 * whole device), where a cudaMalloc would fail or break the budget, and one
 * that keeps its streams pipelined and cannot afford the device-wide
 * synchronisation that cudaMalloc / cudaFree may cause.
 *   psi        device, (ld, jj, layers) column-major, node values (sdata)
 *   periodic_j 0: closed basin; 1: channel periodic in j (full row weights,
 *              the kinetic-energy cells of row 1 wrap to row jj, and the
 *              area (ii - 1) jj), as pq_energy does for a channel context
 *   h, s2      host, layers entries (strat%h, strat%s2)
 *   out        device, layers + 1 doubles: ekin(1:layers), then epot
 *   stream     cudaStream_t to order the work on (NULL: legacy default stream)
 * Limits: jj <= PQ_NOALLOC_MAX_JJ, layers <= PQ_MAX_LAYERS; larger sizes
 * return PQ_ERR_ARG.  The reduction's scratch (row partials and a counter,
 * about 300 KB) is a fixed array inside the library that every GPU which
 * loads it keeps until exit; all calls share it and it keeps the last
 * call's contents (each call clears the counter it needs at zero), so calls
 * whose device work overlaps race and must be serialised by the caller.
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before starting any stream capture.  Asynchronous: `out` is valid once
 * the stream has reached the call. */
#define PQ_NOALLOC_MAX_JJ 4097
PQ_API int pq_energy_noalloc(const double* psi, int ii, int jj, int layers, int ld, int periodic_j,
                             const double* h, const double* s2, double* out, void* stream);

/* Tile parameters of the step kernels (defaults per grid size are set by
 * pq_create; results do not depend on them).
 *   cab_kernel CABARET step formulation: 0 one CTA per 28 x 16 tile and
 *              layer; 1 warp sweeps down bands of cab_band rows of a
 *              32-column strip, claimed from a queue by resident warps;
 *              2 the same with two columns per lane (64-column strips; the
 *              mixed form only).  Default: tiles up to jj = 700, then
 *              sweeps; two-column sweeps in the mixed form above jj = 1500
 *   cab_band   output rows per sweep, 4..128 (default: 8 up to 300 rows,
 *              32 up to 700, then 24 (FP64) or 16 (mixed) up to 1500, and
 *              40 (FP64) or 24 (mixed) above)
 *   dst_group  row groups per DST CTA: a CTA holds dst_group * layers
 *              warps (0: automatic, 1); layers * dst_group <= 8
 *   dst_lanes, dst_lanes_inv  lanes per (row, mode) unit of the forward
 *              and the inverse row DSTs, a power of two up to 64 with
 *              (ii - 1) / 2 / lanes values per lane in 2..32 (0: default,
 *              one warp up to ii = 513, two warps from ii = 1025 forward and
 *              ii = 2049 inverse where the layers fit); units wider than a
 *              warp synchronise by named barriers.  A CTA (layers * rows *
 *              lanes threads) must stay within 320 threads with 16 values
 *              per lane, 256 otherwise. */
typedef struct pq_tuning {
    int cab_band;
    int dst_group;
    int cab_kernel;
    int dst_lanes;
    int dst_lanes_inv;
    int pdl;            /* 1: programmatic dependent launch of the step kernels,
                           each scheduled while its predecessor finishes (it
                           waits for the predecessor's results before reading
                           anything); 0 (default): one after another, which
                           measured 0-5 % faster on B200 */
    int dst_algo;       /* row DSTs of the mixed form's baroclinic modes:
                           PQ_DST_BUTTERFLY (FP32 FFT in registers, the default)
                           or PQ_DST_TENSOR (dense DST-matrix products on the
                           tensor cores, three-term BF16 split with FP32
                           accumulation; ii >= 65); 0 keeps the current one.
                           The FP64 form and the barotropic mode always use
                           the FP64 butterfly. */
    int reserved[1];
} pq_tuning;
#define PQ_DST_BUTTERFLY 1
#define PQ_DST_TENSOR 2
/* The autotuner: times the step's inversion with each row-DST algorithm
 * this context supports (the butterfly, and for the mixed form the tensor-
 * core DST) on its own stream, selects the faster, and returns it in
 * *choice (PQ_DST_*).  The decision is cached per (ii, jj, L, channel) for
 * the process, so later contexts of the same shape take it without timing.
 * The model state is left as it was (psi and the scalars are restored).
 * Call it between steps, not while a stream capture is in progress. */
PQ_API int pq_autotune(pq_ctx* ctx, int* choice);
PQ_API int pq_set_tuning(pq_ctx* ctx, const pq_tuning* t);
PQ_API int pq_get_tuning(pq_ctx* ctx, pq_tuning* t);

/* ---- batched Helmholtz solves ---------------------------------------- */

/* Many independent helm problems (qg3p_helmholtz.F90:614-769, each with its
 * own helm_cache) of mixed sizes and mode counts, solved by grouped launches
 * captured in one CUDA graph.  Member k is an (ii[k], jj[k], layers[k])
 * problem whose layer l has the Helmholtz constant ss[sum_{q<k} layers[q] + l];
 * its right-hand side goes in with pq_batch_set_rhs and the solution, with
 * helm's in-place semantics (row ii zeroed, boundary entries untouched), comes
 * out with pq_batch_get.  The data stay on the device between solves. */
typedef struct pq_batch pq_batch;
PQ_API int pq_batch_create(pq_batch** out, int n, const int* ii, const int* jj, const int* layers,
                           const double* ss, int device);
/* The same with a precision: PQ_PREC_FP64 (pq_batch_create), or
 * PQ_PREC_MIXED -- every member's first layer (the barotropic, ss = 0
 * problem of a stratified model) keeps the FP64 transforms, the other
 * layers are transformed in FP32, the tridiagonal solves stay FP64 -- with
 * dst_algo PQ_DST_BUTTERFLY (FP32 FFT), PQ_DST_TENSOR (tensor-core DST,
 * three-term BF16 split, where ii >= 65 and L >= 2) or 0 (per DST class
 * (ii, L), whichever is faster when timed at creation). */
PQ_API int pq_batch_create_ex(pq_batch** out, int n, const int* ii, const int* jj, const int* layers,
                              const double* ss, int precision, int dst_algo, int device);
/* The row-DST algorithm member k's FP32 layers use (PQ_DST_*). */
PQ_API int pq_batch_member_dst_algo(const pq_batch* b, int k);
PQ_API void pq_batch_destroy(pq_batch* b);
PQ_API const char* pq_batch_last_error(const pq_batch* b);
PQ_API size_t pq_batch_device_bytes(const pq_batch* b);
PQ_API void* pq_batch_stream(pq_batch* b);
PQ_API int pq_batch_set_rhs(pq_batch* b, int k, const double* rhs, int ptr_kind);
PQ_API int pq_batch_get(pq_batch* b, int k, double* out, int ptr_kind);
PQ_API int pq_batch_solve_async(pq_batch* b); /* all members, on pq_batch_stream */
PQ_API int pq_batch_sync(pq_batch* b);
/* set_rhs + solve + get for every member (zeta[k] in/out), then sync. */
PQ_API int pq_batch_helm(pq_batch* b, double* const* zeta, int ptr_kind);
/* Kernel launches one solve makes (3 phases x classes, plus two per member
 * whose layers take the tensor-core DST). */
PQ_API int pq_batch_launch_count(const pq_batch* b);

/* ---- serving: many model runs, continuously batched --------------------- */

/* Runs (CABARET, fixed dt) are queued by pq_server_submit and admitted while
 * the device bytes of the admitted and pooled contexts stay within
 * hbm_budget_bytes.  Each pq_server_poll retires finished runs, admits
 * queued ones (initialisation + first step) and advances every active run
 * with one launch per kernel per shape group and step: the group with the
 * most work per step by up to max_steps steps, cheaper groups
 * proportionally more (up to 64 max_steps), each group up to its nearest
 * member's end, so that small runs keep their own pace.  A
 * run's result is bit-identical to running it alone (pq_init_perturb +
 * pq_step).  Contexts of finished runs are pooled by configuration and
 * reused. */
typedef struct pq_server pq_server;
PQ_API int pq_server_create(pq_server** out, size_t hbm_budget_bytes, int device);
PQ_API void pq_server_destroy(pq_server* s);
PQ_API const char* pq_server_last_error(const pq_server* s);
/* zeta_ic: (ii, jj, L) host array, copied.  PQ_ERR_BUDGET: the run alone
 * exceeds the budget. */
PQ_API int pq_server_submit(pq_server* s, const pq_model_desc* desc, const double* zeta_ic, int nsteps, long* id);
PQ_API int pq_server_poll(pq_server* s, int max_steps, int* active, int* queued);
/* 0 queued, 1 running, 2 finished, 3 failed, -1 unknown id.  A run fails
 * alone -- the others carry on -- when its device status reports a NaN
 * psiC or energy (where the reference aborts the program,
 * qg3p_aux.F90:504-510, qg3p_diagnostics.F90:858-861; checked after every
 * round) or when its admission fails (an invalid description, a failed
 * allocation); its context is destroyed. */
PQ_API int pq_server_status(pq_server* s, long id);
/* psi (ii, jj, L) of a finished run and t3 = {submitted, started, finished}
 * in seconds of pq_server_clock; releases the run (PQ_ERR_NOTFOUND after).
 * For a failed run: t3 (finished = when it failed), no psi, and the run's
 * error code (PQ_ERR_NAN, PQ_ERR_ARG, PQ_ERR_NOMEM, ...) with
 * pq_server_last_error giving its message. */
PQ_API int pq_server_collect(pq_server* s, long id, double* psi, double* t3);
PQ_API size_t pq_server_device_bytes(const pq_server* s);
PQ_API double pq_server_clock(const pq_server* s);
PQ_API long pq_server_launches(const pq_server* s);

/* ---- ensembles: many runs of one configuration stepped together ---------
 * n members share a configuration (CABARET, fixed dt, closed basin) and a
 * stream.  Each member is initialised (START_PERTURB, qg3.F90:365-404) from
 * its own initial PV; then every step (the timestep_loop body,
 * qg3.F90:590-957) is one launch per kernel over all members, replayed as
 * CUDA graphs, so that many small or medium runs fill the GPU.  A member's
 * results are the same as the run alone.  pq_ensemble_member gives a
 * member's context for pq_get_field / pq_energy / pq_write_checkpoint (call
 * pq_ensemble_sync first); do not step a member on its own, nor change its
 * settings (pq_set_tuning, pq_average) once the ensemble has stepped: the
 * merged launches use the members' descriptors as they were at the first
 * step.  The row-DST
 * algorithm (pq_ensemble_autotune / pq_ensemble_set_dst_algo, as pq_autotune
 * and pq_tuning.dst_algo) is chosen before the first step. */
typedef struct pq_ensemble pq_ensemble;
PQ_API int pq_ensemble_create(pq_ensemble** out, int n, const pq_model_desc* desc, int device);
PQ_API void pq_ensemble_destroy(pq_ensemble* e);
PQ_API const char* pq_ensemble_last_error(const pq_ensemble* e);
PQ_API int pq_ensemble_size(const pq_ensemble* e);
PQ_API pq_ctx* pq_ensemble_member(pq_ensemble* e, int k);
PQ_API void* pq_ensemble_stream(pq_ensemble* e);
PQ_API int pq_ensemble_init(pq_ensemble* e, int k, const double* zeta_ic, int ptr_kind);
PQ_API int pq_ensemble_autotune(pq_ensemble* e, int* choice);
PQ_API int pq_ensemble_set_dst_algo(pq_ensemble* e, int algo);
/* nsteps steps of every member, enqueued on pq_ensemble_stream; _sync
 * waits and reports a NaN psiC or energy of any member (PQ_ERR_NAN, the
 * member named in the message). */
PQ_API int pq_ensemble_step_async(pq_ensemble* e, int nsteps);
PQ_API int pq_ensemble_sync(pq_ensemble* e);
PQ_API int pq_ensemble_step(pq_ensemble* e, int nsteps);

/* Number of kernel launches the last pq_step enqueued. */
PQ_API long pq_last_launch_count(const pq_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* PEQUOD_B200_H */

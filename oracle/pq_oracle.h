/*
 * pq_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of PEQUOD's serial (one MPI rank) QG time-step hot
 * path, used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg as the parity checker.  Nothing in the pequod_b200 product links,
 * loads or calls this library.
 *
 * Parity status: pinned.  The restatement is checked against the reference's
 * own known-answer tests (unittest/test_helmholtz.F90, test_laplace_bc.F90,
 * test_mean.F90, test_energy_2.F90, test_stratification.F90,
 * test_cabaret_cfl.F90, test_eigendecompose.F90, test_inverse.F90,
 * test_solve.F90) in tests/test_oracle_kats.py.  The reference itself
 * (Fortran 2003 + MPI + LAPACK) cannot be compiled in this environment, so
 * there is no oracle/_ref build.
 *
 * Array conventions follow the reference exactly: Fortran column-major, i
 * (the first, "meridional" index) fastest, 1-based in the comments.
 *   sdata arrays      (ii,   jj,   L)
 *   full data arrays  (ii+2, jj+2, L)   one-node halo, sdata = data(2:ii+1, 2:jj+1, :)
 *   FLUX_II faces     (ii+3, jj+2, L)
 *   FLUX_JJ faces     (ii+2, jj+3, L)
 * qg3p_base.F90:1322-1323, 2808-2818.
 */
#ifndef PQ_ORACLE_H
#define PQ_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Velocity boundary condition types, qg3p_diagnostics.F90:57-58. */
#define OR_BC_PARTIAL_SLIP 1
#define OR_BC_NO_SLIP 2
#define OR_BC_FREE_SLIP 3

/* ---- stratification (qg3p_diagnostics.F90:125-450) ---------------------- */
void or_strat_l2(double rd_bcl, double h1, double h2, double* s1, double* s2);
void or_strat_l3(double rd_bcl1, double rd_bcl2, double h1, double h2, double h3,
                 double* s1, double* s21, double* s22, double* s3);
/* Full stratification object from layer thicknesses and s1(2:L), s2(1:L-1)
 * (allocate_stratification_parameters, :210-236).  Outputs are the scaled
 * h, s1, s2 (length L; s1[0] and s2[L-1] are set to 0), ss (L), and the
 * L x L column-major modes_to_z / z_to_modes matrices. */
int or_strat_from_parameters(int layers, const double* h, const double* s1_in,
                             const double* s2_in, double l_scale,
                             double* h_out, double* s1_out, double* s2_out,
                             double* ss, double* m2z, double* z2m);
/* Stratification from deformation radii (allocate_stratification_l1/l2/l3).
 * rd has layers-1 entries. */
int or_strat_from_rd(int layers, const double* rd, const double* h, double l_scale,
                     double* h_out, double* s1_out, double* s2_out,
                     double* ss, double* m2z, double* z2m);
/* Small dense linear algebra used by the stratification set-up
 * (replaces the LAPACK calls in lapack_interfaces.F90). */
int or_eigen_real_tridiag(int n, const double* a, double* eigval, double* eigvec);
int or_inverse(int n, const double* a, double* ainv);
int or_solve(int n, const double* a, const double* rhs, double* x);
double or_determinant(int n, const double* a);

/* ---- Helmholtz solver (qg3p_helmholtz.F90) ------------------------------ */
typedef struct or_helm_cache or_helm_cache;
or_helm_cache* or_helm_create(int ii, int jj, int layers, const double* ss, int periodic_j);
void or_helm_destroy(or_helm_cache* h);
/* helm(helm_c, zeta): zeta(ii, jj, layers) in/out. */
int or_helm(or_helm_cache* h, double* zeta);
/* Raw FFTPACK-convention sine transform of x(1:n+1), n = ii - 2. */
int or_sint(or_helm_cache* h, double* x);

/* ---- Dirichlet boundary conditions (qg3p_laplace_bc.F90) ---------------- */
void or_add_laplace_bc_rhs(int ii, int jj, int layers, int periodic_j,
                           double bc, double bc_d, double* rhs);
void or_apply_dirichlet_bc(int ii, int jj, int layers, int periodic_j,
                           double bc, double bc_d, double* zeta);

/* ---- reductions (qg3p_diagnostics.F90:669-863) -------------------------- */
double or_mean(int ii, int jj, int periodic_j, const double* psi);
/* psi is a full data array (ii+2, jj+2, L); h, s2 as stratification. */
void or_energy(int ii, int jj, int layers, int periodic_j, const double* h,
               const double* s2, const double* psi, double* ekin, double* epot);

/* ---- double-gyre driver set-up (qg3.F90:150-307) ------------------------ */
typedef struct {
    int ii, jj, layers;
    double basinscale;        /* cm */
    double dt;                /* s */
    double f0, beta;          /* s^-1, cm^-1 s^-1 */
    double H[8];              /* cm */
    double gprime[8];         /* cm s^-2, interfaces 1..L-1 */
    double tau;               /* cm^2 s^-2 */
    double wind_asym, wind_tilt, wind_shift;
    double visc, visc_bot;    /* cm^2 s^-1, s^-1 */
    double alpha;             /* cm; >= 1e100: free slip */
    int partial_slip;
    double max_dt;            /* s */
    double u_scale;           /* cm s^-1 */
} or_physical;

typedef struct {
    double l_scale, t_scale;
    double dt, max_dt, alpha, viscosity, visc_bot;
    int bc_type;
    double beta[8], h[8], s1[8], s2[8], ss[8];
    double m2z[64], z2m[64];  /* L x L column-major, leading dimension L */
} or_setup;

/* Non-dimensional model parameters and the layer-1 wind forcing (ii, jj)
 * of the double gyre, from the physical parameters alone. */
int or_setup_double_gyre(const or_physical* p, or_setup* out, double* wind);
/* Seeded synthetic initial PV, (ii, jj, L) sdata. */
int or_make_ic(int ii, int jj, int layers, unsigned long long seed, double amplitude, double sigma,
               double* out);

/* ---- full model, one rank, closed basin or channel --------------------- */
typedef struct {
    int ii, jj, layers;
    int periodic_j;       /* 0: closed basin */
    int scheme;           /* 0: CABARET (qg3.F90 CABARET branch), 1: leapfrog */
    int limiter;          /* CABARET_LIMITER */
    int bc_type;          /* OR_BC_* */
    double alpha;         /* non-dimensional partial-slip parameter */
    double dt;            /* non-dimensional time step */
    double viscosity, visc_bot;
    int adapt_dt;
    double target_cfl, max_dt, max_dt_increase;
    double ra_nu, ra_alpha;   /* leapfrog Robert-Asselin-Williams filter */
    const double* beta;       /* [L] */
    const double* h;          /* [L] non-dimensional thicknesses */
    const double* s1;         /* [L] */
    const double* s2;         /* [L] */
    const double* ss;         /* [L] */
    const double* m2z;        /* [L*L] */
    const double* z2m;        /* [L*L] */
    const double* force_wind; /* [ii*jj] or NULL */
} or_params;

typedef struct or_model or_model;
or_model* or_model_create(const or_params* p);
void or_model_destroy(or_model* m);
/* START_PERTURB initialisation (qg3.F90:365-404 and :450-459, plus the
 * forward-Euler start :463-497 for leapfrog).  zeta_ic: (ii, jj, L) sdata, or
 * (ii, jj, L, 2) for leapfrog. */
int or_model_init(or_model* m, const double* zeta_ic);
/* n time steps (one timestep_loop body each; one leapfrog sub-step each). */
int or_model_step(or_model* m, int nsteps);
/* Copy a state field out in reference layout.  Names: "psi", "zeta", "rel",
 * "zeta_old", "ui", "uj", "uimo", "ujmo", "zeta_fi", "zeta_fj", "res",
 * "res_beta" (leapfrog: "psi2", "zeta2", "rel2", "zeta_old2" for level 2).
 * Returns the number of doubles, or -1 for an unknown name.  out may be NULL
 * to query the size. */
long or_model_get(or_model* m, const char* name, double* out);
long or_model_set(or_model* m, const char* name, const double* in);
/* One CABARET step split at the reference's data output / exit point:
 * or_model_step_to_dump leaves the state its checkpoint holds,
 * or_model_finish_step completes the step (corrector, zeta_old, time). */
int or_model_step_to_dump(or_model* m);
int or_model_finish_step(or_model* m);
/* Time average of psi (qg3.F90:502-503, 672-680, 725): enable clears the
 * sum; steps whose model time (after the first half increment) exceeds
 * threshold = max_spin - start_time add dt * psi.  get returns
 * diagnostic_time and copies the sum (ii, jj, L). */
void or_model_average(or_model* m, int enable, double threshold);
/* enable = 2 also accumulates the 23 quad eddy covariances (qg3.F90:683-721);
 * or_model_get_quad copies accumulator q (output order) unscaled and returns
 * its length, or -1. */
long or_model_get_quad(or_model* m, int q, double* out);
double or_model_get_average(or_model* m, double* sum);
/* Checkpoint pickup (qg3.F90:314-363, :448-497) on fields loaded with
 * or_model_set; dt is the checkpoint's (CABARET; ignored for leapfrog). */
int or_model_pickup(or_model* m, double dt);
/* Scalars: dt, tweight_a, tweight_u, model_time. */
void or_model_scalars(or_model* m, double* out4);
int or_model_energy(or_model* m, double* ekin, double* epot);
double or_model_cfl(or_model* m);

/* Individual reference routines on reference-layout arrays. */
int or_pv_inversion(or_model* m, const double* zeta_data, double* psi_data);

#ifdef __cplusplus
}
#endif
#endif

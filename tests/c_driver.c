/* A plain C caller of the C ABI (include/pequod_b200.h), the way a Fortran
 * bind(C) module or any other host language calls it: no Python, no torch.
 *   c_driver setup          host-only set-up calls; prints their results
 *   c_driver run <steps>    a 129 x 129 x 3 double gyre on device 0: init,
 *                           steps, energy; prints ekin and epot */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pequod_b200.h"

static void phys129(pq_physical* p) {
    memset(p, 0, sizeof(*p));
    p->ii = p->jj = 129;
    p->layers = 3;
    p->basinscale = 128 * 30.0e5;
    p->dt = 1800.0;
    p->f0 = 9.4e-5;
    p->beta = 1.8e-13;
    p->H[0] = 3.0e4;
    p->H[1] = 7.0e4;
    p->H[2] = 3.0e5;
    p->gprime[0] = 1.5;
    p->gprime[1] = 0.75;
    p->tau = 0.8;
    p->wind_asym = 1.0;
    p->visc = 1.0e6;
    p->visc_bot = 1.0e-7;
    p->alpha = 120.0e5;
    p->partial_slip = 1;
    p->scheme = PQ_SCHEME_CABARET;
    p->limiter = 1;
    p->precision = PQ_PREC_FP64;
    p->target_cfl = 0.1;
    p->max_dt = 86400.0;
    p->max_dt_increase = 1.5;
    p->u_scale = 1.0;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    pq_physical p;
    pq_model_desc d;
    double ts = 0.0;
    double* wind = malloc(sizeof(double) * 129 * 129);
    phys129(&p);
    int rc = pq_setup_double_gyre(&p, &d, wind, &ts);
    if (rc) {
        printf("setup rc=%d\n", rc);
        return 1;
    }
    const size_t n = (size_t)129 * 129 * 3;
    double* ic = malloc(sizeof(double) * n);
    rc = pq_make_ic(129, 129, 3, 7, 1e-7 * ts, 3.0, ic);
    if (rc) return 1;
    if (!strcmp(argv[1], "setup")) {
        printf("t_scale %.17g dt %.17g ss %.17g %.17g %.17g wind %.17g ic %.17g\n", ts, d.dt, d.ss[0], d.ss[1],
               d.ss[2], wind[5 + 129 * 9], ic[1000]);
        /* no device here: creating a context must fail with a status code */
        pq_ctx* c = NULL;
        rc = pq_create(&c, &d, 0);
        printf("create rc=%d\n", rc);
        if (c) pq_destroy(c);
        return 0;
    }
    int steps = argc > 2 ? atoi(argv[2]) : 10;
    pq_ctx* c = NULL;
    rc = pq_create(&c, &d, 0);
    if (rc) {
        printf("create rc=%d %s\n", rc, c ? pq_last_error(c) : "");
        return 1;
    }
    rc = pq_init_perturb(c, ic, PQ_PTR_HOST);
    if (!rc) rc = pq_step(c, steps);
    double ekin[3], epot = 0.0;
    if (!rc) rc = pq_energy(c, ekin, &epot);
    if (rc) {
        printf("rc=%d %s\n", rc, pq_last_error(c));
        pq_destroy(c);
        return 1;
    }
    printf("ekin %.17g %.17g %.17g epot %.17g\n", ekin[0], ekin[1], ekin[2], epot);
    pq_destroy(c);
    free(ic);
    free(wind);
    return 0;
}

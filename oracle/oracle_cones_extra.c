/*
 * oracle_cones_extra.c -- exponential, power and PSD cone projections for
 * the oracle.  TEST INFRASTRUCTURE ONLY (see pdhcg_oracle.h).
 */
#include "pdhcg_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

static void unsupported(const char *what)
{
    fprintf(stderr, "[oracle] %s cones are not restated yet\n", what);
    abort();
}

void oracle_exp_project(double *x, const double *d, const double *q, double tau)
{
    (void)x; (void)d; (void)q; (void)tau;
    unsupported("exponential");
}

void oracle_pow_project(double *x, const double *d, const double *q, double tau, double alpha)
{
    (void)x; (void)d; (void)q; (void)tau; (void)alpha;
    unsupported("power");
}

void oracle_psd_project(int order, double *x)
{
    (void)order; (void)x;
    unsupported("PSD");
}

void oracle_exp_dual_residual(const double *rc, const double *d, double *out)
{
    (void)rc; (void)d; (void)out;
    unsupported("exponential");
}

void oracle_pow_dual_residual(const double *rc, const double *d, double alpha, double *out)
{
    (void)rc; (void)d; (void)alpha; (void)out;
    unsupported("power");
}

void oracle_psd_dual_residual(int order, const double *rc, const double *d, double *out)
{
    (void)order; (void)rc; (void)d; (void)out;
    unsupported("PSD");
}

/*
 * The synchrotron function F(x) = x * int_x^inf K_{5/3}(s) ds, for the
 * checker build.  Test infrastructure, not product code.
 *
 * The reference takes F(x) from GNU GSL (gsl_sf_synchrotron_1, called by
 * SYN_logFx_table, src/Synchrotron.c:31-41, for x <= 300).  GSL is linked as
 * -lgsl (Makefile:26 of the reference) but not vendored, and no version is
 * pinned; it is absent from this image.  This file restates F(x) from its
 * integral definition instead -- not from GSL's code:
 *
 *   K_nu(s) = int_0^inf exp(-s cosh t) cosh(nu t) dt, and
 *   int_x^inf exp(-s cosh t) ds = exp(-x cosh t) / cosh t, so
 *   F(x) = x int_0^inf exp(-x cosh t) cosh(5t/3) / cosh t dt,
 *
 * an even, analytic, double-exponentially decaying integrand, integrated by
 * the trapezoid rule with step 1/32 up to x cosh t = 800.  Checked against a
 * multiprecision Bessel-function quadrature and the small- and large-x
 * asymptotes (tests/test_emission_tables.py).  oracle/shim/ref_shims.c uses
 * it in place of gsl_sf_synchrotron_1, so the reference's own table code
 * (SYN_logFx_table, tracer_fp_synch_data_init_tables) runs in the checker.
 */
#include <math.h>

double oracle_synch_fx(double x)
{
    const double h = 1.0 / 32.0;
    const double r = (800.0 / x > 2.0) ? 800.0 / x : 2.0;
    const double tmax = log(r + sqrt(r * r - 1.0));
    const int n = (int)ceil(tmax / h);
    double s = 0.5 * exp(-x);
    int k;
    for (k = 1; k <= n; k++) {
        const double t = k * h;
        const double e = exp(t), e53 = exp(t * (5.0 / 3.0));
        const double ch = 0.5 * (e + 1.0 / e), ch53 = 0.5 * (e53 + 1.0 / e53);
        s += exp(-x * ch) * (ch53 / ch);
    }
    return x * h * s;
}

/*
 * Stand-in for <gsl/gsl_sf_synchrotron.h>: declares only the GSL symbols that the
 * reference hot-path sources reference.  Their definitions live in
 * oracle/shim/ref_shims.c.  Test infrastructure, not product.
 */
#ifndef CROMA_ORACLE_SHIM_GSL_SF_SYNCHROTRON_H
#define CROMA_ORACLE_SHIM_GSL_SF_SYNCHROTRON_H
double gsl_sf_gamma(double x);
double gsl_sf_hyperg_1F1(double a, double b, double x);
double gsl_sf_hyperg_U(double a, double b, double x);
double gsl_sf_synchrotron_1(double x);
#endif

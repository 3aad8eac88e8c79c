/* Stand-in for <gsl/gsl_sf_bessel.h> (oracle/_ref, test infrastructure).
 * The reference calls one function from it, gsl_sf_bessel_Jn, to build its
 * Bessel table (boundary.cpp:117-123); ref_shim.cpp evaluates it by its own
 * method (see there). */
#ifndef FELIS_REF_SHIM_GSL_SF_BESSEL_H
#define FELIS_REF_SHIM_GSL_SF_BESSEL_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_sf_bessel_Jn(const int n, const double x);
#ifdef __cplusplus
}
#endif
#endif

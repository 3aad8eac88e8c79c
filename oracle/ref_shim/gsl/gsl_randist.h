/* Stand-in for <gsl/gsl_randist.h> (oracle/_ref, test infrastructure).
 * The reference draws its shot-noise coefficients with gsl_ran_gaussian
 * (loadBeam.cpp:227-228, 406-407). */
#ifndef FELIS_REF_SHIM_GSL_RANDIST_H
#define FELIS_REF_SHIM_GSL_RANDIST_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
double gsl_ran_gaussian(const gsl_rng* r, const double sigma);
#ifdef __cplusplus
}
#endif
#endif

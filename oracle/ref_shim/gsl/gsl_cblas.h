/* Stand-in for <gsl/gsl_cblas.h> (oracle/_ref, test infrastructure): boundary.cpp
 * includes this header but calls nothing from it, so it is empty. */
#ifndef FELIS_REF_SHIM_GSL_CBLAS_H
#define FELIS_REF_SHIM_GSL_CBLAS_H
#endif

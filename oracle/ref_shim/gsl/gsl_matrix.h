/* Stand-in for <gsl/gsl_matrix.h> (oracle/_ref, test infrastructure): boundary.cpp
 * includes this header but calls nothing from it, so it is empty. */
#ifndef FELIS_REF_SHIM_GSL_MATRIX_H
#define FELIS_REF_SHIM_GSL_MATRIX_H
#endif

/* Stand-in for <gsl/gsl_matrix_complex_double.h> (oracle/_ref, test infrastructure): boundary.cpp
 * includes this header but calls nothing from it, so it is empty. */
#ifndef FELIS_REF_SHIM_GSL_MATRIX_COMPLEX_DOUBLE_H
#define FELIS_REF_SHIM_GSL_MATRIX_COMPLEX_DOUBLE_H
#endif

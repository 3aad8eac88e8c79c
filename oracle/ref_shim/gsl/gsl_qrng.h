/* Stand-in for <gsl/gsl_qrng.h> (oracle/_ref, test infrastructure).
 * The reference's loaders draw quasi-random points from a 7-dimensional
 * Halton generator (loadBeam.cpp:75, 3D) and a 3-dimensional Sobol generator
 * (loadBeam.cpp:303, 1D); ref_shim.cpp implements both from their published
 * definitions.  The Niederreiter type is declared because loadBeam.cpp names
 * it in commented-out lines only; allocating it ends the process. */
#ifndef FELIS_REF_SHIM_GSL_QRNG_H
#define FELIS_REF_SHIM_GSL_QRNG_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct gsl_qrng_type_s {
  const char* name;
  int kind; /* 1 Halton, 2 Sobol, 3 Niederreiter (not provided) */
} gsl_qrng_type;

typedef struct gsl_qrng_s gsl_qrng;

extern const gsl_qrng_type* gsl_qrng_halton;
extern const gsl_qrng_type* gsl_qrng_sobol;
extern const gsl_qrng_type* gsl_qrng_niederreiter_2;

gsl_qrng* gsl_qrng_alloc(const gsl_qrng_type* T, unsigned int dimension);
int gsl_qrng_get(const gsl_qrng* q, double x[]);
void gsl_qrng_free(gsl_qrng* q);
#ifdef __cplusplus
}
#endif
#endif

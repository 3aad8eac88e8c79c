/* Stand-in for <gsl/gsl_rng.h> (oracle/_ref, test infrastructure).
 * The reference uses the default generator as gsl_rng_env_setup() leaves it:
 * GSL_RNG_SEED from the environment (0 when unset), type MT19937
 * (loadBeam.cpp:66-69, 294-297).  Only that type is provided. */
#ifndef FELIS_REF_SHIM_GSL_RNG_H
#define FELIS_REF_SHIM_GSL_RNG_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct gsl_rng_type_s {
  const char* name;
} gsl_rng_type;

typedef struct gsl_rng_s gsl_rng;

extern const gsl_rng_type* gsl_rng_default;
extern unsigned long int gsl_rng_default_seed;
extern const gsl_rng_type* gsl_rng_mt19937;

const gsl_rng_type* gsl_rng_env_setup(void);
gsl_rng* gsl_rng_alloc(const gsl_rng_type* T);
void gsl_rng_free(gsl_rng* r);
double gsl_rng_uniform(const gsl_rng* r);
double gsl_rng_uniform_pos(const gsl_rng* r);
#ifdef __cplusplus
}
#endif
#endif

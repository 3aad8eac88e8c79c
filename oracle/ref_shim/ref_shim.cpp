// ref_shim.cpp — project-written stand-ins for the MPI and GSL calls that the
// reference's step loop and setup make, so that the reference's own .cpp files
// compile and run here unmodified (oracle/_ref).
//
// TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/felis_ref*, which tests/,
// __graft_entry__.smoke() and bench.py's reference arm run as a child process.
// The product never links it.
//
// Third-party arithmetic restated here (GSL 2.8 is pinned by the reference's
// makefile:9-14 but absent from this machine, so bit-equality with GSL itself
// is not pinned; each piece follows the published definition named below):
//   gsl_sf_bessel_Jn     Bessel's integral J_n(x) = (1/pi) int_0^pi cos(n t - x sin t) dt
//                        by the trapezoidal rule on 256 intervals of the period
//                        (exponentially convergent for a periodic analytic
//                        integrand; aliasing error below J_{256-n}(x), i.e. far
//                        below 1e-17 for the table's x <= 2 pi * 16)
//   gsl_qrng_halton      radical inverse of the point index in the first primes,
//                        first point at index 1 (Halton 1960)
//   gsl_qrng_sobol       Sobol points in Gray-code order (Antonov & Saleev 1979)
//                        with the direction numbers of Bratley & Fox 1988
//                        (ACM TOMS 14:88), 30-bit integers, first point 1/2;
//                        the three dimensions loadBeam.cpp:303 asks for
//   gsl_rng_default      MT19937 (Matsumoto & Nishimura 1998, init_genrand
//                        seeding; GSL maps seed 0 to 4357), uniform = u32 / 2^32
//   gsl_ran_gaussian     Marsaglia's polar method, returning sigma * y * f
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpi.h"
#include "gsl/gsl_qrng.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_sf_bessel.h"

// ---------------------------------------------------------------- MPI ------
namespace {
int g_rank = 0, g_size = 1;
bool g_ranks_read = false;

void read_ranks() {
  if (g_ranks_read) return;
  g_ranks_read = true;
  const char* n = getenv("FELIS_REF_NRANKS");
  const char* r = getenv("FELIS_REF_RANK");
  if (n && r) {
    const int nn = atoi(n), rr = atoi(r);
    if (nn >= 1 && rr >= 0 && rr < nn) {
      g_size = nn;
      g_rank = rr;
    }
  }
}

size_t type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }
}  // namespace

extern "C" {
int MPI_Init(int*, char***) {
  read_ranks();
  return MPI_SUCCESS;
}
int MPI_Finalize(void) {
  fflush(stdout);
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm, int* rank) {
  read_ranks();
  *rank = g_rank;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int* size) {
  read_ranks();
  *size = g_size;
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
  // Only reached when one process plays one of several ranks (timing runs):
  // the message is dropped.
  return MPI_SUCCESS;
}
int MPI_Recv(void* buf, int count, MPI_Datatype type, int, int, MPI_Comm, MPI_Status* st) {
  memset(buf, 0, (size_t)count * type_size(type));
  if (st) st->MPI_SOURCE = st->MPI_TAG = st->MPI_ERROR = 0;
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  if (sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)count * type_size(type));
  return MPI_SUCCESS;
}
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
  if (sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)count * type_size(type));
  return MPI_SUCCESS;
}
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) {
  fflush(stdout);
  fprintf(stderr, "felis_ref: MPI_Abort(%d)\n", code);
  exit(code == 0 ? 1 : code);
}
}  // extern "C"

// ------------------------------------------------------------ Bessel -------
extern "C" double gsl_sf_bessel_Jn(const int n, const double x) {
  // Trapezoidal rule over [0, pi] with M intervals (the integrand is even and
  // 2 pi periodic, so this is the periodic rule with 2M points).
  const int M = 128;
  const double h = M_PI / M;
  double s = 0.5 * (cos(0.0) + cos(n * M_PI - x * sin(M_PI)));
  for (int k = 1; k < M; ++k) {
    const double t = k * h;
    s += cos(n * t - x * sin(t));
  }
  return s / M;
}

// ------------------------------------------------------------ MT19937 ------
struct gsl_rng_s {
  uint32_t mt[624];
  int mti;
};

namespace {
const gsl_rng_type k_mt19937 = {"mt19937"};

void mt_seed(gsl_rng* r, unsigned long s) {
  if (s == 0) s = 4357;
  r->mt[0] = (uint32_t)(s & 0xffffffffUL);
  for (int i = 1; i < 624; ++i)
    r->mt[i] = (uint32_t)(1812433253UL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (uint32_t)i);
  r->mti = 624;
}

uint32_t mt_next(gsl_rng* r) {
  static const uint32_t mag01[2] = {0x0u, 0x9908b0dfu};
  if (r->mti >= 624) {
    int k = 0;
    for (; k < 624 - 397; ++k) {
      const uint32_t y = (r->mt[k] & 0x80000000u) | (r->mt[k + 1] & 0x7fffffffu);
      r->mt[k] = r->mt[k + 397] ^ (y >> 1) ^ mag01[y & 1u];
    }
    for (; k < 623; ++k) {
      const uint32_t y = (r->mt[k] & 0x80000000u) | (r->mt[k + 1] & 0x7fffffffu);
      r->mt[k] = r->mt[k + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1u];
    }
    const uint32_t y = (r->mt[623] & 0x80000000u) | (r->mt[0] & 0x7fffffffu);
    r->mt[623] = r->mt[396] ^ (y >> 1) ^ mag01[y & 1u];
    r->mti = 0;
  }
  uint32_t y = r->mt[r->mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}
}  // namespace

extern "C" {
const gsl_rng_type* gsl_rng_mt19937 = &k_mt19937;
const gsl_rng_type* gsl_rng_default = &k_mt19937;
unsigned long int gsl_rng_default_seed = 0;

const gsl_rng_type* gsl_rng_env_setup(void) {
  const char* t = getenv("GSL_RNG_TYPE");
  if (t && strcmp(t, "mt19937") != 0) {
    fprintf(stderr, "felis_ref: GSL_RNG_TYPE=%s is not provided (only mt19937)\n", t);
    exit(2);
  }
  const char* s = getenv("GSL_RNG_SEED");
  if (s) gsl_rng_default_seed = strtoul(s, nullptr, 0);
  gsl_rng_default = &k_mt19937;
  return gsl_rng_default;
}
gsl_rng* gsl_rng_alloc(const gsl_rng_type*) {
  gsl_rng* r = (gsl_rng*)malloc(sizeof(gsl_rng));
  mt_seed(r, gsl_rng_default_seed);
  return r;
}
void gsl_rng_free(gsl_rng* r) { free(r); }
double gsl_rng_uniform(const gsl_rng* r) { return mt_next(const_cast<gsl_rng*>(r)) / 4294967296.0; }
double gsl_rng_uniform_pos(const gsl_rng* r) {
  double x;
  do {
    x = gsl_rng_uniform(r);
  } while (x == 0);
  return x;
}
double gsl_ran_gaussian(const gsl_rng* r, const double sigma) {
  double x, y, r2;
  do {
    x = -1 + 2 * gsl_rng_uniform_pos(r);
    y = -1 + 2 * gsl_rng_uniform_pos(r);
    r2 = x * x + y * y;
  } while (r2 > 1.0 || r2 == 0);
  return sigma * y * sqrt(-2.0 * log(r2) / r2);
}
}  // extern "C"

// ------------------------------------------------- quasi-random points -----
struct gsl_qrng_s {
  int kind;
  unsigned int dim;
  unsigned long count;
  uint32_t x[8];
  uint32_t v[31][8];  // Sobol direction numbers, v[k][d] for k = 1..30
};

namespace {
const gsl_qrng_type k_halton = {"halton", 1};
const gsl_qrng_type k_sobol = {"sobol", 2};
const gsl_qrng_type k_nied = {"niederreiter-base-2", 3};

// Primitive polynomials of the first Sobol dimensions, as (degree, coefficient
// bits a_1..a_{s-1} of x^s + a_1 x^{s-1} + ... + a_{s-1} x + 1), and the free
// initial direction integers m_1..m_s (Bratley & Fox 1988, table 2).
struct SobolDim {
  int degree;
  unsigned coeffs;
  unsigned m_init[4];
};
const SobolDim k_sobol_dims[] = {
    {0, 0u, {1, 1, 1, 1}},  // first dimension: van der Corput, every m_k = 1
    {1, 0u, {1, 0, 0, 0}},  // x + 1
    {2, 1u, {1, 3, 0, 0}},  // x^2 + x + 1
};

void sobol_init(gsl_qrng* q) {
  const int B = 30;
  for (unsigned d = 0; d < q->dim; ++d) {
    const SobolDim& sd = k_sobol_dims[d];
    uint32_t m[31] = {};
    for (int k = 1; k <= B; ++k) {
      if (sd.degree == 0) {
        m[k] = 1;
      } else if (k <= sd.degree) {
        m[k] = sd.m_init[k - 1];
      } else {
        const int s = sd.degree;
        uint32_t mk = m[k - s] ^ (m[k - s] << s);
        for (int i = 1; i < s; ++i)
          if ((sd.coeffs >> (s - 1 - i)) & 1u) mk ^= m[k - i] << i;
        m[k] = mk;
      }
      q->v[k][d] = m[k] << (B - k);
    }
    q->x[d] = 0;
  }
}
}  // namespace

extern "C" {
const gsl_qrng_type* gsl_qrng_halton = &k_halton;
const gsl_qrng_type* gsl_qrng_sobol = &k_sobol;
const gsl_qrng_type* gsl_qrng_niederreiter_2 = &k_nied;

gsl_qrng* gsl_qrng_alloc(const gsl_qrng_type* T, unsigned int dimension) {
  // The reference draws 7-dimensional Halton and 3-dimensional Sobol points.
  if (T->kind == 3 || dimension > 7 || (T->kind == 2 && dimension > 3)) {
    fprintf(stderr, "felis_ref: quasi-random generator %s of dimension %u is not provided\n", T->name, dimension);
    exit(2);
  }
  gsl_qrng* q = (gsl_qrng*)calloc(1, sizeof(gsl_qrng));
  q->kind = T->kind;
  q->dim = dimension;
  q->count = 0;
  if (q->kind == 2) sobol_init(q);
  return q;
}

int gsl_qrng_get(const gsl_qrng* cq, double x[]) {
  gsl_qrng* q = const_cast<gsl_qrng*>(cq);
  if (q->kind == 1) {
    static const unsigned primes[7] = {2, 3, 5, 7, 11, 13, 17};
    ++q->count;
    for (unsigned d = 0; d < q->dim; ++d) {
      const unsigned p = primes[d];
      double f = 1.0 / p, r = 0.0;
      for (unsigned long c = q->count; c > 0; c /= p) {
        r += f * (double)(c % p);
        f /= p;
      }
      x[d] = r;
    }
    return 0;
  }
  // Sobol: flip the direction number of the lowest zero bit of the count.
  int ell = 1;
  for (unsigned long c = q->count; c & 1ul; c >>= 1) ++ell;
  if (ell > 30) return 1;
  for (unsigned d = 0; d < q->dim; ++d) {
    q->x[d] ^= q->v[ell][d];
    x[d] = (double)q->x[d] / 1073741824.0;
  }
  ++q->count;
  return 0;
}

void gsl_qrng_free(gsl_qrng* q) { free(q); }
}  // extern "C"

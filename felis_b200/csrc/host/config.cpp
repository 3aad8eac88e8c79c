// Host-side setup for the FELIS input format: the parser, the Domain
// scalars, the static tables and the initial state that the reference builds
// once before its step loop (main.cpp:44-90).  Everything here runs once on
// the CPU in FP64; the GPU library consumes its output through felis_params.
//
//   FindParameters      findparam.cpp:30-116
//   parameterSetting    parameterSetting.cpp:42-627
//   boundary            boundary.cpp:20-124 (decomposition, ABC, Bessel table)
//   loadBeam3D          loadBeam.cpp:28-269
//   loadSeed3D          loadSeed.cpp:25-80
//   wakeFunction        wakeField.cpp:53-159
//   updateWakeField     wakeField.cpp:9-50 (+ makeDensity :161-223)
//
// Third-party pieces the reference takes from GSL 2.8 are written here from
// their published definitions (their bit patterns are not pinned against
// GSL, which is absent): gsl_sf_bessel_Jn (power series for x < 1, Miller's
// backward recurrence normalised by J0 + 2 sum J_2k = 1 otherwise),
// gsl_qrng_halton (radical inverse in bases 2, 3, 5, 7, 11, 13, 17, first
// point at index 1), gsl_rng_default = MT19937 (std::mt19937, seed 0 mapped
// to 4357 as GSL does), gsl_rng_uniform (32-bit output / 2^32) and
// gsl_ran_gaussian (Marsaglia's polar method).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <complex>
#include <random>
#include <string>
#include <vector>

#include "../../../include/felis_b200.h"
#include "../lib/load.cuh"
#include "../lib/wake.cuh"

namespace {

const double kMu0 = 1.2566370614e-6;
const double kVelocityC = 299792458.0;
const double kEMass = 9.10938291e-31;
const double kECharge = 1.60217662e-19;
const double kMc2 = 0.510998918;
const double kZ0 = 376.730313668;
const double kPlankH = 4.135667696E-15;

thread_local std::string g_err;

// ---- findparam.cpp:30-116 -------------------------------------------------
// Reads `key` from the rank-th [block] of the file; the value runs from the
// first non-space after '=' to the next space (a trailing newline stays, as
// in the reference, and is ignored by atoi/atof).
bool find_param(const std::string& text, const char* block, int rank, const char* key, std::string* out) {
  size_t pos = 0;
  int count = 0;
  bool in_block = false;
  while (pos <= text.size()) {
    size_t eol = text.find('\n', pos);
    std::string line = text.substr(pos, eol == std::string::npos ? std::string::npos : eol - pos + 1);
    pos = (eol == std::string::npos) ? text.size() + 1 : eol + 1;
    size_t c = line.find("//");
    if (c != std::string::npos) line.resize(c);
    if (!in_block) {
      size_t p = 0;
      while (p < line.size() && line[p] == ' ') ++p;
      if (p < line.size() && line[p] == '[') {
        size_t q = line.find(']', p);
        if (q == std::string::npos) continue;
        ++p;
        while (p < line.size() && line[p] == ' ') ++p;
        const size_t bl = strlen(block);
        if (line.compare(p, bl, block) == 0) {
          size_t r = p + bl;
          while (r < line.size() && line[r] == ' ') ++r;
          if (r < line.size() && line[r] == ']') {
            ++count;
            if (count == rank) in_block = true;
          }
        }
      }
      continue;
    }
    if (line.find('[') != std::string::npos) return false;
    size_t p = 0;
    while (p < line.size() && line[p] == ' ') ++p;
    const size_t kl = strlen(key);
    if (line.compare(p, kl, key) != 0) continue;
    size_t r = p + kl;
    if (r >= line.size() || (line[r] != ' ' && line[r] != '=')) continue;
    while (r < line.size() && line[r] != '=') ++r;
    if (r >= line.size()) continue;
    ++r;
    while (r < line.size() && line[r] == ' ') ++r;
    size_t e = r;
    while (e < line.size() && line[e] != ' ') ++e;
    *out = line.substr(r, e - r);
    return true;
  }
  return false;
}

bool on_off(const std::string& s) { return s.find("ON") != std::string::npos; }

// ---- Bessel J_n (replaces gsl_sf_bessel_Jn, boundary.cpp:121) --------------
double bessel_jn(int n, double x) {
  if (x == 0.0) return n == 0 ? 1.0 : 0.0;
  const double ax = fabs(x);
  double r;
  if (ax < 1.0) {
    // J_n(x) = sum_k (-1)^k (x/2)^(2k+n) / (k! (k+n)!)
    const double h = 0.5 * ax;
    double term = 1.0;
    for (int k = 1; k <= n; ++k) term *= h / k;
    double sum = term;
    const double h2 = h * h;
    for (int k = 1; k < 60; ++k) {
      term *= -h2 / ((double)k * (double)(k + n));
      sum += term;
      if (fabs(term) < 1e-18 * fabs(sum)) break;
    }
    r = sum;
  } else {
    // Miller: J_{k-1} = (2k/x) J_k - J_{k+1} from k = M down, normalised.
    int M = 2 * ((int)(ax + 40.0 + n) / 2);
    double jp1 = 0.0, j = 1e-300, norm = 0.0, want = 0.0;
    for (int k = M; k > 0; --k) {
      const double jm1 = (2.0 * k / ax) * j - jp1;
      jp1 = j;
      j = jm1;  // now J_{k-1}
      if (k - 1 == n) want = j;
      if ((k - 1) % 2 == 0 && k - 1 > 0) norm += 2.0 * j;
      if (fabs(j) > 1e250) {  // rescale to avoid overflow
        j *= 1e-250; jp1 *= 1e-250; norm *= 1e-250; want *= 1e-250;
      }
    }
    norm += j;  // J_0
    r = want / norm;
  }
  if (x < 0.0 && (n & 1)) r = -r;
  return r;
}

// ---- GSL-equivalent generators (loadBeam.cpp:65-91, 182, 227-228) ---------
struct Halton7 {
  unsigned long count = 0;
  void next(double v[7]) {
    static const int primes[7] = {2, 3, 5, 7, 11, 13, 17};
    ++count;
    for (int d = 0; d < 7; ++d) {
      const int p = primes[d];
      double f = 1.0 / p, x = 0.0;
      unsigned long c = count;
      while (c > 0) {
        x += f * (double)(c % p);
        c /= p;
        f /= p;
      }
      v[d] = x;
    }
  }
};

// Three-dimensional Sobol points in Gray-code order (Antonov & Saleev 1979;
// direction numbers of Bratley & Fox 1988, ACM TOMS 14:88): dimension 1 the
// van der Corput sequence, dimension 2 the primitive polynomial x + 1 with
// m1 = 1, dimension 3 x^2 + x + 1 with m1 = 1, m2 = 3; 30-bit integers, so
// point n is its numerator times 2^-30.  The first point is (1/2, 1/2, 1/2).
struct Sobol3 {
  static constexpr int kBits = 30;
  uint32_t v[kBits + 1][3] = {};
  uint32_t x[3] = {0, 0, 0};
  unsigned long count = 0;
  Sobol3() {
    uint32_t m[kBits + 1][3] = {};
    for (int k = 1; k <= kBits; ++k) {
      m[k][0] = 1;
      m[k][1] = k == 1 ? 1 : (2 * m[k - 1][1]) ^ m[k - 1][1];
      m[k][2] = k == 1 ? 1 : (k == 2 ? 3 : (2 * m[k - 1][2]) ^ (4 * m[k - 2][2]) ^ m[k - 2][2]);
      for (int d = 0; d < 3; ++d) v[k][d] = m[k][d] << (kBits - k);
    }
  }
  void next(double out[3]) {
    int c = 1;  // 1-based position of the rightmost zero bit of count
    for (unsigned long n = count; n & 1ul; n >>= 1) ++c;
    for (int d = 0; d < 3; ++d) {
      x[d] ^= v[c][d];
      out[d] = (double)x[d] / (double)(1ul << kBits);
    }
    ++count;
  }
};

struct GslRng {
  std::mt19937 mt;
  explicit GslRng(unsigned long seed) : mt((uint32_t)(seed == 0 ? 4357 : seed)) {}
  double uniform() { return (double)mt() / 4294967296.0; }
  double uniform_pos() {
    double x;
    do { x = uniform(); } while (x == 0.0);
    return x;
  }
  double gaussian(double sigma) {
    double x, y, r2;
    do {
      x = -1 + 2 * uniform_pos();
      y = -1 + 2 * uniform_pos();
      r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0);
    return sigma * y * sqrt(-2.0 * log(r2) / r2);
  }
};

struct Beam {
  int type = 0;  // 1 Polygon, 2 Gaussian
  int numInBeamlet = 0, numBeamlet = 0;
  bool noise = false, transFlat = false;
  double energy = 0, spread = 0, gamma0 = 0, peakCurrent = 0;
  double emitX = 0, emitY = 0, alphaX = 0, alphaY = 0, betaX = 0, betaY = 0;
  std::vector<double> zpoint, zn, Epoint, En, ESpoint, ESn, EmitPoint, EmitN;
  double sigZ = 0, posZ = 0, Echirp = 0;
  int gaussPower = 2;
};

struct UndBlock {
  felis_undulator u{};
  std::vector<double> unitStart, unitEnd, undStart, undEnd, K0;
};
struct QuadBlock {
  felis_quad q{};
  std::vector<double> unitStart, unitEnd, qdStart, qdEnd, g;
};

}  // namespace

struct felis_config {
  felis_params p{};
  std::string path;
  int num_ranks = 1, rank = 0;
  int maxI = 0;
  std::vector<double> abc[4];
  std::vector<double> bessel, wake_e, wakeF;
  std::vector<UndBlock> und;
  std::vector<QuadBlock> quad;
  std::vector<felis_undulator> und_c;
  std::vector<felis_quad> quad_c;
  std::vector<Beam> beams;
  // [Seed]
  double P0 = 0, duration = 0, spotSigR = 0, focus = 0, a0 = 0, zR = 0, laserAlpha = -1, laserPsi = 0;
  double polarity = 0.0;  // D->polarity is never assigned by parameterSetting (stays 0)
  int loadH = 1;
  // [Wake_field]
  int wakeShape = 1, acdc = 1, wakeFieldStep = 0;
  double radius = 0, cond = 0, ctau = 0;
  // [Save]
  double Lz = 0;
  int saveStep = 0, saveStart = 0;
  bool fieldSave = true, particleSave = true;
  // [Phase_shifter] blocks (README.md:57-70; not read by the reference's
  // parser): every shifter's position [m] and phase [pi]
  std::vector<double> ps_z, ps_phase;
};

extern "C" const char* felis_config_error(void) { return g_err.c_str(); }

namespace {

#define NEED(block, rank, key, conv, dst)                                        \
  do {                                                                          \
    std::string v_;                                                             \
    if (find_param(text, block, rank, key, &v_)) dst = conv(v_.c_str());        \
    else { g_err = std::string("in [") + block + "], " + key + " is missing"; return FELIS_NOT_FOUND; } \
  } while (0)
#define OPT(block, rank, key, conv, dst, def)                                   \
  do {                                                                          \
    std::string v_;                                                             \
    if (find_param(text, block, rank, key, &v_)) dst = conv(v_.c_str());        \
    else dst = def;                                                             \
  } while (0)

int to_int(const char* s) { return atoi(s); }
double to_dbl(const char* s) { return atof(s); }
int to_mode(const char* s) {
  if (strstr(s, "Static")) return FELIS_STATIC;
  if (strstr(s, "Time_Dependent")) return FELIS_TIME_DEPENDENT;
  return 0;
}
int to_und(const char* s) {
  if (strstr(s, "BiPolar")) return FELIS_BIPOLAR;
  if (strstr(s, "QuadPolar")) return FELIS_QUADPOLAR;
  return 0;
}
int to_beam(const char* s) {
  if (strstr(s, "Polygon")) return 1;
  if (strstr(s, "Gaussian")) return 2;
  return 0;
}
bool to_onoff(const char* s) { return strstr(s, "ON") != nullptr; }

// parameterSetting.cpp:431-569
felis_status read_beam(const std::string& text, int rank, Beam& LL, bool* found) {
  std::string v;
  *found = false;
  if (!find_param(text, "EBeam", rank, "load_type", &v)) return FELIS_OK;
  LL.type = to_beam(v.c_str());
  if (LL.type == 0) return FELIS_OK;
  *found = true;
  NEED("EBeam", 1, "beam_energy", to_dbl, LL.energy);
  NEED("EBeam", 1, "energy_spread", to_dbl, LL.spread);
  LL.spread *= 0.01;
  NEED("EBeam", 1, "peak_current", to_dbl, LL.peakCurrent);
  NEED("EBeam", 1, "beta_x", to_dbl, LL.betaX);
  NEED("EBeam", 1, "beta_y", to_dbl, LL.betaY);
  NEED("EBeam", 1, "alpha_x", to_dbl, LL.alphaX);
  NEED("EBeam", 1, "alpha_y", to_dbl, LL.alphaY);
  OPT("EBeam", rank, "transverse_flat", to_onoff, LL.transFlat, false);
  NEED("EBeam", 1, "norm_emittance_x", to_dbl, LL.emitX);
  LL.emitX *= 1e-6;
  NEED("EBeam", 1, "norm_emittance_y", to_dbl, LL.emitY);
  LL.emitY *= 1e-6;
  NEED("EBeam", 1, "noise_ONOFF", to_onoff, LL.noise);
  NEED("EBeam", 1, "beamlets_in_bucket", to_int, LL.numBeamlet);
  NEED("EBeam", 1, "number_in_beamlet", to_int, LL.numInBeamlet);
  char name[64];
  auto nodes = [&](const char* cnt_key, const char* zfmt, const char* nfmt, std::vector<double>& zp,
                   std::vector<double>& zn) -> felis_status {
    int n = 0;
    NEED("EBeam", rank, cnt_key, to_int, n);
    zp.assign(n > 0 ? n : 0, 0.0);
    zn.assign(n > 0 ? n : 0, 0.0);
    for (int i = 0; i < n; ++i) {
      snprintf(name, sizeof name, zfmt, i);
      NEED("EBeam", rank, name, to_dbl, zp[i]);
      snprintf(name, sizeof name, nfmt, i);
      NEED("EBeam", rank, name, to_dbl, zn[i]);
    }
    return FELIS_OK;
  };
  if (LL.type == 1) {
    felis_status st;
    if ((st = nodes("z_nodes", "z%d", "z_n%d", LL.zpoint, LL.zn)) != FELIS_OK) return st;
    if ((st = nodes("energy_nodes", "energy_z%d", "energy_n%d", LL.Epoint, LL.En)) != FELIS_OK) return st;
    if ((st = nodes("energySpread_nodes", "energySpread_z%d", "energySpread_n%d", LL.ESpoint, LL.ESn)) != FELIS_OK) return st;
    if ((st = nodes("emit_nodes", "emit_z%d", "emit_n%d", LL.EmitPoint, LL.EmitN)) != FELIS_OK) return st;
  } else {
    NEED("EBeam", rank, "sigma_z", to_dbl, LL.sigZ);
    OPT("EBeam", rank, "gaussian_power", to_dbl, LL.gaussPower, 2);
    NEED("EBeam", rank, "position_z", to_dbl, LL.posZ);
    NEED("EBeam", rank, "energy_chirp", to_dbl, LL.Echirp);
  }
  LL.gamma0 = LL.energy / kMc2 + 1.0;
  return FELIS_OK;
}

// parameterSetting.cpp:345-429
felis_status read_und(const std::string& text, int rank, double gamma0, double ks, UndBlock& UB, bool* found) {
  felis_undulator& UL = UB.u;
  int quadTaperId = 30000;
  double linTaper = 0, quadTaper = 0;
  *found = false;
  OPT("Undulator", rank, "undulator_type", to_und, UL.type, 0);
  OPT("Undulator", rank, "numbers", to_int, UL.numbers, 0);
  OPT("Undulator", rank, "in_air", to_onoff, UL.air, false);
  if (UL.type == 0) return FELIS_OK;
  *found = true;
  NEED("Undulator", rank, "lambdaU", to_dbl, UL.lambdaU);
  UL.lambdaU *= 0.01;
  UL.K0_alpha = 1;
  if (UL.numbers > 0) {
    const int n = UL.numbers;
    UB.unitStart.assign(n, 0.0); UB.unitEnd.assign(n, 0.0);
    UB.undStart.assign(n, 0.0); UB.undEnd.assign(n, 0.0); UB.K0.assign(n, 0.0);
    NEED("Undulator", rank, "unit_start", to_dbl, UB.unitStart[0]);
    NEED("Undulator", rank, "unit_end", to_dbl, UB.unitEnd[0]);
    NEED("Undulator", rank, "undulator_start", to_dbl, UB.undStart[0]);
    NEED("Undulator", rank, "undulator_end", to_dbl, UB.undEnd[0]);
    OPT("Undulator", rank, "linear_taper", to_dbl, linTaper, 0.0);
    linTaper /= sqrt(2.0);
    OPT("Undulator", rank, "quad_taper", to_dbl, quadTaper, 0.0);
    quadTaper /= sqrt(2.0);
    OPT("Undulator", rank, "slope_K", to_dbl, UL.slopeK, 0.0);
    UL.slopeK /= sqrt(2.0);
    OPT("Undulator", rank, "quad_taper_start_index", to_int, quadTaperId, 30000);
    NEED("Undulator", rank, "polarity", to_dbl, UL.ue);
    OPT("Undulator", rank, "K0_alpha", to_int, UL.K0_alpha, 1);
    const double ku = 2 * M_PI / UL.lambdaU;
    std::string v;
    if (find_param(text, "Undulator", rank, "K0", &v)) UB.K0[0] = atof(v.c_str());
    else UB.K0[0] = sqrt((4 * gamma0 * gamma0 * ku / ks - 2) / (1.0 + UL.ue * UL.ue));
    const double K0 = UB.K0[0];
    const double unitLength = UB.unitEnd[0] - UB.unitStart[0];
    const double undStart = UB.undStart[0] - UB.unitStart[0];
    const double undLength = UB.undEnd[0] - UB.undStart[0];
    for (int i = 1; i < n; ++i) {
      UB.unitStart[i] = UB.unitEnd[i - 1];
      UB.unitEnd[i] = UB.unitStart[i] + unitLength;
      UB.undStart[i] = UB.unitStart[i] + undStart;
      UB.undEnd[i] = UB.undStart[i] + undLength;
      if (i >= quadTaperId)
        UB.K0[i] = K0 + i * linTaper + (i - quadTaperId) * (i - quadTaperId) * quadTaper;
      else
        UB.K0[i] = K0 + i * linTaper;
    }
    // Optional explicit per-unit K list (K0_list = k0,k1,...): an extension
    // for taper studies; absent in reference inputs.
    if (find_param(text, "Undulator", rank, "K0_list", &v)) {
      const char* s = v.c_str();
      for (int i = 0; i < n && *s; ++i) {
        char* end;
        UB.K0[i] = strtod(s, &end);
        if (end == s) break;
        s = (*end == ',') ? end + 1 : end;
      }
    }
  }
  return FELIS_OK;
}

// parameterSetting.cpp:287-338
felis_status read_quad(const std::string& text, int rank, QuadBlock& QB) {
  felis_quad& QD = QB.q;
  OPT("Quad", rank, "numbers", to_int, QD.numbers, 0);
  if (QD.numbers > 0) {
    const int n = QD.numbers;
    QB.unitStart.assign(n, 0.0); QB.unitEnd.assign(n, 0.0);
    QB.qdStart.assign(n, 0.0); QB.qdEnd.assign(n, 0.0); QB.g.assign(n, 0.0);
    NEED("Quad", rank, "unit_start", to_dbl, QB.unitStart[0]);
    NEED("Quad", rank, "unit_end", to_dbl, QB.unitEnd[0]);
    NEED("Quad", rank, "quad_start", to_dbl, QB.qdStart[0]);
    NEED("Quad", rank, "quad_end", to_dbl, QB.qdEnd[0]);
    NEED("Quad", rank, "g", to_dbl, QB.g[0]);
    const double unitLength = QB.unitEnd[0] - QB.unitStart[0];
    const double qdStart = QB.qdStart[0] - QB.unitStart[0];
    const double qdLength = QB.qdEnd[0] - QB.qdStart[0];
    const double g = QB.g[0];
    for (int i = 1; i < n; ++i) {
      QB.unitStart[i] = QB.unitEnd[i - 1];
      QB.unitEnd[i] = QB.unitStart[i] + unitLength;
      QB.qdStart[i] = QB.unitStart[i] + qdStart;
      QB.qdEnd[i] = QB.qdStart[i] + qdLength;
      QB.g[i] = g;
    }
  }
  return FELIS_OK;
}

typedef std::complex<double> cplx;
// Complex division in the expansion the reference's -ffast-math build selects
// (limited range, reciprocal); the GPU library and the CPU restatement use it too.
inline cplx cdiv_fast(cplx a, cplx b) {
  const double inv = 1.0 / (b.real() * b.real() + b.imag() * b.imag());
  return cplx((a.real() * b.real() + a.imag() * b.imag()) * inv, (a.imag() * b.real() - a.real() * b.imag()) * inv);
}
inline cplx cmul_plain(cplx a, cplx b) {
  return cplx(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

// boundary.cpp:73-106
void build_abc(felis_config* c) {
  felis_params& p = c->p;
  const int nx = p.nx, ny = p.ny, Lx = p.abc_n, Ly = p.abc_n;
  const double sig0 = p.abc_sig, dx = p.dx, dy = p.dy, dz = p.dz, ks = p.ks;
  std::vector<double> sigX(nx, 0.0), sigY(ny, 0.0);
  for (int i = 0; i < Lx; ++i) sigX[i] = sig0 * (Lx - i) * (Lx - i) / (1.0 * Lx * Lx);
  for (int i = nx - Lx; i < nx; ++i) sigX[i] = sig0 * (i - nx + Lx) * (i - nx + Lx) / (1.0 * Lx * Lx);
  for (int j = 0; j < Ly; ++j) sigY[j] = sig0 * (Ly - j) * (Ly - j) / (1.0 * Ly * Ly);
  for (int j = ny - Ly; j < ny; ++j) sigY[j] = sig0 * (j - ny + Ly) * (j - ny + Ly) / (1.0 * Ly * Ly);
  std::vector<cplx> sX(nx), sY(ny), al(nx, 0.0), alP(nx, 0.0), be(ny, 0.0), beP(ny, 0.0);
  for (int i = 0; i < nx; ++i) sX[i] = cplx(1.0 + 0.0 * sigX[i], sigX[i]);
  for (int j = 0; j < ny; ++j) sY[j] = cplx(1.0 + 0.0 * sigY[j], sigY[j]);
  const cplx mIdz(-0.0 * dz, -1.0 * dz);
  auto scl = [](cplx a, double s) { return cplx(a.real() * s, a.imag() * s); };
  auto add = [](cplx a, cplx b) { return cplx(a.real() + b.real(), a.imag() + b.imag()); };
  for (int i = 1; i < nx - 1; ++i) {
    const double k2 = 2.0 * ks * dx * dx;
    al[i] = cdiv_fast(mIdz, cmul_plain(scl(sX[i], k2), add(sX[i], sX[i - 1])));
    alP[i] = cdiv_fast(mIdz, cmul_plain(scl(sX[i], k2), add(sX[i], sX[i + 1])));
  }
  for (int j = 1; j < ny - 1; ++j) {
    const double k2 = 2.0 * ks * dy * dy;
    be[j] = cdiv_fast(mIdz, cmul_plain(scl(sY[j], k2), add(sY[j], sY[j - 1])));
    beP[j] = cdiv_fast(mIdz, cmul_plain(scl(sY[j], k2), add(sY[j], sY[j + 1])));
  }
  auto store = [](std::vector<double>& dst, const std::vector<cplx>& src) {
    dst.resize(2 * src.size());
    for (size_t k = 0; k < src.size(); ++k) { dst[2 * k] = src[k].real(); dst[2 * k + 1] = src[k].imag(); }
  };
  store(c->abc[0], al); store(c->abc[1], alP); store(c->abc[2], be); store(c->abc[3], beP);
  p.abc_alpha = c->abc[0].data(); p.abc_alpha_p = c->abc[1].data();
  p.abc_beta = c->abc[2].data(); p.abc_beta_p = c->abc[3].data();
}

// wakeField.cpp:53-159
void wake_function(felis_config* c) {
  const felis_params& p = c->p;
  const int sliceN = p.global_slice_n;
  const double dZ = p.num_slice * p.lambda0;
  const double radius = c->radius, cond = c->cond, ctau = c->ctau;
  const double s0 = pow(2.0 * radius * radius / kZ0 / cond, 1.0 / 3.0);
  const double maxK = 20, maxX = 2000, minK = 0.0, minX = 0.0;
  const int numK = 1000, numX = 50000;
  const double dK = maxK / (numK * 1.0), dX = maxX / (numX * 1.0);
  std::vector<double> impZ(numK + 1, 0.0);
  const cplx I(0.0, 1.0);
  if (c->wakeShape == 1) {
    for (int i = 1; i <= numK; ++i) {
      const double k = minK + i * dK;
      cplx csum = 0.0;
      for (int j = 0; j <= numX; ++j) {
        const double x = minX + j * dX;
        cplx ccal;
        if (x == 0.0) ccal = sqrt(k) / (2.0 + k * k * k - 2.0 * sqrt(k) * k);
        else if (x > 320) ccal = 0.0;
        else {
          const cplx cdino = 2.0 / (1.0 - I) / std::sqrt(k - I * k * k * ctau / s0) * cosh(x) - I * k * sinh(x) / x;
          ccal = 1.0 / cosh(x) / cdino;
        }
        csum += ccal * dX;
      }
      impZ[i] = csum.real();
    }
  } else if (c->wakeShape == 2) {
    for (int i = 1; i <= numK; ++i) {
      const double k = minK + i * dK;
      if (c->acdc == 1) {
        const cplx cdino = sqrt(2.0 * s0 / ctau) / k * (I + s0 * 0.5 / k / ctau) - I * 0.5 * k;
        impZ[i] = (1.0 / cdino).real();
      } else {
        const double dino = 2.0 / k + 0.25 * k * k - sqrt(k);
        impZ[i] = 1.0 / sqrt(k) / dino;
      }
    }
  }
  const double coef = kZ0 * 3e8 / M_PI / radius / radius / M_PI;
  c->wakeF.assign(sliceN, 0.0);
  for (int i = 0; i < sliceN; ++i) {
    const double z = (i * dZ) / s0;
    double sum = 0.0;
    for (double j = 0; j <= numK; ++j) {
      const double k = minK + j * dK;
      sum += impZ[(int)j] * cos(k * z) * dK;
    }
    c->wakeF[i] += sum * coef;
  }
}

felis_status load_config(felis_config* c) {
  FILE* f = fopen(c->path.c_str(), "rb");
  if (!f) { g_err = "cannot open " + c->path; return FELIS_IO; }
  std::string text;
  char buf[65536];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  fclose(f);
  felis_params& p = c->p;
  p.abi_version = FELIS_ABI_VERSION;
  p.precision = FELIS_FP64;
  double photon_energy = 0;
  std::string v;
  NEED("Domain", 1, "dimension", to_int, p.dimension);
  NEED("Domain", 1, "mode", to_mode, p.mode);
  NEED("Domain", 1, "photon_energy", to_dbl, photon_energy);
  p.ks = photon_energy * 2 * M_PI / (kPlankH * kVelocityC);
  p.lambda0 = 2 * M_PI / p.ks;
  NEED("Save", 1, "total_length", to_dbl, c->Lz);
  NEED("Save", 1, "save_step", to_int, c->saveStep);
  NEED("Save", 1, "save_start", to_int, c->saveStart);
  OPT("Save", 1, "field_save", to_onoff, c->fieldSave, true);
  OPT("Save", 1, "particle_save", to_onoff, c->particleSave, true);
  NEED("Domain", 1, "minX", to_dbl, p.min_x); p.min_x *= 1e-6;
  NEED("Domain", 1, "maxX", to_dbl, p.max_x); p.max_x *= 1e-6;
  NEED("Domain", 1, "minY", to_dbl, p.min_y); p.min_y *= 1e-6;
  NEED("Domain", 1, "maxY", to_dbl, p.max_y); p.max_y *= 1e-6;
  NEED("Domain", 1, "minZ", to_dbl, p.min_z); p.min_z *= 1e-6;
  NEED("Domain", 1, "maxZ", to_dbl, p.max_z); p.max_z *= 1e-6;
  NEED("Domain", 1, "nx", to_int, p.nx);
  NEED("Domain", 1, "ny", to_int, p.ny);
  p.dx = (p.max_x - p.min_x) / (p.nx * 1.0);
  p.dy = (p.max_y - p.min_y) / (p.ny * 1.0);
  p.nx += 1;
  p.ny += 1;
  if (p.dimension == 1) { p.nx = 1; p.ny = 1; p.dx = 0.0; p.dy = 0.0; }
  OPT("Domain", 1, "ABC_N", to_int, p.abc_n, 10);
  OPT("Domain", 1, "ABC_coef", to_dbl, p.abc_sig, 1);
  OPT("Domain", 1, "num_harmony", to_int, p.num_harmony, 1);
  if (p.num_harmony < 1 || p.num_harmony > FELIS_MAX_HARMONY) { g_err = "num_harmony out of range"; return FELIS_UNSUPPORTED; }
  for (int i = 0; i < p.num_harmony; ++i) {
    char key[32];
    snprintf(key, sizeof key, "harmony%d", i);
    NEED("Domain", 1, key, to_int, p.harmony[i]);
  }
  OPT("Domain", 1, "lambdaUs_in_iteration", to_int, p.num_lambda_u, 1);
  NEED("Domain", 1, "slices_in_bucket", to_int, p.num_slice);
  if (p.num_slice < p.num_lambda_u) { g_err = "slices_in_bucket < lambdaUs_in_iteration"; return FELIS_BAD_ARG; }
  for (int rank = 1;; ++rank) {
    Beam LL;
    bool found;
    felis_status st = read_beam(text, rank, LL, &found);
    if (st != FELIS_OK) return st;
    if (!found) break;
    c->beams.push_back(LL);
  }
  p.num_species = (int)c->beams.size();
  if (p.num_species < 1 || p.num_species > FELIS_MAX_SPECIES) { g_err = "no [EBeam] block"; return FELIS_NOT_FOUND; }
  p.gamma0 = c->beams[0].gamma0;
  // 1D model: each species' matched spot area (solveField.cpp:455-462)
  for (int s = 0; s < p.num_species; ++s) {
    const Beam& LL = c->beams[s];
    const double emitX = LL.emitX / p.gamma0, emitY = LL.emitY / p.gamma0;
    const double gammaX = (1 + LL.alphaX * LL.alphaX) / LL.betaX;
    const double gammaY = (1 + LL.alphaY * LL.alphaY) / LL.betaY;
    const double sigX = sqrt(emitX / gammaX), sigY = sqrt(emitY / gammaY);
    p.beam_area[s] = 2.0 * M_PI * sigX * sigY;
  }
  for (int rank = 1;; ++rank) {
    UndBlock UB;
    bool found;
    felis_status st = read_und(text, rank, p.gamma0, p.ks, UB, &found);
    if (st != FELIS_OK) return st;
    if (!found) break;
    c->und.push_back(UB);
  }
  if (c->und.empty() || c->und[0].K0.empty()) { g_err = "no [Undulator] block with units"; return FELIS_NOT_FOUND; }
  {
    const UndBlock& U0 = c->und[0];
    p.K0_init = U0.K0[0];
    p.ue_init = U0.u.ue;
    p.K0_alpha_init = U0.u.K0_alpha;
    p.und_type_init = U0.u.type;
    p.lambdaU_init = U0.u.lambdaU;
    const double ku = 2.0 * M_PI / U0.u.lambdaU;
    p.gam_r = sqrt(0.5 * p.ks / ku * (1 + 0.5 * (1 + p.ue_init * p.ue_init) * p.K0_init * p.K0_init));
  }
  for (int rank = 1;; ++rank) {
    QuadBlock QB;
    felis_status st = read_quad(text, rank, QB);
    if (st != FELIS_OK) return st;
    if (QB.q.numbers <= 0) break;
    c->quad.push_back(QB);
  }
  OPT("Domain", 1, "number_azimuthal_mode", to_int, p.scf_mode, 1);
  OPT("Domain", 1, "number_longitudinal_mode", to_int, p.scl_mode, 1);
  if (find_param(text, "Domain", 1, "radial_grids", &v)) p.nr = atoi(v.c_str());
  else p.nr = (int)sqrt(p.nx * p.nx + p.ny * p.ny);
  p.dr = sqrt((p.max_x - p.min_x) * (p.max_x - p.min_x) + (p.max_y - p.min_y) * (p.max_y - p.min_y)) / (1.0 * p.nx);
  if (p.dimension == 1) { p.nr = 1; p.dr = 0.0; p.scf_mode = 1; }
  OPT("Bessel_table", 1, "num_grids", to_int, p.bessel_rows, 2001);
  NEED("Seed", 1, "power", to_dbl, c->P0);
  NEED("Seed", 1, "spot_sigma_R", to_dbl, c->spotSigR); c->spotSigR *= 1e-6;
  NEED("Seed", 1, "rms_duration", to_dbl, c->duration); c->duration *= 1e-15;
  NEED("Seed", 1, "focus", to_dbl, c->focus);
  OPT("Seed", 1, "loading_harmonics", to_int, c->loadH, 1);
  double seed_ue = 0.0;
  OPT("Seed", 1, "polarity", to_dbl, seed_ue, 0.0);
  OPT("Seed", 1, "laser_alpha", to_dbl, c->laserAlpha, -1.0);
  p.spot_sig_r = c->spotSigR;
  const double area = 2.0 * M_PI * c->spotSigR * c->spotSigR;
  c->a0 = sqrt(c->P0 * 2.0 * kZ0 / area) * kECharge / (kEMass * kVelocityC * kVelocityC * p.ks * c->loadH);
  c->zR = 2.0 * c->spotSigR * c->spotSigR * p.ks * (1.0 * c->loadH);
  {
    const std::complex<double> U = (1.0 - seed_ue * seed_ue + std::complex<double>(0, 1) * 2.0 * seed_ue) / (1.0 + seed_ue * seed_ue);
    c->laserPsi = std::arg(U);
  }
  if (p.mode == FELIS_STATIC) { p.min_z = 0.0; p.max_z = p.lambda0 * p.num_slice; }
  p.dz = c->und[0].u.lambdaU * p.num_lambda_u;
  p.max_step = (int)(c->Lz / p.dz + 1);
  int sliceN = (int)((p.max_z - p.min_z) / (p.lambda0 * p.num_slice));
  if (sliceN > 50000 || sliceN < -50000) { g_err = "too many slices"; return FELIS_BAD_ARG; }
  if (p.mode == FELIS_STATIC) sliceN = 1;
  if (sliceN < 1) { g_err = "no slices"; return FELIS_BAD_ARG; }
  p.global_slice_n = sliceN;
  OPT("Wake_field", 1, "activate", to_onoff, p.wake_on, true);
  OPT("Wake_field", 1, "update_step", to_int, c->wakeFieldStep, p.max_step);
  {
    std::string s;
    c->wakeShape = 1;
    if (find_param(text, "Wake_field", 1, "shape", &s)) {
      if (strstr(s.c_str(), "Flat")) c->wakeShape = 1;
      else if (strstr(s.c_str(), "Circular")) c->wakeShape = 2;
      else c->wakeShape = 0;
    }
    c->acdc = 1;
    if (find_param(text, "Wake_field", 1, "ac_dc", &s)) {
      if (strstr(s.c_str(), "AC")) c->acdc = 1;
      else if (strstr(s.c_str(), "DC")) c->acdc = 2;
      else c->acdc = 0;
    }
  }
  NEED("Wake_field", 1, "radius", to_dbl, c->radius);
  OPT("Wake_field", 1, "conductivity", to_dbl, c->cond, 3.03e7);
  if (c->acdc == 1) { OPT("Wake_field", 1, "ctau", to_dbl, c->ctau, 2.4e-6); }
  else c->ctau = 0.0;
  // every [Phase_shifter] block: `number` shifters at start_position +
  // k interval_length, each delaying the electrons by `phase` pi
  for (int rank = 1;; ++rank) {
    int number = 0;
    double start = 0, interval = 0, phase = 0;
    OPT("Phase_shifter", rank, "number", to_int, number, 0);
    if (number <= 0) break;
    OPT("Phase_shifter", rank, "start_position", to_dbl, start, 0.0);
    OPT("Phase_shifter", rank, "interval_length", to_dbl, interval, 0.0);
    OPT("Phase_shifter", rank, "phase", to_dbl, phase, 0.0);
    for (int k = 0; k < number; ++k) {
      c->ps_z.push_back(start + k * interval);
      c->ps_phase.push_back(phase);
    }
  }

  // boundary.cpp:33-46: contiguous slice blocks per rank
  {
    const int nT = c->num_ranks, remain = sliceN % nT, base = sliceN / nT;
    int lo = 0;
    for (int r = 0; r < nT; ++r) {
      const int cnt = (r < remain) ? base + 1 : base;
      if (r == c->rank) { p.min_i = lo; c->maxI = lo + cnt; }
      lo += cnt;
    }
    p.slice_n = c->maxI - p.min_i;
  }
  if (p.dimension == 3) build_abc(c);
  // boundary.cpp:108-124
  {
    const int Hmax = p.harmony[p.num_harmony - 1];
    const double BesselMax = Hmax * 2.0 * M_PI;
    p.d_bessel = BesselMax / (double)p.bessel_rows;
    p.bessel_cols = (Hmax + 1) / 2 + 1;
    c->bessel.assign((size_t)p.bessel_rows * p.bessel_cols, 0.0);
    for (int i = 0; i < p.bessel_rows; ++i) {
      const double xi = p.d_bessel * i;
      for (int j = 0; j < p.bessel_cols; ++j) c->bessel[(size_t)i * p.bessel_cols + j] = bessel_jn(j, xi);
    }
    p.bessel = c->bessel.data();
  }
  c->wake_e.assign(sliceN, 0.0);
  p.wake_e = c->wake_e.data();
  for (auto& U : c->und) {
    U.u.unit_start = U.unitStart.data(); U.u.unit_end = U.unitEnd.data();
    U.u.und_start = U.undStart.data(); U.u.und_end = U.undEnd.data(); U.u.K0 = U.K0.data();
    c->und_c.push_back(U.u);
  }
  for (auto& Q : c->quad) {
    Q.q.unit_start = Q.unitStart.data(); Q.q.unit_end = Q.unitEnd.data();
    Q.q.qd_start = Q.qdStart.data(); Q.q.qd_end = Q.qdEnd.data(); Q.q.g = Q.g.data();
    c->quad_c.push_back(Q.q);
  }
  p.num_undulators = (int)c->und_c.size();
  p.num_quads = (int)c->quad_c.size();
  p.undulators = c->und_c.data();
  p.quads = c->quad_c.empty() ? nullptr : c->quad_c.data();
  p.num_phase_shifts = (int32_t)c->ps_z.size();
  p.phase_shift_z = c->ps_z.empty() ? nullptr : c->ps_z.data();
  p.phase_shift_phase = c->ps_phase.empty() ? nullptr : c->ps_phase.data();
  return FELIS_OK;
}

}  // namespace

extern "C" {

felis_status felis_config_load(const char* path, int32_t num_ranks, int32_t rank, felis_config** out) {
  if (!path || !out || num_ranks < 1 || rank < 0 || rank >= num_ranks) {
    g_err = "felis_config_load: bad argument";
    return FELIS_BAD_ARG;
  }
  felis_config* c = new felis_config();
  c->path = path;
  c->num_ranks = num_ranks;
  c->rank = rank;
  const felis_status st = load_config(c);
  if (st != FELIS_OK) {
    delete c;
    *out = nullptr;
    return st;
  }
  *out = c;
  return FELIS_OK;
}

void felis_config_free(felis_config* c) { delete c; }
const felis_params* felis_config_params(const felis_config* c) { return c ? &c->p : nullptr; }

}  // extern "C"

namespace {

// Per-slice quantities of loadBeam.cpp (current profile, energy, spread, the
// matched transverse sizes, beamlet count and macro weight) for slice sl;
// gamma0 carries over from the previous slice when the profile sets none, as
// in the reference's loop.
struct SliceLoad {
  double dGam, sigX, sigY, sigXPrime, sigYPrime, delTX, delTY, remacro, eNumbers, ESn0;
  int beamlets;
};

SliceLoad slice_load(const felis_params& p, const Beam& LL, int sl, double macro, double& gamma0) {
  SliceLoad L{};
  const double bucketZ = p.lambda0 * p.num_slice;
  double n0 = 0.0, En0 = 0.0, ESn0 = 0.0;
  const double posZ = (sl + p.min_i) * bucketZ + p.min_z;
  if (LL.type == 1) {
    for (size_t l = 0; l + 1 < LL.zpoint.size(); ++l)
      if (posZ >= LL.zpoint[l] && posZ < LL.zpoint[l + 1])
        n0 = (LL.zn[l + 1] - LL.zn[l]) / (LL.zpoint[l + 1] - LL.zpoint[l]) * (posZ - LL.zpoint[l]) + LL.zn[l];
    for (size_t l = 0; l + 1 < LL.Epoint.size(); ++l)
      if (posZ >= LL.Epoint[l] && posZ < LL.Epoint[l + 1])
        En0 = (LL.En[l + 1] - LL.En[l]) / (LL.Epoint[l + 1] - LL.Epoint[l]) * (posZ - LL.Epoint[l]) + LL.En[l];
    gamma0 = LL.energy * En0 / kMc2 + 1.0;
    for (size_t l = 0; l + 1 < LL.ESpoint.size(); ++l)
      if (posZ >= LL.ESpoint[l] && posZ < LL.ESpoint[l + 1])
        ESn0 = (LL.ESn[l + 1] - LL.ESn[l]) / (LL.ESpoint[l + 1] - LL.ESpoint[l]) * (posZ - LL.ESpoint[l]) + LL.ESn[l];
  } else if (LL.type == 2) {
    const double phase = pow((posZ - LL.posZ) / LL.sigZ, LL.gaussPower);
    n0 = exp(-phase);
    gamma0 = (LL.energy + LL.Echirp * (posZ - LL.posZ)) / kMc2 + 1.0;
  }
  L.ESn0 = ESn0;
  L.dGam = LL.spread * gamma0 * ESn0;
  const double emitX = LL.emitX / gamma0, emitY = LL.emitY / gamma0;
  const double gammaX = (1 + LL.alphaX * LL.alphaX) / LL.betaX;
  const double gammaY = (1 + LL.alphaY * LL.alphaY) / LL.betaY;
  L.sigX = sqrt(emitX / gammaX); L.sigY = sqrt(emitY / gammaY);
  L.sigXPrime = sqrt(emitX * gammaX); L.sigYPrime = sqrt(emitY * gammaY);
  const double distanceX = sqrt(fabs((LL.betaX - 1.0 / gammaX) / gammaX));
  const double distanceY = sqrt(fabs((LL.betaY - 1.0 / gammaY) / gammaY));
  const double vz = sqrt(gamma0 * gamma0 - 1.0) / gamma0;
  L.delTX = distanceX / vz; L.delTY = distanceY / vz;
  if (vz == 0.0) L.delTX = L.delTY = 0.0;
  L.beamlets = LL.numBeamlet * n0;
  L.remacro = (L.beamlets > 0) ? macro * (double)LL.numBeamlet / (double)L.beamlets * n0 : 0.0;
  L.eNumbers = L.remacro * LL.numInBeamlet;
  if (L.eNumbers < 10) L.eNumbers = 10;
  return L;
}

// loadBeam.cpp:271-446 (1D): the same per-slice setup; per beamlet a Sobol
// point (phase, energy by Box-Muller) and the noise amplitudes; no
// transverse coordinates.  Counts first (arrays NULL), then the particles.
felis_status load_beam_1d(felis_config* c, int species, uint64_t seed, int64_t* counts, double* xo, double* yo,
                          double* pxo, double* pyo, double* tho, double* gao, double* wo) {
  const felis_params& p = c->p;
  const Beam& LL = c->beams[species];
  const int maxH = p.harmony[p.num_harmony - 1];
  const int numInBeamlet = LL.numInBeamlet;
  double gamma0 = LL.energy / kMc2 + 1;
  const double bucketZ = p.lambda0 * p.num_slice;
  const int ptclCnt = numInBeamlet * LL.numBeamlet;
  const double dPhi = 2.0 * M_PI * p.num_slice;
  const double div = 2.0 * M_PI / (1.0 * numInBeamlet);
  const double noiseONOFF = LL.noise ? 1.0 : 0.0;
  const double macro = LL.peakCurrent / kECharge / kVelocityC * bucketZ / (double)ptclCnt;
  const bool fill = xo != nullptr;
  GslRng ran(seed);
  Sobol3 q1;
  double v1[3] = {0.0, 0.0, 0.0};
  for (int ii = 0; ii < c->rank; ++ii) q1.next(v1);  // randskip = myrank
  int64_t out_idx = 0;
  for (int sl = 0; sl < p.slice_n; ++sl) {
    const SliceLoad L = slice_load(p, LL, sl, macro, gamma0);
    const int64_t total = (int64_t)L.beamlets * numInBeamlet;
    if (!fill) {
      counts[sl] = total;
      continue;
    }
    if (counts[sl] != total) { g_err = "felis_config_load_beam: counts changed"; return FELIS_BAD_ARG; }
    wo[sl] = L.remacro;
    std::vector<double> an(maxH + 1, 0.0), bn(maxH + 1, 0.0);
    for (int b = 0; b < L.beamlets; ++b) {
      q1.next(v1);
      const double th = v1[0];
      double gam = (v1[1] == 0.0) ? 1e-10 : v1[1];
      const double tmp = sqrt(-2.0 * log(gam)) * cos(v1[2] * 2.0 * M_PI);
      gam = gamma0 + L.dGam * tmp;
      const double theta0 = th * dPhi;
      for (int m = 1; m <= maxH; ++m) {
        const double sigma = sqrt(2.0 / L.eNumbers / (1.0 * m * m));
        an[m] = ran.gaussian(sigma);
        bn[m] = ran.gaussian(sigma);
      }
      for (int n = 0; n < numInBeamlet; ++n) {
        const int64_t k = out_idx++;
        xo[k] = 0.0; yo[k] = 0.0; pxo[k] = 0.0; pyo[k] = 0.0; gao[k] = gam;
        const double theta = theta0 + n * div;
        double noise = 0.0;
        for (int m = 1; m <= maxH; ++m) noise += an[m] * cos(m * theta) + bn[m] * sin(m * theta);
        tho[k] = theta + noise * noiseONOFF;
      }
    }
  }
  return FELIS_OK;
}

}  // namespace

extern "C" {

// loadBeam.cpp:28-269 (3D).  Counts first (arrays NULL), then the particles.
felis_status felis_config_load_beam(felis_config* c, int32_t species, uint64_t seed, int64_t* counts, double* xo,
                                    double* yo, double* pxo, double* pyo, double* tho, double* gao, double* wo) {
  if (!c || species < 0 || species >= (int)c->beams.size() || !counts) {
    g_err = "felis_config_load_beam: bad argument";
    return FELIS_BAD_ARG;
  }
  const felis_params& p = c->p;
  if (p.dimension == 1) return load_beam_1d(c, species, seed, counts, xo, yo, pxo, pyo, tho, gao, wo);
  if (p.dimension != 3) { g_err = "dimension must be 1 or 3"; return FELIS_UNSUPPORTED; }
  const Beam& LL = c->beams[species];
  const int maxH = p.harmony[p.num_harmony - 1];
  const int numInBeamlet = LL.numInBeamlet;
  double gamma0 = LL.energy / kMc2 + 1;
  const double current = LL.peakCurrent;
  const double bucketZ = p.lambda0 * p.num_slice;
  const int ptclCnt = numInBeamlet * LL.numBeamlet;
  const double noiseONOFF = LL.noise ? 1.0 : 0.0;
  const double dPhi = 2.0 * M_PI * p.num_slice;
  const double div = 2.0 * M_PI / (1.0 * numInBeamlet);
  const double macro = current / kECharge / kVelocityC * bucketZ / (double)ptclCnt;
  const bool fill = xo != nullptr;
  GslRng ran(seed);
  Halton7 q1;
  double v1[7] = {0};
  for (int ii = 0; ii < c->rank; ++ii) q1.next(v1);  // randskip = myrank
  int64_t out_idx = 0;
  for (int sl = 0; sl < p.slice_n; ++sl) {
    const SliceLoad L = slice_load(p, LL, sl, macro, gamma0);
    const double dGam = L.dGam, sigX = L.sigX, sigY = L.sigY, sigXPrime = L.sigXPrime, sigYPrime = L.sigYPrime;
    const double delTX = L.delTX, delTY = L.delTY, remacro = L.remacro, eNumbers = L.eNumbers, ESn0 = L.ESn0;
    const int beamlets = L.beamlets;
    const int64_t total = (int64_t)beamlets * numInBeamlet;
    if (!fill) {
      counts[sl] = total;
      continue;
    }
    if (counts[sl] != total) { g_err = "felis_config_load_beam: counts changed"; return FELIS_BAD_ARG; }
    wo[sl] = remacro;
    std::vector<double> an(maxH + 1, 0.0), bn(maxH + 1, 0.0);
    for (int b = 0; b < beamlets; ++b) {
      q1.next(v1);
      const double theta0 = v1[4] * dPhi;
      double r1 = v1[0]; if (r1 == 0.0) r1 = 1e-10;
      const double r2 = v1[1];
      double pr1 = v1[2]; if (pr1 == 0.0) pr1 = 1e-10;
      const double pr2 = v1[3];
      double gam = v1[5]; if (gam == 0.0) gam = 1e-10;
      double x, y, xPrime, yPrime;
      if (!LL.transFlat) {
        double coef = sqrt(-2.0 * log(r1));
        x = coef * cos(2.0 * M_PI * r2) * sigX;
        y = coef * sin(2.0 * M_PI * r2) * sigY;
        coef = sqrt(-2.0 * log(pr1));
        xPrime = coef * cos(2.0 * M_PI * pr2) * sigXPrime;
        yPrime = coef * sin(2.0 * M_PI * pr2) * sigYPrime;
      } else {
        double coef = sqrt(r1);
        x = coef * cos(2.0 * M_PI * r2) * sigX;
        y = coef * sin(2.0 * M_PI * r2) * sigY;
        coef = sqrt(-2.0 * log(pr1));
        xPrime = coef * cos(2.0 * M_PI * pr2) * sigXPrime;
        yPrime = coef * sin(2.0 * M_PI * pr2) * sigYPrime;
      }
      const double tmp = sqrt(-2.0 * log(gam)) * cos(v1[6] * 2.0 * M_PI);
      gam = gamma0 + dGam * tmp * ESn0;
      const double pz = sqrt((gam * gam - 1.0) / (1.0 + xPrime * xPrime + yPrime * yPrime));
      const double px = xPrime * pz, py = yPrime * pz;
      x -= delTX * px / gam;
      y -= delTY * py / gam;
      for (int m = 1; m <= maxH; ++m) {
        const double sigma = sqrt(2.0 / eNumbers / (1.0 * m * m));
        an[m] = ran.gaussian(sigma);
        bn[m] = ran.gaussian(sigma);
      }
      for (int n = 0; n < numInBeamlet; ++n) {
        const int64_t k = out_idx++;
        xo[k] = x; yo[k] = y; pxo[k] = px; pyo[k] = py; gao[k] = gam;
        const double theta = theta0 + n * div;
        double noise = 0.0;
        for (int m = 1; m <= maxH; ++m) noise += an[m] * cos(m * theta) + bn[m] * sin(m * theta);
        tho[k] = theta + noise * noiseONOFF;
      }
    }
  }
  return FELIS_OK;
}

// felis_config_load_beam with the per-beamlet work on the device (k_load.cu):
// the host computes the per-slice setup and draws the noise amplitudes from
// the same random stream in the same order.
felis_status felis_config_load_beam_device(felis_config* c, int32_t species, uint64_t seed, int64_t* counts,
                                           double* xo, double* yo, double* pxo, double* pyo, double* tho,
                                           double* gao, double* wo) {
  if (!c || species < 0 || species >= (int)c->beams.size() || !counts) {
    g_err = "felis_config_load_beam_device: bad argument";
    return FELIS_BAD_ARG;
  }
  const felis_params& p = c->p;
  if (p.dimension != 3) { g_err = "the device loader is 3D only (felis_config_load_beam loads 1D beams)"; return FELIS_UNSUPPORTED; }
  const Beam& LL = c->beams[species];
  const int maxH = p.harmony[p.num_harmony - 1];
  const int numInBeamlet = LL.numInBeamlet;
  double gamma0 = LL.energy / kMc2 + 1;
  const double bucketZ = p.lambda0 * p.num_slice;
  const int ptclCnt = numInBeamlet * LL.numBeamlet;
  const double macro = LL.peakCurrent / kECharge / kVelocityC * bucketZ / (double)ptclCnt;
  const bool fill = xo != nullptr;
  if (fill && (!yo || !pxo || !pyo || !tho || !gao || !wo)) {
    g_err = "felis_config_load_beam_device: null array";
    return FELIS_BAD_ARG;
  }
  std::vector<felis::LoadSlice> ls(p.slice_n);
  std::vector<double> eN(p.slice_n);
  int64_t beamlets_total = 0;
  for (int sl = 0; sl < p.slice_n; ++sl) {
    const SliceLoad L = slice_load(p, LL, sl, macro, gamma0);
    const int64_t total = (int64_t)L.beamlets * numInBeamlet;
    if (!fill) {
      counts[sl] = total;
      continue;
    }
    if (counts[sl] != total) { g_err = "felis_config_load_beam_device: counts changed"; return FELIS_BAD_ARG; }
    wo[sl] = L.remacro;
    ls[sl] = felis::LoadSlice{gamma0, L.dGam, L.sigX, L.sigY, L.sigXPrime, L.sigYPrime, L.delTX, L.delTY, L.ESn0,
                              beamlets_total, L.beamlets, 0};
    eN[sl] = L.eNumbers;
    beamlets_total += L.beamlets;
  }
  if (!fill) return FELIS_OK;
  // the noise amplitudes in the host loader's draw order
  GslRng ran(seed);
  std::vector<double> noise((size_t)std::max<int64_t>(beamlets_total, 1) * 2 * maxH);
  size_t q = 0;
  for (int sl = 0; sl < p.slice_n; ++sl)
    for (int b = 0; b < ls[sl].beamlets; ++b)
      for (int m = 1; m <= maxH; ++m) {
        const double sigma = sqrt(2.0 / eN[sl] / (1.0 * m * m));
        noise[q++] = ran.gaussian(sigma);
        noise[q++] = ran.gaussian(sigma);
      }
  felis::LoadSlice* d_ls = nullptr;
  double* d_noise = nullptr;
  cudaError_t e = cudaMalloc(&d_ls, ls.size() * sizeof(felis::LoadSlice));
  if (e == cudaSuccess) e = cudaMalloc(&d_noise, noise.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d_ls, ls.data(), ls.size() * sizeof(felis::LoadSlice), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_noise, noise.data(), noise.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    felis::LoadArgs a{};
    a.slices = d_ls; a.noise = d_noise; a.S = p.slice_n; a.maxH = maxH; a.num_in_beamlet = numInBeamlet;
    a.trans_flat = LL.transFlat ? 1 : 0; a.noise_on = LL.noise ? 1.0 : 0.0;
    a.dPhi = 2.0 * M_PI * p.num_slice; a.div = 2.0 * M_PI / (1.0 * numInBeamlet);
    a.halton0 = (uint64_t)c->rank;  // randskip = myrank
    a.x = xo; a.y = yo; a.px = pxo; a.py = pyo; a.theta = tho; a.gamma = gao;
    e = felis::launch_load_beam(a, 0);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (d_ls) cudaFree(d_ls);
  if (d_noise) cudaFree(d_noise);
  if (e != cudaSuccess) {
    g_err = std::string("felis_config_load_beam_device: ") + cudaGetErrorString(e);
    return FELIS_CUDA_ERROR;
  }
  return FELIS_OK;
}

// loadSeed.cpp:25-80 — writes harmonic `hidx` (all (slice_n+2) planes;
// ghost planes and other harmonics are left to the caller, zero initially).
felis_status felis_config_load_seed(felis_config* c, int32_t hidx, double* ux, double* uy) {
  if (!c || !ux || !uy) return FELIS_BAD_ARG;
  const felis_params& p = c->p;
  if (p.dimension != 3 && p.dimension != 1) return FELIS_UNSUPPORTED;
  int h_pick = 0;
  for (int h = 0; h < p.num_harmony; ++h)
    if (p.harmony[h] == c->loadH) h_pick = h;
  const size_t N = (size_t)p.nx * p.ny, total = (size_t)(p.slice_n + 2) * N;
  for (size_t k = 0; k < 2 * total; ++k) { ux[k] = 0.0; uy[k] = 0.0; }
  if (hidx != h_pick) return FELIS_OK;
  if (p.dimension == 1) {
    // loadSeed.cpp:82-111: one amplitude per slice (z from minZ itself)
    const double bucketZ1 = p.lambda0 * p.num_slice, sigmaZ1 = c->duration * kVelocityC;
    const double invSigma21 = 1.0 / sigmaZ1 / sigmaZ1;
    const double factor = sqrt(1.0 + c->polarity * c->polarity) * 0.5;
    const std::complex<double> ph = std::exp(std::complex<double>(0.0, 1.0) * c->laserPsi);
    for (int sl = 0; sl < p.slice_n; ++sl) {
      const double z = (sl + p.min_i) * bucketZ1 + p.min_z;
      const double amp = factor * c->a0 * exp(-0.25 * z * z * invSigma21);
      const std::complex<double> vx = amp * (1.0 + c->laserAlpha * ph), vy = amp * (-1.0 + c->laserAlpha * ph);
      ux[2 * (sl + 1)] = vx.real(); ux[2 * (sl + 1) + 1] = vx.imag();
      uy[2 * (sl + 1)] = vy.real(); uy[2 * (sl + 1) + 1] = vy.imag();
    }
    return FELIS_OK;
  }
  const double a0 = c->a0, dx = p.dx, dy = p.dy;
  const int nx = p.nx, ny = p.ny;
  const double bucketZ = p.lambda0 * p.num_slice;
  const double sigmaZ = c->duration * kVelocityC;
  const double invSigma2 = 1.0 / sigmaZ / sigmaZ;
  const double minZ = p.min_z + p.lambda0 * 0.5;
  const double zR = c->zR, focus = c->focus, ks = p.ks;
  const double sigR = sqrt(2.0) * c->spotSigR;
  const double factor = sqrt(1.0 + c->polarity * c->polarity) * 0.5;
  const std::complex<double> I(0.0, 1.0);
  const std::complex<double> pol_x = 1.0 + c->laserAlpha * std::exp(I * c->laserPsi);
  const std::complex<double> pol_y = -1.0 + c->laserAlpha * std::exp(I * c->laserPsi);
  double curv = 1e100;
  for (int sl = 0; sl < p.slice_n; ++sl) {
    const int sliceI = sl + 1;
    const double z = (sl + p.min_i) * bucketZ + minZ;
    const double delZ = z - focus;
    const double ampZ = a0 * exp(-0.25 * z * z * invSigma2);
    if (delZ == 0.0) curv = 1e100;
    else curv = delZ * (1.0 + zR * zR / (delZ * delZ));
    const double gouy = atan(delZ / zR);
    const double w = sigR * sqrt(1.0 + delZ * delZ / (zR * zR));
    for (int idxI = 0; idxI < nx; ++idxI) {
      const double x = p.min_x + idxI * dx;
      for (int idxJ = 0; idxJ < ny; ++idxJ) {
        const double y = p.min_y + idxJ * dy;
        const double r2 = x * x + y * y;
        const double phase = -r2 / (2.0 * w * w);
        const std::complex<double> compPhase = I * (ks * delZ + ks * r2 / (2.0 * curv) - gouy);
        const std::complex<double> amp = factor * (ampZ * sigR / w) * std::exp(compPhase + phase);
        const std::complex<double> vx = amp * pol_x, vy = amp * pol_y;
        const size_t k = (size_t)sliceI * N + (size_t)idxJ * nx + idxI;
        ux[2 * k] = vx.real(); ux[2 * k + 1] = vx.imag();
        uy[2 * k] = vy.real(); uy[2 * k + 1] = vy.imag();
      }
    }
  }
  return FELIS_OK;
}

// wakeField.cpp:9-50 with makeDensity (:161-223); den[s] = sum over species of
// weight * count for global slice s (length global_slice_n).
felis_status felis_config_wake(felis_config* c, const double* den_in, double* wake_e) {
  if (!c || !den_in || !wake_e) return FELIS_BAD_ARG;
  const felis_params& p = c->p;
  const int sliceN = p.global_slice_n;
  if (c->wakeF.empty()) wake_function(c);
  const double dZ = p.num_slice * p.lambda0;
  std::vector<double> den(den_in, den_in + sliceN);
  double totalCnt = 0.0;
  for (double v : den) totalCnt += v;
  if (totalCnt > 0.0) {
    const double norm = 1.0 / (totalCnt * dZ);
    for (double& v : den) v *= norm;
  }
  for (int i = 0; i < sliceN; ++i) wake_e[i] = 0.0;
  const double coef = totalCnt * 1.602e-19;
  for (int i = sliceN - 1; i >= 0; --i)
    for (int ii = i; ii >= 0; --ii) wake_e[ii] += den[i] * c->wakeF[i - ii] * dZ * coef;
  for (int i = 0; i < sliceN; ++i) c->wake_e[i] = wake_e[i];
  return FELIS_OK;
}

// The same on the device: wakeFunction (wakeField.cpp:53-159) when no wake
// function is cached yet, and the convolution of updateWakeField
// (wakeField.cpp:9-50) in the reference's order.  The density is normalised
// on the host as in felis_config_wake.
felis_status felis_config_wake_device(felis_config* c, const double* den_in, double* wake_e) {
  if (!c || !den_in || !wake_e) return FELIS_BAD_ARG;
  const felis_params& p = c->p;
  const int sliceN = p.global_slice_n;
  const double dZ = p.num_slice * p.lambda0;
  std::vector<double> den(den_in, den_in + sliceN);
  double totalCnt = 0.0;
  for (double v : den) totalCnt += v;
  if (totalCnt > 0.0) {
    const double norm = 1.0 / (totalCnt * dZ);
    for (double& v : den) v *= norm;
  }
  const double coef = totalCnt * 1.602e-19;
  const size_t S = (size_t)std::max(sliceN, 1);
  double *d_imp = nullptr, *d_wf = nullptr, *d_den = nullptr, *d_we = nullptr;
  cudaError_t e = cudaMalloc(&d_imp, (felis::kWakeNumK + 1) * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_wf, S * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_den, S * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_we, S * sizeof(double));
  const bool compute = c->wakeF.empty();
  if (e == cudaSuccess && compute) {
    felis::WakeArgs a{};
    a.shape = c->wakeShape; a.acdc = c->acdc; a.S = sliceN; a.dZ = dZ;
    a.s0 = pow(2.0 * c->radius * c->radius / kZ0 / c->cond, 1.0 / 3.0);
    a.ctau = c->ctau;
    a.coef = kZ0 * 3e8 / M_PI / c->radius / c->radius / M_PI;
    a.impZ = d_imp; a.wakeF = d_wf;
    e = felis::launch_wake_function(a, 0);
  } else if (e == cudaSuccess && sliceN > 0) {
    e = cudaMemcpy(d_wf, c->wakeF.data(), sliceN * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && sliceN > 0) e = cudaMemcpy(d_den, den.data(), sliceN * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = felis::launch_wake_field(d_den, d_wf, sliceN, dZ, coef, d_we, 0);
  if (e == cudaSuccess && sliceN > 0) e = cudaMemcpy(wake_e, d_we, sliceN * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && compute) {
    c->wakeF.assign(sliceN, 0.0);
    if (sliceN > 0) e = cudaMemcpy(c->wakeF.data(), d_wf, sliceN * sizeof(double), cudaMemcpyDeviceToHost);
  }
  for (double* q : {d_imp, d_wf, d_den, d_we})
    if (q) cudaFree(q);
  if (e != cudaSuccess) {
    if (compute) c->wakeF.clear();
    g_err = std::string("felis_config_wake_device: ") + cudaGetErrorString(e);
    return FELIS_CUDA_ERROR;
  }
  for (int i = 0; i < sliceN; ++i) c->wake_e[i] = wake_e[i];
  return FELIS_OK;
}

// The cached wake function (wakeField.cpp:128-140), global slice distances.
felis_status felis_config_wake_function(felis_config* c, double* wake_f) {
  if (!c || !wake_f) return FELIS_BAD_ARG;
  if (c->wakeF.empty()) wake_function(c);
  std::copy(c->wakeF.begin(), c->wakeF.end(), wake_f);
  return FELIS_OK;
}

}  // extern "C"

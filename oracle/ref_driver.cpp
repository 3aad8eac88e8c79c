// ref_driver.cpp — runs the reference's own setup and step loop, compiled
// from its unmodified sources, and writes the results as raw binary files.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref/felis_ref*).  tests/,
// __graft_entry__.smoke() and bench.py's reference arm run it as a child
// process in a scratch directory (the reference writes its text outputs --
// totalEnergy, twissFile, bFactor, wakeE, impZ, normDen -- into the current
// directory).  The product never runs it.
//
// What it calls, all from the reference (file:line):
//   parameterSetting     parameterSetting.cpp:42-285
//   boundary             boundary.cpp:20-130
//   wakeFunction         wakeField.cpp:53-159
//   loadSeed, loadBeam   loadSeed.cpp:10-80, loadBeam.cpp:14-269 (fresh start)
//   updateWakeField      wakeField.cpp:9-50
//   updateTotalEnergy    updateTotalEnergy.cpp:7-87
//   calculate_twiss      twiss.cpp:7-99
//   updatebFactor        saveFile.cpp:109-172
//   solveField           solveField.cpp:49-78
//   updateK_quadG        updateK_quadG.cpp:8-94
//   transversePush       particlePush.cpp:32-117
//   push_theta_gamma, drift_theta_gamma   particlePush.cpp:15-29, 119-195
//   periodicParticles    rearrangeParticles.cpp:77-114
//   shiftField           solveField.cpp:19-47 (+ fieldShareZ.cpp:39-78)
// in the order of main.cpp:44-90 (setup) and main.cpp:92-156 (loop), which is
// restated below without the saves and progress prints.  A restart from an
// injected state follows main.cpp:58-67: the initial state replaces loadSeed
// and loadBeam, and updateWakeField runs once before the loop.
//
// Usage: felis_ref INPUT OUTDIR [options]
//   --state DIR       initial state from DIR (same files as written below)
//                     instead of loadSeed + loadBeam
//   --bessel FILE     replace the Bessel table after boundary() (bn x orders
//                     doubles, row-major)
//   --from N --to N   iteration range (default 0 .. maxStep)
//   --setup           write the Domain scalars and tables after setup
//   --initial         write the initial state (after loading) to OUTDIR/init
//   --no-final        do not write the final state
//   --time W          time the loop after W untimed iterations (timing.txt)
// Files (little-endian raw arrays): Ux_<h>.bin, Uy_<h>.bin ((S+2) ny nx
// complex128, ghost planes included), Ez_<l>.bin, p<s>_{x,y,px,py,theta,gamma}
// .bin (float64, slice-major), p<s>_offsets.bin (int64, S+1),
// p<s>_weights.bin (float64, S), energyX.bin / energyY.bin (iterations x H,
// the sums of |U|^2 updateTotalEnergy stores), wakeE.bin (the wake energy loss
// per global slice as the loop left it), setup.txt, meta.txt (sizes).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <chrono>
#include <string>
#include <vector>

#include "mesh.h"
#include "mpi.h"

void wakeFunction(Domain* D, int iteration);
void updateWakeField(Domain* D, int iteration);

namespace {

[[noreturn]] void die(const std::string& msg) {
  fprintf(stderr, "felis_ref: %s\n", msg.c_str());
  exit(3);
}

template <class T>
void write_raw(const std::string& path, const T* data, size_t n) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) die("cannot write " + path);
  if (n && fwrite(data, sizeof(T), n, f) != n) die("short write " + path);
  fclose(f);
}

template <class T>
std::vector<T> read_raw(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) die("cannot read " + path);
  fseek(f, 0, SEEK_END);
  const long bytes = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<T> v((size_t)bytes / sizeof(T));
  if (!v.empty() && fread(v.data(), sizeof(T), v.size(), f) != v.size()) die("short read " + path);
  fclose(f);
  return v;
}

bool exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

void write_state(Domain& D, const std::string& dir) {
  mkdir(dir.c_str(), 0755);
  for (int h = 0; h < D.numHarmony; ++h) {
    write_raw(dir + "/Ux_" + std::to_string(h) + ".bin", D.Ux[h].data(), D.Ux[h].size());
    write_raw(dir + "/Uy_" + std::to_string(h) + ".bin", D.Uy[h].data(), D.Uy[h].size());
  }
  for (int l = 0; l < D.SCLmode; ++l)
    write_raw(dir + "/Ez_" + std::to_string(l) + ".bin", D.Ez[l].data(), D.Ez[l].size());
  const char* names[6] = {"x", "y", "px", "py", "theta", "gamma"};
  for (int s = 0; s < D.nSpecies; ++s) {
    std::vector<double> cols[6];
    std::vector<int64_t> offs(1, 0);
    std::vector<double> w;
    for (int i = 1; i <= D.subSliceN; ++i) {
      ptclList* p = D.particle[i].head[s]->pt;
      const std::vector<double>* src[6] = {&p->x, &p->y, &p->px, &p->py, &p->theta, &p->gamma};
      for (int c = 0; c < 6; ++c) cols[c].insert(cols[c].end(), src[c]->begin(), src[c]->end());
      offs.push_back(offs.back() + (int64_t)p->x.size());
      w.push_back(p->weight);
      if (p->next) die("more than one particle node in a slice");
    }
    const std::string pre = dir + "/p" + std::to_string(s) + "_";
    for (int c = 0; c < 6; ++c) write_raw(pre + names[c] + ".bin", cols[c].data(), cols[c].size());
    write_raw(pre + "offsets.bin", offs.data(), offs.size());
    write_raw(pre + "weights.bin", w.data(), w.size());
  }
}

void read_state(Domain& D, const std::string& dir) {
  for (int h = 0; h < D.numHarmony; ++h) {
    for (int pol = 0; pol < 2; ++pol) {
      const std::string f = dir + (pol ? "/Uy_" : "/Ux_") + std::to_string(h) + ".bin";
      std::vector<cplx> u = read_raw<cplx>(f);
      std::vector<cplx>& dst = pol ? D.Uy[h] : D.Ux[h];
      if (u.size() != dst.size()) die("field size mismatch in " + f);
      dst = u;
    }
  }
  const char* names[6] = {"x", "y", "px", "py", "theta", "gamma"};
  for (int s = 0; s < D.nSpecies; ++s) {
    const std::string pre = dir + "/p" + std::to_string(s) + "_";
    std::vector<double> cols[6];
    for (int c = 0; c < 6; ++c) cols[c] = read_raw<double>(pre + names[c] + ".bin");
    std::vector<int64_t> offs = read_raw<int64_t>(pre + "offsets.bin");
    std::vector<double> w = read_raw<double>(pre + "weights.bin");
    if ((int)offs.size() != D.subSliceN + 1 || (int)w.size() != D.subSliceN)
      die("particle offsets/weights do not match the slice count");
    for (int i = 1; i <= D.subSliceN; ++i) {
      ptclList* p = new ptclList();
      const size_t a = (size_t)offs[i - 1], b = (size_t)offs[i];
      std::vector<double>* dst[6] = {&p->x, &p->y, &p->px, &p->py, &p->theta, &p->gamma};
      for (int c = 0; c < 6; ++c) dst[c]->assign(cols[c].begin() + a, cols[c].begin() + b);
      p->weight = w[i - 1];
      p->next = D.particle[i].head[s]->pt;
      D.particle[i].head[s]->pt = p;
    }
  }
}

void write_setup(Domain& D, const std::string& dir) {
  FILE* f = fopen((dir + "/setup.txt").c_str(), "w");
  if (!f) die("cannot write setup.txt");
#define I_(k) fprintf(f, #k " %d\n", (int)D.k)
#define D_(k) fprintf(f, #k " %.17g\n", (double)D.k)
  I_(dimension); I_(mode); I_(numHarmony); I_(maxStep); I_(saveStep); I_(saveStart);
  I_(sliceN); I_(subSliceN); I_(nx); I_(ny); I_(minI); I_(maxI); I_(abcN); I_(nSpecies);
  I_(numSlice); I_(undType); I_(numLambdaU); I_(nUnd); I_(nQuad); I_(SCLmode); I_(SCFmode);
  I_(nr); I_(BesselMaxOrder); I_(bn); I_(loadH); I_(wakeShape); I_(ac_dc); I_(wakeONOFF);
  I_(wakeFieldStep);
  D_(ks); D_(lambda0); D_(minX); D_(maxX); D_(minY); D_(maxY); D_(minZ); D_(maxZ); D_(Lz);
  D_(dz); D_(dx); D_(dy); D_(gamR); D_(abcSig); D_(gamma0); D_(lambdaU); D_(ku); D_(K0);
  D_(K0_alpha); D_(ue); D_(dr); D_(BesselMax); D_(dBessel); D_(laserAlpha); D_(P0);
  D_(duration); D_(spotSigR); D_(a0); D_(zR); D_(focus); D_(polarity); D_(laserPsi);
  D_(radius); D_(cond); D_(ctau); D_(totalCnt);
#undef I_
#undef D_
  for (int h = 0; h < D.numHarmony; ++h) fprintf(f, "harmony%d %d\n", h, D.harmony[h]);
  for (size_t s = 0; s < D.loadList.size(); ++s) {
    const LoadList& L = D.loadList[s];
    fprintf(f, "beam%zu.gamma0 %.17g\nbeam%zu.peakCurrent %.17g\nbeam%zu.spread %.17g\n", s, L.gamma0, s,
            L.peakCurrent, s, L.spread);
    fprintf(f, "beam%zu.numBeamlet %d\nbeam%zu.numInBeamlet %d\n", s, L.numBeamlet, s, L.numInBeamlet);
  }
  for (size_t u = 0; u < D.undList.size(); ++u) {
    const UndList& U = D.undList[u];
    for (size_t n = 0; n < U.K0.size(); ++n)
      fprintf(f, "und%zu.%zu %.17g %.17g %.17g %.17g %.17g\n", u, n, U.unitStart[n], U.unitEnd[n], U.undStart[n],
              U.undEnd[n], U.K0[n]);
  }
  fclose(f);
  if (D.dimension == 3) {
    write_raw(dir + "/abc_alpha.bin", D.ABCalpha.data(), D.ABCalpha.size());
    write_raw(dir + "/abc_alphaP.bin", D.ABCalphaP.data(), D.ABCalphaP.size());
    write_raw(dir + "/abc_beta.bin", D.ABCbeta.data(), D.ABCbeta.size());
    write_raw(dir + "/abc_betaP.bin", D.ABCbetaP.data(), D.ABCbetaP.size());
  }
  std::vector<double> bes;
  for (auto& row : D.BesselJ) bes.insert(bes.end(), row.begin(), row.end());
  write_raw(dir + "/bessel.bin", bes.data(), bes.size());
  write_raw(dir + "/wakeF.bin", D.wakeF.data(), D.wakeF.size());
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) die("usage: felis_ref INPUT OUTDIR [--state DIR] [--bessel FILE] [--from N] [--to N] "
                    "[--setup] [--initial] [--no-final] [--time W]");
  const std::string input = argv[1], out = argv[2];
  std::string state, bessel;
  int it0 = 0, it1 = -1, warm = -1;
  bool want_setup = false, want_initial = false, want_final = true;
  for (int a = 3; a < argc; ++a) {
    const std::string k = argv[a];
    auto val = [&]() -> std::string {
      if (a + 1 >= argc) die("missing value after " + k);
      return argv[++a];
    };
    if (k == "--state") state = val();
    else if (k == "--bessel") bessel = val();
    else if (k == "--from") it0 = atoi(val().c_str());
    else if (k == "--to") it1 = atoi(val().c_str());
    else if (k == "--setup") want_setup = true;
    else if (k == "--initial") want_initial = true;
    else if (k == "--no-final") want_final = false;
    else if (k == "--time") warm = atoi(val().c_str());
    else die("unknown option " + k);
  }
  mkdir(out.c_str(), 0755);
  if (!exists(input)) die("no input file " + input);

  MPI_Init(&argc, &argv);
  Domain D{};
  parameterSetting(&D, input.c_str());
  boundary(&D);
  if (!bessel.empty()) {
    std::vector<double> t = read_raw<double>(bessel);
    if (t.size() != (size_t)D.bn * D.BesselMaxOrder) die("Bessel table size mismatch");
    for (int i = 0; i < D.bn; ++i)
      for (int j = 0; j < D.BesselMaxOrder; ++j) D.BesselJ[i][j] = t[(size_t)i * D.BesselMaxOrder + j];
  }
  wakeFunction(&D, 0);

  if (state.empty()) {
    loadSeed(&D, 0);
    int s = 0;
    for (auto& LL : D.loadList) loadBeam(&D, LL, s++, 0);
  } else {
    read_state(D, state);
  }
  const bool td = D.mode == OperationMode::Time_Dependent;
  if (it0 != 0 && td) updateWakeField(&D, it0);
  if (it1 < 0 || it1 > D.maxStep) it1 = D.maxStep;
  if (want_setup) write_setup(D, out);
  if (want_initial) write_state(D, out + "/init");

  using clk = std::chrono::steady_clock;
  clk::time_point t_start = clk::now();
  int timed_from = warm >= 0 ? it0 + warm : it0;
  for (int iteration = it0; iteration < it1; ++iteration) {
    if (iteration == timed_from) t_start = clk::now();
    if (iteration % D.wakeFieldStep == 0 && td) updateWakeField(&D, iteration);
    updateTotalEnergy(&D, iteration);
    calculate_twiss(D, iteration);
    updatebFactor(D, iteration);
    solveField(&D, iteration);
    updateK_quadG(&D, iteration, 0);
    if (D.dimension == 3) transversePush(&D, iteration);
    updateK_quadG(&D, iteration, 0.5);
    if (D.dimension == 3) transversePush(&D, iteration);
    if (D.driftFlag == false) push_theta_gamma(&D, iteration);
    else drift_theta_gamma(D, iteration);
    periodicParticles(D, iteration);
    if (D.driftFlag == false && td) shiftField(D, iteration);
  }
  const double secs = std::chrono::duration<double>(clk::now() - t_start).count();

  if (warm >= 0) {
    double np = 0;
    for (int s = 0; s < D.nSpecies; ++s)
      for (int i = 1; i <= D.subSliceN; ++i) np += (double)D.particle[i].head[s]->pt->x.size();
    FILE* f = fopen((out + "/timing.txt").c_str(), "w");
    fprintf(f, "seconds %.9g\niterations %d\nparticles %.0f\nslices %d\nnx %d\nny %d\nharmonics %d\n", secs,
            it1 - timed_from, np, D.subSliceN, D.nx, D.ny, D.numHarmony);
    fclose(f);
  }
  {
    FILE* f = fopen((out + "/meta.txt").c_str(), "w");
    if (!f) die("cannot write meta.txt");
    fprintf(f, "harmonics %d\nspecies %d\nslices %d\nny %d\nnx %d\niterations %d\n", D.numHarmony, D.nSpecies,
            D.subSliceN, D.ny, D.nx, it1);
    fclose(f);
  }
  std::vector<double> ex, ey;
  for (int it = 0; it < it1; ++it)
    for (int h = 0; h < D.numHarmony; ++h) {
      ex.push_back(D.totalEnergyX[it][h]);
      ey.push_back(D.totalEnergyY[it][h]);
    }
  write_raw(out + "/energyX.bin", ex.data(), ex.size());
  write_raw(out + "/energyY.bin", ey.data(), ey.size());
  if (want_final) write_state(D, out);
  write_raw(out + "/wakeE.bin", D.wakeE.data(), D.wakeE.size());
  MPI_Finalize();
  return 0;
}

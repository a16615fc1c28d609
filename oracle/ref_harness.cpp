// Harness that drives the reference's own RunZustand/RunDynamik code
// (test infrastructure: the compiled reference checker under oracle/_ref).
//
// Pattern follows the reference's profiling driver (main_profile.cpp:123-139):
// RunZustand::init, then RunDynamik routines called directly. Positions and
// results are exchanged as raw little-endian binary files:
//   position file: int32 N1, int32 N2, then for species 1 and 2 in turn
//                  int32 git[N][2] followed by double rel[N][2].
// Commands:
//   init   SEED OUT.pos                  seeded init (startpos_methode of the build)
//   forces IN.pos OUT.bin                WCA11, WCA22, WCA12, kap on IN; dumps
//                                        F1_WCA,F1kap,F2_WCA,F2kap (double[N][2])
//                                        then rhox.re, Fx.re, Fy.re, Fx.im (Z*Z each)
//   steps  IN.pos NSTEPS NOISE|- EVERY OUT.bin
//                                        zeitschritt() NSTEPS times; NOISE holds the
//                                        injected u values (2*(N1+N2) per step); every
//                                        EVERY steps appends double dt_sum and a
//                                        position record (git int32[N][2], rel double[N][2]
//                                        per species)
//   lists  IN.pos OUT.bin                per species, per cell (i major, j minor):
//                                        int32 count then the neighbour-list ids
//   time   SEED NSTEPS WARMUP            seeded init then time zeitschritt(); prints
//   timefile IN.pos NSTEPS WARMUP        the same from the positions in IN.pos
//                                        one JSON line with seconds per step
//   stepsphilox IN.pos NSTEPS KEY|zero STRIDE CKPTS OUT.bin
//                                        zeitschritt() NSTEPS times with injected
//                                        noise drawn here per step: the Philox
//                                        uniform-disk uniforms of key KEY (the
//                                        oracle's bdo_philox_noise, the stream the
//                                        CUDA library draws), or u = 0.5 (xi = 0,
//                                        noiseless) for "zero". After each step
//                                        listed in CKPTS (comma separated) appends
//                                        int32 step, double dt_sum, then for the
//                                        particles 0, STRIDE, 2*STRIDE, ... of the
//                                        combined index (species 1 first) int32
//                                        git[2] and double rel[2] each.
//   obs    IN.pos OUT.bin                the in-run observables of RunObs on IN:
//                                        record_korrelationsfunktion11/12/22 and
//                                        record_ftrho_unkorrigiert (auswertung.cpp:
//                                        110-188, 262-375); dumps int32 korr_bins,
//                                        double g11, g12, g22 [korr_bins], int32
//                                        nq, int32 qabs2[nq], double ftrho1_re,
//                                        ftrho1_im, ftrho2_re, ftrho2_im [nq]
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include <fftw3.h>

#define private public
#define protected public
#include "parameter.h"
#include "signaturen2.h"
#undef private
#undef protected

void seam_seed(uint64_t seed);
void seam_inject(const double* u, size_t n);
size_t seam_injected_left();
size_t seam_drawn();
extern "C" void bdo_philox_noise(uint64_t seed, uint64_t step, int N1, int N2, int gauss,
                                 double* xi, double* u);

static void die(const char* msg) {
  std::fprintf(stderr, "ref_harness: %s\n", msg);
  std::exit(2);
}

static void write_pos(FILE* f, RunZustand& r) {
  int32_t hdr[2] = {N1, N2};
  std::fwrite(hdr, sizeof(int32_t), 2, f);
  const int Ns[2] = {N1, N2};
  int** git[2] = {r.r1_git, r.r2_git};
  double** rel[2] = {r.r1_rel, r.r2_rel};
  for (int s = 0; s < 2; s++) {
    for (int i = 0; i < Ns[s]; i++) {
      int32_t g[2] = {git[s][i][0], git[s][i][1]};
      std::fwrite(g, sizeof(int32_t), 2, f);
    }
    for (int i = 0; i < Ns[s]; i++) std::fwrite(rel[s][i], sizeof(double), 2, f);
  }
}

static void read_pos(const char* path, RunZustand& r) {
  FILE* f = std::fopen(path, "rb");
  if (!f) die("cannot open position file");
  int32_t hdr[2];
  if (std::fread(hdr, sizeof(int32_t), 2, f) != 2) die("short position header");
  if (hdr[0] != N1 || hdr[1] != N2) die("position file N1/N2 do not match the build");
  const int Ns[2] = {N1, N2};
  int** git[2] = {r.r1_git, r.r2_git};
  double** rel[2] = {r.r1_rel, r.r2_rel};
  for (int s = 0; s < 2; s++) {
    for (int i = 0; i < Ns[s]; i++) {
      int32_t g[2];
      if (std::fread(g, sizeof(int32_t), 2, f) != 2) die("short git");
      git[s][i][0] = g[0];
      git[s][i][1] = g[1];
    }
    for (int i = 0; i < Ns[s]; i++)
      if (std::fread(rel[s][i], sizeof(double), 2, f) != 2) die("short rel");
  }
  std::fclose(f);
}

// Fresh run with positions from IN (seeded init first so every buffer the
// reference allocates in RunZustand::init exists), then rebuild the
// neighbour lists exactly as RunDynamik::init does after an init routine.
static void load_run(RunZustand& r, const char* in) {
  seam_seed(12345);
  r.init(0);
  read_pos(in, r);
  r.dyn.init();
}

static void dump_forces(FILE* f, RunZustand& r) {
  auto& d = r.dyn;
  for (int i = 0; i < N1; i++) std::fwrite(d.F1_WCA[i], sizeof(double), 2, f);
  for (int i = 0; i < N1; i++) std::fwrite(d.F1kap[i], sizeof(double), 2, f);
  for (int i = 0; i < N2; i++) std::fwrite(d.F2_WCA[i], sizeof(double), 2, f);
  for (int i = 0; i < N2; i++) std::fwrite(d.F2kap[i], sizeof(double), 2, f);
  const int Z = densGrid_Zellen;
  for (int k = 0; k < Z * Z; k++) std::fwrite(&d.rhox[k][0], sizeof(double), 1, f);
  for (int k = 0; k < Z * Z; k++) std::fwrite(&d.Fx[k][0], sizeof(double), 1, f);
  for (int k = 0; k < Z * Z; k++) std::fwrite(&d.Fy[k][0], sizeof(double), 1, f);
  for (int k = 0; k < Z * Z; k++) std::fwrite(&d.Fx[k][1], sizeof(double), 1, f);
}

int main(int argc, char** argv) {
  if (argc < 2) die("usage: init|forces|steps|lists|time ...");
  std::string cmd = argv[1];
  if (cmd == "init") {
    if (argc != 4) die("init SEED OUT.pos");
    seam_seed(std::strtoull(argv[2], nullptr, 10));
    RunZustand r;
    r.init(0);
    FILE* f = std::fopen(argv[3], "wb");
    write_pos(f, r);
    std::fclose(f);
    return 0;
  }
  if (cmd == "forces") {
    if (argc != 4) die("forces IN.pos OUT.bin");
    RunZustand r;
    load_run(r, argv[2]);
    r.dyn.berechne_WCA11();
    r.dyn.berechne_WCA22();
    r.dyn.addiere_WCA12();
    r.dyn.berechne_kapkraefte();
    FILE* f = std::fopen(argv[3], "wb");
    dump_forces(f, r);
    std::fclose(f);
    return 0;
  }
  if (cmd == "steps") {
    if (argc != 7) die("steps IN.pos NSTEPS NOISE|- EVERY OUT.bin");
    RunZustand r;
    load_run(r, argv[2]);
    const long nsteps = std::atol(argv[3]);
    const long every = std::atol(argv[5]);
    std::vector<double> noise;
    const size_t per_step = 2 * (size_t)(N1 + N2);
    if (std::string(argv[4]) != "-") {
      FILE* nf = std::fopen(argv[4], "rb");
      if (!nf) die("cannot open noise file");
      noise.resize(per_step * nsteps);
      if (std::fread(noise.data(), sizeof(double), noise.size(), nf) != noise.size())
        die("short noise file");
      std::fclose(nf);
    }
    FILE* f = std::fopen(argv[6], "wb");
    double tsum = 0.0;
    for (long s = 0; s < nsteps; s++) {
      if (!noise.empty()) seam_inject(noise.data() + per_step * s, per_step);
      tsum += r.dyn.zeitschritt(1.0);
      if (!noise.empty() && !noWCA && seam_injected_left() != 0)
        die("injected noise not fully consumed (rejection triggered)");
      if ((s + 1) % every == 0) {
        std::fwrite(&tsum, sizeof(double), 1, f);
        write_pos(f, r);
      }
    }
    std::fclose(f);
    return 0;
  }
  if (cmd == "stepsphilox") {
    if (argc != 8) die("stepsphilox IN.pos NSTEPS KEY|zero STRIDE CKPTS OUT.bin");
    RunZustand r;
    load_run(r, argv[2]);
    const long nsteps = std::atol(argv[3]);
    const bool zero = std::string(argv[4]) == "zero";
    const uint64_t key = zero ? 0 : std::strtoull(argv[4], nullptr, 10);
    const long stride = std::atol(argv[5]);
    if (stride < 1) die("STRIDE must be >= 1");
    std::vector<long> ckpts;
    {
      std::stringstream ss(argv[6]);
      std::string item;
      while (std::getline(ss, item, ',')) ckpts.push_back(std::atol(item.c_str()));
    }
    const size_t per_step = 2 * (size_t)(N1 + N2);
    std::vector<double> u(per_step, 0.5), xi(per_step);
    FILE* f = std::fopen(argv[7], "wb");
    if (!f) die("cannot open output");
    double tsum = 0.0;
    int** git[2] = {r.r1_git, r.r2_git};
    double** rel[2] = {r.r1_rel, r.r2_rel};
    for (long s = 0; s < nsteps; s++) {
      if (!zero) bdo_philox_noise(key, (uint64_t)s, N1, N2, 0, xi.data(), u.data());
      seam_inject(u.data(), per_step);
      tsum += r.dyn.zeitschritt(1.0);
      if (!noWCA && seam_injected_left() != 0)
        die("injected noise not fully consumed (rejection triggered)");
      bool ck = false;
      for (long c : ckpts) ck = ck || (c == s + 1);
      if (!ck) continue;
      int32_t st = (int32_t)(s + 1);
      std::fwrite(&st, sizeof(int32_t), 1, f);
      std::fwrite(&tsum, sizeof(double), 1, f);
      for (long p = 0; p < (long)N1 + N2; p += stride) {
        const int sp = p < N1 ? 0 : 1;
        const long i = p < N1 ? p : p - N1;
        int32_t g[2] = {git[sp][i][0], git[sp][i][1]};
        std::fwrite(g, sizeof(int32_t), 2, f);
        std::fwrite(rel[sp][i], sizeof(double), 2, f);
      }
      std::fflush(f);
    }
    std::fclose(f);
    return 0;
  }
  if (cmd == "obs") {
    if (argc != 4) die("obs IN.pos OUT.bin");
    RunZustand r;
    load_run(r, argv[2]);
    auto& o = r.obs;
    // obs_init only sets these up when the auswerten_* switches are on, which
    // the generated parameter.h keeps off
    o.g11 = o.g12 = o.g22 = nullptr;
    o.ftrho1_re = o.ftrho1_im = o.ftrho2_re = o.ftrho2_im = nullptr;
    o.init_korrelationsfunktion();
    o.record_korrelationsfunktion11(0);
    o.record_korrelationsfunktion12(0);
    o.record_korrelationsfunktion22(0);
    o.init_ftrho();
    o.record_ftrho_unkorrigiert(0);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) die("cannot open output");
    const int32_t kb = korr_bins;
    std::fwrite(&kb, sizeof(int32_t), 1, f);
    for (auto* g : {o.g11, o.g12, o.g22}) std::fwrite(g[0].data(), sizeof(double), korr_bins, f);
    const int32_t nq = (int32_t)o.ftrho_qabs2.size();
    std::fwrite(&nq, sizeof(int32_t), 1, f);
    for (int q : o.ftrho_qabs2) {
      const int32_t w = q;
      std::fwrite(&w, sizeof(int32_t), 1, f);
    }
    for (auto* v : {o.ftrho1_re, o.ftrho1_im, o.ftrho2_re, o.ftrho2_im})
      std::fwrite(v[0].data(), sizeof(double), nq, f);
    std::fclose(f);
    return 0;
  }
  if (cmd == "lists") {
    if (argc != 4) die("lists IN.pos OUT.bin");
    RunZustand r;
    load_run(r, argv[2]);
    FILE* f = std::fopen(argv[3], "wb");
    for (int s = 0; s < 2; s++) {
      auto lists = s == 0 ? r.dyn.erwNachbarn1 : r.dyn.erwNachbarn2;
      for (int i = 0; i < nachList_Zellen; i++)
        for (int j = 0; j < nachList_Zellen; j++) {
          int32_t n = (int32_t)lists[i][j].size();
          std::fwrite(&n, sizeof(int32_t), 1, f);
          for (int v : lists[i][j]) {
            int32_t w = v;
            std::fwrite(&w, sizeof(int32_t), 1, f);
          }
        }
    }
    std::fclose(f);
    return 0;
  }
  if (cmd == "time" || cmd == "timefile") {
    if (argc != 5) die("time SEED|IN.pos NSTEPS WARMUP");
    const long nsteps = std::atol(argv[3]);
    const long warm = std::atol(argv[4]);
    RunZustand r;
    if (cmd == "time") {
      seam_seed(std::strtoull(argv[2], nullptr, 10));
      r.init(0);
    } else {
      load_run(r, argv[2]);
    }
    for (long s = 0; s < warm; s++) r.dyn.zeitschritt(1.0);
    auto t0 = std::chrono::steady_clock::now();
    double tsum = 0.0;
    for (long s = 0; s < nsteps; s++) tsum += r.dyn.zeitschritt(1.0);
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"steps\": %ld, \"seconds\": %.9g, \"sec_per_step\": %.9g, \"N\": %d, \"t_sim\": %.9g}\n",
                nsteps, sec, sec / (double)nsteps, N1 + N2, tsum);
    return 0;
  }
  die("unknown command");
  return 2;
}

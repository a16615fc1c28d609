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

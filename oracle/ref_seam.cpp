// RNG link seam for the compiled reference checker (test infrastructure).
//
// Replaces the reference's zufall.cpp at link time. The reference draws all
// randomness through zufall_gleichverteilt_vonbis(a, b) = a + (b-a)*u with
// u = uniform_real_distribution<double>(0,1) over an mt19937_64 seeded with
// time(NULL) (reference zufall.cpp:18-39). This seam keeps that exact stream
// but takes the seed from the harness, and can instead hand out a prescribed
// sequence of u values ("injected noise"): the reference's noise routine
// (dynamik_methoden.cpp:1317-1339) turns each pair (u_x, u_y) into
// xi = sqrt(5)*(2u-1), so injecting u = (xi/sqrt(5)+1)/2 reproduces a chosen xi.
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>

namespace {
std::mt19937_64 g_gen(0);
std::uniform_real_distribution<double> g_dist(0.0, 1.0);
const double* g_inj = nullptr;
size_t g_inj_n = 0;
size_t g_inj_pos = 0;
size_t g_drawn = 0;
}  // namespace

void seam_seed(uint64_t seed) { g_gen.seed(seed); }

void seam_inject(const double* u, size_t n) {
  g_inj = u;
  g_inj_n = n;
  g_inj_pos = 0;
}

size_t seam_injected_left() { return g_inj ? g_inj_n - g_inj_pos : 0; }
size_t seam_drawn() { return g_drawn; }

double zufall_gleichverteilt() {
  ++g_drawn;
  if (g_inj) {
    if (g_inj_pos >= g_inj_n) {
      std::fprintf(stderr, "seam: injected stream exhausted\n");
      std::exit(3);
    }
    return g_inj[g_inj_pos++];
  }
  return g_dist(g_gen);
}

void init_rng() {}

double zufall_gleichverteilt_vonbis(double min, double max) {
  return min + (max - min) * zufall_gleichverteilt();
}

int zufall_Int(int N) { return ((int)(N * zufall_gleichverteilt())) % N; }

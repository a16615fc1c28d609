/*
 * bd_oracle — CPU restatement (FP64, plain C) of the reference's
 * force-and-integrate step. TEST INFRASTRUCTURE ONLY: it is the checker the
 * tests, smoke() and bench.py's CPU-baseline leg compare the CUDA library
 * against; the product never links or calls it.
 *
 * It follows the reference routine by routine (file:line cited at each
 * function in bd_oracle.c), including the order of every floating-point
 * operation and the history-dependent neighbour-list order, so that its
 * results are bit-identical to the compiled reference (pinned by
 * tests/test_oracle_vs_reference.py and the golden fixtures).
 * Parameters are runtime values with the names of reference parameter.h.
 */
#ifndef BD_ORACLE_H
#define BD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bdo_params {
  int N1, N2;
  double L;
  int densGrid_Schema;
  int FFT_samples;
  double lambda_kapillar, kapillar_vorfaktor, T, dt_max, max_reisedistanz;
  double sigma11_22, sigma11_12, Gamma2_1, eps22_11, eps12_11, f2_f1;
  int idgas_only, noWCA, noRNG, quickInit, restrictRadial;
  double maxPairWCA;
  double obs_dt;
  int startpos_methode;
  double startpos_kreisradius;
} bdo_params;

/* noise sources */
enum {
  BDO_NOISE_REF_STREAM = 0, /* reference: uniform disk from seeded mt19937_64 */
  BDO_NOISE_INJECTED = 1,   /* reference: uniform disk from caller's u values */
  BDO_NOISE_PHILOX_DISK = 2, /* uniform disk, Philox4x32-10 counter stream */
  BDO_NOISE_PHILOX_GAUSS = 3, /* Gaussian N(0,1), Philox4x32-10 + Box-Muller */
  BDO_NOISE_NONE = 4
};

typedef struct bdo_ctx bdo_ctx;

bdo_ctx* bdo_create(const bdo_params* p, uint64_t seed);
void bdo_destroy(bdo_ctx* c);

int bdo_nachList_Zellen(const bdo_ctx* c);
double bdo_nachList_Breite(const bdo_ctx* c);

/* positions, reference layout: git int32[N][2], rel double[N][2] */
int bdo_init_positions(bdo_ctx* c, int methode);
void bdo_set_positions(bdo_ctx* c, int species, const int32_t* git, const double* rel);
void bdo_get_positions(const bdo_ctx* c, int species, int32_t* git, double* rel);

/* routines with the reference's names */
void bdo_WCA_init(bdo_ctx* c);
void bdo_kapkraefte_init(bdo_ctx* c);
void bdo_berechne_WCA11(bdo_ctx* c);
void bdo_berechne_WCA22(bdo_ctx* c);
void bdo_addiere_WCA12(bdo_ctx* c);
void bdo_berechne_kapkraefte(bdo_ctx* c);
void bdo_gridDensity(bdo_ctx* c, int schema);
void bdo_inv_gridDensity(bdo_ctx* c, int schema);
void bdo_berechne_zufallskraefte(bdo_ctx* c);
double bdo_optimaler_zeitschritt(bdo_ctx* c);
void bdo_refresh_erwNachbar(bdo_ctx* c);
double bdo_zeitschritt(bdo_ctx* c, double tmax);
double bdo_zeitschritte(bdo_ctx* c, int n); /* n steps, returns summed dt */
double bdo_zeitschritt_mrd(bdo_ctx* c, double mrd); /* step with travel bound mrd */

/* kind: 0 WCA, 1 KAP, 2 NOISE; out double[N][2] */
void bdo_get_forces(const bdo_ctx* c, int kind, int species, double* out);
/* which: 0 rhox.re, 1 Fx.re, 2 Fy.re, 3 Fx.im ; out double[Z*Z], index k*Z+l */
void bdo_get_grid(const bdo_ctx* c, int which, double* out);
/* neighbour list of cell (i,j) of a species; returns its length, copies up to cap ids */
int bdo_get_list(const bdo_ctx* c, int species, int i, int j, int32_t* out, int cap);
/* number of out-of-range mesh indices met (the reference writes rhox[-1] there) */
long bdo_oob_count(const bdo_ctx* c);

void bdo_set_noise(bdo_ctx* c, int mode, uint64_t seed);
void bdo_inject_uniforms(bdo_ctx* c, const double* u, size_t n);
void bdo_set_step(bdo_ctx* c, uint64_t step);
uint64_t bdo_get_step(const bdo_ctx* c);

/* Philox noise as the CUDA library draws it, for the given per-run key,
 * step and particle counts. xi: double[(N1+N2)][2] (species 1 first).
 * u (optional): the accepted uniforms (2 per particle, disk mode only) that
 * make the reference's own noise routine produce the same xi. */
void bdo_philox_noise(uint64_t seed, uint64_t step, int N1, int N2, int gauss,
                      double* xi, double* u);
void bdo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* mt19937_64 + uniform_real_distribution<double>(0,1), as the reference draws */
double bdo_uniform(bdo_ctx* c);

/* snapshot text exactly as RunObs::schreibe_pos (auswertung.cpp:631-648) */
int bdo_schreibe_pos(const bdo_ctx* c, const char* path1, const char* path2, int nr,
                     int write_header);

/* Local densities of the offline analysis (main_auswertung.cpp:182-390):
 * snapgrid_num (parameter.h:174), the TSC-gridded densities of both species
 * (g1, g2: double[n*n], index k*n + l, k along x; x1, x2: absolute
 * positions double[N][2]), and from them the histograms (hist: int[4][bins]
 * = rho1, rho2, rho1+rho2, rho1-rho2) and threshold counts (over: int[7] =
 * rho over rho_thresh[0..2], |drho|/rho over drho_thresh[0..3]). */
int bdo_snapgrid_num(double L, double snapgrid_crude);
void bdo_lokale_dichte(int n, double width, int N1, const double* x1, int N2, const double* x2,
                       double* g1, double* g2);
void bdo_rhohist(int n, const double* g1, const double* g2, int bins, double dbin,
                 const double* rho_thresh, const double* drho_thresh, int* hist, int* over);

#ifdef __cplusplus
}
#endif
#endif

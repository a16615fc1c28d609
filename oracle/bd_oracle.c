/*
 * bd_oracle.c — FP64 CPU restatement of the reference's timestep path.
 * TEST INFRASTRUCTURE (the oracle): used only by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg as the checker. Never linked by the product.
 *
 * Each routine cites the reference routine it restates. Floating-point
 * expressions keep the reference's evaluation order so that, with the same
 * FFT (oracle/fftw_shim) and without FMA contraction, results match the
 * compiled reference bit for bit. Known reference defects are reproduced
 * except where they are undefined behaviour:
 *   - out-of-range mesh index (reference iw() returns -1 and the caller
 *     writes rhox[-1], allgemeine_methoden.cpp:242-250): the oracle wraps the
 *     index periodically and counts the event (bdo_oob_count).
 */
#include "bd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

/* ------------------------------------------------------------------ */
/* growable int list with the reference's vector<int> push_back / erase */
typedef struct {
  int32_t* v;
  int n, cap;
} ilist;

static void il_push(ilist* l, int32_t x) {
  if (l->n == l->cap) {
    l->cap = l->cap ? 2 * l->cap : 8;
    l->v = (int32_t*)realloc(l->v, sizeof(int32_t) * l->cap);
  }
  l->v[l->n++] = x;
}

/* erwListe_rem (dynamik_methoden.cpp:1398-1417): erase first occurrence */
static void il_rem(ilist* l, int32_t k) {
  int i;
  for (i = 0; i < l->n; i++)
    if (l->v[i] == k) break;
  if (i == l->n) return; /* reference would erase end(): undefined; ignore */
  memmove(l->v + i, l->v + i + 1, sizeof(int32_t) * (l->n - i - 1));
  l->n--;
}

/* ------------------------------------------------------------------ */
/* mt19937_64 (Matsumoto-Nishimura 64-bit Mersenne Twister), the engine the
 * reference seeds in zufall.cpp:18 */
typedef struct {
  uint64_t mt[312];
  int idx;
} mt64;

static void mt64_seed(mt64* m, uint64_t s) {
  m->mt[0] = s;
  for (int i = 1; i < 312; i++)
    m->mt[i] = 6364136223846793005ULL * (m->mt[i - 1] ^ (m->mt[i - 1] >> 62)) + (uint64_t)i;
  m->idx = 312;
}

static uint64_t mt64_next(mt64* m) {
  static const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
  static const uint64_t MA = 0xB5026F5AA96619E9ULL;
  if (m->idx >= 312) {
    for (int i = 0; i < 312; i++) {
      uint64_t x = (m->mt[i] & UM) | (m->mt[(i + 1) % 312] & LM);
      uint64_t xa = x >> 1;
      if (x & 1ULL) xa ^= MA;
      m->mt[i] = m->mt[(i + 156) % 312] ^ xa;
    }
    m->idx = 0;
  }
  uint64_t y = m->mt[m->idx++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= y >> 43;
  return y;
}

/* ------------------------------------------------------------------ */
struct bdo_ctx {
  bdo_params p;
  int N1, N2, C, Z;
  double B, dx, dq, zweihoch1_6, drho;
  int32_t* git[2];
  double* rel[2];
  double* F_WCA[2];
  double* Fkap[2];
  double* Fnoise[2];
  ilist* erw[2]; /* C*C lists, index i*C+j */
  fftw_complex *rhox, *rhok, *Fxk, *Fyk, *Fx, *Fy;
  double *sinxG, *sinyG;
  fftw_plan fwd, bx, by;
  int noise_mode;
  mt64 gen;
  const double* inj;
  size_t inj_n, inj_pos;
  uint64_t philox_seed;
  uint64_t step;
  long oob;
};

double bdo_uniform(bdo_ctx* c) {
  if (c->noise_mode == BDO_NOISE_INJECTED && c->inj) {
    if (c->inj_pos >= c->inj_n) {
      fprintf(stderr, "bd_oracle: injected stream exhausted\n");
      abort();
    }
    return c->inj[c->inj_pos++];
  }
  /* uniform_real_distribution<double>(0,1): one 64-bit draw scaled by 2^-64,
   * values that round up to 1 map to the largest double below 1 */
  uint64_t x = mt64_next(&c->gen);
  double r = (double)x * 0x1p-64;
  if (r >= 1.0) r = nextafter(1.0, 0.0);
  return r * (1.0 - 0.0) + 0.0;
}

/* zufall_gleichverteilt_vonbis (zufall.cpp:35-39) */
static double vonbis(bdo_ctx* c, double a, double b) { return a + (b - a) * bdo_uniform(c); }

/* iw (allgemeine_methoden.cpp:242-250); out-of-range wraps and is counted */
static int iw(bdo_ctx* c, int i, int j) {
  const int Z = c->Z;
  if (i >= Z || j >= Z || i < 0 || j < 0) {
    c->oob++;
    i = ((i % Z) + Z) % Z;
    j = ((j % Z) + Z) % Z;
  }
  return i * Z + j;
}

bdo_ctx* bdo_create(const bdo_params* p, uint64_t seed) {
  bdo_ctx* c = (bdo_ctx*)calloc(1, sizeof(*c));
  c->p = *p;
  c->N1 = p->N1;
  c->N2 = p->N2;
  /* parameter.h:171-209 */
  c->zweihoch1_6 = pow(2.0, 1.0 / 6.0);
  c->C = (int)floor(p->L / c->zweihoch1_6);
  c->B = p->L / ((double)c->C);
  c->dx = p->L / p->FFT_samples;
  c->Z = p->FFT_samples;
  c->dq = 2.0 * M_PI / p->L;
  c->drho = 1.0 / (c->dx * c->dx); /* gridRoutinen.cpp:28 */
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++) {
    size_t n = Ns[s] > 0 ? (size_t)Ns[s] : 1;
    c->git[s] = (int32_t*)calloc(2 * n, sizeof(int32_t));
    c->rel[s] = (double*)calloc(2 * n, sizeof(double));
    c->F_WCA[s] = (double*)calloc(2 * n, sizeof(double));
    c->Fkap[s] = (double*)calloc(2 * n, sizeof(double));
    c->Fnoise[s] = (double*)calloc(2 * n, sizeof(double));
    c->erw[s] = (ilist*)calloc((size_t)c->C * c->C, sizeof(ilist));
  }
  mt64_seed(&c->gen, seed);
  c->noise_mode = BDO_NOISE_REF_STREAM;
  bdo_kapkraefte_init(c);
  return c;
}

void bdo_destroy(bdo_ctx* c) {
  if (!c) return;
  for (int s = 0; s < 2; s++) {
    free(c->git[s]);
    free(c->rel[s]);
    free(c->F_WCA[s]);
    free(c->Fkap[s]);
    free(c->Fnoise[s]);
    for (int k = 0; k < c->C * c->C; k++) free(c->erw[s][k].v);
    free(c->erw[s]);
  }
  fftw_destroy_plan(c->fwd);
  fftw_destroy_plan(c->bx);
  fftw_destroy_plan(c->by);
  fftw_free(c->rhox);
  fftw_free(c->rhok);
  fftw_free(c->Fxk);
  fftw_free(c->Fyk);
  fftw_free(c->Fx);
  fftw_free(c->Fy);
  free(c->sinxG);
  free(c->sinyG);
  free(c);
}

int bdo_nachList_Zellen(const bdo_ctx* c) { return c->C; }
double bdo_nachList_Breite(const bdo_ctx* c) { return c->B; }

/* ------------------------------------------------------------------ */
/* initialisers (dynamik_methoden.cpp:1647-1851) */
static void set_cell(bdo_ctx* c, int s, int i, int jc, int kc, double relx, double rely) {
  c->git[s][2 * i] = jc;
  c->git[s][2 * i + 1] = kc;
  c->rel[s][2 * i] = relx;
  c->rel[s][2 * i + 1] = rely;
}

int bdo_init_positions(bdo_ctx* c, int methode) {
  const double B = c->B, L = c->p.L;
  const int Ns[2] = {c->N1, c->N2};
  switch (methode) {
    case 1: /* init_zufallspos :1647-1678, including the (int) x / B precedence */
      for (int s = 0; s < 2; s++)
        for (int i = 0; i < Ns[s]; i++) {
          double x = vonbis(c, 0.0, L);
          double y = vonbis(c, 0.0, L);
          int jc = (int)((double)((int)x) / B);
          int kc = (int)((double)((int)y) / B);
          set_cell(c, s, i, jc, kc, x - jc * B, y - kc * B);
        }
      break;
    case 3: { /* init_gitterstart :1762-1789 */
      if (c->N2 != 0) return -1;
      double wurzelN = ceil(sqrt((double)c->N1));
      double schrittweite = L / wurzelN;
      int index = 0;
      for (int i = 0; i < wurzelN && index < c->N1; i++)
        for (int j = 0; j < wurzelN; j++) {
          double x = i * schrittweite;
          double y = j * schrittweite;
          int ic = (int)(x / B);
          int jc = (int)(y / B);
          set_cell(c, 0, index, ic, jc, x - ic * B, y - jc * B);
          if (++index == c->N1) break;
        }
      break;
    }
    case 4: /* init_allegleich :1681-1711 */
      for (int s = 0; s < 2; s++) {
        double x = vonbis(c, 0.0, L);
        double y = vonbis(c, 0.0, L);
        int jc = (int)(x / B);
        int kc = (int)(y / B);
        for (int i = 0; i < Ns[s]; i++) set_cell(c, s, i, jc, kc, x - jc * B, y - kc * B);
      }
      break;
    case 5: { /* init_kreisscheibe :1714-1758 */
      const double rad = c->p.startpos_kreisradius;
      const double rad2 = rad * rad;
      for (int s = 0; s < 2; s++)
        for (int i = 0; i < Ns[s]; i++) {
          double x, y;
          do {
            x = vonbis(c, -rad, rad);
            y = vonbis(c, -rad, rad);
          } while (x * x + y * y > rad2);
          x += 0.5 * L;
          y += 0.5 * L;
          int jc = (int)(x / B);
          int kc = (int)(y / B);
          set_cell(c, s, i, jc, kc, x - jc * B + 0.03, y - kc * B + 0.03);
        }
      break;
    }
    case 6: { /* init_kernundring :1792-1828 */
      const double mitte = 0.5 * L;
      if (c->N1 != 1 || c->N2 < 3) return -1;
      {
        double x = mitte, y = mitte;
        int ic = (int)(x / B), jc = (int)(y / B);
        set_cell(c, 0, 0, ic, jc, x - ic * B, y - jc * B);
      }
      for (int t = 0; t < c->N2; t++) {
        double x = mitte + c->p.startpos_kreisradius * cos(2 * M_PI * (double)t / c->N2);
        double y = mitte + c->p.startpos_kreisradius * sin(2 * M_PI * (double)t / c->N2);
        int ic = (int)(x / B), jc = (int)(y / B);
        set_cell(c, 1, t, ic, jc, x - ic * B, y - jc * B);
      }
      break;
    }
    case 7: { /* init_posKrafttest :1830-1851 */
      if (c->N2 != 0 || c->N1 != 2) return -1;
      double x = 0.5 * c->dx, y = 0.5 * c->dx;
      int g0 = (int)(x / B), g1 = (int)(y / B);
      set_cell(c, 0, 0, g0, g1, x - g0 * B, y - g1 * B);
      y = 0.55 * c->dx;
      int h1 = (int)(y / B);
      set_cell(c, 0, 1, g0, h1, c->rel[0][0], y - h1 * B);
      break;
    }
    default:
      return -1;
  }
  /* a disk or ring wider than the box puts cells outside [0, C): the
   * reference then indexes its lists out of range; refuse instead */
  for (int s = 0; s < 2; s++)
    for (int i = 0; i < 2 * Ns[s]; i++)
      if (c->git[s][i] < 0 || c->git[s][i] >= c->C) return -2;
  bdo_WCA_init(c);
  return 0;
}

void bdo_set_positions(bdo_ctx* c, int species, const int32_t* git, const double* rel) {
  const int n = species == 0 ? c->N1 : c->N2;
  memcpy(c->git[species], git, sizeof(int32_t) * 2 * (size_t)n);
  memcpy(c->rel[species], rel, sizeof(double) * 2 * (size_t)n);
}

void bdo_get_positions(const bdo_ctx* c, int species, int32_t* git, double* rel) {
  const int n = species == 0 ? c->N1 : c->N2;
  if (git) memcpy(git, c->git[species], sizeof(int32_t) * 2 * (size_t)n);
  if (rel) memcpy(rel, c->rel[species], sizeof(double) * 2 * (size_t)n);
}

/* ------------------------------------------------------------------ */
/* WCA_init (dynamik_methoden.cpp:459-526): every particle into the 3x3 lists */
static void nine_cells(int C, int k, int l, int* x, int* y) {
  x[0] = (k - 1 + C) % C;
  x[1] = k;
  x[2] = (k + 1) % C;
  y[0] = (l - 1 + C) % C;
  y[1] = l;
  y[2] = (l + 1) % C;
}

void bdo_WCA_init(bdo_ctx* c) {
  const int C = c->C;
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++) {
    for (int k = 0; k < C * C; k++) c->erw[s][k].n = 0;
    for (int t = 0; t < Ns[s]; t++) {
      int x[3], y[3];
      nine_cells(C, c->git[s][2 * t], c->git[s][2 * t + 1], x, y);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) il_push(&c->erw[s][x[i] * C + y[j]], t);
    }
  }
}

/* refresh_erwNachbar (dynamik_methoden.cpp:216-325) */
void bdo_refresh_erwNachbar(bdo_ctx* c) {
  const int C = c->C;
  const double B = c->B;
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++)
    for (int t = 0; t < Ns[s]; t++) {
      double* r = c->rel[s] + 2 * t;
      int32_t* g = c->git[s] + 2 * t;
      if (r[0] < 0.0 || r[0] > B || r[1] < 0.0 || r[1] > B) {
        int x[3], y[3];
        nine_cells(C, g[0], g[1], x, y);
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) il_rem(&c->erw[s][x[i] * C + y[j]], t);
        int ic = (int)floor((g[0] * B + r[0]) / B);
        int jc = (int)floor((g[1] * B + r[1]) / B);
        ic = (ic + C) % C;
        jc = (jc + C) % C;
        r[0] = fmod(r[0] + B, B);
        r[1] = fmod(r[1] + B, B);
        g[0] = ic;
        g[1] = jc;
        nine_cells(C, ic, jc, x, y);
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) il_push(&c->erw[s][x[i] * C + y[j]], t);
      }
    }
}

/* abstand2_* (allgemeine_methoden.cpp:100-166) */
static double abstand2(const bdo_ctx* c, int si, int i, int sj, int j) {
  const double B = c->B, L = c->p.L;
  double xi_abs = c->git[si][2 * i] * B + c->rel[si][2 * i];
  double xj_abs = c->git[sj][2 * j] * B + c->rel[sj][2 * j];
  double yi_abs = c->git[si][2 * i + 1] * B + c->rel[si][2 * i + 1];
  double yj_abs = c->git[sj][2 * j + 1] * B + c->rel[sj][2 * j + 1];
  double tmp1 = xi_abs - xj_abs;
  double tmp2 = xi_abs - xj_abs + L;
  double tmp3 = xi_abs - xj_abs - L;
  double m23 = (tmp3 * tmp3 < tmp2 * tmp2) ? tmp3 * tmp3 : tmp2 * tmp2;
  double dx2 = (m23 < tmp1 * tmp1) ? m23 : tmp1 * tmp1;
  tmp1 = yi_abs - yj_abs;
  tmp2 = yi_abs - yj_abs + L;
  tmp3 = yi_abs - yj_abs - L;
  m23 = (tmp3 * tmp3 < tmp2 * tmp2) ? tmp3 * tmp3 : tmp2 * tmp2;
  double dy2 = (m23 < tmp1 * tmp1) ? m23 : tmp1 * tmp1;
  return dx2 + dy2;
}

/* absolute-coordinate difference with the reference's periodic shift
 * (e.g. dynamik_methoden.cpp:659-683) */
static void pair_delta(const bdo_ctx* c, int si, int i, int sj, int j, double a2, double* pdx,
                       double* pdy) {
  const double B = c->B, L = c->p.L;
  double x1 = c->git[si][2 * i] * B + c->rel[si][2 * i];
  double y1 = c->git[si][2 * i + 1] * B + c->rel[si][2 * i + 1];
  double x2 = c->git[sj][2 * j] * B + c->rel[sj][2 * j];
  double y2 = c->git[sj][2 * j + 1] * B + c->rel[sj][2 * j + 1];
  double dx = x1 - x2;
  double dy = y1 - y2;
  if (dx * dx + dy * dy > a2) {
    if ((dx - L) * (dx - L) < dx * dx)
      x2 += L;
    else if ((dx + L) * (dx + L) < dx * dx)
      x2 -= L;
    dx = x1 - x2;
    if ((dy - L) * (dy - L) < dy * dy)
      y2 += L;
    else if ((dy + L) * (dy + L) < dy * dy)
      y2 -= L;
    dy = y1 - y2;
  }
  *pdx = dx;
  *pdy = dy;
}

/* berechne_WCA11 (dynamik_methoden.cpp:617-702) */
void bdo_berechne_WCA11(bdo_ctx* c) {
  double* F = c->F_WCA[0];
  for (int i = 0; i < c->N1; i++) F[2 * i] = F[2 * i + 1] = 0.0;
  if (c->p.idgas_only) return;
  const double cut = c->zweihoch1_6 * c->zweihoch1_6;
  for (int i = 0; i < c->N1; i++) {
    const ilist* l = &c->erw[0][c->git[0][2 * i] * c->C + c->git[0][2 * i + 1]];
    for (int q = 0; q < l->n; q++) {
      const int j = l->v[q];
      if (i == j) continue;
      double a2 = abstand2(c, 0, i, 0, j);
      if (a2 > cut) continue;
      double dx, dy;
      pair_delta(c, 0, i, 0, j, a2, &dx, &dy);
      double a_8 = 1.0 / (a2 * a2 * a2 * a2);
      double a_14 = 1.0 / (a2 * a2 * a2 * a2 * a2 * a2 * a2);
      double abs_F = 4.0 * 6.0 * (2.0 * a_14 - a_8);
      if (abs_F > c->p.maxPairWCA) abs_F = c->p.maxPairWCA;
      F[2 * i] += abs_F * dx;
      F[2 * i + 1] += abs_F * dy;
    }
  }
}

/* berechne_WCA22 (dynamik_methoden.cpp:790-879) */
void bdo_berechne_WCA22(bdo_ctx* c) {
  double* F = c->F_WCA[1];
  for (int i = 0; i < c->N2; i++) F[2 * i] = F[2 * i + 1] = 0.0;
  if (c->p.idgas_only) return;
  const double cut = c->zweihoch1_6 * c->zweihoch1_6;
  const double s = c->p.sigma11_22;
  for (int i = 0; i < c->N2; i++) {
    const ilist* l = &c->erw[1][c->git[1][2 * i] * c->C + c->git[1][2 * i + 1]];
    for (int q = 0; q < l->n; q++) {
      const int j = l->v[q];
      if (i == j) continue;
      double a2 = abstand2(c, 1, i, 1, j);
      if (a2 * s * s > cut) continue;
      double dx, dy;
      pair_delta(c, 1, i, 1, j, a2, &dx, &dy);
      a2 *= s * s;
      dx *= s;
      dy *= s;
      double a_8 = 1.0 / (a2 * a2 * a2 * a2);
      double a_14 = 1.0 / (a2 * a2 * a2 * a2 * a2 * a2 * a2);
      double abs_F = c->p.eps22_11 * s * 4.0 * 6.0 * (2.0 * a_14 - a_8);
      if (abs_F > c->p.maxPairWCA) abs_F = c->p.maxPairWCA;
      F[2 * i] += abs_F * dx;
      F[2 * i + 1] += abs_F * dy;
    }
  }
}

/* addiere_WCA12 (dynamik_methoden.cpp:973-1059) */
void bdo_addiere_WCA12(bdo_ctx* c) {
  if (c->p.idgas_only) return;
  double* F1 = c->F_WCA[0];
  double* F2 = c->F_WCA[1];
  const double cut = c->zweihoch1_6 * c->zweihoch1_6;
  const double s = c->p.sigma11_12;
  for (int i = 0; i < c->N1; i++) {
    const ilist* l = &c->erw[1][c->git[0][2 * i] * c->C + c->git[0][2 * i + 1]];
    for (int q = 0; q < l->n; q++) {
      const int j2 = l->v[q];
      double a2 = abstand2(c, 0, i, 1, j2);
      if (a2 * s * s > cut) continue;
      double dx, dy;
      pair_delta(c, 0, i, 1, j2, a2, &dx, &dy);
      a2 *= s * s;
      dx *= s;
      dy *= s;
      double a_8 = 1.0 / (a2 * a2 * a2 * a2);
      double a_14 = 1.0 / (a2 * a2 * a2 * a2 * a2 * a2 * a2);
      double abs_F = c->p.eps12_11 * s * 4.0 * 6.0 * (2.0 * a_14 - a_8);
      if (abs_F > c->p.maxPairWCA) abs_F = c->p.maxPairWCA;
      F1[2 * i] += abs_F * dx;
      F1[2 * i + 1] += abs_F * dy;
      F2[2 * j2] -= abs_F * dx;
      F2[2 * j2 + 1] -= abs_F * dy;
    }
  }
}

/* ------------------------------------------------------------------ */
/* G (dynamik_methoden.cpp:1384-1394) */
static double Gfun(const bdo_ctx* c, int j, int k) {
  const int Z = c->Z;
  const double dx = c->dx, dq = c->dq;
  double qx = dq * (((int)(j + Z * 0.5)) % Z - 0.5 * Z);
  double qy = dq * (((int)(k + Z * 0.5)) % Z - 0.5 * Z);
  if (j == 0 && k == 0 && c->p.lambda_kapillar > 0.2 * c->p.L) return 0.0;
  return 1.0 / (4 * sin(0.5 * qx * dx) * sin(0.5 * qx * dx) / dx / dx +
                4 * sin(0.5 * qy * dx) * sin(0.5 * qy * dx) / dx / dx +
                1.0 / (c->p.lambda_kapillar * c->p.lambda_kapillar));
}

/* kapkraefte_init (dynamik_methoden.cpp:529-613) */
void bdo_kapkraefte_init(bdo_ctx* c) {
  const int Z = c->Z;
  if (!c->rhox) {
    size_t bytes = sizeof(fftw_complex) * (size_t)Z * Z;
    c->rhox = (fftw_complex*)fftw_malloc(bytes);
    c->rhok = (fftw_complex*)fftw_malloc(bytes);
    c->Fxk = (fftw_complex*)fftw_malloc(bytes);
    c->Fyk = (fftw_complex*)fftw_malloc(bytes);
    c->Fx = (fftw_complex*)fftw_malloc(bytes);
    c->Fy = (fftw_complex*)fftw_malloc(bytes);
    memset(c->rhox, 0, bytes);
    c->sinxG = (double*)malloc(sizeof(double) * (size_t)Z * Z);
    c->sinyG = (double*)malloc(sizeof(double) * (size_t)Z * Z);
    const double dq = c->dq, dx = c->dx, kap = c->p.kapillar_vorfaktor;
    for (int j = 0; j < Z; j++)
      for (int k = 0; k < Z; k++) {
        double q = dq * ((j + (int)(Z * 0.5)) % Z - 0.5 * Z);
        c->sinxG[j * Z + k] = kap * sin(q * dx) / dx * Gfun(c, j, k) / Z / Z;
        q = dq * ((k + (int)(Z * 0.5)) % Z - 0.5 * Z);
        c->sinyG[j * Z + k] = kap * sin(q * dx) / dx * Gfun(c, j, k) / Z / Z;
      }
    c->fwd = fftw_plan_dft_2d(Z, Z, c->rhox, c->rhok, FFTW_FORWARD, FFTW_ESTIMATE);
    c->bx = fftw_plan_dft_2d(Z, Z, c->Fxk, c->Fx, FFTW_BACKWARD, FFTW_ESTIMATE);
    c->by = fftw_plan_dft_2d(Z, Z, c->Fyk, c->Fy, FFTW_BACKWARD, FFTW_ESTIMATE);
  }
}

/* grid weights shared by the assignment and interpolation routines */
typedef struct {
  int k, kl, kr, l, ll, lr;
  double xl, xe, xr, yl, ye, yr;
} stencil;

static void stencil_cic(bdo_ctx* c, double x, double y, stencil* s) {
  const int Z = c->Z;
  const double dx = c->dx;
  s->k = (int)(x / dx);
  s->kl = (s->k - 1 + Z) % Z;
  s->kr = (s->k + 1) % Z;
  s->l = (int)(y / dx);
  s->ll = (s->l - 1 + Z) % Z;
  s->lr = (s->l + 1) % Z;
  double tmp = x / dx - (s->k + 0.5);
  s->xe = 1.0 - fabs(tmp);
  if (tmp < 0.0) {
    s->xl = -tmp;
    s->xr = 0.0;
  } else {
    s->xl = 0.0;
    s->xr = tmp;
  }
  tmp = y / dx - (s->l + 0.5);
  s->ye = 1.0 - fabs(tmp);
  if (tmp < 0.0) {
    s->yl = -tmp;
    s->yr = 0.0;
  } else {
    s->yl = 0.0;
    s->yr = tmp;
  }
}

static void stencil_tsc(bdo_ctx* c, double x, double y, stencil* s) {
  const int Z = c->Z;
  const double dx = c->dx;
  s->k = (int)(x / dx);
  s->kl = (s->k - 1 + Z) % Z;
  s->kr = (s->k + 1) % Z;
  s->l = (int)(y / dx);
  s->ll = (s->l - 1 + Z) % Z;
  s->lr = (s->l + 1) % Z;
  double d = x - (s->k + 0.5) * dx;
  s->xe = 0.75 - d * d / dx / dx;
  double tmp = fabs((d + dx) / dx);
  s->xl = 0.5 * (1.5 - tmp) * (1.5 - tmp);
  tmp = fabs((d - dx) / dx);
  s->xr = 0.5 * (1.5 - tmp) * (1.5 - tmp);
  d = y - (s->l + 0.5) * dx;
  s->ye = 0.75 - d * d / dx / dx;
  tmp = fabs((d + dx) / dx);
  s->yl = 0.5 * (1.5 - tmp) * (1.5 - tmp);
  tmp = fabs((d - dx) / dx);
  s->yr = 0.5 * (1.5 - tmp) * (1.5 - tmp);
}

/* gridDensity_NGP/CIC/TSC (gridRoutinen.cpp:31-76,131-280,412-547) */
void bdo_gridDensity(bdo_ctx* c, int schema) {
  const int Z = c->Z;
  const double B = c->B, drho = c->drho, f2 = c->p.f2_f1;
  for (int k = 0; k < Z * Z; k++) c->rhox[k][0] = 0.0;
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++) {
    if (s == 1 && c->N2 == 0) return;
    for (int i = 0; i < Ns[s]; i++) {
      double x = c->git[s][2 * i] * B + c->rel[s][2 * i];
      double y = c->git[s][2 * i + 1] * B + c->rel[s][2 * i + 1];
      if (schema == 0) {
        int k = (int)(x / c->dx);
        int l = (int)(y / c->dx);
        if (s == 0)
          c->rhox[iw(c, k, l)][0] += drho;
        else
          c->rhox[iw(c, k, l)][0] += drho * f2;
        continue;
      }
      stencil st;
      if (schema == 1)
        stencil_cic(c, x, y, &st);
      else
        stencil_tsc(c, x, y, &st);
      const int ks[3] = {st.kl, st.k, st.kr};
      const int ls[3] = {st.ll, st.l, st.lr};
      const double wx[3] = {st.xl, st.xe, st.xr};
      const double wy[3] = {st.yl, st.ye, st.yr};
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          if (s == 0)
            c->rhox[iw(c, ks[a], ls[b])][0] += wx[a] * wy[b] * drho;
          else
            c->rhox[iw(c, ks[a], ls[b])][0] += wx[a] * wy[b] * drho * f2;
        }
    }
  }
}

/* inv_gridDensity_NGP/CIC/TSC (gridRoutinen.cpp:81-126,284-407,551-668) */
void bdo_inv_gridDensity(bdo_ctx* c, int schema) {
  const double B = c->B, f2 = c->p.f2_f1;
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++) {
    double* F = c->Fkap[s];
    for (int i = 0; i < Ns[s]; i++) F[2 * i] = F[2 * i + 1] = 0.0;
  }
  for (int s = 0; s < 2; s++) {
    if (s == 1 && c->N2 == 0) return;
    double* F = c->Fkap[s];
    for (int i = 0; i < Ns[s]; i++) {
      double x = c->git[s][2 * i] * B + c->rel[s][2 * i];
      double y = c->git[s][2 * i + 1] * B + c->rel[s][2 * i + 1];
      if (schema == 0) {
        int k = (int)(x / c->dx);
        int l = (int)(y / c->dx);
        int g = iw(c, k, l);
        if (s == 0) {
          F[2 * i] = c->Fx[g][0];
          F[2 * i + 1] = c->Fy[g][0];
        } else {
          /* reference reads the imaginary part of Fx here (gridRoutinen.cpp:123) */
          F[2 * i] = f2 * c->Fx[g][0];
          F[2 * i + 1] = f2 * c->Fx[g][1];
        }
        continue;
      }
      stencil st;
      if (schema == 1)
        stencil_cic(c, x, y, &st);
      else
        stencil_tsc(c, x, y, &st);
      fftw_complex* Fx = c->Fx;
      fftw_complex* Fy = c->Fy;
#define FX(a, b) Fx[iw(c, a, b)][0]
#define FY(a, b) Fy[iw(c, a, b)][0]
      F[2 * i] = st.xl * (st.yl * FX(st.kl, st.ll) + st.ye * FX(st.kl, st.l) + st.yr * FX(st.kl, st.lr));
      F[2 * i + 1] = st.xl * (st.yl * FY(st.kl, st.ll) + st.ye * FY(st.kl, st.l) + st.yr * FY(st.kl, st.lr));
      F[2 * i] += st.xe * (st.yl * FX(st.k, st.ll) + st.ye * FX(st.k, st.l) + st.yr * FX(st.k, st.lr));
      F[2 * i + 1] += st.xe * (st.yl * FY(st.k, st.ll) + st.ye * FY(st.k, st.l) + st.yr * FY(st.k, st.lr));
      F[2 * i] += st.xr * (st.yl * FX(st.kr, st.ll) + st.ye * FX(st.kr, st.l) + st.yr * FX(st.kr, st.lr));
      F[2 * i + 1] += st.xr * (st.yl * FY(st.kr, st.ll) + st.ye * FY(st.kr, st.l) + st.yr * FY(st.kr, st.lr));
#undef FX
#undef FY
      if (s == 1) {
        F[2 * i] *= f2;
        F[2 * i + 1] *= f2;
      }
    }
  }
}

/* berechne_kapkraefte (dynamik_methoden.cpp:1180-1233) */
void bdo_berechne_kapkraefte(bdo_ctx* c) {
  const int Ns[2] = {c->N1, c->N2};
  if (c->p.idgas_only) {
    for (int s = 0; s < 2; s++)
      for (int i = 0; i < Ns[s]; i++) c->Fkap[s][2 * i] = c->Fkap[s][2 * i + 1] = 0.0;
    return;
  }
  bdo_gridDensity(c, c->p.densGrid_Schema);
  fftw_execute(c->fwd);
  const int ZZ = c->Z * c->Z;
  for (int j = 0; j < ZZ; j++) {
    c->Fxk[j][0] = -c->sinxG[j] * c->rhok[j][1];
    c->Fxk[j][1] = c->sinxG[j] * c->rhok[j][0];
    c->Fyk[j][0] = -c->sinyG[j] * c->rhok[j][1];
    c->Fyk[j][1] = c->sinyG[j] * c->rhok[j][0];
  }
  fftw_execute(c->bx);
  fftw_execute(c->by);
  bdo_inv_gridDensity(c, c->p.densGrid_Schema);
}

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC11). */
void bdo_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* One particle's noise, drawn as the CUDA library draws it: counter
 * (particle index over both species, step lo, step hi, attempt), key = seed.
 * Disk mode: 23-bit integers a, b per candidate; t = 2a + 1 - 2^23;
 * accept if ta^2 + tb^2 <= 2^46 (the disk of radius sqrt 5 in units of
 * sqrt 5); xi = sqrt(5) * t * 2^-23; the matching reference uniform is
 * u = (2a + 1) * 2^-24.
 * Gauss mode: Box-Muller on u1 = (r0>>8 + 1) 2^-24, u2 = (r1>>8) 2^-24. */
static void philox_particle(uint64_t seed, uint64_t step, uint32_t pid, int gauss, double* xi,
                            double* u) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  if (gauss) {
    uint32_t ctr[4] = {pid, (uint32_t)step, (uint32_t)(step >> 32), 0u};
    uint32_t r[4];
    bdo_philox4x32_10(ctr, key, r);
    double u1 = ((double)(r[0] >> 8) + 1.0) * 0x1p-24;
    double u2 = (double)(r[1] >> 8) * 0x1p-24;
    double rad = sqrt(-2.0 * log(u1));
    xi[0] = rad * cos(2.0 * M_PI * u2);
    xi[1] = rad * sin(2.0 * M_PI * u2);
    return;
  }
  for (uint32_t att = 0;; att++) {
    uint32_t ctr[4] = {pid, (uint32_t)step, (uint32_t)(step >> 32), att};
    uint32_t r[4];
    bdo_philox4x32_10(ctr, key, r);
    for (int h = 0; h < 2; h++) {
      int64_t a = r[2 * h] >> 9, b = r[2 * h + 1] >> 9;
      int64_t ta = 2 * a + 1 - (1 << 23), tb = 2 * b + 1 - (1 << 23);
      if (ta * ta + tb * tb <= (int64_t)1 << 46) {
        const double w5 = sqrt(5.0);
        xi[0] = w5 * ((double)ta * 0x1p-23);
        xi[1] = w5 * ((double)tb * 0x1p-23);
        if (u) {
          u[0] = (double)(2 * a + 1) * 0x1p-24;
          u[1] = (double)(2 * b + 1) * 0x1p-24;
        }
        return;
      }
    }
  }
}

void bdo_philox_noise(uint64_t seed, uint64_t step, int N1, int N2, int gauss, double* xi,
                      double* u) {
  for (int p = 0; p < N1 + N2; p++)
    philox_particle(seed, step, (uint32_t)p, gauss, xi + 2 * p, u ? u + 2 * p : NULL);
}

/* berechne_zufallskraefte (dynamik_methoden.cpp:1317-1339) */
void bdo_berechne_zufallskraefte(bdo_ctx* c) {
  const int Ns[2] = {c->N1, c->N2};
  if (c->noise_mode == BDO_NOISE_PHILOX_DISK || c->noise_mode == BDO_NOISE_PHILOX_GAUSS) {
    const int gauss = c->noise_mode == BDO_NOISE_PHILOX_GAUSS;
    for (int s = 0; s < 2; s++)
      for (int i = 0; i < Ns[s]; i++)
        philox_particle(c->philox_seed, c->step, (uint32_t)(s == 0 ? i : c->N1 + i), gauss,
                        c->Fnoise[s] + 2 * i, NULL);
    return;
  }
  if (c->noise_mode == BDO_NOISE_NONE) {
    for (int s = 0; s < 2; s++)
      for (int i = 0; i < Ns[s]; i++) c->Fnoise[s][2 * i] = c->Fnoise[s][2 * i + 1] = 0.0;
    return;
  }
  const double wurzelfuenf = sqrt(5.0);
  for (int s = 0; s < 2; s++)
    for (int i = 0; i < Ns[s]; i++) {
      double x, y;
      do {
        x = wurzelfuenf * vonbis(c, -1.0, 1.0);
        y = wurzelfuenf * vonbis(c, -1.0, 1.0);
      } while (x * x + y * y > 5.0);
      c->Fnoise[s][2 * i] = x;
      c->Fnoise[s][2 * i + 1] = y;
    }
}

/* optimaler_zeitschritt (dynamik_methoden.cpp:1420-1491) */
double bdo_optimaler_zeitschritt(bdo_ctx* c) {
  double ret = c->p.dt_max;
  const double mrd = c->p.max_reisedistanz;
  const double T = c->p.T;
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++)
    for (int t = 0; t < Ns[s]; t++)
      for (int d = 0; d < 2; d++) {
        double F = c->F_WCA[s][2 * t + d] + c->Fkap[s][2 * t + d];
        double nz = c->Fnoise[s][2 * t + d];
        double v;
        if (fabs(F) < 1.0e-5) {
          v = mrd * mrd / (2.0 * T * nz * nz);
        } else {
          double u = nz * sqrt(0.5 * T) / F;
          double w = sqrt(u * u + mrd / fabs(F));
          v = (w - fabs(u)) * (w - fabs(u));
        }
        ret = (v < ret) ? v : ret; /* std::min(ret, v) */
      }
  return ret;
}

/* zeitschritt (dynamik_methoden.cpp:74-163) */
double bdo_zeitschritt(bdo_ctx* c, double tmax) {
  if (tmax <= 0.0) return 1.0e10;
  bdo_berechne_WCA11(c);
  bdo_berechne_WCA22(c);
  bdo_addiere_WCA12(c);
  bdo_berechne_kapkraefte(c);
  if (!c->p.noWCA)
    bdo_berechne_zufallskraefte(c);
  else
    for (int s = 0; s < 2; s++) {
      const int n = s == 0 ? c->N1 : c->N2;
      for (int i = 0; i < n; i++) c->Fnoise[s][2 * i] = c->Fnoise[s][2 * i + 1] = 0.0;
    }
  const double deltat = bdo_optimaler_zeitschritt(c);
  const double T = c->p.T, B = c->B, L = c->p.L;
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? c->N1 : c->N2;
    for (int t = 0; t < n; t++) {
      double* Fw = c->F_WCA[s] + 2 * t;
      double* Fk = c->Fkap[s] + 2 * t;
      double* Fn = c->Fnoise[s] + 2 * t;
      double ddx = deltat * (Fw[0] + Fk[0]) + sqrt(2.0 * T * deltat) * Fn[0];
      double ddy = deltat * (Fw[1] + Fk[1]) + sqrt(2.0 * T * deltat) * Fn[1];
      double* r = c->rel[s] + 2 * t;
      r[0] += ddx;
      r[1] += ddy;
      if (s == 1 && c->p.restrictRadial) {
        const double mitte = 0.5 * L;
        const int32_t* g = c->git[1] + 2 * t;
        double x = g[0] * B + r[0];
        double y = g[1] * B + r[1];
        double dxm = mitte - x;
        double dym = mitte - y;
        double abst = sqrt(dxm * dxm + dym * dym);
        double x_soll = mitte + abst * cos(2 * M_PI * (int)t / c->N2);
        double y_soll = mitte + abst * sin(2 * M_PI * (int)t / c->N2);
        r[0] += (x_soll - x);
        r[1] += (y_soll - y);
      }
    }
  }
  bdo_refresh_erwNachbar(c);
  c->step++;
  return deltat;
}

/* A step of length optimaler_zeitschritt(mrd) (dynamik_methoden.cpp:
 * 1495-1560: the travel bound mrd in place of max_reisedistanz), otherwise
 * zeitschritt; the device's zeitschritt_debug step. */
double bdo_zeitschritt_mrd(bdo_ctx* c, double mrd) {
  const double keep = c->p.max_reisedistanz;
  c->p.max_reisedistanz = mrd;
  const double dt = bdo_zeitschritt(c, 1.0);
  c->p.max_reisedistanz = keep;
  return dt;
}

double bdo_zeitschritte(bdo_ctx* c, int n) {
  double t = 0.0;
  for (int i = 0; i < n; i++) t += bdo_zeitschritt(c, 1.0);
  return t;
}

void bdo_get_forces(const bdo_ctx* c, int kind, int species, double* out) {
  const int n = species == 0 ? c->N1 : c->N2;
  const double* src = kind == 0 ? c->F_WCA[species] : kind == 1 ? c->Fkap[species] : c->Fnoise[species];
  memcpy(out, src, sizeof(double) * 2 * (size_t)n);
}

void bdo_get_grid(const bdo_ctx* c, int which, double* out) {
  const int ZZ = c->Z * c->Z;
  for (int k = 0; k < ZZ; k++) {
    switch (which) {
      case 0: out[k] = c->rhox[k][0]; break;
      case 1: out[k] = c->Fx[k][0]; break;
      case 2: out[k] = c->Fy[k][0]; break;
      default: out[k] = c->Fx[k][1]; break;
    }
  }
}

int bdo_get_list(const bdo_ctx* c, int species, int i, int j, int32_t* out, int cap) {
  const ilist* l = &c->erw[species][i * c->C + j];
  int n = l->n < cap ? l->n : cap;
  if (out && n > 0) memcpy(out, l->v, sizeof(int32_t) * n);
  return l->n;
}

long bdo_oob_count(const bdo_ctx* c) { return c->oob; }

void bdo_set_noise(bdo_ctx* c, int mode, uint64_t seed) {
  c->noise_mode = mode;
  if (mode == BDO_NOISE_REF_STREAM) mt64_seed(&c->gen, seed);
  c->philox_seed = seed;
}

void bdo_inject_uniforms(bdo_ctx* c, const double* u, size_t n) {
  c->noise_mode = BDO_NOISE_INJECTED;
  c->inj = u;
  c->inj_n = n;
  c->inj_pos = 0;
}

void bdo_set_step(bdo_ctx* c, uint64_t step) { c->step = step; }
uint64_t bdo_get_step(const bdo_ctx* c) { return c->step; }

/* obs_init header (auswertung.cpp:52-75) and schreibe_pos (:631-648) */
int bdo_schreibe_pos(const bdo_ctx* c, const char* path1, const char* path2, int nr,
                     int write_header) {
  const char* paths[2] = {path1, path2};
  const int Ns[2] = {c->N1, c->N2};
  for (int s = 0; s < 2; s++) {
    if (s == 1 && c->N2 == 0) break;
    FILE* f = fopen(paths[s], write_header ? "w" : "a");
    if (!f) return -1;
    if (write_header) fprintf(f, "# Format: t TAB x TAB y \n\n");
    for (int i = 0; i < Ns[s]; i++) {
      double x = c->rel[s][2 * i] + c->B * c->git[s][2 * i];
      double y = c->rel[s][2 * i + 1] + c->B * c->git[s][2 * i + 1];
      fprintf(f, "%g \t %g \t %g \n", nr * c->p.obs_dt, x, y);
    }
    fprintf(f, "\n");
    fclose(f);
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * Local densities of the offline analysis (main_auswertung.cpp:182-390).
 * snapgrid_num as parameter.h:174 computes it. */
int bdo_snapgrid_num(double L, double snapgrid_crude) {
  return 2 * (int)(L / (2 * snapgrid_crude) + 0.5);
}

/* TSC weights of one coordinate on the snapshot lattice
 * (main_auswertung.cpp:225-250): cell k = (int)(x/width) % n, its
 * neighbours, and the fractions in the left / centre / right cell. */
static void snap_tsc(double x, double width, int n, int* kk, double* wt) {
  int k = (int)(x / width);
  k = k % n;
  kk[0] = (k - 1 + n) % n;
  kk[1] = k;
  kk[2] = (k + 1) % n;
  const double d = x - (k + 0.5) * width;
  wt[1] = 0.75 - d * d / (width * width);
  double tmp = fabs((d + width) / width);
  wt[0] = 0.5 * (1.5 - tmp) * (1.5 - tmp);
  tmp = fabs((d - width) / width);
  wt[2] = 0.5 * (1.5 - tmp) * (1.5 - tmp);
}

/* Gridded densities (main_auswertung.cpp:184-300): every particle adds
 * w_x w_y drho (drho = 1/width^2) to nine cells, species 1 into g1 and
 * species 2 into g2, particles in order, cells in the reference's order
 * (left, centre, right along x, each over left, centre, right along y).
 * x1, x2: absolute positions double[N][2]; g1, g2: double[n*n], index
 * k*n + l with k along x. */
void bdo_lokale_dichte(int n, double width, int N1, const double* x1, int N2, const double* x2,
                       double* g1, double* g2) {
  const double drho = 1. / (width * width);
  for (int s = 0; s < 2; s++) {
    double* g = s == 0 ? g1 : g2;
    const double* x = s == 0 ? x1 : x2;
    const int N = s == 0 ? N1 : N2;
    for (int c = 0; c < n * n; c++) g[c] = 0.0;
    for (int i = 0; i < N; i++) {
      int kx[3], ky[3];
      double wx[3], wy[3];
      snap_tsc(x[2 * i], width, n, kx, wx);
      snap_tsc(x[2 * i + 1], width, n, ky, wy);
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) g[kx[a] * n + ky[b]] += wx[a] * wy[b] * drho;
    }
  }
}

/* Histogram bin as main_auswertung.cpp:337-355: (int) truncation of
 * v = value/drho - 0.5 (+ bins/2 for the difference), clamped to the range.
 * Values at or above `bins` are clamped before the conversion. */
static int snap_bin(double v, int bins) {
  if (v >= bins) return bins - 1;
  int b = (int)v;
  return b < 0 ? 0 : b;
}

/* Histograms and threshold counts (main_auswertung.cpp:302-390).
 * hist: int[4][bins] = rho1Hist, rho2Hist, rhoHist, drhoHist (counts, the
 * reference prints count / n^2); over: int[7] = cells with rho1+rho2 over
 * rho_thresh[0..2], then cells with |rho1-rho2|/(rho1+rho2) over
 * drho_thresh[0..3] (an empty cell gives 0/0 and is not counted). */
void bdo_rhohist(int n, const double* g1, const double* g2, int bins, double dbin,
                 const double* rho_thresh, const double* drho_thresh, int* hist, int* over) {
  for (int i = 0; i < 4 * bins; i++) hist[i] = 0;
  for (int i = 0; i < 7; i++) over[i] = 0;
  for (int c = 0; c < n * n; c++) {
    const double rho1 = g1[c], rho2 = g2[c];
    const double rho = rho1 + rho2, drho = rho1 - rho2;
    for (int t = 0; t < 3; t++)
      if (rho > rho_thresh[t]) over[t]++;
    for (int t = 0; t < 4; t++)
      if (fabs(drho) / rho > drho_thresh[t]) over[3 + t]++;
    hist[2 * bins + snap_bin(rho / dbin - 0.5, bins)]++;
    hist[0 * bins + snap_bin(rho1 / dbin - 0.5, bins)]++;
    hist[1 * bins + snap_bin(rho2 / dbin - 0.5, bins)]++;
    hist[3 * bins + snap_bin(drho / dbin - 0.5 + bins / 2, bins)]++;
  }
}

/*
 * FP64 implementation of the FFTW3-API subset declared in fftw3.h.
 * Test infrastructure: linked only by the oracle (bd_oracle.c) and by the
 * compiled reference checker under oracle/_ref. Never part of the product.
 *
 * Algorithm: self-sorting (Stockham) mixed-radix DFT. A length-n transform is
 * factored into radices 4, 2, 3, 5 and any remaining primes; pass q with
 * radix R and span Ns (product of earlier radices) maps
 *     v_r = in[j + r n/R] * w^(r (j mod Ns)),  w = exp(sign 2 pi i / (Ns R))
 *     out[(j div Ns) Ns R + (j mod Ns) + m Ns] = sum_r v_r exp(sign 2 pi i r m / R)
 * for j in [0, n/R). After the last pass the output is in natural order.
 * A 2D transform is rows (length n1) followed by columns (length n0), the
 * columns processed in blocks of 8 so each row segment read is contiguous.
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int n;
  int nstage;
  int radix[64];
  int span[64];
  double* tw[64]; /* tw[q][(k*(R-1) + r-1)*2 + {0,1}] */
  double* roots;  /* generic-radix roots, max radix */
  int maxr;
  int sign;
} plan1d;

struct fftw_plan_s {
  int n0, n1;
  fftw_complex* in;
  fftw_complex* out;
  plan1d row, col;
  double* work; /* scratch: max(n0, n1) * 8 complex * 2 buffers */
};

void* fftw_malloc(size_t n) {
  void* p = NULL;
  if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
  return p;
}

void fftw_free(void* p) { free(p); }

static void plan1d_init(plan1d* p, int n, int sign) {
  memset(p, 0, sizeof(*p));
  p->n = n;
  p->sign = sign;
  int m = n;
  int ns = 1;
  p->maxr = 1;
  while (m > 1) {
    int r;
    if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else if (m % 3 == 0) r = 3;
    else if (m % 5 == 0) r = 5;
    else {
      r = 7;
      while (m % r) r += 2;
      if (r > 64) abort(); /* radices above 64 are not supported by this shim */
    }
    int q = p->nstage++;
    p->radix[q] = r;
    p->span[q] = ns;
    p->tw[q] = (double*)malloc(sizeof(double) * 2 * (size_t)ns * (r > 1 ? r - 1 : 1));
    for (int k = 0; k < ns; k++)
      for (int rr = 1; rr < r; rr++) {
        double ang = sign * 2.0 * M_PI * (double)(rr * (long long)k) / (double)(ns * (long long)r);
        p->tw[q][((size_t)k * (r - 1) + rr - 1) * 2 + 0] = cos(ang);
        p->tw[q][((size_t)k * (r - 1) + rr - 1) * 2 + 1] = sin(ang);
      }
    if (r > p->maxr) p->maxr = r;
    ns *= r;
    m /= r;
  }
  if (p->maxr > 5) {
    p->roots = (double*)malloc(sizeof(double) * 2 * p->maxr * p->maxr);
  }
}

static void plan1d_free(plan1d* p) {
  for (int q = 0; q < p->nstage; q++) free(p->tw[q]);
  free(p->roots);
}

/* One length-n transform of `batch` interleaved sequences: element e of
 * sequence b sits at x[(e*batch + b)*2]. Result is written back into x. */
static void plan1d_exec(const plan1d* p, double* x, double* y, int batch) {
  const int n = p->n;
  double* a = x;
  double* b = y;
  for (int q = 0; q < p->nstage; q++) {
    const int R = p->radix[q];
    const int Ns = p->span[q];
    const int nR = n / R;
    const double* tw = p->tw[q];
    const double s = (double)p->sign;
    for (int j = 0; j < nR; j++) {
      const int k = j % Ns;
      const int idxD = (j / Ns) * Ns * R + k;
      for (int bb = 0; bb < batch; bb++) {
        double vr[64], vi[64];
        for (int r = 0; r < R; r++) {
          const double* src = a + ((size_t)(j + r * nR) * batch + bb) * 2;
          double re = src[0], im = src[1];
          if (r > 0) {
            const double c = tw[((size_t)k * (R - 1) + r - 1) * 2];
            const double sn = tw[((size_t)k * (R - 1) + r - 1) * 2 + 1];
            const double t = re * c - im * sn;
            im = re * sn + im * c;
            re = t;
          }
          vr[r] = re;
          vi[r] = im;
        }
        double orr[64], oi[64];
        if (R == 2) {
          orr[0] = vr[0] + vr[1]; oi[0] = vi[0] + vi[1];
          orr[1] = vr[0] - vr[1]; oi[1] = vi[0] - vi[1];
        } else if (R == 4) {
          const double s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
          const double d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
          const double s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
          const double d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
          orr[0] = s0r + s1r; oi[0] = s0i + s1i;
          orr[2] = s0r - s1r; oi[2] = s0i - s1i;
          /* V1 = d0 + s*i*d1, V3 = d0 - s*i*d1 */
          orr[1] = d0r - s * d1i; oi[1] = d0i + s * d1r;
          orr[3] = d0r + s * d1i; oi[3] = d0i - s * d1r;
        } else if (R == 3) {
          const double c = -0.5;
          const double sn = s * 0.86602540378443864676;
          const double t1r = vr[1] + vr[2], t1i = vi[1] + vi[2];
          const double t2r = vr[0] + c * t1r, t2i = vi[0] + c * t1i;
          const double t3r = sn * (vr[1] - vr[2]), t3i = sn * (vi[1] - vi[2]);
          orr[0] = vr[0] + t1r; oi[0] = vi[0] + t1i;
          orr[1] = t2r - t3i; oi[1] = t2i + t3r;
          orr[2] = t2r + t3i; oi[2] = t2i - t3r;
        } else {
          for (int m = 0; m < R; m++) {
            double accr = 0.0, acci = 0.0;
            for (int r = 0; r < R; r++) {
              const long long e = ((long long)r * m) % R;
              const double ang = s * 2.0 * M_PI * (double)e / (double)R;
              const double c = cos(ang), sn = sin(ang);
              accr += vr[r] * c - vi[r] * sn;
              acci += vr[r] * sn + vi[r] * c;
            }
            orr[m] = accr;
            oi[m] = acci;
          }
        }
        for (int m = 0; m < R; m++) {
          double* dst = b + ((size_t)(idxD + m * Ns) * batch + bb) * 2;
          dst[0] = orr[m];
          dst[1] = oi[m];
        }
      }
    }
    double* t = a;
    a = b;
    b = t;
  }
  if (a != x) memcpy(x, a, sizeof(double) * 2 * (size_t)n * batch);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags) {
  (void)flags;
  struct fftw_plan_s* p = (struct fftw_plan_s*)calloc(1, sizeof(*p));
  p->n0 = n0;
  p->n1 = n1;
  p->in = in;
  p->out = out;
  plan1d_init(&p->row, n1, sign);
  plan1d_init(&p->col, n0, sign);
  int mx = n0 > n1 ? n0 : n1;
  p->work = (double*)malloc(sizeof(double) * 2 * (size_t)mx * 8 * 2);
  return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags) {
  return fftw_plan_dft_2d(1, n, in, out, sign, flags);
}

void fftw_execute(const fftw_plan p) {
  const int n0 = p->n0, n1 = p->n1;
  double* out = (double*)p->out;
  if (p->out != p->in) memcpy(out, p->in, sizeof(fftw_complex) * (size_t)n0 * n1);
  double* w0 = p->work;
  double* w1 = p->work + 2 * (size_t)(n0 > n1 ? n0 : n1) * 8;
  /* rows */
  if (n1 > 1)
    for (int r = 0; r < n0; r++) {
      double* row = out + 2 * (size_t)r * n1;
      memcpy(w0, row, sizeof(double) * 2 * n1);
      plan1d_exec(&p->row, w0, w1, 1);
      memcpy(row, w0, sizeof(double) * 2 * n1);
    }
  /* columns, 8 at a time */
  if (n0 > 1)
    for (int c0 = 0; c0 < n1; c0 += 8) {
      const int nb = (n1 - c0) < 8 ? (n1 - c0) : 8;
      for (int r = 0; r < n0; r++)
        for (int b = 0; b < nb; b++) {
          w0[((size_t)r * nb + b) * 2] = out[((size_t)r * n1 + c0 + b) * 2];
          w0[((size_t)r * nb + b) * 2 + 1] = out[((size_t)r * n1 + c0 + b) * 2 + 1];
        }
      plan1d_exec(&p->col, w0, w1, nb);
      for (int r = 0; r < n0; r++)
        for (int b = 0; b < nb; b++) {
          out[((size_t)r * n1 + c0 + b) * 2] = w0[((size_t)r * nb + b) * 2];
          out[((size_t)r * n1 + c0 + b) * 2 + 1] = w0[((size_t)r * nb + b) * 2 + 1];
        }
    }
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  plan1d_free(&p->row);
  plan1d_free(&p->col);
  free(p->work);
  free(p);
}

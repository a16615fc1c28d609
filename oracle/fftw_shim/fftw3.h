/*
 * Minimal FFTW3-API shim (test infrastructure for the oracle only).
 *
 * FFTW3 is not installed in this image and the reference does not vendor or
 * pin it (reference Makefile:2 takes it from $FFTW_INC_DIR/$FFTW_LIB_DIR).
 * This header declares exactly the subset of the FFTW3 public interface the
 * reference calls (dynamik_methoden.cpp:554-607,1206,1221-1222;
 * auswertung.cpp:471-481,540), with FFTW's documented conventions:
 *   - fftw_complex is double[2] (re, im), row-major 2D arrays;
 *   - FFTW_FORWARD = -1 computes sum_x f(x) exp(-2 pi i k x / n),
 *     FFTW_BACKWARD = +1 uses exp(+2 pi i k x / n); neither is normalised.
 * The implementation (fftw_shim.c) is an FP64 mixed-radix Stockham FFT
 * written for this project. It is NOT the product: only the oracle and the
 * compiled reference checker link it.
 */
#ifndef BD_FFTW_SHIM_H
#define BD_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out,
                           int sign, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif

// Register-radix FFT for power-of-two lengths (the particle-mesh transforms
// of meshes with Z = 2^a).
//
// Stockham autosort formulation (Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC 2008): a pass of
// radix R over a length-N sequence with sub-transform length Ns takes
// butterfly j from elements j + t*N/R, multiplies element t by
// exp(sg*2*pi*i*(j mod Ns)*t/(Ns*R)), transforms the R values in registers
// and writes them to (j div Ns)*Ns*R + (j mod Ns) + t*Ns. Input and output
// are in natural order, so no permutation pass is needed anywhere.
//
// Twiddles of a butterfly: the powers w^(2^b) come from the table, every
// other power is a product of at most four of them (a few ulp in FP32).
//
// Every thread holds E elements per pass (E/R butterflies of radix R), E
// the schedule's largest radix (16, or 8 for lengths 32, 64 and 512 whose
// passes are all radix 8 or less; N below 16: E = N), so a sequence needs
// N/E threads and one pass is: read all elements into registers, barrier,
// compute, write in place, barrier. The passes use radix 16 where possible:
// 2048 = 16*16*8 takes three passes. Which butterflies a thread holds does
// not change any butterfly's arithmetic, so E does not change the results.
//
// Shared-memory layout: sequence b starts at s + b*ss, element e sits at
// pad16(e) = e + e/16 (one float2 of padding per 16), which keeps the
// strided accesses of every pass free of bank conflicts. Twiddles come from
// the run's table tw[m] = exp(-2*pi*i*m/Z) with Z = 2^lz >= N.
#pragma once

#include <cuda_runtime.h>

#include "bd_fft.cuh"

namespace bd {

__device__ __forceinline__ int pad16(int e) { return e + (e >> 4); }

// The pointer, opaque to the compiler: a kernel that loops over items
// launders its shared-memory base once per item, so the per-thread addresses
// of the passes are not hoisted out of the loop (which would keep hundreds
// of them live and spill).
template <class T>
__device__ __forceinline__ T* opaque(T* p) {
  asm volatile("" : "+l"(p));
  return p;
}
__host__ __device__ constexpr int fft2_stride(int n) { return n + (n >> 4) + 8; }

// Elements a thread holds in a length-2^logn transform: the radix of the
// schedule's first (largest) pass, 2^ceil(logn / ceil(logn / 4)) (Fft2Sched).
__host__ __device__ constexpr int fft2_e(int logn) {
  return logn < 4 ? (1 << logn) : (1 << ((logn + (logn + 3) / 4 - 1) / ((logn + 3) / 4)));
}
// threads one sequence of length 2^logn needs
__host__ __device__ constexpr int fft2_tps(int logn) { return (1 << logn) / fft2_e(logn); }

template <int R>
__device__ __forceinline__ void dftr(float2* v, float sg);

template <>
__device__ __forceinline__ void dftr<2>(float2* v, float) {
  const float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

// X[k] = sum_n v[n] w^(nk), w = exp(sg*2*pi*i/4) = sg*i
template <>
__device__ __forceinline__ void dftr<4>(float2* v, float sg) {
  const float2 s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
  const float2 s1 = cadd(v[1], v[3]), d1 = csub(v[1], v[3]);
  v[0] = cadd(s0, s1);
  v[2] = csub(s0, s1);
  v[1] = make_float2(d0.x - sg * d1.y, d0.y + sg * d1.x);
  v[3] = make_float2(d0.x + sg * d1.y, d0.y - sg * d1.x);
}

// 8 = 4 x 2: two length-4 transforms of the even and odd elements, then
// X[k] = E[k] + w8^k O[k], X[k+4] = E[k] - w8^k O[k].
template <>
__device__ __forceinline__ void dftr<8>(float2* v, float sg) {
  constexpr float c = 0.70710678118654752440f;  // sqrt(1/2)
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  dftr<4>(e, sg);
  dftr<4>(o, sg);
  // o[k] *= exp(sg*2*pi*i*k/8)
  o[1] = make_float2(c * (o[1].x - sg * o[1].y), c * (o[1].y + sg * o[1].x));
  o[2] = make_float2(-sg * o[2].y, sg * o[2].x);
  o[3] = make_float2(-c * (o[3].x + sg * o[3].y), c * (sg * o[3].x - o[3].y));
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

// 16 = 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2. Length-4 transforms over n1 for
// each n2, twiddle w16^(n2 k1), length-4 transforms over n2.
template <>
__device__ __forceinline__ void dftr<16>(float2* v, float sg) {
  constexpr float c1 = 0.92387953251128675613f;  // cos(pi/8)
  constexpr float s1 = 0.38268343236508977173f;  // sin(pi/8)
  constexpr float h = 0.70710678118654752440f;   // sqrt(1/2)
  float2 y[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    y[n2][0] = v[n2];
    y[n2][1] = v[n2 + 4];
    y[n2][2] = v[n2 + 8];
    y[n2][3] = v[n2 + 12];
    dftr<4>(y[n2], sg);
  }
  // w16^m = (cos(2 pi m/16), sg sin(2 pi m/16)) for m = n2*k1
  const float2 w1 = make_float2(c1, sg * s1), w2 = make_float2(h, sg * h);
  const float2 w3 = make_float2(s1, sg * c1), w6 = make_float2(-h, sg * h);
  const float2 w9 = make_float2(-c1, -sg * s1);
  y[1][1] = cmul(y[1][1], w1);
  y[1][2] = cmul(y[1][2], w2);
  y[1][3] = cmul(y[1][3], w3);
  y[2][1] = cmul(y[2][1], w2);
  y[2][2] = make_float2(-sg * y[2][2].y, sg * y[2][2].x);  // w16^4 = sg*i
  y[2][3] = cmul(y[2][3], w6);
  y[3][1] = cmul(y[3][1], w3);
  y[3][2] = cmul(y[3][2], w6);
  y[3][3] = cmul(y[3][3], w9);
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    float2 z[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
    dftr<4>(z, sg);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = z[k2];
  }
}

// One Stockham pass: radix 2^LOGR, sub-transform length 2^LOGNS, over nseq
// sequences of length 2^LOGN. Threads beyond nseq*N/E only join the barriers.
template <int LOGN, int LOGR, int LOGNS, bool TWS>
__device__ __forceinline__ void fft2_pass(float2* s, int ss, int nseq, const float2* __restrict__ tw,
                                          int lz, float sg) {
  constexpr int N = 1 << LOGN, R = 1 << LOGR;
  constexpr int E = fft2_e(LOGN);
  static_assert(E >= R && E % R == 0, "a thread holds whole butterflies");
  constexpr int TPS = N / E;  // threads per sequence
  constexpr int NB = E / R;   // butterflies per thread
  constexpr int NR = N / R;
  const int g = threadIdx.x;
  const int b = g / TPS, i = g - b * TPS;
  const bool act = b < nseq;
  float2* q = s + b * ss;
  float2 v[E];
  if (act) {
#pragma unroll
    for (int u = 0; u < NB; u++)
#pragma unroll
      for (int t = 0; t < R; t++) v[u * R + t] = q[pad16(u * TPS + i + t * NR)];
  }
  __syncthreads();
  if (act) {
#pragma unroll
    for (int u = 0; u < NB; u++) {
      const int j = u * TPS + i;
      const int k = j & ((1 << LOGNS) - 1);
      if (LOGNS > 0) {
        // w^t for t = 2^b from the table, the others as products of at
        // most four table values (w^t = w^(top bit of t) * w^(rest))
        const int sh = lz - LOGNS - LOGR;
        float2 w[R];
#pragma unroll
        for (int t = 1; t < R; t++) {
          if ((t & (t - 1)) == 0) {
            w[t] = TWS ? tw[(k * t) << sh] : __ldg(&tw[(k * t) << sh]);
            if (sg > 0.f) w[t].y = -w[t].y;
          } else {
            const int hb = 1 << (31 - __clz(t));
            w[t] = cmul(w[hb], w[t - hb]);
          }
          v[u * R + t] = cmul(v[u * R + t], w[t]);
        }
      }
      dftr<R>(&v[u * R], sg);
      const int d = ((j >> LOGNS) << (LOGNS + LOGR)) + k;
#pragma unroll
      for (int t = 0; t < R; t++) q[pad16(d + (t << LOGNS))] = v[u * R + t];
    }
  }
  __syncthreads();
}

// Pass schedule: ceil(remaining bits / 4) passes left, the bits spread evenly.
// TWS: the twiddle table tw is a copy in shared memory (kernels that loop
// over items keep it there; global-memory twiddle loads would be hoisted
// out of the loop by the compiler and exhaust the registers).
template <int LOGN, int DONE, bool TWS = false>
struct Fft2Sched {
  static __device__ __forceinline__ void run(float2* s, int ss, int nseq, const float2* tw, int lz,
                                             float sg) {
    constexpr int rem = LOGN - DONE;
    constexpr int left = (rem + 3) / 4;
    constexpr int bits = (rem + left - 1) / left;
    fft2_pass<LOGN, bits, DONE, TWS>(s, ss, nseq, tw, lz, sg);
    Fft2Sched<LOGN, DONE + bits, TWS>::run(s, ss, nseq, tw, lz, sg);
  }
};
template <int LOGN, bool TWS>
struct Fft2Sched<LOGN, LOGN, TWS> {
  static __device__ __forceinline__ void run(float2*, int, int, const float2*, int, float) {}
};

// Fft2Sched<LOGN, 0>::run transforms nseq sequences of length 2^LOGN in
// place (sg = -1 forward, +1 inverse, unnormalised) with nseq * N/E threads;
// the caller syncs before, the last pass ends with a barrier.

}  // namespace bd

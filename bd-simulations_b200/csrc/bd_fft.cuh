// Shared-memory FFT building blocks for the particle-mesh path.
//
// A CTA transforms `nseq` sequences of length n = 2^a 3^b that sit
// interleaved in shared memory: element e of sequence b is s[e*nseq + b]
// (nseq a power of two). Forward transforms use decimation in frequency
// (natural order in, digit-reversed order out), inverse transforms use
// decimation in time (digit-reversed order in, natural order out). A
// forward/inverse pair therefore needs no permutation pass: whatever acts
// between them (the Green's-function multiply) finds spectrum index k at
// position fft_pos(k).
//
// Stages use radix 4, 2 and 3 (FftPlan::r, in decimation-in-frequency
// order). Twiddles come from the run's table tw[t] = exp(-2 pi i t / Z); a
// length-n transform with n | Z reads it with stride Z/n.
#pragma once

#include <cuda_runtime.h>

namespace bd {

struct FftPlan {
  int n;
  int ns;
  int r[16];
  int pow2;    // every radix a power of two: block indices by shifts
  int lh[16];  // log2 of the butterfly span h = m/r of stage q (pow2 plans)
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// frequency k -> storage position after the forward (DIF) transform
__device__ __forceinline__ int fft_pos(const FftPlan& P, int k) {
  int m = P.n, pos = 0;
  for (int q = 0; q < P.ns; q++) {
    const int r = P.r[q];
    m /= r;
    pos += (k % r) * m;
    k /= r;
  }
  return pos;
}

// storage position -> frequency
__device__ __forceinline__ int fft_freq(const FftPlan& P, int pos) {
  int m = P.n, k = 0, mul = 1;
  for (int q = 0; q < P.ns; q++) {
    const int r = P.r[q];
    m /= r;
    k += ((pos / m) % r) * mul;
    mul *= r;
  }
  return k;
}

// in-register DFT of radix r (2, 3, 4); sg = -1 forward, +1 inverse
__device__ __forceinline__ void dft_small(float2* v, int r, float sg) {
  if (r == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (r == 4) {
    const float2 s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
    const float2 s1 = cadd(v[1], v[3]), d1 = csub(v[1], v[3]);
    v[0] = cadd(s0, s1);
    v[2] = csub(s0, s1);
    // V1 = d0 + sg*i*d1, V3 = d0 - sg*i*d1
    v[1] = make_float2(d0.x - sg * d1.y, d0.y + sg * d1.x);
    v[3] = make_float2(d0.x + sg * d1.y, d0.y - sg * d1.x);
  } else {  // 3
    const float sn = sg * 0.866025403784438646763723f;
    const float2 t1 = cadd(v[1], v[2]);
    const float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    const float2 t3 = make_float2(sn * (v[1].x - v[2].x), sn * (v[1].y - v[2].y));
    v[0] = cadd(v[0], t1);
    v[1] = make_float2(t2.x - t3.y, t2.y + t3.x);
    v[2] = make_float2(t2.x + t3.y, t2.y - t3.x);
  }
}

// Decimation-in-frequency stages. inv selects the sign (+1 when true).
// Caller syncs before; every stage ends with a sync.
__device__ inline void fft_dif(float2* s, const FftPlan& P, int lognseq, const float2* tw,
                               int twstride, bool inv) {
  const int n = P.n, nseq = 1 << lognseq;
  const float sg = inv ? 1.f : -1.f;
  int m = n;
  for (int q = 0; q < P.ns; q++) {
    const int r = P.r[q];
    const int h = m / r;
    const int tws = (n / m) * twstride;
    const int total = (n / r) << lognseq;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int b = idx & (nseq - 1);
      const int qq = idx >> lognseq;
      const int g = P.pow2 ? (qq >> P.lh[q]) : qq / h;
      const int e = qq - g * h;
      const int base = g * m + e;
      float2 v[4];
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (t < r) v[t] = s[((base + t * h) << lognseq) | b];
      dft_small(v, r, sg);
#pragma unroll
      for (int u = 1; u < 4; u++)
        if (u < r) {
          float2 w = __ldg(&tw[e * u * tws]);
          if (inv) w.y = -w.y;
          v[u] = cmul(v[u], w);
        }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (u < r) s[((base + u * h) << lognseq) | b] = v[u];
    }
    __syncthreads();
    m = h;
  }
}

// Decimation-in-time stages: the forward stages undone in reverse order.
__device__ inline void fft_dit(float2* s, const FftPlan& P, int lognseq, const float2* tw,
                               int twstride, bool inv) {
  const int n = P.n, nseq = 1 << lognseq;
  const float sg = inv ? 1.f : -1.f;
  int m = 1;
  for (int q = P.ns - 1; q >= 0; q--) {
    const int r = P.r[q];
    m *= r;  // block size of DIF stage q
    const int h = m / r;
    const int tws = (n / m) * twstride;
    const int total = (n / r) << lognseq;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int b = idx & (nseq - 1);
      const int qq = idx >> lognseq;
      const int g = P.pow2 ? (qq >> P.lh[q]) : qq / h;
      const int e = qq - g * h;
      const int base = g * m + e;
      float2 v[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (u < r) v[u] = s[((base + u * h) << lognseq) | b];
#pragma unroll
      for (int u = 1; u < 4; u++)
        if (u < r) {
          float2 w = __ldg(&tw[e * u * tws]);
          if (inv) w.y = -w.y;
          v[u] = cmul(v[u], w);
        }
      dft_small(v, r, sg);
#pragma unroll
      for (int t = 0; t < 4; t++)
        if (t < r) s[((base + t * h) << lognseq) | b] = v[t];
    }
    __syncthreads();
  }
}

}  // namespace bd

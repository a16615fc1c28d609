// Shared device-side definitions: per-run descriptors, particle records,
// Philox4x32-10, mesh stencils and the WCA pair law.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bd_fft.cuh"

namespace bd {

// Particle record, 16 bytes, kept sorted by (cell, pid):
//   ox, oy : in-cell offset (the reference's r?_rel, FP32 here)
//   cell   : linear cell index ic*C + jc (the reference's r?_git pair)
//   pid    : particle index over both species (species 2 starts at N1)
struct __align__(16) Rec {
  float ox, oy;
  int cell;
  int pid;
};

enum Scheme { NGP = 0, CIC = 1, TSC = 2 };
enum NoiseKind { NOISE_DISK = 0, NOISE_GAUSS = 1, NOISE_NONE = 2 };

enum RunFlags : int {
  F_IDGAS = 1,          // idgas_only: no WCA and no capillary force
  F_NOWCA = 2,          // noWCA: noise switched off (reference gates noise on it)
  F_RADIAL = 4,         // restrictRadial projection of species 2
  F_NGP_REFCOMPAT = 8,  // NGP species-2 y force from Im(Fx) (= 0), as the reference
  F_ADAPTIVE = 16,      // travel-bounded adaptive dt (optimaler_zeitschritt)
  F_SMALLBOX = 32,      // fewer than 7 cells per side: pair distances need the periodic wrap
};

// Error bits reported per run (RunDyn::err)
enum ErrBits : int {
  E_DEPOSIT_OVERFLOW = 1,  // staged particle set of a mesh tile exceeded capacity
  E_NONFINITE = 2,         // a particle position became NaN/Inf
  E_BARRIER_TIMEOUT = 4,   // a grid-wide barrier of the fused step gave up waiting
};

// Immutable per-run description (device copy in an array indexed by run).
struct RunDesc {
  int N1, N2, N;
  int C;        // cells per side (nachList_Zellen)
  int Z;        // mesh points per side (densGrid_Zellen)
  FftPlan plan_half;  // length Z/2 (row transform of the real density)
  FftPlan plan_full;  // length Z
  int scheme;
  int flags;
  int noise;
  float L, B, invB;
  float dx, invdx;
  float invC, z_over_L;  // mesh coordinate split
  // WCA: prefactors 24*eps*sigma, sigma, sigma^2 as the reference scales
  float wpre[3], wsig[3], wsig2[3];  // index 0: 11, 1: 22, 2: 12
  float cut2;                        // (2^(1/6))^2
  float maxPair;
  float q2;      // f2_f1
  float drho;    // 1/dx^2
  float T;
  float dt_max, mrd;
  double L_d, B_d, T_d, dt_max_d;
  unsigned long long seed;
  int fx_shift;  // fixed-point exponent of the deposit accumulator
  int wfx_shift; // fixed-point exponent of the WCA force sums
  // device memory owned by the run
  Rec* recA;        // sorted state
  Rec* recB;        // integrate output (old order); its cell is the sort key
  int* count;       // per cell count (C*C)
  int* start;       // per cell exclusive scan (C*C + 1)
  int* chunk_sum;   // per scan chunk: particles counted into its cells
  int* chunk_off;   // per scan chunk: exclusive prefix of chunk_sum
  float* rho;       // Z*Z, index k*Z + l (k = x index)
  float2* spec;     // Z*(Z/2) packed half spectrum after the row transform: power-of-two
                    // meshes by column (slot j of row k at j*Z + k), others by row (k*(Z/2) + j)
  float4* spec2;    // Z*(Z/2): (Fx'.re, Fx'.im, Fy'.re, Fy'.im)
  float2* H;        // Z*Z force grid (Fx, Fy)
  float* green;     // (Z/2+1)*Z, index ky*Z + kx: kapillar_vorfaktor*G/Z^2
  float* sxt;       // Z: sin(qx dx)/dx
  float* syt;       // Z/2+1: sin(qy dx)/dx
  float2* tw;       // Z: exp(-2 pi i t / Z)
  int* pos_full;    // Z: storage position of frequency k after a length-Z forward transform
  int* freq_full;   // Z: frequency held at storage position p
  int* pos_half;    // Z/2: the same for the length-Z/2 row transform
  float2* Fw;       // per pid: WCA force (drop-in routines)
  float2* Fk;       // per pid: capillary force
  float2* Fn;       // per pid: noise
  // Z*Z 64-bit fixed-point density sums of the fused and pipelined steps
  // (nullptr in the descriptions other kernels receive): the move deposits
  // the new positions, the next forward row pass consumes them and clears
  // the words
  unsigned long long* dacc;
};

// Mutable per-run state on the device.
struct RunDyn {
  unsigned long long step;  // Philox step counter
  long long steps_left;     // batched stepping stops a run at zero
  double t;                 // simulated time
  float dt;                 // time step used by the current step
  unsigned int dt_bits;     // min-reduction of the adaptive bound (float bits)
  int err;
  int sorting;  // set by the step's chunk scan: the run takes part in this sort
  int pad;
  int moved[2];       // particles of species 1, 2 that left their cell in this step
  int moved_last[2];  // the same for the last completed step
};

// ------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC11).
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
#ifdef __CUDA_ARCH__
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]);
#else
    const uint32_t hi0 = (uint32_t)(((uint64_t)0xD2511F53u * c[0]) >> 32);
    const uint32_t hi1 = (uint32_t)(((uint64_t)0xCD9E8D57u * c[2]) >> 32);
#endif
    const uint32_t lo0 = 0xD2511F53u * c[0];
    const uint32_t lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0;
    const uint32_t n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Noise vector of one particle for one step.
//  disk : uniform in the disk of radius sqrt(5) (the reference's noise,
//         dynamik_methoden.cpp:1317-1339), by rejection on 23-bit integers
//  gauss: N(0,1) per component by Box-Muller
__device__ __forceinline__ float2 particle_noise(int kind, unsigned long long seed,
                                        unsigned long long step, uint32_t pid) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  if (kind == NOISE_GAUSS) {
    uint32_t c[4] = {pid, (uint32_t)step, (uint32_t)(step >> 32), 0u};
    philox4x32_10(c, k0, k1);
    const float u1 = (float)((c[0] >> 8) + 1u) * 0x1p-24f;
    const float u2 = (float)(c[1] >> 8) * 0x1p-24f;
    const float rad = sqrtf(-2.0f * logf(u1));
    float s, co;
    sincospif(2.0f * u2, &s, &co);
    return make_float2(rad * co, rad * s);
  }
  if (kind == NOISE_DISK) {
    const float w5 = 2.2360679774997896964f;
    for (uint32_t att = 0; att < 64u; att++) {
      uint32_t c[4] = {pid, (uint32_t)step, (uint32_t)(step >> 32), att};
      philox4x32_10(c, k0, k1);
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const long long a = c[2 * h] >> 9, b = c[2 * h + 1] >> 9;
        const long long ta = 2 * a + 1 - (1LL << 23), tb = 2 * b + 1 - (1LL << 23);
        if (ta * ta + tb * tb <= (1LL << 46))
          return make_float2(w5 * ((float)ta * 0x1p-23f), w5 * ((float)tb * 0x1p-23f));
      }
    }
    return make_float2(0.f, 0.f);  // 2^-128 probability
  }
  return make_float2(0.f, 0.f);
}

// ------------------------------------------------------------------
// Mesh stencil of a particle. The mesh coordinate u = x/dx of
// x = ic*B + off is split exactly as u = ic*Z/C + off*Z/L: the integer part
// of ic*Z/C is taken in integer arithmetic so the FP32 fraction stays small
// and precise at any box size.
struct Stencil {
  int k, l;           // central mesh point (wrapped into [0, Z))
  float wx[3], wy[3];  // weights for k-1, k, k+1 (resp. l)
};

// q = num / C, r = num % C for 0 <= num < 2^24 through the FP32 reciprocal:
// num is exact in FP32 and the quotient estimate is off by at most one.
__device__ __forceinline__ int divmod_c(int num, int C, float invC, int& r) {
  int q = (int)((float)num * invC);
  r = num - q * C;
  if (r < 0) {
    q--;
    r += C;
  } else if (r >= C) {
    q++;
    r -= C;
  }
  return q;
}

// (ic, jc) of a linear cell index ic*C + jc
__device__ __forceinline__ void cell_ij(const RunDesc& R, int cell, int& ic, int& jc) {
  ic = divmod_c(cell, R.C, R.invC, jc);
}

__device__ __forceinline__ void mesh_axis(const RunDesc& R, int ic, float off, int& k, float& t) {
  const int num = ic * R.Z;
  int r;
  const int q = divmod_c(num, R.C, R.invC, r);
  const float f = (float)r * R.invC + off * R.z_over_L;
  const float fl = floorf(f);
  t = f - fl;
  if (t >= 1.0f) t = 0.0f, k = q + (int)fl + 1;
  else k = q + (int)fl;
  // the position lies in (-B, L + B]: k in (-Z, 2Z), one conditional wrap
  if (k < 0) k += R.Z;
  else if (k >= R.Z) k -= R.Z;
}

// weights as the reference's grid routines (gridRoutinen.cpp): NGP puts all
// weight on k; CIC: xexakt = 1-|d|, one neighbour gets |d|; TSC:
// 0.75-d^2 and 0.5(0.5 -+ d)^2, with d the offset from the cell centre in
// mesh units.
__device__ __forceinline__ void axis_weights(int scheme, float t, float w[3]) {
  const float d = t - 0.5f;
  if (scheme == CIC) {
    w[1] = 1.0f - fabsf(d);
    w[0] = d < 0.0f ? -d : 0.0f;
    w[2] = d < 0.0f ? 0.0f : d;
  } else if (scheme == TSC) {
    w[1] = 0.75f - d * d;
    const float a = 0.5f - d, b = 0.5f + d;
    w[0] = 0.5f * a * a;
    w[2] = 0.5f * b * b;
  } else {
    w[0] = 0.0f;
    w[1] = 1.0f;
    w[2] = 0.0f;
  }
}

__device__ inline void make_stencil(const RunDesc& R, const Rec& p, Stencil& s) {
  const int ic = p.cell / R.C, jc = p.cell - (p.cell / R.C) * R.C;
  float tx, ty;
  mesh_axis(R, ic, p.ox, s.k, tx);
  mesh_axis(R, jc, p.oy, s.l, ty);
  axis_weights(R.scheme, tx, s.wx);
  axis_weights(R.scheme, ty, s.wy);
}

// WCA pair force coefficient (dynamik_methoden.cpp:617-702,790-879,973-1059):
// with a2 and d scaled by sigma, abs_F = 24 eps sigma (2 a2^-7 - a2^-4),
// capped at maxPairWCA; force = abs_F * d. Written as pre*a^-4*(2a^-3-1) so
// that coincident particles give the cap rather than NaN.
__device__ inline float wca_coef(float a2s, float pre, float maxPair) {
  const float inv = 1.0f / a2s;
  const float i3 = inv * inv * inv;
  float f = pre * (i3 * inv) * (2.0f * i3 - 1.0f);
  return f > maxPair ? maxPair : f;
}

}  // namespace bd

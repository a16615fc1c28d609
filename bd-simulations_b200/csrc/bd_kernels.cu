// Device kernels of the force-and-integrate step.
//
// One step of every run in a batch is the launch sequence
//   deposit -> fft_rows_fwd -> fft_cols -> fft_rows_inv      (capillary mesh)
//   integrate                                                (WCA + mesh force
//                                                             + noise + update
//                                                             + re-binning)
//   scan_partial -> scan_final -> scatter -> fixup -> step_end (cell sort)
// Each kernel walks a list of work items (run, a, b, c) so that runs of
// different sizes share one launch. All reductions are order-independent or
// run in a fixed order, so results do not depend on scheduling.
#include <algorithm>
#include <cstdio>
#include <cuda/atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "bd_common.cuh"
#include "bd_fft.cuh"
#include "bd_fft2.cuh"
#include "bd_kernels.h"

namespace bd {

__device__ __forceinline__ int wrapi(int a, int m) {
  a %= m;
  return a < 0 ? a + m : a;
}

// a in (-m, 2m) into [0, m)
__device__ __forceinline__ int wrap1(int a, int m) {
  return a < 0 ? a + m : (a >= m ? a - m : a);
}

__device__ __forceinline__ bool run_active(const RunDyn* dyn, int run) {
  return dyn[run].steps_left > 0;
}

// Load of data that earlier kernels wrote: through the read-only cache when
// NC, or a plain (coherent) load where the same kernel also writes it (the
// fused step).
template <bool NC, class T>
__device__ __forceinline__ T ldm(const T* p) {
  if constexpr (NC) return __ldg(p);
  else return *p;
}

// Exclusive scan over the CTA (any multiple of 32 threads up to 1024);
// sh: 32 ints of shared scratch. All threads must call it.
__device__ inline int block_excl_scan(int v, int* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  const int base = w > 0 ? sh[w - 1] : 0;
  const int r = base + x - v;
  __syncthreads();
  return r;
}

// In-place exclusive scan of n counts stored with a stride: a[k*stride] ->
// out[k*stride + 1]; writes the total to out[n*stride]. All threads call it.
__device__ inline void block_scan_strided(const int* cnt, int* out, int n, int stride, int* tmp32) {
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int s0 = threadIdx.x * per;
  int loc = 0;
  for (int q = 0; q < per; q++)
    if (s0 + q < n) loc += cnt[(s0 + q) * stride];
  int ex = block_excl_scan(loc, tmp32);
  for (int q = 0; q < per; q++)
    if (s0 + q < n) {
      out[(s0 + q) * stride] = ex;
      ex += cnt[(s0 + q) * stride];
    }
  if (threadIdx.x == blockDim.x - 1) out[n * stride] = ex;
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Charge assignment (gridRoutinen.cpp:31-76, 131-280, 412-547).
// One CTA owns a MT x MT tile of mesh points and gathers every particle whose
// stencil can reach it (the cell rows covering the tile plus halo, located
// through the cell-sorted order). Contributions are rounded to fixed point
// (|value| <= 2^30 units of 2^-fx_shift) and accumulate in shared memory as
// 64-bit sums kept in two 32-bit words (fx_add), so the sum is exact and
// independent of the order in which threads add; the owner writes its tile
// once, without global atomics.

// 64-bit fixed-point add from 32-bit shared-memory atomics (much faster on
// this GPU than 64-bit ones): the carry out of the low word is read off the
// returned old value, so lo/hi always hold the exact sum modulo 2^64,
// whatever the order of the additions.
__device__ __forceinline__ void fx_add(unsigned* lo, unsigned* hi, int a, int v) {
  const unsigned u = (unsigned)v;
  const unsigned old = atomicAdd(&lo[a], u);
  const unsigned h = (unsigned)(v >> 31) + (old + u < old ? 1u : 0u);
  if (h) atomicAdd(&hi[a], h);
}

// Deposit of the MT x MT tile at mesh (x0, y0); smem holds the 2*MT*MT
// accumulator words and the segment table, s_tmp 32 ints. All threads call.
__device__ inline void deposit_tile(const RunDesc& R, int scheme, int x0, int y0, int MT, unsigned char* smem,
                                    int* s_tmp) {
  unsigned* acc_lo = (unsigned*)smem;
  unsigned* acc_hi = acc_lo + MT * MT;
  int* seg = (int*)(acc_hi + MT * MT);  // [nseg][3]: global begin, length, prefix
  for (int i = threadIdx.x; i < 2 * MT * MT; i += blockDim.x) acc_lo[i] = 0u;
  // cell rows/columns that can reach this tile: offsets lie in (-B, 2B]
  const float rB = R.dx * R.invB;
  int ilo = (int)floorf((x0 - 1) * rB) - 2, ihi = (int)floorf((x0 + MT + 1) * rB) + 1;
  int jlo = (int)floorf((y0 - 1) * rB) - 2, jhi = (int)floorf((y0 + MT + 1) * rB) + 1;
  if (ihi - ilo + 1 >= R.C) ilo = 0, ihi = R.C - 1;
  if (jhi - jlo + 1 >= R.C) jlo = 0, jhi = R.C - 1;
  const int ncx = ihi - ilo + 1;
  // per cell row at most two contiguous particle segments (periodic wrap)
  const int jl = wrapi(jlo, R.C);
  const int ncy = jhi - jlo + 1;
  const bool split = jl + ncy > R.C;
  const int nseg = ncx * (split ? 2 : 1);
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) {
    const int row = split ? s >> 1 : s;
    const int part = split ? (s & 1) : 0;
    const int ic = wrapi(ilo + row, R.C);
    int a, b;
    if (!split) {
      a = jl;
      b = jl + ncy;
    } else if (part == 0) {
      a = jl;
      b = R.C;
    } else {
      a = 0;
      b = jl + ncy - R.C;
    }
    const int gb = R.start[ic * R.C + a];
    const int ge = R.start[ic * R.C + b];
    seg[3 * s] = gb;
    seg[3 * s + 1] = ge - gb;
  }
  __syncthreads();
  block_scan_strided(seg + 1, seg + 2, nseg, 3, s_tmp);
  const int total = seg[3 * nseg + 2];
  const float scale = __int_as_float((127 + R.fx_shift) << 23);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (seg[3 * mid + 2] <= t) lo = mid;
      else hi = mid - 1;
    }
    const Rec p = R.recA[seg[3 * lo] + (t - seg[3 * lo + 2])];
    int ic, jc;
    cell_ij(R, p.cell, ic, jc);
    int k, l;
    float tx, ty;
    mesh_axis(R, ic, p.ox, k, tx);
    mesh_axis(R, jc, p.oy, l, ty);
    const float q = p.pid < R.N1 ? 1.0f : R.q2;
    if (scheme == NGP) {
      const int lk = wrap1(k - x0, R.Z), ll = wrap1(l - y0, R.Z);
      if (lk < MT && ll < MT) {
        float c = R.drho;
        if (p.pid >= R.N1) c *= q;
        fx_add(acc_lo, acc_hi, lk * MT + ll, __float2int_rn(c * scale));
      }
      continue;
    }
    float wx[3], wy[3];
    axis_weights(scheme, tx, wx);
    axis_weights(scheme, ty, wy);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int lk = wrap1(k + a - 1 - x0, R.Z);
      if (lk >= MT) continue;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        const int ll = wrap1(l + b - 1 - y0, R.Z);
        if (ll >= MT) continue;
        float c = wx[a] * wy[b] * R.drho;
        if (p.pid >= R.N1) c *= q;
        fx_add(acc_lo, acc_hi, lk * MT + ll, __float2int_rn(c * scale));
      }
    }
  }
  __syncthreads();
  const double inv = 1.0 / (double)scale;
  for (int i = threadIdx.x; i < MT * MT; i += blockDim.x) {
    const int lk = i / MT, ll = i - (i / MT) * MT;
    const long long acc = (long long)(((unsigned long long)acc_hi[i] << 32) | acc_lo[i]);
    R.rho[(size_t)(x0 + lk) * R.Z + y0 + ll] = (float)((double)acc * inv);
  }
  __syncthreads();
}

// The same contributions as deposit_tile, of one particle, added straight to
// the fused step's accumulator R.dacc with 64-bit integer atomics (mesh point
// k*Z + l); the integer sums, and so the density, are those of the tiles.
__device__ __forceinline__ void deposit_acc(const RunDesc& R, const Rec& p) {
  int ic, jc;
  cell_ij(R, p.cell, ic, jc);
  int k, l;
  float tx, ty;
  mesh_axis(R, ic, p.ox, k, tx);
  mesh_axis(R, jc, p.oy, l, ty);
  const float scale = __int_as_float((127 + R.fx_shift) << 23);
  const float q = p.pid < R.N1 ? 1.0f : R.q2;
  unsigned long long* acc = R.dacc;
  if (R.scheme == NGP) {
    float c = R.drho;
    if (p.pid >= R.N1) c *= q;
    atomicAdd(&acc[(size_t)k * R.Z + l], (unsigned long long)(long long)__float2int_rn(c * scale));
    return;
  }
  float wx[3], wy[3];
  axis_weights(R.scheme, tx, wx);
  axis_weights(R.scheme, ty, wy);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const size_t row = (size_t)wrap1(k + a - 1, R.Z) * R.Z;
#pragma unroll
    for (int b = 0; b < 3; b++) {
      float c = wx[a] * wy[b] * R.drho;
      if (p.pid >= R.N1) c *= q;
      atomicAdd(&acc[row + wrap1(l + b - 1, R.Z)], (unsigned long long)(long long)__float2int_rn(c * scale));
    }
  }
}

__global__ void __launch_bounds__(256) k_deposit(const RunDesc* __restrict__ runs,
                                                 const RunDyn* __restrict__ dyn,
                                                 const Item* __restrict__ items, int nitems,
                                                 int scheme_override, int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_tmp[32];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    if (require_active && !run_active(dyn, I.run)) continue;
    const RunDesc& R = runs[I.run];
    const int scheme = scheme_override >= 0 ? scheme_override : R.scheme;
    const int MT = I.c;
    deposit_tile(R, scheme, I.a * MT, I.b * MT, MT, smem, s_tmp);
  }
}

// ---------------------------------------------------------------------------
// Row pass, forward: each mesh row (fixed x index k) is real; it is packed as
// Z/2 complex values z[m] = rho[2m] + i rho[2m+1], transformed, and unpacked
// into the half spectrum X[j], j in [0, Z/2]. The two purely real bins j = 0
// and j = Z/2 share slot 0 as (X[0], X[Z/2]).
__global__ void __launch_bounds__(FFT_THREADS) k_fft_rows_fwd(const RunDesc* __restrict__ runs,
                                                      const RunDyn* __restrict__ dyn,
                                                      const Item* __restrict__ items, int nitems,
                                                      int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* s = (float2*)smem;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    if (require_active && !run_active(dyn, I.run)) continue;
    const RunDesc& R = runs[I.run];
    const int Z = R.Z, n = Z >> 1;
    const int lr = I.c;  // log2(rows in this item)
    const int row0 = I.a;
    for (int i = threadIdx.x; i < (n << lr); i += blockDim.x) {
      const int b = i / n, m = i - b * n;
      const float2 v = *reinterpret_cast<const float2*>(&R.rho[(size_t)(row0 + b) * Z + 2 * m]);
      s[(m << lr) | b] = v;
    }
    __syncthreads();
    fft_dif(s, R.plan_half, lr, R.tw, 2, false);
    for (int i = threadIdx.x; i < (n << lr); i += blockDim.x) {
      const int b = i / n, j = i - b * n;
      const float2 zj = s[(__ldg(&R.pos_half[j]) << lr) | b];
      const float2 zc = s[(__ldg(&R.pos_half[j == 0 ? 0 : n - j]) << lr) | b];
      float2 out;
      if (j == 0) {
        out = make_float2(zj.x + zj.y, zj.x - zj.y);
      } else {
        // E = (zj + conj zc)/2, O = (zj - conj zc)/(2i), X = E + w^j O
        const float2 E = make_float2(0.5f * (zj.x + zc.x), 0.5f * (zj.y - zc.y));
        const float2 O = make_float2(0.5f * (zj.y + zc.y), -0.5f * (zj.x - zc.x));
        out = cadd(E, cmul(__ldg(&R.tw[j]), O));
      }
      R.spec[(size_t)(row0 + b) * n + j] = out;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Column pass: forward transform over x of W spectrum columns, multiply by
// i*sin(q dx)/dx*G(q) for both force components (dynamik_methoden.cpp:
// 1210-1216 with the tables of :585-593), inverse transform over x of both
// fields. Column 0 holds the packed real pair (ky = 0, ky = Z/2): its
// transform C = A + iB is split into A and B, each multiplied by its own
// Green's factor and packed again for the inverse.
__global__ void __launch_bounds__(FFT_THREADS) k_fft_cols(const RunDesc* __restrict__ runs,
                                                  const RunDyn* __restrict__ dyn,
                                                  const Item* __restrict__ items, int nitems,
                                                  int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    if (require_active && !run_active(dyn, I.run)) continue;
    const RunDesc& R = runs[I.run];
    const int Z = R.Z, n = Z >> 1;
    const int lw = I.c, W = 1 << lw;
    const int col0 = I.a;
    float2* sA = (float2*)smem;
    float2* sB = sA + ((size_t)Z << lw);
    for (int i = threadIdx.x; i < (Z << lw); i += blockDim.x) {
      const int k = i >> lw, c = i & (W - 1);
      sA[i] = R.spec[(size_t)k * n + col0 + c];
    }
    __syncthreads();
    fft_dif(sA, R.plan_full, lw, R.tw, 1, false);
    // columns other than the packed one: independent per element
    for (int i = threadIdx.x; i < (Z << lw); i += blockDim.x) {
      const int pos = i >> lw, c = i & (W - 1);
      const int j = col0 + c;
      if (j == 0) continue;
      const int kx = __ldg(&R.freq_full[pos]);
      const float g = __ldg(&R.green[(size_t)j * Z + kx]);
      const float gx = __ldg(&R.sxt[kx]) * g;
      const float gy = __ldg(&R.syt[j]) * g;
      const float2 v = sA[i];
      sA[i] = make_float2(-gx * v.y, gx * v.x);
      sB[i] = make_float2(-gy * v.y, gy * v.x);
    }
    if (col0 == 0) {
      // packed column: read partners before anyone overwrites column 0
      constexpr int MAXIT = 16;
      float2 P[MAXIT], Q[MAXIT];
      int cnt = 0;
      for (int pos = threadIdx.x; pos < Z && cnt < MAXIT; pos += blockDim.x, cnt++) {
        const int kx = __ldg(&R.freq_full[pos]);
        const int km = kx == 0 ? 0 : Z - kx;
        const float2 Cv = sA[pos << lw];
        const float2 Cm = sA[__ldg(&R.pos_full[km]) << lw];
        // A = (C + conj Cm)/2 ; B = (C - conj Cm)/(2i)
        const float2 A = make_float2(0.5f * (Cv.x + Cm.x), 0.5f * (Cv.y - Cm.y));
        const float2 Bv = make_float2(0.5f * (Cv.y + Cm.y), -0.5f * (Cv.x - Cm.x));
        const float gA = __ldg(&R.green[kx]);
        const float gB = __ldg(&R.green[(size_t)n * Z + kx]);
        const float sx = __ldg(&R.sxt[kx]);
        const float syA = __ldg(&R.syt[0]), syB = __ldg(&R.syt[n]);
        // i*s*g*A, then P = FxA + i FxB, Q = FyA + i FyB
        const float2 FxA = make_float2(-sx * gA * A.y, sx * gA * A.x);
        const float2 FxB = make_float2(-sx * gB * Bv.y, sx * gB * Bv.x);
        const float2 FyA = make_float2(-syA * gA * A.y, syA * gA * A.x);
        const float2 FyB = make_float2(-syB * gB * Bv.y, syB * gB * Bv.x);
        P[cnt] = make_float2(FxA.x - FxB.y, FxA.y + FxB.x);
        Q[cnt] = make_float2(FyA.x - FyB.y, FyA.y + FyB.x);
      }
      __syncthreads();
      cnt = 0;
      for (int pos = threadIdx.x; pos < Z && cnt < MAXIT; pos += blockDim.x, cnt++) {
        sA[pos << lw] = P[cnt];
        sB[pos << lw] = Q[cnt];
      }
    }
    __syncthreads();
    fft_dit(sA, R.plan_full, lw, R.tw, 1, true);
    fft_dit(sB, R.plan_full, lw, R.tw, 1, true);
    for (int i = threadIdx.x; i < (Z << lw); i += blockDim.x) {
      const int k = i >> lw, c = i & (W - 1);
      const float2 a = sA[i], b = sB[i];
      R.spec2[(size_t)k * n + col0 + c] = make_float4(a.x, a.y, b.x, b.y);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Row pass, inverse: both force grids are real, so one complex inverse
// transform of H = Fx' + i Fy' over the full y spectrum (Hermitian
// extension of the half spectra) yields Fx + i Fy, stored as float2.
__global__ void __launch_bounds__(FFT_THREADS) k_fft_rows_inv(const RunDesc* __restrict__ runs,
                                                      const RunDyn* __restrict__ dyn,
                                                      const Item* __restrict__ items, int nitems,
                                                      int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* s = (float2*)smem;
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    if (require_active && !run_active(dyn, I.run)) continue;
    const RunDesc& R = runs[I.run];
    const int Z = R.Z, n = Z >> 1;
    const int lr = I.c;
    const int row0 = I.a;
    for (int i = threadIdx.x; i < (Z << lr); i += blockDim.x) {
      const int b = i / Z, j = i - b * Z;
      const size_t rb = (size_t)(row0 + b) * n;
      float2 h;
      if (j == 0) {
        const float4 v = R.spec2[rb];
        h = make_float2(v.x, v.z);
      } else if (j == n) {
        const float4 v = R.spec2[rb];
        h = make_float2(v.y, v.w);
      } else if (j < n) {
        const float4 v = R.spec2[rb + j];
        h = make_float2(v.x - v.w, v.y + v.z);
      } else {
        const float4 v = R.spec2[rb + (Z - j)];
        h = make_float2(v.x + v.w, -v.y + v.z);
      }
      s[(__ldg(&R.pos_full[j]) << lr) | b] = h;
    }
    __syncthreads();
    fft_dit(s, R.plan_full, lr, R.tw, 1, true);
    for (int i = threadIdx.x; i < (Z << lr); i += blockDim.x) {
      const int b = i / Z, l = i - b * Z;
      R.H[(size_t)(row0 + b) * Z + l] = s[(l << lr) | b];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Power-of-two meshes: the same three passes with the register-radix
// Stockham transform (bd_fft2.cuh), natural order throughout. Items are
// sized on the host so that one item's sequences need at most blockDim.x
// threads.

// Row pass, forward, of rows row0 .. row0 + 2^lr - 1 (layout as
// k_fft_rows_fwd). tw: the run's twiddle table, in shared memory when TWS.
// FROM_ACC (fused step): the rows come from the fixed-point accumulator
// R.dacc, converted as deposit_tile converts its sums; the density is also
// stored to R.rho and the accumulator words are cleared for the next step.
template <int LZ, bool TWS, bool FROM_ACC = false>
__device__ __forceinline__ void fft2_rows_fwd_item(const RunDesc& R, int row0, int lr, float2* s,
                                                   const float2* tw) {
  constexpr int Z = 1 << LZ, n = Z >> 1, lz = LZ, ln = LZ - 1;
  constexpr int ss = fft2_stride(n);
  float2* src = reinterpret_cast<float2*>(R.rho) + (size_t)row0 * n;
  if (FROM_ACC) {
    ulonglong2* acc = reinterpret_cast<ulonglong2*>(R.dacc) + (size_t)row0 * n;
    const double inv = 1.0 / (double)__int_as_float((127 + R.fx_shift) << 23);
    for (int i = threadIdx.x; i < (n << lr); i += blockDim.x) {
      const int b = i >> ln, m = i & (n - 1);
      const ulonglong2 a = acc[i];
      const float2 v = make_float2((float)((double)(long long)a.x * inv), (float)((double)(long long)a.y * inv));
      s[b * ss + pad16(m)] = v;
      src[i] = v;
      acc[i] = make_ulonglong2(0ull, 0ull);
    }
  } else {
    for (int i = threadIdx.x; i < (n << lr); i += blockDim.x) {
      const int b = i >> ln, m = i & (n - 1);
      s[b * ss + pad16(m)] = src[i];
    }
  }
  __syncthreads();
  Fft2Sched<LZ - 1, 0, TWS>::run(s, ss, 1 << lr, tw, lz, -1.f);
  // the half spectrum is stored by column (slot j of row k at spec[j*Z + k]),
  // so the column pass reads whole columns. Consecutive threads take groups
  // of rb = min(2^lr, 4) consecutive rows of one slot (a whole 32-byte sector
  // of a column from 4 rows on), then the next slot: at most rb-way bank
  // conflicts on the rows' shared-memory reads.
  const int lrb = lr < 2 ? lr : 2;
  const int rbm = (1 << lrb) - 1;
  for (int i = threadIdx.x; i < (n << lr); i += blockDim.x) {
    const int rest = i >> lrb;
    const int j = rest & (n - 1), b = ((rest >> ln) << lrb) + (i & rbm);
    const float2 zj = s[b * ss + pad16(j)];
    const float2 zc = s[b * ss + pad16((n - j) & (n - 1))];
    float2 out;
    if (j == 0) {
      out = make_float2(zj.x + zj.y, zj.x - zj.y);
    } else {
      // E = (zj + conj zc)/2, O = (zj - conj zc)/(2i), X = E + w^j O
      const float2 E = make_float2(0.5f * (zj.x + zc.x), 0.5f * (zj.y - zc.y));
      const float2 O = make_float2(0.5f * (zj.y + zc.y), -0.5f * (zj.x - zc.x));
      out = cadd(E, cmul(TWS ? tw[j] : __ldg(&tw[j]), O));
    }
    R.spec[(size_t)j * Z + row0 + b] = out;
  }
  __syncthreads();
}

// Green's multiply of the packed column (ky = 0 and ky = Z/2 travel as
// C = A + iB): split with the partner Cm = C[-kx], multiply A and B by
// i*s*g with their own factors, pack the Fx and Fy results again.
__device__ __forceinline__ void packed_green(const RunDesc& R, int kx, float2 Cv, float2 Cm, int n, int Z,
                                             float sy0, float syn, float2& P, float2& Q) {
  // A = (C + conj Cm)/2 ; B = (C - conj Cm)/(2i)
  const float2 A = make_float2(0.5f * (Cv.x + Cm.x), 0.5f * (Cv.y - Cm.y));
  const float2 Bv = make_float2(0.5f * (Cv.y + Cm.y), -0.5f * (Cv.x - Cm.x));
  const float gA = __ldg(&R.green[kx]);
  const float gB = __ldg(&R.green[(size_t)n * Z + kx]);
  const float sx = __ldg(&R.sxt[kx]);
  const float2 FxA = make_float2(-sx * gA * A.y, sx * gA * A.x);
  const float2 FxB = make_float2(-sx * gB * Bv.y, sx * gB * Bv.x);
  const float2 FyA = make_float2(-sy0 * gA * A.y, sy0 * gA * A.x);
  const float2 FyB = make_float2(-syn * gB * Bv.y, syn * gB * Bv.x);
  P = make_float2(FxA.x - FxB.y, FxA.y + FxB.x);
  Q = make_float2(FyA.x - FyB.y, FyA.y + FyB.x);
}

// Column pass (as k_fft_cols) of the 2^lw adjacent half-spectrum columns
// from col0; smem holds 2 * 2^lw sequences.
template <int LZ, bool TWS>
__device__ __forceinline__ void fft2_cols_item(const RunDesc& R, int col0, int lw, float2* sA, const float2* tw) {
  constexpr int Z = 1 << LZ, n = Z >> 1, lz = LZ;
  constexpr int ss = fft2_stride(Z);
  const int W = 1 << lw;
  float2* sB = sA + W * ss;
  // the row pass stored the half spectrum by column: whole columns are read
  const float2* src = R.spec + (size_t)col0 * Z;
  for (int i = threadIdx.x; i < (Z << lw); i += blockDim.x) {
    const int c = i >> lz, k = i & (Z - 1);
    sA[c * ss + pad16(k)] = src[i];
  }
  __syncthreads();
  Fft2Sched<LZ, 0, TWS>::run(sA, ss, W, tw, lz, -1.f);
  for (int i = threadIdx.x; i < (Z << lw); i += blockDim.x) {
    const int c = i >> lz, kx = i & (Z - 1);
    const int j = col0 + c;
    if (j == 0) continue;
    const float g = __ldg(&R.green[(size_t)j * Z + kx]);
    const float gx = __ldg(&R.sxt[kx]) * g;
    const float gy = __ldg(&R.syt[j]) * g;
    const int a = c * ss + pad16(kx);
    const float2 v = sA[a];
    sA[a] = make_float2(-gx * v.y, gx * v.x);
    sB[a] = make_float2(-gy * v.y, gy * v.x);
  }
  if (col0 == 0) {
    // packed column (ky = 0, ky = Z/2): C = A + iB. Element kx of A, B
    // needs C[kx] and C[-kx], so one thread handles both of a pair and
    // writes them in place.
    const float sy0 = __ldg(&R.syt[0]), syn = __ldg(&R.syt[n]);
    for (int kx = threadIdx.x; kx <= n; kx += blockDim.x) {
      const int km = (Z - kx) & (Z - 1);
      const float2 Ck = sA[pad16(kx)], Cm = sA[pad16(km)];
      float2 P, Q;
      packed_green(R, kx, Ck, Cm, n, Z, sy0, syn, P, Q);
      sA[pad16(kx)] = P;
      sB[pad16(kx)] = Q;
      if (km != kx) {
        packed_green(R, km, Cm, Ck, n, Z, sy0, syn, P, Q);
        sA[pad16(km)] = P;
        sB[pad16(km)] = Q;
      }
    }
  }
  __syncthreads();
  if (2 * W * fft2_tps(lz) <= (int)blockDim.x) {
    Fft2Sched<LZ, 0, TWS>::run(sA, ss, 2 * W, tw, lz, 1.f);  // sB follows sA: 2W sequences
  } else {
    Fft2Sched<LZ, 0, TWS>::run(sA, ss, W, tw, lz, 1.f);
    Fft2Sched<LZ, 0, TWS>::run(sB, ss, W, tw, lz, 1.f);
  }
  for (int i = threadIdx.x; i < (Z << lw); i += blockDim.x) {
    const int k = i >> lw, c = i & (W - 1);
    const float2 a = sA[c * ss + pad16(k)], b = sB[c * ss + pad16(k)];
    R.spec2[(size_t)k * n + col0 + c] = make_float4(a.x, a.y, b.x, b.y);
  }
  __syncthreads();
}

// Row pass, inverse (as k_fft_rows_inv), of rows row0 .. row0 + 2^lr - 1.
template <int LZ, bool TWS>
__device__ __forceinline__ void fft2_rows_inv_item(const RunDesc& R, int row0, int lr, float2* s, const float2* tw) {
  constexpr int Z = 1 << LZ, n = Z >> 1, lz = LZ;
  constexpr int ss = fft2_stride(Z);
  for (int i = threadIdx.x; i < (Z << lr); i += blockDim.x) {
    const int b = i >> lz, j = i & (Z - 1);
    const float4* rb = R.spec2 + (size_t)(row0 + b) * n;
    float2 h;
    if (j == 0) {
      const float4 v = rb[0];
      h = make_float2(v.x, v.z);
    } else if (j == n) {
      const float4 v = rb[0];
      h = make_float2(v.y, v.w);
    } else if (j < n) {
      const float4 v = rb[j];
      h = make_float2(v.x - v.w, v.y + v.z);
    } else {
      const float4 v = rb[Z - j];
      h = make_float2(v.x + v.w, -v.y + v.z);
    }
    s[b * ss + pad16(j)] = h;
  }
  __syncthreads();
  Fft2Sched<LZ, 0, TWS>::run(s, ss, 1 << lr, tw, lz, 1.f);
  float2* dst = R.H + (size_t)row0 * Z;
  for (int i = threadIdx.x; i < (Z << lr); i += blockDim.x) {
    const int b = i >> lz, l = i & (Z - 1);
    dst[i] = s[b * ss + pad16(l)];
  }
  __syncthreads();
}

// The three passes as kernels, one item per CTA (an item loop around the
// transform with twiddles from global memory makes the compiler hoist the
// twiddle loads of every pass and spill).
template <int LZ>
__global__ void __launch_bounds__(FFT2_THREADS) k_fft2_rows_fwd(const RunDesc* __restrict__ runs,
                                                         const RunDyn* __restrict__ dyn,
                                                         const Item* __restrict__ items, int nitems,
                                                         int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  if ((int)blockIdx.x >= nitems) return;
  const Item I = items[blockIdx.x];
  if (require_active && !run_active(dyn, I.run)) return;
  const RunDesc& R = runs[I.run];
  fft2_rows_fwd_item<LZ, false>(R, I.a, I.c, (float2*)smem, R.tw);
}

template <int LZ>
__global__ void __launch_bounds__(FFT2_THREADS) k_fft2_cols(const RunDesc* __restrict__ runs,
                                                     const RunDyn* __restrict__ dyn,
                                                     const Item* __restrict__ items, int nitems,
                                                     int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  if ((int)blockIdx.x >= nitems) return;
  const Item I = items[blockIdx.x];
  if (require_active && !run_active(dyn, I.run)) return;
  const RunDesc& R = runs[I.run];
  fft2_cols_item<LZ, false>(R, I.a, I.c, (float2*)smem, R.tw);
}

// Meshes of 2048 and more: the column pass with 1024 threads, so that an
// item holds 2-4 adjacent columns (a 2048-point column alone needs 128
// threads per transform and 256 for the joint inverse) and each row's read
// of the half spectrum fills a 32-byte sector instead of a quarter of one.
template <int LZ>
__global__ void __launch_bounds__(FFT2_WIDE_THREADS) k_fft2_cols_wide(const RunDesc* __restrict__ runs,
                                                                      const RunDyn* __restrict__ dyn,
                                                                      const Item* __restrict__ items, int nitems,
                                                                      int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  if ((int)blockIdx.x >= nitems) return;
  const Item I = items[blockIdx.x];
  if (require_active && !run_active(dyn, I.run)) return;
  const RunDesc& R = runs[I.run];
  fft2_cols_item<LZ, false>(R, I.a, I.c, (float2*)smem, R.tw);
}

template <int LZ>
__global__ void __launch_bounds__(FFT2_THREADS) k_fft2_rows_inv(const RunDesc* __restrict__ runs,
                                                         const RunDyn* __restrict__ dyn,
                                                         const Item* __restrict__ items, int nitems,
                                                         int require_active) {
  extern __shared__ __align__(16) unsigned char smem[];
  if ((int)blockIdx.x >= nitems) return;
  const Item I = items[blockIdx.x];
  if (require_active && !run_active(dyn, I.run)) return;
  const RunDesc& R = runs[I.run];
  fft2_rows_inv_item<LZ, false>(R, I.a, I.c, (float2*)smem, R.tw);
}

// ---------------------------------------------------------------------------
// Per-particle physics shared by the staged and the global neighbour paths.

// Interpolated capillary force (gridRoutinen.cpp:81-126, 284-407, 551-668).
template <bool NC>
__device__ inline float2 mesh_force(const RunDesc& R, const Rec& p, int ic, int jc, int scheme) {
  int k, l;
  float tx, ty;
  mesh_axis(R, ic, p.ox, k, tx);
  mesh_axis(R, jc, p.oy, l, ty);
  const bool sp2 = p.pid >= R.N1;
  if (scheme == NGP) {
    const float2 h = ldm<NC>(&R.H[(size_t)k * R.Z + l]);
    if (!sp2) return h;
    // species 2 reads the imaginary part of the x grid in the reference
    // (gridRoutinen.cpp:123), which is zero up to rounding
    if (R.flags & F_NGP_REFCOMPAT) return make_float2(R.q2 * h.x, 0.0f);
    return make_float2(R.q2 * h.x, R.q2 * h.y);
  }
  float wx[3], wy[3];
  axis_weights(scheme, tx, wx);
  axis_weights(scheme, ty, wy);
  const int km = k == 0 ? R.Z - 1 : k - 1, kp = k == R.Z - 1 ? 0 : k + 1;
  const int lm = l == 0 ? R.Z - 1 : l - 1, lp = l == R.Z - 1 ? 0 : l + 1;
  const int ks[3] = {km, k, kp};
  float fx = 0.f, fy = 0.f;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float2* row = R.H + (size_t)ks[a] * R.Z;
    const float2 h0 = ldm<NC>(&row[lm]), h1 = ldm<NC>(&row[l]), h2 = ldm<NC>(&row[lp]);
    fx += wx[a] * (wy[0] * h0.x + wy[1] * h1.x + wy[2] * h2.x);
    fy += wx[a] * (wy[0] * h0.y + wy[1] * h1.y + wy[2] * h2.y);
  }
  if (sp2) {
    fx *= R.q2;
    fy *= R.q2;
  }
  return make_float2(fx, fy);
}

// WCA parameters of one particle against neighbours of its own and of the
// other species (dynamik_methoden.cpp:679-686, 851-865, 1021-1035), held in
// registers for its pair loop. mask selects pair types (1: 11, 2: 22, 4: 12).
struct WcaP {
  float pre_s, sig_s, sig2_s;  // same species
  float pre_x, sig_x, sig2_x;  // other species
  float B, cut2, maxPair, L;
  float scale;                 // 2^wfx_shift: pair terms are summed in 64-bit fixed point
  int N1;
  bool sp, on_s, on_x, smallbox;
};

__device__ __forceinline__ WcaP wca_params(const RunDesc& R, const Rec& p, int mask) {
  WcaP W;
  W.sp = p.pid >= R.N1;
  const int ts = W.sp ? 1 : 0;
  W.pre_s = R.wpre[ts];
  W.sig_s = R.wsig[ts];
  W.sig2_s = R.wsig2[ts];
  W.pre_x = R.wpre[2];
  W.sig_x = R.wsig[2];
  W.sig2_x = R.wsig2[2];
  W.on_s = (mask & (W.sp ? 2 : 1)) != 0;
  W.on_x = (mask & 4) != 0;
  W.B = R.B;
  W.cut2 = R.cut2;
  W.maxPair = R.maxPair;
  W.L = R.L;
  W.N1 = R.N1;
  W.smallbox = (R.flags & F_SMALLBOX) != 0;
  W.scale = __int_as_float((127 + R.wfx_shift) << 23);
  return W;
}

// WCA contribution of neighbour q on particle p, added to the fixed-point
// sum (fx, fy): rounded once per pair term, the sum does not depend on the
// order in which neighbours are visited. da, db: cell step from p's cell to
// q's cell.
__device__ __forceinline__ void wca_pair(const WcaP& W, const Rec& p, const Rec& q, int da, int db, long long& fx,
                                         long long& fy) {
  const bool same = (q.pid >= W.N1) == W.sp;
  if (!(same ? W.on_s : W.on_x)) return;
  float dx = (p.ox - q.ox) - (float)da * W.B;
  float dy = (p.oy - q.oy) - (float)db * W.B;
  // minimum image, as abstand2_* (allgemeine_methoden.cpp:100-166). With
  // offsets in (-B, 2B] and neighbouring cells |d| < 3B, which is below L/2
  // from 7 cells per side on; only smaller boxes need the wrap.
  if (W.smallbox) {
    dx -= W.L * rintf(dx / W.L);
    dy -= W.L * rintf(dy / W.L);
  }
  const float a2 = dx * dx + dy * dy;
  const float a2s = a2 * (same ? W.sig2_s : W.sig2_x);
  if (a2s > W.cut2) return;
  const float coef = wca_coef(a2s, same ? W.pre_s : W.pre_x, W.maxPair);
  const float sg = same ? W.sig_s : W.sig_x;
  fx += __float2ll_rn(coef * (dx * sg) * W.scale);
  fy += __float2ll_rn(coef * (dy * sg) * W.scale);
}

// Re-binning of one axis after a move (refresh_erwNachbar,
// dynamik_methoden.cpp:216-325): the cell moves by floor(off/B) and the
// offset becomes fmod(off + B, B). For off in [-B, 0) the new offset is
// off + B, kept as is when FP32 rounds it to B (a legal offset) instead of
// wrapping to 0, which would move the particle by a whole cell. For
// off < -B the reference's fmod keeps a negative offset; reproduced.
__device__ inline void rebin_axis(float off, float B, int& n, float& no) {
  if (off >= 0.0f && off < B) {
    n = 0;
    no = off;
  } else if (off == B) {
    n = 1;
    no = 0.0f;
  } else if (off > B && off < 2.0f * B) {
    n = 1;
    no = off - B;
  } else if (off < 0.0f && off >= -B) {
    n = -1;
    no = off + B;
  } else if (off >= 2.0f * B) {
    const float fl = floorf(off / B);
    n = (int)fl;
    no = fmaf(-fl, B, off);
    if (no >= B) {
      no -= B;
      n++;
    } else if (no < 0.0f) {
      no += B;
      n--;
    }
  } else if (off < -B) {
    n = (int)floorf(off / B);
    no = fmodf(off + B, B);
  } else {  // NaN
    n = 0;
    no = off;
  }
}

struct StepOut {
  Rec r;
  int key;
};

// Euler-Maruyama update (zeitschritt, dynamik_methoden.cpp:117-157) and
// re-binning of one particle.
__device__ inline Rec move_particle(const RunDesc& R, Rec p, float2 F, float2 xi, float dt,
                                    int* err, bool apply = true) {
  if (apply) {
    const float sq = sqrtf(2.0f * R.T * dt);
    p.ox += dt * F.x + sq * xi.x;
    p.oy += dt * F.y + sq * xi.y;
  }
  if (apply && (R.flags & F_RADIAL) && p.pid >= R.N1) {
    int ic, jc;
    cell_ij(R, p.cell, ic, jc);
    const double mitte = 0.5 * R.L_d;
    const double x = ic * R.B_d + (double)p.ox;
    const double y = jc * R.B_d + (double)p.oy;
    const double dxm = mitte - x, dym = mitte - y;
    const double abst = sqrt(dxm * dxm + dym * dym);
    const int t = p.pid - R.N1;
    // cos / sin of 2 pi t / N2 as sincospi (no large-argument reduction path)
    double sn, cs;
    sincospi(2.0 * t / R.N2, &sn, &cs);
    p.ox = (float)((double)p.ox + (mitte + abst * cs - x));
    p.oy = (float)((double)p.oy + (mitte + abst * sn - y));
  }
  if (!isfinite(p.ox) || !isfinite(p.oy)) {
    atomicOr(err, E_NONFINITE);
    return p;
  }
  if (p.ox < 0.0f || p.ox > R.B || p.oy < 0.0f || p.oy > R.B) {
    int nx, ny;
    float ox, oy;
    rebin_axis(p.ox, R.B, nx, ox);
    rebin_axis(p.oy, R.B, ny, oy);
    int ic, jc;
    cell_ij(R, p.cell, ic, jc);
    const int icn = wrapi(ic + nx, R.C), jcn = wrapi(jc + ny, R.C);
    p.cell = icn * R.C + jcn;
    p.ox = ox;
    p.oy = oy;
  }
  return p;
}

// optimaler_zeitschritt bound of one component (dynamik_methoden.cpp:1420-1491):
// dt < (w-|u|)^2 with u = xi sqrt(T/2)/F, w = sqrt(u^2 + m/|F|). In FP32
// w - |u| cancels when u^2 >> m/|F|, so it is evaluated as the equal
// (m/|F|) / (w + |u|).
__device__ inline float dt_bound(float F, float nz, float mrd, float T) {
  if (fabsf(F) < 1.0e-5f) return mrd * mrd / (2.0f * T * nz * nz);
  const float u = nz * sqrtf(0.5f * T) / F;
  const float a = mrd / fabsf(F);
  const float w = sqrtf(u * u + a);
  const float d = a / (w + fabsf(u));
  return d * d;
}


template <bool NC, bool DEP>
__device__ inline void finish_particle(const RunDesc& R, RunDyn& D, int mode, int mask,
                                       const Rec& p, int ic, int jc, int gi, float2 Fw);

template <bool NC>
__device__ __forceinline__ Rec ldrec(const Rec* q) {
  const int4 v = ldm<NC>(reinterpret_cast<const int4*>(q));
  Rec r;
  r.ox = __int_as_float(v.x);
  r.oy = __int_as_float(v.y);
  r.cell = v.z;
  r.pid = v.w;
  return r;
}

// WCA sum of particle p (at global index self, cell (ic, jc)) over the 3x3
// neighbour cells, read straight from the cell-sorted array: per neighbour
// row the cells jc-1, jc, jc+1 form one contiguous range unless the row
// wraps. The fixed-point sum makes the result independent of the order of
// the particles within a cell.
template <bool NC>
__device__ inline float2 wca_direct(const RunDesc& R, const Rec& p, int ic, int jc, int self, int m) {
  long long fx = 0, fy = 0;
  const WcaP W = wca_params(R, p, m);
  const int C = R.C;
  const Rec* rec = R.recA;
  const int* start = R.start;
  if (jc >= 1 && jc <= C - 2) {
    // per neighbour row one contiguous range (cells jc-1 .. jc+1); the six
    // bounds are loaded together
    int beg[3], end[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int row = wrap1(ic + a - 1, C) * C;
      beg[a] = ldm<NC>(&start[row + jc - 1]);
      end[a] = ldm<NC>(&start[row + jc + 2]);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int cmid = wrap1(ic + a - 1, C) * C + jc;
      if constexpr (!NC) {
        // fused step (registers to spare): the next record is requested
        // before the current pair is evaluated
        Rec q;
        if (beg[a] < end[a]) q = ldrec<NC>(&rec[beg[a]]);
        for (int j = beg[a]; j < end[a]; j++) {
          Rec qn = q;
          if (j + 1 < end[a]) qn = ldrec<NC>(&rec[j + 1]);
          if (j != self) wca_pair(W, p, q, a - 1, q.cell - cmid, fx, fy);
          q = qn;
        }
      } else {
        for (int j = beg[a]; j < end[a]; j++) {
          if (j == self) continue;
          const Rec q = ldrec<NC>(&rec[j]);
          wca_pair(W, p, q, a - 1, q.cell - cmid, fx, fy);
        }
      }
    }
  } else {
#pragma unroll 1
    for (int da = -1; da <= 1; da++) {
      const int row = wrap1(ic + da, C) * C;
#pragma unroll 1
      for (int db = -1; db <= 1; db++) {
        const int g = row + wrap1(jc + db, C);
        const int beg = ldm<NC>(&start[g]), end = ldm<NC>(&start[g + 1]);
        for (int j = beg; j < end; j++) {
          if (j == self) continue;
          wca_pair(W, p, ldrec<NC>(&rec[j]), da, db, fx, fy);
        }
      }
    }
  }
  const double inv = 1.0 / (double)W.scale;
  return make_float2((float)((double)fx * inv), (float)((double)fy * inv));
}

// Forces and (MODE_STEP) the move of the particle at sorted index gi; DEP:
// the move also deposits the new position into R.dacc.
template <bool NC, bool DEP>
__device__ __forceinline__ void particle_item(const RunDesc& R, RunDyn& D, int gi, int mode, int mask) {
  const Rec p = ldrec<NC>(&R.recA[gi]);
  int ic, jc;
  cell_ij(R, p.cell, ic, jc);
  int m = mask;
  if (mode == MODE_SET) m &= p.pid >= R.N1 ? 2 : 1;
  if (R.flags & F_IDGAS) m = 0;
  const float2 Fw = m ? wca_direct<NC>(R, p, ic, jc, gi, m) : make_float2(0.f, 0.f);
  finish_particle<NC, DEP>(R, D, mode, mask, p, ic, jc, gi, Fw);
}

// One thread per particle of the cell-sorted array.
// deposit (MODE_STEP): the move adds the next step's density to each run's
// accumulator R.dacc (the pipelined stage step, whose forward row pass reads it)
// MINB: CTAs per SM the compiler keeps registers for (4: at most 64
// registers; 5: at most 51, more warps resident, a few values reloaded from
// local memory); the batch autotuner picks one, the arithmetic is the same.
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_particles(const RunDesc* __restrict__ runs,
                                                   RunDyn* __restrict__ dyn,
                                                   const Item* __restrict__ items, int nitems,
                                                   int mode, int mask, int require_active, int deposit) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    // the pipelined step (deposit): the run's first block records whether
    // the run takes part in this step, for the sort and transform kernels
    // that follow (the step end changes the budget while they run)
    if (deposit && I.a == 0 && threadIdx.x == 0) dyn[I.run].sorting = run_active(dyn, I.run) ? 1 : 0;
    if (require_active && !run_active(dyn, I.run)) continue;
    const RunDesc& R = runs[I.run];
    const int gi = I.a * blockDim.x + threadIdx.x;
    if (gi >= R.N) continue;
    if (deposit) particle_item<true, true>(R, dyn[I.run], gi, mode, mask);
    else particle_item<true, false>(R, dyn[I.run], gi, mode, mask);
  }
}


// Count particle gi into its new cell (an add whose result nobody waits for;
// the scatter takes the slots) and into the per-chunk total for the scan,
// added once per group of lanes in the same chunk (neighbouring particles of
// the cell-sorted order mostly share one). The cell is the key: the scatter
// reads it from the record recB[gi].
__device__ __forceinline__ void count_into_cell(const RunDesc& R, int gi, int key) {
  atomicAdd(&R.count[key], 1);
  const int ch = key / SCAN_CHUNK;
  const unsigned grp = __match_any_sync(__activemask(), ch);
  if ((threadIdx.x & 31) == __ffs(grp) - 1) atomicAdd(&R.chunk_sum[ch], __popc(grp));
}

// Everything after the WCA sum: store it (MODE_SET/ADD), or add the mesh
// force and the noise and store the forces (MODE_FORCES) or move and re-bin
// (MODE_STEP).
template <bool NC, bool DEP>
__device__ inline void finish_particle(const RunDesc& R, RunDyn& D, int mode, int mask,
                                       const Rec& p, int ic, int jc, int gi, float2 Fw) {
  const bool sp2 = p.pid >= R.N1;
  if (mode == MODE_SET) {
    if ((mask & (sp2 ? 2 : 1))) R.Fw[p.pid] = Fw;
    return;
  }
  if (mode == MODE_ADD) {
    float2 f = R.Fw[p.pid];
    f.x += Fw.x;
    f.y += Fw.y;
    R.Fw[p.pid] = f;
    return;
  }
  const float2 Fk = (R.flags & F_IDGAS) ? make_float2(0.f, 0.f) : mesh_force<NC>(R, p, ic, jc, R.scheme);
  float2 xi = make_float2(0.f, 0.f);
  if (!(R.flags & F_NOWCA)) xi = particle_noise(R.noise, R.seed, D.step, (uint32_t)p.pid);
  if (mode == MODE_FORCES) {
    R.Fw[p.pid] = Fw;
    R.Fk[p.pid] = Fk;
    R.Fn[p.pid] = xi;
    float bnd = fminf(dt_bound(Fw.x + Fk.x, xi.x, R.mrd, R.T), dt_bound(Fw.y + Fk.y, xi.y, R.mrd, R.T));
    if (!(bnd >= 0.f)) bnd = 3.0e38f;  // NaN never wins the minimum (std::min semantics)
    if (bnd < R.dt_max) atomicMin(&D.dt_bits, __float_as_uint(bnd));
    return;
  }
  // MODE_STEP
  const float2 F = make_float2(Fw.x + Fk.x, Fw.y + Fk.y);
  const Rec np = move_particle(R, p, F, xi, R.dt_max, &D.err);
  R.recB[gi] = np;
  count_into_cell(R, gi, np.cell);
  // the fused step and the pipelined stage step: the next step's density
  if constexpr (DEP) deposit_acc(R, np);
  if (np.cell != p.cell) atomicAdd(&D.moved[sp2 ? 1 : 0], 1);  // num_Zellwechsel of TimestepInfo
}

// Move from stored forces (adaptive dt: the reduced bound; fixed dt: dt_max),
// or with refresh_only re-bin the current positions without moving
// (refresh_erwNachbar on caller-modified offsets).
__global__ void __launch_bounds__(256) k_move(const RunDesc* __restrict__ runs,
                                              RunDyn* __restrict__ dyn,
                                              const Item* __restrict__ items, int nitems,
                                              int require_active, int refresh_only) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    if (require_active && !run_active(dyn, I.run)) continue;
    const RunDesc& R = runs[I.run];
    RunDyn& D = dyn[I.run];
    const int gi = I.a * blockDim.x + threadIdx.x;
    if (gi >= R.N) continue;
    const Rec p = R.recA[gi];
    Rec np;
    if (refresh_only) {
      np = move_particle(R, p, make_float2(0.f, 0.f), make_float2(0.f, 0.f), 0.f, &D.err, false);
    } else {
      const float2 Fw = R.Fw[p.pid], Fk = R.Fk[p.pid], xi = R.Fn[p.pid];
      const float dt = (R.flags & F_ADAPTIVE) ? fminf(R.dt_max, __uint_as_float(D.dt_bits)) : R.dt_max;
      np = move_particle(R, p, make_float2(Fw.x + Fk.x, Fw.y + Fk.y), xi, dt, &D.err);
    }
    R.recB[gi] = np;
    count_into_cell(R, gi, np.cell);
    if (np.cell != p.cell) atomicAdd(&D.moved[p.pid >= R.N1 ? 1 : 0], 1);
  }
}

// Keys of an unsorted upload in recB (initial sort).
__global__ void __launch_bounds__(256) k_count(const RunDesc* __restrict__ runs,
                                               const Item* __restrict__ items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    const RunDesc& R = runs[I.run];
    const int gi = I.a * blockDim.x + threadIdx.x;
    if (gi >= R.N) continue;
    count_into_cell(R, gi, R.recB[gi].cell);
  }
}

// ---------------------------------------------------------------------------
// Counting sort by cell: exclusive scan of the counts (the per-chunk totals
// come from the counting kernels; one CTA per run scans them, then every
// chunk of SCAN_CHUNK cells scans its counts from its offset), scatter by
// (start + atomic slot), then a fix-up that orders every cell holding two or
// more particles by particle index. The result is the order a stable sort by
// cell of the particle-index order gives, which is the reference's
// neighbour-list order after WCA_init (ascending index).

// End of a step (one thread per run): advance the Philox step counter, the
// simulated time and the steps budget; re-arm the adaptive dt reduction.
__device__ inline void end_step(const RunDesc& R, RunDyn& D, int adaptive) {
  double dt = R.dt_max_d;
  if (adaptive && (R.flags & F_ADAPTIVE)) {
    const float b = __uint_as_float(D.dt_bits);
    dt = b < R.dt_max ? (double)b : R.dt_max_d;
  }
  D.dt = (float)dt;
  D.t += dt;
  D.step++;
  D.steps_left--;
  D.dt_bits = __float_as_uint(3.0e38f);
  D.moved_last[0] = D.moved[0];
  D.moved_last[1] = D.moved[1];
  D.moved[0] = D.moved[1] = 0;
}

// Exclusive scan of one run's chunk totals into chunk_off; clears the
// totals. With end_step (the fused step's sort) its thread 0 also ends the
// run's step: the particle kernels that read the step counter and the dt
// bound are done, the scan and the scatter do not read them.
__global__ void __launch_bounds__(1024) k_chunk_scan(const RunDesc* __restrict__ runs, RunDyn* __restrict__ dyn,
                                                     int run0, int nruns, int end_step_flag, int adaptive,
                                                     int require_active) {
  __shared__ int sh[32];
  // up to 1024 * CPT chunks: C <= 4095 gives at most 8188
  constexpr int CPT = 8;
  for (int run = run0 + blockIdx.x; run < run0 + nruns; run += gridDim.x) {
    // the scan and the scatter of this sort follow this decision, taken
    // before end_step changes the steps budget
    const bool on = !require_active || run_active(dyn, run);
    __syncthreads();
    if (threadIdx.x == 0) dyn[run].sorting = on ? 1 : 0;
    if (!on) continue;
    const RunDesc& R = runs[run];
    const int nch = (R.C * R.C + SCAN_CHUNK - 1) / SCAN_CHUNK;
    const int k0 = threadIdx.x * CPT;
    int v[CPT];
    int loc = 0;
#pragma unroll
    for (int k = 0; k < CPT; k++) {
      v[k] = k0 + k < nch ? R.chunk_sum[k0 + k] : 0;
      loc += v[k];
    }
    int ex = block_excl_scan(loc, sh);
#pragma unroll
    for (int k = 0; k < CPT; k++)
      if (k0 + k < nch) {
        R.chunk_off[k0 + k] = ex;
        R.chunk_sum[k0 + k] = 0;
        ex += v[k];
      }
    if (end_step_flag && threadIdx.x == 0) end_step(R, dyn[run], adaptive);
    __syncthreads();
  }
}

// Scan of one chunk's counts from its offset into start[]; clears the
// counts for the next sort. CTAs stride over the chunks and load the next
// chunk's counts before scanning the current one, so loads stay in flight.
struct ScanChunk {
  const RunDesc* R;
  int chunk, ncells;
  bool on;
  int v[SCAN_CHUNK / 256];
};

__device__ __forceinline__ void scan_load(const RunDesc* __restrict__ runs, const RunDyn* __restrict__ dyn,
                                          const Item& I, int require_active, ScanChunk& S) {
  constexpr int PER = SCAN_CHUNK / 256;
  S.R = &runs[I.run];
  S.chunk = I.a;
  S.on = !require_active || dyn[I.run].sorting;
  S.ncells = S.R->C * S.R->C;
  const int base = I.a * SCAN_CHUNK;
  const int c0 = base + threadIdx.x * PER;
  const int* cnt = S.R->count;
  if (base + SCAN_CHUNK <= S.ncells) {
    const int4 a = __ldcg(reinterpret_cast<const int4*>(&cnt[c0]));
    const int4 b = __ldcg(reinterpret_cast<const int4*>(&cnt[c0 + 4]));
    S.v[0] = a.x, S.v[1] = a.y, S.v[2] = a.z, S.v[3] = a.w;
    S.v[4] = b.x, S.v[5] = b.y, S.v[6] = b.z, S.v[7] = b.w;
  } else {
#pragma unroll
    for (int k = 0; k < PER; k++) S.v[k] = c0 + k < S.ncells ? __ldcg(&cnt[c0 + k]) : 0;
  }
}

// start[] of one chunk from its counts v (eight per thread) and its offset.
// The counts stay: the scatter counts them down to zero as it takes slots.
// All threads call; sh: 32 ints.
__device__ __forceinline__ void scan_chunk_store(const RunDesc& R, int chunk, int ncells, const int* v, int off,
                                                 int* sh) {
  constexpr int PER = SCAN_CHUNK / 256;
  const int base = chunk * SCAN_CHUNK;
  const int c0 = base + threadIdx.x * PER;
  int loc = 0;
#pragma unroll
  for (int k = 0; k < PER; k++) loc += v[k];
  int acc = block_excl_scan(loc, sh) + off;
  int w[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) {
    w[k] = acc;
    acc += v[k];
  }
  if (base + SCAN_CHUNK <= ncells) {
    *reinterpret_cast<int4*>(&R.start[c0]) = make_int4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<int4*>(&R.start[c0 + 4]) = make_int4(w[4], w[5], w[6], w[7]);
  } else {
#pragma unroll
    for (int k = 0; k < PER; k++)
      if (c0 + k < ncells) R.start[c0 + k] = w[k];
  }
  if (base + SCAN_CHUNK >= ncells && threadIdx.x == 0) R.start[ncells] = R.N;
  __syncthreads();  // sh is reused by the next scan
}

__global__ void __launch_bounds__(256) k_scan(const RunDesc* __restrict__ runs, const RunDyn* __restrict__ dyn,
                                              const Item* __restrict__ items, int nitems, int require_active) {
  static_assert(SCAN_CHUNK == 2048, "eight counts per thread");
  __shared__ int sh[32];
  int it = blockIdx.x;
  if (it >= nitems) return;
  ScanChunk cur, nxt;
  scan_load(runs, dyn, items[it], require_active, cur);
  for (;;) {
    const int itn = it + gridDim.x;
    if (itn < nitems) scan_load(runs, dyn, items[itn], require_active, nxt);
    if (cur.on) scan_chunk_store(*cur.R, cur.chunk, cur.ncells, cur.v, cur.R->chunk_off[cur.chunk], sh);
    if (itn >= nitems) break;
    it = itn;
    cur = nxt;
  }
}

// Particle gi of the old order to start[cell] + slot, the slot taken by
// counting the cell's count down (which leaves it zero for the next sort).
__device__ __forceinline__ void scatter_particle(const RunDesc& R, int gi) {
  const Rec q = R.recB[gi];
  const int slot = atomicSub(&R.count[q.cell], 1) - 1;
  R.recA[R.start[q.cell] + slot] = q;
}

// Places every particle at start[cell] + slot (slots in atomic order: the
// order within a cell is arbitrary and no result depends on it).
__global__ void __launch_bounds__(256) k_scatter(const RunDesc* __restrict__ runs,
                                                 const RunDyn* __restrict__ dyn,
                                                 const Item* __restrict__ items, int nitems,
                                                 int require_active) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    if (require_active && !dyn[I.run].sorting) continue;
    const RunDesc& R = runs[I.run];
    const int gi = I.a * blockDim.x + threadIdx.x;
    if (gi >= R.N) continue;
    scatter_particle(R, gi);
  }
}


// ---------------------------------------------------------------------------
// Pipelined stage step: any number of runs on power-of-two meshes with a
// fixed dt, six launches per step. As in the fused step, the move deposits
// the next step's density (the same fixed-point integers as the tiles, into
// each run's R.dacc), and the transform of the new density runs beside the
// cell sort:
//   k_particles     forces, noise, move, re-binning, counts, next density;
//                   marks the runs that take part (`sorting`)
//   then, on two streams joined at the step's end:
//   k_pipe_scan -> k_pipe_scatter (step end)
//   k_pipe_fft<1> forward rows -> k_pipe_fft<2> columns + Green
//                 -> k_pipe_fft<0> inverse rows (the next step's force grids)
// Each kernel keeps its own registers and shared memory. Every transform CTA
// takes one item, of any mesh size (log2 Z in Item.b): no loop wraps a
// transform, whose per-thread offsets and twiddles the compiler would
// otherwise keep live across iterations.
#define BD_PIPE_SIZES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)

// pass 0: inverse rows, 1: forward rows from R.dacc, 2: columns + Green
template <int PASS>
__device__ __forceinline__ void pipe_fft_item(const RunDesc& R, const Item& I, float2* s) {
  switch (I.b) {
#define BD_CASE(L)                                                      \
  case L:                                                               \
    if (PASS == 0) fft2_rows_inv_item<L, false>(R, I.a, I.c, s, R.tw);       \
    else if (PASS == 1) fft2_rows_fwd_item<L, false, true>(R, I.a, I.c, s, R.tw); \
    else fft2_cols_item<L, false>(R, I.a, I.c, s, R.tw);                    \
    break;
    BD_PIPE_SIZES(BD_CASE)
#undef BD_CASE
    default:
      break;
  }
}

// One transform item per CTA, of any mesh size (pass as pipe_fft_item).
// Every pass checks `sorting` (whether the run takes part in this step,
// recorded by the particle kernel): the passes run beside the cell sort,
// whose last kernel ends the step and changes the step budget.
// Registers bounded for four CTAs per SM (64; a few values spill): the
// passes are bound by load latency, and the fourth CTA hides more of it
// (256-run ensemble: three passes 0.138 -> 0.129 ms).
template <int PASS>
__global__ void __launch_bounds__(FFT2_THREADS, 4) k_pipe_fft(const RunDesc* __restrict__ runs,
                                                            RunDyn* __restrict__ dyn,
                                                            const Item* __restrict__ items, int nitems) {
  extern __shared__ __align__(16) unsigned char smem[];
  if ((int)blockIdx.x >= nitems) return;
  const Item I = items[blockIdx.x];
  if (!((volatile const RunDyn*)dyn)[I.run].sorting) return;
  pipe_fft_item<PASS>(runs[I.run], I, (float2*)smem);
}

// Scan chunk c of run R (256 threads, all call): its offset is the sum of
// the run's earlier chunk totals, formed here (no separate chunk scan).
__device__ __forceinline__ void scan_chunk_item(const RunDesc& R, int c, int* s_tmp) {
  static_assert(SCAN_CHUNK == 2048, "eight counts per thread");
  const int ncells = R.C * R.C;
  int loc = 0;
  for (int k = threadIdx.x; k < c; k += blockDim.x) loc += R.chunk_sum[k];
  const int ex = block_excl_scan(loc, s_tmp);
  if (threadIdx.x == blockDim.x - 1) s_tmp[0] = ex + loc;
  __syncthreads();
  const int off = s_tmp[0];
  __syncthreads();
  constexpr int PER = SCAN_CHUNK / 256;
  const int c0 = c * SCAN_CHUNK + threadIdx.x * PER;
  int cv[PER];
#pragma unroll
  for (int k = 0; k < PER; k++) cv[k] = c0 + k < ncells ? R.count[c0 + k] : 0;
  scan_chunk_store(R, c, ncells, cv, off, s_tmp);
}

// PIPE_SCAN_GROUP chunks of one run per CTA (Item.a: the first): the counts
// (8 per chunk and thread) are requested before the offset, the sum of the run's
// earlier chunk totals, so both round trips overlap; one exclusive scan over
// the group. The starts are those of the per-chunk scan (one exclusive scan
// of the run's counts), so the group size is a free choice.
__global__ void __launch_bounds__(256) k_pipe_scan(const RunDesc* __restrict__ runs,
                                                   RunDyn* __restrict__ dyn,
                                                   const Item* __restrict__ groups, int ngroup) {
  constexpr int PER = PIPE_SCAN_GROUP * SCAN_CHUNK / 256;
  static_assert(PER % 4 == 0, "whole int4 vectors per thread");
  __shared__ int s_tmp[32];
  if ((int)blockIdx.x >= ngroup) return;
  const Item I = groups[blockIdx.x];
  if (!dyn[I.run].sorting) return;
  const RunDesc& R = runs[I.run];
  const int ncells = R.C * R.C, c0 = I.a;
  const int g0 = c0 * SCAN_CHUNK;
  const int base = g0 + threadIdx.x * PER;
  int v[PER];
  if (base + PER <= ncells) {
#pragma unroll
    for (int k = 0; k < PER; k += 4) {
      const int4 q = *reinterpret_cast<const int4*>(&R.count[base + k]);
      v[k] = q.x;
      v[k + 1] = q.y;
      v[k + 2] = q.z;
      v[k + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < PER; k++) v[k] = base + k < ncells ? R.count[base + k] : 0;
  }
  int pre = 0;
  for (int k = threadIdx.x; k < c0; k += blockDim.x) pre += R.chunk_sum[k];
  int tot = 0;
#pragma unroll
  for (int k = 0; k < PER; k++) tot += v[k];
  // the offset: the block's sum of pre, read after the scan of pre
  const int ex_pre = block_excl_scan(pre, s_tmp);
  if (threadIdx.x == blockDim.x - 1) s_tmp[0] = ex_pre + pre;
  __syncthreads();
  const int off = s_tmp[0];
  __syncthreads();
  int acc = block_excl_scan(tot, s_tmp) + off;
  if (base + PER <= ncells) {
#pragma unroll
    for (int k = 0; k < PER; k += 4) {
      int4 w;
      w.x = acc;
      acc += v[k];
      w.y = acc;
      acc += v[k + 1];
      w.z = acc;
      acc += v[k + 2];
      w.w = acc;
      acc += v[k + 3];
      *reinterpret_cast<int4*>(&R.start[base + k]) = w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < PER; k++) {
      if (base + k < ncells) R.start[base + k] = acc;
      acc += v[k];
    }
  }
  if (g0 + PIPE_SCAN_GROUP * SCAN_CHUNK >= ncells && threadIdx.x == 0) R.start[ncells] = R.N;
}

// Scatter of particles [a * PIPE_SCATTER_UNIT, +PIPE_SCATTER_UNIT) of run R:
// four per thread, their loads and slot atomics issued together.
__device__ __forceinline__ void scatter_unit(const RunDesc& R, int a) {
  constexpr int Q = PIPE_SCATTER_UNIT / 256;
  const int g0 = a * PIPE_SCATTER_UNIT + threadIdx.x;
  Rec q[Q];
  int slot[Q], st[Q];
#pragma unroll
  for (int k = 0; k < Q; k++)
    if (g0 + 256 * k < R.N) q[k] = R.recB[g0 + 256 * k];
#pragma unroll
  for (int k = 0; k < Q; k++)
    if (g0 + 256 * k < R.N) {
      slot[k] = atomicSub(&R.count[q[k].cell], 1) - 1;
      st[k] = R.start[q[k].cell];
    }
#pragma unroll
  for (int k = 0; k < Q; k++)
    if (g0 + 256 * k < R.N) R.recA[st[k] + slot[k]] = q[k];
}

// One scatter unit per CTA, then, spread over all threads of the launch, the
// chunk totals of every sorting run cleared and (by its first chunk's
// thread) the run's step ended.
__global__ void __launch_bounds__(256) k_pipe_scatter(const RunDesc* __restrict__ runs, RunDyn* __restrict__ dyn,
                                                      const Item* __restrict__ units, int nunit,
                                                      const Item* __restrict__ chunks, int nchunk) {
  if ((int)blockIdx.x < nunit) {
    const Item I = units[blockIdx.x];
    if (dyn[I.run].sorting) scatter_unit(runs[I.run], I.a);
  }
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nchunk; c += gridDim.x * blockDim.x) {
    const Item I = chunks[c];
    if (!dyn[I.run].sorting) continue;
    runs[I.run].chunk_sum[I.a] = 0;
    if (I.a == 0) end_step(runs[I.run], dyn[I.run], 0);
  }
}

// ---------------------------------------------------------------------------
// Drop-in single routines.

// inv_gridDensity_*: Fk[pid] from the current force grid with `scheme`.
__global__ void __launch_bounds__(256) k_interp(const RunDesc* __restrict__ runs,
                                                const Item* __restrict__ items, int nitems,
                                                int scheme) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    const RunDesc& R = runs[I.run];
    const int gi = I.a * blockDim.x + threadIdx.x;
    if (gi >= R.N) continue;
    const Rec p = R.recA[gi];
    int ic, jc;
    cell_ij(R, p.cell, ic, jc);
    R.Fk[p.pid] = (R.flags & F_IDGAS) ? make_float2(0.f, 0.f) : mesh_force<true>(R, p, ic, jc, scheme);
  }
}

// berechne_zufallskraefte: Fn[pid] for the current step.
__global__ void __launch_bounds__(256) k_noise(const RunDesc* __restrict__ runs,
                                               const RunDyn* __restrict__ dyn,
                                               const Item* __restrict__ items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    const RunDesc& R = runs[I.run];
    const int pid = I.a * blockDim.x + threadIdx.x;
    if (pid >= R.N) continue;
    R.Fn[pid] = (R.flags & F_NOWCA) ? make_float2(0.f, 0.f)
                                    : particle_noise(R.noise, R.seed, dyn[I.run].step, (uint32_t)pid);
  }
}

// optimaler_zeitschritt over the stored force/noise buffers.
__global__ void __launch_bounds__(256) k_dtbound(const RunDesc* __restrict__ runs,
                                                 RunDyn* __restrict__ dyn,
                                                 const Item* __restrict__ items, int nitems) {
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const Item I = items[it];
    const RunDesc& R = runs[I.run];
    const int pid = I.a * blockDim.x + threadIdx.x;
    if (pid >= R.N) continue;
    const float2 Fw = R.Fw[pid], Fk = R.Fk[pid], xi = R.Fn[pid];
    float bnd = fminf(dt_bound(Fw.x + Fk.x, xi.x, R.mrd, R.T), dt_bound(Fw.y + Fk.y, xi.y, R.mrd, R.T));
    if (!(bnd >= 0.f)) bnd = 3.0e38f;
    if (bnd < R.dt_max) atomicMin(&dyn[I.run].dt_bits, __float_as_uint(bnd));
  }
}

// Green's function tables in FP64 (kapkraefte_init and G,
// dynamik_methoden.cpp:585-593, 1384-1394), stored FP32:
//   green[ky][kx] = kapillar_vorfaktor * G(kx, ky) / Z^2, ky in [0, Z/2] (stored by
//   column, so a column pass reads it contiguously)
//   sxt[kx] = sin(qx dx)/dx, syt[ky] = sin(qy dx)/dx
__global__ void k_green(float* __restrict__ green, float* __restrict__ sxt,
                        float* __restrict__ syt, int Z, double kap, double lambda, double L) {
  const int n = Z / 2;
  const double dx = L / Z, dq = 2.0 * 3.14159265358979323846 / L;
  const long long total = (long long)Z * (n + 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int ky = (int)(i / Z), kx = (int)(i - (long long)ky * Z);
    const double qx = dq * (((kx + n) % Z) - 0.5 * Z);
    const double qy = dq * (((ky + n) % Z) - 0.5 * Z);
    double G;
    if (kx == 0 && ky == 0 && lambda > 0.2 * L) G = 0.0;
    else {
      const double sx = sin(0.5 * qx * dx), sy = sin(0.5 * qy * dx);
      G = 1.0 / (4 * sx * sx / dx / dx + 4 * sy * sy / dx / dx + 1.0 / (lambda * lambda));
    }
    green[i] = (float)(kap * G / Z / Z);
    if (ky == 0) sxt[kx] = (float)(sin(qx * dx) / dx);
    if (kx == 0) syt[ky] = (float)(sin(qy * dx) / dx);
  }
}

// ---------------------------------------------------------------------------
// Fused step: one run on a power-of-two mesh up to 1024^2 with a fixed dt.
// Every stage of the step runs in one cooperative launch (all CTAs
// resident), separated by grid-wide barriers: the launch and drain gaps
// between the stage kernels disappear, which is most of a step's time on
// meshes this small. Data written within the launch is read
// with plain (coherent) loads, never through the read-only cache.

constexpr unsigned BAR_MAX_POLLS = 1u << 22;
// set in the arrival counter by a CTA whose wait gave up: every CTA that
// sees it fails the barrier
constexpr unsigned BAR_POISON = 0x80000000u;

// Grid-wide barrier: bar[0] counts arrivals (a release add; waiters poll it
// with acquire loads until it reaches target = barriers so far x grid), so
// the writes of every CTA before the barrier are visible to all after it.
// bar[1] counts CTAs leaving the launch; the last one clears both words for
// the next launch. A wait gives up after max_polls polls: it sets the poison
// bit with a compare-and-swap that succeeds only while the count is short of
// the target, so either the last arrival comes first and every CTA passes,
// or the poison comes first and every CTA (late arrivals included) fails
// this barrier and returns: no CTA runs past a failed barrier. The failure
// is reported as E_BARRIER_TIMEOUT; the host clears the words.
__device__ bool grid_barrier(unsigned* bar, unsigned target, unsigned max_polls, int* err, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> c(bar[0]);
    c.fetch_add(1u, cuda::memory_order_release);
    int ok = 1;
    for (unsigned polls = 0;; polls++) {
      unsigned v = c.load(cuda::memory_order_acquire);
      if (v & BAR_POISON) {
        ok = 0;
        break;
      }
      if (v >= target) break;
      if (polls >= max_polls) {
        while (!(v & BAR_POISON) && v < target)
          if (c.compare_exchange_weak(v, v | BAR_POISON, cuda::memory_order_acq_rel, cuda::memory_order_acquire))
            v |= BAR_POISON;
        if (v & BAR_POISON) {
          ok = 0;
          atomicOr(err, E_BARRIER_TIMEOUT);
        }
        break;
      }
      __nanosleep(20);
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

__device__ void grid_exit(unsigned* bar) {
  if (threadIdx.x == 0 && atomicAdd(&bar[1], 1u) == gridDim.x - 1) {
    atomicExch(&bar[0], 0u);
    atomicExch(&bar[1], 0u);
  }
}

constexpr size_t FUSED_TW_BYTES(int lz) { return (((size_t)8 << lz) + 255) & ~(size_t)255; }

// The run's description is a kernel parameter (constant bank), so its fields
// take no registers across the phases.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bring this CTA's share (1/G, 256-byte aligned pieces) of a device array
// into L2 with one bulk prefetch (no data moves to the SM; the base must be
// 16-byte aligned, as cudaMalloc's are). Issued by one thread.
__device__ __forceinline__ void l2_prefetch_share(const void* base, size_t bytes, int b, int G) {
  const size_t per = ((bytes + G - 1) / G + 255) & ~(size_t)255;
  const size_t off = (size_t)b * per;
  if (off >= bytes) return;
  const size_t len = (bytes - off < per ? bytes - off : per) & ~(size_t)15;
  if (len == 0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char*)base + off), "r"((unsigned)len)
               : "memory");
}

// ts (optional, FUSED_PHASES + 1 entries): CTA 0 records the global timer
// at the start and after every phase's barrier.
template <int LZ>
__global__ void __launch_bounds__(256, 2) k_fused(const __grid_constant__ RunDesc R, RunDyn* __restrict__ dyn,
                                               const __grid_constant__ FusedPlan P, unsigned* bar,
                                               unsigned long long* ts) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_tmp[32];
  __shared__ int s_ok;
  constexpr int Z = 1 << LZ;
  RunDyn& D = dyn[0];
  volatile RunDyn& Dv = dyn[0];
  // the spectrum rows of this CTA's inverse row item go to L2 first, then the
  // twiddles are requested together with the step budget (independent loads,
  // all from DRAM after the caches were flushed)
  if (threadIdx.x == 0 && (int)blockIdx.x < P.nri)
    l2_prefetch_share(R.spec2 + ((size_t)blockIdx.x << P.lri) * (Z / 2), ((size_t)1 << P.lri) * (Z / 2) * sizeof(float4),
                      0, 1);
  constexpr int TWR = (Z + 255) / 256;
  float2 twr[TWR];
#pragma unroll
  for (int k = 0; k < TWR; k++)
    if (threadIdx.x + 256 * k < Z) twr[k] = R.tw[threadIdx.x + 256 * k];
  // the budget is checked after the inverse row pass (which only rebuilds
  // the force grid from the unchanged spectrum), so its load does not hold up
  // the start; nothing in this launch changes it before the end
  const long long steps_left = Dv.steps_left;
  // What the later phases read first from memory (particles, cell starts and
  // counts in the particle pass, and the density accumulator its move adds
  // to; the Green's tables in the column pass) is requested into L2 now,
  // behind the inverse row pass.
  if (threadIdx.x == 0) {
    const int nZ = (1 << LZ) / 2 + 1;
    l2_prefetch_share(R.green, (size_t)(1 << LZ) * nZ * sizeof(float), blockIdx.x, gridDim.x);
    l2_prefetch_share(R.recA, (size_t)R.N * sizeof(Rec), blockIdx.x, gridDim.x);
    l2_prefetch_share(R.start, ((size_t)R.C * R.C + 1) * sizeof(int), blockIdx.x, gridDim.x);
    l2_prefetch_share(R.count, (size_t)R.C * R.C * sizeof(int), blockIdx.x, gridDim.x);
    l2_prefetch_share(R.dacc, ((size_t)1 << (2 * LZ)) * sizeof(unsigned long long), blockIdx.x, gridDim.x);
    if (blockIdx.x == 0) {
      l2_prefetch_share(R.sxt, (size_t)(1 << LZ) * sizeof(float), 0, 1);
      l2_prefetch_share(R.syt, (size_t)nZ * sizeof(float), 0, 1);
    }
  }
  float2* tws = (float2*)smem;
  float2* work = (float2*)(smem + FUSED_TW_BYTES(LZ));
#pragma unroll
  for (int k = 0; k < TWR; k++)
    if (threadIdx.x + 256 * k < Z) tws[threadIdx.x + 256 * k] = twr[k];
  const unsigned G = gridDim.x;
  // each CTA takes an equal contiguous share of the particles (the busiest
  // SM then holds two shares, not two full CTAs of 256 while others hold one)
  const int per = (R.N + (int)G - 1) / (int)G;
  const int ncells = R.C * R.C;
  const int b = blockIdx.x;
  unsigned ep = 0;
  int ph = 0;
  const bool rec = ts && b == 0 && threadIdx.x == 0;
  if (rec) ts[ph] = global_ns();
  const unsigned maxp = P.max_polls ? P.max_polls : BAR_MAX_POLLS;
  // next grid barrier; false: it failed, the CTA returns. The recovery-path
  // test makes one CTA leave instead of arriving (CTA-uniform condition).
  auto barrier = [&]() -> bool {
    if (P.skip_barrier == (int)ep + 1 && b == P.skip_cta) return false;
    return grid_barrier(bar, ++ep * G, maxp, &D.err, &s_ok);
  };
#define BD_BARRIER()        \
  if (!barrier()) return; \
  if (rec) ts[++ph] = global_ns()
  // The mesh transform is pipelined across the step boundary: this step's
  // density was deposited by the previous step's move and its forward row
  // and column passes ran beside that step's scan and scatter (or, after the
  // positions changed elsewhere, the host ran them before this launch). The
  // step starts at the inverse row pass. A transform item runs at most once
  // per call site and CTA (the host sizes them so; a loop around a transform
  // would make the compiler keep the addresses of all its passes live).
  if (b < P.nri) fft2_rows_inv_item<LZ, true>(R, b << P.lri, P.lri, work, tws);
  BD_BARRIER();
  if (steps_left <= 0) {  // uniform
    grid_exit(bar);
    return;
  }
  // forces, noise, move, re-binning, counts, the next step's density
  for (int i = threadIdx.x; i < per; i += blockDim.x) {
    const int gi = b * per + i;
    if (gi < R.N) particle_item<false, true>(R, D, gi, MODE_STEP, 7);
  }
  BD_BARRIER();
  // chunk offsets: each CTA sums the totals before its chunk (few chunks),
  // else CTA 0 scans them first
  const bool own = P.nch <= 512;
  if (!own) {
    if (b == 0) {
      int loc = 0;
      const int per = (P.nch + blockDim.x - 1) / blockDim.x, k0 = threadIdx.x * per;
      for (int k = 0; k < per; k++)
        if (k0 + k < P.nch) loc += R.chunk_sum[k0 + k];
      int ex = block_excl_scan(loc, s_tmp);
      for (int k = 0; k < per; k++)
        if (k0 + k < P.nch) {
          const int v = R.chunk_sum[k0 + k];
          R.chunk_off[k0 + k] = ex;
          ex += v;
        }
    }
    if (!barrier()) return;
  }
  for (int c = b; c < P.nch; c += G) {
    int off;
    if (own) {
      int loc = 0;
      for (int k = threadIdx.x; k < c; k += blockDim.x) loc += R.chunk_sum[k];
      const int ex = block_excl_scan(loc, s_tmp);
      __syncthreads();  // every thread has read s_tmp
      if (threadIdx.x == blockDim.x - 1) s_tmp[0] = ex + loc;
      __syncthreads();
      off = s_tmp[0];
      __syncthreads();
    } else {
      off = R.chunk_off[c];
    }
    constexpr int PER = SCAN_CHUNK / 256;
    const int c0 = c * SCAN_CHUNK + threadIdx.x * PER;
    int v[PER];
#pragma unroll
    for (int k = 0; k < PER; k++) v[k] = c0 + k < ncells ? R.count[c0 + k] : 0;
    scan_chunk_store(R, c, ncells, v, off, s_tmp);
  }
  // beside the scan: the next step's forward row pass over the density the
  // move deposited (items on the CTAs from the top down, the scan's chunks
  // are on the lowest)
  {
    const int it = (int)G - 1 - b;
    if (it < P.nrf) fft2_rows_fwd_item<LZ, true, true>(R, it << P.lrf, P.lrf, work, tws);
  }
  BD_BARRIER();
  for (int i = threadIdx.x; i < per; i += blockDim.x) {
    const int gi = b * per + i;
    if (gi < R.N) scatter_particle(R, gi);
  }
  // beside the scatter: the next step's column pass and Green's multiply
  {
    const int it = (int)G - 1 - b;
    if (it < P.ncl) fft2_cols_item<LZ, true>(R, it << P.lw, P.lw, work, tws);
  }
  if (b == 0) {
    for (int k = threadIdx.x; k < P.nch; k += blockDim.x) R.chunk_sum[k] = 0;
    if (threadIdx.x == 0) end_step(R, D, 0);
  }
  if (ts) {
    // the last phase ends when every CTA has scattered and transformed
    if (!barrier()) return;
    if (rec) ts[++ph] = global_ns();
  }
  grid_exit(bar);
#undef BD_BARRIER
}

#define BD_FUSED_SIZES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

int fused_configure(FusedPlan& P, int device) {
  const int Z = 1 << P.lz, n = Z / 2;
  const size_t rf = (size_t)(1 << P.lrf) * fft2_stride(n) * 8;
  const size_t cl = (size_t)2 * (1 << P.lw) * fft2_stride(Z) * 8;
  const size_t ri = (size_t)(1 << P.lri) * fft2_stride(Z) * 8;
  P.smem = FUSED_TW_BYTES(P.lz) + std::max(rf, std::max(cl, ri));
  int nsm = 0, per = 0;
  cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return (int)e;
  switch (P.lz) {
#define BD_CASE(L)                                                                                \
  case L:                                                                                         \
    e = cudaFuncSetAttribute(k_fused<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem); \
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fused<L>, 256, P.smem); \
    break;
    BD_FUSED_SIZES(BD_CASE)
#undef BD_CASE
    default:
      return (int)cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return (int)e;
  if (per <= 0) return (int)cudaErrorInvalidConfiguration;
  // two CTAs per SM: more make every grid barrier slower than they gain
  P.grid = std::min(per, 2) * nsm;
  return 0;
}

int launch_fused(const RunDesc& run, RunDyn* dyn, const FusedPlan& P, unsigned* bar, cudaStream_t s,
                 unsigned long long* ts) {
  cudaError_t e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P.grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = P.smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  RunDesc rd = run;
  rd.dacc = P.dacc;  // only the fused kernel's copy carries the accumulator
  switch (P.lz) {
#define BD_CASE(L)                                                 \
  case L:                                                          \
    e = cudaLaunchKernelEx(&cfg, k_fused<L>, rd, dyn, P, bar, ts); \
    break;
    BD_FUSED_SIZES(BD_CASE)
#undef BD_CASE
    default:
      return (int)cudaErrorInvalidValue;
  }
  return (int)e;
}

// ---------------------------------------------------------------------------
// Two-launch pipelined step (any number of runs on power-of-two meshes with a
// fixed dt): the particle kernel, then one cooperative launch that holds the
// rest of the step and the start of the next, its phases separated by grid
// barriers:
//   C  scan chunks and the next forward row items (of the runs the particle
//      kernel marked as taking part)
//   D  scatter (PIPE_SCATTER_UNIT particles per unit) and the next column +
//      Green items; chunk totals cleared and steps ended
//   A  inverse row items of the runs that took part (the next step's force
//      grids; a run that did not keeps its spectrum and its grids)
// Unit u of a phase goes to CTA u mod G. The host interleaves transform
// items with scan chunks (and with scatter units) in one list, so every CTA
// holds a share of both kinds and on every SM the latency-bound transforms
// run beside the bandwidth-bound sort, which two kernels on two streams did
// not: the first kernel's CTAs filled the GPU before the second's started.


// meshes of the two-launch form (the host keeps larger ones on six launches)
#define BD_TAIL_FFT_SIZES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)

// A transform item called from the unit loops: not inlined, so the compiler
// cannot hoist the per-thread offsets and twiddle addresses of every pass
// and mesh size out of the loop (kept live across it, they spill).
// The dynamic shared memory is named here, not passed: a pointer parameter
// would be generic and every transform access a generic load.
template <int PASS, int L>
__device__ __noinline__ void tail_fft_sized(const RunDesc* R, int a, int c) {
  extern __shared__ __align__(16) unsigned char smem[];
  float2* s = (float2*)smem;
  if (PASS == 0) fft2_rows_inv_item<L, false>(*R, a, c, s, R->tw);
  else if (PASS == 1) fft2_rows_fwd_item<L, false, true>(*R, a, c, s, R->tw);
  else fft2_cols_item<L, false>(*R, a, c, s, R->tw);
}

template <int PASS>
__device__ __forceinline__ void tail_fft_item(const RunDesc* R, const Item& I) {
  switch (I.b) {
#define BD_CASE(L)                                \
  case L:                                         \
    tail_fft_sized<PASS, L>(R, I.a, I.c);         \
    break;
    BD_TAIL_FFT_SIZES(BD_CASE)
#undef BD_CASE
    default:
      break;
  }
}

// ts (optional, 4 entries): CTA 0 records the global timer at the start and
// after phases C, D and A (a barrier closes A when ts is given).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_pipe_tail(const RunDesc* __restrict__ runs, RunDyn* dyn,
                                                          const __grid_constant__ PipeTail P, unsigned* bar,
                                                          unsigned long long* ts) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_tmp[32];
  __shared__ int s_ok;
  const unsigned G = gridDim.x;
  const int b = blockIdx.x, nt = blockDim.x;
  unsigned ep = 0;
  const bool rec = ts && b == 0 && threadIdx.x == 0;
  if (rec) ts[0] = global_ns();
  const unsigned maxp = P.max_polls ? P.max_polls : BAR_MAX_POLLS;
  // which runs take part in this step: recorded by the particle kernel
  // before this launch; read with volatile loads (the run's state line may
  // sit in this SM's L1 while the step end in phase D changes it)
  volatile const RunDyn* dv = dyn;
  for (int u = b; u < P.ncu; u += G) {
    const Item I = P.cunits[u];
    if (!dv[I.run].sorting) continue;
    const RunDesc& R = runs[I.run];
    if (I.b < 0) scan_chunk_item(R, I.a, s_tmp);
    else tail_fft_item<1>(&R, I);
  }
  if (!grid_barrier(bar, ++ep * G, maxp, &dyn[0].err, &s_ok)) return;
  if (rec) ts[1] = global_ns();
  for (int u = b; u < P.ndu; u += G) {
    const Item I = P.dunits[u];
    if (!dv[I.run].sorting) continue;
    const RunDesc& R = runs[I.run];
    if (I.b < 0) scatter_unit(R, I.a);
    else tail_fft_item<2>(&R, I);
  }
  for (int c = b * nt + threadIdx.x; c < P.nchunk; c += (int)G * nt) {
    const Item I = P.chunks[c];
    if (!dv[I.run].sorting) continue;
    runs[I.run].chunk_sum[I.a] = 0;
    if (I.a == 0) end_step(runs[I.run], dyn[I.run], 0);
  }
  if (!grid_barrier(bar, ++ep * G, maxp, &dyn[0].err, &s_ok)) return;
  if (rec) ts[2] = global_ns();
  for (int u = b; u < P.ninv; u += G) {
    const Item I = P.inv[u];
    if (dv[I.run].sorting) tail_fft_item<0>(&runs[I.run], I);
  }
  if (ts) {
    if (!grid_barrier(bar, ++ep * G, maxp, &dyn[0].err, &s_ok)) return;
    if (rec) ts[3] = global_ns();
  }
  grid_exit(bar);
}

#define BD_TAIL_SHAPES(X) X(2) X(3) X(4)

int pipe_tail_configure(PipeTail& P, int device) {
  int nsm = 0, per = 0;
  cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return (int)e;
  switch (P.minb) {
#define BD_CASE(M)                                                                                   \
  case M:                                                                                            \
    e = cudaFuncSetAttribute(k_pipe_tail<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem); \
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pipe_tail<M>, 256, P.smem); \
    break;
    BD_TAIL_SHAPES(BD_CASE)
#undef BD_CASE
    default:
      return (int)cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return (int)e;
  if (per <= 0) return (int)cudaErrorInvalidConfiguration;
  P.grid = std::min(per, P.minb) * nsm;
  return 0;
}

int launch_pipe_tail(const RunDesc* runs, RunDyn* dyn, const PipeTail& P, unsigned* bar, cudaStream_t s,
                     unsigned long long* ts) {
  cudaError_t e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P.grid);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = P.smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  switch (P.minb) {
#define BD_CASE(M)                                                         \
  case M:                                                                  \
    e = cudaLaunchKernelEx(&cfg, k_pipe_tail<M>, runs, dyn, P, bar, ts); \
    break;
    BD_TAIL_SHAPES(BD_CASE)
#undef BD_CASE
    default:
      return (int)cudaErrorInvalidValue;
  }
  return (int)e;
}

// ---------------------------------------------------------------------------
// TimestepInfo diagnostics (zeitschritt_debug, dynamik_methoden.cpp:168-211,
// and the *_debug force routines) plus the WCA potential energy and virial
// in FP64. One thread per particle of the sorted array, after the forces of
// the current positions are in Fw/Fk/Fn (per particle index):
//  - the largest |F| of each force kind, as (|F|^2 bits << 32 | index) maxima;
//  - the pairs the reference's WCA loops examine: same-species neighbours of
//    every particle (i != j) and type-2 neighbours of every type-1 particle
//    (berechne_WCA11/22 and addiere_WCA12 loop over the 3x3 cells);
//  - over all pairs within the cutoff, each seen from both ends and halved:
//    U = 4 eps (s^-12 - s^-6) + eps with s = r*sigma (the potential whose
//    gradient is the uncapped WCA force), and r.F with the force the step
//    uses (capped at maxPairWCA).
struct DiagAcc {
  double energy, virial;
  unsigned long long maxF[3];  // WCA, capillary, noise
  unsigned long long pairs;
};

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

__global__ void __launch_bounds__(256) k_diag(const RunDesc* __restrict__ runs, DiagAcc* __restrict__ acc) {
  const RunDesc& R = runs[0];
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, w = 0.0;
  unsigned long long pairs = 0, mx[3] = {0, 0, 0};
  if (gi < R.N) {
    const Rec p = R.recA[gi];
    const float2* Fs[3] = {R.Fw, R.Fk, R.Fn};
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float2 f = Fs[k][p.pid];
      const float m = f.x * f.x + f.y * f.y;
      mx[k] = ((unsigned long long)__float_as_uint(m) << 32) | (unsigned)p.pid;
    }
    if (!(R.flags & F_IDGAS)) {
      const int C = R.C;
      int ic, jc;
      cell_ij(R, p.cell, ic, jc);
      const bool sp = p.pid >= R.N1;
      for (int da = -1; da <= 1; da++) {
        const int row = wrap1(ic + da, C) * C;
        for (int db = -1; db <= 1; db++) {
          const int g = row + wrap1(jc + db, C);
          for (int j = R.start[g]; j < R.start[g + 1]; j++) {
            if (j == gi) continue;
            const Rec q = R.recA[j];
            const bool sq = q.pid >= R.N1;
            if (sp == sq || !sp) pairs++;
            const int t = sp == sq ? (sp ? 1 : 0) : 2;
            double dx = ((double)p.ox - (double)q.ox) - da * R.B_d;
            double dy = ((double)p.oy - (double)q.oy) - db * R.B_d;
            if (R.flags & F_SMALLBOX) {
              dx -= R.L_d * rint(dx / R.L_d);
              dy -= R.L_d * rint(dy / R.L_d);
            }
            const double sig = R.wsig[t];
            const double a2s = (dx * dx + dy * dy) * sig * sig;
            if (a2s > (double)R.cut2) continue;
            const double eps = (double)R.wpre[t] / (24.0 * sig);
            const double i2 = 1.0 / a2s, i6 = i2 * i2 * i2;
            e += 4.0 * eps * (i6 * i6 - i6) + eps;
            double f = (double)R.wpre[t] * i6 * i2 * (2.0 * i6 - 1.0);  // 24 eps sigma (2 s^-14 - s^-8)
            if (f > (double)R.maxPair) f = R.maxPair;
            w += f * a2s / sig;  // r . F = f * sigma * r^2
          }
        }
      }
    }
  }
  // block reductions, one atomic per block and quantity
  __shared__ double s_e[8], s_w[8];
  __shared__ unsigned long long s_p[8], s_m[3][8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    w += __shfl_xor_sync(0xffffffffu, w, o);
    pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) mx[k] = warp_max_u64(mx[k]);
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_e[wid] = e;
    s_w[wid] = w;
    s_p[wid] = pairs;
    for (int k = 0; k < 3; k++) s_m[k][wid] = mx[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double te = 0.0, tw = 0.0;
    unsigned long long tp = 0, tm[3] = {0, 0, 0};
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
      te += s_e[k];
      tw += s_w[k];
      tp += s_p[k];
      for (int q = 0; q < 3; q++) tm[q] = s_m[q][k] > tm[q] ? s_m[q][k] : tm[q];
    }
    atomicAdd(&acc->energy, 0.5 * te);
    atomicAdd(&acc->virial, 0.5 * tw);
    atomicAdd(&acc->pairs, tp);
    for (int q = 0; q < 3; q++) atomicMax(&acc->maxF[q], tm[q]);
  }
}

int launch_diag(const RunDesc* runs, int N, void* acc, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(DiagAcc), s);
  if (e != cudaSuccess) return (int)e;
  k_diag<<<(N + 255) / 256, 256, 0, s>>>(runs, (DiagAcc*)acc);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

size_t diag_bytes() { return sizeof(DiagAcc); }

// ---------------------------------------------------------------------------
// Observables computed from the resident state (the reference's in-run
// auswertung.cpp, validation tools here).

// Pair-distance histogram for g11 / g12 / g22 (record_korrelationsfunktion11/
// 12/22, auswertung.cpp:110-188): every pair once (11, 22: the lower particle
// index of the pair counts; 12: type 1 against type 2), minimum-image
// distance in FP64 from the cell and offset, bin (int)(r / dr). One thread
// per particle of the sorted array searches the cells within `range` of its
// own (the whole box when the range covers it); the CTA counts in shared
// memory and adds to hist[bins] once.
__global__ void __launch_bounds__(256) k_korr(const RunDesc* __restrict__ runs, int which, int bins, double dr,
                                              int range, unsigned long long* __restrict__ hist) {
  extern __shared__ unsigned sh_hist[];
  const RunDesc& R = runs[0];
  for (int b = threadIdx.x; b < bins; b += blockDim.x) sh_hist[b] = 0u;
  __syncthreads();
  const int C = R.C;
  const bool all_rows = 2 * range + 1 >= C;
  for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < R.N; gi += gridDim.x * blockDim.x) {
    const Rec p = R.recA[gi];
    const int si = p.pid >= R.N1;
    if ((which == 0 && si != 0) || (which == 1 && si != 0) || (which == 2 && si != 1)) continue;
    const int want = which == 1 ? 1 : si;
    int ic, jc;
    cell_ij(R, p.cell, ic, jc);
    const double xi = ic * R.B_d + (double)p.ox, yi = jc * R.B_d + (double)p.oy;
    const int nrows = all_rows ? C : 2 * range + 1;
    for (int a = 0; a < nrows; a++) {
      const int row = all_rows ? a : wrapi(ic - range + a, C);
      // columns jc-range .. jc+range as at most two contiguous runs
      int segs[2][2];
      int ns = 1;
      if (all_rows) {
        segs[0][0] = 0, segs[0][1] = C;
      } else {
        const int j0 = wrapi(jc - range, C), len = 2 * range + 1;
        if (j0 + len <= C) {
          segs[0][0] = j0, segs[0][1] = j0 + len;
        } else {
          segs[0][0] = j0, segs[0][1] = C, segs[1][0] = 0, segs[1][1] = j0 + len - C;
          ns = 2;
        }
      }
      for (int sgi = 0; sgi < ns; sgi++) {
        const int beg = R.start[row * C + segs[sgi][0]], end = R.start[row * C + segs[sgi][1]];
        for (int j = beg; j < end; j++) {
          const Rec q = R.recA[j];
          const int sj = q.pid >= R.N1;
          if (sj != want) continue;
          if (which != 1 && q.pid >= p.pid) continue;  // each pair once
          int qi, qj;
          cell_ij(R, q.cell, qi, qj);
          double dx = xi - (qi * R.B_d + (double)q.ox);
          double dy = yi - (qj * R.B_d + (double)q.oy);
          dx -= R.L_d * rint(dx / R.L_d);
          dy -= R.L_d * rint(dy / R.L_d);
          const int idx = (int)(sqrt(dx * dx + dy * dy) / dr);
          if (idx >= 0 && idx < bins) atomicAdd(&sh_hist[idx], 1u);
        }
      }
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < bins; b += blockDim.x)
    if (sh_hist[b]) atomicAdd(&hist[b], (unsigned long long)sh_hist[b]);
}

// Density Fourier sums of one species on the lattice k = dq (i, j),
// 0 <= i, j < qbins, i^2 + j^2 <= qbins^2 (record_ftrho_unkorrigiert,
// auswertung.cpp:307-380): re + i im = sum over particles of exp(i k.r), in
// FP64. Each thread owns up to FT_KPT lattice points and sums over the
// particles its CTA stages in shared memory; one atomic add per CTA and point.
constexpr int FT_KPT = 16;
__global__ void __launch_bounds__(256) k_ftrho(const RunDesc* __restrict__ runs, int species, int qbins, double dq,
                                               double* __restrict__ re, double* __restrict__ im) {
  __shared__ double sx[256], sy[256];
  __shared__ int sn;
  const RunDesc& R = runs[0];
  const int nk = qbins * qbins;
  double ar[FT_KPT], ai[FT_KPT];
#pragma unroll
  for (int m = 0; m < FT_KPT; m++) ar[m] = ai[m] = 0.0;
  for (int base = blockIdx.x * 256; base < R.N; base += gridDim.x * 256) {
    if (threadIdx.x == 0) sn = 0;
    __syncthreads();
    const int gi = base + threadIdx.x;
    if (gi < R.N) {
      const Rec p = R.recA[gi];
      if ((p.pid >= R.N1) == (species == 1)) {
        int ic, jc;
        cell_ij(R, p.cell, ic, jc);
        const int slot = atomicAdd(&sn, 1);
        sx[slot] = ic * R.B_d + (double)p.ox;
        sy[slot] = jc * R.B_d + (double)p.oy;
      }
    }
    __syncthreads();
    const int n = sn;
#pragma unroll
    for (int m = 0; m < FT_KPT; m++) {
      const int k = threadIdx.x + m * 256;
      if (k >= nk) break;
      const int i = k / qbins, j = k - (k / qbins) * qbins;
      if (i * i + j * j > qbins * qbins) continue;
      for (int t = 0; t < n; t++) {
        double sn_, cs;
        sincos(dq * (sx[t] * i + sy[t] * j), &sn_, &cs);
        ar[m] += cs;
        ai[m] += sn_;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int m = 0; m < FT_KPT; m++) {
    const int k = threadIdx.x + m * 256;
    if (k >= nk) break;
    if (ar[m] != 0.0 || ai[m] != 0.0) {
      atomicAdd(&re[k], ar[m]);
      atomicAdd(&im[k], ai[m]);
    }
  }
}

int launch_korr(const RunDesc* runs, int N, int which, int bins, double dr, int range, unsigned long long* hist,
                cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)bins * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return (int)e;
  const int grid = std::max(1, std::min((N + 255) / 256, 148 * 8));
  k_korr<<<grid, 256, (size_t)bins * sizeof(unsigned), s>>>(runs, which, bins, dr, range, hist);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

int launch_ftrho(const RunDesc* runs, int N, int species, int qbins, double dq, double* re, double* im,
                 cudaStream_t s) {
  const size_t nk = (size_t)qbins * qbins;
  cudaError_t e = cudaMemsetAsync(re, 0, nk * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(im, 0, nk * sizeof(double), s);
  if (e != cudaSuccess) return (int)e;
  const int grid = std::max(1, std::min((N + 255) / 256, 148 * 4));
  k_ftrho<<<grid, 256, 0, s>>>(runs, species, qbins, dq, re, im);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// Local densities of the offline analysis (main_auswertung.cpp:182-390),
// from the resident state. Lattice of n x n cells of width w = L/n; each
// particle adds w_x w_y drho (drho = 1/w^2) to nine cells with FP64 atomic
// adds. A fixed-point sum would be order-independent, but its absolute
// resolution turns cells holding only the tail of a TSC weight (values near
// 1e-19) into empty cells, and the reference counts such a cell in the
// |rho1 - rho2| / rho thresholds; FP64 adds keep every cell's value to a few
// ulp of itself. All weight arithmetic is written with explicit
// round-to-nearest operations, so no product is fused into a following add
// and each contribution equals the reference's FP64 expression.
__device__ __forceinline__ void snap_tsc(double x, double w, int n, int* kk, double* wt) {
  int k = __double2int_rz(__ddiv_rn(x, w));  // (int)(x/width)
  k = k % n;
  if (k < 0) k += n;  // x < 0 (never from the integrator) stays on the lattice
  kk[0] = (k - 1 + n) % n;
  kk[1] = k;
  kk[2] = (k + 1) % n;
  const double d = __dsub_rn(x, __dmul_rn((double)k + 0.5, w));
  wt[1] = __dsub_rn(0.75, __ddiv_rn(__dmul_rn(d, d), __dmul_rn(w, w)));
  double t = 1.5 - fabs(__ddiv_rn(__dadd_rn(d, w), w));
  wt[0] = __dmul_rn(__dmul_rn(0.5, t), t);
  t = 1.5 - fabs(__ddiv_rn(__dsub_rn(d, w), w));
  wt[2] = __dmul_rn(__dmul_rn(0.5, t), t);
}

__global__ void __launch_bounds__(256) k_lokdens(const RunDesc* __restrict__ runs, LdSnap sp,
                                                 double* __restrict__ grid) {
  const RunDesc& R = runs[0];
  const size_t cells = (size_t)sp.n * sp.n;
  for (int gi = blockIdx.x * blockDim.x + threadIdx.x; gi < R.N; gi += gridDim.x * blockDim.x) {
    const Rec p = R.recA[gi];
    const int s = p.pid >= R.N1;
    int ic, jc;
    cell_ij(R, p.cell, ic, jc);
    const double x = __dadd_rn(__dmul_rn((double)ic, R.B_d), (double)p.ox);
    const double y = __dadd_rn(__dmul_rn((double)jc, R.B_d), (double)p.oy);
    int kx[3], ky[3];
    double wx[3], wy[3];
    snap_tsc(x, sp.w, sp.n, kx, wx);
    snap_tsc(y, sp.w, sp.n, ky, wy);
    double* G = grid + s * cells;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++)
        atomicAdd(&G[(size_t)kx[a] * sp.n + ky[b]], __dmul_rn(__dmul_rn(wx[a], wy[b]), sp.drho));
  }
}

// Histogram bin of main_auswertung.cpp:337-355: (int) truncation of v,
// clamped to [0, bins); values at or above bins are clamped before the
// conversion.
__device__ __forceinline__ int snap_bin(double v, int bins) {
  if (v >= (double)bins) return bins - 1;
  const int b = __double2int_rz(v);
  return b < 0 ? 0 : b;
}

// Histograms and threshold counts over the lattice (main_auswertung.cpp:
// 302-390). hist: [4][bins] counts (rho1, rho2, rho1+rho2, rho1-rho2), then
// [7] threshold counts.
__global__ void __launch_bounds__(256) k_rhohist(const LdHist hp, const double* __restrict__ grid,
                                                 unsigned* __restrict__ hist) {
  extern __shared__ unsigned sh_rh[];
  const int bins = hp.bins, nb = 4 * bins + 7;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sh_rh[i] = 0u;
  __syncthreads();
  const size_t cells = (size_t)hp.n * hp.n;
  unsigned over[7] = {0u, 0u, 0u, 0u, 0u, 0u, 0u};
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
    const double rho1 = grid[c], rho2 = grid[cells + c];
    const double rho = __dadd_rn(rho1, rho2), drho = __dsub_rn(rho1, rho2);
#pragma unroll
    for (int t = 0; t < 3; t++) over[t] += rho > hp.rho_thresh[t];
    const double q = __ddiv_rn(fabs(drho), rho);  // 0/0 for an empty cell: never over
#pragma unroll
    for (int t = 0; t < 4; t++) over[3 + t] += q > hp.drho_thresh[t];
    atomicAdd(&sh_rh[0 * bins + snap_bin(__dsub_rn(__ddiv_rn(rho1, hp.dbin), 0.5), bins)], 1u);
    atomicAdd(&sh_rh[1 * bins + snap_bin(__dsub_rn(__ddiv_rn(rho2, hp.dbin), 0.5), bins)], 1u);
    atomicAdd(&sh_rh[2 * bins + snap_bin(__dsub_rn(__ddiv_rn(rho, hp.dbin), 0.5), bins)], 1u);
    atomicAdd(&sh_rh[3 * bins + snap_bin(__dadd_rn(__dsub_rn(__ddiv_rn(drho, hp.dbin), 0.5), (double)(bins / 2)),
                                         bins)],
              1u);
  }
#pragma unroll
  for (int t = 0; t < 7; t++) {
    const unsigned v = __reduce_add_sync(0xffffffffu, over[t]);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&sh_rh[4 * bins + t], v);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    if (sh_rh[i]) atomicAdd(&hist[i], sh_rh[i]);
}

int launch_lokdens(const RunDesc* runs, int N, const LdSnap& sp, const LdHist& hp, double* grid, unsigned* hist,
                   cudaStream_t s) {
  const size_t cells = (size_t)sp.n * sp.n;
  cudaError_t e = cudaMemsetAsync(grid, 0, 2 * cells * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, (4 * (size_t)hp.bins + 7) * sizeof(unsigned), s);
  if (e != cudaSuccess) return (int)e;
  if (N > 0) k_lokdens<<<std::max(1, std::min((N + 255) / 256, 148 * 8)), 256, 0, s>>>(runs, sp, grid);
  const int g2 = (int)std::max<size_t>(1, std::min<size_t>((cells + 255) / 256, 148 * 4));
  k_rhohist<<<g2, 256, (4 * (size_t)hp.bins + 7) * sizeof(unsigned), s>>>(hp, grid, hist);
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// ---------------------------------------------------------------------------
// host-side launchers

#define BD_LAUNCH_CHECK()                                                                    \
  do {                                                                                       \
    cudaError_t e__ = cudaGetLastError();                                                    \
    if (e__ != cudaSuccess) {                                                                \
      std::fprintf(stderr, "bd: %s:%d: launch: %s\n", __FILE__, __LINE__, cudaGetErrorString(e__)); \
      return (int)e__;                                                                       \
    }                                                                                        \
  } while (0)

static inline int grid_for(int n, int cap) { return n < cap ? (n > 0 ? n : 1) : cap; }

// SMs of the current device (asked once per device)
static int sm_count() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

size_t deposit_smem(int mt_max, int rows_max) {
  return (size_t)mt_max * mt_max * 8 + (size_t)(3 * 2 * rows_max + 4) * 4;  // lo + hi words, segments
}

int launch_deposit(const RunDesc* runs, const RunDyn* dyn, const Item* items, int n, int mt_max,
                   int rows_max, int scheme_override, int require_active, cudaStream_t s) {
  if (n <= 0) return 0;
  const size_t sm = deposit_smem(mt_max, rows_max);
  k_deposit<<<grid_for(n, 65535), 256, sm, s>>>(runs, dyn, items, n, scheme_override, require_active);
  BD_LAUNCH_CHECK();
  return 0;
}

// the power-of-two kernels of every mesh size 8..4096, by log2(Z)
#define BD_FFT2_SIZES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)

static int launch_fft2(int pass, int lz, const RunDesc* runs, const RunDyn* dyn, const FftPass& p,
                       int require_active, cudaStream_t s) {
  if (p.n <= 0) return 0;
  switch (lz) {
#define BD_CASE(L)                                                                                      \
  case L:                                                                                               \
    if (pass == 0)                                                                                      \
      k_fft2_rows_fwd<L><<<p.n, p.threads, p.smem, s>>>(runs, dyn, p.items, p.n, require_active);      \
    else if (pass == 1)                                                                                 \
      if (p.threads > FFT2_THREADS)                                                                      \
        k_fft2_cols_wide<L><<<p.n, p.threads, p.smem, s>>>(runs, dyn, p.items, p.n, require_active);   \
      else                                                                                              \
        k_fft2_cols<L><<<p.n, p.threads, p.smem, s>>>(runs, dyn, p.items, p.n, require_active);        \
    else                                                                                                \
      k_fft2_rows_inv<L><<<p.n, p.threads, p.smem, s>>>(runs, dyn, p.items, p.n, require_active);      \
    break;
    BD_FFT2_SIZES(BD_CASE)
#undef BD_CASE
    default:
      return (int)cudaErrorInvalidValue;
  }
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_fft(const RunDesc* runs, const RunDyn* dyn, const FftPass gen[3], const Fft2Group* g2, int ng2,
               int require_active, cudaStream_t s, cudaEvent_t* ev, int npass) {
  for (int pass = 0; pass < npass && pass < 3; pass++) {
    const FftPass& g = gen[pass];
    if (g.n > 0) {
      if (pass == 0)
        k_fft_rows_fwd<<<grid_for(g.n, 65535), FFT_THREADS, g.smem, s>>>(runs, dyn, g.items, g.n, require_active);
      else if (pass == 1)
        k_fft_cols<<<grid_for(g.n, 65535), FFT_THREADS, g.smem, s>>>(runs, dyn, g.items, g.n, require_active);
      else
        k_fft_rows_inv<<<grid_for(g.n, 65535), FFT_THREADS, g.smem, s>>>(runs, dyn, g.items, g.n, require_active);
      BD_LAUNCH_CHECK();
    }
    for (int k = 0; k < ng2; k++) {
      const int e = launch_fft2(pass, g2[k].lz, runs, dyn, g2[k].pass[pass], require_active, s);
      if (e) return e;
    }
    if (ev) cudaEventRecord(ev[pass], s);
  }
  return 0;
}

int launch_particles(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, int mode,
                     int mask, int require_active, cudaStream_t s, int deposit, int shape) {
  if (n <= 0) return 0;
  // The pipelined step (deposit): one wave of resident CTAs, each taking
  // items blockIdx.x, +gridDim.x, ... (256-run ensemble: particle phase
  // 0.429 -> 0.407 ms). Otherwise one CTA per item: for one large run the
  // resident wave was slower (0.152 -> 0.190 ms; two waves 0.179).
  // resident CTAs per SM of each shape, asked once per process (every
  // device of one process is taken to be the same GPU model)
  static int resident[2] = {0, 0};
  const int sh = shape == PART_SHAPE_5CTA ? 1 : 0;
  if (!resident[sh]) {
    int per = 0;
    const cudaError_t e = sh ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_particles<5>, 256, 0)
                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_particles<4>, 256, 0);
    resident[sh] = (e == cudaSuccess && per > 0) ? per : 1;
  }
  const int g = deposit ? grid_for(n, resident[sh] * sm_count()) : grid_for(n, 65535);
  if (sh)
    k_particles<5><<<g, 256, 0, s>>>(runs, dyn, items, n, mode, mask, require_active, deposit);
  else
    k_particles<4><<<g, 256, 0, s>>>(runs, dyn, items, n, mode, mask, require_active, deposit);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_pipe_fft(int pass, const RunDesc* runs, RunDyn* dyn, const Item* items, int n, size_t smem,
                    cudaStream_t s) {
  if (n <= 0) return 0;
  if (pass == 0) k_pipe_fft<0><<<n, FFT2_THREADS, smem, s>>>(runs, dyn, items, n);
  else if (pass == 1) k_pipe_fft<1><<<n, FFT2_THREADS, smem, s>>>(runs, dyn, items, n);
  else k_pipe_fft<2><<<n, FFT2_THREADS, smem, s>>>(runs, dyn, items, n);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_pipe_scan(const RunDesc* runs, RunDyn* dyn, const Item* groups, int ngroup, cudaStream_t s) {
  if (ngroup <= 0) return 0;
  k_pipe_scan<<<ngroup, 256, 0, s>>>(runs, dyn, groups, ngroup);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_pipe_scatter(const RunDesc* runs, RunDyn* dyn, const Item* units, int nunit, const Item* chunks,
                        int nchunk, cudaStream_t s) {
  if (nunit + nchunk <= 0) return 0;
  k_pipe_scatter<<<nunit > 0 ? nunit : 1, 256, 0, s>>>(runs, dyn, units, nunit, chunks, nchunk);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_move(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, int require_active,
                int refresh_only, cudaStream_t s) {
  if (n <= 0) return 0;
  k_move<<<grid_for(n, 65535), 256, 0, s>>>(runs, dyn, items, n, require_active, refresh_only);
  BD_LAUNCH_CHECK();
  return 0;
}

// Records in particle-index order (dst[pid] = src[i]), for the copy of a
// run's positions to the host: the host then writes the caller's arrays in
// order instead of at scattered indices.
__global__ void __launch_bounds__(256) k_records_by_pid(const Rec* __restrict__ src, Rec* __restrict__ dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Rec q = src[i];
    if ((unsigned)q.pid < (unsigned)n) dst[q.pid] = q;  // every pid of a run is in [0, n)
  }
}

int launch_records_by_pid(const Rec* src, Rec* dst, int n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_records_by_pid<<<std::min((n + 255) / 256, 4096), 256, 0, s>>>(src, dst, n);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_count(const RunDesc* runs, const Item* items, int n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_count<<<grid_for(n, 65535), 256, 0, s>>>(runs, items, n);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_sort(const RunDesc* runs, RunDyn* dyn, int run0, int nruns, const Item* chunks, int nchunks,
                const Item* parts, int nparts, int end_step_flag, int adaptive, int require_active, cudaStream_t s,
                cudaEvent_t* ev) {
  if (nchunks > 0) {
    k_chunk_scan<<<nruns, 1024, 0, s>>>(runs, dyn, run0, nruns, end_step_flag, adaptive, require_active);
    BD_LAUNCH_CHECK();
    k_scan<<<grid_for(nchunks, 148 * 8), 256, 0, s>>>(runs, dyn, chunks, nchunks, require_active);
    BD_LAUNCH_CHECK();
  }
  if (ev) cudaEventRecord(ev[0], s);
  if (nparts > 0) {
    k_scatter<<<grid_for(nparts, 65535), 256, 0, s>>>(runs, dyn, parts, nparts, require_active);
    BD_LAUNCH_CHECK();
  }
  if (ev) {
    cudaEventRecord(ev[1], s);
    cudaEventRecord(ev[2], s);
  }
  return 0;
}


int launch_interp(const RunDesc* runs, const Item* items, int n, int scheme, cudaStream_t s) {
  if (n <= 0) return 0;
  k_interp<<<grid_for(n, 65535), 256, 0, s>>>(runs, items, n, scheme);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_noise(const RunDesc* runs, const RunDyn* dyn, const Item* items, int n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_noise<<<grid_for(n, 65535), 256, 0, s>>>(runs, dyn, items, n);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_dtbound(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_dtbound<<<grid_for(n, 65535), 256, 0, s>>>(runs, dyn, items, n);
  BD_LAUNCH_CHECK();
  return 0;
}

int launch_green(float* green, float* sxt, float* syt, int Z, double kap, double lambda,
                 double L, cudaStream_t s) {
  const long long total = (long long)Z * (Z / 2 + 1);
  const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
  k_green<<<blocks, 256, 0, s>>>(green, sxt, syt, Z, kap, lambda, L);
  BD_LAUNCH_CHECK();
  return 0;
}

int set_kernel_attributes() {
  cudaError_t e;
  e = cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_fft_rows_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_fft_rows_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
#define BD_ATTR(L)                                                                                     \
  e = cudaFuncSetAttribute(k_fft2_rows_fwd<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM); \
  if (e != cudaSuccess) return (int)e;                                                                  \
  e = cudaFuncSetAttribute(k_fft2_cols<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);     \
  if (e != cudaSuccess) return (int)e;                                                                  \
  e = cudaFuncSetAttribute(k_fft2_cols_wide<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM); \
  if (e != cudaSuccess) return (int)e;                                                                  \
  e = cudaFuncSetAttribute(k_fft2_rows_inv<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM); \
  if (e != cudaSuccess) return (int)e;
  BD_FFT2_SIZES(BD_ATTR)
#undef BD_ATTR
  e = cudaFuncSetAttribute(k_deposit, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_pipe_fft<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_pipe_fft<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_pipe_fft<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, MAX_FFT_SMEM);
  if (e != cudaSuccess) return (int)e;
  return 0;
}

}  // namespace bd

// Density assignment that allocates nothing (bd_gridDensity_noalloc).
//
// Callers that cannot allocate device memory at call time use it: a host that
// runs under a fixed device-memory budget set up front (a memory pool sized
// once, a process that must not grow its footprint while another job shares
// the GPU), or code that must not reach the CUDA allocator from a latency-
// critical path. It is the deposit of bd_gridDensity_NGP/CIC/TSC
// (gridRoutinen.cpp:31-137, 223-343, 451-560) for positions already in device
// memory, with no bd_ctx and none of its cell-sorted state: every particle
// adds its stencil into a file-scope fixed-point accumulator with global
// atomics, and a second pass writes rho. Contributions and the fixed-point
// scale are those of the library's tile deposit, and integer sums do not
// depend on the order of the additions, so rho is identical to the one
// bd_gridDensity_* produces on the same positions.
//
// Scratch: one file-scope __device__ array of BD_NOALLOC_MAX_Z^2 64-bit
// accumulators (8 MiB), shared by every call in the process on that device.
// Each call zeroes the part it uses (and *nskipped) before it deposits, on the
// caller's stream. Two calls that overlap on the device (different streams, or
// different host threads without ordering) race on the array and both results
// are undefined; calls on one stream are ordered and safe.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress while that device is current, once per device and
// process (which may load the module). Make that first call before any stream
// capture begins on that device. The caller's buffers and stream belong to the
// device that is current at the call (rho is checked; BD_ERR_ARG otherwise).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "bd_api.h"
#include "bd_common.cuh"
#include "bd_host.h"

namespace bd {
namespace {

constexpr int kMaxZ = BD_NOALLOC_MAX_Z;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_noalloc_acc[(size_t)kMaxZ * kMaxZ];

std::mutex g_setup_mu;
unsigned long long* g_acc_ptr[kMaxDevices] = {};

__global__ void k_noalloc_zero(unsigned long long* __restrict__ acc, int n, int* nskipped) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[i] = 0ull;
  if (nskipped && blockIdx.x == 0 && threadIdx.x == 0) *nskipped = 0;
}

// One thread per particle (species 1 first, then species 2). Mesh index and
// weights come from the same device functions as the tile deposit; positions
// outside the reference's invariants (0 <= git < C, -B < rel <= 2B) are
// skipped and counted.
__global__ void __launch_bounds__(256) k_noalloc_deposit(const __grid_constant__ RunDesc R, int scheme,
                                                         const int32_t* __restrict__ git1,
                                                         const double* __restrict__ rel1,
                                                         const int32_t* __restrict__ git2,
                                                         const double* __restrict__ rel2, float B,
                                                         unsigned long long* __restrict__ acc,
                                                         int* nskipped) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.N) return;
  const bool s2 = i >= R.N1;
  const int j = s2 ? i - R.N1 : i;
  const int32_t* g = s2 ? git2 : git1;
  const double* r = s2 ? rel2 : rel1;
  const int ic = g[2 * j], jc = g[2 * j + 1];
  const float ox = (float)r[2 * j], oy = (float)r[2 * j + 1];
  const bool ok = ic >= 0 && ic < R.C && jc >= 0 && jc < R.C && ox > -B && ox <= 2.0f * B && oy > -B &&
                  oy <= 2.0f * B;
  if (!ok) {
    if (nskipped) atomicAdd(nskipped, 1);
    return;
  }
  // under the range check above mesh_axis wraps k and l into [0, Z), as the
  // tile deposit relies on
  int k, l;
  float tx, ty;
  mesh_axis(R, ic, ox, k, tx);
  mesh_axis(R, jc, oy, l, ty);
  const float scale = __int_as_float((127 + R.fx_shift) << 23);
  const float q = s2 ? R.q2 : 1.0f;
  if (scheme == NGP) {
    float c = R.drho;
    if (s2) c *= q;
    atomicAdd(&acc[(size_t)k * R.Z + l], (unsigned long long)__float2ll_rn(c * scale));
    return;
  }
  float wx[3], wy[3];
  axis_weights(scheme, tx, wx);
  axis_weights(scheme, ty, wy);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    int kk = k + a - 1;
    kk = kk < 0 ? kk + R.Z : (kk >= R.Z ? kk - R.Z : kk);
#pragma unroll
    for (int b = 0; b < 3; b++) {
      int ll = l + b - 1;
      ll = ll < 0 ? ll + R.Z : (ll >= R.Z ? ll - R.Z : ll);
      float c = wx[a] * wy[b] * R.drho;
      if (s2) c *= q;
      atomicAdd(&acc[(size_t)kk * R.Z + ll], (unsigned long long)__float2ll_rn(c * scale));
    }
  }
}

__global__ void k_noalloc_store(const unsigned long long* __restrict__ acc, int n, int fx_shift,
                                float* __restrict__ rho) {
  const double inv = 1.0 / (double)__int_as_float((127 + fx_shift) << 23);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    rho[i] = (float)((double)(long long)acc[i] * inv);
}

// Device address of the accumulator on the current device, looked up once.
int noalloc_scratch(unsigned long long** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return BD_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return BD_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_acc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_acc);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return BD_ERR_CUDA;
    }
    g_acc_ptr[dev] = (unsigned long long*)p;
  }
  *out = g_acc_ptr[dev];
  return BD_OK;
}

}  // namespace
}  // namespace bd

extern "C" int bd_gridDensity_noalloc(const bd_params* p, int scheme, const int32_t* git1,
                                      const double* rel1, const int32_t* git2, const double* rel2,
                                      float* rho, int* nskipped, void* stream) {
  using namespace bd;
  if (!p || !rho || !git1 || !rel1) return BD_ERR_ARG;
  if (scheme < NGP || scheme > TSC) return BD_ERR_ARG;
  if (p->N2 > 0 && (!git2 || !rel2)) return BD_ERR_ARG;
  const int v = params_validate(p);
  if (v != BD_OK) return v;
  if (p->FFT_samples > kMaxZ) return BD_ERR_UNSUPPORTED;  // mesh larger than the scratch array
  bd_derived dv;
  params_derived(p, &dv);
  // the scalars the tile deposit reads, computed as the engine computes them
  RunDesc R;
  memset(&R, 0, sizeof(R));
  const int C = dv.nachList_Zellen, Z = p->FFT_samples, N = p->N1 + p->N2;
  const double dx = dv.densGrid_Breite;
  R.C = C;
  R.Z = Z;
  R.N = N;
  R.N1 = p->N1;
  R.N2 = p->N2;
  R.invC = (float)(1.0 / C);
  R.z_over_L = (float)(Z / p->L);
  R.q2 = (float)p->f2_f1;
  R.drho = (float)(1.0 / (dx * dx));
  {
    const double unit = (1.0 / (dx * dx)) * std::max(1.0, std::fabs(p->f2_f1));
    const int E = (int)std::floor(30.0 - std::log2(unit));
    R.fx_shift = std::max(-120, std::min(120, E));
  }
  unsigned long long* acc = nullptr;
  const int st = noalloc_scratch(&acc);
  if (st != BD_OK) return st;
  // the scratch belongs to the current device: rho must too (an attribute
  // query, no allocation)
  {
    cudaPointerAttributes a;
    int dev = -1;
    if (cudaPointerGetAttributes(&a, rho) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) {
      cudaGetLastError();
      return BD_ERR_ARG;
    }
    if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != dev) return BD_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int ZZ = Z * Z;
  k_noalloc_zero<<<592, 256, 0, s>>>(acc, ZZ, nskipped);
  k_noalloc_deposit<<<(N + 255) / 256, 256, 0, s>>>(R, scheme, git1, rel1, git2, rel2, (float)dv.nachList_Breite,
                                                    acc, nskipped);
  k_noalloc_store<<<592, 256, 0, s>>>(acc, ZZ, R.fx_shift, rho);
  if (cudaGetLastError() != cudaSuccess) return BD_ERR_CUDA;
  return BD_OK;
}

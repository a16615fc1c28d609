// Engine implementation: per-run device memory, the batched launch plan and
// graph capture of the fused step.
#include "bd_engine.h"

#include <algorithm>
#include <cstdio>
#include <climits>
#include <cmath>
#include <cstring>

#include "bd_fft2.cuh"
#include "bd_host.h"

namespace bd {

int status_from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return BD_OK;
  if (e == cudaErrorMemoryAllocation) return BD_ERR_NOMEM;
  return BD_ERR_CUDA;
}

// a failing CUDA call other than an allocation is reported on stderr with
// its place, then turned into a status
#define CK(x)                                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) {                                                                   \
      if (e_ != cudaErrorMemoryAllocation)                                                     \
        std::fprintf(stderr, "bd: %s:%d: %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
      return status_from_cuda(e_);                                                             \
    }                                                                                          \
  } while (0)
#define RK(x)                                   \
  do {                                          \
    int r_ = (x);                               \
    if (r_ != 0) return r_ > 0 ? BD_ERR_CUDA : r_; \
  } while (0)

static const long long STEPS_UNLIMITED = LLONG_MAX / 4;

// Host -> device copies go through the engine's stream and complete before
// the call returns. A plain cudaMemcpy runs on the legacy stream, which the
// engine's non-blocking stream is not ordered after, and from pageable
// memory it may return before the data lands: a kernel launched next on the
// engine's stream could read the old contents.
static cudaError_t h2d(cudaStream_t s, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}
// the same without the synchronisation, for a group of copies whose host
// buffers outlive the synchronisation that ends the group
static cudaError_t h2d_nosync(cudaStream_t s, void* dst, const void* src, size_t bytes) {
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
}
// device -> host, after everything queued on the engine's stream
static cudaError_t d2h(cudaStream_t s, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

static int build_fft_plan(int n, FftPlan& P) {
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  P.ns = 0;
  int m = n;
  while (m % 4 == 0 && P.ns < 16) P.r[P.ns++] = 4, m /= 4;
  while (m % 2 == 0 && P.ns < 16) P.r[P.ns++] = 2, m /= 2;
  while (m % 3 == 0 && P.ns < 16) P.r[P.ns++] = 3, m /= 3;
  if (m != 1) return -1;
  P.pow2 = 1;
  int mm = n;
  for (int q = 0; q < P.ns; q++) {
    if (P.r[q] == 3) P.pow2 = 0;
    const int h = mm / P.r[q];
    int l = 0;
    while ((1 << l) < h) l++;
    P.lh[q] = l;
    mm = h;
  }
  return 0;
}

// digit-reversal maps of a plan, as fft_pos / fft_freq compute them
static void plan_maps(const FftPlan& P, std::vector<int>& pos_of_freq, std::vector<int>* freq_of_pos) {
  pos_of_freq.assign(P.n, 0);
  if (freq_of_pos) freq_of_pos->assign(P.n, 0);
  for (int k0 = 0; k0 < P.n; k0++) {
    int k = k0, m = P.n, pos = 0;
    for (int q = 0; q < P.ns; q++) {
      m /= P.r[q];
      pos += (k % P.r[q]) * m;
      k /= P.r[q];
    }
    pos_of_freq[k0] = pos;
    if (freq_of_pos) (*freq_of_pos)[pos] = k0;
  }
}

static size_t r256(size_t b) { return (b + 255) & ~(size_t)255; }
static bool pow2(int z) { return z > 0 && (z & (z - 1)) == 0; }
static int ilog2(int z) {
  int l = 0;
  while ((2 << l) <= z) l++;
  return l;
}

// A run can step with the density deposited in the move (fused step or
// pipelined stage step): a power-of-two mesh, a fixed dt, a mesh at all.
static bool deposit_in_move(const bd_params& p) {
  bd_derived dv;
  params_derived(&p, &dv);
  return pow2(p.FFT_samples) && dv.fixed_dt && !p.idgas_only;
}

// launch geometry of one run
static void geometry(RunHost& r) {
  const int Z = r.Z, C = r.C;
  r.mt = 4;
  for (int c : {64, 48, 32, 24, 16, 12, 8, 6, 4})
    if (Z % c == 0) {
      r.mt = c;
      break;
    }
  r.rows_max = std::min(C, (int)std::ceil((r.mt + 2.0) * C / Z) + 6);
  // rows per row-pass item: about 2048 complex values (4 per thread), at
  // most 32 KB of shared memory; build_plan thins items when a launch would
  // have too few of them for the machine
  int lr = 0;
  while ((2 << lr) * (Z / 2) <= 2048 && (2 << lr) * (Z / 2) * 8 <= 32768 && Z % (2 << lr) == 0) lr++;
  r.lrf = lr;
  lr = 0;
  while ((2 << lr) * Z <= 2048 && (2 << lr) * Z * 8 <= 32768 && Z % (2 << lr) == 0) lr++;
  r.lri = lr;
  // columns per column-pass item: 4 (one 32-byte sector per row) when they fit
  int lw = 2;
  while (lw > 0 && ((size_t)2 * ((size_t)Z << lw) * 8 > (size_t)MAX_FFT_SMEM || (Z / 2) % (1 << lw)))
    lw--;
  r.lw = lw;
}

size_t Engine::footprint_of(const bd_params& p) {
  bd_derived dv;
  params_derived(&p, &dv);
  const size_t N = (size_t)p.N1 + p.N2, C = dv.nachList_Zellen, Z = p.FFT_samples;
  const size_t cc = C * C, n = Z / 2;
  size_t b = 0;
  b += 2 * r256(N * sizeof(Rec)) + 3 * r256(N * 8);
  b += r256(cc * 4) + r256((cc + 1) * 4) + 2 * r256(((cc + SCAN_CHUNK - 1) / SCAN_CHUNK) * 4);
  if (!p.idgas_only)
    b += r256(Z * Z * 4) + r256(Z * n * 8) + r256(Z * n * 16) + r256(Z * Z * 8) +
         r256(Z * (n + 1) * 4) + r256(Z * 4) + r256((n + 1) * 4) + r256(Z * 8) +
         2 * r256(Z * 4) + r256(n * 4);
  if (deposit_in_move(p)) b += r256(Z * Z * 8);  // density accumulator
  return b;
}

// a run's arrays go back to the engine's pool in stream order (no device
// synchronisation, the memory stays mapped for the next run)
static void free_run_memory(RunDesc& d, cudaStream_t s) {
  void* ptrs[] = {d.recA, d.recB,  d.count, d.start,    d.chunk_sum, d.chunk_off,
                  d.rho,  d.spec,  d.spec2, d.H,    d.green, d.sxt,      d.syt,
                  d.tw,   d.Fw,    d.Fk,    d.Fn,   d.pos_full, d.freq_full, d.pos_half, d.dacc};
  for (void* q : ptrs)
    if (q) cudaFreeAsync(q, s);
}

Engine::~Engine() {
  drop_graphs();
  for (auto* r : runs) {
    free_run_memory(r->d, stream);
    if (r->d_sort) cudaFreeAsync(r->d_sort, stream);
    delete r;
  }
  if (stream) cudaStreamSynchronize(stream);
  if (h_stage) cudaFreeHost(h_stage);
  if (ev_stage) cudaEventDestroy(ev_stage);
  for (auto& e : ev_piece)
    if (e) cudaEventDestroy(e);
  if (pool) cudaMemPoolDestroy(pool);
  if (d_runs) cudaFree(d_runs);
  if (d_dyn) cudaFree(d_dyn);
  if (d_items) cudaFree(d_items);
  if (d_bar) cudaFree(d_bar);
  for (int k = 0; k < 2; k++) {
    if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
    if (ev_join[k]) cudaEventDestroy(ev_join[k]);
  }
  if (stream2) cudaStreamDestroy(stream2);
  if (stream) cudaStreamDestroy(stream);
}

int Engine::init(int dev) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return BD_ERR_CUDA;
  if (dev < 0 || dev >= n) return BD_ERR_ARG;
  device = dev;
  CK(cudaSetDevice(dev));
  CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&ev_stage, cudaEventDisableTiming));
  for (auto& e : ev_piece) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (int k = 0; k < 2; k++) {
    CK(cudaEventCreateWithFlags(&ev_fork[k], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
  }
  // the runs' arrays come from a stream-ordered pool of this engine that
  // keeps freed memory mapped: runs joining and leaving a served batch then
  // cost no device-wide allocation or synchronisation
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  CK(cudaMemPoolCreate(&pool, &props));
  uint64_t keep = UINT64_MAX;
  CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  RK(set_kernel_attributes());
  return BD_OK;
}

template <class T>
static cudaError_t dalloc(T*& p, size_t n, size_t& acc, cudaMemPool_t pool, cudaStream_t s) {
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  acc += r256(bytes);
  return cudaMallocFromPoolAsync((void**)&p, bytes, pool, s);
}

int Engine::add_run(const bd_params& p, uint64_t seed, RunHost** out) {
  int st = params_validate(&p);
  if (st) return st;
  CK(cudaSetDevice(device));
  RK(download_dyn());  // keep the device state of the runs already there
  tables_ok = false;
  descs_ok = false;
  planned = false;
  drop_graphs();
  auto* r = new RunHost();
  r->p = p;
  r->seed = seed;
  r->gen.seed(seed);
  bd_derived dv;
  params_derived(&p, &dv);
  r->C = dv.nachList_Zellen;
  r->Z = p.FFT_samples;
  r->N = p.N1 + p.N2;
  r->B = dv.nachList_Breite;
  r->dx = dv.densGrid_Breite;
  r->adaptive = !dv.fixed_dt;
  r->idgas = p.idgas_only != 0;
  RunDesc& d = r->d;
  std::memset(&d, 0, sizeof(d));
  d.N1 = p.N1;
  d.N2 = p.N2;
  d.N = r->N;
  d.C = r->C;
  d.Z = r->Z;
  if (build_fft_plan(r->Z / 2, d.plan_half) || build_fft_plan(r->Z, d.plan_full)) {
    delete r;
    return BD_ERR_UNSUPPORTED;
  }
  d.scheme = p.densGrid_Schema;
  d.flags = (p.idgas_only ? F_IDGAS : 0) | (p.noWCA ? F_NOWCA : 0) |
            (p.restrictRadial ? F_RADIAL : 0) | (p.ngp_ref_compat ? F_NGP_REFCOMPAT : 0) |
            (r->adaptive ? F_ADAPTIVE : 0) | (r->C < 7 ? F_SMALLBOX : 0);
  d.noise = p.noise_kind == BD_NOISE_GAUSS ? NOISE_GAUSS
            : p.noise_kind == BD_NOISE_NONE ? NOISE_NONE
                                            : NOISE_DISK;
  d.L = (float)p.L;
  d.B = (float)r->B;
  d.invB = (float)(1.0 / r->B);
  d.dx = (float)r->dx;
  d.invdx = (float)(1.0 / r->dx);
  d.invC = (float)(1.0 / r->C);
  d.z_over_L = (float)(r->Z / p.L);
  // WCA pair types 11, 22, 12 (dynamik_methoden.cpp:679-686, 851-865, 1021-1035)
  d.wpre[0] = 24.0f;
  d.wsig[0] = 1.0f;
  d.wsig2[0] = 1.0f;
  d.wpre[1] = (float)(p.eps22_11 * p.sigma11_22 * 4.0 * 6.0);
  d.wsig[1] = (float)p.sigma11_22;
  d.wsig2[1] = (float)(p.sigma11_22 * p.sigma11_22);
  d.wpre[2] = (float)(p.eps12_11 * p.sigma11_12 * 4.0 * 6.0);
  d.wsig[2] = (float)p.sigma11_12;
  d.wsig2[2] = (float)(p.sigma11_12 * p.sigma11_12);
  d.cut2 = (float)(dv.zweihoch1_6 * dv.zweihoch1_6);
  d.maxPair = (float)p.maxPairWCA;
  d.q2 = (float)p.f2_f1;
  d.drho = (float)(1.0 / (r->dx * r->dx));
  d.T = (float)p.T;
  d.dt_max = (float)p.dt_max;
  d.mrd = (float)std::min(p.max_reisedistanz, 1e30);
  d.L_d = p.L;
  d.B_d = r->B;
  d.T_d = p.T;
  d.dt_max_d = p.dt_max;
  d.seed = seed;
  {
    const double unit = (1.0 / (r->dx * r->dx)) * std::max(1.0, std::fabs(p.f2_f1));
    // one contribution is at most unit: |value| <= 2^30 after scaling
    int E = (int)std::floor(30.0 - std::log2(unit));
    d.fx_shift = std::max(-120, std::min(120, E));
  }
  {
    // one WCA pair term is at most maxPairWCA * 3B * sigma: 2^50 after
    // scaling, so a particle's sum has room for 2^13 capped pairs
    const double smax = std::max(1.0, std::max(p.sigma11_22, p.sigma11_12));
    const double big = std::max(1e-30, p.maxPairWCA * 3.0 * r->B * smax);
    const int E = (int)std::floor(50.0 - std::log2(big));
    d.wfx_shift = std::max(-100, std::min(100, E));
  }
  geometry(*r);
  // device memory
  const size_t N = r->N, cc = (size_t)r->C * r->C, Z = r->Z, n = Z / 2;
  size_t acc = 0;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
  };
  A(dalloc(d.recA, N, acc, pool, stream));
  A(dalloc(d.recB, N, acc, pool, stream));
  A(dalloc(d.Fw, N, acc, pool, stream));
  A(dalloc(d.Fk, N, acc, pool, stream));
  A(dalloc(d.Fn, N, acc, pool, stream));
  A(dalloc(d.count, cc, acc, pool, stream));
  A(dalloc(d.start, cc + 1, acc, pool, stream));
  A(dalloc(d.chunk_sum, (cc + SCAN_CHUNK - 1) / SCAN_CHUNK, acc, pool, stream));
  A(dalloc(d.chunk_off, (cc + SCAN_CHUNK - 1) / SCAN_CHUNK, acc, pool, stream));
  if (!r->idgas) {
    A(dalloc(d.rho, Z * Z, acc, pool, stream));
    A(dalloc(d.spec, Z * n, acc, pool, stream));
    A(dalloc(d.spec2, Z * n, acc, pool, stream));
    A(dalloc(d.H, Z * Z, acc, pool, stream));
    A(dalloc(d.green, Z * (n + 1), acc, pool, stream));
    A(dalloc(d.sxt, Z, acc, pool, stream));
    A(dalloc(d.syt, n + 1, acc, pool, stream));
    A(dalloc(d.tw, Z, acc, pool, stream));
    A(dalloc(d.pos_full, Z, acc, pool, stream));
    A(dalloc(d.freq_full, Z, acc, pool, stream));
    A(dalloc(d.pos_half, n, acc, pool, stream));
  }
  if (deposit_in_move(p)) A(dalloc(d.dacc, Z * Z, acc, pool, stream));
  r->bytes = acc;
  runs.push_back(r);  // owned from here on (freed by the destructor on error)
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // the arrays exist before host copies
  if (e != cudaSuccess) {
    runs.pop_back();
    free_run_memory(r->d, stream);
    delete r;
    cudaGetLastError();
    return status_from_cuda(e);
  }
  CK(cudaMemsetAsync(d.count, 0, cc * sizeof(int), stream));
  CK(cudaMemsetAsync(d.chunk_sum, 0, ((cc + SCAN_CHUNK - 1) / SCAN_CHUNK) * 4, stream));
  CK(cudaMemsetAsync(d.Fw, 0, N * sizeof(float2), stream));
  CK(cudaMemsetAsync(d.Fk, 0, N * sizeof(float2), stream));
  CK(cudaMemsetAsync(d.Fn, 0, N * sizeof(float2), stream));
  CK(cudaMemsetAsync(d.recA, 0, N * sizeof(Rec), stream));
  if (d.dacc) CK(cudaMemsetAsync(d.dacc, 0, Z * Z * sizeof(unsigned long long), stream));
  if (!r->idgas) {
    // kapkraefte_init: twiddles and Green's tables (FP64, stored FP32)
    std::vector<float2> tw(Z);
    for (size_t t = 0; t < Z; t++) {
      const double a = -2.0 * M_PI * (double)t / (double)Z;
      tw[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    CK(h2d_nosync(stream, d.tw, tw.data(), Z * sizeof(float2)));
    std::vector<int> pf, fp, ph;
    plan_maps(d.plan_full, pf, &fp);
    plan_maps(d.plan_half, ph, nullptr);
    CK(h2d_nosync(stream, d.pos_full, pf.data(), Z * sizeof(int)));
    CK(h2d_nosync(stream, d.freq_full, fp.data(), Z * sizeof(int)));
    CK(h2d_nosync(stream, d.pos_half, ph.data(), n * sizeof(int)));
    RK(launch_green(d.green, d.sxt, d.syt, r->Z, p.kapillar_vorfaktor, p.lambda_kapillar, p.L, stream));
    CK(cudaMemsetAsync(d.H, 0, Z * Z * sizeof(float2), stream));
    CK(cudaStreamSynchronize(stream));  // the tables' host buffers end here
  }
  r->dyn.step = 0;
  r->dyn.steps_left = STEPS_UNLIMITED;
  r->dyn.t = 0.0;
  r->dyn.dt = 0.f;
  float big = 3.0e38f;
  std::memcpy(&r->dyn.dt_bits, &big, 4);
  r->dyn.err = 0;
  r->dyn.sorting = 0;
  r->dyn.pad = 0;
  if (out) *out = r;
  return BD_OK;
}

int Engine::remove_run(size_t idx) {
  if (idx >= runs.size()) return BD_ERR_ARG;
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  RK(download_dyn());
  tables_ok = false;
  descs_ok = false;
  planned = false;
  drop_graphs();
  RunHost* r = runs[idx];
  free_run_memory(r->d, stream);
  if (r->d_sort) cudaFreeAsync(r->d_sort, stream);
  delete r;
  runs.erase(runs.begin() + idx);
  return BD_OK;
}

void Engine::drop_graphs() {
  if (g1) cudaGraphExecDestroy(g1);
  if (gK) cudaGraphExecDestroy(gK);
  g1 = gK = nullptr;
}

// The fused step applies to one run with a mesh, a power-of-two mesh side
// from 8 to 1024 and a fixed dt; its transform items are sized so that one
// CTA handles at most one (at least two CTAs per SM are resident at ~100
// registers per thread).
int Engine::plan_fused() {
  fused = false;
  if (runs.size() != 1) return BD_OK;
  const RunHost& r = *runs[0];
  const int Z = r.Z;
  if (!r.d.dacc || Z < 8 || Z > 1024) return BD_OK;
  FusedPlan P{};
  P.lz = ilog2(Z);
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  // CTAs: two per SM once the particles fill a CTA per SM; a small run takes
  // fewer (at least 32), so that its grid barriers wait on fewer arrivals
  const int blocks = (r.N + 255) / 256;
  const int gmin = blocks >= nsm ? 2 * nsm : std::max(32, blocks);
  auto size_items = [&](int count, int tps, int& l, int& n) {
    l = 0;
    while ((count >> l) > gmin && ((2 << l) * tps) <= FFT2_THREADS && (count >> (l + 1)) >= 1) l++;
    n = count >> l;
  };
  size_items(Z, fft2_tps(P.lz - 1), P.lrf, P.nrf);
  size_items(Z / 2, fft2_tps(P.lz), P.lw, P.ncl);
  size_items(Z, fft2_tps(P.lz), P.lri, P.nri);
  P.nch = (int)(((long long)r.C * r.C + SCAN_CHUNK - 1) / SCAN_CHUNK);
  // the forward row items run beside the scan chunks, on the other CTAs
  // where the threads allow
  while (P.nrf + P.nch > gmin && P.nrf > 1 && ((2 << P.lrf) * fft2_tps(P.lz - 1)) <= FFT2_THREADS) {
    P.lrf++;
    P.nrf >>= 1;
  }
  const int e = fused_configure(P, device);
  if (e) {
    cudaGetLastError();
    return BD_OK;  // not available: the stage kernels run instead
  }
  P.grid = std::min(P.grid, std::max(gmin, std::max(P.nrf, std::max(P.ncl, P.nri))));
  if (P.nrf > P.grid || P.ncl > P.grid || P.nri > P.grid) return BD_OK;
  if (!d_bar) {
    CK(cudaMalloc(&d_bar, 2 * sizeof(unsigned)));
    CK(cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), stream));
  }
  // the run's density accumulator (cleared again by the prologue that
  // precedes the first fused step)
  P.dacc = r.d.dacc;
  fplan = P;
  dep_valid = false;
  fused = true;
  return BD_OK;
}

// The run table on the device: every run's description, and its mutable
// state, which is authoritative on the device once uploaded (tables_ok) until
// the set of runs changes (download_dyn first).
int Engine::upload_tables() {
  CK(cudaSetDevice(device));
  if (tables_ok && descs_ok) return BD_OK;  // nothing changed since the last upload
  if (runs.size() > d_runs_cap) {
    CK(cudaStreamSynchronize(stream));
    if (tables_ok) RK(download_dyn());
    if (d_runs) cudaFree(d_runs);
    if (d_dyn) cudaFree(d_dyn);
    d_runs = nullptr;
    d_dyn = nullptr;
    d_runs_cap = runs.size() + runs.size() / 2 + 4;
    CK(cudaMalloc(&d_runs, d_runs_cap * sizeof(RunDesc)));
    CK(cudaMalloc(&d_dyn, d_runs_cap * sizeof(RunDyn)));
    tables_ok = false;
  }
  std::vector<RunDesc> hd(runs.size());
  for (size_t k = 0; k < runs.size(); k++) {
    hd[k] = runs[k]->d;
    if (!piped) hd[k].dacc = nullptr;  // only the pipelined stage step deposits through the table
  }
  std::vector<RunDyn> hy;
  if (!runs.empty()) CK(h2d_nosync(stream, d_runs, hd.data(), hd.size() * sizeof(RunDesc)));
  if (!tables_ok) {
    hy.resize(runs.size());
    for (size_t k = 0; k < runs.size(); k++) hy[k] = runs[k]->dyn;
    if (!runs.empty()) CK(h2d_nosync(stream, d_dyn, hy.data(), hy.size() * sizeof(RunDyn)));
    tables_ok = true;
  }
  CK(cudaStreamSynchronize(stream));  // hd and hy end here
  descs_ok = true;
  return BD_OK;
}

// The pinned staging buffer, at least `bytes` long, once the last copy that
// used it has ended (the host may write it).
int Engine::stage_buffer(size_t bytes, void** out) {
  CK(cudaEventSynchronize(ev_stage));
  if (bytes > h_stage_cap) {
    if (h_stage) CK(cudaFreeHost(h_stage));
    h_stage = nullptr;
    h_stage_cap = 0;
    const size_t cap = std::max<size_t>(bytes + bytes / 4, 4096);
    CK(cudaHostAlloc(&h_stage, cap, cudaHostAllocDefault));
    h_stage_cap = cap;
  }
  *out = h_stage;
  return BD_OK;
}

// the device state of every run back into the host mirrors (one copy)
int Engine::download_dyn() {
  if (!tables_ok || runs.empty()) return BD_OK;
  std::vector<RunDyn> hy(runs.size());
  CK(cudaStreamSynchronize(stream));
  CK(d2h(stream, hy.data(), d_dyn, hy.size() * sizeof(RunDyn)));
  for (size_t k = 0; k < runs.size(); k++) runs[k]->dyn = hy[k];
  return BD_OK;
}

int Engine::build_plan() {
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));  // earlier work may still read the old tables
  drop_graphs();
  dep_valid = false;  // the next fused or pipelined step starts with the prologue
  descs_ok = false;   // the descriptions depend on the plan (the accumulator of piped runs)
  std::vector<Item> all, dep, part, chunk;
  // FFT items: [0] meshes with a factor 3, [1 + lz] power-of-two meshes 2^lz
  std::vector<Item> fl[14][3];
  size_t fsm[14][3] = {};
  int fthr[14][3] = {};
  mt_max = 0;
  rows_max = 0;
  split = false;
  // FFT item sizes: the per-run sizes, halved while a pass of the whole
  // launch has fewer than fft_items_min items (default: two per SM; the
  // transforms' arithmetic does not depend on how sequences are grouped into
  // items). Power-of-two meshes
  // take as many sequences per item as FFT2_THREADS threads transform at
  // once (Z/16 threads per length-Z sequence).
  const size_t nr = runs.size();
  // the pipelined stage step (decided below) runs every transform item with
  // FFT2_THREADS threads; the classic column pass of meshes of 2048 and more
  // takes FFT2_WIDE_THREADS, so an item holds several columns
  bool pipe_runs = nr >= 2;
  for (auto* r : runs) pipe_runs = pipe_runs && r->d.dacc != nullptr;
  std::vector<int> lrf(nr), lri(nr), lw(nr);
  for (size_t k = 0; k < nr; k++) {
    const RunHost& r = *runs[k];
    const int Z = r.Z;
    if (pow2(Z)) {
      const int lz = ilog2(Z);
      lrf[k] = std::min(ilog2(FFT2_THREADS / fft2_tps(lz - 1)), lz);
      lri[k] = std::min(ilog2(FFT2_THREADS / fft2_tps(lz)), lz);
      // columns per item: both inverse transforms of the item run at once
      const int cthr = (lz >= 11 && !pipe_runs) ? FFT2_WIDE_THREADS : FFT2_THREADS;
      lw[k] = std::min(ilog2(cthr / (2 * fft2_tps(lz))), lz - 1);
    } else {
      lrf[k] = r.lrf;
      lri[k] = r.lri;
      lw[k] = r.lw;
    }
  }
  auto thin = [&](std::vector<int>& l, auto count) {
    for (;;) {
      long long items = 0;
      for (size_t k = 0; k < nr; k++)
        if (!runs[k]->idgas) items += count(k, l[k]);
      if (items >= fft_items_min) break;
      bool changed = false;
      for (size_t k = 0; k < nr; k++)
        if (l[k] > 0) l[k]--, changed = true;
      if (!changed) break;
    }
  };
  // deposit tiles: the largest that still give the launch dep_tiles_min tiles
  // (default: one per SM)
  std::vector<int> mt(nr), rmax(nr);
  for (size_t k = 0; k < nr; k++) mt[k] = runs[k]->mt;
  for (;;) {
    long long tiles = 0;
    for (size_t k = 0; k < nr; k++)
      if (!runs[k]->idgas) tiles += (long long)(runs[k]->Z / mt[k]) * (runs[k]->Z / mt[k]);
    if (tiles >= dep_tiles_min) break;
    bool changed = false;
    for (size_t k = 0; k < nr; k++)
      if (mt[k] >= 32 && mt[k] % 2 == 0 && runs[k]->Z % (mt[k] / 2) == 0) mt[k] /= 2, changed = true;
    if (!changed) break;
  }
  for (size_t k = 0; k < nr; k++) {
    const RunHost& r = *runs[k];
    rmax[k] = std::min(r.C, (int)std::ceil((mt[k] + 2.0) * r.C / r.Z) + 6);
  }
  thin(lrf, [&](size_t k, int l) { return (long long)(runs[k]->Z >> l); });
  thin(lri, [&](size_t k, int l) { return (long long)(runs[k]->Z >> l); });
  thin(lw, [&](size_t k, int l) { return (long long)((runs[k]->Z / 2) >> l); });
  for (size_t k = 0; k < runs.size(); k++) {
    RunHost& r = *runs[k];
    const int run = (int)k, Z = r.Z, n = Z / 2, C = r.C;
    if (r.adaptive) split = true;
    for (int b = 0; b < (r.N + 255) / 256; b++) part.push_back({run, b, 0, 0});
    if (!r.idgas) {
      for (int tx = 0; tx < Z / mt[k]; tx++)
        for (int ty = 0; ty < Z / mt[k]; ty++) dep.push_back({run, tx, ty, mt[k]});
      const int lz = ilog2(Z);
      const int P = pow2(Z) ? 1 + lz : 0;
      for (int row = 0; row < Z; row += 1 << lrf[k]) fl[P][0].push_back({run, row, 0, lrf[k]});
      for (int col = 0; col < n; col += 1 << lw[k]) fl[P][1].push_back({run, col, 0, lw[k]});
      for (int row = 0; row < Z; row += 1 << lri[k]) fl[P][2].push_back({run, row, 0, lri[k]});
      if (P) {
        fsm[P][0] = std::max(fsm[P][0], (size_t)(1 << lrf[k]) * fft2_stride(n) * 8);
        fsm[P][1] = std::max(fsm[P][1], (size_t)2 * (1 << lw[k]) * fft2_stride(Z) * 8);
        fsm[P][2] = std::max(fsm[P][2], (size_t)(1 << lri[k]) * fft2_stride(Z) * 8);
        fthr[P][0] = std::max(fthr[P][0], (1 << lrf[k]) * fft2_tps(lz - 1));
        // both inverse column transforms at once when the threads allow
        fthr[P][1] = std::max(fthr[P][1], std::min(lz >= 11 && !pipe_runs ? FFT2_WIDE_THREADS : FFT2_THREADS,
                                                   2 * (1 << lw[k]) * fft2_tps(lz)));
        fthr[P][2] = std::max(fthr[P][2], (1 << lri[k]) * fft2_tps(lz));
      } else {
        fsm[0][0] = std::max(fsm[0][0], (size_t)(1 << lrf[k]) * n * 8);
        fsm[0][1] = std::max(fsm[0][1], (size_t)2 * ((size_t)Z << lw[k]) * 8);
        fsm[0][2] = std::max(fsm[0][2], (size_t)(1 << lri[k]) * Z * 8);
      }
      mt_max = std::max(mt_max, mt[k]);
      rows_max = std::max(rows_max, rmax[k]);
    }
    const long long cc = (long long)C * C;
    for (int c = 0; c < (int)((cc + SCAN_CHUNK - 1) / SCAN_CHUNK); c++) chunk.push_back({run, c, 0, 0});
  }
  auto put = [&](std::vector<Item>& v, int& off, int& cnt) {
    off = (int)all.size();
    cnt = (int)v.size();
    all.insert(all.end(), v.begin(), v.end());
  };
  put(dep, off_dep, n_dep);
  fft_gen = FftSet();
  fft_p2.clear();
  for (int P = 0; P < 14; P++) {
    if (fl[P][0].empty()) continue;
    FftSet f;
    f.lz = P ? P - 1 : 0;
    for (int q = 0; q < 3; q++) {
      put(fl[P][q], f.off[q], f.n[q]);
      f.sm[q] = fsm[P][q];
      // whole warps, at least one
      f.thr[q] = P ? std::max(32, std::min(q == 1 ? FFT2_WIDE_THREADS : FFT2_THREADS, (fthr[P][q] + 31) / 32 * 32))
                   : FFT_THREADS;
    }
    if (P) fft_p2.push_back(f);
    else fft_gen = f;
  }
  put(part, off_part, n_part);
  put(chunk, off_chunk, n_chunk);
  off_part_all = off_part;
  n_part_all = n_part;
  // pipelined stage step: several runs, every one depositing in the move. A
  // single run takes the fused step (mesh up to 1024^2) or the classic stage
  // kernels: alone on a large mesh, the tile deposit is cheaper than the
  // move's atomics and its transforms leave the sort nothing to overlap with
  piped = pipe_runs;
  if (piped) {
    std::vector<Item> pl[3];
    size_t psm[3] = {0, 0, 0};
    for (int P = 1; P < 14; P++)
      for (int q = 0; q < 3; q++) {
        for (Item I : fl[P][q]) {
          I.b = P - 1;  // log2 Z
          pl[q].push_back(I);
        }
        psm[q] = std::max(psm[q], fsm[P][q]);
      }
    put(pl[2], off_pinv, n_pinv);
    put(pl[0], off_pfwd, n_pfwd);
    put(pl[1], off_pcol, n_pcol);
    sm_pinv = psm[2];
    sm_pfwd = psm[0];
    sm_pcol = psm[1];
    std::vector<Item> su;  // scatter units (Item.b = -1)
    for (size_t k = 0; k < runs.size(); k++)
      for (int a = 0; a < (runs[k]->N + PIPE_SCATTER_UNIT - 1) / PIPE_SCATTER_UNIT; a++)
        su.push_back({(int)k, a, -1, 0});
    n_cu = n_du = 0;
    if (pipe_form == PIPE_TWO) {
      // two-launch form only (served mixes rebuild the plan every tick): each
      // phase's transform items spread evenly through its other units (scan
      // chunks, scatter units; Item.b = -1)
      auto interleave = [](const std::vector<Item>& F, const std::vector<Item>& S) {
        const size_t nf = F.size(), ns = S.size(), n = nf + ns;
        std::vector<Item> out;
        out.reserve(n);
        size_t i = 0, j = 0;
        for (size_t k = 0; k < n; k++) {
          if (i < nf && (j >= ns || i * n <= k * nf)) out.push_back(F[i++]);
          else out.push_back(S[j++]);
        }
        return out;
      };
      std::vector<Item> sc = chunk;
      for (Item& I : sc) I.b = -1;
      std::vector<Item> cu = interleave(pl[0], sc), du = interleave(pl[1], su);
      put(cu, off_cu, n_cu);
      put(du, off_du, n_du);
    }
    // six-launch form: the scan's chunk groups
    std::vector<Item> grp;
    for (const Item& I : chunk)
      if (I.a % PIPE_SCAN_GROUP == 0) grp.push_back(I);
    put(grp, off_pscan, n_pscan);
    put(su, off_psu, n_psu);
  }
  if (all.size() > d_items_cap) {
    if (d_items) cudaFree(d_items);
    d_items = nullptr;
    d_items_cap = all.size() + all.size() / 2 + 16;
    CK(cudaMalloc(&d_items, d_items_cap * sizeof(Item)));
  }
  if (!all.empty())
    CK(h2d(stream, d_items, all.data(), all.size() * sizeof(Item)));
  RK(upload_tables());
  RK(plan_fused());
  RK(plan_tail());
  planned = true;
  int st = make_graphs();
  if (st != BD_OK && fused) {
    // the cooperative launch could not be captured: stage kernels instead
    cudaGetLastError();
    drop_graphs();
    fused = false;
    st = make_graphs();
  }
  return st;
}

// One fused step of every run. ev (optional, 10 events) brackets the stages:
// ev[0] | deposit | ev[1] | row FFT | ev[2] | column FFT | ev[3] | inverse
// row FFT | ev[4] | particles (+ move) | ev[5] | count scan (+ step end) |
// ev[6] | scatter | ev[7] .. ev[9] (no further launches)
int Engine::enqueue_step(cudaStream_t s, cudaEvent_t* ev) {
  if (fused && !ev) {
    FusedPlan P = fplan;
    if (fault_barrier > 0) {
      P.skip_barrier = fault_barrier;
      P.skip_cta = P.grid - 1;
      P.max_polls = fault_polls;
      fault_barrier = 0;
    }
    const int e = launch_fused(runs[0]->d, d_dyn, P, d_bar, s);
    return e ? BD_ERR_CUDA : BD_OK;
  }
  if (piped && !ev) return pipe_form == PIPE_TWO && tail_ok ? enqueue_pipe2(s) : enqueue_pipe(s, nullptr);
  // the classic stage kernels leave no pipeline state (they run here for the
  // stage timings of a fused or pipelined plan too)
  if (fused || piped) RK(dep_invalidate());
  if (ev) cudaEventRecord(ev[0], s);
  if (n_dep > 0) RK(launch_deposit(d_runs, d_dyn, it(off_dep), n_dep, mt_max, rows_max, -1, 1, s));
  if (ev) cudaEventRecord(ev[1], s);
  if (n_dep > 0)
    RK(enqueue_fft(1, s, ev ? ev + 2 : nullptr));
  else if (ev)
    for (int k = 2; k <= 4; k++) cudaEventRecord(ev[k], s);
  if (split) {
    RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, MODE_FORCES, 7, 1, s, 0, part_shape));
    RK(launch_move(d_runs, d_dyn, it(off_part), n_part, 1, 0, s));
  } else {
    RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, MODE_STEP, 7, 1, s, 0, part_shape));
  }
  if (ev) cudaEventRecord(ev[5], s);
  RK(launch_sort(d_runs, d_dyn, 0, (int)runs.size(), it(off_chunk), n_chunk, it(off_part), n_part, 1,
                 split ? 1 : 0, 1, s, ev ? ev + 6 : nullptr));
  if (ev) cudaEventRecord(ev[9], s);
  return BD_OK;
}

// One pipelined stage step on stream s (and stream2 for the next transform,
// forked and joined through events, so a capture of s records both
// branches). The particle kernel marks the runs that take part (`sorting`);
// then two chains run side by side, joined once at the end: the cell sort
// (scan, then scatter and step end) on s, and on stream2 the transform of
// the new positions (forward rows from the density the move deposited,
// columns + Green, inverse rows), which leaves the next step's force grids.
// Nothing in one chain reads what the other writes (the scatter's step end
// changes the budget and counters, which the transforms do not read; they
// take the flag). ev (optional, FUSED_PHASES + 1 events): recorded on s at
// the start, after the particles, after the scan and after the join (the
// inverse rows, phase 0, run inside the last phase: reported as 0).
int Engine::enqueue_pipe(cudaStream_t s, cudaEvent_t* ev) {
  if (ev) CK(cudaEventRecord(ev[0], s));
  if (ev) CK(cudaEventRecord(ev[1], s));
  RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, MODE_STEP, 7, 1, s, 1, part_shape));
  if (ev) CK(cudaEventRecord(ev[2], s));
  CK(cudaEventRecord(ev_fork[0], s));
  CK(cudaStreamWaitEvent(stream2, ev_fork[0], 0));
  RK(launch_pipe_fft(1, d_runs, d_dyn, it(off_pfwd), n_pfwd, sm_pfwd, stream2));
  RK(launch_pipe_fft(2, d_runs, d_dyn, it(off_pcol), n_pcol, sm_pcol, stream2));
  RK(launch_pipe_fft(0, d_runs, d_dyn, it(off_pinv), n_pinv, sm_pinv, stream2));
  RK(launch_pipe_scan(d_runs, d_dyn, it(off_pscan), n_pscan, s));
  if (ev) CK(cudaEventRecord(ev[3], s));
  RK(launch_pipe_scatter(d_runs, d_dyn, it(off_psu), n_psu, it(off_chunk), n_chunk, s));
  CK(cudaEventRecord(ev_join[0], stream2));
  CK(cudaStreamWaitEvent(s, ev_join[0], 0));
  if (ev) CK(cudaEventRecord(ev[4], s));
  return BD_OK;
}

// One two-launch pipelined step on stream s: the particle kernel, then the
// cooperative tail (scan | next forward rows, scatter | next columns, step
// end, the next step's inverse rows). ts (optional): the tail's timestamps.
int Engine::enqueue_pipe2(cudaStream_t s, unsigned long long* ts) {
  RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, MODE_STEP, 7, 1, s, 1, part_shape));
  return launch_pipe_tail(d_runs, d_dyn, tplan, d_bar, s, ts) ? BD_ERR_CUDA : BD_OK;
}

int Engine::set_step_form(int form, int ctas) {
  pipe_form = form;
  if (form == PIPE_TWO && ctas) tail_minb = ctas;
  if (!planned) return BD_OK;
  CK(cudaSetDevice(device));
  return build_plan();
}

// Launch shape of the two-launch form's cooperative kernel (pipelined plans)
// at tail_minb CTAs per SM; tail_ok stays false when it cannot be resident
// (the six-launch form runs instead).
int Engine::plan_tail() {
  tail_ok = false;
  if (!piped || pipe_form != PIPE_TWO) return BD_OK;
  for (auto* r : runs)
    if (r->Z > 1024) return BD_OK;  // the tail's transforms are compiled up to 1024 points
  PipeTail P{};
  P.cunits = it(off_cu);
  P.ncu = n_cu;
  P.dunits = it(off_du);
  P.ndu = n_du;
  P.chunks = it(off_chunk);
  P.nchunk = n_chunk;
  P.inv = it(off_pinv);
  P.ninv = n_pinv;
  P.smem = std::max(sm_pinv, std::max(sm_pfwd, sm_pcol));
  P.minb = tail_minb;
  if (pipe_tail_configure(P, device)) {
    cudaGetLastError();
    return BD_OK;
  }
  if (!d_bar) {
    CK(cudaMalloc(&d_bar, 2 * sizeof(unsigned)));
    CK(cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), stream));
  }
  tplan = P;
  tail_ok = true;
  return BD_OK;
}

int Engine::enqueue_fft(int require_active, cudaStream_t s, cudaEvent_t* ev) {
  FftPass gen[3];
  for (int q = 0; q < 3; q++) gen[q] = {it(fft_gen.off[q]), fft_gen.n[q], fft_gen.sm[q], fft_gen.thr[q]};
  Fft2Group g2[16];
  const int ng = (int)std::min<size_t>(fft_p2.size(), 16);
  for (int k = 0; k < ng; k++) {
    const FftSet& f = fft_p2[k];
    g2[k].lz = f.lz;
    for (int q = 0; q < 3; q++) g2[k].pass[q] = {it(f.off[q]), f.n[q], f.sm[q], f.thr[q]};
  }
  return launch_fft(d_runs, d_dyn, gen, g2, ng, require_active, s, ev);
}

int Engine::launches_per_step() const {
  if (fused) return 1;
  if (piped && pipe_form == PIPE_TWO && tail_ok) return 2;  // particles, cooperative tail
  if (piped) return 6;  // particles, then scan and scatter beside three transform passes
  int n = 0;
  if (n_dep > 0) {
    n += 1;
    for (int q = 0; q < 3; q++) {
      n += fft_gen.n[q] > 0;
      for (const FftSet& f : fft_p2) n += f.n[q] > 0;
    }
  }
  n += split ? 2 : 1;
  n += (n_chunk > 0 ? 2 : 0) + (n_part > 0);
  return n;
}

int Engine::timestep_info(bd_timestep_info* info) {
  if (runs.size() != 1 || !info) return BD_ERR_ARG;
  RunHost& r = *runs[0];
  if (!r.has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  // forces, noise and dt bound of the current positions and step
  if (!r.idgas) {
    RK(deposit(-1));
    RK(fft());
  }
  {
    float big = 3.0e38f;
    unsigned bits;
    std::memcpy(&bits, &big, 4);
    CK(cudaStreamSynchronize(stream));
    CK(h2d(stream, &d_dyn[0].dt_bits, &bits, 4));
  }
  RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, MODE_FORCES, 7, 0, stream));
  void* acc = nullptr;
  CK(cudaMalloc(&acc, diag_bytes()));
  int st = launch_diag(d_runs, r.N, acc, stream);
  struct {
    double energy, virial;
    unsigned long long maxF[3];
    unsigned long long pairs;
  } h{};
  if (!st && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
  if (!st && d2h(stream, &h, acc, sizeof(h)) != cudaSuccess) st = BD_ERR_CUDA;
  cudaFree(acc);
  if (st) return st > 0 ? BD_ERR_CUDA : st;
  RunDyn y;
  CK(d2h(stream, &y, d_dyn, sizeof(y)));
  std::memset(info, 0, sizeof(*info));
  info->num_WCA_berechnet = (long long)h.pairs;
  const int N1 = r.p.N1;
  float2* arr[3] = {r.d.Fw, r.d.Fk, r.d.Fn};
  int pids[3];
  double fx[3], fy[3];
  for (int k = 0; k < 3; k++) {
    const int pid = (int)(h.maxF[k] & 0xffffffffull);
    float2 f;
    CK(d2h(stream, &f, arr[k] + pid, sizeof(f)));
    pids[k] = pid;
    fx[k] = f.x;
    fy[k] = f.y;
  }
  info->maxWCAx = fx[0], info->maxWCAy = fy[0];
  info->maxWCAtype = pids[0] < N1 ? 1 : 2, info->maxWCAindex = pids[0] < N1 ? pids[0] : pids[0] - N1;
  info->maxKapx = fx[1], info->maxKapy = fy[1];
  info->maxKaptype = pids[1] < N1 ? 1 : 2, info->maxKapindex = pids[1] < N1 ? pids[1] : pids[1] - N1;
  info->maxRNDx = fx[2], info->maxRNDy = fy[2];
  info->maxRNDtype = pids[2] < N1 ? 1 : 2, info->maxRNDindex = pids[2] < N1 ? pids[2] : pids[2] - N1;
  float b;
  std::memcpy(&b, &y.dt_bits, 4);
  info->dt = (r.adaptive && (double)b < r.p.dt_max) ? (double)b : r.p.dt_max;
  info->num_Zellwechsel1 = y.moved_last[0];
  info->num_Zellwechsel2 = y.moved_last[1];
  info->E_WCA = r.idgas ? 0.0 : h.energy;
  info->virial_WCA = r.idgas ? 0.0 : h.virial;
  // entries of the erweiterte Nachbarlisten of the largest-WCA particle
  std::vector<int32_t> g1(2 * (size_t)N1 + 2), g2(2 * (size_t)r.p.N2 + 2);
  int32_t* gp[2] = {g1.data(), g2.data()};
  double* qp[2] = {nullptr, nullptr};
  RK(get_positions_both(0, gp, qp));
  const int s0 = pids[0] < N1 ? 0 : 1, i0 = pids[0] < N1 ? pids[0] : pids[0] - N1;
  const int ic = gp[s0][2 * i0], jc = gp[s0][2 * i0 + 1], C = r.C;
  int cnt[2] = {0, 0};
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? N1 : r.p.N2;
    for (int t = 0; t < n; t++) {
      const int di = ((gp[s][2 * t] - ic) % C + C) % C, dj = ((gp[s][2 * t + 1] - jc) % C + C) % C;
      if ((di <= 1 || di == C - 1) && (dj <= 1 || dj == C - 1)) cnt[s]++;
    }
  }
  info->maxWCA_numWW1 = cnt[0];
  info->maxWCA_numWW2 = cnt[1];
  return BD_OK;
}

// zeitschritt_debug (dynamik_methoden.cpp:168-211): one step whose length is
// optimaler_zeitschritt(mrd) (:1495-1560, travel bound mrd in place of
// max_reisedistanz, capped at dt_max), with the TimestepInfo of its forces.
// The run's descriptor carries the bound and the adaptive flag for this step
// only. The step itself is the regular one (zeitschritt's force, noise and
// restrictRadial rules); the cell changes reported are this step's.
int Engine::zeitschritt_debug(double mrd, bd_timestep_info* info, double* dt) {
  if (runs.size() != 1 || !info || !(mrd > 0.0)) return BD_ERR_ARG;
  RunHost& r = *runs[0];
  if (!r.has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  CK(cudaStreamSynchronize(stream));
  RunDesc d = r.d;
  d.mrd = (float)std::min(mrd, 1e30);
  d.flags |= F_ADAPTIVE;
  CK(h2d(stream, d_runs, &d, sizeof(d)));
  const bool was_adaptive = r.adaptive;
  r.adaptive = true;
  int st = timestep_info(info);
  if (st == BD_OK && launch_move(d_runs, d_dyn, it(off_part), n_part, 0, 0, stream)) st = BD_ERR_CUDA;
  if (st == BD_OK && launch_sort(d_runs, d_dyn, 0, 1, it(off_chunk), n_chunk, it(off_part), n_part, 1, 1, 0,
                                 stream, nullptr))
    st = BD_ERR_CUDA;
  if (st == BD_OK) st = dep_invalidate();
  if (st == BD_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
  r.adaptive = was_adaptive;
  const cudaError_t e = h2d(stream, d_runs, &r.d, sizeof(r.d));
  if (st != BD_OK) return st;
  if (e != cudaSuccess) return BD_ERR_CUDA;
  RK(sync_check());
  RunDyn y;
  CK(d2h(stream, &y, d_dyn, sizeof(y)));
  info->num_Zellwechsel1 = y.moved_last[0];
  info->num_Zellwechsel2 = y.moved_last[1];
  info->dt = y.dt;
  if (dt) *dt = y.dt;
  return BD_OK;
}

int Engine::korrelation(int which, double dr, int bins, double* g) {
  if (runs.size() != 1 || !g || which < 0 || which > 2 || !(dr > 0.0) || bins <= 0) return BD_ERR_ARG;
  if (bins > 8192) return BD_ERR_UNSUPPORTED;  // one CTA's shared-memory histogram
  RunHost& r = *runs[0];
  if (!r.has_pos) return BD_ERR_STATE;
  const int N1 = r.p.N1, N2 = r.p.N2;
  const double L = r.p.L, pi = 3.14159265358979323846;
  double v;
  if (which == 0) {
    v = N1 > 1 ? 2.0 / ((N1 - 1) * pi * (N1 / L / L) * dr * dr) : 0.0;
  } else if (which == 1) {
    v = (N1 > 1 && N2 > 0) ? 1.0 / ((N1 - 1) * pi * (N2 / L / L) * dr * dr) : 0.0;
  } else {
    v = N2 > 1 ? 2.0 / ((N2 - 1) * pi * (N2 / L / L) * dr * dr) : 0.0;
  }
  if (v == 0.0) {
    for (int b = 0; b < bins; b++) g[b] = 0.0;
    return BD_OK;
  }
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  // offsets lie in (-B, 2B]: three extra cells cover every pair closer than bins*dr
  const int range = (int)std::ceil(bins * dr / r.B) + 3;
  unsigned long long* d_h = nullptr;
  CK(cudaMalloc(&d_h, (size_t)bins * sizeof(unsigned long long)));
  std::vector<unsigned long long> h(bins);
  int st = launch_korr(d_runs, r.N, which, bins, dr, range, d_h, stream);
  if (!st && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
  if (!st && d2h(stream, h.data(), d_h, h.size() * sizeof(unsigned long long)) != cudaSuccess)
    st = BD_ERR_CUDA;
  cudaFree(d_h);
  if (st) return st > 0 ? BD_ERR_CUDA : st;
  for (int b = 0; b < bins; b++) g[b] = (double)h[b] * v / (2 * b + 1);
  return BD_OK;
}

int Engine::ftrho(int species, int qbins, double dq, double* re, double* im) {
  if (runs.size() != 1 || !re || !im || species < 0 || species > 1 || qbins <= 0) return BD_ERR_ARG;
  if (qbins > 64) return BD_ERR_UNSUPPORTED;
  RunHost& r = *runs[0];
  if (!r.has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  const size_t nk = (size_t)qbins * qbins;
  double* d = nullptr;
  CK(cudaMalloc(&d, 2 * nk * sizeof(double)));
  int st = launch_ftrho(d_runs, r.N, species, qbins, dq, d, d + nk, stream);
  if (!st && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
  if (!st && (d2h(stream, re, d, nk * sizeof(double)) != cudaSuccess ||
              d2h(stream, im, d + nk, nk * sizeof(double)) != cudaSuccess))
    st = BD_ERR_CUDA;
  cudaFree(d);
  return st > 0 ? BD_ERR_CUDA : st;
}

int Engine::lokale_dichte(const bd_lokdens_params& lp, double* rho1, double* rho2, int32_t* hist,
                          int32_t* over) {
  if (runs.size() != 1) return BD_ERR_ARG;
  RunHost& r = *runs[0];
  const int n = bd::snapgrid_num(r.p.L, lp.snapgrid_crude);
  if (n <= 0 || lp.rhohist_bins <= 0 || !(lp.rhohist_drho > 0.0)) return BD_ERR_ARG;
  if (n > BD_SNAPGRID_MAX || lp.rhohist_bins > BD_RHOHIST_MAX_BINS) return BD_ERR_UNSUPPORTED;
  if (!r.has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  const double w = r.p.L / n;
  LdSnap sp;
  LdHist hp;
  sp.n = hp.n = n;
  sp.w = w;
  sp.drho = 1. / (w * w);  // main_auswertung.cpp:28
  hp.bins = lp.rhohist_bins;
  hp.dbin = lp.rhohist_drho;
  for (int t = 0; t < 3; t++) hp.rho_thresh[t] = lp.rho_thresh[t];
  for (int t = 0; t < 4; t++) hp.drho_thresh[t] = lp.drho_thresh[t];
  const size_t cells = (size_t)n * n, nh = 4 * (size_t)hp.bins + 7;
  char* d = nullptr;
  CK(cudaMalloc(&d, 2 * cells * sizeof(double) + nh * sizeof(unsigned)));
  double* d_grid = (double*)d;
  unsigned* d_hist = (unsigned*)(d + 2 * cells * sizeof(double));
  int st = launch_lokdens(d_runs, r.N, sp, hp, d_grid, d_hist, stream);
  std::vector<unsigned> h(nh);
  if (!st && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
  if (!st && d2h(stream, h.data(), d_hist, nh * sizeof(unsigned)) != cudaSuccess)
    st = BD_ERR_CUDA;
  if (!st && rho1 && d2h(stream, rho1, d_grid, cells * sizeof(double)) != cudaSuccess)
    st = BD_ERR_CUDA;
  if (!st && rho2 &&
      d2h(stream, rho2, d_grid + cells, cells * sizeof(double)) != cudaSuccess)
    st = BD_ERR_CUDA;
  cudaFree(d);
  if (st) return st > 0 ? BD_ERR_CUDA : st;
  if (hist)
    for (size_t i = 0; i < 4 * (size_t)hp.bins; i++) hist[i] = (int32_t)h[i];
  if (over)
    for (int t = 0; t < 7; t++) over[t] = (int32_t)h[4 * (size_t)hp.bins + t];
  return BD_OK;
}

int Engine::fused_phase_times(int nsteps, double* ms, int nphases) {
  if (nsteps <= 0 || nphases < FUSED_PHASES) return BD_ERR_ARG;
  for (auto* r : runs)
    if (!r->has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  if (piped) return pipe_phase_times(nsteps, ms, nphases);
  if (!fused) return BD_ERR_STATE;
  RK(fused_prologue());
  unsigned long long* d_ts = nullptr;
  CK(cudaMalloc(&d_ts, (FUSED_PHASES + 1) * sizeof(unsigned long long)));
  double acc[FUSED_PHASES] = {0};
  int st = BD_OK;
  for (int k = 0; k < nsteps && st == BD_OK; k++) {
    if (launch_fused(runs[0]->d, d_dyn, fplan, d_bar, stream, d_ts)) st = BD_ERR_CUDA;
    unsigned long long h[FUSED_PHASES + 1];
    if (st == BD_OK && cudaMemcpyAsync(h, d_ts, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      st = BD_ERR_CUDA;
    if (st == BD_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
    if (st == BD_OK)
      for (int i = 0; i < FUSED_PHASES; i++) acc[i] += (double)(h[i + 1] - h[i]) * 1e-6;
  }
  cudaFree(d_ts);
  if (st != BD_OK) return st;
  RK(sync_check());
  for (int i = 0; i < FUSED_PHASES; i++) ms[i] = acc[i] / nsteps;
  for (int i = FUSED_PHASES; i < nphases; i++) ms[i] = 0.0;
  return BD_OK;
}

// The pipelined stage step's phases in the fused step's four slots: events
// around the particle kernel and the scan, then to the join (the scatter
// beside the transform chain, whose inverse rows fill slot 0's place: slot 0
// stays 0), summed over nsteps steps.
int Engine::pipe_phase_times(int nsteps, double* ms, int nphases) {
  RK(fused_prologue());
  if (pipe_form == PIPE_TWO && tail_ok) return pipe2_phase_times(nsteps, ms, nphases);
  cudaEvent_t ev[FUSED_PHASES + 1];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  double acc[FUSED_PHASES] = {0};
  int st = BD_OK;
  for (int k = 0; k < nsteps && st == BD_OK; k++) {
    st = enqueue_pipe(stream, ev);
    if (st == BD_OK && cudaEventSynchronize(ev[4]) != cudaSuccess) st = BD_ERR_CUDA;
    for (int i = 0; i < FUSED_PHASES && st == BD_OK; i++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      acc[i] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (st != BD_OK) return st;
  RK(sync_check());
  for (int i = 0; i < FUSED_PHASES; i++) ms[i] = acc[i] / nsteps;
  for (int i = FUSED_PHASES; i < nphases; i++) ms[i] = 0.0;
  return BD_OK;
}

// The two-launch step's phases: events around the particle kernel, the
// tail's own timestamps for the rest (its inverse rows are the next step's;
// averaged over nsteps steps, they stand for this one's).
int Engine::pipe2_phase_times(int nsteps, double* ms, int nphases) {
  cudaEvent_t ev[2];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  unsigned long long* d_ts = nullptr;
  CK(cudaMalloc(&d_ts, 4 * sizeof(unsigned long long)));
  double acc[FUSED_PHASES] = {0};
  int st = BD_OK;
  for (int k = 0; k < nsteps && st == BD_OK; k++) {
    if (cudaEventRecord(ev[0], stream) != cudaSuccess) st = BD_ERR_CUDA;
    if (st == BD_OK)
      st = launch_particles(d_runs, d_dyn, it(off_part), n_part, MODE_STEP, 7, 1, stream, 1, part_shape)
               ? BD_ERR_CUDA
               : BD_OK;
    if (st == BD_OK && cudaEventRecord(ev[1], stream) != cudaSuccess) st = BD_ERR_CUDA;
    if (st == BD_OK && launch_pipe_tail(d_runs, d_dyn, tplan, d_bar, stream, d_ts)) st = BD_ERR_CUDA;
    unsigned long long h[4];
    if (st == BD_OK && cudaMemcpyAsync(h, d_ts, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      st = BD_ERR_CUDA;
    if (st == BD_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = BD_ERR_CUDA;
    if (st == BD_OK) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[0], ev[1]);
      acc[0] += (double)(h[3] - h[2]) * 1e-6;
      acc[1] += t;
      acc[2] += (double)(h[1] - h[0]) * 1e-6;
      acc[3] += (double)(h[2] - h[1]) * 1e-6;
    }
  }
  cudaFree(d_ts);
  for (auto& e : ev) cudaEventDestroy(e);
  if (st != BD_OK) return st;
  RK(sync_check());
  for (int i = 0; i < FUSED_PHASES; i++) ms[i] = acc[i] / nsteps;
  for (int i = FUSED_PHASES; i < nphases; i++) ms[i] = 0.0;
  return BD_OK;
}

int Engine::stage_times(int nsteps, double* ms, int nstages) {
  if (nsteps <= 0 || nstages < 9) return BD_ERR_ARG;
  for (auto* r : runs)
    if (!r->has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  cudaEvent_t ev[10];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  double acc[9] = {0};
  int st = BD_OK;
  for (int k = 0; k < nsteps && st == BD_OK; k++) {
    st = enqueue_step(stream, ev);
    if (st != BD_OK) break;
    if (cudaEventSynchronize(ev[9]) != cudaSuccess) {
      st = BD_ERR_CUDA;
      break;
    }
    for (int i = 0; i < 9; i++) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      acc[i] += t;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (st != BD_OK) return st;
  for (int i = 0; i < 9; i++) ms[i] = acc[i] / nsteps;
  for (int i = 9; i < nstages; i++) ms[i] = 0.0;
  return BD_OK;
}

// Mean device time of one deposit + transform pass of every run (all runs,
// active or not) with the current plan: one untimed pass, then reps timed.
// Only rho and the spectra / force grids are written, from the positions.
// reps mesh passes of every run with the current plan: the pipelined step's
// three transform launches, or the classic deposit and transform launches.
// Positions are not touched; the pipeline state is marked stale (the next
// step recomputes the spectrum).
int Engine::time_mesh_passes(int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
  RK(dep_invalidate());
  for (int k = 0; k <= reps; k++) {
    if (k == 1) CK(cudaEventRecord(e0, stream));
    if (piped) {
      RK(launch_pipe_fft(1, d_runs, d_dyn, it(off_pfwd), n_pfwd, sm_pfwd, stream));
      RK(launch_pipe_fft(2, d_runs, d_dyn, it(off_pcol), n_pcol, sm_pcol, stream));
      RK(launch_pipe_fft(0, d_runs, d_dyn, it(off_pinv), n_pinv, sm_pinv, stream));
    } else {
      RK(launch_deposit(d_runs, d_dyn, it(off_dep), n_dep, mt_max, rows_max, -1, 0, stream));
      RK(enqueue_fft(0, stream, nullptr));
    }
  }
  CK(cudaEventRecord(e1, stream));
  CK(cudaEventSynchronize(e1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  *ms = (double)t / reps;
  return BD_OK;
}

// reps launches of the step's particle kernel in the given shape (MODE_STEP
// with the deposit of a pipelined plan; MODE_FORCES for adaptive-dt plans),
// the first untimed. What they leave (cell counts, chunk totals, the step's
// records in recB, density accumulators, forces, the per-run counters) is
// put back by tune_particles.
int Engine::time_particles(int shape, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
  for (int k = 0; k <= reps; k++) {
    if (k == 1) CK(cudaEventRecord(e0, stream));
    RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, split ? MODE_FORCES : MODE_STEP, 7, 1, stream,
                        piped ? 1 : 0, shape));
  }
  CK(cudaEventRecord(e1, stream));
  CK(cudaEventSynchronize(e1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  *ms = (double)t / reps;
  return BD_OK;
}

// The particle kernel's shape: each timed on this batch and the faster kept.
// The runs' state is put back afterwards: the device run table (counters,
// step budget) from a copy, every run's cell counts and chunk totals to zero
// (as a step leaves them), and the pipeline state marked stale (the next
// step recomputes the density and spectrum of the unchanged positions).
int Engine::tune_particles(int reps, cudaEvent_t e0, cudaEvent_t e1, bd_tune_result* out) {
  out->particle_shape = part_shape;
  if (n_part == 0) return BD_OK;
  RK(upload_tables());
  RunDyn* saved = nullptr;
  CK(cudaMallocFromPoolAsync((void**)&saved, runs.size() * sizeof(RunDyn), pool, stream));
  int st = status_from_cuda(
      cudaMemcpyAsync(saved, d_dyn, runs.size() * sizeof(RunDyn), cudaMemcpyDeviceToDevice, stream));
  const int shapes[2] = {PART_SHAPE_DEFAULT, PART_SHAPE_5CTA};
  double t[2] = {0.0, 0.0};
  for (int k = 0; k < 2 && st == BD_OK; k++) st = time_particles(shapes[k], reps, e0, e1, &t[k]);
  if (cudaMemcpyAsync(d_dyn, saved, runs.size() * sizeof(RunDyn), cudaMemcpyDeviceToDevice, stream) !=
      cudaSuccess && st == BD_OK)
    st = BD_ERR_CUDA;
  cudaFreeAsync(saved, stream);
  for (auto* r : runs) {
    const size_t cc = (size_t)r->C * r->C;
    if (cudaMemsetAsync(r->d.count, 0, cc * sizeof(int), stream) != cudaSuccess && st == BD_OK) st = BD_ERR_CUDA;
    if (cudaMemsetAsync(r->d.chunk_sum, 0, ((cc + SCAN_CHUNK - 1) / SCAN_CHUNK) * sizeof(int), stream) !=
            cudaSuccess &&
        st == BD_OK)
      st = BD_ERR_CUDA;
  }
  RK(dep_invalidate());
  if (cudaStreamSynchronize(stream) != cudaSuccess && st == BD_OK) st = BD_ERR_CUDA;
  if (st != BD_OK) return st;
  out->particle_default_ms = t[part_shape == PART_SHAPE_5CTA ? 1 : 0];
  part_shape = t[1] < t[0] ? PART_SHAPE_5CTA : PART_SHAPE_DEFAULT;
  out->particle_shape = part_shape;
  out->particle_best_ms = std::min(t[0], t[1]);
  out->candidates += 2;
  return BD_OK;
}

int Engine::autotune(int reps, bd_tune_result* out) {
  if (reps <= 0 || !out) return BD_ERR_ARG;
  if (runs.empty()) return BD_ERR_STATE;
  for (auto* r : runs)
    if (!r->has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  if (fused) return BD_ERR_STATE;
  std::memset(out, 0, sizeof(*out));
  const int dep0 = dep_tiles_min, fft0 = fft_items_min;
  out->dep_tiles_min = dep0;
  out->fft_items_min = fft0;
  out->dep_tile_max = mt_max;
  out->particle_shape = part_shape;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return BD_ERR_CUDA;
  }
  if (n_dep == 0) {  // no mesh work (ideal-gas runs only): the particle kernel alone
    int st = tune_particles(reps, e0, e1, out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    RK(st);
    return build_plan();  // graphs with the chosen shape
  }
  // classic plans: deposit tiles x transform items; pipelined plans deposit
  // in the move, so only the transform items per launch are chosen (down to
  // a few rows or columns per item)
  static const int cand[6] = {148, 296, 592, 1184, 2368, 4736};
  const bool pipe_plan = piped;
  const int ndep = pipe_plan ? 1 : 4, nfft = pipe_plan ? 6 : 4;
  int st = time_mesh_passes(reps, e0, e1, &out->default_ms);
  double best = out->default_ms;
  int bd = dep0, bf = fft0;
  for (int i = 0; i < ndep && st == BD_OK; i++)
    for (int j = 0; j < nfft && st == BD_OK; j++) {
      dep_tiles_min = pipe_plan ? dep0 : cand[i];
      fft_items_min = cand[j];
      st = build_plan();
      double ms = 0.0;
      if (st == BD_OK) st = time_mesh_passes(reps, e0, e1, &ms);
      if (st != BD_OK) break;
      out->candidates++;
      if (ms < best) best = ms, bd = cand[i], bf = cand[j];
    }
  // the chosen plan (the starting one when a candidate failed), then the
  // particle kernel's shape on it; the graphs are built with both
  dep_tiles_min = st == BD_OK ? bd : dep0;
  fft_items_min = st == BD_OK ? bf : fft0;
  int st2 = build_plan();
  if (st == BD_OK && st2 == BD_OK) st2 = tune_particles(reps, e0, e1, out);
  if (st == BD_OK && st2 == BD_OK) st2 = build_plan();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != BD_OK) return st;
  if (st2 != BD_OK) return st2;
  out->dep_tiles_min = dep_tiles_min;
  out->fft_items_min = fft_items_min;
  out->dep_tile_max = mt_max;
  out->best_ms = best;
  return BD_OK;
}

int Engine::make_graphs() {
  if (runs.empty()) return BD_OK;
  for (int which = 0; which < 2; which++) {
    const int nst = which == 0 ? 1 : K;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    int st = BD_OK;
    for (int i = 0; i < nst && st == BD_OK; i++) st = enqueue_step(stream);
    cudaError_t e = cudaStreamEndCapture(stream, &g);
    if (st != BD_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return st != BD_OK ? st : status_from_cuda(e);
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    (which == 0 ? g1 : gK) = ex;
  }
  return BD_OK;
}

int Engine::step(long long nsteps) {
  if (nsteps < 0) return BD_ERR_ARG;
  // every kernel assumes the cell-sorted state (start[] tables) exists
  for (auto* r : runs)
    if (!r->has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  if (runs.empty()) return BD_OK;
  if ((fused || piped) && nsteps > 0) RK(fused_prologue());
  if (fused && fault_barrier > 0 && nsteps > 0) {  // the faulted step is a direct launch
    RK(enqueue_step(stream));
    nsteps--;
  }
  while (nsteps >= K) {
    CK(cudaGraphLaunch(gK, stream));
    nsteps -= K;
  }
  // the fused step alone is one kernel: launched directly rather than as a
  // one-node graph
  if (fused)
    while (nsteps-- > 0) RK(enqueue_step(stream));
  while (nsteps-- > 0) CK(cudaGraphLaunch(g1, stream));
  return BD_OK;
}

int Engine::sync_check() {
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  if (!tables_ok) return BD_OK;
  std::vector<RunDyn> hy(runs.size());
  if (!runs.empty()) CK(d2h(stream, hy.data(), d_dyn, hy.size() * sizeof(RunDyn)));
  for (auto& y : hy) {
    if (y.err & E_NONFINITE) return BD_ERR_NONFINITE;
    if (y.err & E_BARRIER_TIMEOUT) {
      RK(recover_fused());
      return BD_ERR_TIMEOUT;
    }
  }
  return BD_OK;
}

// A fused step whose grid barrier failed ran no phase past that barrier (the
// barrier fails for every CTA or for none), so its positions (recA) are those
// before the step, and the step counter, time and budget did not advance.
// What the phases before the barrier left behind is cleared: the barrier
// words, the cell counts, chunk totals and density accumulator the move adds
// to, the moved-cell counters and the error bit; the cell starts (which the
// scan may have rebuilt for the new keys) come back from a counting sort of
// the unchanged records; the next fused step recomputes the spectrum
// (prologue). The step can then be taken again with the same bits.
int Engine::recover_fused() {
  if (d_bar) CK(cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), stream));
  for (size_t k = 0; k < runs.size(); k++) {
    RunDesc& d = runs[k]->d;
    const size_t cc = (size_t)runs[k]->C * runs[k]->C;
    CK(cudaMemsetAsync(d.count, 0, cc * sizeof(int), stream));
    CK(cudaMemsetAsync(d.chunk_sum, 0, ((cc + SCAN_CHUNK - 1) / SCAN_CHUNK) * sizeof(int), stream));
    RunDyn y;
    CK(d2h(stream, &y, d_dyn + k, sizeof(RunDyn)));
    y.err &= ~E_BARRIER_TIMEOUT;
    y.moved[0] = y.moved[1] = 0;
    CK(h2d(stream, d_dyn + k, &y, sizeof(RunDyn)));
    if (runs[k]->has_pos) {
      CK(cudaMemcpyAsync(d.recB, d.recA, (size_t)runs[k]->N * sizeof(Rec), cudaMemcpyDeviceToDevice, stream));
      RK(sort_uploaded_run(k));
    }
  }
  for (auto* r : runs)
    if (r->d.dacc) CK(cudaMemsetAsync(r->d.dacc, 0, (size_t)r->Z * r->Z * sizeof(unsigned long long), stream));
  dep_valid = false;
  CK(cudaStreamSynchronize(stream));
  return BD_OK;
}

int Engine::inject_barrier_timeout(int barrier, unsigned max_polls) {
  if (barrier < 1 || barrier > 3 || max_polls == 0) return BD_ERR_ARG;
  for (auto* r : runs)
    if (!r->has_pos) return BD_ERR_STATE;
  CK(cudaSetDevice(device));
  if (!planned) RK(build_plan());
  if (!fused) return BD_ERR_STATE;
  fault_barrier = barrier;
  fault_polls = max_polls;
  return BD_OK;
}

int Engine::get_dyn(size_t run, RunDyn* dd) {
  if (run >= runs.size()) return BD_ERR_ARG;
  CK(cudaSetDevice(device));
  if (!tables_ok) {
    *dd = runs[run]->dyn;
    return BD_OK;
  }
  CK(cudaStreamSynchronize(stream));
  CK(d2h(stream, dd, d_dyn + run, sizeof(RunDyn)));
  return BD_OK;
}

int Engine::set_dyn_field_step(size_t run, unsigned long long stp) {
  if (run >= runs.size()) return BD_ERR_ARG;
  RK(upload_tables());
  CK(cudaStreamSynchronize(stream));
  CK(h2d(stream, &d_dyn[run].step, &stp, sizeof(stp)));
  return BD_OK;
}

int Engine::set_dyn_time(size_t run, double t, float dt) {
  if (run >= runs.size()) return BD_ERR_ARG;
  RK(upload_tables());
  CK(cudaStreamSynchronize(stream));
  CK(h2d(stream, &d_dyn[run].t, &t, sizeof(t)));
  CK(h2d(stream, &d_dyn[run].dt, &dt, sizeof(dt)));
  return BD_OK;
}

int Engine::set_steps_left(size_t run, long long n) {
  if (run >= runs.size()) return BD_ERR_ARG;
  if (!tables_ok) {
    runs[run]->dyn.steps_left = n;
    return BD_OK;
  }
  CK(cudaStreamSynchronize(stream));
  CK(h2d(stream, &d_dyn[run].steps_left, &n, sizeof(n)));
  return BD_OK;
}

int Engine::get_dyn_all(std::vector<RunDyn>& out) {
  CK(cudaSetDevice(device));
  out.resize(runs.size());
  if (runs.empty()) return BD_OK;
  if (!tables_ok) {
    for (size_t k = 0; k < runs.size(); k++) out[k] = runs[k]->dyn;
    return BD_OK;
  }
  CK(cudaStreamSynchronize(stream));
  CK(d2h(stream, out.data(), d_dyn, runs.size() * sizeof(RunDyn)));
  return BD_OK;
}

int Engine::set_steps_left_all(const std::vector<long long>& n) {
  if (n.size() != runs.size()) return BD_ERR_ARG;
  RK(upload_tables());
  std::vector<RunDyn> y;
  RK(get_dyn_all(y));
  for (size_t k = 0; k < y.size(); k++) y[k].steps_left = n[k];
  if (!y.empty()) CK(h2d(stream, d_dyn, y.data(), y.size() * sizeof(RunDyn)));
  return BD_OK;
}

// Records [t0, t1) of a run in the reference layout: cell (ic, jc) =
// (cell / C, cell % C), offsets widened to double, written at the
// particle's index. The quotient comes from a double reciprocal (exact for
// cells below 2^24 after the one-step correction).
static void records_to_layout(const Rec* h, long long t0, long long t1, int N1, int C, int32_t* git[2],
                              double* rel[2]) {
  const double invC = 1.0 / (double)C;
  for (long long t = t0; t < t1; t++) {
    const Rec& q = h[t];
    const int s = q.pid >= N1;
    const int i = s ? q.pid - N1 : q.pid;
    int ic = (int)((double)q.cell * invC);
    int jc = q.cell - ic * C;
    if (jc < 0) {
      ic--;
      jc += C;
    } else if (jc >= C) {
      ic++;
      jc -= C;
    }
    if (git[s]) {
      git[s][2 * i] = ic;
      git[s][2 * i + 1] = jc;
    }
    if (rel[s]) {
      rel[s][2 * i] = (double)q.ox;
      rel[s][2 * i + 1] = (double)q.oy;
    }
  }
}

// Particles [t0, t1) (index over both species) of the reference layout into
// records; false if one lies outside the cells or the legal offsets.
static bool layout_to_records(int32_t* const git[2], double* const rel[2], Rec* h, long long t0, long long t1,
                              int N1, int C, float B) {
  for (long long t = t0; t < t1; t++) {
    const int s = t >= N1;
    const long long i = s ? t - N1 : t;
    const int gx = git[s][2 * i], gy = git[s][2 * i + 1];
    const float fx = (float)rel[s][2 * i], fy = (float)rel[s][2 * i + 1];
    if (gx < 0 || gx >= C || gy < 0 || gy >= C) return false;
    if (!(fx > -B && fx <= 2.0f * B && fy > -B && fy <= 2.0f * B)) return false;
    h[t].ox = fx;
    h[t].oy = fy;
    h[t].cell = gx * C + gy;
    h[t].pid = (int)t;
  }
  return true;
}

// Position copies go in pieces of at least this many particles (at most
// MAX_COPY_PIECES of them), converted on the host pool's threads in
// parallel; a download's pieces convert as soon as their copies have ended.
static const long long COPY_PIECE = 8192;

static int copy_pieces(long long n) {
  return (int)std::min<long long>(Engine::max_copy_pieces(), (n + COPY_PIECE - 1) / COPY_PIECE);
}

HostPool::HostPool(int workers) {
  for (int k = 0; k < workers; k++) th_.emplace_back([this] { work(); });
}

HostPool::~HostPool() {
  {
    std::lock_guard<std::mutex> g(m_);
    stop_ = true;
  }
  cv_.notify_all();
  for (auto& t : th_) t.join();
}

// Take and run tasks of job generation g until none is left. Tasks are
// taken under the lock, so a thread that woke late for an earlier job takes
// none of a later one; the job stays in place until all its tasks are done.
void HostPool::drain(unsigned g) {
  for (;;) {
    int k;
    {
      std::lock_guard<std::mutex> l(m_);
      if (gen_ != g || next_ >= njob_) return;
      k = next_++;
    }
    (*job_)(k);
    done_.fetch_add(1);
  }
}

void HostPool::work() {
  unsigned seen = 0;
  for (;;) {
    {
      std::unique_lock<std::mutex> l(m_);
      cv_.wait(l, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
    }
    drain(seen);
  }
}

void HostPool::run_ordered(int n, const std::function<void(int)>& fn, const std::function<void(int)>& after) {
  if (n <= 0) return;
  std::unique_ptr<std::atomic<int>[]> fin(new std::atomic<int>[n]);
  for (int k = 0; k < n; k++) fin[k].store(0);
  const std::function<void(int)> task = [&](int k) {
    fn(k);
    fin[k].store(1, std::memory_order_release);
  };
  unsigned g;
  {
    std::lock_guard<std::mutex> l(m_);
    job_ = &task;
    njob_ = n;
    next_ = 0;
    done_.store(0);
    g = ++gen_;
  }
  cv_.notify_all();
  if (th_.empty()) drain(g);  // no workers: the caller converts everything first
  for (int k = 0; k < n; k++) {
    while (!fin[k].load(std::memory_order_acquire)) std::this_thread::yield();
    after(k);
  }
  while (done_.load() < n) std::this_thread::yield();
}

void HostPool::run(int n, const std::function<void(int)>& fn) {
  if (n <= 0) return;
  unsigned g;
  {
    std::lock_guard<std::mutex> l(m_);
    job_ = &fn;
    njob_ = n;
    next_ = 0;
    done_.store(0);
    g = ++gen_;
  }
  cv_.notify_all();
  drain(g);
  while (done_.load() < n) std::this_thread::yield();
}

HostPool& Engine::host_pool() {
  if (!hpool) {
    const unsigned hc = std::thread::hardware_concurrency();
    hpool.reset(new HostPool((int)std::min(7u, hc > 1 ? hc - 1 : 1u)));
  }
  return *hpool;
}

int Engine::set_all_positions(size_t run, int32_t* git[2], double* rel[2]) {
  if (run >= runs.size()) return BD_ERR_ARG;
  RunHost& r = *runs[run];
  CK(cudaSetDevice(device));
  void* buf = nullptr;
  RK(stage_buffer((size_t)std::max(r.N, 1) * sizeof(Rec), &buf));
  Rec* h = static_cast<Rec*>(buf);
  const float B = (float)r.B;
  RK(upload_tables());  // the sort needs the run table only, not the launch plan
  // converted piece by piece on the host pool's threads, each piece copied
  // into recB (scratch until the sort) as soon as it and the ones before it
  // are converted: positions out of range stop the call before the sort, the
  // run's state untouched
  const int np = copy_pieces(r.N);
  const long long per = np > 0 ? (r.N + np - 1) / np : 0;
  std::vector<char> ok(np, 1);
  bool all_ok = true;
  cudaError_t ce = cudaSuccess;
  host_pool().run_ordered(
      np,
      [&](int k) {
        const long long t0 = k * per, t1 = std::min<long long>(r.N, t0 + per);
        if (t0 < t1) ok[k] = layout_to_records(git, rel, h, t0, t1, r.p.N1, r.C, B) ? 1 : 0;
      },
      [&](int k) {
        const long long t0 = k * per, t1 = std::min<long long>(r.N, t0 + per);
        all_ok = all_ok && ok[k];
        if (all_ok && ce == cudaSuccess && t0 < t1)
          ce = cudaMemcpyAsync(r.d.recB + t0, h + t0, (size_t)(t1 - t0) * sizeof(Rec), cudaMemcpyHostToDevice, stream);
      });
  CK(ce);
  CK(cudaEventRecord(ev_stage, stream));  // the staging buffer is free once the copies end
  if (!all_ok) return BD_ERR_RANGE;
  RK(sort_uploaded_run(run));
  r.has_pos = true;
  return BD_OK;
}

int Engine::sort_uploaded() {
  for (size_t k = 0; k < runs.size(); k++) RK(sort_uploaded_run(k));
  return BD_OK;
}

// Counting sort of the run's uploaded records (recB) into recA, queued on the
// engine's stream (every later access is ordered after it). Its work items
// are uploaded once, by the run's first sort.
int Engine::sort_uploaded_run(size_t run) {
  RunHost& r = *runs[run];
  if (!r.d_sort) {
    const long long cc = (long long)r.C * r.C;
    r.n_sort_part = (r.N + 255) / 256;
    r.n_sort_chunk = (int)((cc + SCAN_CHUNK - 1) / SCAN_CHUNK);
    CK(cudaMallocFromPoolAsync((void**)&r.d_sort, ((size_t)r.n_sort_part + r.n_sort_chunk) * sizeof(Item),
                               pool, stream));
    r.sort_items_run = -1;
  }
  // the items carry the run's index in the table: rebuilt when it changed
  // (runs before it left)
  if (r.sort_items_run != (int)run) {
    std::vector<Item> v((size_t)r.n_sort_part + r.n_sort_chunk);
    for (int b = 0; b < r.n_sort_part; b++) v[b] = {(int)run, b, 0, 0};
    for (int c = 0; c < r.n_sort_chunk; c++) v[r.n_sort_part + c] = {(int)run, c, 0, 0};
    CK(h2d(stream, r.d_sort, v.data(), v.size() * sizeof(Item)));
    r.sort_items_run = (int)run;
  }
  Item* dp = r.d_sort;
  Item* dch = r.d_sort + r.n_sort_part;
  int st = BD_OK;
  if (r.n_sort_part > 0) st = launch_count(d_runs, dp, r.n_sort_part, stream);
  if (!st)
    st = launch_sort(d_runs, d_dyn, (int)run, 1, dch, r.n_sort_chunk, dp, r.n_sort_part, 0, 0, 0, stream);
  if (!st) st = dep_invalidate();
  return st > 0 ? BD_ERR_CUDA : st;
}

int Engine::set_positions(size_t run, int species, const int32_t* git, const double* rel) {
  if (run >= runs.size() || species < 0 || species > 1) return BD_ERR_ARG;
  RunHost& r = *runs[run];
  std::vector<int32_t> g[2];
  std::vector<double> q[2];
  const int Ns[2] = {r.p.N1, r.p.N2};
  for (int s = 0; s < 2; s++) {
    g[s].resize(2 * (size_t)Ns[s] + 2);
    q[s].resize(2 * (size_t)Ns[s] + 2);
    if (s == species) {
      std::memcpy(g[s].data(), git, sizeof(int32_t) * 2 * Ns[s]);
      std::memcpy(q[s].data(), rel, sizeof(double) * 2 * Ns[s]);
    } else {
      RK(get_positions(run, s, g[s].data(), q[s].data()));
    }
  }
  int32_t* gp[2] = {g[0].data(), g[1].data()};
  double* qp[2] = {q[0].data(), q[1].data()};
  return set_all_positions(run, gp, qp);
}

int Engine::get_positions(size_t run, int species, int32_t* git, double* rel) {
  if (run >= runs.size() || species < 0 || species > 1) return BD_ERR_ARG;
  int32_t* g[2] = {nullptr, nullptr};
  double* q[2] = {nullptr, nullptr};
  g[species] = git;
  q[species] = rel;
  return get_positions_both(run, g, q);
}

int Engine::get_records(size_t run, std::vector<Rec>& out) {
  if (run >= runs.size()) return BD_ERR_ARG;
  RunHost& r = *runs[run];
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(stream));
  out.resize(r.N);
  if (r.N > 0) CK(d2h(stream, out.data(), r.d.recA, out.size() * sizeof(Rec)));
  return BD_OK;
}

// The run's records, one device -> host copy into the pinned staging buffer
// after everything queued on the engine's stream, then written out in the
// reference layout.
int Engine::get_positions_both(size_t run, int32_t* git[2], double* rel[2]) {
  if (run >= runs.size()) return BD_ERR_ARG;
  RunHost& r = *runs[run];
  CK(cudaSetDevice(device));
  void* buf = nullptr;
  RK(stage_buffer((size_t)std::max(r.N, 1) * sizeof(Rec), &buf));
  Rec* h = static_cast<Rec*>(buf);
  // the records in particle order (into recB, scratch between steps), so
  // that the caller's arrays are written in order; copied piece by piece
  // after everything queued on the stream, each piece converted as soon as
  // its copy has ended, while the next ones move
  RK(launch_records_by_pid(r.d.recA, r.d.recB, r.N, stream) ? BD_ERR_CUDA : BD_OK);
  const int npieces = copy_pieces(r.N);
  const long long per = npieces > 0 ? (r.N + npieces - 1) / npieces : 0;
  for (int k = 0; k < npieces; k++) {
    const long long t0 = k * per, t1 = std::min<long long>(r.N, t0 + per);
    if (t0 >= t1) break;
    CK(cudaMemcpyAsync(h + t0, r.d.recB + t0, (size_t)(t1 - t0) * sizeof(Rec), cudaMemcpyDeviceToHost, stream));
    CK(cudaEventRecord(ev_piece[k], stream));
  }
  // each piece converted on a pool thread once its copy has ended
  std::vector<cudaError_t> err(npieces, cudaSuccess);
  const int dev = device;
  host_pool().run(npieces, [&](int k) {
    const long long t0 = k * per, t1 = std::min<long long>(r.N, t0 + per);
    if (t0 >= t1) return;
    cudaError_t e = cudaSetDevice(dev);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev_piece[k]);
    err[k] = e;
    if (e == cudaSuccess) records_to_layout(h, t0, t1, r.p.N1, r.C, git, rel);
  });
  for (int k = 0; k < npieces; k++) CK(err[k]);
  return BD_OK;
}

// ---- drop-in routines on run 0 ------------------------------------------
int Engine::wca(int mode, int mask) {
  if (runs.empty() || !runs[0]->has_pos) return BD_ERR_STATE;
  if (!planned) RK(build_plan());
  RK(launch_particles(d_runs, d_dyn, it(off_part), n_part, mode, mask, 0, stream));
  return BD_OK;
}

int Engine::deposit(int scheme) {
  if (runs.empty() || !runs[0]->has_pos) return BD_ERR_STATE;
  if (!planned) RK(build_plan());
  if (runs.empty() || runs[0]->idgas) return BD_OK;
  RK(dep_invalidate());  // rho, and after fft() the spectra, change
  RK(launch_deposit(d_runs, d_dyn, it(off_dep), n_dep, mt_max, rows_max, scheme, 0, stream));
  return BD_OK;
}

int Engine::fft() {
  if (!planned) RK(build_plan());
  if (runs.empty() || runs[0]->idgas) return BD_OK;
  RK(dep_invalidate());
  RK(enqueue_fft(0, stream, nullptr));
  return BD_OK;
}

int Engine::interp(int scheme) {
  if (runs.empty() || !runs[0]->has_pos) return BD_ERR_STATE;
  if (!planned) RK(build_plan());
  RK(launch_interp(d_runs, it(off_part_all), n_part_all, scheme, stream));
  return BD_OK;
}

int Engine::kap(int scheme) {
  if (!planned) RK(build_plan());
  if (runs.empty()) return BD_OK;
  if (runs[0]->idgas) {
    CK(cudaMemsetAsync(runs[0]->d.Fk, 0, runs[0]->N * sizeof(float2), stream));
    return BD_OK;
  }
  RK(deposit(scheme));
  RK(fft());
  RK(interp(scheme));
  return BD_OK;
}

int Engine::noise() {
  if (!planned) RK(build_plan());
  RK(launch_noise(d_runs, d_dyn, it(off_part_all), n_part_all, stream));
  return BD_OK;
}

int Engine::dtbound(double* dt) {
  if (!planned) RK(build_plan());
  if (runs.empty()) return BD_ERR_STATE;
  float big = 3.0e38f;
  unsigned int bits;
  std::memcpy(&bits, &big, 4);
  CK(cudaStreamSynchronize(stream));
  CK(h2d(stream, &d_dyn[0].dt_bits, &bits, 4));
  RK(launch_dtbound(d_runs, d_dyn, it(off_part_all), n_part_all, stream));
  CK(cudaStreamSynchronize(stream));
  CK(d2h(stream, &bits, &d_dyn[0].dt_bits, 4));
  float b;
  std::memcpy(&b, &bits, 4);
  const double dmax = runs[0]->p.dt_max;
  *dt = ((double)b < dmax) ? (double)b : dmax;
  // leave the reduction armed for the next step
  CK(h2d(stream, &d_dyn[0].dt_bits, &big, 4));
  return BD_OK;
}

int Engine::refresh() {
  if (runs.empty() || !runs[0]->has_pos) return BD_ERR_STATE;
  if (!planned) RK(build_plan());
  if (runs.empty()) return BD_OK;
  RK(launch_move(d_runs, d_dyn, it(off_part_all), n_part_all, 0, 1, stream));
  RK(launch_sort(d_runs, d_dyn, 0, (int)runs.size(), it(off_chunk), n_chunk, it(off_part), n_part, 0, 0,
                 0, stream));
  return dep_invalidate();
}

// The fused step's pipeline state (spec2 of the current positions, dacc
// clear) no longer holds: the next fused step is preceded by the prologue.
int Engine::dep_invalidate() {
  dep_valid = false;
  return BD_OK;
}

// deposit + forward row and column passes with the stage kernels: what a
// fused or pipelined step expects to find
int Engine::fused_prologue() {
  if (dep_valid) return BD_OK;
  for (auto* r : runs)
    if (r->d.dacc) CK(cudaMemsetAsync(r->d.dacc, 0, (size_t)r->Z * r->Z * sizeof(unsigned long long), stream));
  RK(launch_deposit(d_runs, d_dyn, it(off_dep), n_dep, mt_max, rows_max, -1, 0, stream));
  FftPass gen[3];
  for (int q = 0; q < 3; q++) gen[q] = {it(fft_gen.off[q]), fft_gen.n[q], fft_gen.sm[q], fft_gen.thr[q]};
  Fft2Group g2[16];
  const int ng = (int)std::min<size_t>(fft_p2.size(), 16);
  for (int k = 0; k < ng; k++) {
    const FftSet& f = fft_p2[k];
    g2[k].lz = f.lz;
    for (int q = 0; q < 3; q++) g2[k].pass[q] = {it(f.off[q]), f.n[q], f.sm[q], f.thr[q]};
  }
  // the fused step starts with the inverse row pass; the pipelined step's
  // transform chain ends with it, so its first step finds the force grids
  RK(launch_fft(d_runs, d_dyn, gen, g2, ng, 0, stream, nullptr, piped ? 3 : 2));
  dep_valid = true;
  return BD_OK;
}

int Engine::get_forces(int kind, int species, double* out) {
  if (runs.empty() || species < 0 || species > 1 || kind < 0 || kind > 2) return BD_ERR_ARG;
  RunHost& r = *runs[0];
  CK(cudaStreamSynchronize(stream));
  const int lo = species == 0 ? 0 : r.p.N1;
  const int cnt = species == 0 ? r.p.N1 : r.p.N2;
  std::vector<float2> h(cnt + 1);
  const float2* src = kind == 0 ? r.d.Fw : kind == 1 ? r.d.Fk : r.d.Fn;
  if (cnt > 0) CK(d2h(stream, h.data(), src + lo, cnt * sizeof(float2)));
  for (int i = 0; i < cnt; i++) {
    out[2 * i] = h[i].x;
    out[2 * i + 1] = h[i].y;
  }
  return BD_OK;
}

int Engine::get_grid(int which, double* out) {
  if (runs.empty() || which < 0 || which > 2) return BD_ERR_ARG;
  RunHost& r = *runs[0];
  if (r.idgas) return BD_ERR_STATE;
  CK(cudaStreamSynchronize(stream));
  const size_t ZZ = (size_t)r.Z * r.Z;
  if (which == 0) {
    std::vector<float> h(ZZ);
    CK(d2h(stream, h.data(), r.d.rho, ZZ * sizeof(float)));
    for (size_t k = 0; k < ZZ; k++) out[k] = h[k];
  } else {
    std::vector<float2> h(ZZ);
    CK(d2h(stream, h.data(), r.d.H, ZZ * sizeof(float2)));
    for (size_t k = 0; k < ZZ; k++) out[k] = which == 1 ? h[k].x : h[k].y;
  }
  return BD_OK;
}

}  // namespace bd

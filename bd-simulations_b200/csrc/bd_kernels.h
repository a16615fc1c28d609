// Host-visible declarations of the kernel launchers (bd_kernels.cu).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace bd {

struct RunDesc;
struct RunDyn;

// Work item of a batched launch: run index plus up to three coordinates
// whose meaning depends on the kernel (tile, row group, block, chunk).
struct Item {
  int run, a, b, c;
};

enum CellblockMode { MODE_STEP = 0, MODE_SET = 1, MODE_ADD = 2, MODE_FORCES = 3 };

constexpr int SCAN_CHUNK = 2048;
constexpr int FFT_THREADS = 512;
constexpr int MAX_FFT_SMEM = 200 * 1024;

size_t deposit_smem(int mt_max, int rows_max);

int set_kernel_attributes();
int launch_deposit(const RunDesc* runs, const RunDyn* dyn, const Item* items, int n, int mt_max,
                   int rows_max, int scheme_override, int require_active, cudaStream_t s);
int launch_fft(const RunDesc* runs, const RunDyn* dyn, const Item* rf, int nrf, size_t sm_rf,
               const Item* cl, int ncl, size_t sm_cl, const Item* ri, int nri, size_t sm_ri,
               int require_active, cudaStream_t s, cudaEvent_t* ev = nullptr);
int launch_particles(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, int mode,
                     int mask, int require_active, cudaStream_t s);
int launch_move(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, int require_active,
                int refresh_only, cudaStream_t s);
int launch_count(const RunDesc* runs, const Item* items, int n, cudaStream_t s);
int launch_sort(const RunDesc* runs, const RunDyn* dyn, const Item* chunks, int nchunks,
                const Item* parts, int nparts, const Item* cells, int ncells, int require_active,
                cudaStream_t s, cudaEvent_t* ev = nullptr);
int launch_step_end(const RunDesc* runs, RunDyn* dyn, int nruns, int adaptive, cudaStream_t s);
int launch_interp(const RunDesc* runs, const Item* items, int n, int scheme, cudaStream_t s);
int launch_noise(const RunDesc* runs, const RunDyn* dyn, const Item* items, int n, cudaStream_t s);
int launch_dtbound(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, cudaStream_t s);
int launch_green(float* green, float* sxt, float* syt, int Z, double kap, double lambda,
                 double L, cudaStream_t s);

}  // namespace bd

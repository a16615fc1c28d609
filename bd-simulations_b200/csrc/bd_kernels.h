// Host-visible declarations of the kernel launchers (bd_kernels.cu).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace bd {

struct RunDesc;
struct RunDyn;
struct Rec;

// Work item of a batched launch: run index plus up to three coordinates
// whose meaning depends on the kernel (tile, row group, block, chunk).
struct Item {
  int run, a, b, c;
};

enum CellblockMode { MODE_STEP = 0, MODE_SET = 1, MODE_ADD = 2, MODE_FORCES = 3 };

constexpr int SCAN_CHUNK = 2048;
constexpr int FFT_THREADS = 512;
constexpr int FFT2_THREADS = 256;  // power-of-two path (register-radix transform)
constexpr int FFT2_WIDE_THREADS = 1024;  // column pass of meshes of 2048 and more (several columns per item)
constexpr int MAX_FFT_SMEM = 200 * 1024;

// One FFT launch: its items, dynamic shared memory and threads per CTA.
struct FftPass {
  const Item* items;
  int n;
  size_t smem;
  int threads;
};

size_t deposit_smem(int mt_max, int rows_max);

int set_kernel_attributes();
int launch_deposit(const RunDesc* runs, const RunDyn* dyn, const Item* items, int n, int mt_max,
                   int rows_max, int scheme_override, int require_active, cudaStream_t s);
// the three power-of-two passes of all runs with mesh 2^lz
struct Fft2Group {
  int lz;
  FftPass pass[3];
};

// rows forward, columns + Green, rows inverse: gen[] the kernels for meshes
// with a factor 3 (radix 4/2/3), g2[] one group per power-of-two mesh size;
// ev[0..2] (optional) recorded after each pass; npass < 3 stops early
int launch_fft(const RunDesc* runs, const RunDyn* dyn, const FftPass gen[3], const Fft2Group* g2, int ng2,
               int require_active, cudaStream_t s, cudaEvent_t* ev = nullptr, int npass = 3);
// deposit (MODE_STEP): also add the new positions to each run's R.dacc.
// shape: the compiled form of the particle kernel (same arithmetic):
// PART_SHAPE_DEFAULT (registers for four 256-thread CTAs per SM) or
// PART_SHAPE_5CTA (for five)
enum PartShape { PART_SHAPE_DEFAULT = 0, PART_SHAPE_5CTA = 1 };
int launch_particles(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, int mode,
                     int mask, int require_active, cudaStream_t s, int deposit = 0,
                     int shape = PART_SHAPE_DEFAULT);
// Pipelined stage step (power-of-two meshes, fixed dt, every run with its
// R.dacc): particles (launch_particles with deposit), then the scan and the
// scatter with the step end beside the transform of the new density:
// forward rows (pass 1), columns + Green (pass 2), inverse rows (pass 0).
// Transform items carry log2 Z in Item.b; smem is the largest item's shared
// memory; runs whose `sorting` flag is clear are skipped.
int launch_pipe_fft(int pass, const RunDesc* runs, RunDyn* dyn, const Item* items, int n, size_t smem,
                    cudaStream_t s);
// the six-launch form's scan: one CTA per group of PIPE_SCAN_GROUP chunks of
// one run (Item.a: its first chunk), and its scatter: one CTA per unit of
// PIPE_SCATTER_UNIT particles (Item.a: the unit's index in the run), then
// the chunk totals cleared and the steps ended
// two chunks per CTA: 41 us for the 256-run ensemble's scan, four: 55 us
constexpr int PIPE_SCAN_GROUP = 2;
constexpr int PIPE_SCATTER_UNIT = 1024;
int launch_pipe_scan(const RunDesc* runs, RunDyn* dyn, const Item* groups, int ngroup, cudaStream_t s);
int launch_pipe_scatter(const RunDesc* runs, RunDyn* dyn, const Item* units, int nunit, const Item* chunks,
                        int nchunk, cudaStream_t s);
// Two-launch form of the pipelined step: launch_particles (with deposit),
// then one cooperative launch of the sort and the transforms, phases C (scan
// chunks and next forward rows), D (scatter, next columns + Green, step end)
// and A (inverse rows: the next step's force grids). Unit lists:
// Item.b >= 3 a transform item (log2 Z), Item.b < 0 a scan chunk (C, Item.a)
// or a scatter unit of PIPE_SCATTER_UNIT particles (D, Item.a).
struct PipeTail {
  const Item* cunits;
  int ncu;
  const Item* dunits;
  int ndu;
  const Item* chunks;  // every chunk of every run (totals cleared, steps ended)
  int nchunk;
  const Item* inv;     // inverse row items
  int ninv;
  unsigned max_polls;  // grid-barrier poll bound (0: the default, about a second)
  size_t smem;    // the largest transform item's shared memory
  int minb;       // CTAs per SM the registers are bounded for (2, 3 or 4)
  int grid;       // filled by pipe_tail_configure
};
int pipe_tail_configure(PipeTail& P, int device);
// bar: the two grid-barrier words (zero; each launch leaves them zero); ts
// (optional): 4 device timestamps (ns), start and the ends of C, D and A
int launch_pipe_tail(const RunDesc* runs, RunDyn* dyn, const PipeTail& P, unsigned* bar, cudaStream_t s,
                     unsigned long long* ts = nullptr);
int launch_move(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, int require_active,
                int refresh_only, cudaStream_t s);
int launch_count(const RunDesc* runs, const Item* items, int n, cudaStream_t s);
// dst[src[i].pid] = src[i] for the n records of one run
int launch_records_by_pid(const Rec* src, Rec* dst, int n, cudaStream_t s);
// scan of the cell counts (chunk offsets of runs run0 .. run0+nruns-1, then
// chunks) and scatter (particles); end_step_flag: also end the step of every
// run (adaptive: take the reduced dt bound)
int launch_sort(const RunDesc* runs, RunDyn* dyn, int run0, int nruns, const Item* chunks, int nchunks,
                const Item* parts, int nparts, int end_step_flag, int adaptive, int require_active, cudaStream_t s,
                cudaEvent_t* ev = nullptr);
// Fused step (one run, power-of-two mesh 2^lz with lz in [3, 10], fixed dt):
// work sizes of its phases
struct FusedPlan {
  int lz;
  int lrf, nrf;    // row items: 2^lrf rows, nrf items
  int lw, ncl;     // column items
  int lri, nri;    // inverse row items
  int nch;         // scan chunks
  size_t smem;     // dynamic shared memory
  int grid;        // CTAs (all resident: cooperative launch)
  unsigned long long* dacc;  // Z*Z density accumulator, zero between fused steps
  // grid-barrier waits give up after this many polls (0: the default bound,
  // about a second); a wait that gives up fails that barrier for every CTA
  unsigned max_polls;
  // recovery-path test: CTA skip_cta returns instead of arriving at barrier
  // skip_barrier (1-based; 0: none), so every other CTA's wait gives up
  int skip_barrier, skip_cta;
};
// fills smem and grid (occupancy of the cooperative kernel); returns 0 or a
// cudaError_t
int fused_configure(FusedPlan& P, int device);
// one step of one run (its description by value, its state in *dyn); bar:
// the two device words of the grid barrier, zero before the first launch
// (each launch leaves them zero). The FFT item counts nrf, ncl, nri must not
// exceed grid. The step starts from the column-transformed, Green-multiplied
// spectrum of the current positions (spec2), which the previous fused step
// leaves behind; otherwise deposit + forward row and column passes must run
// first (the stage kernels). It leaves the same for the next step, with the
// accumulator dacc cleared again.
// ts (optional): FUSED_PHASES + 1 device timestamps (ns) of the phase ends:
// [0] inverse row FFT [1] particles (forces, noise, move, next density)
// [2] cell-count scan + next row FFT [3] scatter + next column FFT + Green
constexpr int FUSED_PHASES = 4;
int launch_fused(const RunDesc& run, RunDyn* dyn, const FusedPlan& P, unsigned* bar, cudaStream_t s,
                 unsigned long long* ts = nullptr);
// TimestepInfo reductions of run 0 into acc (diag_bytes() of device memory):
// energy, virial (double), largest |F|^2 << 32 | index of WCA, capillary,
// noise forces (uint64 x 3), examined WCA pairs (uint64)
int launch_diag(const RunDesc* runs, int N, void* acc, cudaStream_t s);
size_t diag_bytes();
// observables of run 0: pair-distance counts hist[bins] (which 0: 11,
// 1: 12, 2: 22; cells searched within `range` of each particle's) and the
// density Fourier sums re/im[qbins*qbins] of one species
int launch_korr(const RunDesc* runs, int N, int which, int bins, double dr, int range, unsigned long long* hist,
                cudaStream_t s);
int launch_ftrho(const RunDesc* runs, int N, int species, int qbins, double dq, double* re, double* im,
                 cudaStream_t s);
// local densities of run 0 (main_auswertung.cpp:182-390): the TSC lattice
// grid[2][n*n] (FP64, species 1 then 2), then the histograms hist[4][bins]
// and threshold counts hist[4*bins .. +7]
struct LdSnap {
  int n;
  double w, drho;
};
struct LdHist {
  int n, bins;
  double dbin;
  double rho_thresh[3];
  double drho_thresh[4];
};
int launch_lokdens(const RunDesc* runs, int N, const LdSnap& sp, const LdHist& hp, double* grid, unsigned* hist,
                   cudaStream_t s);
int launch_interp(const RunDesc* runs, const Item* items, int n, int scheme, cudaStream_t s);
int launch_noise(const RunDesc* runs, const RunDyn* dyn, const Item* items, int n, cudaStream_t s);
int launch_dtbound(const RunDesc* runs, RunDyn* dyn, const Item* items, int n, cudaStream_t s);
int launch_green(float* green, float* sxt, float* syt, int Z, double kap, double lambda,
                 double L, cudaStream_t s);

}  // namespace bd

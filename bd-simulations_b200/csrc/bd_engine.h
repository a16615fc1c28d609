// Engine: device state of one or many runs and the launch plan of a step.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "bd_api.h"
#include "bd_common.cuh"
#include "bd_kernels.h"

namespace bd {

struct RunHost {
  bd_params p{};
  uint64_t seed = 0;
  std::mt19937_64 gen;  // the initialisers' stream
  RunDesc d{};          // host mirror holding the device pointers
  RunDyn dyn{};         // saved device state while the launch plan is rebuilt
  int C = 0, Z = 0, N = 0;
  double B = 0, dx = 0;
  int mt = 0, rows_max = 0, lrf = 0, lw = 0, lri = 0;
  bool adaptive = false, idgas = false;
  bool has_pos = false;  // positions uploaded and cell-sorted
  size_t bytes = 0;
  // work items of this run's own counting sort (particle blocks, then scan
  // chunks), built and uploaded once by its first sort
  Item* d_sort = nullptr;
  int n_sort_part = 0, n_sort_chunk = 0;
  int sort_items_run = -1;  // the run index the items were built for
  // observation files (RunObs)
  std::string pos1, pos2;
  long long obs_nr = 0;
  double t_obs = 0.0;
};

// Host threads for the per-call conversions of positions between the
// reference layout and the device records: run(n, fn) calls fn(k) for every
// k in [0, n) on the workers and the calling thread and returns once all are
// done. Workers wait on a condition variable between calls. One call at a
// time per pool (the engine's calls come from one thread).
class HostPool {
 public:
  explicit HostPool(int workers);
  ~HostPool();
  void run(int n, const std::function<void(int)>& fn);
  // fn(k) on the workers; after(k) on the calling thread, in order of k, as
  // soon as fn(0..k) have returned
  void run_ordered(int n, const std::function<void(int)>& fn, const std::function<void(int)>& after);

 private:
  void work();
  void drain(unsigned g);
  std::vector<std::thread> th_;
  std::mutex m_;  // guards everything below but done_
  std::condition_variable cv_;
  const std::function<void(int)>* job_ = nullptr;
  int njob_ = 0, next_ = 0;
  unsigned gen_ = 0;
  bool stop_ = false;
  std::atomic<int> done_{0};
};

class Engine {
 public:
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<RunHost*> runs;

  ~Engine();
  int init(int dev);
  // allocate a run's device memory (positions empty until uploaded)
  int add_run(const bd_params& p, uint64_t seed, RunHost** out = nullptr);
  int remove_run(size_t idx);  // frees its memory; plan must be rebuilt
  // rebuild the run table, the work lists and the graphs
  int build_plan();

  // positions in the reference layout; set also sorts (WCA_init)
  int set_positions(size_t run, int species, const int32_t* git, const double* rel);
  int set_all_positions(size_t run, int32_t* git[2], double* rel[2]);
  int get_positions(size_t run, int species, int32_t* git, double* rel);
  int get_positions_both(size_t run, int32_t* git[2], double* rel[2]);
  int get_records(size_t run, std::vector<Rec>& out);  // the cell-sorted records, one copy
  int sort_uploaded();  // counting sort of every run's recB into recA
  int sort_uploaded_run(size_t run);

  int step(long long nsteps);  // fused steps for every run
  int sync_check();            // synchronise and report run errors
  int get_dyn(size_t run, RunDyn* d);
  int set_dyn_field_step(size_t run, unsigned long long step);
  int set_dyn_time(size_t run, double t, float dt);
  int set_steps_left(size_t run, long long n);
  // per-run step budgets for the next steps (one copy each way)
  int set_steps_left_all(const std::vector<long long>& n);
  int get_dyn_all(std::vector<RunDyn>& out);

  // drop-in routines (single run, run index 0)
  int wca(int mode, int mask);
  int kap(int scheme);
  int deposit(int scheme);
  int fft();
  int interp(int scheme);
  int noise();
  int dtbound(double* dt);
  int refresh();
  int get_forces(int kind, int species, double* out);
  int get_grid(int which, double* out);

  size_t footprint_of(const bd_params& p);
  int launches_per_step() const;
  int stage_times(int nsteps, double* ms, int nstages);
  // stage-kernel plan targets: build_plan halves deposit tiles and transform
  // items until one launch has at least this many (autotune() picks them)
  int dep_tiles_min = 148, fft_items_min = 296;
  // compiled form of the step's particle kernel (PartShape; autotune() picks it)
  int part_shape = PART_SHAPE_DEFAULT;
  // form of the pipelined step (set_step_form; same bits either way):
  // PIPE_SIX: six launches on two streams; PIPE_TWO: the particle kernel and
  // one cooperative launch of everything else
  enum { PIPE_SIX = 0, PIPE_TWO = 1 };
  int pipe_form = PIPE_SIX;  // the faster on every mix measured on a B200
  int tail_minb = 4;  // CTAs per SM of the cooperative launch (2, 3 or 4)
  int set_step_form(int form, int ctas);  // rebuilds the plan and graphs
  int autotune(int reps, bd_tune_result* out);
  int fused_phase_times(int nsteps, double* ms, int nphases);  // fused or pipelined step
  int pipe_phase_times(int nsteps, double* ms, int nphases);
  int pipe2_phase_times(int nsteps, double* ms, int nphases);
  int timestep_info(bd_timestep_info* info);
  int zeitschritt_debug(double mrd, bd_timestep_info* info, double* dt);
  int korrelation(int which, double dr, int bins, double* g);
  int ftrho(int species, int qbins, double dq, double* re, double* im);
  int lokale_dichte(const bd_lokdens_params& lp, double* rho1, double* rho2, int32_t* hist, int32_t* over);
  bool uses_fused() const { return fused; }
  bool uses_pipeline() const { return piped; }
  // recovery-path test: the next fused step has CTA (grid - 1) leave instead
  // of arriving at grid barrier `barrier` (1..3) and every wait give up after
  // max_polls polls; BD_ERR_STATE without the fused step
  int inject_barrier_timeout(int barrier, unsigned max_polls);

 private:
  RunDesc* d_runs = nullptr;
  RunDyn* d_dyn = nullptr;
  size_t d_runs_cap = 0;
  Item* d_items = nullptr;
  size_t d_items_cap = 0;
  // offsets into d_items
  int off_dep = 0, n_dep = 0;
  // FFT launches, passes [0] rows forward [1] columns + Green [2] rows
  // inverse: one set for meshes with a factor 3, one per power-of-two size
  struct FftSet {
    int lz = 0;
    int off[3] = {}, n[3] = {}, thr[3] = {};
    size_t sm[3] = {};
  };
  FftSet fft_gen;
  std::vector<FftSet> fft_p2;
  int off_part = 0, n_part = 0, off_chunk = 0, n_chunk = 0;
  int off_part_all = 0, n_part_all = 0;  // particle items incl. idgas runs
  int mt_max = 0, rows_max = 0;
  bool split = false;
  cudaMemPool_t pool = nullptr;  // the runs' device arrays (stream-ordered, kept mapped)
  bool planned = false;    // work lists, fused plan and graphs built for the current runs
  bool tables_ok = false;  // d_runs / d_dyn hold the current runs (device state authoritative)
  bool descs_ok = false;   // d_runs holds the current runs' descriptions (cleared when they change)
  int upload_tables();
  // pinned host buffer of the position copies (records in and out): copies
  // from it run asynchronously at full link speed; ev_stage marks the end of
  // the last copy that uses it, waited on before the host writes it again
  void* h_stage = nullptr;
  size_t h_stage_cap = 0;
  cudaEvent_t ev_stage = nullptr;
  int stage_buffer(size_t bytes, void** out);
  // the device -> host copies of a run's records go in up to this many
  // pieces, each with its event, converted as they arrive
  static constexpr int MAX_COPY_PIECES = 64;

 public:
  static constexpr int max_copy_pieces() { return MAX_COPY_PIECES; }

 private:
  cudaEvent_t ev_piece[MAX_COPY_PIECES] = {};
  // converts the pieces in parallel (created by the first copy)
  std::unique_ptr<HostPool> hpool;
  HostPool& host_pool();
  int download_dyn();
  // fused step (one run, power-of-two mesh up to 1024^2, fixed dt): one
  // cooperative launch per step instead of the stage kernels
  bool fused = false;
  FusedPlan fplan{};
  unsigned* d_bar = nullptr;
  // pipelined stage step (power-of-two meshes, fixed dt, two or more runs):
  // six launches per step, the density deposited in the move, its transform
  // beside the cell sort. Its transform items of every mesh size (log2 Z in
  // Item.b) and their shared memory:
  bool piped = false;
  // its second stream (the transform kernels beside the sort) and the events
  // that fork and join it
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork[2] = {nullptr, nullptr}, ev_join[2] = {nullptr, nullptr};
  int enqueue_pipe(cudaStream_t s, cudaEvent_t* ev);
  int off_pinv = 0, n_pinv = 0, off_pfwd = 0, n_pfwd = 0, off_pcol = 0, n_pcol = 0;
  size_t sm_pinv = 0, sm_pfwd = 0, sm_pcol = 0;
  int off_pscan = 0, n_pscan = 0;  // groups of PIPE_SCAN_GROUP scan chunks
  int off_psu = 0, n_psu = 0;      // scatter units of PIPE_SCATTER_UNIT particles
  // two-launch form (pipe_form PIPE_TWO): the particle kernel, then one
  // cooperative launch of the sort, the next transforms and the next step's
  // inverse rows. Its unit lists (phase C: forward rows among scan chunks,
  // phase D: columns among scatter units) and launch shape:
  int off_cu = 0, n_cu = 0, off_du = 0, n_du = 0;
  PipeTail tplan{};
  bool tail_ok = false;  // the cooperative tail kernel fits (else six launches)
  int enqueue_pipe2(cudaStream_t s, unsigned long long* ts = nullptr);
  // fused and pipelined steps: whether the spectrum (spec2) belongs to the
  // current positions, with every run's density accumulator (RunDesc::dacc)
  // zero; cleared when positions change outside those steps (stream-ordered)
  bool dep_valid = false;
  int dep_invalidate();
  int fused_prologue();
  // one-shot fault of the next fused launch (inject_barrier_timeout)
  int fault_barrier = 0;
  unsigned fault_polls = 0;
  // after a failed grid barrier: the run back at its state before the step
  int recover_fused();
  cudaGraphExec_t g1 = nullptr, gK = nullptr;
  int K = 16;

  int enqueue_step(cudaStream_t s, cudaEvent_t* ev = nullptr);
  int enqueue_fft(int require_active, cudaStream_t s, cudaEvent_t* ev);
  int time_mesh_passes(int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms);
  int time_particles(int shape, int reps, cudaEvent_t e0, cudaEvent_t e1, double* ms);
  int tune_particles(int reps, cudaEvent_t e0, cudaEvent_t e1, bd_tune_result* out);
  int plan_fused();
  int plan_tail();
  int make_graphs();
  void drop_graphs();
  Item* it(int off) { return d_items + off; }
};

int status_from_cuda(cudaError_t e);

}  // namespace bd

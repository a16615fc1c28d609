/*
 * bd_api.h — C ABI of the B200 Brownian-dynamics timestep library
 * (libbd_b200.so). Drop-in for the force-and-integrate path of
 * BD-Simulations: parameters keep the names of parameter.h, the routines keep
 * the names of RunZustand::RunDynamik (signaturen2.h:68-188), and snapshots
 * keep the pos1_<run+1>.txt / pos2_<run+1>.txt text format.
 *
 * Conventions (differences from the reference are deliberate):
 *  - every call returns an int status (BD_OK = 0, negative on error) where
 *    the reference returns void and prints to cout;
 *  - parameters are a runtime struct where the reference compiles consts;
 *  - device memory belongs to the context; host buffers belong to the caller
 *    and are copied; layouts at the boundary are the reference's: positions as
 *    git int32[N][2] (cell indices) and rel double[N][2] (in-cell offsets),
 *    forces as double[N][2], mesh grids as double[Z*Z] with index k*Z + l
 *    (k the x index, allgemeine_methoden.cpp:242-250);
 *  - calls on one context are not thread-safe; distinct contexts may be
 *    driven from distinct host threads;
 *  - there is no CPU fallback: without a usable CUDA device bd_create returns
 *    BD_ERR_CUDA.
 */
#ifndef BD_API_H
#define BD_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BD_OK 0
#define BD_ERR_ARG (-1)         /* invalid argument or parameter set */
#define BD_ERR_CUDA (-2)        /* CUDA runtime error / no device */
#define BD_ERR_UNSUPPORTED (-3) /* parameter outside the supported range */
#define BD_ERR_RANGE (-4)       /* position outside the reference's invariants */
#define BD_ERR_STATE (-5)       /* call not valid in the current state */
#define BD_ERR_IO (-6)          /* file could not be opened / parsed */
#define BD_ERR_NOMEM (-7)       /* device memory or admission budget exhausted */
#define BD_ERR_NONFINITE (-8)   /* a particle position became NaN or Inf */
#define BD_ERR_NOTFOUND (-9)    /* unknown request id */
#define BD_ERR_TIMEOUT (-10)    /* a device-side wait gave up (grid barrier of the fused
                                   step); the step did not take place, the run is back at
                                   its state before it and the context stays usable */

/* noise distributions (extension: the reference draws the uniform disk) */
#define BD_NOISE_DISK 0  /* uniform on the disk of radius sqrt(5), dynamik_methoden.cpp:1317-1339 */
#define BD_NOISE_GAUSS 1 /* N(0,1) per component */
#define BD_NOISE_NONE 2  /* noiseless */

/* force kinds for bd_get_forces */
#define BD_FORCE_WCA 0
#define BD_FORCE_KAP 1
#define BD_FORCE_NOISE 2

/* mesh grids for bd_get_grid */
#define BD_GRID_DENSITY 0
#define BD_GRID_FX 1
#define BD_GRID_FY 2

/* Run parameters; names, meaning and defaults of parameter.h:14-139. */
typedef struct bd_params {
  int N1, N2;
  double L;
  int densGrid_Schema; /* 0 NGP, 1 CIC, 2 TSC */
  int FFT_samples;     /* mesh points per side; 2^a 3^b, 8..4096 */
  double lambda_kapillar, kapillar_vorfaktor, T, dt_max, max_reisedistanz;
  double sigma11_22, sigma11_12, Gamma2_1, eps22_11, eps12_11, f2_f1;
  int idgas_only, noWCA, noRNG, quickInit, restrictRadial, debugmode, krafttestmode;
  double maxPairWCA;
  int max_write_interval, runs, jobs, maxThreads;
  double obs_dt;
  int obs_anzahl;
  int startpos_methode;
  double startpos_kreisradius;
  /* extensions without a parameter.h counterpart */
  int noise_kind;     /* BD_NOISE_*, default BD_NOISE_DISK */
  int ngp_ref_compat; /* 1 (default): NGP species-2 y force read from Im(Fx), i.e. 0 */
} bd_params;

/* Derived constants, computed as parameter.h:171-209. */
typedef struct bd_derived {
  double zweihoch1_6;
  int nachList_Zellen;
  double nachList_Breite;
  double densGrid_Breite;
  int densGrid_Zellen;
  double dq;
  int fixed_dt; /* 1 when max_reisedistanz >= 1e20: dt = dt_max every step */
} bd_derived;

typedef struct bd_ctx bd_ctx;       /* one run (RunZustand + RunDynamik) */
typedef struct bd_batch bd_batch;   /* many independent runs stepped together */
typedef struct bd_server bd_server; /* continuous-batching request loop */

const char* bd_version(void);
const char* bd_status_string(int status);
int bd_device_count(int* n);

/* parameter.h:14-139 as shipped, plus the extension defaults */
int bd_params_default(bd_params* p);
/* reads a parameter.h-style file (const <type> name = expr;) over the defaults */
int bd_params_from_header(const char* path, bd_params* p);
/* parameter.h:171-209 */
int bd_params_derived(const bd_params* p, bd_derived* d);

/* ---- one run ------------------------------------------------------------ */
/* RunZustand::init allocation + RunDynamik::init (allgemeine_methoden.cpp:256-320,
 * 361-364); positions start empty until bd_init_positions / bd_set_positions.
 * seed seeds the host mt19937_64 of the initialisers (zufall.cpp:18, seeded
 * with time(NULL) there) and keys the device Philox noise stream. */
int bd_create(const bd_params* p, uint64_t seed, int device, bd_ctx** out);
int bd_destroy(bd_ctx* c);
/* startpos_methode switch (allgemeine_methoden.cpp:276-303): 1 random
 * (init_zufallspos, dynamik_methoden.cpp:1647-1678), 3 grid, 4 all-same,
 * 5 disk, 6 core+ring, 7 force test; 2 (file) is bd_init_pos_aus_datei */
int bd_init_positions(bd_ctx* c, int methode);
/* init_pos_aus_datei (dynamik_methoden.cpp:1578-1643) with the rel = x - git*B
 * fix; file format: two header lines, then "idx TAB type TAB x TAB y" rows */
int bd_init_pos_aus_datei(bd_ctx* c, const char* path);
/* set/get r?_git, r?_rel of one species (0 or 1); set requires
 * 0 <= git < nachList_Zellen and -B < rel <= 2B, and rebuilds the cell order
 * (WCA_init) without re-binning */
int bd_set_positions(bd_ctx* c, int species, const int32_t* git, const double* rel);
int bd_get_positions(bd_ctx* c, int species, int32_t* git, double* rel);
/* both species in one host<->device copy (16 bytes per particle each way) */
int bd_set_positions_all(bd_ctx* c, const int32_t* git1, const double* rel1,
                         const int32_t* git2, const double* rel2);
int bd_get_positions_all(bd_ctx* c, int32_t* git1, double* rel1, int32_t* git2, double* rel2);

/* WCA_init (dynamik_methoden.cpp:459-526): counting sort by cell */
int bd_WCA_init(bd_ctx* c);
/* kapkraefte_init (dynamik_methoden.cpp:529-613): Green's tables in FP64 */
int bd_kapkraefte_init(bd_ctx* c);
/* berechne_WCA11 (:617-702), berechne_WCA22 (:790-879), addiere_WCA12 (:973-1059) */
int bd_berechne_WCA11(bd_ctx* c);
int bd_berechne_WCA22(bd_ctx* c);
int bd_addiere_WCA12(bd_ctx* c);
/* berechne_kapkraefte (:1180-1233) */
int bd_berechne_kapkraefte(bd_ctx* c);
/* gridDensity_* / inv_gridDensity_* (gridRoutinen.cpp:31-668) */
int bd_gridDensity_NGP(bd_ctx* c);
int bd_gridDensity_CIC(bd_ctx* c);
int bd_gridDensity_TSC(bd_ctx* c);
int bd_inv_gridDensity_NGP(bd_ctx* c);
int bd_inv_gridDensity_CIC(bd_ctx* c);
int bd_inv_gridDensity_TSC(bd_ctx* c);
/* berechne_zufallskraefte (:1317-1339) for the current step */
int bd_berechne_zufallskraefte(bd_ctx* c);
/* optimaler_zeitschritt (:1420-1491) over the current force/noise buffers */
int bd_optimaler_zeitschritt(bd_ctx* c, double* dt);
/* refresh_erwNachbar (:216-325) */
int bd_refresh_erwNachbar(bd_ctx* c);
/* zeitschritt (:74-163): one fused step; *dt_out = the step length used
 * (tmax is ignored as in the reference; tmax <= 0 returns BD_ERR_ARG and
 * *dt_out = 1e10) */
int bd_zeitschritt(bd_ctx* c, double tmax, double* dt_out);
/* nsteps fused steps replayed from captured CUDA graphs; *t_out = simulated time */
int bd_zeitschritte(bd_ctx* c, long long nsteps, double* t_out);
/* zeitschritte_bis_obs (:444-455): steps until the time since the last
 * observation point reaches obs_dt; *nsteps_out = steps taken */
int bd_zeitschritte_bis_obs(bd_ctx* c, long long* nsteps_out);
/* RunDynamik::TimestepInfo (signaturen2.h:71-145): what zeitschritt_debug
 * (dynamik_methoden.cpp:168-211) records about the forces of the current
 * positions and step, without moving. Indices count within the species,
 * types are 1 or 2. Extensions: the WCA potential energy
 * sum 4 eps (s^-12 - s^-6) + eps over pairs within the cutoff (s = r*sigma,
 * the potential of the uncapped force) and the virial sum r.F of the WCA
 * force the step uses, both reduced in FP64. */
typedef struct bd_timestep_info {
  long long num_WCA_berechnet; /* pairs the WCA11/22/12 loops examine */
  double maxWCAx, maxWCAy;     /* largest WCA force */
  int maxWCAtype, maxWCAindex;
  int maxWCA_numWW1, maxWCA_numWW2; /* type-1 / type-2 particles in its 3x3 cells */
  double maxKapx, maxKapy;     /* largest capillary force */
  int maxKaptype, maxKapindex;
  double maxRNDx, maxRNDy;     /* largest noise vector */
  int maxRNDtype, maxRNDindex;
  double dt;                   /* the step the next zeitschritt takes */
  int num_Zellwechsel1, num_Zellwechsel2; /* cell changes in the last completed step */
  double E_WCA, virial_WCA;
} bd_timestep_info;
int bd_zeitschritt_info(bd_ctx* c, bd_timestep_info* info);
/* zeitschritt_debug (dynamik_methoden.cpp:168-211): one step of length
 * optimaler_zeitschritt(mrd) (:1495-1560: the travel bound mrd in place of
 * max_reisedistanz, at most dt_max, also for fixed-dt runs), recording the
 * TimestepInfo of its forces; num_Zellwechsel1/2 are this step's cell
 * changes, dt (and *dt_out, may be NULL) its length. The step is
 * zeitschritt's: the reference's debug variants examine the wrong cell in
 * WCA11 (dynamik_methoden.cpp:725), never fill maxWCA, draw noise under noWCA
 * and skip restrictRadial; none of that is reproduced. */
int bd_zeitschritt_debug(bd_ctx* c, double mrd, bd_timestep_info* info, double* dt_out);
/* Observables of the resident state, the reference's in-run analysis
 * (auswertung.cpp), here the tools of the statistical comparison:
 * g11 / g12 / g22 (record_korrelationsfunktion11/12/22, auswertung.cpp:
 * 110-188; which 0, 1, 2): pair counts in korr_bins bins of width korr_dr
 * (every pair once, minimum image, FP64 distances), normalised as the
 * reference: g[b] = count * vorfaktor / (2b + 1). korr_bins <= 8192; the
 * reference's korr_rmax = L/2 makes it an all-pairs sum, so pick the range
 * to fit the run's size. */
int bd_korrelationsfunktion(bd_ctx* c, int which, double korr_dr, int korr_bins, double* g);
/* rho(k) of one species (record_ftrho_unkorrigiert, auswertung.cpp:307-380):
 * re + i im = sum over the particles of exp(i k.r) for k = dq (i, j),
 * 0 <= i, j < qbins (<= 64), i^2 + j^2 <= qbins^2, index i*qbins + j, zero
 * outside the disk; FP64. The reference's species-1 loop takes y from the x
 * offset (auswertung.cpp:333); this one uses y. */
int bd_ftrho(bd_ctx* c, int species, int qbins, double dq, double* re, double* im);
/* Local densities of the offline analysis program (main_auswertung.cpp:
 * 182-390), computed from the resident state. Its compile-time constants
 * (parameter.h:109-124,161,174) become a parameter block: */
typedef struct bd_lokdens_params {
  double snapgrid_crude; /* lattice width about this: snapgrid_num =
                            2*(int)(L/(2*snapgrid_crude)+0.5), width L/snapgrid_num */
  int rhohist_bins;      /* histogram bins (<= BD_RHOHIST_MAX_BINS) */
  double rhohist_drho;   /* bin width: bin b holds rhohist_drho*(b+0.5) */
  double rho_thresh[3];  /* count cells with rho1+rho2 over each */
  double drho_thresh[4]; /* count cells with |rho1-rho2|/(rho1+rho2) over each */
} bd_lokdens_params;
#define BD_SNAPGRID_MAX 16384
#define BD_RHOHIST_MAX_BINS 2048
/* the shipped values: 0.5, 100, 0.01, {0.1, 0.2, 0.5}, {0.1, 0.2, 0.5, 0.99} */
void bd_lokdens_params_default(bd_lokdens_params* lp);
/* the same names read from a parameter.h (absent names keep their value) */
int bd_lokdens_params_from_header(const char* parameter_h_path, bd_lokdens_params* lp);
/* snapgrid_num of a run (parameter.h:174) */
int bd_snapgrid_num(const bd_params* p, const bd_lokdens_params* lp, int* n);
/* The TSC-gridded densities (localDens/rho<t>.txt, main_auswertung.cpp:
 * 184-300): every particle adds w_x w_y / width^2 to nine cells;
 * rho1 / rho2: double[n*n], index k*n + l, k along x (NULL: not copied).
 * Positions are the resident FP64 values cell*B + offset (the program
 * itself reads %g text). Cells are summed with FP64 atomic adds: each value
 * is within a few ulp of the reference's particle-order sum, and the order
 * of the adds, so the last bits, may change from call to call.
 * hist: int32[4][rhohist_bins] cell counts of rho1, rho2, rho1+rho2 and
 * rho1-rho2 (rhoHist.txt / drhoHist.txt print count / n^2); over: int32[7]
 * counts over rho_thresh[0..2] then drho_thresh[0..3] (rhoThresh.txt /
 * drhoThresh.txt; a cell with rho1+rho2 = 0 is never over a drho
 * threshold). Any output may be NULL. */
int bd_lokale_dichte(bd_ctx* c, const bd_lokdens_params* lp, double* rho1, double* rho2,
                     int32_t* hist, int32_t* over);
/* The program's output files for frame nr (t = nr*obs_dt), in its formats
 * (main_auswertung.cpp:60-77,205-210,290-296,357-375): writes
 * <dir>/localDens/rho<nr>.txt (the directory is created) and appends a frame
 * to <dir>/rhoHist.txt, drhoHist.txt, rhoThresh.txt, drhoThresh.txt, which
 * nr == 0 creates afresh with the program's headers. */
int bd_schreibe_lokale_dichte(bd_ctx* c, const bd_lokdens_params* lp, const char* dir, int nr);
/* F?_WCA / F?kap / F?_noise of one species as double[N][2]: the forces the
 * last force routine (bd_berechne_*, bd_berechne_zufallskraefte), TimestepInfo
 * call (bd_zeitschritt_info, bd_zeitschritt_debug) or adaptive-dt step left.
 * A fixed-dt step keeps its forces in registers and does not store them (the
 * reference's arrays hold the last step's; call bd_zeitschritt_info for the
 * forces of the current positions). */
int bd_get_forces(bd_ctx* c, int kind, int species, double* out);
/* rhox / Fx / Fy mesh as double[Z*Z] */
int bd_get_grid(bd_ctx* c, int which, double* out);
/* erwNachbarn?[i][j]: particles of `species` in cells (i+-1, j+-1), built
 * from the current cell keys, in ascending particle index; *n = full length.
 * Right after WCA_init this is the reference's own list (dynamik_methoden.cpp:
 * 459-526). After steps the set is the reference's, but its order is not:
 * refresh_erwNachbar (:216-325, 1398-1417) erases a particle that changed
 * cell from the lists it leaves and appends it to the lists it enters, so the
 * reference's order records the history of cell changes. No result here
 * depends on that order: the WCA pair terms and the density are summed in
 * 64-bit fixed point, exact in any order (in the reference the order only
 * changes the last bits of its FP64 sums). */
int bd_get_list(bd_ctx* c, int species, int i, int j, int32_t* out, int cap, int* n);
int bd_get_step(bd_ctx* c, uint64_t* step);
int bd_set_step(bd_ctx* c, uint64_t step);
int bd_get_time(bd_ctx* c, double* t);
int bd_sync(bd_ctx* c);
/* RunObs::obs_init (auswertung.cpp:52-75): opens <dir>/pos1_<run+1>.txt (and
 * pos2_<run+1>.txt when N2 != 0) and writes the header */
int bd_obs_init(bd_ctx* c, int run, const char* dir);
/* RunObs::schreibe_pos (auswertung.cpp:631-648): appends a frame at t = nr*obs_dt */
int bd_schreibe_pos(bd_ctx* c, int nr);
/* resumable binary snapshot (no counterpart in the reference, whose only
 * restart input is the text startpos.txt): cells, the exact FP32 in-cell
 * offsets, the Philox step counter, the simulated time and the observation
 * schedule of the run. Stepping on from a loaded snapshot gives the same bits
 * as stepping on without the interruption. load requires a context created
 * with the same physical parameters and seed (else BD_ERR_ARG); the format
 * belongs to this library build (BD_ERR_IO for a file it does not know). */
int bd_snapshot_save(bd_ctx* c, const char* path);
int bd_snapshot_load(bd_ctx* c, const char* path);
/* host-only formatter of one frame in the same format (header when append == 0) */
int bd_write_pos_frame(const char* path, int append, double t, int n, const int32_t* git,
                       const double* rel, double nachList_Breite);
/* host-only: the initialisers of bd_init_positions into caller arrays */
int bd_init_positions_host(const bd_params* p, uint64_t seed, int methode, int32_t* git1,
                           double* rel1, int32_t* git2, double* rel2);

/* ---- batch of independent runs (the reference's runs loop, main.cpp:130) -- */
/* every run initialised with its startpos_methode from its own seed */
int bd_batch_create(const bd_params* runs, const uint64_t* seeds, int nruns, int device,
                    bd_batch** out);
int bd_batch_destroy(bd_batch* b);
int bd_batch_step(bd_batch* b, long long nsteps);
int bd_batch_sync(bd_batch* b);
int bd_batch_nruns(bd_batch* b, int* n);
int bd_batch_get_positions(bd_batch* b, int run, int species, int32_t* git, double* rel);
int bd_batch_set_positions(bd_batch* b, int run, int species, const int32_t* git,
                           const double* rel);
/* both species of one run in one host<->device copy and one cell sort (as
 * bd_set_positions_all / bd_get_positions_all; git2, rel2 may be NULL when
 * the run has no species 2) */
int bd_batch_set_positions_all(bd_batch* b, int run, const int32_t* git1, const double* rel1,
                               const int32_t* git2, const double* rel2);
int bd_batch_get_positions_all(bd_batch* b, int run, int32_t* git1, double* rel1, int32_t* git2,
                               double* rel2);
int bd_batch_get_time(bd_batch* b, int run, double* t);
/* bytes of device memory one run with these parameters holds */
int bd_run_footprint(const bd_params* p, size_t* bytes);

/* ---- density assignment without allocation (no counterpart in the
 * reference; its gridDensity_* routines, gridRoutinen.cpp:31-560, work on a
 * RunZustand) ----------------------------------------------------------- */
/* largest mesh side the no-allocation deposit accepts (its scratch array) */
#define BD_NOALLOC_MAX_Z 1024
/* rho = gridDensity_<scheme> of the given positions, identical to
 * bd_gridDensity_* + bd_get_grid(BD_GRID_DENSITY) on the same positions, for
 * callers that cannot allocate device memory at call time. Every pointer
 * except p is DEVICE memory owned by the caller, on the device that is
 * current at the call, as is `stream` (rho on another device: BD_ERR_ARG);
 * git?/rel? in the boundary
 * layout (int32[N?][2], double[N?][2]; git2/rel2 may be NULL when N2 == 0),
 * rho float[Z*Z] (index k*Z + l), nskipped (may be NULL) receives the number
 * of particles outside 0 <= git < nachList_Zellen, -B < rel <= 2B, which are
 * left out. Work is enqueued on `stream` (a cudaStream_t, NULL = default
 * stream); the call does not wait for it. Scratch is one 8 MiB file-scope
 * device array per device, shared by all calls: calls that overlap on the
 * device race and give undefined results; calls ordered on one stream are
 * safe. The first call on each device looks the array up (once, with that
 * device current); make it before any stream capture on that device.
 * FFT_samples > BD_NOALLOC_MAX_Z returns BD_ERR_UNSUPPORTED; scheme outside
 * 0..2 or missing pointers BD_ERR_ARG. */
int bd_gridDensity_noalloc(const bd_params* p, int scheme, const int32_t* git1, const double* rel1,
                           const int32_t* git2, const double* rel2, float* rho, int* nskipped,
                           void* stream);

/* ---- instrumentation (no counterpart in the reference; its only timing is
 * the steps/s print of main.cpp:268-276) ---------------------------------- */
/* the cudaStream_t the context launches on, for CUDA-event timing */
int bd_get_stream(bd_ctx* c, void** stream);
int bd_batch_get_stream(bd_batch* b, void** stream);
/* kernel launches one fused step makes (all runs of a batch together) */
int bd_launches_per_step(bd_ctx* c, int* n);
int bd_batch_launches_per_step(bd_batch* b, int* n);
/* runs nsteps fused steps with CUDA events between the stages and returns
 * the mean device time per step of each stage in ms:
 * [0] deposit [1] row FFT [2] column FFT + Green [3] inverse row FFT
 * [4] per-particle forces/update [5] cell-count scan (+ step end)
 * [6] scatter [7], [8] 0 (no further launches); nstages >= 9 */
int bd_stage_times(bd_ctx* c, int nsteps, double* ms, int nstages);
int bd_batch_stage_times(bd_batch* b, int nsteps, double* ms, int nstages);
/* Plan autotuning (no counterpart in the reference, which has one run on one
 * CPU thread). A batch's stage-kernel plan cuts every run's mesh work into
 * deposit tiles (a square of mesh points per CTA) and transform items (rows
 * or columns per CTA); the plan halves them until a launch has at least
 * dep_tiles_min tiles and fft_items_min items (defaults 148 and 296: one and
 * two per SM). bd_batch_autotune builds the plan for each candidate, times
 * reps mesh passes of every run with CUDA events on the batch's stream and
 * keeps the fastest plan for the later steps. Candidates: for the pipelined
 * stage step (runs on power-of-two meshes with a fixed dt; the density is
 * deposited in the move) fft_items_min in {148, 296, 592, 1184, 2368, 4736},
 * timing its three transform launches; otherwise every pair of targets in
 * {148, 296, 592, 1184}², timing the deposit and transform launches. On
 * the chosen plan it then times the step's particle kernel (forces, noise,
 * move, counts; one thread per particle, 256 per CTA) in its two compiled
 * shapes, registers for four or for five CTAs per SM (64 or 51 registers a
 * thread: more warps resident, some values reloaded), reps launches each, and
 * keeps the faster for the step graphs. Only knobs that leave every result
 * unchanged are tuned: every plan and shape gives the same bits
 * (fixed-point density and force sums, the same transform per sequence),
 * so the transform's radix schedule, which sets its rounding, is fixed per
 * mesh size; the runs' positions, step counters and noise streams are not
 * touched: the density and force grids are recomputed from the current
 * positions, as the next step does anyway, and what the timed particle
 * launches leave (cell counts, chunk totals, per-run counters, the density
 * accumulators) is put back to its state before the call.
 * BD_ERR_STATE when the batch steps in one fused launch (no tile or item
 * plan to choose); a batch of ideal-gas runs only has no mesh work, and
 * only the particle kernel's shape is timed (candidates 2). BD_ERR_ARG for
 * a missing batch or result or reps <= 0. */
typedef struct bd_tune_result {
  int dep_tiles_min;   /* chosen targets */
  int fft_items_min;
  int dep_tile_max;    /* largest deposit tile edge (mesh points) of the chosen plan */
  int candidates;      /* plans and particle-kernel shapes timed */
  double default_ms;   /* deposit + transforms per pass with the plan the call started from */
  double best_ms;      /* the same with the chosen plan */
  int particle_shape;  /* chosen particle-kernel shape: 0 four CTAs per SM, 1 five */
  double particle_default_ms; /* one particle launch in the shape the call started from */
  double particle_best_ms;    /* the same in the chosen shape */
} bd_tune_result;
int bd_batch_autotune(bd_batch* b, int reps, bd_tune_result* out);
/* Form of the pipelined stage step (no counterpart in the reference), for
 * batches of runs on power-of-two meshes with a fixed dt. form 0 (the
 * default): six launches; the particle kernel, then the cell sort (scan,
 * then scatter and step end) on one stream beside the transform of the new
 * positions (forward rows, columns + Green, inverse rows: the next step's
 * force grids) on a second, joined at the step's end; ctas_per_sm must be 0.
 * form 1: two launches, the particle kernel and one cooperative launch that
 * holds the scan beside the forward row pass, the scatter beside the column
 * pass and then the inverse row pass, separated by grid barriers, for meshes
 * up to 1024^2; ctas_per_sm (2, 3 or 4; 0 keeps the current, initially 4)
 * bounds that launch's registers. Every form gives the same bits.
 * bd_batch_launches_per_step reports 6 or 2 afterwards (form 1 falls back
 * to six launches where its cooperative launch cannot be resident or a mesh
 * is larger than 1024^2). BD_ERR_ARG for other values. */
int bd_batch_set_step_form(bd_batch* b, int form, int ctas_per_sm);
/* one run on a power-of-two mesh up to 1024^2 with a fixed dt steps in one
 * cooperative launch per step (the fused step); bd_launches_per_step then
 * reports 1 and bd_stage_times times the stage kernels instead. Runs on
 * power-of-two meshes with a fixed dt otherwise (a batch of two or more of
 * them) step in six launches per step (the pipelined stage step;
 * bd_launches_per_step reports 6): the particle kernel, then the cell sort
 * beside the transform of the new density on a second stream. This runs
 * nsteps steps and returns the mean time per step of each phase in ms (the
 * fused step: device timestamps at its grid-wide barriers; the pipelined
 * step: CUDA events on the library stream). The mesh transform is pipelined
 * across steps (the next step's density is deposited by the move):
 * fused step: [0] inverse row FFT [1] per-particle forces/update/next
 * density [2] cell-count scan + next row FFT [3] scatter + next column FFT +
 * Green (+ step end); pipelined step: [0] 0 (its inverse rows run in [3])
 * [1] the particle kernel [2] the scan [3] the scatter and step end beside
 * the forward row, column + Green and inverse row passes, to their join;
 * BD_ERR_STATE when the context uses neither; nphases >= 4 */
int bd_fused_phase_times(bd_ctx* c, int nsteps, double* ms, int nphases);
/* the same for a batch */
int bd_batch_phase_times(bd_batch* b, int nsteps, double* ms, int nphases);
/* Test of the failure path of the fused step's bounded device waits (no
 * counterpart in the reference, whose routines only print and return,
 * dynamik_methoden.cpp:80-83, 624-627, 1202). The next fused step has one
 * CTA leave instead of arriving at grid barrier `barrier` (1: after the
 * inverse row pass, 2: after the particle pass, 3: after the scan), and every
 * wait of that launch gives up after max_polls polls instead of about a
 * second. The waits then give up and the launch returns without a fault.
 * The next synchronising call (bd_zeitschritte, bd_sync; bd_zeitschritt with
 * a fixed dt only queues the step) returns BD_ERR_TIMEOUT, after which the
 * run is back at its state before the failed step and steps on with the
 * bits of a run that never failed. BD_ERR_STATE when the context does not
 * use the fused step; BD_ERR_ARG for barrier outside 1..3 or max_polls 0. */
int bd_inject_barrier_timeout(bd_ctx* c, int barrier, unsigned max_polls);

/* ---- serving: continuous batching of run requests ----------------------- */
typedef struct bd_serve_opts {
  int device;
  size_t hbm_budget;    /* bytes of device memory admitted runs may hold (0: 80% of free) */
  int max_runs;         /* at most this many runs on the device at once (0: no limit) */
  int steps_per_tick;   /* steps every active run advances per tick (graph length) */
  const char* snapshot_dir; /* NULL: snapshots kept in memory only */
} bd_serve_opts;

#define BD_REQ_QUEUED 0
#define BD_REQ_RUNNING 1
#define BD_REQ_DONE 2
#define BD_REQ_CANCELLED 3
#define BD_REQ_FAILED 4

typedef struct bd_req_status {
  int state;
  long long steps_done;
  long long steps_total;
  int snapshots;
  double submit_s, admit_s, finish_s; /* host clock, seconds since server start */
  int error;
} bd_req_status;

typedef struct bd_serve_stats {
  long long completed;
  long long particle_steps;
  double wall_s;
  double p50_latency_s, p99_latency_s, max_latency_s;
  int active, queued;
  size_t hbm_in_use;
  double step_s;  /* time in the batched step launches (CUDA events), summed over ticks */
  double host_s;  /* the rest of the ticks, of which: */
  double admit_s; /* admission: allocation, initial positions, first sort */
  double plan_s;  /* launch-plan and graph rebuilds after runs joined or left, and the
                     batch autotuner (bd_batch_autotune on the resident mix once it holds
                     2^20 particles, again whenever it has doubled since) */
  double fetch_s; /* snapshot and result copies to the host, retirement */
} bd_serve_stats;

int bd_serve_create(const bd_serve_opts* o, bd_server** out);
int bd_serve_destroy(bd_server* s);
/* queue a run: nsteps fused steps; a snapshot every snapshot_every steps
 * (0: none); returns BD_ERR_NOMEM if the run alone exceeds the budget */
int bd_serve_submit(bd_server* s, const bd_params* p, uint64_t seed, long long nsteps,
                    int snapshot_every, long long* req_id);
int bd_serve_cancel(bd_server* s, long long req_id);
int bd_serve_poll(bd_server* s, long long req_id, bd_req_status* st);
/* one tick: admit queued requests that fit, advance every active run by up to
 * steps_per_tick steps, take due snapshots, retire finished runs;
 * *active = runs still on the device */
int bd_serve_tick(bd_server* s, int* active);
/* final positions of a finished request (kept until bd_serve_release) */
int bd_serve_result(bd_server* s, long long req_id, int species, int32_t* git, double* rel);
int bd_serve_release(bd_server* s, long long req_id);
/* latest snapshot frame of a request, in the pos-file layout */
int bd_serve_snapshot(bd_server* s, long long req_id, int species, long long* step,
                      int32_t* git, double* rel);
int bd_serve_stats_get(bd_server* s, bd_serve_stats* st);

#ifdef __cplusplus
}
#endif

#endif

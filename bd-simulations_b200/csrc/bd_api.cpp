// extern "C" entry points of libbd_b200.so (declared in include/bd_api.h).
#include "bd_api.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "bd_engine.h"
#include "bd_host.h"

using bd::Engine;
using bd::RunHost;

struct bd_ctx {
  Engine e;
  long double t_obs = 0.0L;  // time since the last observation point
  long long obs_nr = 0;
  std::string pos1, pos2;
  bool obs_open = false;
};

struct bd_batch {
  Engine e;
};

#define RK(x)                \
  do {                       \
    int r_ = (x);            \
    if (r_ != BD_OK) return r_; \
  } while (0)

static int init_run_positions(Engine& e, size_t run, int methode) {
  RunHost& r = *e.runs[run];
  std::vector<int32_t> g1(2 * (size_t)r.p.N1 + 2, 0), g2(2 * (size_t)r.p.N2 + 2, 0);
  std::vector<double> q1(2 * (size_t)r.p.N1 + 2, 0.0), q2(2 * (size_t)r.p.N2 + 2, 0.0);
  int32_t* g[2] = {g1.data(), g2.data()};
  double* q[2] = {q1.data(), q2.data()};
  int st = bd::init_positions_host(&r.p, r.gen, methode, g, q);
  if (st != BD_OK) return st;
  return e.set_all_positions(run, g, q);
}

extern "C" {

const char* bd_version(void) { return "bd_b200 1.0 (sm_100a)"; }

const char* bd_status_string(int s) {
  switch (s) {
    case BD_OK: return "ok";
    case BD_ERR_ARG: return "invalid argument";
    case BD_ERR_CUDA: return "CUDA error or no device";
    case BD_ERR_UNSUPPORTED: return "unsupported parameter";
    case BD_ERR_RANGE: return "position out of range";
    case BD_ERR_STATE: return "invalid state";
    case BD_ERR_IO: return "file error";
    case BD_ERR_NOMEM: return "out of device memory or budget";
    case BD_ERR_NONFINITE: return "non-finite position";
    case BD_ERR_NOTFOUND: return "unknown request";
    case BD_ERR_TIMEOUT: return "device wait gave up; step not taken";
    default: return "unknown status";
  }
}

int bd_device_count(int* n) {
  if (!n) return BD_ERR_ARG;
  *n = 0;
  if (cudaGetDeviceCount(n) != cudaSuccess) {
    *n = 0;
    cudaGetLastError();
  }
  return BD_OK;
}

int bd_params_default(bd_params* p) {
  if (!p) return BD_ERR_ARG;
  bd::params_default(p);
  return BD_OK;
}

int bd_params_from_header(const char* path, bd_params* p) {
  if (!path || !p) return BD_ERR_ARG;
  return bd::params_from_header(path, p);
}

int bd_params_derived(const bd_params* p, bd_derived* d) {
  if (!p || !d) return BD_ERR_ARG;
  bd::params_derived(p, d);
  return BD_OK;
}

int bd_run_footprint(const bd_params* p, size_t* bytes) {
  if (!p || !bytes) return BD_ERR_ARG;
  int st = bd::params_validate(p);
  if (st) return st;
  Engine tmp;
  *bytes = tmp.footprint_of(*p);
  return BD_OK;
}

int bd_write_pos_frame(const char* path, int append, double t, int n, const int32_t* git,
                       const double* rel, double B) {
  if (!path || n < 0) return BD_ERR_ARG;
  return bd::write_pos_frame(path, append, t, n, git, rel, B);
}

int bd_init_positions_host(const bd_params* p, uint64_t seed, int methode, int32_t* git1,
                           double* rel1, int32_t* git2, double* rel2) {
  if (!p) return BD_ERR_ARG;
  int st = bd::params_validate(p);
  if (st) return st;
  std::mt19937_64 gen(seed);
  int32_t* g[2] = {git1, git2};
  double* q[2] = {rel1, rel2};
  std::vector<int32_t> dg;
  std::vector<double> dq;
  if (p->N2 > 0 && (!git2 || !rel2)) return BD_ERR_ARG;
  if (!git1 || !rel1) return BD_ERR_ARG;
  if (p->N2 == 0) {
    dg.resize(2);
    dq.resize(2);
    g[1] = dg.data();
    q[1] = dq.data();
  }
  return bd::init_positions_host(p, gen, methode, g, q);
}

// ---- single run ----------------------------------------------------------
int bd_create(const bd_params* p, uint64_t seed, int device, bd_ctx** out) {
  if (!p || !out) return BD_ERR_ARG;
  *out = nullptr;
  int st = bd::params_validate(p);
  if (st) return st;
  bd_ctx* c = new (std::nothrow) bd_ctx();
  if (!c) return BD_ERR_NOMEM;
  st = c->e.init(device);
  if (st == BD_OK) st = c->e.add_run(*p, seed);
  if (st == BD_OK) st = c->e.build_plan();
  if (st == BD_OK) {
    // RunZustand::init: positions from startpos_methode (file start: empty)
    const int m = p->startpos_methode;
    if (m != 2) {
      int s2 = init_run_positions(c->e, 0, m);
      if (s2 != BD_OK && s2 != BD_ERR_ARG) st = s2;
    }
  }
  if (st != BD_OK) {
    delete c;
    return st;
  }
  *out = c;
  return BD_OK;
}

int bd_destroy(bd_ctx* c) {
  delete c;
  return BD_OK;
}

int bd_init_positions(bd_ctx* c, int methode) {
  if (!c) return BD_ERR_ARG;
  if (methode == 2) return BD_ERR_ARG;
  return init_run_positions(c->e, 0, methode);
}

int bd_init_pos_aus_datei(bd_ctx* c, const char* path) {
  if (!c || !path) return BD_ERR_ARG;
  RunHost& r = *c->e.runs[0];
  std::vector<int32_t> g1(2 * (size_t)r.p.N1 + 2), g2(2 * (size_t)r.p.N2 + 2);
  std::vector<double> q1(2 * (size_t)r.p.N1 + 2), q2(2 * (size_t)r.p.N2 + 2);
  int32_t* g[2] = {g1.data(), g2.data()};
  double* q[2] = {q1.data(), q2.data()};
  RK(bd::init_pos_from_file(&r.p, path, g, q));
  return c->e.set_all_positions(0, g, q);
}

int bd_set_positions(bd_ctx* c, int species, const int32_t* git, const double* rel) {
  if (!c || !git || !rel) return BD_ERR_ARG;
  return c->e.set_positions(0, species, git, rel);
}

int bd_get_positions(bd_ctx* c, int species, int32_t* git, double* rel) {
  if (!c) return BD_ERR_ARG;
  return c->e.get_positions(0, species, git, rel);
}

int bd_set_positions_all(bd_ctx* c, const int32_t* git1, const double* rel1,
                         const int32_t* git2, const double* rel2) {
  if (!c || !git1 || !rel1) return BD_ERR_ARG;
  RunHost& r = *c->e.runs[0];
  if (r.p.N2 > 0 && (!git2 || !rel2)) return BD_ERR_ARG;
  int32_t dg[2] = {0, 0};
  double dq[2] = {0, 0};
  int32_t* g[2] = {const_cast<int32_t*>(git1), git2 ? const_cast<int32_t*>(git2) : dg};
  double* q[2] = {const_cast<double*>(rel1), rel2 ? const_cast<double*>(rel2) : dq};
  return c->e.set_all_positions(0, g, q);
}

int bd_get_positions_all(bd_ctx* c, int32_t* git1, double* rel1, int32_t* git2, double* rel2) {
  if (!c) return BD_ERR_ARG;
  int32_t* g[2] = {git1, git2};
  double* q[2] = {rel1, rel2};
  return c->e.get_positions_both(0, g, q);
}

int bd_WCA_init(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  // the cell order is rebuilt whenever positions are set; sort again from
  // the current state for callers that mirror the reference's call order
  RunHost& r = *c->e.runs[0];
  std::vector<int32_t> g1(2 * (size_t)r.p.N1 + 2), g2(2 * (size_t)r.p.N2 + 2);
  std::vector<double> q1(2 * (size_t)r.p.N1 + 2), q2(2 * (size_t)r.p.N2 + 2);
  RK(c->e.get_positions(0, 0, g1.data(), q1.data()));
  RK(c->e.get_positions(0, 1, g2.data(), q2.data()));
  int32_t* g[2] = {g1.data(), g2.data()};
  double* q[2] = {q1.data(), q2.data()};
  return c->e.set_all_positions(0, g, q);
}

int bd_kapkraefte_init(bd_ctx* c) { return c ? BD_OK : BD_ERR_ARG; }

int bd_berechne_WCA11(bd_ctx* c) { return c ? c->e.wca(bd::MODE_SET, 1) : BD_ERR_ARG; }
int bd_berechne_WCA22(bd_ctx* c) { return c ? c->e.wca(bd::MODE_SET, 2) : BD_ERR_ARG; }
int bd_addiere_WCA12(bd_ctx* c) { return c ? c->e.wca(bd::MODE_ADD, 4) : BD_ERR_ARG; }

int bd_berechne_kapkraefte(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  return c->e.kap(c->e.runs[0]->p.densGrid_Schema);
}

int bd_gridDensity_NGP(bd_ctx* c) { return c ? c->e.deposit(0) : BD_ERR_ARG; }
int bd_gridDensity_CIC(bd_ctx* c) { return c ? c->e.deposit(1) : BD_ERR_ARG; }
int bd_gridDensity_TSC(bd_ctx* c) { return c ? c->e.deposit(2) : BD_ERR_ARG; }

static int inv_grid(bd_ctx* c, int scheme) {
  if (!c) return BD_ERR_ARG;
  // the force grid comes from the transforms of the current density
  RK(c->e.fft());
  return c->e.interp(scheme);
}
int bd_inv_gridDensity_NGP(bd_ctx* c) { return inv_grid(c, 0); }
int bd_inv_gridDensity_CIC(bd_ctx* c) { return inv_grid(c, 1); }
int bd_inv_gridDensity_TSC(bd_ctx* c) { return inv_grid(c, 2); }

int bd_berechne_zufallskraefte(bd_ctx* c) { return c ? c->e.noise() : BD_ERR_ARG; }

int bd_optimaler_zeitschritt(bd_ctx* c, double* dt) {
  if (!c || !dt) return BD_ERR_ARG;
  return c->e.dtbound(dt);
}

int bd_refresh_erwNachbar(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  RK(c->e.refresh());
  return c->e.sync_check();
}

int bd_zeitschritt(bd_ctx* c, double tmax, double* dt_out) {
  if (!c) return BD_ERR_ARG;
  if (tmax <= 0.0) {
    if (dt_out) *dt_out = 1.0e10;
    return BD_ERR_ARG;
  }
  RK(c->e.step(1));
  RunHost& r = *c->e.runs[0];
  double dt = r.p.dt_max;
  if (r.adaptive) {
    bd::RunDyn y;
    RK(c->e.get_dyn(0, &y));
    dt = y.dt;
    if (y.err & bd::E_NONFINITE) return BD_ERR_NONFINITE;
  }
  c->t_obs += (long double)dt;
  if (dt_out) *dt_out = dt;
  return BD_OK;
}

int bd_zeitschritte(bd_ctx* c, long long nsteps, double* t_out) {
  if (!c || nsteps < 0) return BD_ERR_ARG;
  bd::RunDyn y0;
  RK(c->e.get_dyn(0, &y0));
  RK(c->e.step(nsteps));
  RK(c->e.sync_check());
  bd::RunDyn y;
  RK(c->e.get_dyn(0, &y));
  c->t_obs += (long double)(y.t - y0.t);
  if (t_out) *t_out = y.t;
  return BD_OK;
}

int bd_zeitschritte_bis_obs(bd_ctx* c, long long* nsteps_out) {
  if (!c) return BD_ERR_ARG;
  RunHost& r = *c->e.runs[0];
  const long double obs_dt = r.p.obs_dt;
  long long n = 0;
  if (!r.adaptive) {
    long double t = c->t_obs;
    while (t < obs_dt) {
      t += (long double)r.p.dt_max;
      n++;
    }
    RK(c->e.step(n));
    RK(c->e.sync_check());
    c->t_obs = t;
  } else {
    while (c->t_obs < obs_dt) {
      double dt;
      RK(bd_zeitschritt(c, 1.0, &dt));
      n++;
    }
  }
  if (nsteps_out) *nsteps_out = n;
  return BD_OK;
}

int bd_get_forces(bd_ctx* c, int kind, int species, double* out) {
  if (!c || !out) return BD_ERR_ARG;
  return c->e.get_forces(kind, species, out);
}

int bd_get_grid(bd_ctx* c, int which, double* out) {
  if (!c || !out) return BD_ERR_ARG;
  return c->e.get_grid(which, out);
}

int bd_get_list(bd_ctx* c, int species, int i, int j, int32_t* out, int cap, int* n) {
  if (!c || species < 0 || species > 1) return BD_ERR_ARG;
  RunHost& r = *c->e.runs[0];
  const int C = r.C;
  if (i < 0 || i >= C || j < 0 || j >= C) return BD_ERR_ARG;
  const int cnt = species == 0 ? r.p.N1 : r.p.N2;
  std::vector<int32_t> g(2 * (size_t)cnt + 2);
  RK(c->e.get_positions(0, species, g.data(), nullptr));
  std::vector<int32_t> ids;
  for (int t = 0; t < cnt; t++) {
    const int di = ((g[2 * t] - i) % C + C) % C, dj = ((g[2 * t + 1] - j) % C + C) % C;
    if ((di <= 1 || di == C - 1) && (dj <= 1 || dj == C - 1)) ids.push_back(t);
  }
  if (n) *n = (int)ids.size();
  if (out)
    for (int k = 0; k < std::min(cap, (int)ids.size()); k++) out[k] = ids[k];
  return BD_OK;
}

// ---- resumable snapshot ----------------------------------------------------
// Binary, little-endian, for the same library build:
//   "BDSNAP01", uint32 version (1), uint32 sizeof(bd_params), bd_params,
//   uint64 seed, uint64 step, double t, float dt, double t_obs, int64 obs_nr,
//   int32 N1, int32 N2, then per particle (species 1, then 2, by index)
//   int32 git[2] and float32 rel[2] -- the device representation exactly.
namespace {
constexpr char kSnapMagic[8] = {'B', 'D', 'S', 'N', 'A', 'P', '0', '1'};

bool same_physics(const bd_params& a, const bd_params& b) {
  return a.N1 == b.N1 && a.N2 == b.N2 && a.L == b.L && a.densGrid_Schema == b.densGrid_Schema &&
         a.FFT_samples == b.FFT_samples && a.lambda_kapillar == b.lambda_kapillar &&
         a.kapillar_vorfaktor == b.kapillar_vorfaktor && a.T == b.T && a.dt_max == b.dt_max &&
         a.max_reisedistanz == b.max_reisedistanz && a.sigma11_22 == b.sigma11_22 &&
         a.sigma11_12 == b.sigma11_12 && a.eps22_11 == b.eps22_11 && a.eps12_11 == b.eps12_11 &&
         a.f2_f1 == b.f2_f1 && a.idgas_only == b.idgas_only && a.noWCA == b.noWCA &&
         a.restrictRadial == b.restrictRadial && a.maxPairWCA == b.maxPairWCA &&
         a.noise_kind == b.noise_kind && a.ngp_ref_compat == b.ngp_ref_compat;
}
}  // namespace

int bd_snapshot_save(bd_ctx* c, const char* path) {
  if (!c || !path) return BD_ERR_ARG;
  RunHost& r = *c->e.runs[0];
  if (!r.has_pos) return BD_ERR_STATE;
  bd::RunDyn y;
  RK(c->e.get_dyn(0, &y));
  const int N1 = r.p.N1, N2 = r.p.N2;
  std::vector<int32_t> g1(2 * (size_t)N1 + 2), g2(2 * (size_t)N2 + 2);
  std::vector<double> q1(2 * (size_t)N1 + 2), q2(2 * (size_t)N2 + 2);
  int32_t* gp[2] = {g1.data(), g2.data()};
  double* qp[2] = {q1.data(), q2.data()};
  RK(c->e.get_positions_both(0, gp, qp));
  FILE* f = std::fopen(path, "wb");
  if (!f) return BD_ERR_IO;
  bool ok = std::fwrite(kSnapMagic, 1, 8, f) == 8;
  const uint32_t ver = 1, psz = sizeof(bd_params);
  const uint64_t seed = r.seed, step = y.step;
  const double t = y.t, t_obs = (double)c->t_obs;
  const float dt = y.dt;
  const int64_t obs_nr = c->obs_nr;
  ok = ok && std::fwrite(&ver, 4, 1, f) == 1 && std::fwrite(&psz, 4, 1, f) == 1;
  ok = ok && std::fwrite(&r.p, sizeof(bd_params), 1, f) == 1;
  ok = ok && std::fwrite(&seed, 8, 1, f) == 1 && std::fwrite(&step, 8, 1, f) == 1;
  ok = ok && std::fwrite(&t, 8, 1, f) == 1 && std::fwrite(&dt, 4, 1, f) == 1;
  ok = ok && std::fwrite(&t_obs, 8, 1, f) == 1 && std::fwrite(&obs_nr, 8, 1, f) == 1;
  ok = ok && std::fwrite(&N1, 4, 1, f) == 1 && std::fwrite(&N2, 4, 1, f) == 1;
  const int32_t* gs[2] = {g1.data(), g2.data()};
  const double* qs[2] = {q1.data(), q2.data()};
  for (int s = 0; s < 2 && ok; s++) {
    const int n = s == 0 ? N1 : N2;
    for (int i = 0; i < n && ok; i++) {
      const float rel[2] = {(float)qs[s][2 * i], (float)qs[s][2 * i + 1]};
      ok = std::fwrite(&gs[s][2 * i], 4, 2, f) == 2 && std::fwrite(rel, 4, 2, f) == 2;
    }
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? BD_OK : BD_ERR_IO;
}

int bd_snapshot_load(bd_ctx* c, const char* path) {
  if (!c || !path) return BD_ERR_ARG;
  RunHost& r = *c->e.runs[0];
  FILE* f = std::fopen(path, "rb");
  if (!f) return BD_ERR_IO;
  struct Closer {
    FILE* f;
    ~Closer() { std::fclose(f); }
  } closer{f};
  char magic[8];
  uint32_t ver = 0, psz = 0;
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kSnapMagic, 8) != 0) return BD_ERR_IO;
  if (std::fread(&ver, 4, 1, f) != 1 || ver != 1) return BD_ERR_IO;
  if (std::fread(&psz, 4, 1, f) != 1 || psz != sizeof(bd_params)) return BD_ERR_IO;
  bd_params p;
  uint64_t seed = 0, step = 0;
  double t = 0.0, t_obs = 0.0;
  float dt = 0.f;
  int64_t obs_nr = 0;
  int32_t N1 = 0, N2 = 0;
  if (std::fread(&p, sizeof(p), 1, f) != 1 || std::fread(&seed, 8, 1, f) != 1 ||
      std::fread(&step, 8, 1, f) != 1 || std::fread(&t, 8, 1, f) != 1 || std::fread(&dt, 4, 1, f) != 1 ||
      std::fread(&t_obs, 8, 1, f) != 1 || std::fread(&obs_nr, 8, 1, f) != 1 ||
      std::fread(&N1, 4, 1, f) != 1 || std::fread(&N2, 4, 1, f) != 1)
    return BD_ERR_IO;
  // the run must be the one that was saved: same physics and noise key
  if (!same_physics(p, r.p) || seed != r.seed || N1 != r.p.N1 || N2 != r.p.N2) return BD_ERR_ARG;
  std::vector<int32_t> g[2];
  std::vector<double> q[2];
  for (int s = 0; s < 2; s++) {
    const int n = s == 0 ? N1 : N2;
    g[s].resize(2 * (size_t)n + 2);
    q[s].resize(2 * (size_t)n + 2);
    for (int i = 0; i < n; i++) {
      float rel[2];
      if (std::fread(&g[s][2 * i], 4, 2, f) != 2 || std::fread(rel, 4, 2, f) != 2) return BD_ERR_IO;
      q[s][2 * i] = rel[0];
      q[s][2 * i + 1] = rel[1];
    }
  }
  int32_t* gp[2] = {g[0].data(), g[1].data()};
  double* qp[2] = {q[0].data(), q[1].data()};
  RK(c->e.set_all_positions(0, gp, qp));
  RK(c->e.set_dyn_field_step(0, step));
  RK(c->e.set_dyn_time(0, t, dt));
  c->t_obs = t_obs;
  c->obs_nr = obs_nr;
  return BD_OK;
}

int bd_get_step(bd_ctx* c, uint64_t* step) {
  if (!c || !step) return BD_ERR_ARG;
  bd::RunDyn y;
  RK(c->e.get_dyn(0, &y));
  *step = y.step;
  return BD_OK;
}

int bd_set_step(bd_ctx* c, uint64_t step) {
  if (!c) return BD_ERR_ARG;
  return c->e.set_dyn_field_step(0, step);
}

int bd_get_time(bd_ctx* c, double* t) {
  if (!c || !t) return BD_ERR_ARG;
  bd::RunDyn y;
  RK(c->e.get_dyn(0, &y));
  *t = y.t;
  return BD_OK;
}

int bd_sync(bd_ctx* c) { return c ? c->e.sync_check() : BD_ERR_ARG; }

int bd_obs_init(bd_ctx* c, int run, const char* dir) {
  if (!c) return BD_ERR_ARG;
  std::string d = dir && *dir ? std::string(dir) + "/" : std::string();
  c->pos1 = d + "pos1_" + std::to_string(run + 1) + ".txt";
  c->pos2 = d + "pos2_" + std::to_string(run + 1) + ".txt";
  RunHost& r = *c->e.runs[0];
  RK(bd::write_pos_frame(c->pos1.c_str(), 0, 0.0, 0, nullptr, nullptr, r.B));
  if (r.p.N2 != 0) RK(bd::write_pos_frame(c->pos2.c_str(), 0, 0.0, 0, nullptr, nullptr, r.B));
  c->obs_open = true;
  c->obs_nr = 0;
  return BD_OK;
}

int bd_schreibe_pos(bd_ctx* c, int nr) {
  if (!c) return BD_ERR_ARG;
  if (!c->obs_open) return BD_ERR_STATE;
  RunHost& r = *c->e.runs[0];
  const int Ns[2] = {r.p.N1, r.p.N2};
  const std::string* paths[2] = {&c->pos1, &c->pos2};
  for (int s = 0; s < 2; s++) {
    if (s == 1 && r.p.N2 == 0) break;
    std::vector<int32_t> g(2 * (size_t)Ns[s] + 2);
    std::vector<double> q(2 * (size_t)Ns[s] + 2);
    RK(c->e.get_positions(0, s, g.data(), q.data()));
    RK(bd::write_pos_frame(paths[s]->c_str(), 1, nr * r.p.obs_dt, Ns[s], g.data(), q.data(), r.B));
  }
  // RunZustand::obs_point (auswertung.cpp:78-93): time since obs restarts
  c->t_obs = 0.0L;
  c->obs_nr++;
  return BD_OK;
}

// ---- batch ------------------------------------------------------------------
int bd_batch_create(const bd_params* runs, const uint64_t* seeds, int nruns, int device,
                    bd_batch** out) {
  if (!runs || !seeds || nruns <= 0 || !out) return BD_ERR_ARG;
  *out = nullptr;
  for (int k = 0; k < nruns; k++) RK(bd::params_validate(&runs[k]));
  bd_batch* b = new (std::nothrow) bd_batch();
  if (!b) return BD_ERR_NOMEM;
  int st = b->e.init(device);
  for (int k = 0; k < nruns && st == BD_OK; k++) st = b->e.add_run(runs[k], seeds[k]);
  if (st == BD_OK) st = b->e.build_plan();
  for (int k = 0; k < nruns && st == BD_OK; k++) {
    const int m = runs[k].startpos_methode;
    if (m != 2) {
      int s2 = init_run_positions(b->e, k, m);
      if (s2 != BD_OK && s2 != BD_ERR_ARG) st = s2;
    }
  }
  if (st != BD_OK) {
    delete b;
    return st;
  }
  *out = b;
  return BD_OK;
}

int bd_batch_destroy(bd_batch* b) {
  delete b;
  return BD_OK;
}

int bd_batch_step(bd_batch* b, long long nsteps) { return b ? b->e.step(nsteps) : BD_ERR_ARG; }
int bd_batch_sync(bd_batch* b) { return b ? b->e.sync_check() : BD_ERR_ARG; }

int bd_batch_nruns(bd_batch* b, int* n) {
  if (!b || !n) return BD_ERR_ARG;
  *n = (int)b->e.runs.size();
  return BD_OK;
}

int bd_batch_get_positions(bd_batch* b, int run, int species, int32_t* git, double* rel) {
  if (!b || run < 0) return BD_ERR_ARG;
  return b->e.get_positions((size_t)run, species, git, rel);
}

int bd_batch_set_positions(bd_batch* b, int run, int species, const int32_t* git,
                           const double* rel) {
  if (!b || run < 0 || !git || !rel) return BD_ERR_ARG;
  return b->e.set_positions((size_t)run, species, git, rel);
}

int bd_batch_set_positions_all(bd_batch* b, int run, const int32_t* git1, const double* rel1,
                               const int32_t* git2, const double* rel2) {
  if (!b || run < 0 || (size_t)run >= b->e.runs.size() || !git1 || !rel1) return BD_ERR_ARG;
  const bd::RunHost& r = *b->e.runs[run];
  if (r.p.N2 > 0 && (!git2 || !rel2)) return BD_ERR_ARG;
  int32_t dg[2] = {0, 0};
  double dq[2] = {0, 0};
  int32_t* g[2] = {const_cast<int32_t*>(git1), git2 ? const_cast<int32_t*>(git2) : dg};
  double* q[2] = {const_cast<double*>(rel1), rel2 ? const_cast<double*>(rel2) : dq};
  return b->e.set_all_positions((size_t)run, g, q);
}

int bd_batch_get_positions_all(bd_batch* b, int run, int32_t* git1, double* rel1, int32_t* git2,
                               double* rel2) {
  if (!b || run < 0 || (size_t)run >= b->e.runs.size()) return BD_ERR_ARG;
  int32_t* g[2] = {git1, git2};
  double* q[2] = {rel1, rel2};
  return b->e.get_positions_both((size_t)run, g, q);
}

int bd_get_stream(bd_ctx* c, void** stream) {
  if (!c || !stream) return BD_ERR_ARG;
  *stream = (void*)c->e.stream;
  return BD_OK;
}

int bd_batch_get_stream(bd_batch* b, void** stream) {
  if (!b || !stream) return BD_ERR_ARG;
  *stream = (void*)b->e.stream;
  return BD_OK;
}

int bd_launches_per_step(bd_ctx* c, int* n) {
  if (!c || !n) return BD_ERR_ARG;
  *n = c->e.launches_per_step();
  return BD_OK;
}

int bd_batch_launches_per_step(bd_batch* b, int* n) {
  if (!b || !n) return BD_ERR_ARG;
  *n = b->e.launches_per_step();
  return BD_OK;
}

int bd_stage_times(bd_ctx* c, int nsteps, double* ms, int nstages) {
  if (!c || !ms) return BD_ERR_ARG;
  return c->e.stage_times(nsteps, ms, nstages);
}

int bd_zeitschritt_info(bd_ctx* c, bd_timestep_info* info) {
  if (!c || !info) return BD_ERR_ARG;
  return c->e.timestep_info(info);
}

int bd_zeitschritt_debug(bd_ctx* c, double mrd, bd_timestep_info* info, double* dt_out) {
  if (!c || !info) return BD_ERR_ARG;
  double dt = 0.0;
  RK(c->e.zeitschritt_debug(mrd, info, &dt));
  c->t_obs += (long double)dt;
  if (dt_out) *dt_out = dt;
  return BD_OK;
}

int bd_korrelationsfunktion(bd_ctx* c, int which, double korr_dr, int korr_bins, double* g) {
  return c ? c->e.korrelation(which, korr_dr, korr_bins, g) : BD_ERR_ARG;
}

int bd_ftrho(bd_ctx* c, int species, int qbins, double dq, double* re, double* im) {
  return c ? c->e.ftrho(species, qbins, dq, re, im) : BD_ERR_ARG;
}

void bd_lokdens_params_default(bd_lokdens_params* lp) {
  if (lp) bd::lokdens_params_default(lp);
}

int bd_lokdens_params_from_header(const char* path, bd_lokdens_params* lp) {
  if (!path || !lp) return BD_ERR_ARG;
  return bd::lokdens_params_from_header(path, lp);
}

int bd_snapgrid_num(const bd_params* p, const bd_lokdens_params* lp, int* n) {
  if (!p || !lp || !n) return BD_ERR_ARG;
  *n = bd::snapgrid_num(p->L, lp->snapgrid_crude);
  return *n > 0 ? BD_OK : BD_ERR_ARG;
}

int bd_lokale_dichte(bd_ctx* c, const bd_lokdens_params* lp, double* rho1, double* rho2, int32_t* hist,
                     int32_t* over) {
  if (!c || !lp) return BD_ERR_ARG;
  return c->e.lokale_dichte(*lp, rho1, rho2, hist, over);
}

int bd_schreibe_lokale_dichte(bd_ctx* c, const bd_lokdens_params* lp, const char* dir, int nr) {
  if (!c || !lp || !dir || nr < 0) return BD_ERR_ARG;
  const bd_params& p = c->e.runs[0]->p;
  const int n = bd::snapgrid_num(p.L, lp->snapgrid_crude);
  if (n <= 0 || n > BD_SNAPGRID_MAX) return n <= 0 ? BD_ERR_ARG : BD_ERR_UNSUPPORTED;
  if (lp->rhohist_bins <= 0 || lp->rhohist_bins > BD_RHOHIST_MAX_BINS) return BD_ERR_ARG;
  const size_t cells = (size_t)n * n;
  std::vector<double> g1(cells), g2(cells);
  std::vector<int32_t> hist(4 * (size_t)lp->rhohist_bins), over(7);
  RK(c->e.lokale_dichte(*lp, g1.data(), g2.data(), hist.data(), over.data()));
  return bd::write_lokdens_frame(dir, lp, n, p.L / n, nr, p.obs_dt, g1.data(), g2.data(), hist.data(),
                                 over.data());
}

int bd_fused_phase_times(bd_ctx* c, int nsteps, double* ms, int nphases) {
  if (!c || !ms) return BD_ERR_ARG;
  return c->e.fused_phase_times(nsteps, ms, nphases);
}

int bd_batch_phase_times(bd_batch* b, int nsteps, double* ms, int nphases) {
  if (!b || !ms) return BD_ERR_ARG;
  return b->e.fused_phase_times(nsteps, ms, nphases);
}

int bd_inject_barrier_timeout(bd_ctx* c, int barrier, unsigned max_polls) {
  if (!c) return BD_ERR_ARG;
  return c->e.inject_barrier_timeout(barrier, max_polls);
}

int bd_batch_stage_times(bd_batch* b, int nsteps, double* ms, int nstages) {
  if (!b || !ms) return BD_ERR_ARG;
  return b->e.stage_times(nsteps, ms, nstages);
}

int bd_batch_autotune(bd_batch* b, int reps, bd_tune_result* out) {
  if (!b || !out || reps <= 0) return BD_ERR_ARG;
  return b->e.autotune(reps, out);
}

int bd_batch_set_step_form(bd_batch* b, int form, int ctas_per_sm) {
  if (!b || form < 0 || form > 1 || ctas_per_sm < 0) return BD_ERR_ARG;
  if (form == 1 && (ctas_per_sm == 1 || ctas_per_sm > 4)) return BD_ERR_ARG;
  if (form == 0 && ctas_per_sm != 0) return BD_ERR_ARG;
  return b->e.set_step_form(form, ctas_per_sm);
}

int bd_batch_get_time(bd_batch* b, int run, double* t) {
  if (!b || !t || run < 0) return BD_ERR_ARG;
  bd::RunDyn y;
  RK(b->e.get_dyn((size_t)run, &y));
  *t = y.t;
  return BD_OK;
}

}  // extern "C"

// Host-side pieces of the C ABI that need no GPU: parameters (defaults,
// parameter.h parser, derived constants), the reference's position
// initialisers and the pos-file formatter.
#include <cctype>
#include <climits>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <random>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "bd_api.h"
#include "bd_host.h"

namespace bd {

// parameter.h:14-139 as shipped
void params_default(bd_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->N1 = 2000;
  p->N2 = 2000;
  p->L = 300.0;
  p->densGrid_Schema = 2;
  p->FFT_samples = 384;
  p->lambda_kapillar = 25.0;
  p->kapillar_vorfaktor = 1.111111111;
  p->T = 24.3055555;
  p->dt_max = 0.005;
  p->max_reisedistanz = 0.24;
  p->sigma11_22 = 1.0;
  p->sigma11_12 = 0.5 * (1.0 + p->sigma11_22);
  p->Gamma2_1 = p->sigma11_22;
  p->eps22_11 = 1.0;
  p->eps12_11 = 1.0;
  p->f2_f1 = -1.0;
  p->idgas_only = 0;
  p->noWCA = 0;
  p->noRNG = 0;
  p->quickInit = 1;
  p->restrictRadial = 0;
  p->debugmode = 0;
  p->krafttestmode = 0;
  p->maxPairWCA = 1.0e5;
  p->max_write_interval = 900;
  p->runs = 1;
  p->jobs = 1;
  p->maxThreads = 1;
  p->obs_dt = 0.2;
  p->obs_anzahl = 12;
  p->startpos_methode = 1;
  p->startpos_kreisradius = 4.5 * p->lambda_kapillar;
  p->noise_kind = BD_NOISE_DISK;
  p->ngp_ref_compat = 1;
}

// parameter.h:171-209
void params_derived(const bd_params* p, bd_derived* d) {
  d->zweihoch1_6 = std::pow(2.0, 1.0 / 6.0);
  d->nachList_Zellen = (int)std::floor(p->L / d->zweihoch1_6);
  d->nachList_Breite = p->L / ((double)d->nachList_Zellen);
  d->densGrid_Breite = p->L / p->FFT_samples;
  d->densGrid_Zellen = p->FFT_samples;
  d->dq = 2.0 * M_PI / p->L;
  d->fixed_dt = p->max_reisedistanz >= 1e20 ? 1 : 0;
}

static bool pow23(int n) {
  if (n <= 0) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

int params_validate(const bd_params* p) {
  if (p->N1 < 1 || p->N2 < 0) return BD_ERR_ARG;  // parameter.h:13: N1 must not be zero
  if ((long long)p->N1 + p->N2 >= (1LL << 30)) return BD_ERR_UNSUPPORTED;
  if (!(p->L > 0.0) || !std::isfinite(p->L)) return BD_ERR_ARG;
  if (p->densGrid_Schema < 0 || p->densGrid_Schema > 2) return BD_ERR_ARG;
  if (p->FFT_samples < 8 || p->FFT_samples > 4096 || p->FFT_samples % 2) return BD_ERR_UNSUPPORTED;
  if (!pow23(p->FFT_samples)) return BD_ERR_UNSUPPORTED;
  bd_derived d;
  params_derived(p, &d);
  // fewer than 3 cells per side makes the 3x3 neighbour cells coincide
  if (d.nachList_Zellen < 3) return BD_ERR_UNSUPPORTED;
  // cell and mesh indices stay below 2^24 (exact FP32 index arithmetic on the device)
  if (d.nachList_Zellen > 4095) return BD_ERR_UNSUPPORTED;
  if (!(p->dt_max > 0.0) || !(p->T >= 0.0)) return BD_ERR_ARG;
  if (p->noise_kind < 0 || p->noise_kind > 2) return BD_ERR_ARG;
  return BD_OK;
}

// ---------------------------------------------------------------------------
// parameter.h reader: `const <type> <name> = <expr>;` with + - * / (), number
// literals, previously defined names, M_PI, pow(), floor(), sqrt(), ceil(),
// C casts (int)/(double) and true/false. string constants are skipped.
namespace {
struct Parser {
  const char* s;
  std::map<std::string, double>& vars;
  bool ok = true;
  void ws() {
    while (*s && std::isspace((unsigned char)*s)) s++;
  }
  bool eat(char c) {
    ws();
    if (*s == c) {
      s++;
      return true;
    }
    return false;
  }
  std::string ident() {
    ws();
    std::string r;
    while (*s && (std::isalnum((unsigned char)*s) || *s == '_')) r += *s++;
    return r;
  }
  double primary() {
    ws();
    if (*s == '(') {
      // cast or parenthesised expression
      const char* save = s;
      s++;
      std::string id = ident();
      ws();
      if ((id == "int" || id == "double" || id == "float" || id == "long") && *s == ')') {
        s++;
        double v = unary();
        return id == "int" || id == "long" ? (double)(long long)v : v;
      }
      s = save + 1;
      double v = expr();
      if (!eat(')')) ok = false;
      return v;
    }
    if (std::isdigit((unsigned char)*s) || *s == '.') {
      char* e;
      double v = std::strtod(s, &e);
      s = e;
      while (*s == 'f' || *s == 'F' || *s == 'L' || *s == 'l' || *s == 'u' || *s == 'U') s++;
      return v;
    }
    std::string id = ident();
    if (id.empty()) {
      ok = false;
      return 0;
    }
    if (id == "true") return 1;
    if (id == "false") return 0;
    if (id == "M_PI") return M_PI;
    if (id == "pow" || id == "floor" || id == "sqrt" || id == "ceil" || id == "fabs") {
      if (!eat('(')) {
        ok = false;
        return 0;
      }
      double a = expr(), b = 0;
      if (id == "pow") {
        if (!eat(',')) ok = false;
        b = expr();
      }
      if (!eat(')')) ok = false;
      if (id == "pow") return std::pow(a, b);
      if (id == "floor") return std::floor(a);
      if (id == "ceil") return std::ceil(a);
      if (id == "fabs") return std::fabs(a);
      return std::sqrt(a);
    }
    auto it = vars.find(id);
    if (it == vars.end()) {
      ok = false;
      return 0;
    }
    return it->second;
  }
  double unary() {
    if (eat('-')) return -unary();
    if (eat('+')) return unary();
    return primary();
  }
  double term() {
    double v = unary();
    for (;;) {
      if (eat('*')) v *= unary();
      else if (eat('/')) v /= unary();
      else return v;
    }
  }
  double expr() {
    double v = term();
    for (;;) {
      if (eat('+')) v += term();
      else if (eat('-')) v -= term();
      else return v;
    }
  }
};

// drops // and /* */ comments and preprocessor lines
std::string strip_comments(const std::string& in) {
  std::string out;
  bool line_start = true;
  for (size_t i = 0; i < in.size(); i++) {
    if (line_start && in[i] == '#') {
      while (i < in.size() && in[i] != '\n') i++;
      out += '\n';
      continue;
    }
    if (in[i] != ' ' && in[i] != '\t') line_start = in[i] == '\n';
    if (in[i] == '/' && i + 1 < in.size() && in[i + 1] == '/') {
      while (i < in.size() && in[i] != '\n') i++;
      out += '\n';
      line_start = true;
    } else if (in[i] == '/' && i + 1 < in.size() && in[i + 1] == '*') {
      i += 2;
      while (i + 1 < in.size() && !(in[i] == '*' && in[i + 1] == '/')) i++;
      i++;
    } else {
      out += in[i];
    }
  }
  return out;
}
}  // namespace

// every `const <type> name = expr;` of a parameter.h, evaluated in order
static int header_vars(const char* path, std::map<std::string, double>& vars) {
  FILE* f = std::fopen(path, "r");
  if (!f) return BD_ERR_IO;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  std::fclose(f);
  text = strip_comments(text);
  // statements separated by ';' 
  size_t pos = 0;
  while (pos < text.size()) {
    size_t end = text.find(';', pos);
    if (end == std::string::npos) break;
    std::string st = text.substr(pos, end - pos);
    pos = end + 1;
    const char* c = st.c_str();
    while (*c && std::isspace((unsigned char)*c)) c++;
    if (std::strncmp(c, "const", 5) != 0) continue;
    c += 5;
    // type
    while (*c && std::isspace((unsigned char)*c)) c++;
    std::string type;
    while (*c && (std::isalnum((unsigned char)*c) || *c == '_' || *c == ':')) type += *c++;
    if (type == "string" || type == "std::string" || type == "char") continue;
    // one or more "name = expr" separated by commas at top level
    std::string rest(c);
    int depth = 0;
    std::vector<std::string> decls;
    std::string cur;
    for (char ch : rest) {
      if (ch == '(') depth++;
      if (ch == ')') depth--;
      if (ch == ',' && depth == 0) {
        decls.push_back(cur);
        cur.clear();
      } else {
        cur += ch;
      }
    }
    decls.push_back(cur);
    for (auto& dcl : decls) {
      size_t eq = dcl.find('=');
      if (eq == std::string::npos) continue;
      std::string name = dcl.substr(0, eq);
      name.erase(0, name.find_first_not_of(" \t\r\n"));
      name.erase(name.find_last_not_of(" \t\r\n") + 1);
      Parser ps{dcl.c_str() + eq + 1, vars};
      double v = ps.expr();
      if (!ps.ok) return BD_ERR_IO;
      if (type == "int") v = (double)(long long)v;
      vars[name] = v;
    }
  }
  return BD_OK;
}

int params_from_header(const char* path, bd_params* p) {
  std::map<std::string, double> vars;
  const int st = header_vars(path, vars);
  if (st) return st;
#define GETI(nm) \
  if (vars.count(#nm)) p->nm = (int)vars[#nm];
#define GETD(nm) \
  if (vars.count(#nm)) p->nm = vars[#nm];
  GETI(N1) GETI(N2) GETD(L) GETI(densGrid_Schema) GETI(FFT_samples) GETD(lambda_kapillar)
  GETD(kapillar_vorfaktor) GETD(T) GETD(dt_max) GETD(max_reisedistanz) GETD(sigma11_22)
  GETD(sigma11_12) GETD(Gamma2_1) GETD(eps22_11) GETD(eps12_11) GETD(f2_f1) GETI(idgas_only)
  GETI(noWCA) GETI(noRNG) GETI(quickInit) GETI(restrictRadial) GETI(debugmode)
  GETI(krafttestmode) GETD(maxPairWCA) GETI(max_write_interval) GETI(runs) GETI(jobs)
  GETI(maxThreads) GETD(obs_dt) GETI(obs_anzahl) GETI(startpos_methode)
  GETD(startpos_kreisradius)
#undef GETI
#undef GETD
  return BD_OK;
}

// parameter.h:109-124,161 as shipped
void lokdens_params_default(bd_lokdens_params* lp) {
  lp->snapgrid_crude = 0.5;
  lp->rhohist_bins = 100;
  lp->rhohist_drho = 0.01;
  lp->rho_thresh[0] = 0.1, lp->rho_thresh[1] = 0.2, lp->rho_thresh[2] = 0.5;
  lp->drho_thresh[0] = 0.1, lp->drho_thresh[1] = 0.2, lp->drho_thresh[2] = 0.5, lp->drho_thresh[3] = 0.99;
}

int lokdens_params_from_header(const char* path, bd_lokdens_params* lp) {
  std::map<std::string, double> vars;
  const int st = header_vars(path, vars);
  if (st) return st;
  auto get = [&](const char* nm, double& out) {
    if (vars.count(nm)) out = vars[nm];
  };
  get("snapgrid_crude", lp->snapgrid_crude);
  get("rhohist_drho", lp->rhohist_drho);
  if (vars.count("rhohist_bins")) lp->rhohist_bins = (int)vars["rhohist_bins"];
  const char* rt[3] = {"rho_thresh1", "rho_thresh2", "rho_thresh3"};
  const char* dt[4] = {"drho_thresh1", "drho_thresh2", "drho_thresh3", "drho_thresh4"};
  for (int t = 0; t < 3; t++) get(rt[t], lp->rho_thresh[t]);
  for (int t = 0; t < 4; t++) get(dt[t], lp->drho_thresh[t]);
  return BD_OK;
}

// parameter.h:174
int snapgrid_num(double L, double snapgrid_crude) {
  if (!(snapgrid_crude > 0.0) || !(L > 0.0)) return 0;
  const double v = L / (2 * snapgrid_crude) + 0.5;
  return v < (double)INT_MAX / 2 ? 2 * (int)v : 0;
}

// ---------------------------------------------------------------------------
// Initialisers (dynamik_methoden.cpp:1647-1851). The generator is the
// reference's: std::mt19937_64 with uniform_real_distribution<double>(0,1)
// and zufall_gleichverteilt_vonbis(a, b) = a + (b-a) u (zufall.cpp:18-39).
struct Uniform {
  std::mt19937_64& g;
  std::uniform_real_distribution<double> dist{0.0, 1.0};
  double vonbis(double a, double b) { return a + (b - a) * dist(g); }
};

int init_positions_host(const bd_params* p, std::mt19937_64& gen, int methode, int32_t* git[2],
                        double* rel[2]) {
  bd_derived d;
  params_derived(p, &d);
  const double B = d.nachList_Breite, L = p->L;
  const int Ns[2] = {p->N1, p->N2};
  Uniform U{gen};
  auto set = [&](int s, int i, int jc, int kc, double rx, double ry) {
    git[s][2 * i] = jc;
    git[s][2 * i + 1] = kc;
    rel[s][2 * i] = rx;
    rel[s][2 * i + 1] = ry;
  };
  switch (methode) {
    case 1:  // init_zufallspos, including the (int) x / B precedence
      for (int s = 0; s < 2; s++)
        for (int i = 0; i < Ns[s]; i++) {
          double x = U.vonbis(0.0, L);
          double y = U.vonbis(0.0, L);
          int jc = (int)((double)((int)x) / B);
          int kc = (int)((double)((int)y) / B);
          set(s, i, jc, kc, x - jc * B, y - kc * B);
        }
      return BD_OK;
    case 3: {  // init_gitterstart
      if (p->N2 != 0) return BD_ERR_ARG;
      double wurzelN = std::ceil(std::sqrt((double)p->N1));
      double schritt = L / wurzelN;
      int index = 0;
      for (int i = 0; i < wurzelN && index < p->N1; i++)
        for (int j = 0; j < wurzelN; j++) {
          double x = i * schritt, y = j * schritt;
          int ic = (int)(x / B), jc = (int)(y / B);
          set(0, index, ic, jc, x - ic * B, y - jc * B);
          if (++index == p->N1) break;
        }
      return BD_OK;
    }
    case 4:  // init_allegleich
      for (int s = 0; s < 2; s++) {
        double x = U.vonbis(0.0, L);
        double y = U.vonbis(0.0, L);
        int jc = (int)(x / B), kc = (int)(y / B);
        for (int i = 0; i < Ns[s]; i++) set(s, i, jc, kc, x - jc * B, y - kc * B);
      }
      return BD_OK;
    case 5: {  // init_kreisscheibe
      const double rad = p->startpos_kreisradius, rad2 = rad * rad;
      for (int s = 0; s < 2; s++)
        for (int i = 0; i < Ns[s]; i++) {
          double x, y;
          do {
            x = U.vonbis(-rad, rad);
            y = U.vonbis(-rad, rad);
          } while (x * x + y * y > rad2);
          x += 0.5 * L;
          y += 0.5 * L;
          int jc = (int)(x / B), kc = (int)(y / B);
          set(s, i, jc, kc, x - jc * B + 0.03, y - kc * B + 0.03);
        }
      return BD_OK;
    }
    case 6: {  // init_kernundring
      if (p->N1 != 1 || p->N2 < 3) return BD_ERR_ARG;
      const double mitte = 0.5 * L;
      {
        int ic = (int)(mitte / B), jc = (int)(mitte / B);
        set(0, 0, ic, jc, mitte - ic * B, mitte - jc * B);
      }
      for (int t = 0; t < p->N2; t++) {
        double x = mitte + p->startpos_kreisradius * std::cos(2 * M_PI * (double)t / p->N2);
        double y = mitte + p->startpos_kreisradius * std::sin(2 * M_PI * (double)t / p->N2);
        int ic = (int)(x / B), jc = (int)(y / B);
        set(1, t, ic, jc, x - ic * B, y - jc * B);
      }
      return BD_OK;
    }
    case 7: {  // init_posKrafttest
      if (p->N2 != 0 || p->N1 != 2) return BD_ERR_ARG;
      const double dx = d.densGrid_Breite;
      double x = 0.5 * dx, y = 0.5 * dx;
      int g0 = (int)(x / B), g1 = (int)(y / B);
      set(0, 0, g0, g1, x - g0 * B, y - g1 * B);
      y = 0.55 * dx;
      int h1 = (int)(y / B);
      set(0, 1, g0, h1, rel[0][0], y - h1 * B);
      return BD_OK;
    }
    default:
      return BD_ERR_ARG;
  }
}

// init_pos_aus_datei (dynamik_methoden.cpp:1578-1643): two header lines,
// then N1 rows "idx TAB 1 TAB x TAB y" and N2 rows with type 2, read with
// %g into float as the reference does. The offset is x - git*B (the
// reference subtracts rel*B, an uninitialised value).
int init_pos_from_file(const bd_params* p, const char* path, int32_t* git[2], double* rel[2]) {
  FILE* in = std::fopen(path, "r");
  if (!in) return BD_ERR_IO;
  char buffer[1000];
  if (!std::fgets(buffer, sizeof(buffer), in) || !std::fgets(buffer, sizeof(buffer), in)) {
    std::fclose(in);
    return BD_ERR_IO;
  }
  bd_derived d;
  params_derived(p, &d);
  const double B = d.nachList_Breite;
  const int Ns[2] = {p->N1, p->N2};
  for (int s = 0; s < 2; s++)
    for (int zeile = 0; zeile < Ns[s]; zeile++) {
      int nr, typ;
      float xf, yf;
      if (std::fscanf(in, "%d \t %d \t %g \t %g", &nr, &typ, &xf, &yf) != 4 || nr != zeile ||
          typ != s + 1) {
        std::fclose(in);
        return BD_ERR_IO;
      }
      double x = xf, y = yf;
      if (x < 0.0 || x > p->L || y < 0.0 || y > p->L) {
        std::fclose(in);
        return BD_ERR_RANGE;
      }
      int gx = (int)(x / B), gy = (int)(y / B);
      if (gx >= d.nachList_Zellen) gx = d.nachList_Zellen - 1;
      if (gy >= d.nachList_Zellen) gy = d.nachList_Zellen - 1;
      git[s][2 * zeile] = gx;
      git[s][2 * zeile + 1] = gy;
      rel[s][2 * zeile] = x - gx * B;
      rel[s][2 * zeile + 1] = y - gy * B;
    }
  std::fclose(in);
  return BD_OK;
}

// RunObs::obs_init header and RunObs::schreibe_pos rows (auswertung.cpp:57-68,
// 631-648): "%g \t %g \t %g \n" of t, x = rel + B*git, y; blank line per frame.
// The analysis program's output (main_auswertung.cpp): the headers written
// when it opens its files (:60-77), the gridded densities
// localDens/rho<nr>.txt (:205-210,290-296), the histogram and threshold
// lines (:357-375). Times print as nr * obs_dt.
int write_lokdens_frame(const char* dir, const bd_lokdens_params* lp, int n, double width, int nr,
                        double obs_dt, const double* g1, const double* g2, const int32_t* hist,
                        const int32_t* over) {
  const std::string base = std::string(dir) + "/";
  if (mkdir((base + "localDens").c_str(), 0777) != 0 && errno != EEXIST) return BD_ERR_IO;
  const double t = nr * obs_dt;
  const int bins = lp->rhohist_bins;
  const double pref = 1. / (n * n);
  FILE* f = std::fopen((base + "localDens/rho" + std::to_string(nr) + ".txt").c_str(), "w");
  if (!f) return BD_ERR_IO;
  std::fprintf(f, "# Format: t x y rho1 rho2 \n");
  std::fprintf(f, "# where x and y are the center of the cell. \n\n");
  for (int k = 0; k < n; k++)
    for (int l = 0; l < n; l++)
      std::fprintf(f, "%g \t %g \t %g \t %g \t %g \n", t, (k + 0.5) * width, (l + 0.5) * width,
                   g1[(size_t)k * n + l], g2[(size_t)k * n + l]);
  std::fprintf(f, "\n");
  std::fclose(f);
  const char* mode = nr == 0 ? "w" : "a";
  FILE* rh = std::fopen((base + "rhoHist.txt").c_str(), mode);
  FILE* dh = std::fopen((base + "drhoHist.txt").c_str(), mode);
  FILE* rt = std::fopen((base + "rhoThresh.txt").c_str(), mode);
  FILE* dt = std::fopen((base + "drhoThresh.txt").c_str(), mode);
  int st = (rh && dh && rt && dt) ? BD_OK : BD_ERR_IO;
  if (st == BD_OK && nr == 0) {
    std::fprintf(rh, "# Format: t TAB dens TAB fraction of space with <rho1 TAB rho2 TAB rho1+rho2> = dens \n\n");
    std::fprintf(dh, "# Format: t TAB rho1-rho2 TAB fraction of space with this rho1-rho2\n\n");
    std::fprintf(rt, "# Format: t TAB #cells over thresh1 TAB #cells over thresh2 TAB #cells over thresh3\n");
    std::fprintf(rt, "# where thresh1=%g, thresh2=%g, thresh3=%g\n\n", lp->rho_thresh[0], lp->rho_thresh[1],
                 lp->rho_thresh[2]);
    std::fprintf(dt,
                 "# Format: t TAB #cells with |rho1-rho2|/(rho1+rho2) over thresh1 TAB same thresh2 TAB same "
                 "thresh3 TAB same thresh4\n");
    std::fprintf(dt, "# where thresh1=%g, thresh2=%g, thresh3=%g, thresh4=%g\n\n", lp->drho_thresh[0],
                 lp->drho_thresh[1], lp->drho_thresh[2], lp->drho_thresh[3]);
  }
  if (st == BD_OK) {
    std::fprintf(rt, "%g \t %g \t %g \t %g \n", t, over[0] * pref, over[1] * pref, over[2] * pref);
    std::fprintf(dt, "%g \t %g \t %g \t %g \t %g \n", t, over[3] * pref, over[4] * pref, over[5] * pref,
                 over[6] * pref);
    for (int b = 0; b < bins; b++) {
      std::fprintf(rh, "%g \t %g \t %g \t %g \t %g \n", t, lp->rhohist_drho * (b + 0.5), pref * hist[b],
                   pref * hist[bins + b], pref * hist[2 * bins + b]);
      std::fprintf(dh, "%g \t %g \t %g \n", t, lp->rhohist_drho * (b + 0.5 - bins / 2), pref * hist[3 * bins + b]);
    }
    std::fprintf(rh, "\n");
    std::fprintf(dh, "\n");
  }
  for (FILE* x : {rh, dh, rt, dt})
    if (x) std::fclose(x);
  return st;
}

int write_pos_frame(const char* path, int append, double t, int n, const int32_t* git,
                    const double* rel, double B) {
  FILE* f = std::fopen(path, append ? "a" : "w");
  if (!f) return BD_ERR_IO;
  if (!append) std::fprintf(f, "# Format: t TAB x TAB y \n\n");
  if (n > 0 && git && rel) {
    for (int i = 0; i < n; i++) {
      double x = rel[2 * i] + B * git[2 * i];
      double y = rel[2 * i + 1] + B * git[2 * i + 1];
      std::fprintf(f, "%g \t %g \t %g \n", t, x, y);
    }
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return BD_OK;
}

}  // namespace bd

// C++ mirror of the reference's run interface (signaturen2.h:29-434) over the
// C ABI of libbd_b200.so: class and routine names, argument meaning and the
// error behaviour (a message on std::cout, then return) are the reference's,
// so code written against RunZustand / RunZustand::RunDynamik compiles
// against this header with the parameters taken from a bd_params struct
// instead of compile-time constants.
#pragma once

#include <cstdint>
#include <cstdio>
#include <ctime>
#include <iostream>
#include <string>
#include <vector>

#include "bd_api.h"

namespace bdb {

class RunZustand {
 public:
  class RunDynamik {
   public:
    bd_ctx* ctx = nullptr;
    int N1 = 0, N2 = 0;

    // TimestepInfo (signaturen2.h:71-145): the record zeitschritt_debug
    // fills, with its console report
    struct TimestepInfo : bd_timestep_info {
      TimestepInfo() { reset(); }
      void reset() {
        bd_timestep_info& b = *this;
        b = bd_timestep_info{};
        maxWCAtype = maxWCAindex = maxWCA_numWW1 = maxWCA_numWW2 = -1;
        maxKaptype = maxKapindex = maxRNDtype = maxRNDindex = -1;
        dt = -1.0;
      }
      void ausgabe() const {
        std::cout << "WCA-Wechselwirkung: " << num_WCA_berechnet << " WW wurden berechnet." << std::endl;
        std::cout << "stärkste WCA-WW: Wirkt auf Teilchen " << maxWCAindex << ", Typ " << maxWCAtype
                  << ". Sie beträgt (" << maxWCAx << "," << maxWCAy << "). In den Nachbarlisten sind "
                  << maxWCA_numWW1 << "+" << maxWCA_numWW2 << " Einträge." << std::endl;
        std::cout << "Es haben " << num_Zellwechsel1 << "+" << num_Zellwechsel2
                  << " Teilchen ihre Zelle verlassen." << std::endl
                  << std::endl;
        std::cout << "Kapillarwechselwirkung: stärkste Kraft wirkt auf Teilchen " << maxKapindex << ", Typ "
                  << maxKaptype << ". Sie beträgt (" << maxKapx << "," << maxKapy << ")." << std::endl
                  << std::endl;
        std::cout << "Zufallskräfte: stärkste Kraft wirkt auf Teilchen " << maxRNDindex << ", Typ " << maxRNDtype
                  << ". Sie beträgt (" << maxRNDx << "," << maxRNDy << "). " << std::endl
                  << std::endl;
        std::cout << "-> Schrittweite: dt=" << dt << std::endl << std::flush;
      }
    };

    // zeitschritt_debug (dynamik_methoden.cpp:168-211): a step bounded by
    // travel distance mrd, recording its TimestepInfo; returns its length
    double zeitschritt_debug(double mrd, TimestepInfo& info, bool silent) {
      info.reset();
      double dt = 1.0e10;
      report(bd_zeitschritt_debug(ctx, mrd, &info, &dt), "zeitschritt_debug");
      if (!silent) info.ausgabe();
      return dt;
    }

    // zeitschritt (dynamik_methoden.cpp:74-163): returns the step length
    double zeitschritt(double tmax) {
      double dt = 1.0e10;
      const int s = bd_zeitschritt(ctx, tmax, &dt);
      if (s == BD_ERR_ARG)
        std::cout << "Fehler: Negative Zeitschrittweite " << tmax << " gefordert, breche ab!"
                  << std::endl;
      else report(s, "zeitschritt");
      return dt;
    }
    void berechne_kapkraefte() { report(bd_berechne_kapkraefte(ctx), "berechne_kapkraefte"); }
    void berechne_WCA11() { report(bd_berechne_WCA11(ctx), "berechne_WCA11"); }
    void berechne_WCA22() { report(bd_berechne_WCA22(ctx), "berechne_WCA22"); }
    void addiere_WCA12() { report(bd_addiere_WCA12(ctx), "addiere_WCA12"); }
    void refresh_erwNachbar() { report(bd_refresh_erwNachbar(ctx), "refresh_erwNachbar"); }
    void berechne_zufallskraefte() {
      report(bd_berechne_zufallskraefte(ctx), "berechne_zufallskraefte");
    }
    double optimaler_zeitschritt() {
      double dt = 0.0;
      report(bd_optimaler_zeitschritt(ctx, &dt), "optimaler_zeitschritt");
      return dt;
    }
    void init() {
      report(bd_WCA_init(ctx), "WCA_init");
      report(bd_kapkraefte_init(ctx), "kapkraefte_init");
    }
    // krafttest getters (signaturen2.h:182-188): y force on particle 1 of species 1
    double getFKap() { return force(BD_FORCE_KAP, 1, 1); }
    double getF() { return force(BD_FORCE_KAP, 1, 1) + force(BD_FORCE_WCA, 1, 1); }

   private:
    double force(int kind, int i, int comp) {
      std::vector<double> f(2 * (size_t)N1);
      report(bd_get_forces(ctx, kind, 0, f.data()), "get_forces");
      return f[2 * (size_t)i + comp];
    }
    static void report(int s, const char* what) {
      if (s != BD_OK) std::cout << "Fehler in " << what << ": " << bd_status_string(s) << std::endl;
    }
  };

  RunDynamik dyn;
  int nr = 0;
  long double t = 0.0L;  // simulated time since the last observation point
  int obs_nr = 0;
  int schritte_seit_obs = 0;
  bd_params p{};

  RunZustand() = default;
  explicit RunZustand(const bd_params& params, int device = 0) : p(params), device_(device) {}
  RunZustand(const RunZustand&) = delete;
  RunZustand& operator=(const RunZustand&) = delete;
  ~RunZustand() {
    if (dyn.ctx) bd_destroy(dyn.ctx);
  }

  // RunZustand::init (allgemeine_methoden.cpp:256-320): positions by
  // startpos_methode, cell order, Green's tables, observation files. The
  // run number seeds the initialisers (the reference seeds with time(NULL)).
  void init(int run, uint64_t seed) {
    nr = run;
    obs_nr = 0;
    t = 0.0L;
    if (dyn.ctx) bd_destroy(dyn.ctx);
    dyn.ctx = nullptr;
    const int s = bd_create(&p, seed, device_, &dyn.ctx);
    if (s != BD_OK) {
      std::cout << "Fehler: bd_create: " << bd_status_string(s) << std::endl;
      return;
    }
    dyn.N1 = p.N1;
    dyn.N2 = p.N2;
    if (p.startpos_methode == 2 && bd_init_pos_aus_datei(dyn.ctx, "startpos.txt") != BD_OK)
      std::cout << "Fehler beim Lesen der Inputdatei startpos.txt" << std::endl;
    bd_obs_init(dyn.ctx, run, obs_dir_.c_str());
  }
  void set_obs_dir(const std::string& d) { obs_dir_ = d; }

  // zeitschritte_bis_obs (dynamik_methoden.cpp:444-455)
  void zeitschritte_bis_obs(time_t last_write) {
    (void)last_write;
    long long n = 0;
    const int s = bd_zeitschritte_bis_obs(dyn.ctx, &n);
    if (s != BD_OK) std::cout << "Fehler: zeitschritte_bis_obs: " << bd_status_string(s) << std::endl;
    schritte_seit_obs += (int)n;
  }

  // obs_point (auswertung.cpp:78-93): the snapshot observable
  void obs_point(int nr_obspoint) {
    bd_schreibe_pos(dyn.ctx, nr_obspoint);
    schritte_seit_obs = 0;
    t = 0.0L;
    obs_nr++;
  }

  void schreibe_obs() {}  // in-run observables other than the snapshots are off by default

 private:
  int device_ = 0;
  std::string obs_dir_;
};

}  // namespace bdb

// bdkap: drop-in for the reference's simulation driver (main.cpp:73-323) on
// libbd_b200.so. Reads a parameter.h (the reference's parameter file format),
// runs `runs` runs of obs_anzahl observation intervals and writes
// pos1_<run+1>.txt / pos2_<run+1>.txt like RunObs (auswertung.cpp:52-93).
//
//   bdkap [parameter.h] [--seed S] [--device D] [--out DIR]
//
// Differences: the initialisers are seeded from --seed + run (the reference
// seeds from time(NULL)); in debugmode every re-initialisation of the dt
// sweep takes the next seed.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <iostream>
#include <string>
#include <vector>

#include "RunZustand.hpp"
#include "bd_api.h"

int main(int argc, char** argv) {
  std::string header = "parameter.h", out = ".";
  uint64_t seed = (uint64_t)time(nullptr);
  int device = 0;
  for (int i = 1; i < argc; i++) {
    if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) seed = std::strtoull(argv[++i], nullptr, 10);
    else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--out") && i + 1 < argc) out = argv[++i];
    else header = argv[i];
  }
  bd_params p;
  bd_params_default(&p);
  if (bd_params_from_header(header.c_str(), &p) != BD_OK) {
    std::cout << "Fehler: " << header << " nicht lesbar" << std::endl;
    return 1;
  }
  const auto t_start = std::chrono::steady_clock::now();
  for (int run = 0; run < p.runs; run++) {
    // RunZustand::ausgabe_jeansgroessen (allgemeine_methoden.cpp:324-348)
    const double rho = (p.N1 + p.N2) / (p.L * p.L);
    const double rho_c = 2.0 / std::sqrt(3.0);
    std::cout << "Jeans-Zeit: \t\t" << 1.0 / (rho * p.kapillar_vorfaktor) << std::endl;
    std::cout << "Jeans-Wellenzahl:\t"
              << std::sqrt(p.kapillar_vorfaktor / p.T * rho /
                           (1 - 3 * rho * rho / rho_c / rho_c - 8 * rho * rho * rho / (rho_c * rho_c * rho_c)))
              << std::endl;
    bdb::RunZustand r(p, device);
    r.set_obs_dir(out);
    r.init(run, seed + (uint64_t)run);
    if (!r.dyn.ctx) return 2;
    r.obs_point(0);
    if (p.krafttestmode) {
      // two-particle force scan (main.cpp:220-248): particle 1 moves along y
      FILE* f = std::fopen((out + "/kapkraft.txt").c_str(), "w");
      std::fprintf(f, "#Format: r Fkap Ftotal\n\n");
      bd_derived d;
      bd_params_derived(&p, &d);
      std::vector<int32_t> g(2 * (size_t)p.N1);
      std::vector<double> q(2 * (size_t)p.N1);
      bd_get_positions(r.dyn.ctx, 0, g.data(), q.data());
      for (double t = 0.001; t < 5.0; t += 0.01) {
        const double origin = g[0] * d.nachList_Breite + q[0];
        const double y = origin + t;
        g[3] = (int)(y / d.nachList_Breite);
        q[3] = y - g[3] * d.nachList_Breite;
        bd_set_positions(r.dyn.ctx, 0, g.data(), q.data());
        r.dyn.berechne_kapkraefte();
        r.dyn.berechne_WCA11();
        std::fprintf(f, "%g \t %g \t %g \n", t, r.dyn.getFKap(), r.dyn.getF());
      }
      std::fclose(f);
      return 0;
    }
    if (p.debugmode) {
      // travel-distance sweep (main.cpp:156-218): for mrd = 1, 0.95, ... > 0.01
      // re-initialise, average |F_WCA,max| and dt over 50 debug steps early
      // and over 50 after max(50, 1.5/mrd) regular steps
      r.obs_point(0);
      bdb::RunZustand::RunDynamik::TimestepInfo info;
      FILE* debugfile1 = std::fopen((out + "/mrd_data1.txt").c_str(), "w");
      FILE* debugfile2 = std::fopen((out + "/mrd_data2.txt").c_str(), "w");
      if (!debugfile1 || !debugfile2) return 3;
      std::fprintf(debugfile1, "# Mittelwerte über 50 Zeitschritte. Früh = erste 50 Zeitschritte. \n");
      std::fprintf(debugfile2, "# Mittelwerte über 50 Zeitschritte. Spät = nach 1000 Zeitschritten \n");
      std::fprintf(debugfile1, "# Format: mrd TAB <F_WCA_max> TAB |F_WCA_highest| TAB dt \n\n");
      std::fprintf(debugfile2, "# Format: mrd TAB <F_WCA_max> TAB |F_WCA_highest| TAB dt \n\n");
      uint64_t init_seed = seed + (uint64_t)run;
      auto fifty = [&](double mrd, FILE* f) {
        double F_mittel = 0.0, F_highest = 0.0, dt_mittel = 0.0;
        for (int count = 0; count < 50; count++) {
          r.dyn.zeitschritt_debug(mrd, info, true);
          dt_mittel += info.dt / 50.0;
          const double F = std::sqrt(info.maxWCAx * info.maxWCAx + info.maxWCAy * info.maxWCAy);
          F_mittel += F / 50.0;
          if (F > F_highest) F_highest = F;
        }
        std::fprintf(f, "%g \t %g \t %g \t %g \n", mrd, F_mittel, F_highest, dt_mittel);
      };
      for (double mrd = 1.0; mrd > 0.01; mrd *= 0.95) {
        std::cout << "mrd=" << mrd << std::endl;
        r.init(run, ++init_seed);
        if (!r.dyn.ctx) return 2;
        fifty(mrd, debugfile1);
        int num_skip = (int)(1.5 / mrd);
        if (num_skip < 50) num_skip = 50;
        for (int count = 0; count < num_skip; count++) r.dyn.zeitschritt(0.1);
        fifty(mrd, debugfile2);
      }
      std::fclose(debugfile1);
      std::fclose(debugfile2);
      return 0;
    }
    std::cout << "Run " << run << ": initial positions written, starting timesteps." << std::endl;
    auto last = std::chrono::steady_clock::now();
    for (int obs_nr = 1; obs_nr < p.obs_anzahl; obs_nr++) {
      r.zeitschritte_bis_obs(time(nullptr));
      const int steps = r.schritte_seit_obs;
      const auto now = std::chrono::steady_clock::now();
      const double sec = std::chrono::duration<double>(now - last).count();
      std::cout << "\nRun " << run << ": recording obs-Point " << r.obs_nr + 1 << " / " << p.obs_anzahl
                << ".\n";
      std::cout << "Run " << run << ": " << steps << " steps since CP. Avg dt: " << p.obs_dt / steps
                << ". Performance: " << (sec > 0 ? steps / sec : 0.0) << " steps/s." << std::endl;
      r.obs_point(obs_nr);
      last = std::chrono::steady_clock::now();
    }
  }
  std::cout << "Time since program launch: "
            << std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count()
            << " seconds." << std::endl;
  return 0;
}

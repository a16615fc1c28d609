// Host-only helpers shared by the engine and the C ABI (bd_host.cpp).
#pragma once

#include <cstdint>
#include <random>

#include "bd_api.h"

namespace bd {

void params_default(bd_params* p);
void params_derived(const bd_params* p, bd_derived* d);
int params_validate(const bd_params* p);
int params_from_header(const char* path, bd_params* p);
void lokdens_params_default(bd_lokdens_params* lp);
int lokdens_params_from_header(const char* path, bd_lokdens_params* lp);
int snapgrid_num(double L, double snapgrid_crude);
// the analysis program's files for frame nr (main_auswertung.cpp:60-77,
// 184-375); g1, g2: double[n*n]; hist int32[4][bins]; over int32[7]
int write_lokdens_frame(const char* dir, const bd_lokdens_params* lp, int n, double width, int nr,
                        double obs_dt, const double* g1, const double* g2, const int32_t* hist,
                        const int32_t* over);
int init_positions_host(const bd_params* p, std::mt19937_64& gen, int methode, int32_t* git[2],
                        double* rel[2]);
int init_pos_from_file(const bd_params* p, const char* path, int32_t* git[2], double* rel[2]);
int write_pos_frame(const char* path, int append, double t, int n, const int32_t* git,
                    const double* rel, double B);

}  // namespace bd

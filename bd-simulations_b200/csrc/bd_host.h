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
int init_positions_host(const bd_params* p, std::mt19937_64& gen, int methode, int32_t* git[2],
                        double* rel[2]);
int init_pos_from_file(const bd_params* p, const char* path, int32_t* git[2], double* rel[2]);
int write_pos_frame(const char* path, int append, double t, int n, const int32_t* git,
                    const double* rel, double B);

}  // namespace bd

// GGX directional-albedo table used by the energy compensation of the Substitute material.
#pragma once

#include "../../include/sprout_b200.h"

namespace spb {

constexpr int Ggx_table_size = 32;

// Row-major [alpha index][cos_theta_o index], both sampled at i / 31; computed once.
float const* ggx_albedo_table();

}  // namespace spb

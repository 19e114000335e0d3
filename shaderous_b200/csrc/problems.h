// Host-side initial conditions (problems.cpp).
#pragma once
#include <cstdint>

#include "../../include/shaderous_b200.h"

namespace shz {

// Float64 primitives (rho, vx, vy, vz, p, s) of planes k0..k1-1, x fastest.
int problem_prims(const shz_config& c, const shz_problem& p, int k0, int k1, double* out);
bool problem_known(int kind);
// Conserved float32 state of `count` cells from float64 primitives, rounded once.
void prims_to_state(const double* w, double gamma, int64_t count, float* u1, float* u2);

}  // namespace shz

// Host-side initial conditions (problems.cpp).
#pragma once
#include <cstdint>

#include "../../include/shaderous_b200.h"

namespace shz {

// A problem with its derived constants (the Sedov deposit's radius and pressure, the box).
struct ProblemCtx {
  shz_problem p;
  double gamma;
  int nd;
  double L[3];
  double sedov_r = 0, sedov_p = 0;
};
ProblemCtx prepare_problem(const shz_config& c, const shz_problem& p);
// Float64 primitives at one cell centre (box centred on 0); `cell` numbers it for seeded noise.
void sample_problem(const ProblemCtx& q, double x, double y, double z, uint64_t cell, double* w);
// Float64 primitives (rho, vx, vy, vz, p, s) of planes k0..k1-1, x fastest.
int problem_prims(const shz_config& c, const shz_problem& p, int k0, int k1, double* out);
bool problem_known(int kind);
// Conserved float32 state of `count` cells from float64 primitives, rounded once.
void prims_to_state(const double* w, double gamma, int64_t count, float* u1, float* u2);

}  // namespace shz

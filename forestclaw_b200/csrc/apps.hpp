// apps.hpp -- host-side application callbacks of the built-in problems
// (the qinit / setaux / tagging a ForestClaw app installs in its vtables).
#pragma once
#include "fc2d_b200.h"
#include "host_forest.hpp"

namespace fcb {

// setaux for one patch into aux (maux*nxy doubles, Fortran layout).
void app_setaux(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, double* aux);
// qinit for one patch into q (meqn*nxy doubles, ghosts included).
void app_qinit(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, const double* aux, double* q);
// The sphere app's rotation: unit axis and angular speed (psi = omega (axis . x)).
void app_sphere_flow(const fc2d_b200_options_t& o, double axis[3], double* omega);
// Constant state imposed by mthbc = 0 sides (shock-bubble inflow); false if the app has none.
bool app_inflow_state(const fc2d_b200_options_t& o, double* q);
// The tagging criterion in force (FC2D_B200_TAG_*, TAG_APP resolved to the app's own).
int tag_criterion(const fc2d_b200_options_t& o);
// Refinement test of one patch on the host (tag4refinement at initialization).
int app_tag_refine(const fc2d_b200_options_t& o, const Dims& d, const PatchInfo& P, const double* q);

}  // namespace fcb

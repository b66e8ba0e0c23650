// MD integrator kernels (md.cu).
#pragma once

#include "tgap_internal.h"

namespace tgap {

// velocity_verlet (src/md/md_utils.f90:486-532): masses in eV fs^2 / A^2, no fixed atoms.
int velocity_verlet(tgap_context *ctx, int n, double *pos, double *pos_prev, double *vel,
                    const double *forces, double *forces_prev, const double *mass, double dt,
                    double dt_prev, int first_step);

}  // namespace tgap

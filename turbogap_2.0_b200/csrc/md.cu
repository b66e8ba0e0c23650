// Velocity Verlet on the device (src/md/md_utils.f90:486-532), FP64. A non-finite force is
// recorded in the device check word (reported as TGAP_ERR_NUMERIC by the next state read).
//
// After the update velocities are synchronous with positions_prev and positions are dt
// ahead: v(t) = v(t-dt) + 0.5 (F + F_prev) / m dt_prev (skipped on the first step),
// x(t+dt) = x(t) + v dt + 0.5 F / m dt^2, F_prev = F.
#include "md_kernels.h"

namespace tgap {

__global__ void k_velocity_verlet(int n, double *__restrict__ pos, double *__restrict__ pos_prev,
                                  double *__restrict__ vel, const double *__restrict__ f,
                                  double *__restrict__ f_prev, const double *__restrict__ mass,
                                  double dt, double dt_prev, int first_step, int *check)
{
    pdl_enter();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 3 * n) return;
    const int i = g / 3;
    const double m = mass[i];
    double v = vel[g];
    const double fg = f[g];
    if (!isfinite(fg)) check_fail(check, kCheckNonFinite, i, g - 3 * i);
    if (!first_step) v = v + 0.5 * (fg + f_prev[g]) / m * dt_prev;
    vel[g] = v;
    const double x = pos[g];
    pos_prev[g] = x;
    f_prev[g] = fg;
    pos[g] = x + v * dt + 0.5 * fg / m * (dt * dt);
}

int velocity_verlet(tgap_context *ctx, int n, double *pos, double *pos_prev, double *vel,
                    const double *forces, double *forces_prev, const double *mass, double dt,
                    double dt_prev, int first_step)
{
    if (n <= 0) return TGAP_OK;
    const int T = 256;
    StageScope sc(ctx, "velocity_verlet");
    TGAP_CUDA(ctx, launch_pdl(k_velocity_verlet, dim3((3 * n + T - 1) / T), dim3(T), 0, ctx->stream, n, pos,
                              pos_prev, vel, forces, forces_prev, mass, dt, dt_prev, first_step, ctx->d_check));
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}

}  // namespace tgap

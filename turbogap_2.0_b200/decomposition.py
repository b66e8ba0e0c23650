"""Atom decomposition over the ranks of a process group (one process per GPU).

TurboGAP splits the sites of a structure over its MPI ranks (split_tasks, src/utils/misc.f90:88-111),
each rank evaluates the energies of its own sites and their force and virial contributions on every
atom, and collect_calculation (src/mpi/mpi_utils.f90:515-545) sums the ranks; the integrator then
runs on the replicated positions. Here each rank drives its own GPU: the system's site range
(tgap_system_set_site_range) restricts the descriptor centres to the rank's share, one all-reduce
over torch.distributed (NCCL between GPUs, gloo on the host) sums forces, energies and virials in one
contiguous buffer, and every rank applies the same velocity Verlet update (tgap_velocity_verlet) to
the same summed forces, so the positions stay identical on all ranks without a broadcast.
"""
import ctypes as C

from .native import TGAP_FP64, check


def split_tasks(n_sites, n_tasks, rank):
    """0-based [beg, end) of rank's sites: the first n_sites % n_tasks ranks take one more
    (misc.f90:88-111, whose 1-based i_beg/i_end are beg + 1 and end)."""
    if n_tasks < 1 or not 0 <= rank < n_tasks:
        raise ValueError("rank outside the task count")
    q, r = divmod(n_sites, n_tasks)
    if rank < r:
        beg = rank * (q + 1)
        return beg, beg + q + 1
    beg = r * (q + 1) + (rank - r) * q
    return beg, beg + q


def collect(buf, dist=None, group=None):
    """Sums a rank's partial outputs over the group in place (collect_calculation); with no
    process group the buffer is already the total."""
    if dist is not None and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    return buf


class ShardedMD:
    """NVE velocity Verlet with the sites split over the ranks of a process group.

    Every rank holds the whole system (positions replicated, neighbor lists over all atoms) and
    evaluates only its own sites; forces, energies and virials are summed over the ranks by one
    all-reduce per step, then each rank integrates all atoms. With one rank it is plain MD.
    Steps are eager (the all-reduce sits between the force evaluation and the integrator)."""

    def __init__(self, ctx, system, models, masses_amu, dt, rebuild_every=10, precision=TGAP_FP64,
                 dist=None, group=None):
        import numpy as np
        import torch
        self.ctx, self.system, self.models = ctx, system, list(models)
        self.dt, self.rebuild_every, self.precision = float(dt), int(rebuild_every), precision
        self.dist, self.group = dist, group
        world = dist.get_world_size(group) if dist is not None and dist.is_initialized() else 1
        rank = dist.get_rank(group) if dist is not None and dist.is_initialized() else 0
        n = system.n_atoms
        self.n = n
        self.range = split_tasks(n, world, rank)
        system.set_site_range(*self.range)
        # forces (3n), energies (n), virials (9 per structure): one buffer, one collective
        nst = system.n_structures
        self.out = torch.zeros(4 * n + 9 * nst, dtype=torch.float64, device="cuda")
        self.forces = self.out[:3 * n]
        self.energies = self.out[3 * n:4 * n]
        self.virial = self.out[4 * n:]
        self.mass = torch.as_tensor(np.asarray(masses_amu, dtype=np.float64) * 103.6426965268,
                                    device="cuda")  # read_files.f90:333
        self.vel = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
        self.pos_prev = torch.zeros_like(self.vel)
        self.forces_prev = torch.zeros_like(self.vel)
        self.step = 0

    def set_velocities(self, v):
        import numpy as np
        import torch
        self.vel.copy_(torch.as_tensor(np.asarray(v, dtype=np.float64).reshape(-1)))

    def _forces(self, rebuild):
        import torch
        self.system.update(rebuild)
        self.out.zero_()
        torch.cuda.synchronize()
        self.system.compute_device(self.models, self.precision, self.energies.data_ptr(), self.forces.data_ptr(),
                                   self.virial.data_ptr())
        self.ctx.synchronize()
        collect(self.out, self.dist, self.group)

    def run(self, n_steps):
        L = self.ctx._L
        pos = C.c_void_p(self.system.device_positions())
        for _ in range(int(n_steps)):
            self._forces(self.step % self.rebuild_every == 0)
            check(L.tgap_velocity_verlet(self.ctx.h, self.n, pos, C.c_void_p(self.pos_prev.data_ptr()),
                                         C.c_void_p(self.vel.data_ptr()), C.c_void_p(self.forces.data_ptr()),
                                         C.c_void_p(self.forces_prev.data_ptr()), C.c_void_p(self.mass.data_ptr()),
                                         self.dt, self.dt, int(self.step == 0)), self.ctx.h, "tgap_velocity_verlet")
            self.step += 1
        self.ctx.synchronize()

    def state(self):
        """Host copies: positions, velocities, forces (n, 3), potential and kinetic energy of the
        last evaluated step (energies summed over the ranks)."""
        import numpy as np
        n = self.n
        v = self.vel.cpu().numpy().reshape(n, 3)
        m = self.mass.cpu().numpy()
        return dict(positions=self.system.get_positions(), velocities=v,
                    forces=self.forces.cpu().numpy().reshape(n, 3), e_pot=float(self.energies.sum()),
                    e_kin=float(0.5 * np.sum(m[:, None] * v * v)))

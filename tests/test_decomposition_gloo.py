"""Atom decomposition (turbogap_b200.decomposition) on the host: split_tasks against the
reference's formula (misc.f90:88-111), and the exchange step with two gloo ranks on the CPU. Each
rank evaluates the energies, forces and virial of its own sites with the oracle, as one MPI rank of
the reference does with its slice of the neighbor list, and collect() sums the ranks
(collect_calculation, mpi_utils.f90:515-545): the sums equal the single-process evaluation, and
every rank holds the same bits afterwards."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _split_tasks_reference(n_sites, n_tasks, rank):
    """misc.f90:88-111 verbatim in its integer arithmetic (1-based i_beg, i_end)."""
    if rank < n_sites % n_tasks:
        i_beg = 1 + rank * (n_sites // n_tasks + 1)
        i_end = (rank + 1) * (n_sites // n_tasks + 1)
    else:
        i_beg = 1 + (n_sites % n_tasks) * (n_sites // n_tasks + 1) + (rank - n_sites % n_tasks) * (n_sites // n_tasks)
        i_end = i_beg + n_sites // n_tasks - 1
    return i_beg, i_end


def test_split_tasks_matches_reference_and_partitions(tg):
    from turbogap_b200 import decomposition as dc
    for n in (1, 7, 64, 4096, 32768, 4099):
        for world in (1, 2, 3, 8):
            prev = 0
            for r in range(world):
                beg, end = dc.split_tasks(n, world, r)
                i_beg, i_end = _split_tasks_reference(n, world, r)
                assert (beg + 1, end) == (i_beg, i_end)
                assert beg == prev
                prev = end
            assert prev == n


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _slice(nb, beg, end):
    st = np.concatenate([[0], np.cumsum(nb["n_neigh"])])
    return {k: (v[beg:end] if k == "n_neigh" else v[st[beg]:st[end]]) for k, v in nb.items()}


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import conftest
    import helpers
    import oracle_lib as orc
    tg = conftest.load_package()
    from turbogap_b200 import decomposition as dc
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    hyp, m = helpers.carbon_model(tg.synth, 40, seed=5, n_pool_structs=1)
    pos, box, sp, _ = tg.synth.random_packing(96, 2.5, 1.2, seed=8)
    n = len(pos)
    nb = orc.build_neighbors(pos, n, *box, 3.7, sp, False)
    beg, end = dc.split_tasks(n, world, rank)
    e, f, v = orc.get_gap_soap(orc.Hypers(hyp), n, _slice(nb, beg, end), sp, 0, m["alphas"], m["Qs"], 1.0, 4.0)
    buf = torch.from_numpy(np.concatenate([f.reshape(-1), e, v.reshape(-1, order="F")]))
    dc.collect(buf, dist)
    out[rank] = buf.numpy().copy()
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_sum_to_the_single_process_result(tg):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers
    import oracle_lib as orc
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        r0, r1 = out[0], out[1]
    assert np.array_equal(r0, r1)  # every rank holds the same summed bits
    hyp, m = helpers.carbon_model(tg.synth, 40, seed=5, n_pool_structs=1)
    pos, box, sp, _ = tg.synth.random_packing(96, 2.5, 1.2, seed=8)
    n = len(pos)
    nb = orc.build_neighbors(pos, n, *box, 3.7, sp, False)
    e, f, v = orc.get_gap_soap(orc.Hypers(hyp), n, nb, sp, 0, m["alphas"], m["Qs"], 1.0, 4.0)
    full = np.concatenate([f.reshape(-1), e, v.reshape(-1, order="F")])
    assert np.max(np.abs(r0 - full)) < 1e-12

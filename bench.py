"""Headline benchmark of the SOAP/GAP energy-and-force path on B200.

Workload (the reference's NVE MD configuration): 4,096 carbon atoms at 2.5 g/cm^3 in a cubic
periodic box (seeded rejection sampling, 1.2 A minimum distance), Maxwell-Boltzmann velocities
at 3000 K, velocity-Verlet NVE with dt = 1 fs, neighbor list rebuilt every 10 steps with a
0.3 A skin; SOAP poly3 n_max = l_max = 8, rcut 3.7/3.2 A, sigma 0.5 A; synthetic GAP with
2,000 sparse points (normalised SOAP vectors of random atoms from 10 further seeded boxes),
zeta = 4, delta = 1 eV, alphas ~ N(0, 1e-6).

A step is one MD step (geometry refresh or rebuild, descriptor, GAP contraction, adjoint force
back-scatter, integrator). `value` is atom-steps/s of the mixed-precision path (FP32 descriptor,
bf16x3 tcgen05 GEMMs, FP64 accumulation), device-timed with CUDA events per step, L2 flushed
(256 MB write) between timed steps. The plain FP64 path is measured the same way and reported
beside it. `e2e` drives the same MD through the host-buffer C ABI call (positions in, energies/
forces/virial out every step, integrator on the host). N > 1 GPUs run independent replicas.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "atom-steps/s & MC moves/s: mixed/surrogate vs plain FP64, 1 B200, at stated RMSE"
WORKLOAD = ("NVE velocity-Verlet MD, 4096 C atoms, 2.5 g/cm3, dt 1 fs, rebuild every 10 steps, "
            "skin 0.3 A, SOAP n_max=l_max=8 rcut 3.7/3.2, GAP 2000 sparse zeta=4")
N_ATOMS = 4096
N_SPARSE = 2000
# neighbor skin of the MC lists: 0.5, 0.7, 0.9 and 1.2 A measured 48, 55, 59 and 60 k mixed moves/s
# (438, 194, 81 and 42 list rebuilds per 20k proposals, each a host round trip)
MC_ATOMS, MC_DENSITY, MC_T, MC_RADIUS, MC_SKIN = 1000, 2.0, 2000.0, 0.2, 1.0
MC_PROPOSALS = 20000
MC_WORKLOAD = ("NVT Metropolis MC, 1000 C atoms, 2.0 g/cm3, 2000 K, single-atom moves uniform in a 0.2 A ball, "
               "local SOAP/GAP update of atoms within rcut of the moved atom (lists with a 1.0 A skin), same SOAP "
               "settings and 2000-sparse GAP as the MD workload; plain GAP MC evaluates 12 (mixed) or 4 (FP64) "
               "proposals side by side and settles them in proposal order (speculative batch: the same chain as one "
               "at a time); 'screened': "
               "delayed acceptance "
               "with a PCA-64 / 128 / 128 SiLU bf16 screen trained on 200k atomic energies of 2000 plain-MC "
               "snapshots, proposals one at a time")
DT = 1.0
REBUILD = 10
SKIN = 0.3
L2_NOTE = ("flushed between timed steps (untimed: 256 MB device write, then a 256 MB read of a second buffer so "
           "the written lines are evicted)")


def _load_package():
    import importlib.util
    if "turbogap_b200" in sys.modules:
        return sys.modules["turbogap_b200"]
    pkg_dir = os.path.join(ROOT, "turbogap_2.0_b200")
    spec = importlib.util.spec_from_file_location(
        "turbogap_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["turbogap_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _workload(tg, seed):
    pos, box, sp, masses = tg.synth.random_packing(N_ATOMS, 2.5, 1.2, seed=seed)
    vel = tg.synth.maxwell_boltzmann(masses, 3000.0, seed=seed + 1)
    return pos, box, sp, masses, vel


def _pool_structures(tg, seed):
    return [tg.synth.random_packing(N_ATOMS, 2.5, 1.2, seed=seed + 100 + k)[:3] for k in range(10)]


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return dict(hbm=p["hbm_gbs"], bf16=p["bf16_tflops"], bf16_sus=p["bf16_tflops_sustained"], src="measured")
    except Exception:
        return dict(hbm=6650.0, bf16=1590.0, bf16_sus=1400.0, src="fallback")


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """SM clock, power and clock-event reasons sampled every ~2 ms through NVML while a timed
    region runs (start() before it, stop() after its synchronize). NVML is queried directly, not
    through nvidia-smi, so a timed region of a few milliseconds still gets samples; the first
    and last samples bracket the region."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device_index):
        self.samples = []
        self.err = None
        self.h = None
        self._stop = threading.Event()
        try:
            import pynvml
            import torch
            self.nv = pynvml
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(device_index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: the line says so
            self.err = f"nvml unavailable: {e}"

    def _sample(self):
        nv = self.nv
        try:
            sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
            try:
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except AttributeError:
                bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
            pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
            self.samples.append((sm, int(bits), pw))
        except Exception as e:
            self.err = str(e)

    def _loop(self):
        while not self._stop.is_set():
            self._sample()
            time.sleep(0.002)

    def start(self):
        if self.h is None:
            return
        self._sample()
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.h is None:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=[self.err], samples=0)
        self._sample()
        self._stop.set()
        self.thread.join(timeout=2)
        sm = [x[0] for x in self.samples]
        reasons = sorted({name for _, bits, _ in self.samples for bit, name in self.REASONS.items() if bits & bit})
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=self.max_mhz, reasons=reasons,
                    samples=len(sm), sm_mhz_min=min(sm) if sm else None,
                    power_w_max=max(x[2] for x in self.samples) if sm else None, source="nvml, 2 ms")


# ----------------------------------------------------------------------------- reference arm

def _oracle_md_steps(orc, hyp, model, pos, box, sp, masses, vel, steps, budget_s, warmup):
    """velocity_verlet MD of the oracle (FP64 CPU restatement), list rebuilt every REBUILD steps
    at rcut + skin, geometry refreshed every step. Returns (steps done, seconds)."""
    H = orc.Hypers(hyp)
    n = len(pos)
    x = pos.copy()
    v = vel.copy()
    xp = np.zeros_like(x)
    fp = np.zeros_like(x)
    mm = masses * 103.6426965268
    dtp = DT
    nb = None
    done = 0
    t0 = None
    for k in range(warmup + steps):
        if k == warmup:
            t0 = time.perf_counter()
        if k % REBUILD == 0 or nb is None:
            nb = orc.build_neighbors(x, n, *box, 3.7 + SKIN, sp, False)
        else:
            nb.update(orc.neighbor_geometry(x, n, *box, nb["n_neigh"], nb["neighbors_list"], sp))
        _, f, _ = orc.get_gap_soap(H, n, nb, sp, 0, model["alphas"], model["Qs"], model["delta"], model["zeta"])
        dtp = orc.velocity_verlet(x, xp, v, f, fp, mm, DT, dtp, k == 0)
        if k >= warmup:
            done += 1
            if time.perf_counter() - t0 > budget_s:
                break
    return done, time.perf_counter() - t0


def _md_config(n_pairs):
    """The `config` of the headline line; both arms report the same one."""
    return {"workload": WORKLOAD, "n_atoms": N_ATOMS, "n_sparse": N_SPARSE, "pairs_in_list": int(n_pairs),
            "l2": L2_NOTE, "parallelism": "single GPU"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    tg = _load_package()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers
    import oracle_lib as orc
    hyp = tg.synth.carbon_hypers()
    pool = [helpers.oracle_descriptors(hyp, p, b, s) for p, b, s in _pool_structures(tg, 1000)]
    model = tg.synth.gap_model(np.concatenate(pool), N_SPARSE, seed=7)
    pos, box, sp, masses, vel = _workload(tg, 0)
    n_pairs = int(orc.build_neighbors(pos, N_ATOMS, *box, 3.7 + SKIN, sp, False)["n_neigh"].sum())
    steps, secs = _oracle_md_steps(orc, hyp, model, pos, box, sp, masses, vel, args.steps, 150.0, args.warmup)
    value = N_ATOMS * steps / secs
    cores = orc.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _md_config(n_pairs),  # the same workload and keys as the GPU arm's line
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{steps} MD steps of the 4096-atom box after {args.warmup} untimed ones on the "
                                   f"host cores (oracle restatement with OpenMP, not TurboGAP; the Fortran "
                                   f"reference cannot be compiled here)"},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- our arm

class L2Flush:
    """Untimed L2 flush between timed steps: write a buffer larger than the 126 MB L2, then read a
    second one, so the timed step starts with a cold L2 holding no dirty lines (their write-back
    would otherwise be charged to the step)."""

    def __init__(self, torch):
        n = 256 * 1024 * 1024 // 4
        self.w = torch.empty(n, dtype=torch.float32, device="cuda")
        self.r = torch.zeros(n, dtype=torch.float32, device="cuda")

    def flush(self):
        self.w.zero_()
        self.r.sum()


def _timed_md(tg, torch, ctx, stream, flush, system, model, masses, vel, precision, steps, warmup):
    md = tg.MD(ctx, system, [model], masses, DT, rebuild_every=REBUILD, precision=precision, use_graph=True)
    md.set_velocities(vel)
    with torch.cuda.stream(stream):
        md.run(warmup)
        ctx.synchronize()
        st0 = md.state()
        l0 = ctx.kernel_launches
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        for k in range(steps):
            flush.flush()
            starts[k].record(stream)
            md.run(1)
            ends[k].record(stream)
        stream.synchronize()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    launches = ctx.kernel_launches - l0
    st1 = md.state()
    md.close()
    return ms, launches, st0, st1


def _timing_report(ctx):
    """Stage totals collected by the library's stage timers (tgap_timing_*), then reset."""
    from turbogap_b200 import native
    import ctypes as C
    L = native.lib()
    cap = 64
    names = C.create_string_buffer(32 * cap)
    tot = np.zeros(cap)
    cnt = np.zeros(cap, np.int64)
    n = C.c_int(0)
    L.tgap_timing_report(ctx.h, cap, names, native.ptr(tot), native.ptr(cnt), C.byref(n))
    out = {}
    for i in range(n.value):
        nm = names.raw[32 * i:32 * (i + 1)].split(b"\0")[0].decode()
        if cnt[i]:
            out[nm] = dict(total_ms=float(tot[i]), launches=int(cnt[i]), avg_us=1e3 * tot[i] / cnt[i])
    L.tgap_timing_reset(ctx.h)
    return out


def _stage_profile(tg, ctx, system, models, masses, vel, precision, steps=20, dt=DT):
    """Per-stage device time of `steps` eager MD steps (CUDA events around every stage)."""
    from turbogap_b200 import native
    L = native.lib()
    md = tg.MD(ctx, system, models, masses, dt, rebuild_every=REBUILD, precision=precision, use_graph=False)
    md.set_velocities(vel)
    md.run(2)
    ctx.synchronize()
    L.tgap_timing_reset(ctx.h)
    L.tgap_timing_enable(ctx.h, 1)
    md.run(steps)
    L.tgap_timing_enable(ctx.h, 0)
    out = _timing_report(ctx)
    md.close()
    return out


def _eval_stage_profile(tg, torch, ctx, system, models, precision, reps):
    """Per-stage device time of `reps` single-point evaluations (tgap_compute on the current list)."""
    from turbogap_b200 import native
    L = native.lib()
    n, nst = system.n_atoms, system.n_structures
    e = torch.zeros(n, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(9 * nst, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    system.compute_device(models, precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    ctx.synchronize()
    L.tgap_timing_reset(ctx.h)
    L.tgap_timing_enable(ctx.h, 1)
    for _ in range(reps):
        system.compute_device(models, precision, e.data_ptr(), f.data_ptr(), v.data_ptr())
    L.tgap_timing_enable(ctx.h, 0)
    return _timing_report(ctx)


FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # B200 CUDA-core FP32, nominal (not measured)


def _work(rows, dim, n_sparse, n_pairs, n_cut, alpha, l_max, n_models=1):
    """Algorithmic work of one evaluation: rows = descriptor rows over all models (each atom is a
    row of the model of its species), n_pairs list pairs, n_cut in-cutoff pairs (self excluded),
    alpha radial functions per neighbor, K_l = (l_max + 1)(l_max + 2) / 2 angular functions."""
    return dict(rows=rows, dim=dim, dim_pad=(dim + 127) // 128 * 128, n_sparse=n_sparse,
                n_sparse_pad=(n_sparse + 127) // 128 * 128, n_pairs=n_pairs, n_cut=n_cut, alpha=alpha,
                l_max=l_max, n_models=n_models)


def _stage_roofline(name, st, evals, total_ms, W, peaks):
    """Roofline of one stage from its CUDA-event time per evaluation (evals evaluations measured)
    and the algorithmic work of one evaluation.

    GEMMs: 2 N D M flops per product (the fused kernel does two: q Qs^T and G Qs), bf16x3 against
    the measured burst bf16 peak (the split executes 3x that, reported as executed_tflops); FP64
    GEMMs against the measured cuBLAS FP64 peak. Descriptor kernels: the contract's HBM figure
    from algorithmic bytes, and beside it the FP32 figure that actually bounds them, 4 alpha K_l
    (forward) or 12 alpha K_l (adjoint) flops per in-cutoff pair, against the nominal FP32 peak.
    """
    t = st["total_ms"] * 1e-3 / evals
    share = st["total_ms"] / total_ms
    base = dict(kernel=name, share=share, us_per_eval=t * 1e6, launches_per_eval=st["launches"] / evals)
    N, D, M = W["rows"], W["dim"], W["n_sparse"]
    if name.startswith("gemm_bf16x3"):
        prods = 2.0 if name.endswith("fused") else 1.0
        ach = prods * 2.0 * N * D * M / t / 1e12
        exe = prods * 3.0 * 2.0 * N * W["dim_pad"] * W["n_sparse_pad"] / t / 1e12
        return dict(base, bound="tensor", achieved=ach, peak=peaks["bf16"], unit="TFLOP/s",
                    frac=ach / peaks["bf16"], frac_of_sustained=ach / peaks["bf16_sus"], executed_tflops=exe,
                    executed_frac=exe / peaks["bf16"], peak_source=peaks["src"] + " bf16 (burst)")
    if name.startswith("dgemm"):
        ach = 2.0 * N * D * M / t / 1e12
        fp64 = peaks.get("fp64")
        return dict(base, bound="fp64 tensor", achieved=ach, peak=fp64, unit="TFLOP/s",
                    frac=ach / fp64 if fp64 else None, peak_source="measured cuBLAS DGEMM 8192^3 (this run)")
    nlm, nmax = (W["l_max"] + 1) ** 2, W["alpha"]
    kl = (W["l_max"] + 1) * (W["l_max"] + 2) // 2
    P, Pc = W["n_pairs"], W["n_cut"]
    fp32 = None
    if name.startswith("soap_forward"):
        # reads the pair list (xyz, r, species: 36 B/pair), writes c, q (+bf16 split), |p|
        byts = 36.0 * P + N * (4.0 * nmax * nlm + 8.0 * W["dim_pad"] + 4.0)
        fp32 = 4.0 * W["alpha"] * kl * Pc
    elif name.startswith("soap_backward"):
        # reads pairs (+ neighbor index), c, q, g; scatters 3 FP64 forces per pair
        byts = 64.0 * P + N * (4.0 * nmax * nlm + 8.0 * W["dim_pad"] + 4.0)
        fp32 = 12.0 * W["alpha"] * kl * Pc
    else:
        byts = 48.0 * P
    ach = byts / t / 1e9
    out = dict(base, bound="hbm", achieved=ach, peak=peaks["hbm"], unit="GB/s", frac=ach / peaks["hbm"],
               peak_source=peaks["src"] + " HBM copy")
    if fp32 is not None and name.endswith("f32"):
        a32 = fp32 / t / 1e12
        out["fp32"] = dict(achieved=a32, peak=FP32_NOMINAL_TFLOPS, unit="TFLOP/s", frac=a32 / FP32_NOMINAL_TFLOPS,
                           peak_source="nominal 148 SM x 128 lanes x 2 x 1.965 GHz", in_cutoff_pairs=Pc)
    return out


def _roofline(stages, evals, W, peaks, traffic=False):
    """Roofline of the dominant stage, plus every costed stage's in `all`."""
    if not stages:
        return None
    total = sum(v["total_ms"] for v in stages.values())
    costed = ("gemm_bf16x3", "soap_forward", "soap_backward", "dgemm")
    rows = {k: _stage_roofline(k, v, evals, total, W, peaks) for k, v in stages.items() if k.startswith(costed)}
    name = max(stages.items(), key=lambda kv: kv[1]["total_ms"])[0]
    dom = dict(rows.get(name) or _stage_roofline(name, stages[name], evals, total, W, peaks))
    dom["traffic"] = _ncu_traffic(name) if traffic else None
    if dom["traffic"] is not None:
        dom["traffic_note"] = "ncu dram read+write bytes per launch (profiles/ncu_traffic.txt)"
    dom["all"] = {k: {kk: vv for kk, vv in v.items() if kk not in ("kernel",)} for k, v in rows.items()}
    return dom


def _fp64_peak(torch):
    """Measured FP64 tensor-core peak of this GPU: cuBLAS DGEMM 8192^3 (torch.matmul), best of 4."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        c = a @ b
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


def _ncu_traffic(kernel):
    """dram bytes per launch of `kernel` from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def _e2e(tg, ctx, system, model, masses, vel, pos0, precision, steps):
    """MD driven through the host-buffer C ABI call (calculate_gap_soap surface): positions
    host->device, energies/forces/virial device->host every step, integrator on the host."""
    from turbogap_b200 import native
    import ctypes as C
    L = native.lib()
    n = len(masses)
    x = np.ascontiguousarray(pos0.copy())
    v = vel.copy()
    mm = (masses * 103.6426965268)[:, None]
    e = np.zeros(n)
    f = np.zeros((n, 3))
    fp = np.zeros((n, 3))
    vir = np.zeros(9)
    arr = (C.c_void_p * 1)(model.h.value)
    v = np.ascontiguousarray(v)
    m_col = np.ascontiguousarray(mm[:, 0])
    # the arrays live for the whole run: their addresses are taken once, and they are registered
    # with the context as pinned host memory, which the call then reads and writes directly
    px, pe, pf, pv, pfp, pm, pvir = (native.ptr(a) for a in (x, e, f, v, fp, m_col, vir))
    for a in (x, e, f, vir):
        native.check(L.tgap_host_register(ctx.h, native.ptr(a), a.nbytes), ctx.h, "tgap_host_register")

    def force(k):
        st = L.tgap_calculate_gap_soap(ctx.h, system.h, 1, arr, int(precision), px, int(k % REBUILD == 0), pe, pf,
                                       pvir)
        native.check(st, ctx.h, "tgap_calculate_gap_soap")

    # warm-up: both call configurations (with and without the list rebuild) run eagerly once and
    # are captured as graphs, as in any MD loop after its first two rebuild intervals
    for k in range(2 * REBUILD + 2):
        force(k)
    x[:] = pos0
    t0 = time.perf_counter()
    for k in range(steps):
        force(k)
        # velocity Verlet on the host (md_utils.f90:486-532), as the reference integrates
        native.check(L.tgap_velocity_verlet_host(n, px, None, pv, pf, pfp, pm, DT, DT, int(k == 0)), ctx.h,
                     "tgap_velocity_verlet_host")
    secs = time.perf_counter() - t0
    for a in (x, e, f, vir):
        native.check(L.tgap_host_unregister(ctx.h, native.ptr(a)), ctx.h, "tgap_host_unregister")
    return dict(value=n * steps / secs, unit="atom-steps/s", h2d_bytes_per_step=8 * 3 * n,
                d2h_bytes_per_step=8 * (4 * n + 9), steps=steps, precision="mixed" if precision else "fp64")


def _cpu_baseline(tg, pos, box, sp, masses, vel, model_np):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as orc
    hyp = tg.synth.carbon_hypers()
    steps, secs = _oracle_md_steps(orc, hyp, model_np, pos, box, sp, masses, vel, 1000, 20.0, 0)
    return dict(value=N_ATOMS * steps / secs, unit="atom-steps/s", cores=orc.num_threads(), kind="port",
                sample=f"{steps} MD steps of the same 4096-atom box (FP64 oracle restatement with OpenMP, "
                       f"materialised dq/dr as in the reference; not TurboGAP itself)")


def _mc_leg(tg, torch, ctx, stream, model, n_prop, seed):
    """MC moves/s of the local-update driver (both precisions) on the 1000-atom box: CUDA events
    around tgap_mc_run (its host loop, list rebuilds and graph launches included)."""
    pos, box, sp, _ = tg.synth.random_packing(MC_ATOMS, MC_DENSITY, 1.2, seed=seed)
    atoms, disp, u = tg.synth.mc_proposals(MC_ATOMS, n_prop + 256, MC_RADIUS, seed=seed + 1)
    out = {}
    for name, prec in (("mixed", tg.TGAP_MIXED), ("fp64", tg.TGAP_FP64)):
        system = tg.System(ctx, [(pos, box, sp)], 3.7 + MC_SKIN)
        mc = tg.MC(ctx, system, [model], MC_T, precision=prec)
        mc.run(atoms[:256], disp[:256], u[:256], logs=False)  # warm-up: graph capture, first rebuilds
        st0 = mc.state()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = mc.run(atoms[256:], disp[256:], u[256:], logs=False)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st1 = mc.state()
        bs = mc.batch_stats()
        out[name] = dict(moves_per_s=n_prop / (ms * 1e-3), us_per_move=1e3 * ms / n_prop,
                         acceptance=r["accepted"] / n_prop, list_rebuilds=st1["rebuilds"] - st0["rebuilds"],
                         proposals_per_speculative_batch=round(bs["settled"] / max(1, bs["batches"]), 3))
        if name == "mixed":
            final = st1
        mc.close()
        system.close()
    screened = _mc_screen_leg(tg, torch, ctx, stream, model, n_prop, seed, final)
    return dict(workload=MC_WORKLOAD, proposals=n_prop, unit="moves/s", value=out["mixed"]["moves_per_s"],
                mixed=out["mixed"], plain_fp64=out["fp64"], screened=screened,
                speedup_mixed_vs_fp64=out["mixed"]["moves_per_s"] / out["fp64"]["moves_per_s"])


def _rdf(pos, box, r_max=6.0, bins=60):
    """g(r) of a cubic periodic box (minimum image), numpy."""
    L = box[0][0]
    n = len(pos)
    d = pos[:, None, :] - pos[None, :, :]
    d -= L * np.round(d / L)
    r = np.sqrt((d ** 2).sum(-1))[np.triu_indices(n, 1)]
    h, edges = np.histogram(r, bins=bins, range=(0.0, r_max))
    shell = 4.0 / 3.0 * np.pi * (edges[1:] ** 3 - edges[:-1] ** 3)
    return h / (shell * n * (n - 1) / 2 / L ** 3)


def _mc_screen_leg(tg, torch, ctx, stream, model, n_prop, seed, plain):
    """The MC workload with the learned screen (delayed acceptance): training on 200k atomic
    energies from 2000 snapshots of plain (exact) MC, then screened moves/s on a fresh chain, and
    the comparison with the plain chain (energy statistics, radial distribution function)."""
    import ctypes as C
    from turbogap_b200 import native
    pos, box, sp, _ = tg.synth.random_packing(MC_ATOMS, MC_DENSITY, 1.2, seed=seed)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + MC_SKIN)
    mc = tg.MC(ctx, system, [model], MC_T, precision=tg.TGAP_MIXED)
    n_snap, gap = 2000, 5
    atoms, disp, u = tg.synth.mc_proposals(MC_ATOMS, n_snap * gap, MC_RADIUS, seed=seed + 7)
    rng = np.random.default_rng(seed + 8)
    q = torch.zeros((MC_ATOMS, model.dim), dtype=torch.float64, device="cuda")
    qs, es = [], []
    t0 = time.perf_counter()
    for k in range(n_snap):
        mc.run(atoms[k * gap:(k + 1) * gap], disp[k * gap:(k + 1) * gap], u[k * gap:(k + 1) * gap], logs=False)
        e_atoms = mc.state()["energies"]
        system.update(False)
        nr = C.c_int(0)
        native.check(native.lib().tgap_descriptors(ctx.h, system.h, model.h, 0, C.c_void_p(q.data_ptr()),
                                                   C.byref(nr)), ctx.h, "descriptors")
        ctx.synchronize()
        pick = rng.choice(MC_ATOMS, size=100, replace=False)
        qs.append(q[torch.as_tensor(pick, device="cuda")].cpu().numpy())
        es.append(e_atoms[pick])
    t_data = time.perf_counter() - t0
    mc.close()
    system.close()
    qs, es = np.concatenate(qs), np.concatenate(es)
    val = rng.random(len(es)) < 0.05
    t0 = time.perf_counter()
    w, fit_log = tg.screen.fit(ctx, qs[~val], es[~val], n_pca=64, hidden=128, epochs=40, batch=512, seed=seed,
                               return_log=True)
    t_fit = time.perf_counter() - t0
    rmse = float(np.sqrt(np.mean((tg.screen.predict(ctx, w, qs[val]) - es[val]) ** 2)))
    # screened chain from the same start on the plain leg's proposals (second deviate added)
    atoms, disp, u1 = tg.synth.mc_proposals(MC_ATOMS, n_prop + 256, MC_RADIUS, seed=seed + 1)
    u = np.stack([u1, np.random.default_rng(seed + 9).random(len(u1))], axis=1)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + MC_SKIN)
    mc = tg.MC(ctx, system, [model], MC_T, precision=tg.TGAP_MIXED)
    mc.set_screen(w)
    mc.run(atoms[:256], disp[:256], u[:256], logs=False)
    torch.cuda.synchronize()
    s0 = mc.screen_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    # no per-proposal logs, as in the plain leg; the screen's decisions come from its counters
    r = mc.run(atoms[256:], disp[256:], u[256:], logs=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st = mc.state()
    ss = mc.screen_stats()
    by_screen = (ss["judged"] - s0["judged"]) - (ss["passed"] - s0["passed"])  # rejected at stage 1
    out = dict(moves_per_s=n_prop / (ms * 1e-3), us_per_move=1e3 * ms / n_prop, acceptance=r["accepted"] / n_prop,
               settled_by_screen=by_screen / n_prop, exact_evaluations_per_move=1.0 - by_screen / n_prop,
               screen_validation_rmse_meV_per_atom=1e3 * rmse, screen_active_at_end=ss["active"],
               fallbacks=ss["fallbacks"], training=dict(
                   snapshots=n_snap, energies=int((~val).sum()), data_s=round(t_data, 1), fit_s=round(t_fit, 2),
                   trainer="device kernels (tgap_screen_train), 40 epochs of 512-row Adam batches",
                   train_rmse_meV_per_atom_first_last_epoch=[round(1e3 * float(np.sqrt(fit_log[0])), 4),
                                                             round(1e3 * float(np.sqrt(fit_log[-1])), 4)]),
               energy_mean_meV_per_atom=1e3 * st["e_total"] / MC_ATOMS,
               plain_energy_mean_meV_per_atom=1e3 * plain["e_total"] / MC_ATOMS,
               rdf_l1_vs_plain=float(np.abs(_rdf(st["positions"], box) - _rdf(plain["positions"], box)).mean()))
    mc.close()
    system.close()
    return out


def _mc_cpu_baseline(tg, model_np, seed, budget_s=10.0):
    """The reference's MC semantics on the host cores: every proposal re-evaluates the whole
    1000-atom box with the FP64 oracle restatement (calculate_mc_step -> full calculate_gap_soap)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as orc
    hyp = tg.synth.carbon_hypers()
    H = orc.Hypers(hyp)
    pos, box, sp, _ = tg.synth.random_packing(MC_ATOMS, MC_DENSITY, 1.2, seed=seed)
    atoms, disp, u = tg.synth.mc_proposals(MC_ATOMS, 100000, MC_RADIUS, seed=seed + 1)
    kb = float(np.float32(8.617333262e-5))

    def energy(x):
        nb = orc.build_neighbors(x, MC_ATOMS, *box, 3.7, sp, False)
        e, _, _ = orc.get_gap_soap(H, MC_ATOMS, nb, sp, 0, model_np["alphas"], model_np["Qs"], model_np["delta"],
                                   model_np["zeta"], False)
        return e.sum()

    x = pos.copy()
    e_cur = energy(x)
    t0 = time.perf_counter()
    k = 0
    while time.perf_counter() - t0 < budget_s:
        y = x.copy()
        y[atoms[k]] += disp[k]
        e_new = energy(y)
        if min(1.0, np.exp(-(e_new - e_cur) / (kb * MC_T))) > u[k]:
            x, e_cur = y, e_new
        k += 1
    secs = time.perf_counter() - t0
    return dict(value=k / secs, unit="moves/s", cores=orc.num_threads(), kind="port",
                sample=f"{k} proposals on the 1000-atom box, full FP64 re-evaluation per proposal as the "
                       f"reference does (oracle restatement with OpenMP; not TurboGAP itself)")


# ----------------------------------------------------------------------------- the other workloads

CFG0_WORKLOAD = ("predict single point: 216-atom carbon, 3x3x3 cubic diamond (a = 3.567 A) with uniform +-0.15 A "
                 "noise per axis; SOAP poly3 n_max = l_max = 8, rcut 3.7/3.2 A, sigma 0.5 A; GAP zeta = 4, delta = 1 eV, "
                 "1000 sparse points from 10 further perturbed supercells, alphas ~ N(0, 1e-6), e0 = 0; energies, "
                 "forces, virial; neighbor build included")
CFG2_WORKLOAD = ("batched single points: 512 periodic carbon cells, atoms log-uniform in [32, 2048], densities uniform "
                 "in [1.5, 3.5] g/cm3, 1.1 A minimum distance, triclinic strain up to 5 %; SOAP n_max = l_max = 8, "
                 "rcut 3.7/3.2; GAP 2000 sparse, zeta = 4; one flat launch per kernel over all cells (persistent "
                 "work-queue descriptor kernels); neighbor build included")
CFG3_WORKLOAD = ("two-species scale MD: 32,768-atom amorphous SiO2 (Si:O = 1:2) at 2.2 g/cm3, minimum distances Si-O 1.4, "
                 "O-O 2.2, Si-Si 2.5 A; species-resolved SOAP n_max 8 + 8, l_max 6, rcut 5.0/4.5 A (952 components); "
                 "one GAP per centre species with 4,000 sparse points from 3 further 4096-atom boxes, zeta = 4; NVE "
                 "velocity Verlet dt = 0.5 fs from Maxwell-Boltzmann velocities at 300 K, list rebuilt every 10 steps "
                 "with a 0.3 A skin; 200 timed steps")
SIO2_DMIN = {("Si", "O"): 1.4, ("O", "O"): 2.2, ("Si", "Si"): 2.5}
SIO2_FRAC = {"Si": 1 / 3, "O": 2 / 3}


def _device_descriptors(tg, torch, ctx, hyp, structs, central_species=0):
    """FP64 descriptors of the given centre species over seeded structures, on the device."""
    import ctypes as C
    from turbogap_b200 import native
    dummy = tg.Model(ctx, hyp, np.zeros((1, tg.synth.soap_dim(hyp))), np.zeros(1), central_species=central_species)
    out = []
    for p, b, s in structs:
        sysp = tg.System(ctx, [(p, b, s)], max(hyp["rcut_hard"]))
        q = torch.zeros((len(s), dummy.dim), dtype=torch.float64, device="cuda")
        nr = C.c_int(0)
        torch.cuda.synchronize()
        native.check(native.lib().tgap_descriptors(ctx.h, sysp.h, dummy.h, 0, C.c_void_p(q.data_ptr()), C.byref(nr)),
                     ctx.h, "descriptors")
        ctx.synchronize()
        out.append(q[:nr.value].cpu().numpy())
        sysp.close()
    dummy.close()
    return np.concatenate(out)


def _single_points(tg, torch, ctx, stream, flush, system, models, reps):
    """Single-point evaluations (neighbor rebuild + energies, forces, virials) in both precisions,
    CUDA events around each one, L2 flushed before each; mixed vs FP64 RMSE of the last ones."""
    n, nst = system.n_atoms, system.n_structures
    res, outs = {}, {}
    for name, prec in (("mixed", tg.TGAP_MIXED), ("fp64", tg.TGAP_FP64)):
        e = torch.zeros(n, dtype=torch.float64, device="cuda")
        f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
        v = torch.zeros(9 * nst, dtype=torch.float64, device="cuda")
        with torch.cuda.stream(stream):
            for _ in range(2):
                system.update(True)
                system.compute_device(models, prec, e.data_ptr(), f.data_ptr(), v.data_ptr())
            ctx.synchronize()
            ms = 0.0
            for _ in range(reps):
                flush.flush()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                system.update(True)
                system.compute_device(models, prec, e.data_ptr(), f.data_ptr(), v.data_ptr())
                s1.record(stream)
                stream.synchronize()
                ms += s0.elapsed_time(s1)
        res[name] = dict(atom_evals_per_s=n * reps / (ms * 1e-3), ms_per_eval=ms / reps, evaluations=reps)
        outs[name] = (e.cpu().numpy(), f.cpu().numpy())
    res["speedup_mixed_vs_fp64"] = res["mixed"]["atom_evals_per_s"] / res["fp64"]["atom_evals_per_s"]
    res["accuracy_vs_fp64"] = dict(
        energy_rmse_meV_per_atom=1e3 * float(np.sqrt(np.mean((outs["mixed"][0] - outs["fp64"][0]) ** 2))),
        force_rmse_meV_per_A=1e3 * float(np.sqrt(np.mean((outs["mixed"][1] - outs["fp64"][1]) ** 2))))
    return res


def _oracle_single_points(tg, hyp, models_np, structs, budget_s):
    """The oracle (FP64, OpenMP) over the structures in order until the budget is spent:
    neighbor build + get_gap_soap with forces per structure, as a predict run does."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers
    import oracle_lib as orc
    atoms, k = 0, 0
    t0 = time.perf_counter()
    while k < len(structs) and (k == 0 or time.perf_counter() - t0 < budget_s):
        pos, box, sp = structs[k]
        helpers.oracle_structure_eval(hyp, models_np, pos, box, sp)
        atoms += len(pos)
        k += 1
    secs = time.perf_counter() - t0
    return atoms / secs, k, atoms, orc.num_threads()


def _in_cutoff_pairs(ctx, structs, rcut):
    """Pairs inside rcut (self excluded) of cells at least 2 rcut wide, from the library's own list."""
    n = 0
    for pos, box, sp in structs:
        nb = ctx.build_neighbors_list(pos, len(pos), *box, rcut, sp)
        n += int(np.sum(nb["n_neigh"])) - len(pos)
    return n


def _md_run_drift(tg, torch, ctx, stream, system, models, masses, vel, dt, precision, warmup, steps):
    """`steps` NVE steps after `warmup` ones, timed as one CUDA-event region (step graphs); the
    total-energy drift over those steps per atom."""
    md = tg.MD(ctx, system, models, masses, dt, rebuild_every=REBUILD, precision=precision, use_graph=True)
    md.set_velocities(vel)
    with torch.cuda.stream(stream):
        md.run(warmup)
        st0 = md.state()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        md.run(steps)
        s1.record(stream)
        stream.synchronize()
    st1 = md.state()
    md.close()
    drift = ((st1["e_pot"] + st1["e_kin"]) - (st0["e_pot"] + st0["e_kin"])) / system.n_atoms
    return s0.elapsed_time(s1), drift


def _cfg0_leg(tg, torch, ctx, stream, flush, peaks, with_cpu):
    hyp = tg.synth.carbon_hypers()
    pool = _device_descriptors(tg, torch, ctx, hyp, [tg.synth.diamond_supercell(3, seed=5000 + k) for k in range(10)])
    m = tg.synth.gap_model(pool, 1000, seed=21)
    pos, box, sp = tg.synth.diamond_supercell(3, a0=3.567, noise=0.15, seed=20)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, [(pos, box, sp)], 3.7)
    out = dict(workload=CFG0_WORKLOAD, unit="atom-evals/s", n_atoms=len(pos), n_sparse=1000)
    out.update(_single_points(tg, torch, ctx, stream, flush, system, [model], 50))
    # the list is built at the model cutoff: every pair but the self slots is inside it
    W = _work(len(pos), tg.synth.soap_dim(hyp), 1000, system.n_pairs, system.n_pairs - len(pos), 8, 8)
    out["roofline"] = _roofline(_eval_stage_profile(tg, torch, ctx, system, [model], tg.TGAP_MIXED, 20), 20, W, peaks)
    if with_cpu:
        v, k, a, cores = _oracle_single_points(tg, hyp, [m], [(pos, box, sp)] * 50, 5.0)
        out["cpu_baseline"] = dict(value=v, unit="atom-evals/s", cores=cores, kind="port",
                                   sample=f"{k} single points of the 216-atom box (oracle restatement, not TurboGAP)")
    system.close()
    model.close()
    return out


def _cfg2_leg(tg, torch, ctx, stream, flush, peaks, with_cpu):
    hyp = tg.synth.carbon_hypers()
    rng = np.random.default_rng(2024)
    sizes = np.exp(rng.uniform(np.log(32), np.log(2048), 512)).astype(int)
    dens = rng.uniform(1.5, 3.5, 512)
    structs = [tg.synth.random_packing(int(n), float(d), 1.1, seed=3000 + k, strain=0.05)[:3]
               for k, (n, d) in enumerate(zip(sizes, dens))]
    further = [tg.synth.random_packing(int(n), float(d), 1.1, seed=9000 + k, strain=0.05)[:3]
               for k, (n, d) in enumerate(zip(sizes[:16], dens[:16]))]
    m = tg.synth.gap_model(_device_descriptors(tg, torch, ctx, hyp, further), 2000, seed=9)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], 1.0, 4.0)
    system = tg.System(ctx, structs, 3.7)
    n = system.n_atoms
    out = dict(workload=CFG2_WORKLOAD, unit="atom-evals/s", n_structures=512, n_atoms=n, n_sparse=2000,
               pairs_in_list=system.n_pairs)
    out.update(_single_points(tg, torch, ctx, stream, flush, system, [model], 5))
    W = _work(n, tg.synth.soap_dim(hyp), 2000, system.n_pairs, system.n_pairs - n, 8, 8)
    out["roofline"] = _roofline(_eval_stage_profile(tg, torch, ctx, system, [model], tg.TGAP_MIXED, 3), 3, W, peaks)
    if with_cpu:
        v, k, a, cores = _oracle_single_points(tg, hyp, [m], structs, 10.0)
        out["cpu_baseline"] = dict(value=v, unit="atom-evals/s", cores=cores, kind="port",
                                   sample=f"the first {k} of the 512 cells ({a} atoms), one single point each "
                                          f"(oracle restatement, not TurboGAP)")
    system.close()
    model.close()
    return out


def _cfg3_leg(tg, torch, ctx, stream, peaks, with_cpu, warmup):
    hyp = tg.synth.sio2_hypers()
    pos, box, sp, masses = tg.synth.random_packing(32768, 2.2, SIO2_DMIN, SIO2_FRAC, seed=3)
    n = len(pos)
    further = [tg.synth.random_packing(4096, 2.2, SIO2_DMIN, SIO2_FRAC, seed=600 + k)[:3] for k in range(3)]
    mods_np, mods = [], []
    for cs, seed in ((1, 61), (2, 62)):
        mm = tg.synth.gap_model(_device_descriptors(tg, torch, ctx, hyp, further, cs), 4000, seed=seed)
        mm["central_species"] = cs
        mods_np.append(mm)
        mods.append(tg.Model(ctx, hyp, mm["Qs"], mm["alphas"], 1.0, 4.0, central_species=cs))
    system = tg.System(ctx, [(pos, box, sp)], 5.0 + SKIN)
    vel = tg.synth.maxwell_boltzmann(masses, 300.0, seed=4)
    out = dict(workload=CFG3_WORKLOAD, unit="atom-steps/s", n_atoms=n, n_sparse=[4000, 4000],
               pairs_in_list=system.n_pairs, l2="inputs larger than L2 (descriptor rows alone exceed 250 MB)")
    steps = 200
    for name, prec in (("mixed", tg.TGAP_MIXED), ("fp64", tg.TGAP_FP64)):
        system.set_positions(pos)
        system.update(True)
        ms, drift = _md_run_drift(tg, torch, ctx, stream, system, mods, masses, vel, 0.5, prec, warmup, steps)
        out[name] = dict(atom_steps_per_s=n * steps / (ms * 1e-3), ms_per_step=ms / steps, steps=steps,
                         energy_drift_meV_per_atom=1e3 * drift)
    out["speedup_mixed_vs_fp64"] = out["mixed"]["atom_steps_per_s"] / out["fp64"]["atom_steps_per_s"]
    system.set_positions(pos)
    system.update(True)
    e64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    f64 = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v64 = torch.zeros(9, dtype=torch.float64, device="cuda")
    e32, f32, v32 = torch.zeros_like(e64), torch.zeros_like(f64), torch.zeros_like(v64)
    torch.cuda.synchronize()
    system.compute_device(mods, tg.TGAP_FP64, e64.data_ptr(), f64.data_ptr(), v64.data_ptr())
    system.compute_device(mods, tg.TGAP_MIXED, e32.data_ptr(), f32.data_ptr(), v32.data_ptr())
    ctx.synchronize()
    out["accuracy_vs_fp64"] = dict(
        energy_rmse_meV_per_atom=1e3 * float(torch.sqrt(torch.mean((e32 - e64) ** 2))),
        force_rmse_meV_per_A=1e3 * float(torch.sqrt(torch.mean((f32 - f64) ** 2))),
        virial_max_abs_diff_eV=float(torch.max(torch.abs(v32 - v64))))
    W = _work(n, tg.synth.soap_dim(hyp), 4000, system.n_pairs, _in_cutoff_pairs(ctx, [(pos, box, sp)], 5.0), 8, 6,
              n_models=2)
    out["roofline"] = _roofline(_eval_stage_profile(tg, torch, ctx, system, mods, tg.TGAP_MIXED, 3), 3, W, peaks)
    if with_cpu:
        sample = tg.synth.random_packing(1536, 2.2, SIO2_DMIN, SIO2_FRAC, seed=65)[:3]
        v, k, a, cores = _oracle_single_points(tg, hyp, mods_np, [sample], 0.0)
        out["cpu_baseline"] = dict(value=v, unit="atom-steps/s", cores=cores, kind="port",
                                   sample="one force evaluation (neighbor build + both models) of a 1536-atom box "
                                          "of the same composition, density, descriptor and models (the per-atom "
                                          "cost of the 32,768-atom box, whose materialised dq/dr would take 27 GB); "
                                          "oracle restatement, not TurboGAP")
    system.close()
    for m in mods:
        m.close()
    return out


def _sharded_leg(tg, torch, ctx, model, dist, world, rank, steps, warmup):
    """Atom decomposition across the ranks (N > 1): one box of 4096 N carbon atoms at the MD
    workload's density, split_tasks over the ranks, one all-reduce of forces, energies and virial
    per step (NCCL), the same velocity Verlet on every rank. Per-GPU work is fixed as N grows
    (weak scaling of the decomposition); device time per step, max over ranks."""
    from turbogap_b200 import decomposition as dc
    n = N_ATOMS * world
    pos, box, sp, masses = tg.synth.random_packing(n, 2.5, 1.2, seed=4242)
    vel = tg.synth.maxwell_boltzmann(masses, 3000.0, seed=4243)
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + SKIN)
    sh = dc.ShardedMD(ctx, system, [model], masses, DT, rebuild_every=REBUILD, precision=tg.TGAP_MIXED, dist=dist)
    sh.set_velocities(vel)
    sh.run(warmup)
    dist.barrier()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    sh.run(steps)
    s1.record()
    torch.cuda.synchronize()
    ms = _over_ranks([s0.elapsed_time(s1)], "max", dist, "cuda")[0]
    st = sh.state()
    system.close()
    return dict(workload=f"NVE MD of one {n}-atom carbon box (2.5 g/cm3, same model and settings as the headline), "
                         f"sites split over {world} ranks (split_tasks), one NCCL all-reduce of forces, energies "
                         f"and virial per step", n_atoms=n, sites_per_rank=sh.range[1] - sh.range[0], steps=steps,
                atom_steps_per_s=n * steps / (ms * 1e-3), ms_per_step=ms / steps, scaling="weak",
                e_pot_per_atom=st["e_pot"] / n)


def _over_ranks(values, op, dist, device):
    """Max or min of per-rank values over the process group (identity without one): each rank
    runs its own replica, and the job is as slow as its slowest rank."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.MIN)
    return [float(v) for v in t.cpu()]


def _job_throughput(world, units_per_rank, ms_max):
    """Whole-job units per second: every rank processed units_per_rank in at most ms_max."""
    return world * units_per_rank / (ms_max * 1e-3)


def run_ours(args):
    import torch
    tg = _load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    seed = 17 * rank
    pos, box, sp, masses, vel = _workload(tg, seed)
    ctx = tg.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    hyp = tg.synth.carbon_hypers()
    # sparse set: descriptors of 10 further seeded boxes, computed on the device (FP64)
    pool = _device_descriptors(tg, torch, ctx, hyp, _pool_structures(tg, 1000 + seed))
    model_np = tg.synth.gap_model(pool, N_SPARSE, seed=7)
    model = tg.Model(ctx, hyp, model_np["Qs"], model_np["alphas"], model_np["delta"], model_np["zeta"])
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + SKIN)
    flush = L2Flush(torch)
    peaks = _peaks()
    peaks["fp64"] = _fp64_peak(torch)
    # launch shapes picked by the autotuner on this system, both precisions (before any graph)
    tuning = system.autotune([model], tg.TGAP_MIXED, reps=5) + system.autotune([model], tg.TGAP_FP64, reps=3)

    # accuracy: single point, mixed vs FP64
    e64 = torch.zeros(N_ATOMS, dtype=torch.float64, device="cuda")
    f64 = torch.zeros(3 * N_ATOMS, dtype=torch.float64, device="cuda")
    v64 = torch.zeros(9, dtype=torch.float64, device="cuda")
    e32, f32, v32 = torch.zeros_like(e64), torch.zeros_like(f64), torch.zeros_like(v64)
    torch.cuda.synchronize()
    system.compute_device([model], tg.TGAP_FP64, e64.data_ptr(), f64.data_ptr(), v64.data_ptr())
    system.compute_device([model], tg.TGAP_MIXED, e32.data_ptr(), f32.data_ptr(), v32.data_ptr())
    ctx.synchronize()
    e_rmse = float(torch.sqrt(torch.mean((e32 - e64) ** 2)))
    f_rmse = float(torch.sqrt(torch.mean((f32 - f64) ** 2)))
    n_pairs = system.n_pairs
    # in-cutoff pairs (r < 3.7 A, self excluded) of the starting box, from the library's own list
    n_cut = _in_cutoff_pairs(ctx, [(pos, box, sp)], 3.7)

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms64, _, _, _ = _timed_md(tg, torch, ctx, stream, flush, system, model, masses, vel, tg.TGAP_FP64,
                              args.steps, args.warmup)
    system.set_positions(pos)
    system.update(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ms, launches, st0, st1 = _timed_md(tg, torch, ctx, stream, flush, system, model, masses, vel, tg.TGAP_MIXED,
                                       args.steps, args.warmup)
    clk = clocks.stop()
    torch.cuda.synchronize()
    ms, ms64 = _over_ranks([ms, ms64], "max", dist, "cuda")
    drift = ((st1["e_pot"] + st1["e_kin"]) - (st0["e_pot"] + st0["e_kin"])) / N_ATOMS
    value = _job_throughput(world, N_ATOMS * args.steps, ms)
    value64 = _job_throughput(world, N_ATOMS * args.steps, ms64)

    # per-kernel times and roofline of the dominant kernel, both precisions
    W = _work(N_ATOMS, tg.synth.soap_dim(hyp), N_SPARSE, n_pairs, n_cut, 8, 8)
    system.set_positions(pos)
    system.update(True)
    stages = _stage_profile(tg, ctx, system, [model], masses, vel, tg.TGAP_MIXED)
    roof = _roofline(stages, 20, W, peaks, traffic=True)
    system.set_positions(pos)
    system.update(True)
    stages64 = _stage_profile(tg, ctx, system, [model], masses, vel, tg.TGAP_FP64, steps=10)
    roof64 = _roofline(stages64, 10, W, peaks)
    # energy conservation over the workload's full 1,000 steps (untimed), both precisions
    long_drift = {}
    for name, prec in (("mixed", tg.TGAP_MIXED), ("fp64", tg.TGAP_FP64)):
        system.set_positions(pos)
        system.update(True)
        ms_l, d_l = _md_run_drift(tg, torch, ctx, stream, system, [model], masses, vel, DT, prec, 1, 1000)
        long_drift[name] = dict(steps=1000, energy_drift_meV_per_atom=1e3 * d_l, ms_per_step=ms_l / 1000)
    system.set_positions(pos)
    system.update(True)
    e2e = _e2e(tg, ctx, system, model, masses, vel, pos, tg.TGAP_MIXED, min(args.steps, 50))
    e2e["value"] = _over_ranks([e2e["value"]], "min", dist, "cuda")[0] * world
    system.set_positions(pos)
    system.update(True)
    e2e64 = _e2e(tg, ctx, system, model, masses, vel, pos, tg.TGAP_FP64, min(args.steps, 20))
    e2e64["value"] = _over_ranks([e2e64["value"]], "min", dist, "cuda")[0] * world
    mc_line = _mc_leg(tg, torch, ctx, stream, model, MC_PROPOSALS, 300 + seed)
    with_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    cpu = None
    if with_cpu:
        cpu = _cpu_baseline(tg, pos, box, sp, masses, vel, model_np)
        mc_line["cpu_baseline"] = _mc_cpu_baseline(tg, model_np, 300 + seed)
    legs = {}
    if world > 1:
        legs["sharded_md"] = _sharded_leg(tg, torch, ctx, model, dist, world, rank, args.steps, args.warmup)
    if world == 1 and not args.headline_only:
        legs["predict_216"] = _cfg0_leg(tg, torch, ctx, stream, flush, peaks, with_cpu)
        legs["batched_512_cells"] = _cfg2_leg(tg, torch, ctx, stream, flush, peaks, with_cpu)
        legs["sio2_32768_md"] = _cfg3_leg(tg, torch, ctx, stream, peaks, with_cpu, args.warmup)
    if rank == 0:
        cfg = _md_config(n_pairs)
        cfg["parallelism"] = f"replicas x{world}" if world > 1 else "single GPU"
        line = {
            "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 descriptor + bf16x3 tensor-core GEMM, f64 accumulation",
            "data": "synthetic (seeded random packing, synthetic GAP model)",
            "config": cfg,
            "plain_fp64": {"value": value64, "unit": "atom-steps/s", "ms_per_step": ms64 / args.steps,
                           "roofline": roof64, "e2e": e2e64,
                           "stages_us_per_step": {k: v["total_ms"] * 1e3 / 10 for k, v in stages64.items()}},
            "speedup_mixed_vs_fp64": value / value64,
            "accuracy_vs_fp64": {"energy_rmse_meV_per_atom": 1e3 * e_rmse, "force_rmse_meV_per_A": 1e3 * f_rmse},
            "energy_drift_meV_per_atom": 1e3 * drift,
            "energy_drift_1000_steps": long_drift,
            "roofline": roof,
            "stages_us_per_step": {k: v["total_ms"] * 1e3 / 20 for k, v in stages.items()},
            "autotune": tuning,
            "cpu_baseline": cpu,
            "mc": mc_line,
            "workloads": legs,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "peaks": {k: peaks[k] for k in ("hbm", "bf16", "bf16_sus", "fp64", "src")},
        }
        print(json.dumps(line), flush=True)
    model.close()
    system.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_profile(args):
    """The MD workload only (no other legs, no CPU baseline): warm-up, then `steps` eager MD steps in
    one precision, for profiler captures of its kernels."""
    import torch
    tg = _load_package()
    torch.cuda.set_device(0)
    pos, box, sp, masses, vel = _workload(tg, 0)
    ctx = tg.Context(0)
    hyp = tg.synth.carbon_hypers()
    pool = _device_descriptors(tg, torch, ctx, hyp, _pool_structures(tg, 1000))
    m = tg.synth.gap_model(pool, N_SPARSE, seed=7)
    model = tg.Model(ctx, hyp, m["Qs"], m["alphas"], m["delta"], m["zeta"])
    system = tg.System(ctx, [(pos, box, sp)], 3.7 + SKIN)
    prec = tg.TGAP_FP64 if args.profile == "fp64" else tg.TGAP_MIXED
    md = tg.MD(ctx, system, [model], masses, DT, rebuild_every=REBUILD, precision=prec, use_graph=False)
    md.set_velocities(vel)
    md.run(args.warmup)
    ctx.synchronize()
    l0 = ctx.kernel_launches
    md.run(args.steps)
    ctx.synchronize()
    st = md.state()
    print(json.dumps({"profile": args.profile, "steps": args.steps, "warmup": args.warmup,
                      "launches": ctx.kernel_launches - l0, "e_pot": st["e_pot"]}), flush=True)
    md.close()
    system.close()
    model.close()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true", help="skip the predict, batched and SiO2 legs")
    ap.add_argument("--profile", choices=["mixed", "fp64"], default=None,
                    help="only the MD workload's steps in one precision (for profiler captures)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

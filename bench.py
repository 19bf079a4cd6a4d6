"""Benchmark of the LGA docking hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--lsmet ad|sw|adam|fire]

Workload (the plain per-ligand configuration): one synthetic receptor
(60^3 grid points at 0.375 A; C, A, N, OA, HD, e and d maps) and one seeded
ligand of 40 heavy atoms with 10 torsions, nrun 100, population 150,
2.5M evaluations per run.  One step = one complete docking of that ligand
(initial population, then generations of GA + local search until the mean
evaluations per run reach 2.5M), through the reference kernel API
(libadgpu_b200).  The metric is score evaluations per second, counted the
way the reference counts them (per-run eval counters), plus ligands/hour.

With N > 1 (torchrun), every rank docks its own ligand on its own GPU: the
ligands are independent, there is no data-path collective (replicas), and
`value` is all ranks' evaluations over the slowest rank's time.

--impl reference times the reference's algorithm on the host cores: the C
restatement of the reference kernels (oracle/, one pose per thread, all
host threads), on inputs prepared by the reference's own front end
(oracle/_ref), one complete generation of the same docking per step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "autodock-gpu_b200")]

import numpy as np  # noqa: E402

WORKLOAD = dict(npts=60, types=["C", "A", "N", "OA", "HD"], n_heavy=40, n_tors=10, nrun=100, pop=150,
                nev=2_500_000, config_id=2, seed=(305419896, 2271560481, 3735928559))
METRIC = "score-evals/s"
UNIT = "evals/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def build_inputs(lsmet: str, rank: int = 0):
    """Seeded synthetic receptor + ligand, prepared by the engine's front end."""
    from adgpu_b200 import frontend, synth
    w = WORKLOAD
    spec = synth.grid_spec(w["npts"], w["types"], seed=12345 + w["config_id"])
    maps = synth.quantize_maps(synth.make_maps(spec))
    grid = frontend.Grid.from_maps(maps, w["types"], spec.spacing, spec.origin)
    mol = synth.ligand_for(w["config_id"], rank, w["n_heavy"], w["n_tors"])
    lines, _ = synth.pdbqt_lines(mol)
    text = "\n".join(lines) + "\n"
    run = frontend.default_dockpars(grid.spacing, w["pop"])
    lig = frontend.Ligand(grid, text, None, run=run, seed=w["seed"], num_runs=w["nrun"])
    return grid, lig


def cost_model(lig):
    """Algorithmic FLOPs per evaluation from the prepared tables:
    40*R_rot + 200*N_i + 80*Q + 25*S_tors + 30*N (energy+gradient) and
    40*R_rot + 100*N_i + 45*Q (energy only); bytes = 96*N_i (3 maps x 8 corners x 4 B)."""
    from adgpu_b200 import abi
    dp = lig.dockpars
    N, Q = dp.num_of_atoms, dp.num_of_intraE_contributors
    ii = np.frombuffer(bytes(lig.tables["interintra"]), np.uint8)
    n_i = int((ii[3072:3072 + N] == 0).sum())
    rl = np.frombuffer(bytes(lig.tables["rotlist"]), np.int32)[:dp.rotbondlist_length]
    r_rot = int(((rl & abi.RLIST_DUMMY_MASK) == 0).sum())
    gr = abi.KcGrads.from_buffer_copy(bytes(lig.tables["grads"]))
    s_tors = int(sum(gr.num_rotating_atoms_per_rotbond[:dp.num_of_genes - 6]))
    grad = 40 * r_rot + 200 * n_i + 80 * Q + 25 * s_tors + 30 * N
    energy = 40 * r_rot + 100 * n_i + 45 * Q
    return dict(N=N, N_i=n_i, Q=Q, R_rot=r_rot, S_tors=s_tors, flop_grad=grad, flop_energy=energy, bytes=96 * n_i)


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region, in
    process through NVML every 0.3 s.  (An `nvidia-smi -lms 200` child
    process sampling the same fields slowed the timed dockings by about 10 %
    on this workload; NVML queries from a thread of this process do not
    measurably.)  Falls back to nvidia-smi when NVML is unavailable."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index: int, interval: float = 0.3):
        self.index = index
        self.interval = interval
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []
        self.running = False

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = None
            try:        # the CUDA device's own GPU, whatever CUDA_VISIBLE_DEVICES maps it to
                import torch
                uuid = str(torch.cuda.get_device_properties(self.index).uuid)
                self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.smax = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.running = True

            def loop():
                while self.running:
                    try:
                        self.samples.append((pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM),
                                             int(reasons(self.h))))
                    except Exception:
                        pass
                    time.sleep(self.interval)
            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.running = False
            self.t.join()
            sm = [float(c) for c, _ in self.samples]
            reasons = sorted({n for _, bits in self.samples for n, b in self.REASON_BITS.items() if bits & b})
            load = [x for x in sm if x > 0.5 * self.smax] or sm
            return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": float(self.smax),
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        load = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


# ---------------------------------------------------------------------------
# CPU side: the oracle (C restatement of the reference kernels, one pose per
# host thread) on inputs prepared by the reference's own front end
# (oracle/_ref), so that neither this repository's library nor its front end
# is on that path.
# ---------------------------------------------------------------------------
def _reference_inputs(config_id: int, npts: int, n_heavy: int, n_tors: int, nrun: int, lsmet: str):
    """Writes the seeded synthetic maps and ligand as .fld/.map/.pdbqt files and
    prepares them with the reference's own front end (oracle/_ref)."""
    import tempfile
    from adgpu_b200 import synth          # numpy only: no library is loaded
    from oracle import oraclepy, refpy
    w = WORKLOAD
    d = tempfile.mkdtemp(prefix=f"adgpu_ref{config_id}_")
    spec = synth.grid_spec(npts, w["types"], seed=12345 + config_id)
    fld = synth.write_maps(spec, synth.make_maps(spec), d)
    lig_path = os.path.join(d, "ligand.pdbqt")
    synth.write_ligand(synth.ligand_for(config_id, 0, n_heavy, n_tors), lig_path)
    job = refpy.RefJob(["--ffile", fld, "--lfile", lig_path, "--nrun", str(nrun), "--seed",
                        ",".join(str(s) for s in w["seed"]), "--lsmet", lsmet, "--heuristics", "0", "--autostop", "0",
                        "--nev", str(w["nev"]), "--psize", str(w["pop"])])
    ht = oraclepy.tables_from_refjob(job)
    return job, ht


class OracleDocking:
    """docking_with_gpu's generation loop (host/src/performdocking.cpp.Cuda:
    684-831) over the oracle's kernels on the host cores."""

    LS = {"ad": "gradient_minad", "sw": "perform_ls", "adam": "gradient_minadam", "fire": "gradient_minfire"}

    def __init__(self, job, ht, lsmet: str, nthreads: int):
        from adgpu_b200 import abi
        self.ht, self.lsmet, self.nt = ht, lsmet, nthreads
        dp = ht.dockpars
        self.R, self.P, self.L = job.info.num_of_runs, dp.pop_size, dp.num_of_lsentities
        n = self.R * self.P
        self.prng = job.blob("prng").copy()
        self.en = np.zeros(n, np.int32)
        self.er = np.zeros(self.R, np.int32)
        ht.bind_state(self.prng, self.en, self.er)
        self.cur = job.blob("initpop").reshape(-1, abi.GENOTYPE_STRIDE)[:n].copy()
        self.ecur = np.zeros(n, np.float32)
        self.nxt, self.enxt = np.zeros_like(self.cur), np.zeros_like(self.ecur)
        ht.call("calc_initpop", n, self.cur, self.ecur, nthreads)
        ht.call("sum_evals", self.R)
        self.generations = 0

    def evals(self) -> int:
        return int(self.er.sum())

    def generation(self):
        T = 64
        self.ht.call("gen_and_eval_newpops", self.R * self.P, T, self.cur, self.ecur, self.nxt, self.enxt, self.nt)
        self.ht.call(self.LS[self.lsmet], self.R * self.L, T, self.nxt, self.enxt, self.nt)
        self.ht.call("sum_evals", self.R)
        self.cur, self.nxt, self.ecur, self.enxt = self.nxt, self.cur, self.enxt, self.ecur
        self.generations += 1

    def run(self, nev: int, ngen: int = 42000):
        """Until the mean evaluations per run reach nev (check_progress, :908-942)."""
        while max(self.evals() / self.R / nev, self.generations / ngen) < 1.0:
            self.generation()


def cpu_baseline(lsmet: str, budget_s: float = 12.0):
    """The workload's docking on the host cores (the oracle): complete
    generations of the plain docking from its initial population for about
    budget_s, plus one complete docking of the small CPU-runnable
    configuration (40^3 maps, 16 heavy atoms / 4 torsions, nrun 10, 2.5M
    evaluations per run)."""
    w = WORKLOAD
    nthreads = os.cpu_count() or 1
    job, ht = _reference_inputs(w["config_id"], w["npts"], w["n_heavy"], w["n_tors"], w["nrun"], lsmet)
    od = OracleDocking(job, ht, lsmet, nthreads)
    e0, t0 = od.evals(), time.perf_counter()
    while time.perf_counter() - t0 < budget_s or od.generations < 1:
        od.generation()
    dt = time.perf_counter() - t0
    v = (od.evals() - e0) / dt
    job1, ht1 = _reference_inputs(1, 40, 16, 4, 10, lsmet)
    d1 = OracleDocking(job1, ht1, lsmet, nthreads)
    t1 = time.perf_counter()
    d1.run(w["nev"])
    s1 = time.perf_counter() - t1
    return {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{od.generations} complete generations (GA + {lsmet} local search + eval sums, 100 runs x 150) "
                      f"of the workload's docking from its initial population ({od.evals() - e0} evals, {dt:.1f} s), "
                      f"inputs prepared by the reference's own front end, on {nthreads} host threads",
            "cfg1_full_docking": {"workload": "40^3 maps, 16 heavy atoms / 4 torsions, nrun 10, pop 150, nev 2.5M, "
                                              f"lsmet {lsmet}", "seconds": s1, "generations": d1.generations,
                                  "evals_per_s": d1.evals() / s1, "ligands_per_hour": 3600.0 / s1}}


def run_reference(args, rank, world):
    """--impl reference: the reference's algorithm (the oracle, a C
    restatement of its kernels; inputs from its own front end) on the host
    cores.  A step is one complete generation of the workload's docking (GA,
    local search and eval sums over all 100 runs), continuing from the
    previous step; value = evaluations / second over the timed steps."""
    if rank != 0:
        return None
    w = WORKLOAD
    nthreads = os.cpu_count() or 1
    job, ht = _reference_inputs(w["config_id"], w["npts"], w["n_heavy"], w["n_tors"], w["nrun"], args.lsmet)
    od = OracleDocking(job, ht, args.lsmet, nthreads)
    for _ in range(args.warmup):
        od.generation()
    e0, t0 = od.evals(), time.perf_counter()
    for _ in range(args.steps):
        od.generation()
    dt = time.perf_counter() - t0
    v = (od.evals() - e0) / dt
    evals_per_docking = w["nrun"] * w["nev"]
    sample = (f"generations {args.warmup + 1}-{args.warmup + args.steps} of the workload's docking ({od.evals() - e0} "
              f"evals, {dt:.1f} s), one generation per step, on {nthreads} host threads")
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(1, args.steps),
            "step": "one complete generation (GA + local search + eval sums, 100 runs x 150 entities)",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": _config(args), "ligands_per_hour": 3600.0 * v / evals_per_docking,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _config(args):
    w = WORKLOAD
    return {"workload": f"plain per-ligand docking: {w['npts']}^3 maps (5 types + e + d), ligand {w['n_heavy']} heavy "
                        f"atoms / {w['n_tors']} torsions, nrun {w['nrun']}, pop {w['pop']}, nev {w['nev']}, "
                        f"lsmet {args.lsmet}",
            "lsmet": args.lsmet, "nrun": w["nrun"], "pop_size": w["pop"], "nev_per_run": w["nev"],
            "grid_points": w["npts"] + 1, "l2": "flushed between timed steps (256 MiB write)",
            "parallelism": f"replicas x{args.gpus}"}


def rank_aggregate(seconds: float, work: float, device, world: int):
    """Whole-job figures of a replicas run: the slowest rank's timed seconds
    (max over ranks) and the work of all ranks (sum), through
    torch.distributed (NCCL on the GPUs; any backend works)."""
    if world <= 1:
        return float(seconds), float(work)
    import torch
    t = torch.tensor([float(seconds)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    w = torch.tensor([float(work)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(w, op=torch.distributed.ReduceOp.SUM)
    return float(t.item()), float(w.item())


def fp32_peak(dev) -> float:
    """Measured FP32 FMA throughput of the device (TFLOP/s), from the
    bench-only probe library (autodock-gpu_b200/csrc/probe)."""
    import ctypes as C
    import torch
    path = os.path.join(ROOT, "autodock-gpu_b200", "lib", "libadgpu_probe.so")
    L = C.CDLL(path)
    L.adgpu_probe_fp32_peak.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
    scratch = torch.empty(4096 * 1024, dtype=torch.float32, device=dev)
    peak = C.c_float(0)
    rc = L.adgpu_probe_fp32_peak(C.c_void_p(scratch.data_ptr()), scratch.numel(), C.byref(peak))
    if rc != 0:
        raise RuntimeError(f"fp32 probe failed ({rc})")
    return float(peak.value)


def _roofline_inputs():
    """DRAM traffic and issue figures per evaluation of the dominant kernel from
    the last ncu capture (profiles/roofline_inputs.json: kernel, case, date)."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "roofline_inputs.json")))
    except Exception:
        return {}


def run_engine(args, rank, world, local_rank):
    import ctypes as C
    import torch
    from adgpu_b200 import device, dock, lib
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = WORKLOAD
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def setup(lsmet):
        grid, lig = build_inputs(lsmet, rank)
        ref_grid = grid.reference_layout()
        job = device.DeviceJob(lig.tables, lig.dockpars, ref_grid, w["nrun"], lig.prng, device=dev)
        job.activate()
        bufs = (*job.population(), *job.population())
        init_dev = torch.from_numpy(lig.initpop).to(dev)
        return grid, lig, ref_grid, job, bufs, init_dev, job.prng.clone()

    def timed_dockings(job, bufs, init_dev, prng0, lsmet, steps):
        times, evals, gens, res = [], 0, 0, None
        for _ in range(steps):
            job.prng.copy_(prng0)
            flush.zero_()
            torch.cuda.synchronize()
            ev_a.record()
            res = dock.dock(job, init_dev, lsmet, w["nev"], 42000, buffers=bufs)
            ev_b.record()
            torch.cuda.synchronize()
            times.append(ev_a.elapsed_time(ev_b) / 1e3)
            evals += int(res.evals_per_run.sum())
            gens += res.generations
        return times, evals, gens, res

    grid, lig, ref_grid, job, bufs, init_dev, prng0 = setup(args.lsmet)
    timed_dockings(job, bufs, init_dev, prng0, args.lsmet, args.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    times, evals, gens, res = timed_dockings(job, bufs, init_dev, prng0, args.lsmet, args.steps)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    loop_stats = dock.last_stats()
    t_all, ev_all = rank_aggregate(sum(times), evals, dev, world)
    ev_all = int(ev_all)
    value = ev_all / t_all
    best = float(res.energies.min().item())

    # --- end to end through the public API with host buffers -------------------
    host_tables, host_pop, host_prng = lig.tables, np.ascontiguousarray(lig.initpop, np.float32), lig.prng
    h2d = ref_grid.nbytes + sum(np.asarray(t).nbytes for t in host_tables.values()) + host_pop.nbytes + host_prng.nbytes
    e2e_times, e2e_evals, d2h = [], 0, 0
    for i in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        j2 = device.DeviceJob(host_tables, lig.dockpars, ref_grid, w["nrun"], host_prng, device=dev)
        j2.activate()
        pop_dev = torch.from_numpy(host_pop).to(dev)
        r2 = dock.dock(j2, pop_dev, args.lsmet, w["nev"], 42000)
        conf_h = r2.conformations.cpu().numpy()
        en_h = r2.energies.cpu().numpy()
        e2e_times.append(time.perf_counter() - t0)
        e2e_evals += int(r2.evals_per_run.sum())
        d2h = conf_h.nbytes + en_h.nbytes + r2.evals_per_run.nbytes
        del j2
    job.activate()
    e2e_t, e2e_all = rank_aggregate(sum(e2e_times), e2e_evals, dev, world)
    e2e_value = e2e_all / e2e_t

    # --- roofline of the dominant kernel: the docking loop's persistent launch ---
    cm = cost_model(lig)
    roof = None
    if rank == 0:
        R, P = w["nrun"], w["pop"]
        c1, e1, c2, e2 = bufs
        durs, loop_evals, ga_evals = [], [], []
        for _ in range(2):
            job.prng.copy_(prng0)
            c1.copy_(init_dev[:R * P])
            job.evals_runs.zero_()
            lib.call("adgpu_calc_initpop", R * P, 64, c1, e1)
            lib.call("adgpu_sum_evals", R, 64)
            flush.zero_()
            torch.cuda.synchronize()
            fin, gn = C.c_int(0), C.c_uint32(0)
            ev_a.record()
            lib.call("adgpu_dock_resident", dock.LSMET[args.lsmet], R, w["nev"], 42000, c1, e1, c2, e2,
                     C.byref(fin), C.byref(gn))
            ev_b.record()
            torch.cuda.synchronize()
            durs.append(ev_a.elapsed_time(ev_b) / 1e3)
            loop_evals.append(int(job.evals_runs.sum().item()) - R * P)
            ga_evals.append(gn.value * R * (P - 1))         # one per new entity, none for the elite
        dur = statistics.mean(durs)
        n_loop, n_ga = statistics.mean(loop_evals), statistics.mean(ga_evals)
        flop_ls = cm["flop_grad"] if args.lsmet != "sw" else cm["flop_energy"]
        flop = (n_loop - n_ga) * flop_ls + n_ga * cm["flop_energy"]
        achieved = flop / dur / 1e12
        peak = fp32_peak(dev)
        ri = _roofline_inputs().get(args.lsmet, {})
        traffic = ri.get("dram_bytes_per_eval")
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic * n_loop if traffic else None,
                "traffic_source": (f"ncu dram__bytes_read+write per evaluation of {ri.get('kernel')} on "
                                   f"{ri.get('case')} (capture of {ri.get('date')}, profiles/roofline_inputs.json) "
                                   "x this launch's evaluations") if traffic else "no capture of this kernel",
                "peak_source": "measured in this run (FMA-chain probe, bench-only libadgpu_probe.so); "
                               "MEASURED_PEAKS.json has no FP32 figure",
                "issue_slots_active": ri.get("issue_active"), "warp_instructions_per_eval": ri.get("warp_instr_per_eval"),
                "kernel": "pipe_kernel (adgpu_dock_resident: the whole generation loop, one persistent launch)",
                "launch_ms": dur * 1e3, "evals_per_launch": n_loop, "ga_evals_per_launch": n_ga,
                "flop_per_eval": {"local_search": flop_ls, "ga": cm["flop_energy"]}, "bytes_per_eval": cm["bytes"],
                "hbm_frac_of_measured": (n_loop * cm["bytes"] / dur / 1e9) / _hbm_peak(),
                "pose_group_utilisation": dock.last_stats().get("utilisation")}

    line = None
    if rank == 0:
        evals_per_docking = w["nrun"] * w["nev"]
        gl = gens // max(1, args.steps)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_all / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": _config(args),
                "ligands_per_hour": 3600.0 * world * args.steps / t_all,
                "generations_per_docking": gl, "best_energy": best,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
                # per docking: initpop, eval sums, then the loop's init, persistent and final kernels
                "gpu_launches": int(args.steps * 5),
                "docking_loop": loop_stats,
                "clocks": clocks, "roofline": roof, "cost_model": cm}
        # the same docking with the other local search of the plain configuration (sw <-> ad)
        other = "sw" if args.lsmet != "sw" else "ad"
        _, _, _, job_o, bufs_o, init_o, prng_o = setup(other)
        timed_dockings(job_o, bufs_o, init_o, prng_o, other, 1)
        t_o, ev_o, g_o, _ = timed_dockings(job_o, bufs_o, init_o, prng_o, other, max(2, min(args.steps, 5)))
        line[f"lsmet_{other}"] = {"value": ev_o / sum(t_o), "unit": UNIT, "ms_per_step": 1e3 * sum(t_o) / len(t_o),
                                  "steps": len(t_o), "generations_per_docking": g_o // len(t_o),
                                  "ligands_per_hour": 3600.0 * len(t_o) / sum(t_o), "docking_loop": dock.last_stats()}
        del job_o, bufs_o
        line["cfg1_gpu"] = gpu_cfg1(dev)
        job.activate()
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.lsmet)
        # the single-GPU samples below run at N = 1 only (under torchrun the
        # other ranks would wait for them at the closing barrier)
        if world > 1:
            args.no_batch = args.no_serve = args.no_result = True
        if not args.no_batch:
            # the batching comparison on a bounded sample of its configuration
            bvp = run_batch(args)
            line["batched_vs_plain"] = {k: bvp[k] for k in ("ligands", "nrun", "nev_per_run", "heavy_atoms", "batched",
                                                            "plain", "batched_over_plain_ligands_per_hour", "tpp_classes",
                                                            "clocks_batched")}
        if not args.no_serve:
            # the serving loop on a shorter request stream (same settings as --mode serve)
            sargs = argparse.Namespace(**vars(args))
            sargs.nreq = 100
            sargs.process_results = True
            sv = run_serve(sargs)
            line["serving"] = {k: sv[k] for k in ("requests", "nrun", "nev_per_run", "receptors",
                                                  "batched_capacity_ligands_per_s", "arrival_rate_per_s",
                                                  "ligands_per_hour", "latency_p50_s", "latency_p90_s", "latency_p99_s",
                                                  "tick_ms", "threads_per_pose", "priority", "results_processed_on_device",
                                                  "clocks")}
        if not args.no_result:
            rr = run_result(args)
            line["result_processing"] = {k: rr[k] for k in ("workload", "gpu_ms_all_entities", "reference_host_ms",
                                                            "speedup_vs_reference", "clusters", "parity")}
        del evals_per_docking
    return line


def gpu_cfg1(dev, steps: int = 3):
    """The small CPU-runnable configuration docked on the GPU: 40^3 maps,
    16 heavy atoms / 4 torsions, nrun 10, pop 150, 2.5M evaluations per run,
    ADADELTA (the docking the CPU baseline times completely)."""
    import torch
    from adgpu_b200 import device, dock, frontend, synth
    w = WORKLOAD
    spec = synth.grid_spec(40, w["types"], seed=12345 + 1)
    grid = frontend.Grid.from_maps(synth.quantize_maps(synth.make_maps(spec)), w["types"], spec.spacing, spec.origin)
    text = "\n".join(synth.pdbqt_lines(synth.ligand_for(1, 0, 16, 4))[0]) + "\n"
    lig = frontend.Ligand(grid, text, None, run=frontend.default_dockpars(grid.spacing, w["pop"]), seed=w["seed"],
                          num_runs=10)
    job = device.DeviceJob(lig.tables, lig.dockpars, grid.reference_layout(), 10, lig.prng, device=dev)
    job.activate()
    bufs = (*job.population(), *job.population())
    init_dev = torch.from_numpy(lig.initpop).to(dev)
    prng0 = job.prng.clone()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts, ev, gens = [], 0, 0
    for i in range(steps + 1):
        job.prng.copy_(prng0)
        torch.cuda.synchronize()
        ea.record()
        r = dock.dock(job, init_dev, "ad", w["nev"], 42000, buffers=bufs)
        eb.record()
        torch.cuda.synchronize()
        if i:
            ts.append(ea.elapsed_time(eb) / 1e3)
            ev += int(r.evals_per_run.sum())
            gens = r.generations
    return {"workload": "40^3 maps, 16 heavy atoms / 4 torsions, nrun 10, pop 150, nev 2.5M, lsmet ad",
            "seconds_per_docking": sum(ts) / len(ts), "evals_per_s": ev / sum(ts), "generations": gens,
            "ligands_per_hour": 3600.0 * len(ts) / sum(ts), "best_energy": float(r.energies.min().item()),
            "docking_loop": dock.last_stats()}


def run_kernel_only(args):
    """--mode ls-kernel: one docking cut after a few generations, then `--steps`
    launches of the local-search kernel alone on that population (the case
    the ncu captures use; --nrun keeps it small)."""
    import torch
    from adgpu_b200 import device, dock, lib
    grid, lig = build_inputs(args.lsmet)
    ref_grid = grid.reference_layout()
    w = WORKLOAD
    nrun = args.nrun or w["nrun"]
    job = device.DeviceJob(lig.tables, lig.dockpars, ref_grid, nrun, lig.prng)
    # the docking that produces the population runs with another group size
    # than the measured launches, so that a profiler can select them by name
    os.environ["ADGPU_THREADS_PER_POSE"] = "32" if args.tpp == 64 else "64"
    job.activate()
    init_dev = torch.from_numpy(lig.initpop[:nrun * w["pop"]]).cuda()
    mid = dock.dock(job, init_dev, args.lsmet, w["nev"], 10)
    os.environ["ADGPU_THREADS_PER_POSE"] = str(args.tpp)
    job.activate()
    entry = {"ad": "adgpu_gradient_minad", "sw": "adgpu_perform_ls", "adam": "adgpu_gradient_minadam",
             "fire": "adgpu_gradient_minfire"}[args.lsmet]
    L = lig.dockpars.num_of_lsentities
    for _ in range(args.steps):
        c, e = mid.conformations.clone(), mid.energies.clone()
        job.evals_new.zero_()
        lib.call(entry, nrun * L, 64, c, e)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "ls-kernel", "kernel": entry, "nrun": nrun, "launches": args.steps,
                      "evals_last_launch": int(job.evals_new.sum().item())}))


def run_loop_kernel(args):
    """--mode loop-kernel: `--steps` pipelined dockings of the workload's ligand
    with --nrun runs of --nev evaluations (the small case the ncu captures of
    the docking loop's persistent kernel use); prints the loop's accounting."""
    import torch
    from adgpu_b200 import device, dock
    grid, lig = build_inputs(args.lsmet)
    ref_grid = grid.reference_layout()
    w = WORKLOAD
    nrun = args.nrun or w["nrun"]
    job = device.DeviceJob(lig.tables, lig.dockpars, ref_grid, nrun, lig.prng)
    job.activate()
    init_dev = torch.from_numpy(lig.initpop[:nrun * w["pop"]]).cuda()
    prng0 = job.prng.clone()
    res = None
    for _ in range(args.steps):
        job.prng.copy_(prng0)
        res = dock.dock(job, init_dev, args.lsmet, args.nev)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "loop-kernel", "lsmet": args.lsmet, "nrun": nrun, "nev": args.nev, "dockings": args.steps,
                      "evals_last": int(res.evals_per_run.sum()), "generations": res.generations,
                      "docking_loop": dock.last_stats()}))


def _ligand_text(config_id, idx, n_heavy, n_tors, types=None):
    from adgpu_b200 import synth
    mol = synth.ligand_for(config_id, idx, n_heavy, n_tors, types=types)
    return "\n".join(synth.pdbqt_lines(mol)[0]) + "\n"


def run_batch(args):
    """--mode batch: ligands docked by the batch engine (all ligands and runs
    admitted at once, one persistent launch) next to plain per-ligand
    dockings through the reference kernel API, same ligands, same budget.
    The batching configuration (--nlig 1024 --nev 2500000: 10-64 heavy atoms,
    0-32 torsions, nrun 20, ADADELTA), or with --batch-config 4 the
    flexible-receptor one (--nlig 256 --nev 2500000 --lsmet adam: 80^3 maps,
    7 types + e + d, 2 flexible residues of 8-10 atoms and 2-4 torsions,
    ligands of 40 heavy atoms / 10 torsions, nrun 50); smaller --nlig / --nev
    give bounded samples of either.  The plain arms dock --plain-sample of the
    ligands one at a time and scale their time to the whole set by cost."""
    import torch
    from adgpu_b200 import device, dock, engine, frontend, synth
    w = WORKLOAD
    cfg4 = getattr(args, "batch_config", 3) == 4
    types = synth.MAP_TYPES_7 if cfg4 else w["types"]
    spec = synth.grid_spec(80 if cfg4 else w["npts"], types, seed=12345 + (4 if cfg4 else 3))
    grid = frontend.Grid.from_maps(synth.quantize_maps(synth.make_maps_fast(spec)), types, spec.spacing, spec.origin)
    rng = np.random.default_rng(3)
    nlig, nrun, nev = args.nlig, (50 if cfg4 else 20), args.nev
    # cfg3: heavy atoms uniform in 10-64, torsions in 0-32; cfg4: ligands as
    # the plain configuration's (40 heavy atoms, 10 torsions), one seed each
    sizes = [(40, 10) if cfg4 else (int(rng.integers(10, 65)), int(rng.integers(0, 33))) for _ in range(nlig)]
    run = frontend.default_dockpars(grid.spacing, 150)
    flex = None
    ltypes = None
    if cfg4:
        frng = np.random.default_rng(77)
        flex = synth.flexres_text([synth.make_flexres(100 + k, int(frng.integers(8, 11)), int(frng.integers(2, 5)),
                                                      anchor=np.array([-3.0 + 6.0 * k, 4.0, 0.0])) for k in range(2)])
        ltypes = (("C", 0.55), ("A", 0.15), ("N", 0.08), ("NA", 0.04), ("OA", 0.13), ("SA", 0.05))
    ligs = [frontend.Ligand(grid, _ligand_text(4 if cfg4 else 3, i, a, t, types=ltypes), flex, run=run,
                            seed=w["seed"], num_runs=nrun)
            for i, (a, t) in enumerate(sizes)]
    # batched: one engine, everything admitted, run to completion
    en = engine.Engine(threads_per_pose=args.engine_tpp)
    rec = en.add_receptor(grid)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    t0 = time.perf_counter()
    ids = [en.submit(lg, rec, args.lsmet, max_evals=nev) for lg in ligs]
    tpps = {}
    for i in ids:
        t = en.info(i)[0]
        tpps[str(t)] = tpps.get(str(t), 0) + 1
    en.run()
    res = [en.result(i) for i in ids]
    t_batch = time.perf_counter() - t0
    clocks = sampler.stop()
    ev_batch = sum(int(r.evals.sum()) for r in res)
    st = en.stats()
    util = st.worker_busy_s / st.worker_span_s if st.worker_span_s > 0 else None
    # plain: one ligand at a time through the kernel API, (a) driven by the
    # reference host's loop (a synchronous call per kernel per generation) --
    # the drop-in -- and (b) with the loop resident on the device
    # sample: every k-th ligand; the plain rate is scaled to the whole set by
    # per-ligand cost (pairs + 8 atoms per evaluation, the engine's weight)
    nplain = min(nlig, args.plain_sample)
    sample = ligs[::max(1, nlig // nplain)][:nplain]
    cost = lambda lg: lg.dockpars.num_of_intraE_contributors + 8.0 * lg.dockpars.num_of_atoms + 64.0  # noqa: E731
    scale = sum(cost(lg) for lg in ligs) / sum(cost(lg) for lg in sample) * len(sample) / nlig
    ref_grid = grid.reference_layout()
    plain = {}
    for name, fn in (("reference_host_loop", dock.dock_host_loop), ("resident_loop", dock.dock)):
        t_plain, ev_plain = 0.0, 0
        for lg in sample:
            job = device.DeviceJob(lg.tables, lg.dockpars, ref_grid, nrun, lg.prng)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            job.activate()
            r = fn(job, lg.initpop, args.lsmet, nev, 42000)
            torch.cuda.synchronize()
            t_plain += time.perf_counter() - t0
            ev_plain += int(r.evals_per_run.sum())
            del job
        plain[name] = {"ligands_sampled": nplain, "seconds": t_plain, "ligands_per_hour": 3600.0 * nplain / t_plain / scale,
                       "evals_per_s": ev_plain / t_plain, "sample_cost_scale": scale}
    lph_b = 3600.0 * nlig / t_batch
    return {"mode": "batch", "config": 4 if cfg4 else 3, "flexres": 2 if cfg4 else 0,
            "ligands": nlig, "nrun": nrun, "nev_per_run": nev, "lsmet": args.lsmet,
            "heavy_atoms": [min(a for a, _ in sizes), max(a for a, _ in sizes)],
            "batched": {"seconds": t_batch, "ligands_per_hour": lph_b, "evals_per_s": ev_batch / t_batch,
                        "worker_utilisation": util, "tasks": int(st.tasks)},
            "plain": plain,
            "batched_over_plain_ligands_per_hour": {k: lph_b / v["ligands_per_hour"] for k, v in plain.items()},
            "tpp_classes": tpps, "clocks_batched": clocks}


def run_serve(args):
    """--mode serve: a Poisson stream of cfg2-sized requests against three
    resident receptors (60^3, 80^3, 100^3 maps, 7 types + e + d), arrival rate
    80% of the measured batched capacity, admission by a fixed device-memory
    budget; p50/p99 request latency (arrival to result) and ligands/hour."""
    import torch
    from adgpu_b200 import engine, frontend, synth
    w = WORKLOAD
    types = synth.MAP_TYPES_7
    grids = []
    for k, n in enumerate((60, 80, 100)):
        spec = synth.grid_spec(n, types, seed=12345 + 5 + k)
        grids.append(frontend.Grid.from_maps(synth.quantize_maps(synth.make_maps_fast(spec)), types, spec.spacing,
                                             spec.origin))
    nrun, nev, nreq = 10, args.nev, args.nreq
    ltypes = (("C", 0.55), ("A", 0.15), ("N", 0.08), ("NA", 0.04), ("OA", 0.13), ("SA", 0.05))
    rng = np.random.default_rng(5)
    texts = [_ligand_text(5, i, 40, 10, types=ltypes) for i in range(nreq)]
    targets = [int(rng.integers(0, 3)) for _ in range(nreq)]
    ligs = [frontend.Ligand(grids[t], texts[i], None, run=frontend.default_dockpars(grids[t].spacing, 150),
                            seed=w["seed"], num_runs=nrun) for i, t in enumerate(targets)]
    budget = args.budget_gb << 30
    natoms = [lg.dockpars.num_of_atoms for lg in ligs]
    # 64 threads per pose unless asked otherwise: a request's latency is the
    # chain of its runs' generations, each ending with its longest local
    # search, which two warps per pose shorten (p50 0.96 s against 1.27 s at
    # 80 % load for 4 % less capacity)
    tpp = args.engine_tpp if args.engine_tpp else 64
    # capacity: a batch of requests run to completion in one launch, by an
    # engine with the serving engine's settings
    cap_n = min(nreq, 48)
    cap = engine.Engine(memory_budget_bytes=budget, threads_per_pose=tpp, priority=args.priority)
    crecs = [cap.add_receptor(g) for g in grids]
    t0 = time.perf_counter()
    ids = [cap.submit(ligs[i], crecs[targets[i]], args.lsmet, max_evals=nev) for i in range(cap_n)]
    cap.run()
    for i in ids:
        cap.result(i)
    capacity = cap_n / (time.perf_counter() - t0)          # ligands / s
    cap.close()
    rate = args.rate if args.rate > 0 else 0.8 * capacity
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    # the serving engine: ticks end on a wall-clock deadline (or a generation count)
    en = engine.Engine(memory_budget_bytes=budget, gens_per_tick=args.gens_per_tick, tick_ms=args.tick_ms,
                       threads_per_pose=tpp, priority=args.priority)
    recs = [en.add_receptor(g) for g in grids]
    # serving loop
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    t_start = time.perf_counter()
    pending, live, lat, queued = list(range(nreq)), {}, [], []
    done_n = 0
    t_submit = t_tick = t_result = 0.0
    while done_n < nreq:
        now = time.perf_counter() - t_start
        while pending and arrivals[pending[0]] <= now:
            queued.append(pending.pop(0))
        ta = time.perf_counter()
        while queued:
            i = queued[0]
            rid = en.submit(ligs[i], recs[targets[i]], args.lsmet, max_evals=nev, raise_on_budget=False)
            if rid is None:
                break
            live[rid] = i
            queued.pop(0)
        tb = time.perf_counter()
        t_submit += tb - ta
        if live:
            en.tick()
            tc = time.perf_counter()
            t_tick += tc - tb
            for rid in [r for r in live if en.done(r)]:
                i = live.pop(rid)
                if args.process_results:
                    en.process_result(rid, natoms[i])
                en.result(rid)
                lat.append(time.perf_counter() - t_start - arrivals[i])
                done_n += 1
            t_result += time.perf_counter() - tc
        else:
            time.sleep(0.001)
    t_total = time.perf_counter() - t_start
    torch.cuda.synchronize()
    clocks = sampler.stop()
    lat = np.array(lat)
    return {"mode": "serve", "requests": nreq, "nrun": nrun, "nev_per_run": nev, "receptors": "60^3, 80^3, 100^3",
            "batched_capacity_ligands_per_s": capacity, "arrival_rate_per_s": rate,
            "ligands_per_hour": 3600.0 * nreq / t_total, "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)), "latency_p90_s": float(np.percentile(lat, 90)),
            "latency_mean_s": float(lat.mean()), "latency_max_s": float(lat.max()), "memory_budget_gb": args.budget_gb,
            "gens_per_tick": args.gens_per_tick, "tick_ms": args.tick_ms, "ticks": int(en.stats().ticks),
            "priority": {0: "least advanced run", 1: "oldest request"}[args.priority],
            "results_processed_on_device": bool(args.process_results), "threads_per_pose": {-1: "tuned"}.get(tpp, tpp),
            "host_seconds": {"submit": t_submit, "tick": t_tick, "results": t_result, "total": t_total,
                             "engine_kernels": en.stats().kernel_s},
            "worker_utilisation": (en.stats().worker_busy_s / en.stats().worker_span_s
                                   if en.stats().worker_span_s > 0 else None), "clocks": clocks}


def run_result(args):
    """--mode result: result processing of one docked ligand of the plain
    workload (60^3 maps, 40 heavy atoms / 10 torsions, nrun 100, pop 150) on
    the device (adgpu_process_result: population ordering, re-scoring, RMSD,
    clustering; host outputs included) against the reference's own
    process_result on one host core (oracle/_ref, files switched off), on the
    same final population."""
    import tempfile
    import torch
    from adgpu_b200 import device, dock, frontend, result, synth
    from oracle import refpy
    w = WORKLOAD
    d = tempfile.mkdtemp(prefix="adgpu_result_")
    spec = synth.grid_spec(w["npts"], w["types"], seed=12345 + w["config_id"])
    fld = synth.write_maps(spec, synth.make_maps(spec), d)
    lig_path = os.path.join(d, "ligand.pdbqt")
    synth.write_ligand(synth.ligand_for(w["config_id"], 0, w["n_heavy"], w["n_tors"]), lig_path)
    seeds = ",".join(str(s) for s in w["seed"])
    ref = refpy.RefJob(["--ffile", fld, "--lfile", lig_path, "--nrun", str(w["nrun"]), "--seed", seeds,
                        "--heuristics", "0", "--autostop", "0", "--psize", str(w["pop"])])
    grid = frontend.Grid.read(fld)
    lig = frontend.Ligand(grid, open(lig_path).read(), None, run=frontend.default_dockpars(grid.spacing, w["pop"]),
                          seed=w["seed"], num_runs=w["nrun"])
    job = device.DeviceJob(lig.tables, lig.dockpars, grid.reference_layout(), w["nrun"], lig.prng)
    job.activate()
    dr = dock.dock(job, lig.initpop, args.lsmet, nev=args.nev)
    pops0, en0 = dr.conformations.clone(), dr.energies.clone()
    R = w["nrun"]

    def gpu_time(rescore_all):
        params = result.default_params(rescore_entities=int(rescore_all))
        ts, out = [], None
        for i in range(args.warmup + args.steps):
            c, e = pops0.clone(), en0.clone()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = result.process_result(lig, job.grid, c, e, R, params)
            t1 = time.perf_counter()
            if i >= args.warmup:
                ts.append(t1 - t0)
        return statistics.median(ts), out, c, e

    t_best, out, c_sorted, e_sorted = gpu_time(False)
    t_all, out_all, _, _ = gpu_time(True)
    hp, he = pops0.cpu().numpy(), en0.cpu().numpy()
    tr, reps = [], 0
    t_start = time.perf_counter()
    while reps < 3 or time.perf_counter() - t_start < 10.0:
        t0 = time.perf_counter()
        rp, re_, rruns, rxyz, rper = ref.process_result(hp, he)
        tr.append(time.perf_counter() - t0)
        reps += 1
    t_ref = statistics.median(tr)
    fields = ("inter_e", "interflex_e", "inter_e_elec", "intra_e", "intraflex_e", "rmsd_from_ref")
    got = np.array([[getattr(r, f) for f in fields] for r in out.runs], np.float64)
    want = np.array([[getattr(r, f) for f in fields] for r in rruns], np.float64)
    same_clusters = all((a.cluster_id, a.cluster_subrank, a.output) == (b.cluster_id, b.cluster_subrank, b.output)
                        for a, b in zip(out.runs, rruns))
    exact = float(np.mean(np.concatenate([(got == want).ravel(), (out.best_xyz == rxyz).ravel(),
                                          (out.peratom == rper).ravel()])))
    return {"mode": "result", "metric": "ligands/s (result processing)", "workload":
            f"one docked ligand ({w['n_heavy']} heavy atoms / {w['n_tors']} torsions, {lig.dockpars.num_of_atoms} "
            f"atoms, {lig.dockpars.num_of_intraE_contributors} pairs), nrun {R}, pop {w['pop']}, {args.lsmet} "
            f"docking at nev {args.nev}",
            "gpu_ms_best_entities": 1e3 * t_best, "gpu_ms_all_entities": 1e3 * t_all,
            "reference_host_ms": 1e3 * t_ref, "reference_reps": reps, "reference_cores": 1,
            "speedup_vs_reference": t_ref / t_all,
            "clusters": len(out.clusters), "parity": {
                "population_order_identical": bool(np.array_equal(c_sorted.cpu().numpy(), rp) and
                                                   np.array_equal(e_sorted.cpu().numpy(), re_, equal_nan=True)),
                "clusters_identical": bool(same_clusters),
                "max_abs_diff": float(np.abs(got - want).max()), "bit_identical_fraction": exact},
            "note": "the reference re-scores every entity of every run in make_resfiles; the device path does so "
                    "with rescore_entities (gpu_ms_all_entities, the like-for-like figure) and otherwise only each "
                    "run's best entity, the only one the .dlg uses"}


def _hbm_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
    except Exception:
        return 6650.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--lsmet", default="ad", choices=["ad", "sw", "adam", "fire"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-plain sample in the default mode")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving sample in the default mode")
    ap.add_argument("--no-result", action="store_true", help="skip the result-processing sample in the default mode")
    ap.add_argument("--mode", default="dock", choices=["dock", "ls-kernel", "loop-kernel", "batch", "serve", "result"])
    ap.add_argument("--nrun", type=int, default=0, help="runs per ligand (ls-kernel / loop-kernel modes)")
    ap.add_argument("--tpp", type=int, default=32, help="threads per pose of the measured launches (ls-kernel mode)")
    ap.add_argument("--engine-tpp", type=int, default=0,
                    help="engine threads per pose (batch / serve modes): 0 = the mode's default (batch: the "
                         "engine's, 32; serve: 64), -1 = tuned per ligand size, or 32, 64, 128")
    ap.add_argument("--nlig", type=int, default=64, help="ligands (batch mode)")
    ap.add_argument("--batch-config", type=int, default=3, choices=[3, 4],
                    help="batch mode workload: 3 (uneven ligands) or 4 (80^3 maps, 2 flexible residues, nrun 50)")
    ap.add_argument("--nev", type=int, default=250_000, help="evaluations per run (batch / serve / loop-kernel modes)")
    ap.add_argument("--plain-sample", type=int, default=16, help="ligands docked one at a time for the plain arm")
    ap.add_argument("--nreq", type=int, default=200, help="requests (serve mode)")
    ap.add_argument("--budget-gb", type=int, default=8, help="engine device-memory budget (serve mode)")
    ap.add_argument("--gens-per-tick", type=int, default=0, help="generations per engine tick (serve mode; 0: no limit)")
    ap.add_argument("--process-results", action="store_true",
                    help="serve mode: each finished request's runs ordered, re-scored and clustered on the device")
    ap.add_argument("--rate", type=float, default=0.0,
                    help="request arrival rate per second (serve mode; 0: 80%% of the measured capacity)")
    ap.add_argument("--tick-ms", type=float, default=50.0, help="wall-clock length of an engine tick (serve mode; 0: none)")
    ap.add_argument("--priority", type=int, default=1, choices=[0, 1],
                    help="serve mode: runs served first, 0 the least advanced, 1 the oldest request's")
    args = ap.parse_args()
    if args.mode == "ls-kernel":
        run_kernel_only(args)
        return
    if args.mode == "loop-kernel":
        run_loop_kernel(args)
        return
    if args.mode in ("batch", "serve", "result"):
        out = {"batch": run_batch, "serve": run_serve, "result": run_result}[args.mode](args)
        print(json.dumps(out), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    line = run_engine(args, rank, world, local_rank)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

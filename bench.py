"""Benchmark of the MCWF ensemble engine (one JSON line on rank 0).

Workload (default): the driven lossy qubit-mode system — two-level atom x mode with
Jaynes-Cummings coupling g=2, kappa=1, gamma=0.5, pump eta=1.5, Delta=0, dimension
2 x 40 = 80, complex128, 4096 trajectories per GPU, RK54 eps=1e-6, dpLimit 0.01 —
evolved through t in [0, 20].  One bench "step" advances every trajectory by Dt=1
(inside the same persistent launch the trajectories take ~10^3 MCWF steps each).
The metric is accepted MCWF trajectory-steps per second (MCWF_Trajectory::step calls,
logger_.step(), MCWF_Trajectory.h:372) summed over all GPUs.

--impl reference times the reference's algorithm on the host cores (the CPU oracle,
a restatement of C++QED's serial Ensemble / MCWF_Trajectory path including the
density-operator average at every Dt) on a bounded sample of the same workload.

Multi-GPU (torchrun): trajectories are sharded, every rank runs its own 4096 with
disjoint pcg/philox streams (weak scaling); the per-interval ensemble sums are
all-reduced (the only exchange) and timing is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (script, args, n_traj per GPU, Dt per step)
    "qbitmode_jc_2x40": ("QbitMode_C++QED",
                         ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC", "0", "--kappa", "1",
                          "--eta", "1.5", "--cutoff", "40", "--g", "2"], 4096, 1.0),
    # the same system in the interaction picture (the reference's default picture): detuned
    # qubit and mode, so the coupling and pump terms carry time-dependent phases
    "qbitmode_jc_2x40_ip": ("QbitMode_C++QED",
                            ["--picture", "IP", "--deltaA", "-1", "--gamma", "0.5", "--deltaC", "2", "--kappa", "1",
                             "--eta", "1.5", "--cutoff", "40", "--g", "2"], 4096, 1.0),
    # particle in a cavity (1particle1mode, ParticleAlongCavity with a cos^2 mode function,
    # no transverse pump): mode cutoff 20 x particle momenta 2^7 = 2560
    "particle_cavity_2560": ("1particle1mode",
                             ["--1p1mconf", "2", "--vClass", "0", "--modeCav", "Cos", "--kCav", "1", "--Unot", "-1",
                              "--eta", "5", "--kappa", "1", "--cutoff", "20", "--fin", "7"], 2048, 0.05),
    "pumped_lossy_mode_30": ("PumpedLossyMode_C++QED",
                             ["--picture", "Sch", "--deltaC", "-1", "--eta", "2", "--kappa", "1", "--cutoff", "30",
                              "--no_quadratures"], 1000, 1.0),
}


# Uneven batch (driven Jaynes-Cummings, qubit x mode): cutoffs uniform in [20, 120],
# g uniform in [1, 10], eta uniform in [0.5, 3], kappa = 1, gamma = 0; one parameter draw per
# system of UNEVEN_PER_SYSTEM trajectories (fixed seed).
UNEVEN = {"uneven_jc_16384": (256, 64, 0.5)}  # name: (systems, trajectories per system, Dt per step)

# Serving: Poisson arrivals (mean SERVING["rate"] requests/s, fixed seed) of ensemble requests
# of 64-1024 trajectories over a library of systems: pumped lossy mode, cutoff 20-200;
# qubit-mode 2 x (10-100); the 6-qubit chain with local decay (dim 64); optomechanics 15 x 30.
# Every request evolves to T with output interval Dt.
SERVING = {"serving_poisson_200": {"rate": 200.0, "requests": 400, "T": 0.5, "Dt": 0.125, "seed": 77}}


def serving_library():
    """(kind, model) pairs: cutoffs on a grid of 10, so a service keeps ~30 systems."""
    import cppqed_b200 as cqg
    lib = []
    for N in range(20, 201, 10):
        lib.append(("mode", cqg.Model("PumpedLossyMode_C++QED",
                                      ["--picture", "Sch", "--deltaC", "-1", "--eta", "2", "--kappa", "1",
                                       "--cutoff", str(N), "--no_quadratures"])))
    for N in range(10, 101, 10):
        lib.append(("qubit-mode", cqg.Model("QbitMode_C++QED",
                                            ["--picture", "Sch", "--deltaA", "0", "--gamma", "0.5", "--deltaC",
                                             "0", "--kappa", "1", "--eta", "1.5", "--cutoff", str(N), "--g", "2"])))
    lib.append(("chain", cqg.Model("QbitChain", ["--nQbit", "6", "--deltaA", "0", "--gamma", "0.2", "--etat", "0.5",
                                                  "--u", "1"])))
    lib.append(("optomechanics", cqg.Model("Optomechanics",
                                           ["--picture", "Sch", "--cutoffOpt", "15", "--cutoffMech", "30",
                                            "--etaOpt", "2", "--kappaOpt", "1", "--deltaCOpt", "-1",
                                            "--kappaMech", "0.1", "--deltaCMech", "-2", "--u", "0.2"])))
    return lib


def serving_requests(cfg, lib):
    """Seeded request list: (arrival s, library index, trajectories, prng stream)."""
    import numpy as np
    rng = np.random.default_rng(cfg["seed"])
    kinds = sorted({k for k, _ in lib})
    by_kind = {k: [i for i, (kk, _) in enumerate(lib) if kk == k] for k in kinds}
    t = 0.0
    out = []
    stream = 1
    for _ in range(cfg["requests"]):
        t += rng.exponential(1.0 / cfg["rate"])
        k = kinds[int(rng.integers(len(kinds)))]
        j = by_kind[k][int(rng.integers(len(by_kind[k])))]
        n = int(rng.integers(64, 1025))
        out.append((t, j, n, stream))
        stream += n
    return out


def uneven_models(n_systems, seed=2024):
    import numpy as np

    import cppqed_b200 as cqg
    rng = np.random.default_rng(seed)
    models = []
    for _ in range(n_systems):
        N = int(rng.integers(20, 121))
        g = rng.uniform(1, 10)
        eta = rng.uniform(0.5, 3)
        args = ["--picture", "Sch", "--deltaA", "0", "--gamma", "0", "--deltaC", "0", "--kappa", "1",
                "--eta", "%.6f" % eta, "--cutoff", str(N), "--g", "%.6f" % g]
        models.append(cqg.Model("QbitMode_C++QED", args))
    return models


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="qbitmode_jc_2x40",
                    choices=sorted(WORKLOADS) + sorted(UNEVEN) + sorted(SERVING))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--rng", default="pcg64", choices=["pcg64", "philox"])
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cta-threads", type=int, default=0,
                    help="force this CTA size on every kernel group (no autotuning)")
    ap.add_argument("--cta-shared-vectors", type=int, default=0,
                    help="with --cta-threads: 1 selects the shared-memory stage vectors (CTA kernel) or the "
                         "high-occupancy instance (warp kernel)")
    ap.add_argument("--yield-steps", type=int, default=0,
                    help="MCWF steps after which a warp hands its trajectory back to the queue (0: default, -1: never)")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the batched-vs-plain, accuracy and serving checks of the default line")
    ap.add_argument("--apply-states", type=int, default=0,
                    help="only time the batched H/i application on this many states of the workload's system")
    ap.add_argument("--apply-reps", type=int, default=20)
    return ap.parse_args()


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML read every 20 ms
    (the device matched by PCI bus id), else nvidia-smi every 200 ms.  Read-only queries."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, max sm MHz, set of reasons)

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.device)
        bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def start(self):
        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.nvml = (nv, h, bits)
            self.stopping = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _poll(self):
        nv, h, bits = self.nvml
        while not self.stopping.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), {n for n, b in bits.items() if r & b}))
            except Exception:
                pass
            self.stopping.wait(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stopping.set()
            self.thread.join(timeout=5)
            source = "nvml, 20 ms"
        elif self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        else:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            source = "nvidia-smi, 200 ms"
            for l in self.lines:
                p = [x.strip() for x in l.split(",")]
                if len(p) < 9:
                    continue
                try:
                    self.samples.append((float(p[1]), float(p[2]),
                                         {n for n, v in zip(self.NAMES, p[5:9]) if v.lower() == "active"}))
                except ValueError:
                    continue
        sms = [a for a, _, _ in self.samples]
        maxes = [b for _, b, _ in self.samples]
        reasons = set().union(*[c for _, _, c in self.samples]) if self.samples else set()
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(sms), "source": source}


def flops_model(model):
    """Algorithmic FLOPs per RK attempt and per extra MCWF-step work, from the system's
    operator structure (complex MAC = 8, complex multiply = 6, real-complex axpy = 4)."""
    import numpy as np
    d = model.desc.contents
    D = model.dim
    # nonzeros of H/i per row: count entries of every term
    nnz = 0
    for i in range(d.n_ham):
        t = d.ham[i]
        L = 3 ** t.rank
        for j in range(L):
            if t.diagonals[j]:
                box = 1
                digits = []
                rem = j
                for _ in range(t.rank):
                    digits.append(rem % 3)
                    rem //= 3
                digits = digits[::-1]
                for a in range(t.rank):
                    N = d.dims[t.axes[a]]
                    box *= N if digits[a] == 0 else N - t.differences[a]
                slices = D // int(np.prod([d.dims[t.axes[a]] for a in range(t.rank)]))
                nnz += box * slices
    rhs = 8.0 * nnz
    per_attempt = 6 * rhs + D * (15 * 4 + 4 * 4 + 5 * 4 + 15)
    per_step = D * (5 + 3 * d.n_jumps)
    return per_attempt, per_step, nnz


def measured_peaks():
    """HBM copy bandwidth and bf16 GEMM peaks measured on this pool (driver-written), else
    the pool's earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


# DRAM bytes of one launch from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum).
# MCWF kernel: the default workload (qubit-mode 2x40, 4096 trajectories, FP64), one Dt = 1
# launch.  Apply kernel: 65,536 states of the same system (the full 1 M-state batch is larger
# than a capture should be); reads are exactly psi + dpsi, part of the dpsi write is still
# in L2 when the launch ends.
# DRAM bytes (read + write) and L2-to-SM bytes per MCWF launch from one ncu capture of the
# first timed launch of each workload (profiles/mcwf*Kernel_*.md), by (workload, precision)
MCWF_TRAFFIC = {("qbitmode_jc_2x40", "fp64"): {"dram": 6.54464e6 + 0.159232e6, "l2_to_sm": 530.862816e6},
                ("particle_cavity_2560", "fp32"): {"dram": 72.08704e6 + 466.320128e6, "l2_to_sm": 14.272849e9},
                ("particle_cavity_2560", "fp64"): {"dram": 619.755264e6 + 2555.67e6, "l2_to_sm": 21.374789e9}}
APPLY_TRAFFIC = {"n_states": 65536, "bytes": 167.799040e6 + 33.929728e6, "algorithmic_bytes": 48.0 * 65536 * 80}


def run_apply(model, n_states=1 << 20, warmup=3, reps=20):
    """Batched H/i application (cqg_system_apply_hamiltonian) on n_states device states:
    48 bytes per state element (read psi, read+write dpsi); timed with CUDA events on the
    launching stream."""
    import ctypes

    import torch

    import cppqed_b200 as cqg

    system = cqg.System(model.desc)
    D = model.dim
    n_states = max(1, min(n_states, (4 << 30) // (48 * D)))  # at most ~4 GB moved per launch
    g = torch.Generator(device="cuda").manual_seed(5)
    psi = torch.randn(n_states, D, dtype=torch.complex128, device="cuda", generator=g)
    dpsi = torch.zeros_like(psi)
    stream = torch.cuda.current_stream()
    lib = cqg.lib()

    def launch():
        rc = lib.cqg_system_apply_hamiltonian(system._h, ctypes.c_void_p(psi.data_ptr()),
                                              ctypes.c_void_p(dpsi.data_ptr()), n_states, 0.0,
                                              ctypes.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(lib.cqg_last_error().decode())

    for _ in range(warmup):
        launch()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    bytes_per = 48.0 * n_states * D
    peak, src = measured_peaks()
    gbs = bytes_per / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "peak_source": src, "ms_per_launch": ms, "bytes_per_launch": bytes_per, "n_states": n_states,
            "traffic": APPLY_TRAFFIC if n_states == APPLY_TRAFFIC["n_states"] else None,
            "kernel": "stagedApplyKernel (cqg_system_apply_hamiltonian)"}


def run_ours(args, rank, world, dev):
    import numpy as np
    import torch

    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A
    from cppqed_b200 import sharding

    script, sargs, n_traj, Dt = WORKLOADS[args.workload]
    model = cqg.Model(script, sargs)
    pars = model.run_pars().mcwf
    pars.rng = A.RNG_PCG64 if args.rng == "pcg64" else A.RNG_PHILOX
    pars.precision = A.FP64 if args.precision == "fp64" else A.FP32
    pars.prng_stream = sharding.first_stream(1, n_traj, rank)
    pars.yield_steps = args.yield_steps
    if args.cta_threads:
        pars.autotune = 0
        pars.cta_threads = args.cta_threads
        pars.cta_shared_vectors = args.cta_shared_vectors
    system = cqg.System(model.desc)
    psi0 = model.initial_state()
    ens = cqg.Ensemble(system, psi0, n_traj, pars)

    def allreduce(x):
        return sharding.allreduce_sum(x, world)

    for _ in range(args.warmup):
        allreduce(ens.run(Dt, 1))
    c0 = ens.counters()
    sampler = ClockSampler(dev)
    if rank == 0:
        sampler.start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    kernel_ms = run_ms = 0.0
    for _ in range(args.steps):
        sums = allreduce(ens.run(Dt, 1))
        k, r = ens.last_ms()
        kernel_ms += k
        run_ms += r
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop() if rank == 0 else None
    c1 = ens.counters()
    d = (c1.astype(np.int64) - c0.astype(np.int64)).sum(axis=0)
    # summed over ranks: accepted steps, ODE attempts, RHS evaluations, failed attempts,
    # dpLimit overshoots, step-backs, jumps
    tot = allreduce(np.array([d[0], d[1], d[3], d[2], d[4], d[5], d[6]], dtype=np.float64))
    tmax = sharding.max_over_ranks([run_ms, kernel_ms], world)
    run_ms_max, kernel_ms_max = float(tmax[0]), float(tmax[1])
    steps_total = float(tot[0])
    value = steps_total / (run_ms_max * 1e-3)

    # end to end through the public API from host buffers: create (upload of the host
    # states), one Dt interval, read-back of the averages, destroy; one untimed call first,
    # as for the device-timed steps (first-use allocations of the engine's buffers)
    e = cqg.Ensemble(system, psi0, n_traj, pars)
    allreduce(e.run(Dt, 1))
    del e
    e2e_steps = 0
    phases = np.zeros(4)  # create (host states uploaded), run (one Dt, sums read back), counters, destroy
    t0 = time.perf_counter()
    n_e2e = max(1, min(3, args.steps))
    for _ in range(n_e2e):
        ta = time.perf_counter()
        e = cqg.Ensemble(system, psi0, n_traj, pars)
        tb = time.perf_counter()
        allreduce(e.run(Dt, 1))
        tc = time.perf_counter()
        e2e_steps += int(e.counters()[:, 0].sum())
        td = time.perf_counter()
        del e
        phases += [tb - ta, tc - tb, td - tc, time.perf_counter() - td]
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_tot = allreduce(np.array([e2e_steps, e2e_s], dtype=np.float64))
    e2e_s = float(sharding.max_over_ranks([e2e_s], world)[0])
    e2e_value = float(e2e_tot[0]) / e2e_s
    # sent per call: the initial state once (replicated on the device), and per trajectory its
    # slot and state offsets, system index, times, random stream and counters
    elem = 16 if args.precision == "fp64" else 8
    h2d = model.dim * elem + n_traj * (8 + 8 + 4 + 8 * 4 + 32 + 64)
    d2h = (model.n_avr + 1) * 8 + 4

    apply = run_apply(model) if rank == 0 else None
    fp64_peak, fp32_peak = cqg.engine.probe_fma_peaks()
    per_attempt, per_step, nnz = flops_model(model)
    flops = float(tot[1]) * per_attempt + steps_total * per_step
    achieved = flops / (kernel_ms_max * 1e-3) / 1e12
    peak = fp64_peak if args.precision == "fp64" else fp32_peak
    return {
        "value": value, "ms_per_step": run_ms_max / args.steps, "steps_total": steps_total,
        "attempts_total": float(tot[1]), "rhs_total": float(tot[2]), "kernel_ms": kernel_ms_max,
        "failed_total": float(tot[3]), "overshoots_total": float(tot[4]), "stepbacks_total": float(tot[5]),
        "jumps_total": float(tot[6]),
        "clocks": clocks, "e2e": {"value": e2e_value, "unit": "trajectory-steps/s", "h2d_bytes_per_step": h2d,
                                  "d2h_bytes_per_step": d2h, "steps_per_call": e2e_steps / n_e2e,
                                  "ms_per_call": dict(zip(("create", "run", "counters", "destroy"),
                                                          [round(1e3 * v / n_e2e, 3) for v in phases]))},
        "roofline": {"bound": "fp64" if args.precision == "fp64" else "fp32", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": MCWF_TRAFFIC.get((args.workload, args.precision), {}).get("dram"),
                     "traffic_l2_to_sm": MCWF_TRAFFIC.get((args.workload, args.precision), {}).get("l2_to_sm"),
                     "peak_source": "measured FMA probe (cqg_probe_fma_peaks) on this GPU",
                     "flops_per_attempt": per_attempt, "nnz_h": nnz},
        "n_traj": n_traj, "model": model, "apply": apply, "plan": ens.plan(),
    }


def run_batched(args, dev):
    """Uneven batch: every system's trajectories in one batch (one persistent launch per
    kernel group, groups concurrent), against the plain path (one FP64 ensemble per system
    and launch, one after another), and the FP32-state variant against FP64 on the same
    random streams."""
    import numpy as np
    import torch

    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A

    n_sys, per, Dt = UNEVEN[args.workload]
    models = uneven_models(n_sys)
    systems = [cqg.System(m.desc) for m in models]
    idx = np.repeat(np.arange(n_sys), per)
    psi0s = [models[j].initial_state() for j in idx]
    n_traj = len(idx)

    def pars_for(precision, stream=1):
        p = models[0].run_pars().mcwf
        p.rng = A.RNG_PCG64 if args.rng == "pcg64" else A.RNG_PHILOX
        p.precision = precision
        p.prng_stream = stream
        return p

    def timed_batch(precision, steps, warmup, sampler=None):
        ens = cqg.Ensemble.batch(systems, idx, psi0s, pars_for(precision))
        for _ in range(warmup):
            ens.run(Dt, 1)
        c0 = ens.counters()
        if sampler:
            sampler.start()
        torch.cuda.synchronize()
        k_ms = r_ms = 0.0
        for _ in range(steps):
            ens.run(Dt, 1)
            k, r = ens.last_ms()
            k_ms += k
            r_ms += r
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        d = ens.counters().astype(np.int64) - c0.astype(np.int64)
        return ens, d, k_ms, r_ms, clocks

    precision = A.FP64 if args.precision == "fp64" else A.FP32
    ens, d, k_ms, r_ms, clocks = timed_batch(precision, args.steps, args.warmup, ClockSampler(dev))
    steps_total = float(d[:, 0].sum())
    value = steps_total / (r_ms * 1e-3)
    plan = ens.plan()

    # roofline: algorithmic FLOPs trajectory by trajectory
    fm = [flops_model(m) for m in models]
    flops = float(sum(d[i, 1] * fm[idx[i]][0] + d[i, 0] * fm[idx[i]][1] for i in range(n_traj)))
    fp64_peak, fp32_peak = cqg.engine.probe_fma_peaks()
    peak = fp64_peak if args.precision == "fp64" else fp32_peak
    achieved = flops / (k_ms * 1e-3) / 1e12

    # FP32-state variant against FP64 on the same streams after the same simulated time:
    # difference of the batch means of every average, in units of the FP64 standard error
    T_steps = args.warmup + args.steps
    e64, _, _, _, _ = timed_batch(A.FP64, T_steps, 0) if precision != A.FP64 else (ens, None, 0, 0, None)
    e32, _, _, _, _ = timed_batch(A.FP32, T_steps, 0) if precision != A.FP32 else (ens, None, 0, 0, None)
    a64 = e64.traj_averages()[:, :models[0].n_avr]
    a32 = e32.traj_averages()[:, :models[0].n_avr]
    se = a64.std(axis=0, ddof=1) / np.sqrt(n_traj)
    z = np.abs(a32.mean(axis=0) - a64.mean(axis=0)) / np.where(se > 0, se, np.inf)
    precision_check = {"observables": models[0].key(), "max_sigma": float(z.max()),
                       "sigma_per_observable": [float(v) for v in z], "t": T_steps * Dt,
                       "note": "FP32-state/FP64-control batch vs the FP64 batch, same pcg64 streams"}
    del e64, e32

    # plain path: one FP64 ensemble per system and launch, one after another, same work
    p_steps = 0
    p_ms = 0.0
    for j in range(n_sys):
        e = cqg.Ensemble(systems[j], models[j].initial_state(), per, pars_for(A.FP64, 1 + j * per))
        for _ in range(T_steps):
            e.run(Dt, 1)
            p_ms += e.last_ms()[1]
        p_steps += int(e.counters()[:, 0].sum())
        del e
    plain_value = p_steps / (p_ms * 1e-3)

    # end to end: batch created from host states, one Dt, averages read back, destroyed;
    # one untimed call first (first-use allocations), then three timed calls
    e = cqg.Ensemble.batch(systems, idx, psi0s, pars_for(precision))
    e.run(Dt, 1)
    del e
    e2e_steps = 0
    t0 = time.perf_counter()
    for _ in range(3):
        e = cqg.Ensemble.batch(systems, idx, psi0s, pars_for(precision))
        e.run(Dt, 1)
        e2e_steps += int(e.counters()[:, 0].sum())
        del e
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    dims = np.array([m.dim for m in models])[idx]
    out = {"metric": "MCWF trajectory-steps/s", "value": value, "unit": "trajectory-steps/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": r_ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if args.precision == "fp64" else "f32-state/f64-control", "data": "synthetic",
           "config": {"workload": args.workload, "systems": n_sys, "trajectories_per_system": per,
                      "n_traj": n_traj, "dim_range": [int(dims.min()), int(dims.max())], "Dt_per_step": Dt,
                      "rng": args.rng, "kernel_groups": plan,
                      "l2_flush": "not needed: states stay on chip"},
           "plain_fp64": {"value": plain_value, "unit": "trajectory-steps/s",
                          "how": "one FP64 ensemble per system and launch, sequential, same Dt intervals"},
           "batched_vs_plain": value / plain_value,
           "precision_check": precision_check,
           "e2e": {"value": e2e_steps / e2e_s, "unit": "trajectory-steps/s",
                   "h2d_bytes_per_step": sum(m.dim for m in models) * (16 if args.precision == "fp64" else 8)
                   + n_traj * (8 + 8 + 4 + 8 * 4 + 32 + 64),
                   "d2h_bytes_per_step": (models[0].n_avr + 1) * 8},
           "roofline": {"bound": "fp64" if args.precision == "fp64" else "fp32", "achieved": achieved,
                        "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                        "peak_source": "measured FMA probe (cqg_probe_fma_peaks) on this GPU"},
           "clocks": clocks, "gpu_launches": sum(1 for _ in plan) * args.steps + 2 * args.steps,
           "counters": {"accepted_steps": steps_total, "ode_attempts": float(d[:, 1].sum()),
                        "kernel_ms": k_ms}}
    return out


def run_serving(args, dev):
    """Requests arrive on a seeded Poisson schedule in real time; the server admits them
    between rounds (continuous batching) and each is timed from its scheduled arrival to
    the end of the round that retires it.  The plain path serves the same requests one at a
    time as FP64 ensembles, one launch per output interval."""
    import numpy as np
    import torch

    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A

    cfg = SERVING[args.workload]
    lib = serving_library()
    systems = [cqg.System(m.desc) for _, m in lib]
    reqs = serving_requests(cfg, lib)
    pars = lib[0][1].run_pars().mcwf
    pars.precision = A.FP64 if args.precision == "fp64" else A.FP32
    pars.rng = A.RNG_PCG64 if args.rng == "pcg64" else A.RNG_PHILOX

    def serve(requests, sampler=None):
        srv = cqg.Server(pars, hbm_budget_bytes=16 << 30, max_trajectories=1 << 17)
        psi0 = [m.initial_state() for _, m in lib]
        arrival = {}
        done = {}
        k = 0
        if sampler:
            sampler.start()
        t0 = time.perf_counter()
        while len(done) < len(requests):
            now = time.perf_counter() - t0
            while k < len(requests) and requests[k][0] <= now:
                a, j, n, stream = requests[k]
                rid = srv.submit(systems[j], psi0[j], n, cfg["T"], cfg["Dt"], stream)
                arrival[rid] = (a, k)
                k += 1
            active, waiting = srv.round()
            now = time.perf_counter() - t0
            for rid in srv.completed():
                rows, steps, _, status = srv.result(rid)
                done[rid] = (now - arrival[rid][0], steps, status)
            if active == 0 and waiting == 0 and k < len(requests):
                time.sleep(max(0.0, requests[k][0] - (time.perf_counter() - t0)))
        wall = time.perf_counter() - t0
        clocks = sampler.stop() if sampler else None
        steps, kernel_ms, rounds = srv.stats()
        lat = np.array([v[0] for v in done.values()]) * 1e3
        bad = sum(1 for v in done.values() if v[2])
        return {"wall_s": wall, "steps": steps, "kernel_ms": kernel_ms, "rounds": rounds, "lat_ms": lat,
                "failed": bad, "clocks": clocks}

    # warm-up: a few requests through a fresh server
    serve([(0.0,) + r[1:] for r in reqs[:max(3, args.warmup)]])
    res = serve(reqs, ClockSampler(dev))
    lat = res["lat_ms"]

    # plain: one FP64 ensemble per request, one launch per output interval, sequentially
    plain_steps = 0
    plain_ms = 0.0
    p64 = lib[0][1].run_pars().mcwf
    p64.precision = A.FP64
    nInt = int(round(cfg["T"] / cfg["Dt"]))
    for (a, j, n, stream) in reqs:
        p64.prng_stream = stream
        e = cqg.Ensemble(systems[j], lib[j][1].initial_state(), n, p64)
        e.run(cfg["Dt"], 1)  # the first run of an ensemble allocates its output buffers
        plain_ms += e.last_ms()[0]
        for _ in range(nInt - 1):
            e.run(cfg["Dt"], 1)
            plain_ms += e.last_ms()[0]
        plain_steps += int(e.counters()[:, 0].sum())
        del e
    plain_value = plain_steps / (plain_ms * 1e-3)
    value = res["steps"] / res["wall_s"]
    device_value = res["steps"] / (res["kernel_ms"] * 1e-3)
    offered = sum(r[2] for r in reqs)
    return {"metric": "MCWF trajectory-steps/s", "value": value, "unit": "trajectory-steps/s", "n_gpus": 1,
            "steps": len(reqs), "warmup": max(3, args.warmup), "ms_per_step": res["wall_s"] * 1e3 / len(reqs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-state/f64-control", "data": "synthetic",
            "config": {"workload": args.workload, "arrival_rate_per_s": cfg["rate"], "requests": len(reqs),
                       "trajectories": offered, "T": cfg["T"], "Dt": cfg["Dt"], "library_systems": len(lib),
                       "hbm_budget_bytes": 16 << 30, "step": "one request (arrival to retirement)"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max()), "mean": float(lat.mean())},
            "device_value": device_value, "rounds": res["rounds"], "failed_requests": res["failed"],
            "plain_fp64": {"value": plain_value, "unit": "trajectory-steps/s",
                           "how": "every request as one FP64 ensemble, one launch per Dt, sequential; "
                                  "device time of the MCWF launches"},
            "served_device_vs_plain": device_value / plain_value,
            "clocks": res["clocks"], "gpu_launches": None,
            "e2e": {"value": value, "unit": "trajectory-steps/s", "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": None}}


# Correctness check 2 of the bench's default line: the FP64 master equation of the qubit-mode
# workload over t in [0, 20], computed by the oracle and committed as a fixture (a CPU test
# recomputes it and requires the same numbers).
MASTER_FIXTURE = os.path.join(ROOT, "tests", "golden", "master_equation_runs.json")


def bonferroni_z(n_comparisons, sigmas=3.0):
    """Per-point z threshold of a 3-sigma family-wise test over n_comparisons points."""
    from scipy.stats import norm
    return float(norm.isf(2 * norm.sf(sigmas) / (2 * n_comparisons)))


def accuracy_summary(precision, n_traj=4096):
    """Ensemble averages of the qubit-mode workload (t in [0, 20], Dt = 1, from the vacuum)
    against the FP64 master equation: per output time and observable, the distance in units
    of the ensemble's standard error (per-trajectory values)."""
    import numpy as np

    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A

    ref = json.load(open(MASTER_FIXTURE))["qbitmode_jc_2x40"]
    model = cqg.Model(ref["script"], ref["args"])
    pars = model.run_pars().mcwf
    pars.precision = precision
    ens = cqg.Ensemble(cqg.System(model.desc), model.initial_state(), n_traj, pars)
    K = int(round(ref["T"] / ref["Dt"]))
    master = np.array(ref["rows"])[1:, 2:]
    z = np.zeros((K, 4))
    for k in range(K):
        ens.run(ref["Dt"], 1)
        per = ens.traj_averages()[:, :model.n_avr]
        # <n>, Re<a>, Im<a>, <sigma_z> = rho11 - rho00 (columns of the qubit-mode key)
        obs = np.stack([per[:, 4], per[:, 6], per[:, 7], per[:, 1] - per[:, 0]], axis=1)
        want = np.array([master[k, 4], master[k, 6], master[k, 7], master[k, 1] - master[k, 0]])
        se = obs.std(axis=0, ddof=1) / np.sqrt(n_traj)
        # an observable that is the same in every trajectory (Im<a> = 0 here) has no spread:
        # floor the error by the integrators' accuracy
        floor = 1e-6 if precision == A.FP64 else 1e-4
        z[k] = np.abs(obs.mean(axis=0) - want) / np.sqrt(se ** 2 + floor ** 2)
    return {"observables": ["<n>", "Re<a>", "Im<a>", "<sigma_z>"], "t": [ref["Dt"] * (k + 1) for k in range(K)],
            "sigma": np.round(z, 3).tolist(), "max_sigma_per_observable": np.round(z.max(axis=0), 3).tolist(),
            "max_sigma": float(z.max()), "bonferroni_3sigma_threshold": bonferroni_z(z.size),
            "within_3sigma": bool(z.max() < bonferroni_z(z.size))}


def uneven_summary(rng, steps=3, warmup=1):
    """The uneven batch (256 driven Jaynes-Cummings systems, D in [40, 240], 64 trajectories
    each): one batch in FP32-state and in FP64, against the plain path (one FP64 ensemble
    per system and launch, one after another), over the same Dt intervals; device time of
    the run calls.  Also the FP32 batch means against the FP64 batch (same streams)."""
    import numpy as np
    import torch

    import cppqed_b200 as cqg
    from cppqed_b200 import _abi as A

    n_sys, per, Dt = UNEVEN["uneven_jc_16384"]
    models = uneven_models(n_sys)
    systems = [cqg.System(m.desc) for m in models]
    idx = np.repeat(np.arange(n_sys), per)
    psi0s = [models[j].initial_state() for j in idx]

    def pars_for(precision, stream=1):
        p = models[0].run_pars().mcwf
        p.rng = A.RNG_PCG64 if rng == "pcg64" else A.RNG_PHILOX
        p.precision = precision
        p.prng_stream = stream
        return p

    def timed(ens):
        for _ in range(warmup):
            ens.run(Dt, 1)
        c0 = ens.counters()[:, 0].astype(np.int64)
        ms = 0.0
        for _ in range(steps):
            ens.run(Dt, 1)
            ms += ens.last_ms()[1]
        return int((ens.counters()[:, 0].astype(np.int64) - c0).sum()), ms

    out = {}
    means = {}
    for name, prec in (("batched_fp32", A.FP32), ("batched_fp64", A.FP64)):
        ens = cqg.Ensemble.batch(systems, idx, psi0s, pars_for(prec))
        st, ms = timed(ens)
        out[name] = st / (ms * 1e-3)
        means[name] = ens.traj_averages()[:, :models[0].n_avr]
        del ens
    p_steps, p_ms = 0, 0.0
    for j in range(n_sys):
        e = cqg.Ensemble(systems[j], models[j].initial_state(), per, pars_for(A.FP64, 1 + j * per))
        st, ms = timed(e)
        p_steps += st
        p_ms += ms
        del e
    torch.cuda.synchronize()
    out["plain_fp64"] = p_steps / (p_ms * 1e-3)
    out["batched_fp32_vs_plain_fp64"] = out["batched_fp32"] / out["plain_fp64"]
    out["batched_fp64_vs_plain_fp64"] = out["batched_fp64"] / out["plain_fp64"]
    out["fp32_vs_fp64_batched"] = out["batched_fp32"] / out["batched_fp64"]
    a64, a32 = means["batched_fp64"], means["batched_fp32"]
    se = a64.std(axis=0, ddof=1) / np.sqrt(len(a64))
    z = np.abs(a32.mean(axis=0) - a64.mean(axis=0)) / np.where(se > 0, se, np.inf)
    out["fp32_vs_fp64_batch_means_max_sigma"] = float(z.max())
    out["config"] = {"systems": n_sys, "trajectories_per_system": per, "Dt": Dt, "warmup_intervals": warmup,
                     "timed_intervals": steps, "unit": "trajectory-steps/s (device time of the run calls)"}
    return out


def north_star_checks(args, dev):
    """Extra keys of the default line: batched and served throughput against the plain
    one-ensemble-per-launch FP64 path, and the accuracy of the FP64 and FP32-state ensembles
    against the FP64 master equation."""
    from cppqed_b200 import _abi as A

    out = {"uneven_batch": uneven_summary(args.rng)}
    out["accuracy_vs_master_equation"] = {
        "workload": "qbitmode_jc_2x40, 4096 trajectories, t in [0, 20], Dt = 1",
        "reference": "FP64 master equation of the oracle (tests/golden/master_equation_runs.json)",
        "fp64": accuracy_summary(A.FP64), "fp32_state": accuracy_summary(A.FP32)}
    sargs = argparse.Namespace(**vars(args))
    sargs.workload = "serving_poisson_200"
    sargs.precision = "fp32"
    srv = run_serving(sargs, dev)
    out["serving"] = {"workload": sargs.workload, "precision": "fp32-state/fp64-control",
                      "latency_ms": srv["latency_ms"], "served_wall_steps_per_s": srv["value"],
                      "served_device_steps_per_s": srv["device_value"],
                      "plain_fp64_device_steps_per_s": srv["plain_fp64"]["value"],
                      "served_device_vs_plain_fp64": srv["served_device_vs_plain"],
                      "requests": srv["config"]["requests"], "failed_requests": srv["failed_requests"]}
    return out


def cpu_sample(args, threads, seconds):
    """Times the oracle (the reference's serial algorithm: Ensemble::advance trajectory by
    trajectory, the density-operator average at every Dt) on a sample of the workload's
    trajectories over the same time window as the device arm: args.warmup untimed intervals
    of Dt, then args.steps timed ones.  The sample (the first n of the trajectories, the same
    random streams) is sized so that the timed part takes about `seconds` on `threads`
    host threads."""
    import cppqed_b200 as cqg
    from tests.oracle_lib import Oracle

    script, sargs, n_traj, Dt = WORKLOADS[args.workload]
    model = cqg.Model(script, sargs)
    pars = model.run_pars().mcwf
    orc = Oracle()
    W, K = args.warmup, max(args.steps, 1)
    # calibrate on a few trajectories: cost of one interval after the warm-up
    probe = max(threads, 4)
    _, secs, _ = orc.ensemble_bench(model, pars, probe, Dt, 1, threads, 1, warm_intervals=W)
    per_traj_interval = secs * threads / probe
    n = int(seconds * threads / (K * max(per_traj_interval, 1e-6)))
    n = max(threads, min(n_traj, n - n % threads if n > threads else threads))
    steps, secs, _ = orc.ensemble_bench(model, pars, n, Dt, K, threads, 1, warm_intervals=W)
    return {"value": steps / secs, "unit": "trajectory-steps/s", "cores": threads, "kind": "port",
            "sample": "trajectories 1..%d of the %d of %s (the same random streams) through the device arm's "
                      "window t in [%g, %g]: %d untimed warm-up intervals, then %d timed intervals of Dt = %g; "
                      "serial Ensemble::advance + rho average per Dt, trajectories split over %d host threads" %
                      (n, n_traj, args.workload, W * Dt, (W + K) * Dt, W, K, Dt, threads),
            "steps": steps, "seconds": secs, "n_sample": n}


def workload_config(args, world):
    """The bench line's config, the same for the device arm and the reference arm."""
    script, sargs, n_traj, Dt = WORKLOADS[args.workload]
    return {"workload": args.workload, "script": script, "args": " ".join(sargs), "n_traj_per_gpu": n_traj,
            "Dt_per_step": Dt, "t_window": [args.warmup * Dt, (args.warmup + args.steps) * Dt], "rng": args.rng,
            "l2_flush": "not needed: states stay on chip; per-step HBM traffic is the state read/write",
            "parallelism": "trajectory-sharded x%d" % world}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and "RANK" in os.environ:
        world = int(os.environ["WORLD_SIZE"])
    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        r = cpu_sample(args, threads, args.cpu_sample_seconds)
        value = r["value"]
        out = {"metric": "MCWF trajectory-steps/s", "value": value, "unit": "trajectory-steps/s",
               "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": 1e3 * r["seconds"] / max(args.steps, 1), "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": workload_config(args, args.gpus),
               "impl": "reference",
               "cpu_baseline": {"value": value, "unit": "trajectory-steps/s", "cores": threads, "kind": "port",
                                "sample": r["sample"]},
               "e2e": {"value": value, "unit": "trajectory-steps/s", "h2d_bytes_per_step": 0,
                       "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    import torch
    torch.cuda.set_device(local)
    if args.workload in UNEVEN:
        print(json.dumps(run_batched(args, local)))
        return
    if args.workload in SERVING:
        print(json.dumps(run_serving(args, local)))
        return
    if args.apply_states:
        import cppqed_b200 as cqg
        script, sargs, _, _ = WORKLOADS[args.workload]
        print(json.dumps(run_apply(cqg.Model(script, sargs), n_states=args.apply_states,
                                   warmup=args.warmup, reps=args.apply_reps)))
        return
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    r = run_ours(args, rank, world, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(args, 1, args.cpu_sample_seconds)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    extras = None
    if rank == 0 and world == 1 and not args.no_extras and args.workload == "qbitmode_jc_2x40":
        extras = north_star_checks(args, local)
    if rank == 0:
        script, sargs, n_traj, Dt = WORKLOADS[args.workload]
        out = {"metric": "MCWF trajectory-steps/s", "value": r["value"], "unit": "trajectory-steps/s",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64" if args.precision == "fp64" else "f32-state/f64-control", "data": "synthetic",
               "config": workload_config(args, world), "kernel_groups": r["plan"],
               "e2e": r["e2e"], "roofline": r["roofline"], "apply_roofline": r["apply"], "cpu_baseline": cpu,
               "clocks": r["clocks"],
               "gpu_launches": 3 * args.steps,
               "counters": {"accepted_steps": r["steps_total"], "ode_attempts": r["attempts_total"],
                            "rhs_evaluations": r["rhs_total"], "failed_attempts": r["failed_total"],
                            "dp_limit_overshoots": r["overshoots_total"], "step_backs": r["stepbacks_total"],
                            "jumps": r["jumps_total"], "kernel_ms": r["kernel_ms"]}}
        if extras is not None:
            out["north_star"] = extras
        print(json.dumps(out))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

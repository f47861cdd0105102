"""Benchmark: beam-splitter updates per second of the MPO boson-sampling circuit.

Workload (synthetic, seeded): N = 64 modes, lossy single photons (eta = 0.3) in the
even modes, Fock cutoff d = 5, bond dimension chi = 1024, complex128; the
interferometer is a seeded Haar unitary (seed 1003) decomposed into a 2016-BS
Clements mesh of 64 brick-wall layers.  One step = one brick-wall layer (31 or 32
beam-splitter updates) in the middle of the circuit, where every interior bond is
saturated at chi = 1024.  The circuit is advanced untimed to layer `--start-layer`,
then W warm-up layers and K timed layers follow.

Arms:
  default            the sm_100a library (libbsmpo) on every rank (replicas)
  --impl reference   the CPU restatement of the reference's CPU update (oracle/) on
                     this host's cores, on a bounded sample of the same circuit
Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
# libbsmpo runs a layer's beam splitters on several streams at once: give the process as
# many hardware work queues as it has worker streams (process-local; read when CUDA
# initialises, so set before torch is imported)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
# load every kernel module at context creation: a module loaded lazily by its first
# launch inside the timed region would stall the concurrent updates
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")
sys.path.insert(0, ROOT)

WORKLOADS = {
    "chi1024": dict(name="boson-sampling MPO, N=64, 32 photons (even modes), eta=0.3, d=5, chi=1024, "
                         "Haar seed 1003 -> 2016-BS Clements mesh",
                    n=64, eta=0.3, d=5, chi=1024, seed=1003),
    # smaller workload (profiling / parity sizes): N=32, 16 photons, eta=0.5, d=4, chi=256
    "chi256": dict(name="boson-sampling MPO, N=32, 16 photons (even modes), eta=0.5, d=4, chi=256, "
                        "Haar seed 1002 -> 496-BS Clements mesh",
                   n=32, eta=0.5, d=4, chi=256, seed=1002),
}
WORKLOAD = WORKLOADS["chi1024"]
METRIC = "BS-updates/s & circuit time at \u03c7=1024 vs plain FP64 GPU path at \u22641e-6 prob err"
# arithmetic type of each path
DTYPES = {"fp64": "f64", "fp64-gram": "f64", "tf32x3": "tf32x3 contractions + f64 Gram/eigen"}
SVD_KERNELS = {"fp64": "jacobi_gram_kernel + jacobi_apply_kernel (one-sided Jacobi SVD rounds)",
               "fp64-gram": "zgemm_grouped_kernel (Gram) + tridiag_kernel + bisect_kernel (Gram route SVD)",
               "tf32x3": "zgemm_grouped_kernel (Gram) + tridiag_kernel + bisect_kernel (Gram route SVD)"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--start-layer", type=int, default=10)
    p.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work per sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-circuit", action="store_true",
                   help="skip the whole-circuit run (all updates from the initial state)")
    p.add_argument("--workload", default="chi1024", choices=sorted(WORKLOADS))
    p.add_argument("--precision", default="fp64-gram", choices=sorted(DTYPES),
                   help="the measured path: fp64-gram (Gram matrix + Hermitian eigenproblem, the "
                        "default) or fp64 (the plain path: one-sided Jacobi)")
    p.add_argument("--workers", type=int, default=0, help="concurrent updates (0: 16, or 8 for fp64)")
    p.add_argument("--also", default="tf32x3",
                   help="comma-separated further precision forms timed on the same layers and "
                        "checked over the whole circuit ('' for none)")
    p.add_argument("--batch", type=int, default=64,
                   help="independent circuits of the batched workload (N in [16, 48], eta in "
                        "[0.2, 0.8], d=4, chi in {128, 256, 512}) run side by side and one by one "
                        "(0: skip)")
    p.add_argument("--batch-conc", default="4,8",
                   help="comma-separated numbers of circuits run side by side in the batched form "
                        "(the fastest is reported)")
    p.add_argument("--no-grad", action="store_true",
                   help="skip the differentiation form (N=24, d=4, chi=256 gradients of a marginal "
                        "loss, checked against central finite differences)")
    p.add_argument("--no-plain", action="store_true",
                   help="skip the plain FP64 path (the metric's denominator) and the error against it")
    p.add_argument("--bs-slice", default=None,
                   help="profiling runs only: START:STOP -- a step runs beam splitters START..STOP-1 "
                        "of its layer (default: the whole layer)")
    p.add_argument("--state-cache", default=None,
                   help="file holding the state at --start-layer: loaded if present (the untimed "
                        "set-up layers are skipped), else written after them; for profiling runs, "
                        "whose per-launch overhead makes the set-up layers slow")
    a = p.parse_args()
    global WORKLOAD, METRIC
    WORKLOAD = WORKLOADS[a.workload]
    if a.workload != "chi1024":
        METRIC = "BS-updates/s (%s circuit) vs plain FP64 GPU path" % a.workload
    return a


def config_dict(args, workers):
    """The workload and how a step is timed (the same dict on both arms)."""
    return {"workload": WORKLOAD["name"],
            "start_layer": args.start_layer,
            "l2": "inputs larger than L2 (state 1.07 GB)" if WORKLOAD["chi"] >= 1024 else "state below L2 size",
            "bs_slice": args.bs_slice or "whole layer", "cutoff": 0.0}


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons while the timed region runs.

    Reads them in-process through NVML every 0.5 s (a spawned nvidia-smi per sample
    initialises NVML each time and competes with the timed process for the driver);
    falls back to nvidia-smi when NVML is not importable.  Reads only."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, cuda_index, period=0.5):
        self.cuda_index = cuda_index
        self.period = period
        self.samples = []   # (sm_mhz, sm_max_mhz, watts, set of reasons)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(cuda_index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            self._h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self._nvml = pynvml
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        n, h = self._nvml, self._h
        sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)
        w = n.nvmlDeviceGetPowerUsage(h) / 1e3
        bits = n.nvmlDeviceGetCurrentClocksEventReasons(h)
        return (float(sm), float(mx), w, {name for name, bit in self.REASONS if bits & bit})

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", "-i", str(self.cuda_index), "--query-gpu=" + self.FIELDS,
                              "--format=csv,noheader,nounits"], capture_output=True,
                             text=True, timeout=5).stdout.strip()
        f = [x.strip() for x in out.split(",")]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        return (float(f[1]), float(f[2]), float(f[3]) if f[3].replace(".", "").isdigit() else 0.0,
                {nm for nm, v in zip(names, f[5:9]) if v.lower() == "active"})

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._sample_nvml() if self._nvml else self._sample_smi())
            except Exception:
                pass
            self._stop.wait(self.period)

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set()
        for smp in self.samples:
            reasons |= smp[3]
        return {"sm_mhz": float(np.median([x[0] for x in self.samples])),
                "sm_max_mhz": max(x[1] for x in self.samples),
                "power_w_max": round(max(x[2] for x in self.samples), 1),
                "reasons": sorted(reasons), "samples": len(self.samples),
                "source": "nvml" if self._nvml else "nvidia-smi"}


def max_over_ranks(x, dist, device):
    """The largest x over the ranks of the process group (x itself on one rank): every
    multi-rank time is the slowest rank's."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(n_units_per_rank, world, seconds):
    """Whole-job rate of `world` replicas that each process n_units_per_rank units, timed
    as the slowest rank's seconds (weak scaling)."""
    return world * n_units_per_rank / seconds


def layers_of(bs):
    n_layers = max(b[0] for b in bs) + 1
    out = [[] for _ in range(n_layers)]
    for (layer, m, th, ph) in bs:
        out[layer].append((m, th, ph))
    return out


def measure_hbm_peak(torch):
    """Copy bandwidth (torch copy of 1 GiB, read + write counted, best of 10): the HBM
    roofline measured in the same run."""
    n = 1 << 30
    a = torch.empty(n, dtype=torch.uint8, device="cuda")
    b = torch.empty_like(a)
    b.copy_(a)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.copy_(a)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n / best / 1e9


def measure_fp64_peak(torch):
    """DGEMM TFLOP/s (torch.matmul float64 8192^3, best of 5) -- the FP64 roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def cpu_sample(budget_s, layers, start_layer=None, state=None):
    """Oracle (CPU restatement) on a bounded sample of the circuit: BS-updates/s."""
    from threadpoolctl import threadpool_info

    from oracle import fock, interferometer, mpo
    w = WORKLOAD
    if state is None:
        st = mpo.initial_state(w["n"], range(0, w["n"], 2), w["eta"], w["d"], w["chi"])
        seq = [op for layer in layers for op in layer]
        label = "first BSs of the circuit from the initial state (small bond dimensions)"
    else:
        st = state
        seq = [op for layer in layers[start_layer:] for op in layer]
        label = "BSs of layer %d onward from the mid-circuit state (bond dimension 1024)" % start_layer
    t0 = time.perf_counter()
    done = 0
    for (m, th, ph) in seq:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, ph), w["d"]))
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    threads = max([i.get("num_threads", 1) for i in threadpool_info()] + [1])
    return {"value": done / el, "unit": "BS-updates/s", "cores": int(threads), "kind": "port",
            "sample": "%d BS updates in %.1f s: %s" % (done, el, label)}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference update on this host's
    cores, on the same workload as our arm -- advanced untimed to --start-layer, then W
    short warm-up samples and K timed samples that continue the circuit from there (each
    a bounded number of updates, --cpu-budget seconds of timed work in total)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from threadpoolctl import threadpool_info

    from bosonsampling_b200 import interferometer
    from oracle import fock, mpo
    w = WORKLOAD
    U, bs, ph = interferometer.circuit(w["n"], w["seed"])
    layers = layers_of(bs)
    st = mpo.initial_state(w["n"], range(0, w["n"], 2), w["eta"], w["d"], w["chi"])
    t_setup = time.perf_counter()
    for L in range(args.start_layer):
        for (m, th, p) in layers[L]:
            mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, p), w["d"]))
    t_setup = time.perf_counter() - t_setup
    seq = iter([op for L in layers[args.start_layer:] for op in L])

    def sample(budget_s):
        t0 = time.perf_counter()
        done = 0
        for (m, th, p) in seq:
            mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, p), w["d"]))
            done += 1
            if time.perf_counter() - t0 > budget_s:
                break
        return done, time.perf_counter() - t0

    for _ in range(args.warmup):
        sample(0.0)                       # one update each
    timed = [sample(args.cpu_budget / max(1, args.steps)) for _ in range(args.steps)]
    n_done = sum(x[0] for x in timed)
    el = sum(x[1] for x in timed)
    v = n_done / el
    threads = max([i.get("num_threads", 1) for i in threadpool_info()] + [1])
    cb = {"value": v, "unit": "BS-updates/s", "cores": int(threads), "kind": "port",
          "sample": "%d BS updates in %.1f s from layer %d of the circuit (bond dimension %d), "
                    "after %.0f s of untimed set-up" % (n_done, el, args.start_layer,
                                                       max(mpo.bond_dims(st)), t_setup)}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "BS-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args, 0),
            "path": "CPU restatement of the reference update (oracle/), FP64, all BLAS threads",
            "step": "a bounded sample of the circuit's BS updates from layer %d on (one CPU layer takes "
                    "~15 s)" % args.start_layer,
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "BS-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# DRAM bytes (read + write) of one tridiag_kernel launch of the largest size class
# (8-CTA clusters, the biggest sector of a centre update at chi = 1024), from the ncu
# capture summarised under profiles/ (cold cache)
TRIDIAG_TRAFFIC = 2941184   # 2.836 MB read + 0.105 MB written


def measured_peaks(path=os.path.join(ROOT, "MEASURED_PEAKS.json")):
    """The pool's measured peaks (copy bandwidth ``hbm_gbs``, bf16 GEMM), or None."""
    try:
        with open(path) as f:
            peaks = json.load(f)
        return peaks if isinstance(peaks, dict) else None
    except (OSError, ValueError):
        return None


def roofline(args, mine, kernel, fp64_peak, hbm_peak, peaks=None):
    """The dominant kernel's roofline.  Gram route: the Householder tridiagonalisation
    (tridiag_kernel, 66-71% of the update's kernel time), whose fused passes stream the
    trailing matrix once per step (read + write, 32 B per complex entry): achieved
    bytes / device time of the phase, one worker, against the pool's measured copy
    bandwidth (``peaks["hbm_gbs"]``), or the copy bandwidth measured in this run when
    that is absent (both reported).  Plain path: the Jacobi rounds' FP64 flops against
    DGEMM measured in this run (the pool's file holds no FP64 figure)."""
    if kernel is not None and kernel["ms"] > 0:
        achieved = kernel["bytes"] / (kernel["ms"] / 1e3) / 1e9
        pool = float(peaks["hbm_gbs"]) if peaks and peaks.get("hbm_gbs") else None
        peak = pool if pool else hbm_peak
        return {"kernel": "tridiag_kernel (Householder tridiagonalisation, four forked size-class launches)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if peak else None,
                "frac_of": "measured",
                "peak_source": ("MEASURED_PEAKS.json hbm_gbs: copy bandwidth measured on this pool's B200s"
                                if pool else
                                "copy bandwidth measured in this run (torch copy of 1 GiB, best of 10)"),
                "peak_in_run": hbm_peak,
                "frac_of_in_run": achieved / hbm_peak if hbm_peak else None,
                "achieved_over": "the phase's device time (CUDA events), one worker, one layer (%d phases)"
                                 % kernel["phases"],
                "bytes": kernel["bytes"], "ms": kernel["ms"],
                "flops_tflops": kernel["flops"] / (kernel["ms"] / 1e3) / 1e12,
                "traffic": TRIDIAG_TRAFFIC, "traffic_unit": "bytes per launch (largest class)"}
    achieved = mine["svd_flops"] / mine["seconds"] / 1e12 if mine["seconds"] > 0 else None
    return {"kernel": SVD_KERNELS[args.precision], "bound": "tensor", "achieved": achieved, "peak": fp64_peak,
            "unit": "TFLOP/s", "frac": (achieved / fp64_peak) if achieved and fp64_peak else None,
            "frac_of": "measured",
            "peak_source": "FP64 DGEMM measured in this run (torch.matmul 8192^3, best of 5)",
            "achieved_over": "timed region (device time); the SVD phases of concurrent updates overlap",
            "traffic": None}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    from bosonsampling_b200 import engine, interferometer

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    w = WORKLOAD
    U, bs, out_phases = interferometer.circuit(w["n"], w["seed"])
    layers = layers_of(bs)
    need = args.start_layer + args.warmup + args.steps
    if need > len(layers):
        raise SystemExit("start-layer + warmup + steps exceeds the %d layers" % len(layers))
    workers = args.workers or (8 if args.precision == "fp64" else 16)
    sim = engine.MPOSimulator(w["n"], w["d"], w["chi"])
    sim.set_workers(workers)
    sim.init_single_photons(range(0, w["n"], 2), w["eta"])

    bs_slice = slice(*[int(x) for x in args.bs_slice.split(":")]) if args.bs_slice else slice(None)

    def layer_ops(L0, count, partial=False):
        return [op for L in range(L0, L0 + count) for op in (layers[L][bs_slice] if partial else layers[L])]

    def run_layers(h, L0, count, partial=False):
        # one library call for `count` consecutive layers, as a whole-circuit run makes it
        # (the library overlaps consecutive layers' independent updates)
        ops = layer_ops(L0, count, partial)
        if ops:
            h.run_mesh([m for (m, _, _) in ops], [t for (_, t, _) in ops], [p for (_, _, p) in ops])

    # untimed: advance to the saturated middle of the circuit on the plain FP64 path, so
    # both paths time the same layers from the same state
    t_setup = time.perf_counter()
    cache = args.state_cache
    if cache and os.path.exists(cache):
        saved = torch.load(cache)
        if saved["workload"] != w["name"] or saved["start_layer"] != args.start_layer:
            raise SystemExit("--state-cache %s holds another workload or start layer" % cache)
        sim.load(saved["gamma"].cuda(), saved["lam"].cuda(), saved["charge"].cuda())
        del saved
    else:
        run_layers(sim, 0, args.start_layer)
        if cache:
            g, l, c = sim.store()
            torch.save({"workload": w["name"], "start_layer": args.start_layer,
                        "gamma": g.cpu(), "lam": l.cpu(), "charge": c.cpu()}, cache)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    dims = sim.bond_dims()
    g0, l0, c0 = sim.store()          # state at --start-layer (device copy)

    first = args.start_layer + args.warmup
    n_bs = len(layer_ops(first, args.steps, partial=True))

    def timed_layers(precision, n_workers):
        """W warm-up layers then K timed layers from the start state; device seconds."""
        sim.load(g0, l0, c0)
        sim.set_precision(precision)
        sim.set_workers(n_workers)
        run_layers(sim, args.start_layer, args.warmup)
        torch.cuda.synchronize()
        sim.set_timing(True)
        launches0 = sim.kernel_launches()
        routes0 = sim.svd_routes()
        ws0 = sim.workspace_stats()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local)
        sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")
        e0.record()
        run_layers(sim, first, args.steps, partial=True)
        e1.record()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        sampler.stop()
        launches = sim.kernel_launches() - launches0
        routes = [a - b for a, b in zip(sim.svd_routes(), routes0)]
        ws1 = sim.workspace_stats()
        svd_ms, svd_flops, svd_launches = sim.jacobi_timing()
        sim.set_timing(False)
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, "cuda")
        tr, P = sim.observables()
        return {"seconds": t, "launches": launches, "svd_ms": svd_ms, "svd_flops": svd_flops,
                "svd_launches": svd_launches, "clocks": sampler.summary(), "trace": tr, "P": P,
                "routes": {"jacobi": routes[0], "gram": routes[1]},
                "workspace_grows": {"device": ws1[0] - ws0[0], "pinned": ws1[1] - ws0[1],
                                    "device_bytes": ws1[2], "pinned_bytes": ws1[3]}}

    # ---- timed, device-resident: the measured path, then the plain FP64 path on the same
    # layers from the same state (the metric's denominator)
    mine = timed_layers(args.precision, workers)
    value = replica_rate(n_bs, world, mine["seconds"])
    plain = None
    if args.precision != "fp64" and not args.no_plain:
        plain = timed_layers("fp64", 8)
        plain["value"] = replica_rate(n_bs, world, plain["seconds"])
    extras = {}
    also = [x for x in args.also.split(",") if x and x != args.precision]
    for form in also:
        r = timed_layers(form, workers)
        r["value"] = replica_rate(n_bs, world, r["seconds"])
        extras[form] = r
    if world > 1:
        dist.barrier()

    # ---- the dominant kernel alone: one worker, one layer, the tridiagonalisation phase
    # timed with CUDA events around its launches (the Gram route's forked size classes)
    kernel = None
    if args.precision != "fp64":
        sim.load(g0, l0, c0)
        sim.set_precision(args.precision)
        sim.set_workers(1)
        run_layers(sim, args.start_layer, args.warmup)
        sim.set_timing(True)
        run_layers(sim, first, 1, partial=True)
        torch.cuda.synchronize()
        td_ms, td_bytes, td_flops, td_phases = sim.tridiag_timing()
        sim.set_timing(False)
        kernel = {"ms": td_ms, "bytes": td_bytes, "flops": td_flops, "phases": td_phases}

    # ---- end to end through the public API with host buffers, over the same K layers: per
    # step (layer) the state goes host -> device, the layer runs, the state comes back
    # device -> host (the next step's input) and the trace is read.  The measured form
    # streams the state (run_mesh_host: per-site copies overlapping the updates); the
    # sequential form copies the whole state in, runs the layer, then copies it out
    def layer_args(L):
        ops = layer_ops(L, 1, True)
        return [m for (m, _, _) in ops], [t for (_, t, _) in ops], [p for (_, _, p) in ops]

    sim.load(g0, l0, c0)
    sim.set_precision(args.precision)
    sim.set_workers(workers)
    run_layers(sim, args.start_layer, args.warmup)
    g1, l1, c1 = sim.store()
    start_host = [g1.cpu().pin_memory(), l1.cpu().pin_memory(), c1.cpu().pin_memory()]
    del g1, l1, c1
    e2e_times = {}
    for form in ("streamed", "sequential"):
        host_in = [x.clone().pin_memory() for x in start_host]
        host_out = [torch.empty_like(x, pin_memory=True) for x in host_in]
        dev = [torch.empty_like(x, device="cuda") for x in host_in] if form == "sequential" else None
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(args.steps):
            if form == "streamed":
                sim.run_mesh_host(*layer_args(first + i), host_in, host_out)
            else:
                for dd, hh in zip(dev, host_in):
                    dd.copy_(hh, non_blocking=True)
                sim.load(*dev)
                sim.run_mesh(*layer_args(first + i))
                gs, ls, cs = sim.store()
                for hh, dd in zip(host_out, (gs, ls, cs)):
                    hh.copy_(dd, non_blocking=True)
            tr_e2e = sim.trace()
            torch.cuda.synchronize()
            host_in, host_out = host_out, host_in
        e2e_times[form] = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        del dev, host_in, host_out
    t_e2e = e2e_times["streamed"]
    state_bytes = sum(x.numel() * x.element_size() for x in start_host)
    h2d = state_bytes * args.steps
    d2h = (state_bytes + 16) * args.steps
    del start_host

    # ---- the whole circuit: every update from the initial state, the output phases and the
    # observables (trace, marginals), one run_mesh call, on the measured path and on the
    # plain FP64 path; the probability error is the largest marginal difference / trace
    circuit = None
    if not args.no_circuit and not args.bs_slice:
        runs = {}
        for prec in ([args.precision] + also +
                     (["fp64"] if args.precision != "fp64" and not args.no_plain else [])):
            with engine.MPOSimulator(w["n"], w["d"], w["chi"]) as full:
                full.set_precision(prec)
                full.set_workers(workers if prec == args.precision else 8)
                full.init_single_photons(range(0, w["n"], 2), w["eta"])
                torch.cuda.synchronize()
                if world > 1:
                    dist.barrier()
                t0 = time.perf_counter()
                full.run_mesh([b[1] for b in bs], [b[2] for b in bs], [b[3] for b in bs])
                tw = full.mesh_truncation()
                full.apply_phases(out_phases)
                trace_c, P_c = full.observables()
                torch.cuda.synchronize()
                runs[prec] = (max_over_ranks(time.perf_counter() - t0, dist, "cuda"), trace_c, P_c, tw)
        t_c, trace_c, P_c, tw_c = runs[args.precision]
        circuit = {"bs_updates": len(bs), "seconds": round(t_c, 3),
                   "value": replica_rate(len(bs), world, t_c), "unit": "BS-updates/s",
                   "trace": float(trace_c.real), "max_truncation_weight": float(np.max(tw_c)),
                   "covers": "all updates from the initial state, output phases, trace and marginals "
                             "(host wall clock, initial state excluded)"}
        if "fp64" in runs and args.precision != "fp64":
            t_p, trace_p, P_p, tw_p = runs["fp64"]
            circuit["plain_fp64_seconds"] = round(t_p, 3)
            circuit["plain_fp64_value"] = replica_rate(len(bs), world, t_p)
            circuit["prob_err_vs_fp64"] = float(np.abs(P_c - P_p).max() / abs(trace_p))
            circuit["trace_err_vs_fp64"] = float(abs(trace_c - trace_p) / abs(trace_p))
            circuit["truncation_weight_err_vs_fp64"] = float(np.abs(tw_c - tw_p).max())
            for form in also:
                t_f, trace_f, P_f, _ = runs[form]
                extras[form]["circuit"] = {"seconds": round(t_f, 3),
                                           "value": replica_rate(len(bs), world, t_f),
                                           "prob_err_vs_fp64": float(np.abs(P_f - P_p).max() / abs(trace_p))}

    # ---- batched form: independent circuits of uneven N and chi, side by side against one
    # by one (host wall clock; every circuit is computed exactly as alone)
    batched = None
    if args.batch > 0 and not args.bs_slice and world == 1:
        specs = engine.batch_circuits(n_circuits=args.batch)
        n_up = sum(len(sp["mesh"]) for sp in specs)
        engine.run_batch(specs[:2], concurrency=2, precision=args.precision)   # warm-up
        best = {}
        for conc, wk in [(1, 8)] + [(int(c), 4) for c in args.batch_conc.split(",") if int(c) > 1]:
            tm = {}
            engine.run_batch(specs, concurrency=conc, precision=args.precision, workers=wk, timing=tm)
            best[conc] = tm["seconds"]
        t_seq = best[1]
        conc_best = min((c for c in best if c > 1), key=lambda c: best[c])
        t_par = best[conc_best]
        batched = {"circuits": len(specs), "bs_updates": n_up,
                   "value": n_up / t_par, "one_by_one_value": n_up / t_seq, "unit": "BS-updates/s",
                   "speedup": t_seq / t_par, "seconds": round(t_par, 3), "one_by_one_seconds": round(t_seq, 3),
                   "n_range": [min(sp["n"] for sp in specs), max(sp["n"] for sp in specs)],
                   "chis": sorted(set(sp["chi"] for sp in specs)),
                   "concurrency": conc_best, "seconds_by_concurrency": {str(c): round(t, 3) for c, t in best.items()},
                   "how": "circuits side by side, one handle + host thread + stream each, 4 worker streams per "
                          "handle (one by one: 8); host wall clock of the meshes, output phases and "
                          "observables, handles created and initialised before"}

    # ---- differentiation form: gradients of the squared distance between the marginals
    # of one circuit and those of a second Haar circuit, with respect to every (theta,
    # phi) and eta, from the adjoint over the recorded updates; checked against
    # central finite differences of the library's forward (h = 1e-6, FP64)
    grad = None
    if not args.no_grad and not args.bs_slice and world == 1:
        from bosonsampling_b200 import adjoint
        gn, gd, gchi, geta, gseed = 24, 4, 256, 0.5, 1005
        _, gbs, gph = interferometer.circuit(gn, gseed)
        _, tbs, tph = interferometer.circuit(gn, gseed + 1)
        photons = list(range(0, gn, 2))
        gth = np.array([b[2] for b in gbs])
        gphi = np.array([b[3] for b in gbs])
        circ = adjoint.DiffCircuit(gn, gd, gchi, photons, gbs, gph)
        tc = adjoint.DiffCircuit(gn, gd, gchi, photons, tbs, tph)
        ttr, tP = tc.run(np.array([b[2] for b in tbs]), np.array([b[3] for b in tbs]), geta)
        tc.close()
        target = tP.real / ttr.real
        t0 = time.perf_counter()
        ttr2, _ = circ.run(gth, gphi, geta)
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        torch.cuda.reset_peak_memory_stats()
        t0 = time.perf_counter()
        gl, g_th, g_ph, g_eta = circ.loss_and_grad(gth, gphi, geta, target)
        torch.cuda.synchronize()
        t_grad = time.perf_counter() - t0
        peak = torch.cuda.max_memory_allocated()
        g_th, g_ph = g_th.cpu().numpy(), g_ph.cpu().numpy()

        def gloss(t, p_, e):
            trc, Pm = circ.run(t, p_, e)
            return float(((Pm.real / trc.real - target) ** 2).sum())
        h, errs, checks = 1e-6, [], []
        nb = len(gth)
        for kind, i in (("theta", 0), ("theta", nb // 2), ("theta", nb - 1), ("phi", 1), ("phi", nb // 3), ("eta", -1)):
            if kind == "eta":
                fd = (gloss(gth, gphi, geta + h) - gloss(gth, gphi, geta - h)) / (2 * h)
                g = g_eta
            else:
                vp, vm = (gth.copy(), gth.copy()) if kind == "theta" else (gphi.copy(), gphi.copy())
                vp[i] += h
                vm[i] -= h
                fd = ((gloss(vp, gphi, geta) - gloss(vm, gphi, geta)) if kind == "theta"
                      else (gloss(gth, vp, geta) - gloss(gth, vm, geta))) / (2 * h)
                g = float(g_th[i] if kind == "theta" else g_ph[i])
            errs.append((g, fd))
            checks.append({"param": kind if kind == "eta" else "%s[%d]" % (kind, i), "adjoint": g,
                           "finite_difference": fd})
        circ.close()
        # relative to each finite difference where it is significant (>= 1e-3 of the largest
        # one checked); for the others the absolute difference against that scale, which
        # the finite difference's own rounding (~1e-16 loss / h) bounds from below
        scale = max(abs(fd) for _, fd in errs)
        for c, (g, fd) in zip(checks, errs):
            c["rel_err"] = abs(g - fd) / abs(fd) if abs(fd) >= 1e-3 * scale else None
            c["abs_err_over_scale"] = abs(g - fd) / scale
        errs = [c["rel_err"] for c in checks if c["rel_err"] is not None]
        grad = {"config": "N=24, 12 photons (even modes), eta=0.5, d=4, chi=256, Haar seed %d -> %d-BS mesh; "
                          "target: marginals of Haar seed %d" % (gseed, nb, gseed + 1),
                "loss": gl, "params": 2 * nb + 1, "forward_seconds": round(t_fwd, 3),
                "loss_and_grad_seconds": round(t_grad, 3), "records": "two sites and three bonds per update",
                "peak_device_bytes": int(peak), "fd_check": checks, "fd_max_rel_err": max(errs),
                "fd_max_abs_err_over_scale": max(c["abs_err_over_scale"] for c in checks),
                "how": "library forward (plain FP64 path) update by update, keeping each update's inputs "
                       "and outputs (two sites, three bonds); hand-written adjoint of the contraction + "
                       "truncated SVD (pair-relative Lorentzian broadening) on the device; gate angles by "
                       "bsmpo_bs_angle_grad"}

    # ---- roofline of the dominant phase: the SVD step (Jacobi rounds, or the Gram GEMM,
    # Householder reduction and bisection of the Gram route), FP64 against measured DGEMM
    fp64_peak = measure_fp64_peak(torch) if rank == 0 else None
    hbm_peak = measure_hbm_peak(torch) if rank == 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import mpo as _mpo
        g, l, c = g0, l0, c0
        # the oracle times the layers after the start state (input data only; the timed
        # CPU work is the oracle's own update)
        st = _mpo.MPOState(w["n"], w["d"], w["chi"], g.cpu().numpy(), l.cpu().numpy(), c.cpu().numpy())
        cpu = cpu_sample(args.cpu_budget, [[(m, th, p) for (m, th, p) in L] for L in layers],
                         start_layer=args.start_layer, state=st)
    if rank == 0:
        # the updates overlap on several streams, so the SVD phases' flops are taken over the
        # whole timed region (device time), not over their summed per-stream durations
        achieved = mine["svd_flops"] / mine["seconds"] / 1e12 if mine["seconds"] > 0 else None
        layer_err = None
        if plain is not None:
            layer_err = float(np.abs(mine["P"] - plain["P"]).max() / abs(plain["trace"]))
        line = {
            "metric": METRIC, "value": value, "unit": "BS-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mine["seconds"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPES[args.precision],
            "data": "synthetic",
            "config": config_dict(args, workers),
            "path": "%s, %d concurrent updates" % (args.precision, workers),
            "step": "one brick-wall layer (31-32 BS updates) of layers %d-%d; the K timed layers go in one "
                    "run_mesh call" % (first, first + args.steps - 1),
            "plain_fp64": None if plain is None else {
                "value": plain["value"], "unit": "BS-updates/s", "ms_per_step": plain["seconds"] / args.steps * 1e3,
                "speedup": value / plain["value"], "launches": plain["launches"],
                "prob_err_after_timed_layers": layer_err,
                "note": "the same K layers from the same start state on the plain path (one-sided Jacobi SVD, "
                        "equal to the CPU oracle at 1e-10)"},
            "e2e": {"value": replica_rate(n_bs, world, t_e2e), "unit": "BS-updates/s",
                    "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                    "covers": "K steps, each: one layer over the host-resident state (run_mesh_host: the "
                              "state's sites stream host->device as the updates need them and device->host "
                              "as they finish), then the trace",
                    "sequential_value": replica_rate(n_bs, world, e2e_times["sequential"]),
                    "sequential_covers": "the same steps with the whole state copied in, loaded, the layer run, "
                                         "stored and copied out one after another"},
            "gpu_launches": int(mine["launches"]),
            "svd_routes": mine["routes"],
            "workspace_grows_in_timed_region": mine["workspace_grows"],
            "roofline": roofline(args, mine, kernel, fp64_peak, hbm_peak, measured_peaks()),
            "precision_forms": {form: {
                "value": r["value"], "unit": "BS-updates/s", "speedup_vs_plain": (r["value"] / plain["value"]) if plain else None,
                "prob_err_after_timed_layers": (float(np.abs(r["P"] - plain["P"]).max() / abs(plain["trace"]))
                                                if plain else None),
                "circuit": r.get("circuit")} for form, r in extras.items()},
            "clocks": mine["clocks"],
            "circuit": circuit,
            "batched": batched,
            "differentiation": grad,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    sim.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

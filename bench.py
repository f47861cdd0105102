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
METRIC = "BS-updates/s (chi=1024 circuit, plain FP64 path)"


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
        METRIC = "BS-updates/s (%s circuit, plain FP64 path)" % a.workload
    return a


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
            "config": {"workload": w["name"], "path": "CPU restatement of the reference update (oracle/)",
                       "step": "bounded sample of the circuit's BS updates from layer %d on" % args.start_layer},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "BS-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


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
    sim = engine.MPOSimulator(w["n"], w["d"], w["chi"])
    sim.init_single_photons(range(0, w["n"], 2), w["eta"])

    bs_slice = slice(*[int(x) for x in args.bs_slice.split(":")]) if args.bs_slice else slice(None)

    def run_layers(L0, count, partial=False):
        # one library call for `count` consecutive layers, as a whole-circuit run makes it
        # (the library overlaps consecutive layers' independent updates)
        ops = [op for L in range(L0, L0 + count) for op in (layers[L][bs_slice] if partial else layers[L])]
        if ops:
            sim.run_mesh([m for (m, _, _) in ops], [t for (_, t, _) in ops], [p for (_, _, p) in ops])

    def run_layer(L, partial=False):
        run_layers(L, 1, partial)

    # untimed: advance to the saturated middle of the circuit
    t_setup = time.perf_counter()
    cache = args.state_cache
    if cache and os.path.exists(cache):
        saved = torch.load(cache)
        if saved["workload"] != w["name"] or saved["start_layer"] != args.start_layer:
            raise SystemExit("--state-cache %s holds another workload or start layer" % cache)
        sim.load(saved["gamma"].cuda(), saved["lam"].cuda(), saved["charge"].cuda())
        del saved
    else:
        run_layers(0, args.start_layer)
        if cache:
            g, l, c = sim.store()
            torch.save({"workload": w["name"], "start_layer": args.start_layer,
                        "gamma": g.cpu(), "lam": l.cpu(), "charge": c.cpu()}, cache)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    dims = sim.bond_dims()
    g0, l0, c0 = sim.store()   # the timed layers restart from this state (device copy)
    g_host = g0.cpu().pin_memory()
    l_host = l0.cpu().pin_memory()
    c_host = c0.cpu().pin_memory()

    run_layers(args.start_layer, args.warmup)
    torch.cuda.synchronize()

    # ---- timed, device-resident: K layers after the warm-up ones
    first = args.start_layer + args.warmup
    n_bs = sum(len(layers[first + i][bs_slice]) for i in range(args.steps))
    sampler = ClockSampler(local)
    sim.set_timing(True)
    launches0 = sim.kernel_launches()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")
    e0.record()
    run_layers(first, args.steps, partial=True)
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    sampler.stop()
    launches = sim.kernel_launches() - launches0
    jac_ms, jac_flops, jac_launches = sim.jacobi_timing()
    sim.set_timing(False)
    t_dev = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, "cuda")
    if world > 1:
        dist.barrier()
    value = replica_rate(n_bs, world, t_dev)

    # ---- end to end through the public API with host buffers: per step the state is
    # copied host -> device and loaded, the layer runs, the state is stored and copied
    # device -> host, and the trace is read back
    e2e_steps = 1
    g_dev = torch.empty_like(g0)
    l_dev = torch.empty_like(l0)
    c_dev = torch.empty_like(c0)
    g_out = torch.empty_like(g_host, pin_memory=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        g_dev.copy_(g_host, non_blocking=True)
        l_dev.copy_(l_host, non_blocking=True)
        c_dev.copy_(c_host, non_blocking=True)
        sim.load(g_dev, l_dev, c_dev)
        run_layer(args.start_layer + i)
        g1, l1, c1 = sim.store()
        g_out.copy_(g1, non_blocking=True)
        tr = sim.trace()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    n_bs_e2e = sum(len(layers[args.start_layer + i]) for i in range(e2e_steps))
    h2d = (g_host.numel() * 16 + l_host.numel() * 8 + c_host.numel() * 4) * e2e_steps
    d2h = (g_out.numel() * 16 + 16) * e2e_steps

    # ---- the whole circuit: every update from the initial state, the output phases and
    # the observables (trace, marginals), in one run_mesh call, on a second handle
    circuit = None
    if not args.no_circuit and not args.bs_slice:
        with engine.MPOSimulator(w["n"], w["d"], w["chi"]) as full:
            full.init_single_photons(range(0, w["n"], 2), w["eta"])
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            full.run_mesh([b[1] for b in bs], [b[2] for b in bs], [b[3] for b in bs])
            full.apply_phases(out_phases)
            trace_c, _ = full.observables()
            torch.cuda.synchronize()
            t_circ = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        circuit = {"bs_updates": len(bs), "seconds": round(t_circ, 3),
                   "value": replica_rate(len(bs), world, t_circ), "unit": "BS-updates/s",
                   "trace": float(trace_c.real),
                   "covers": "all updates from the initial state, output phases, trace and marginals "
                             "(host wall clock, initial state excluded)"}

    # ---- roofline of the dominant kernel (the Jacobi round), FP64 against measured DGEMM
    fp64_peak = measure_fp64_peak(torch) if rank == 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import mpo as _mpo
        g, l, c = sim.store()
        # the oracle times the same layers from the same mid-circuit state (input data
        # only; the timed CPU work is the oracle's own update)
        st = _mpo.MPOState(w["n"], w["d"], w["chi"], g.cpu().numpy(), l.cpu().numpy(), c.cpu().numpy())
        cpu = cpu_sample(args.cpu_budget, [[(m, th, p) for (m, th, p) in L] for L in layers],
                         start_layer=args.start_layer + 1, state=st)
    if rank == 0:
        # the updates of a layer overlap on several streams, so the Jacobi phases' flops are
        # taken over the whole timed region (device time), not over their summed durations
        achieved = jac_flops / t_dev / 1e12 if t_dev > 0 else None
        clocks = sampler.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "BS-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": w["name"], "step": "one brick-wall layer (31-32 BS updates); the K timed layers go in one run_mesh call",
                       "workers": int(os.environ.get("BSMPO_WORKERS", "8")),
                       "timed_layers": [first, first + args.steps - 1], "bs_updates_timed": n_bs,
                       "bond_dims_at_start": [min(dims), max(dims)],
                       "setup_layers_s": round(t_setup, 2),
                       "circuit_time_s_upper_est": round(len(bs) / (value / world), 1),
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (state %.2f GB)" % (g_host.numel() * 16 / 1e9),
                       "bs_slice": args.bs_slice or "whole layer",
                       "cutoff": 0.0},
            "e2e": {"value": replica_rate(n_bs_e2e, world, t_e2e), "unit": "BS-updates/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "roofline": {"kernel": "jacobi_gram_kernel + jacobi_apply_kernel (one-sided Jacobi SVD rounds)",
                         "bound": "tensor", "achieved": achieved, "peak": fp64_peak,
                         "unit": "TFLOP/s", "frac": (achieved / fp64_peak) if achieved and fp64_peak else None,
                         "peak_source": "FP64 DGEMM measured in this run (torch.matmul 8192^3, best of 5)",
                         "achieved_over": "timed region (device time); Jacobi phases of the concurrent updates overlap",
                         "jacobi_stream_ms_sum": jac_ms, "jacobi_launches": jac_launches,
                         # DRAM bytes (read + write) of one early-round jacobi_gram_kernel
                         # launch of this workload, measured with ncu (cold cache)
                         "traffic": 21995008 if args.workload == "chi1024" else None,
                         "traffic_unit": "bytes per launch"},
            "clocks": clocks,
            "circuit": circuit,
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

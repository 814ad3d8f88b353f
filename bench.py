#!/usr/bin/env python
"""Benchmark of the dense statevector path on B200.

Workload (one "step"): the 30-qubit complex128 job -- a seeded U3/CZ brick
circuit of depth 40 followed by a full QFT (2260 gates, the reference's
containment fusion on), then the state's norm, 64 random Pauli-string
expectations and 1e6 shots.  The 16 GiB state is far larger than L2, so no
L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Other workloads (one JSON line each, not the headline):
    --mode serve   the serving stream: Poisson arrivals of mixed requests (12-28
                   qubits, depth 4-40, shots or <H>), the continuous-batching
                   server against the sequential plain loop
    --mode batch   the batched parameter sweep: 16-qubit RY/RZ + CX ansatz, 8
                   layers, 4096 bindings, <H> over 32 weighted Pauli strings
    --mode c64     the complex64 path: 32-qubit brick depth 32, error against the
                   complex128 path at 28 qubits

Multi-GPU: replicas only (the statevector is not sharded); each rank runs
its own job and `value` counts the jobs of all ranks over the slowest rank's
time.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "circuits/s, 30q complex128 job (brick d40 + QFT, norm, 64 Paulis, 1e6 shots)"
UNIT = "circuits/s"


def kernel_launches() -> int:
    """Kernels the library has launched so far (its own counter, mb2_kernel_launches)."""
    import ctypes as C
    from menos_b200 import _lib
    v = C.c_uint64()
    _lib.check(_lib.lib().mb2_kernel_launches(C.byref(v)), None, "mb2_kernel_launches")
    return int(v.value)


def profiled_traffic(n: int):
    """DRAM bytes of one tile-pass launch, from the committed ncu summary
    (measured at 28 qubits, scaled to 2^n: every tile is read and written
    once), or None when the summary is absent."""
    import re
    path = os.path.join(ROOT, "profiles", "k_tile_pass_c2_28q_ncu_full.md")
    try:
        with open(path) as f:
            m = re.search(r"traffic_bytes_per_launch_30q:\s*([0-9.eE+]+)", f.read())
    except OSError:
        return None
    return round(float(m.group(1)) * 2.0 ** (n - 30)) if m else None


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--qubits", type=int, default=30)
    p.add_argument("--depth", type=int, default=40)
    p.add_argument("--shots", type=int, default=1_000_000)
    p.add_argument("--terms", type=int, default=64)
    p.add_argument("--tile", type=int, default=0)
    p.add_argument("--fusion", type=int, default=0,
                   help="job: 0 = the reference's containment fusion; 2..6 = blocks of up to that many qubits")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="with --impl reference: skip timing the reference's own CUDA engine")
    p.add_argument("--validate-cpu", action="store_true",
                   help="with --impl reference: the extrapolated CPU job time against a whole reference run")
    p.add_argument("--mode", default="job", choices=["job", "serve", "batch", "c64", "estimator", "host"])
    p.add_argument("--requests", type=int, default=600)
    p.add_argument("--load", default="4", help="serve: arrival rate / plain-loop capacity (comma list: a sweep)")
    p.add_argument("--qubit-range", default="12,28", help="serve: request qubit counts, uniform in lo,hi")
    p.add_argument("--slots", type=int, default=0, help="serve: concurrent requests (0: the server's default, 16)")
    p.add_argument("--bindings", type=int, default=4096)
    p.add_argument("--window", type=int, default=0, help="host: device window qubits of the windowed sweep (0: n - 1)")
    p.add_argument("--precision", default="c128", choices=["c128", "c64"], help="serve/batch: state precision")
    p.add_argument("--c64-kernel", default="auto", choices=["auto", "tensor", "simt"],
                   help="complex64 passes: tensor cores (split-FP16 GEMMs), FP32 SIMT gates, or automatic")
    return p.parse_args()


def rank_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Clocks:
    """nvidia-smi samples (200 ms) across the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.device = device

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for name, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(world):
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    dist.init_process_group(backend=backend, timeout=timedelta(seconds=600))
    return dist


def dist_max(dist, value: float) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(dist):
    if dist is not None:
        dist.barrier()


# ----------------------------------------------------------------------------
# CPU leg: the reference's own CPU kernels (oracle/_ref), bounded sample.
# ----------------------------------------------------------------------------
def cpu_reference_sample(n, circ, paulis, shots, seed):
    """Times the reference CPU engine's kernels on the job at n qubits over a
    bounded sample -- the first brick layer's gates (each gate of the job is
    one of these shapes), one Pauli expectation and the full sampling walk --
    and extrapolates to the whole job.  Returns (circuits/s, details)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    ref = pyoracle.RefLib()
    threads = ref.default_threads()
    state = np.empty(1 << n, np.complex128)
    state.fill(0.0)  # every page touched before anything is timed
    state[0] = 1.0
    # U3 and CZ timings from one brick layer; CP / H / SWAP timed once each;
    # each gate applied twice and the second (warm) application timed.
    per_kind = {}
    sample_ops = circ.ops[:n + n // 2]
    extra = []
    for kind in ("h", "cp", "swap"):
        for op in circ.ops:
            if op[0] == pyoracle.OP[kind]:
                extra.append(op)
                break
    for oc, qs, ps, _m, _c in sample_ops + extra:
        m = ref.gate_matrix(oc, list(ps) + [0.0] * (3 - len(ps)))
        ref.apply_matrix(state, m, list(qs), threads=threads)
        t0 = time.perf_counter()
        ref.apply_matrix(state, m, list(qs), threads=threads)
        per_kind.setdefault(oc, []).append(time.perf_counter() - t0)
    counts_by_kind = {}
    for oc, *_ in circ.ops:
        counts_by_kind[oc] = counts_by_kind.get(oc, 0) + 1
    t_gates = sum(statistics.mean(per_kind[oc]) * c for oc, c in counts_by_kind.items())
    t0 = time.perf_counter()
    ref.expectation(state, paulis[0][0], paulis[0][1])
    t_term = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.sample(state, shots, seed, [(q, q) for q in range(n)], width=n)
    t_sample = time.perf_counter() - t0
    t_norm = t_term  # one more single-threaded read pass
    job = t_gates + t_norm + len(paulis) * t_term + t_sample
    sampled = sum(len(v) for v in per_kind.values())
    detail = {"gates_timed": sampled, "t_gates_s": round(t_gates, 3), "t_term_s": round(t_term, 4),
              "t_sample_s": round(t_sample, 3), "threads": threads, "isa": ref.kernel_isa()}
    return 1.0 / job, detail, threads, sampled


# ----------------------------------------------------------------------------
def main():
    args = parse()
    rank, world, local = rank_info()
    if args.impl == "reference":
        return main_reference(args, rank, world)
    if args.mode != "job":
        if rank == 0:
            {"serve": main_serve, "batch": main_batch, "c64": main_c64,
             "estimator": main_estimator, "host": main_host}[args.mode](args, local)
        return
    dist = dist_setup(world)
    import numpy as np
    import torch
    from menos_b200 import Context, DeviceState, workloads
    from menos_b200.circuit import to_mb2_ops
    from menos_b200._lib import SweepEstimate, SweepOptions, lib
    import ctypes as C

    torch.cuda.set_device(local)
    n = args.qubits
    circ = workloads.config_c2(n=n, depth=args.depth)
    paulis = workloads.pauli_strings(n, args.terms, 7)
    targets = [(q, q) for q in range(n)]
    ctx = Context(local)
    st = DeviceState(ctx, n)
    stream = torch.cuda.ExternalStream(st.stream_handle())

    def step():
        st.init(0.0)
        stats = st.apply_program(circ, tile_qubits=args.tile, fusion_width=args.fusion)
        norm = st.norm()
        terms = st.expectation(paulis)
        counts = st.sample(args.shots, 1234, targets)
        return stats, norm, terms, counts

    fp64_peak, copy_peak = ctx.probe_rates()
    for _ in range(args.warmup):
        stats, norm, terms, counts = step()
    assert abs(norm - 1.0) < 1e-9, norm

    # ---- device-timed job steps (state resident, circuit from host memory)
    clocks = Clocks(local)
    dist_barrier(dist)
    torch.cuda.synchronize()
    st.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = kernel_launches()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(args.steps):
        stats, norm, terms, counts = step()
    ev1.record(stream)
    ev1.synchronize()
    job_ms = ev0.elapsed_time(ev1)
    launches = kernel_launches() - launches0
    # ---- the sweep alone: average tile-pass launch duration
    sweep_ms = []
    for _ in range(max(2, args.steps)):
        st.init(0.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats = st.apply_program(circ, tile_qubits=args.tile, fusion_width=args.fusion)
        b.record(stream)
        b.synchronize()
        sweep_ms.append(a.elapsed_time(b))
    clk = clocks.stop()
    torch.cuda.synchronize()
    dist_barrier(dist)
    job_ms = dist_max(dist, job_ms)

    # ---- end to end through the engine's public API (host circuit in, host results out)
    from menos_b200 import B200DenseEngine, EngineExecutionRequest, PauliTerm
    eng = B200DenseEngine(local, tile_qubits=args.tile, fusion_width=args.fusion)
    req = EngineExecutionRequest(num_qubits=n, operations=circ, want_counts=True, want_expectation=True,
                                 shots=args.shots, seed=1234, measure_targets=targets, bitstring_width=n,
                                 observable=[PauliTerm(0, 0)] + [PauliTerm(x, z) for x, z in paulis])
    st.free()
    eng.execute(req)
    dist_barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.execute(req)
    e2e_s = dist_max(dist, time.perf_counter() - t0)
    # The copies one execute() makes (the circuit is planned on the host and
    # only its encoded program crosses): the tiled program, the Pauli terms'
    # X and Z masks and the sampler's sorted uniforms in; the terms' values
    # and each shot's basis index out.  The expectation's group tables (a
    # few KB) are not counted.
    arr, _keep = to_mb2_ops(circ)
    est = SweepEstimate()
    rc_est = lib().mb2_estimate_sweep(arr, len(circ.ops), C.byref(SweepOptions(1, 0, args.tile, 0, 0, args.fusion)),
                                      n, C.byref(est))
    n_terms = len(paulis) + 1
    h2d = int(est.h2d_bytes) + 16 * n_terms + 8 * args.shots if rc_est == 0 else None
    d2h = 16 * n_terms + 8 * args.shots

    passes = int(stats.passes)
    sweep_avg = statistics.median(sweep_ms)
    per_launch_ms = sweep_avg / max(passes, 1)
    state_bytes = 16 << n
    achieved = 2 * state_bytes / (per_launch_ms * 1e-3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_src = "measured"
    value = world * args.steps / (job_ms * 1e-3)
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(job_ms / args.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded circuit)",
        "config": {"workload": f"{n}q complex128: brick depth {args.depth} + QFT ({len(circ.ops)} gates), " +
                               ("fusion=containment" if args.fusion == 0 else f"fusion<={args.fusion} qubits") +
                               f", norm + {args.terms} Paulis + {args.shots} shots",
                   "qubits": n, "parallelism": f"replicas x{world}", "l2": "state 16 GiB >> L2 (no flush)",
                   "passes": passes, "blocks": int(stats.blocks), "sweep_ms": round(sweep_avg, 2),
                   "tile_qubits": args.tile or 11},
        "roofline": {"bound": "hbm", "kernel": "k_tile_pass", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": profiled_traffic(n),
                     "traffic_source": "ncu dram__bytes_read+write of one pass at 28 qubits, scaled by the "
                                       "state size (profiles/k_tile_pass_c2_28q_ncu_full.md)",
                     "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": 2 * state_bytes,
                     "blocks_per_launch": round(int(stats.blocks) / max(1, passes), 2),
                     # Blocks x one state pass each / sweep time: what the multi-gate
                     # passes buy; reported beside `achieved`, never as the fraction.
                     "gate_equivalent_gbs": round(int(stats.blocks) * 2 * state_bytes / (sweep_avg * 1e-3) / 1e9, 1)},
        "fp64": {"kernel": "k_tile_pass", "achieved_ops_per_s": round(stats.fp64_ops_per_amp * (1 << n) /
                                                                     (sweep_avg * 1e-3), 1),
                 "peak_ops_per_s": round(fp64_peak, 1), "peak_source": "measured (mb2_probe_rates)",
                 "frac": round(stats.fp64_ops_per_amp * (1 << n) / (sweep_avg * 1e-3) / fp64_peak, 4),
                 "model_ops_per_amp": int(stats.fp64_ops_per_amp), "copy_gbs_probe": round(copy_peak, 1)},
        "e2e": {"value": round(world * args.steps / e2e_s, 4), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, detail, cores, sampled = cpu_reference_sample(n, circ, paulis, args.shots, 1234)
        line["cpu_baseline"] = {"value": round(v, 6), "unit": UNIT, "cores": cores, "kind": "reference",
                                "sample": f"reference CPU kernels (oracle/_ref) at {n} qubits: {sampled} gates "
                                          f"timed, 1 Pauli pass, full 1e6-shot walk; extrapolated to the job",
                                "detail": detail}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def percentile(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


def main_serve(args, local):
    """The serving stream against the sequential plain loop, same requests."""
    import numpy as np
    from menos_b200 import Context, DeviceState, workloads
    from menos_b200.serve import Server
    ctx = Context(local)
    from menos_b200.circuit import PackedCircuit
    nmin, nmax = (int(v) for v in args.qubit_range.split(","))
    reqs = workloads.serving_stream(args.requests, 1.0, 20261201, nmin=nmin, nmax=nmax)
    # Operations packed for the C ABI once, before any timed region, for
    # both arms: the timed work is the engine's, not Python's conversion.
    for r in reqs:
        r["circuit"] = PackedCircuit(r["circuit"])

    def run_plain(r):
        st = DeviceState(ctx, r["circuit"].num_qubits)
        st.init(r["circuit"].global_phase)
        st.apply_program(r["circuit"])
        if r["output"] == "counts":
            out = st.sample(r["shots"], r["seed"], [(q, q) for q in range(r["circuit"].num_qubits)])
        else:
            vals = st.expectation(r["paulis"])
            out = float(sum(c * v.real for c, v in zip(r["coefs"], vals)))
        st.free()
        return out

    for r in reqs[:8]:  # warm-up (planner, allocator, module load)
        run_plain(r)
    # Sequential plain loop: service times, then FIFO latencies for any arrival process.
    service, plain_out = [], []
    t_all = time.perf_counter()
    for r in reqs:
        t0 = time.perf_counter()
        plain_out.append(run_plain(r))
        service.append(time.perf_counter() - t0)
    plain_total = time.perf_counter() - t_all
    plain_rate = len(reqs) / plain_total
    loads = [float(x) for x in str(args.load).split(",")]

    def fifo_latencies(arrivals):
        lat, free_at = [], 0.0
        for a, s in zip(arrivals, service):
            start = max(a, free_at)
            free_at = start + s
            lat.append(free_at - a)
        return lat

    from menos_b200._lib import C64, C128
    prec = C64 if args.precision == "c64" else C128

    def serve(arrive):
        srv = Server(ctx, budget_bytes=160 * 10**9, slots=args.slots)
        done, results, failed = {}, {}, {}
        tickets = {}
        t0 = time.perf_counter()
        i = 0
        while len(done) < len(reqs):
            now = time.perf_counter() - t0
            while i < len(reqs) and (not arrive or arrive[i] <= now):
                r = reqs[i]
                nq = r["circuit"].num_qubits
                if r["output"] == "counts":
                    tk = srv.submit(r["circuit"], "counts", shots=r["shots"], seed=r["seed"],
                                    targets=[(q, q) for q in range(nq)], precision=prec)
                else:
                    tk = srv.submit(r["circuit"], "expectation", paulis=r["paulis"], coefs=r["coefs"],
                                    precision=prec)
                tickets[tk] = i
                i += 1
            for c in srv.poll(timeout_ms=1):
                k = tickets[c["ticket"]]
                done[k] = c["latency_s"]
                if c["status"] != 0:
                    failed[k] = c["status"]
                results[k] = c["counts"] if reqs[k]["output"] == "counts" else c["value"]
        total = time.perf_counter() - t0
        srv.close()
        return done, results, total, failed

    burst_done, burst_res, burst_total, burst_failed = serve(None)
    # The live stream at each load: Poisson arrivals at load x the plain
    # loop's capacity (the stream was drawn at rate 1 and is rescaled).
    live, live_failed, mix_same = [], {}, True
    for load in loads:
        rate = load * plain_rate
        arrivals = [r["arrival_s"] / rate for r in reqs]
        done, res, total, failed = serve(arrivals)
        live_failed.update(failed)
        for k in range(len(reqs)):
            if k not in burst_failed and k not in failed:
                mix_same = mix_same and (burst_res[k] == res[k])
        lat = [done[k] for k in range(len(reqs))]
        plain_lat = fifo_latencies(arrivals)
        live.append({"arrival_rate_per_s": round(rate, 2), "load_vs_plain_capacity": load,
                     "circuits_per_s": round(len(reqs) / total, 2),
                     "p50_ms": round(1e3 * percentile(lat, 50), 2), "p99_ms": round(1e3 * percentile(lat, 99), 2),
                     "plain_fifo_p50_ms": round(1e3 * percentile(plain_lat, 50), 2),
                     "plain_fifo_p99_ms": round(1e3 * percentile(plain_lat, 99), 2)})
    # Each result the same in the burst and in the live mixes; against the
    # complex128 plain loop: identical counts and <H> (complex128), or <H>
    # within the precision path's error (complex64; counts then follow the
    # complex64 probabilities).
    worst_exp, counts_same = 0.0, True
    for k, r in enumerate(reqs):
        if k in burst_failed or k in live_failed:
            continue
        if r["output"] == "counts":
            counts_same = counts_same and (burst_res[k] == plain_out[k])
        else:
            worst_exp = max(worst_exp, abs(burst_res[k] - plain_out[k]))
    line = {
        "metric": "served circuits/s (continuous batching) vs sequential plain loop", "unit": "circuits/s",
        "mode": "serve", "requests": len(reqs), "higher_is_better": True,
        "value": round(len(reqs) / burst_total, 2),
        "plain_loop": {"circuits_per_s": round(plain_rate, 2), "total_s": round(plain_total, 3)},
        "speedup_vs_plain": round(plain_total / burst_total, 2),
        "live": live,
        "failed_requests": {"burst": len(burst_failed), "live": len(live_failed),
                            "statuses": sorted(set(burst_failed.values()) | set(live_failed.values()))},
        "results": {"burst_equals_live": mix_same, "counts_identical_to_plain_c128": counts_same,
                    "max_abs_dH_vs_plain_c128": worst_exp},
        "precision": args.precision,
        "config": {"workload": f"serving stream: qubits {nmin}-{nmax}, depth 4-40 (U3/CZ brick or RY/RZ+CX), "
                               f"4096 shots or <H> over 32 weighted Paulis, {args.precision}, budget 160 GB",
                   "seed": 20261201},
        "data": "synthetic (seeded requests)",
    }
    print(json.dumps(line), flush=True)


def main_batch(args, local):
    """The batched parameter sweep against one plain run per binding."""
    import numpy as np
    import torch
    from menos_b200 import Context, DeviceState, workloads
    from menos_b200.engine import sweep_batch
    ctx = Context(local)
    n, layers, B = 16, 8, args.bindings
    circ = workloads.hea(n, layers, 11)
    params = np.asarray(workloads.hea_bindings(n, layers, B, 12))
    paulis = workloads.pauli_strings(n, 32, 13)
    coefs = workloads.weights(32, 14)
    from menos_b200._lib import C64, C128
    prec = C64 if args.precision == "c64" else C128
    sweep_batch(ctx, circ, params[:64], paulis, coefs, precision=prec)  # warm-up
    torch.cuda.synchronize()
    ts = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        vals, _, stats = sweep_batch(ctx, circ, params, paulis, coefs, precision=prec)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)

    def bound(row):
        c = workloads.hea(n, layers, 11)
        k, ops = 0, []
        for oc, qs, ps, m, cl in c.ops:
            if ps:
                ps = tuple(float(v) for v in row[k:k + len(ps)])
                k += len(ps)
            ops.append((oc, qs, ps, m, cl))
        c.ops = ops
        return c
    sample = min(64, B)
    st = DeviceState(ctx, n)
    t0 = time.perf_counter()
    worst = 0.0
    for b in range(sample):
        st.init(0.0)
        st.apply_program(bound(params[b]), fuse_gates=False)
        v = st.expectation(paulis)
        h = float(sum(c * x.real for c, x in zip(coefs, v)))
        worst = max(worst, abs(h - vals[b]))
    plain_per = (time.perf_counter() - t0) / sample
    line = {
        "metric": "bindings/s, batched parameter sweep (16q RY/RZ+CX x8, <H> over 32 Paulis)", "unit": "bindings/s",
        "mode": "batch", "value": round(B / t, 1), "higher_is_better": True, "bindings": B, "s_per_sweep": round(t, 4),
        "plain_loop": {"bindings_per_s": round(1.0 / plain_per, 1), "sampled_bindings": sample},
        "speedup_vs_plain": round((B / t) * plain_per, 2),
        "max_abs_dH_vs_plain_c128": worst, "passes": int(stats.passes),
        "dtype": "c128 (f64)" if prec == C128 else "c64 (f32 amplitudes, f64 reductions)",
        "config": {"workload": f"hea({n}, {layers}) x {B} bindings, 32 weighted Paulis", "seed": 11},
        "data": "synthetic (seeded angles)",
    }
    print(json.dumps(line), flush=True)


def main_c64(args, local):
    """The complex64 path: 32-qubit throughput, error against complex128 at 28 qubits."""
    import numpy as np
    import torch
    from menos_b200 import Context, DeviceState, workloads
    from menos_b200._lib import C64
    ctx = Context(local)
    paulis = workloads.pauli_strings(28, 64, 21)
    circ28 = workloads.brick(28, 32, 20260929)
    ref = DeviceState(ctx, 28)
    ref.init(0.0)
    ref.apply_program(circ28)
    ref_amps = ref.copy_out()
    ref_exp = ref.expectation(paulis)
    ref.free()
    lo = DeviceState(ctx, 28, precision=C64)
    lo.init(0.0)
    lo.apply_program(circ28, tile_qubits=args.tile, c64_kernel=args.c64_kernel)
    lo.normalize()
    lo_amps = lo.copy_out()
    lo_exp = lo.expectation(paulis)
    lo.free()
    d_amp = float(np.max(np.abs(lo_amps.astype(np.complex128) - ref_amps)))
    d_exp = float(np.max(np.abs(lo_exp - ref_exp)))
    del ref_amps, lo_amps
    n = args.qubits if args.qubits != 30 else 32
    circ = workloads.brick(n, 32, 20260929)
    st = DeviceState(ctx, n, precision=C64)
    stream = torch.cuda.ExternalStream(st.stream_handle())
    st.init(0.0)
    st.apply_program(circ, tile_qubits=args.tile, c64_kernel=args.c64_kernel)
    st.synchronize()
    ts = []
    for _ in range(max(1, args.steps)):
        st.init(0.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats = st.apply_program(circ, tile_qubits=args.tile, c64_kernel=args.c64_kernel)
        st.normalize()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    ms = statistics.median(ts)
    per_pass = ms / max(1, int(stats.passes))
    line = {
        "metric": f"circuits/s, {n}q complex64 brick depth 32 (sweep + renormalisation)", "unit": "circuits/s",
        "mode": "c64", "value": round(1000.0 / ms, 4), "ms_per_circuit": round(ms, 2), "higher_is_better": True,
        "passes": int(stats.passes), "hbm_gbs_per_pass": round(2 * (8 << n) / (per_pass * 1e-3) / 1e9, 1),
        "error_28q_vs_complex128": {"max_abs_amp": d_amp, "max_abs_pauli": d_exp, "paulis": 64},
        "dtype": "c64 (f32 amplitudes, f64 reductions)",
        "config": {"workload": f"brick({n}, 32), state {8 << n >> 30} GiB", "seed": 20260929,
                   "c64_kernel": args.c64_kernel, "tile_qubits": args.tile or "auto"},
        "data": "synthetic (seeded circuit)",
    }
    print(json.dumps(line), flush=True)


def main_estimator(args, local):
    """The Qiskit-shaped Estimator (menos_b200/primitives.py) against the
    reference primitive's loop shape (python/menos/qiskit/estimator.py:
    86-156): one full run per observable of each pub, pub after pub, here
    through this engine's own plain path."""
    import numpy as np
    from menos_b200 import Context, DeviceState, workloads
    from menos_b200.primitives import B200Estimator, bind, observable_terms, parameter_slots
    ctx = Context(local)
    rng = np.random.default_rng(31)
    pubs = []
    for i in range(args.requests if args.requests != 600 else 48):
        n = int(rng.integers(12, 21))
        circ = workloads.brick(n, int(rng.integers(4, 21)), 1000 + i)
        obs = []
        for _ in range(8):
            ps = workloads.pauli_strings(n, 8, int(rng.integers(0, 1 << 30)))
            obs.append([(x, z, float(w)) for (x, z), w in zip(ps, rng.normal(size=8))])
        pubs.append((circ, obs))
    hea = workloads.hea(16, 8, 5)
    values = rng.uniform(-np.pi, np.pi, size=(256, parameter_slots(hea)))
    hobs = [[(x, z, float(w)) for (x, z), w in zip(workloads.pauli_strings(16, 8, 40 + k), rng.normal(size=8))]
            for k in range(4)]

    def loop_run(circ, o):
        st = DeviceState(ctx, circ.num_qubits)
        st.init(circ.global_phase)
        st.apply_program(circ)
        terms = observable_terms(o, circ.num_qubits)
        v = st.expectation([(x, z) for x, z, _ in terms])
        st.free()
        return sum((c * e).real for (_, _, c), e in zip(terms, v))

    est = B200Estimator(ctx, seed=1)
    est.run(pubs[:4])
    loop_run(pubs[0][0], pubs[0][1][0])
    t0 = time.perf_counter()
    res = est.run(pubs)
    t_batched = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref_vals = [[loop_run(c, o) for o in obs] for c, obs in pubs]
    t_loop = time.perf_counter() - t0
    err = max(abs(r["evs"][k] - ref_vals[i][k]) for i, r in enumerate(res) for k in range(8))
    # A parameterised pub: 256 bindings x 4 observables (one batched sweep per observable).
    t0 = time.perf_counter()
    (hr,) = est.run([(hea, [[o] for o in hobs], values)])  # observables (4, 1) x bindings (256,)
    t_hb = time.perf_counter() - t0
    sample = 16
    t0 = time.perf_counter()
    hloop = [[loop_run(bind(hea, values[b]), o) for o in hobs] for b in range(sample)]
    t_hl = (time.perf_counter() - t0) * values.shape[0] / sample
    herr = max(abs(hr["evs"][k, b] - hloop[b][k]) for b in range(sample) for k in range(4))
    line = {
        "metric": "estimator pubs/s (8 observables x 8 Paulis each) vs one run per observable",
        "unit": "pubs/s", "mode": "estimator", "value": round(len(pubs) / t_batched, 3), "higher_is_better": True,
        "loop_pubs_per_s": round(len(pubs) / t_loop, 3), "speedup_vs_loop": round(t_loop / t_batched, 2),
        "max_abs_diff_vs_loop": err,
        "parameterised_pub": {"bindings": int(values.shape[0]), "observables": 4, "seconds": round(t_hb, 4),
                              "loop_seconds_extrapolated": round(t_hl, 3), "speedup": round(t_hl / t_hb, 1),
                              "max_abs_diff_vs_loop": herr},
        "dtype": "c128 (f64)",
        "config": {"workload": f"{len(pubs)} pubs: brick circuits of 12-20 qubits, depth 4-20, 8 observables of "
                               "8 weighted Paulis each; plus hea(16, 8) x 256 bindings x 4 observables", "seed": 31},
        "data": "synthetic (seeded circuits and observables)",
    }
    print(json.dumps(line), flush=True)


def main_host(args, local):
    """The host-resident tier: the job's circuit on a complex128 state in
    pinned, mapped host memory (every pass streams it over PCIe), beside the
    same sweep on a device-resident state."""
    import torch
    from menos_b200 import Context, DeviceState, workloads
    ctx = Context(local)
    n = args.qubits if args.qubits != 30 else 28
    circ = workloads.config_c2(n=n, depth=args.depth)
    paulis = workloads.pauli_strings(n, args.terms, 7)
    out = {}
    for host in (False, True):
        st = DeviceState(ctx, n, host=host)
        stream = torch.cuda.ExternalStream(st.stream_handle())
        warm = workloads.config_c2(n=n, depth=1)
        st.init(0.0)
        st.apply_program(warm)
        st.synchronize()
        st.init(0.0)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        stats = st.apply_program(circ)
        b.record(stream)
        b.synchronize()
        sweep = a.elapsed_time(b)
        t0 = time.perf_counter()
        st.norm()
        st.expectation(paulis)
        st.sample(args.shots, 1234, [(q, q) for q in range(n)])
        outputs = (time.perf_counter() - t0) * 1e3
        out[host] = {"sweep_ms": round(sweep, 2), "passes": int(stats.passes), "outputs_ms": round(outputs, 2),
                     "gbs_per_pass": round(2 * (16 << n) / (sweep / int(stats.passes) * 1e-3) / 1e9, 1)}
        st.free()
    # The same host-resident state through two device windows of
    # 2^(n-1) amplitudes (the chunked tier on the copy engines).
    window = args.window if args.window > 0 else n - 1
    st = DeviceState(ctx, n, host=True)
    st.init(0.0)
    st.apply_program_windowed(workloads.config_c2(n=n, depth=1), window)
    st.init(0.0)
    st.synchronize()
    t0 = time.perf_counter()
    stats = st.apply_program_windowed(circ, window)
    wsweep = (time.perf_counter() - t0) * 1e3
    st.free()
    win = {"sweep_ms": round(wsweep, 2), "window_passes": int(stats.passes), "window_qubits": window,
           "gbs_per_pass": round(2 * (16 << n) / (wsweep / int(stats.passes) * 1e-3) / 1e9, 1)}
    h = out[True]
    line = {
        "metric": f"circuits/s, {n}q complex128 job on a host-resident state (pinned, mapped; streamed over PCIe)",
        "unit": "circuits/s", "mode": "host", "value": round(1000.0 / (h["sweep_ms"] + h["outputs_ms"]), 4),
        "higher_is_better": True, "host": h, "device": out[False], "windowed": win,
        "windowed_circuits_per_s": round(1000.0 / (win["sweep_ms"] + h["outputs_ms"]), 4),
        "dtype": "c128 (f64)",
        "config": {"workload": f"brick({n}, {args.depth}) + QFT, norm + {args.terms} Paulis + {args.shots} shots, "
                               f"state {16 << n >> 30} GiB in host memory, 12-qubit tiles"},
        "data": "synthetic (seeded circuit)",
    }
    print(json.dumps(line), flush=True)


def validate_cpu_baseline(args):
    """The extrapolated CPU figure against one whole job run through the
    reference's DenseEngine::execute (oracle/_ref), both at --qubits (26 by
    default for this check: a full 30-qubit run takes hours)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from menos_b200 import workloads
    n = args.qubits
    circ = workloads.config_c2(n=n, depth=args.depth)
    paulis = workloads.pauli_strings(n, args.terms, 7)
    v, detail, cores, sampled = cpu_reference_sample(n, circ, paulis, args.shots, 1234)
    ref = pyoracle.RefLib()
    oc = pyoracle.Circuit(n)
    oc.ops = list(circ.ops)
    t0 = time.perf_counter()
    ref.run(oc, fuse_gates=True, statevector=False, shots=args.shots, seed=1234,
            targets=[(q, q) for q in range(n)], width=n, paulis=[(0, 0)] + list(paulis))
    whole = time.perf_counter() - t0
    print(json.dumps({"check": "cpu baseline extrapolation vs whole DenseEngine::execute", "qubits": n,
                      "extrapolated_s": round(1.0 / v, 3), "measured_s": round(whole, 3),
                      "ratio": round((1.0 / v) / whole, 3), "threads": cores, "detail": detail}), flush=True)


def reference_gpu_job(n, circ, paulis, shots):
    """The reference's own CUDA dense engine (CudaDenseEngine::execute, its
    src/kernels/cuda built for sm_100a with its -fmad=false by
    oracle/Makefile) on the whole job: wall time of one execute() for the
    request the B200 engine's e2e leg runs (statevector norm as the identity
    term, the Pauli terms, the shots), after a small warm-up run."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from menos_b200 import workloads
    if not os.path.exists(pyoracle.REF_CUDA_SO):
        return {"unavailable": "oracle/_ref/libmenos_ref_cuda.so is not built"}
    ref = pyoracle.RefLib(pyoracle.REF_CUDA_SO)
    warm = pyoracle.Circuit(16)
    warm.ops = list(workloads.config_c2(n=16, depth=2).ops)
    ref.run(warm, engine="cuda", statevector=False, shots=1000, seed=1, targets=[(q, q) for q in range(16)],
            width=16, paulis=[(0, 0)])
    oc = pyoracle.Circuit(n, circ.global_phase)
    oc.ops = list(circ.ops)
    r = ref.run(oc, engine="cuda", fuse_gates=True, statevector=False, shots=shots, seed=1234,
                targets=[(q, q) for q in range(n)], width=n, paulis=[(0, 0)] + list(paulis))
    s = r["seconds"]
    return {"value": round(1.0 / s, 6), "unit": UNIT, "seconds": round(s, 3),
            "engine": "reference CudaDenseEngine::execute (sm_100a, -fmad=false), containment fusion, "
                      "host-side sampling walk",
            "request": f"{n}q brick depth 40 + QFT, identity + {len(paulis)} Pauli terms, {shots} shots"}


def main_reference(args, rank, world):
    if rank != 0:
        return
    if args.validate_cpu:
        return validate_cpu_baseline(args)
    from menos_b200 import workloads
    n = args.qubits
    circ = workloads.config_c2(n=n, depth=args.depth)
    paulis = workloads.pauli_strings(n, args.terms, 7)
    vals, detail, cores, sampled = [], None, 0, 0
    for _ in range(max(1, min(args.steps, 2))):
        v, detail, cores, sampled = cpu_reference_sample(n, circ, paulis, args.shots, 1234)
        vals.append(v)
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000.0 / v, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic (seeded circuit)",
        "config": {"workload": f"{n}q complex128: brick depth {args.depth} + QFT, norm + {args.terms} Paulis + "
                               f"{args.shots} shots", "qubits": n},
        "cpu_baseline": {"value": round(v, 6), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"reference CPU kernels at {n} qubits: {sampled} gates timed, 1 Pauli pass, "
                                   f"full 1e6-shot walk; extrapolated to the job", "detail": detail},
        "e2e": {"value": round(v, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    # Beside the CPU arm, for reference: the reference's own GPU path.
    try:
        import torch
        if torch.cuda.is_available() and not args.no_reference_gpu:
            line["reference_gpu"] = reference_gpu_job(n, circ, paulis, args.shots)
    except Exception as e:  # reported, never fatal to the CPU arm
        line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

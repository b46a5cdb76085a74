"""Benchmark of the B200 gauge-field hot path; prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the "plain FP64 at scale" configuration): a 32^4 periodic SU(3) lattice, FP64 links
(18 reals), hot start from seed 7, Wilson action beta = 6.0, N_hits = 2.  One step = one full
checkerboard heatbath sweep (8 (parity, mu) passes, every link updated once with N_hits hits).
`value` is link-updates/s over all ranks with the field resident in HBM; `e2e` is the same metric
through the C ABI with the configuration uploaded from pinned host memory each step and the
plaquette read back.  The flow part of the metric (site-steps/s of the Wilson flow over the
configuration's 250 steps, FP64 vs FP32 18- and 12-real, the RK3 integrator alone and with clover
Q, E and the plaquette every step, with |dQ|, dE/E and dP against FP64) is measured on the same
configuration and reported under "flow"; each form starts from an idle GPU.  Multi-GPU runs are
independent replicas (weak scaling, no collective on the data path).  The reference arm and the
cpu_baseline leg time the reference's own heatbath code (its hit() per link, staple recomputed per
hit), compiled unchanged into oracle/_ref/libqcb_ref.so, on all host cores, one full sweep of the
same 32^4 configuration per step; where that library is absent they fall back to the oracle's
restatement with the same cost structure.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "ecmc-qcb_b200")

L = (32, 32, 32, 32)
BETA, N_HITS, SEED_HOT, SEED_HB = 6.0, 2, 7, 12345
METRIC = "HB link-upd/s & flow site-steps/s, FP32 vs FP64 at ΔQ<1e-4; serve p50/p99"
S_U = {64: 144, 32: 72}  # bytes of an 18-real link
S_U12 = {64: 96, 32: 48}
S_Z = {64: 64, 32: 32}


def load_package():
    if "ecmc_qcb_b200" in sys.modules:
        return sys.modules["ecmc_qcb_b200"]
    spec = importlib.util.spec_from_file_location("ecmc_qcb_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ecmc_qcb_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    return oracle


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            v = float(json.load(fh)["hbm_gbs"])
        if v > 0:
            return v, "measured"
    except (OSError, ValueError, KeyError, TypeError):
        pass
    return 6650.0, "fallback"


def profile_traffic(name: str):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary (profiles/<name>.md)."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = str(gpu_index)
        try:
            import torch

            self.idx = "GPU-" + str(torch.cuda.get_device_properties(gpu_index).uuid)
        except Exception:
            pass
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler has produced its first line
            t0 = time.time()
            while time.time() - t0 < 5.0:
                if os.fstat(self.f.fileno()).st_size > 0:
                    break
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.05)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int, backend: str | None = None):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK): NCCL on GPUs, gloo on CPU."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return rank, world, local


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: float, ms_max: float, world: int) -> float:
    """Whole-job rate of `world` independent replicas (weak scaling): all ranks' units over the
    slowest rank's time."""
    return world * units_per_rank / (ms_max * 1e-3)


def cuda_timer(qcb, field):
    """CUDA events on the field's own stream (the stream the kernels are launched on)."""
    import torch

    stream = torch.cuda.ExternalStream(field.stream)
    return stream, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


CONFIG = {"workload": "hb_fp64_32^4", "L": list(L), "beta": BETA, "n_hits": N_HITS, "start": "hot seed 7",
          "step": "one full checkerboard sweep (8 (parity,mu) passes, every link updated once)",
          "l2": "inputs larger than L2 (604 MB FP64 field vs 126 MB L2)"}


class CpuHeatbath:
    """The CPU heatbath the GPU arm is compared with, on the 32^4 configuration (hot start seed 7).

    kind "reference": the reference's own mpi::heatbathcb::hit (src/heatbath/heatbath_mpi.cpp:10-33)
    link by link, compiled unchanged into oracle/_ref/libqcb_ref.so, staple recomputed for every hit
    as the reference does, OpenMP over the links of each (parity, mu) set on all host threads, draws
    from the same Philox link streams as the GPU.  kind "port": the oracle's restatement with the same
    cost structure, used only where the reference library is absent."""

    def __init__(self):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        orc = load_oracle()
        orc.set_threads(0)
        U = orc.hot_start(L, SEED_HOT)
        self.V = U.shape[0]
        self.threads = orc.threads()
        import ref

        if ref.available():
            ref.set_threads(0)
            self.kind = "reference"
            self.lat = ref.RefLattice(L[0], U)
            self._sub = lambda sw, p, mu: self.lat.hb_subsweep(BETA, N_HITS, SEED_HB, sw, p, mu)
        else:
            self.kind = "port"
            self.U = U
            self._sub = lambda sw, p, mu: orc.hb_subsweep(self.U, L, BETA, N_HITS, SEED_HB, sw, p, mu, refcost=True)

    def sweep(self, sw: int) -> None:
        for p in (0, 1):
            for mu in range(4):
                self._sub(sw, p, mu)

    def describe(self, what: str) -> str:
        src = ("the reference's hit() compiled unchanged (oracle/_ref)" if self.kind == "reference"
               else "the oracle's restatement of the reference's hit()")
        return (f"{what}; each sweep 8 (parity,mu) passes of V/2 = {self.V // 2} link-updates, N_hits=2, staple "
                f"recomputed per hit; {src}; 1 process x {self.threads} OpenMP threads")


def cpu_sample(seconds: float = 12.0):
    """cpu_baseline leg: full sweeps of the workload on the host cores until `seconds` have passed
    (after one untimed sweep), with the sweep indices the reference arm uses."""
    c = CpuHeatbath()
    c.sweep(0)
    n, t0 = 0, time.perf_counter()
    while True:
        c.sweep(1 + n)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": n * 4 * c.V / el, "unit": "link-upd/s", "cores": c.threads, "kind": c.kind,
            "sample": c.describe(f"{n} full sweeps of 32^4 in {el:.1f} s")}


REF_BUDGET_S = 300.0  # the reference arm's whole run stays within a few minutes


def run_reference(args, rank: int, world: int):
    """The reference arm: W untimed then K timed steps of the workload on the host cores.  A step is
    one full sweep, as in the GPU arm, unless W + K full sweeps would exceed REF_BUDGET_S (judged from
    the first warm-up sweep); then a step is one (parity, mu) pass (V/2 link-updates) and the
    config's "step" says so."""
    if rank != 0:
        return
    c = CpuHeatbath()
    t0 = time.perf_counter()
    c.sweep(0)
    t_sweep = time.perf_counter() - t0
    full = (args.warmup + args.steps) * t_sweep <= REF_BUDGET_S
    times, units = [], 0
    for i in range(1, args.warmup + args.steps):
        t0 = time.perf_counter()
        if full:
            c.sweep(i)
        else:
            c._sub(i // 8, (i // 4) % 2, i % 4)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
            units += 4 * c.V if full else c.V // 2
    if args.warmup == 0:  # the first sweep is the only one of a 0-warm-up run that was timed
        times.append(t_sweep)
        units += 4 * c.V
    tot = sum(times)
    value = units / tot
    cfg = dict(CONFIG)
    cfg["parallelism"] = f"replicas x{args.gpus}"
    if not full:
        cfg["step"] = "one (parity,mu) pass of the sweep (V/2 link-updates): full sweeps exceed the time budget"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "link-upd/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": value, "unit": "link-upd/s", "cores": c.threads, "kind": c.kind,
                         "sample": c.describe(f"{args.steps} timed {'full sweeps' if full else '(parity,mu) passes'} "
                                              f"after {args.warmup} untimed")},
        "e2e": {"value": value, "unit": "link-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


FLOW_STEPS = 250  # t = 5.0 at eps = 0.02: the flow of the 32^4 FP64 configuration
FLOW_COOL_S = 2.0  # idle pause before each timed flow form
# idle pause before each serving arm: the arms are seconds of full load each, and one started right
# after another ran 10-25% slower on some boxes (the power cap); 10 s removed that in A/B runs
SERVE_COOL_S = 10.0


def flow_flops_per_link_stage(prec: int) -> float:
    """Algorithmic flops of one link in one fused RK3 stage, as the kernels form it (complex
    multiply-add 8 flops, multiply 6, add 2):
      staple   6 staples x (36 multiply-adds of the two-row products + 6 multiplies and 3 subtractions
               rebuilding row 3 + 9 adds into A)                                    = 6 x 348 = 2088
      force    -proj(U A) from 6 off-diagonal entries (3 multiply-adds each), 3 imaginary diagonal
               parts and the projection                                            = 204
      RK3      X (and Z) combinations, averaged over the three stages              = 60
      exp      X^2 (27 multiply-adds), t and det X, the 18-step Horner recurrence, q0 + q1 X + q2 X^2
                                                                                   = 542
      update   exp(X) W, full product (27 multiply-adds)                           = 216
      reproject (FP32 links) column Gram-Schmidt in FP64                           = 100"""
    return 2088 + 204 + 60 + 542 + 216 + (100 if prec == 32 else 0)


def flow_block(qcb, src, prec, store, n_steps, hbm_peak, fma_peak, gpu_index=0, measured=True):
    """One flow form on the configuration `src`, timed with CUDA events on the flow's stream.

    Every form starts from the same state: an idle pause of FLOW_COOL_S first, because under the
    1 kW power cap a form timed right after another inherits its power draw (a stage runs 10-20%
    slower for a few hundred ms after a sustained FP64 flow).  Then
      (a) n_steps RK3 steps after 3 warm-up steps, replayed as CUDA graphs: site-steps/s of the
          integrator;
      (b) 20 more steps with per-launch event timing (plain launches): the mean stage-kernel
          duration, for the HBM roofline and the pipe fraction;
      (c) if `measured`, the configuration's measured flow: the copy of `src`, n_steps RK3 steps
          and clover Q, E and the plaquette at every one of the n_steps + 1 times
          (qcb_flow_measure), after the same idle pause.
    SM clocks and throttle reasons are sampled over all three."""
    V = src.V
    time.sleep(FLOW_COOL_S)
    fl = qcb.GradientFlow(src, 0.02, prec=prec, store=store)
    f = fl.field
    stream, e0, e1 = cuda_timer(qcb, f)
    with Clocks(gpu_index) as clk:
        fl.rk3_step(4)
        f.sync()
        e0.record(stream)
        fl.rk3_step(n_steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        f.timing(True)
        f.timing_reset()
        fl.rk3_step(20)
        nl, kms = f.timing_read(qcb.K_FLOW)
        f.timing(False)
        ms_meas = None
        if measured:
            # untimed warm-up: the first measured flow of a flow state allocates its clover-halves
            # buffer and captures the measurement graphs (one per buffer parity)
            fl.measure(src, 4, 1, plaquette=True)
            time.sleep(FLOW_COOL_S)
            e0.record(stream)
            fl.measure(src, n_steps + 1, 1, plaquette=True)
            e1.record(stream)
            e1.synchronize()
            ms_meas = e0.elapsed_time(e1)
    s_u = (S_U12 if store == 1 else S_U)[prec]
    bytes_stage = V * 4 * (2 * s_u) + V * 4 * S_Z[prec] * (4 / 3)  # per stage: read+write U, Z traffic averaged
    stage_ms = kms / nl
    achieved = bytes_stage / (stage_ms * 1e-3) / 1e9
    flops_stage = 4 * V * flow_flops_per_link_stage(prec)
    tflops = flops_stage / (stage_ms * 1e-3) / 1e12
    fl.close()
    out = {"site_steps_per_s": V * n_steps / (ms * 1e-3), "rk3_steps": n_steps, "ms_per_rk3": ms / n_steps,
           "launch": "CUDA graph replays (two RK3 steps each)", "stage_kernel_ms": stage_ms,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                        "frac": achieved / hbm_peak},
           "pipe": {"bound": f"fp{prec}", "achieved": tflops, "peak": fma_peak[prec], "unit": "TFLOP/s",
                    "frac": tflops / fma_peak[prec], "flops_per_site_step": 12 * flow_flops_per_link_stage(prec),
                    "peak_kind": "measured FMA rate (qcb_diag_fma_rate)"},
           "clocks": clk.summary()}
    if ms_meas is not None:
        out["measured_flow"] = {"rk3_steps": n_steps, "measurements": n_steps + 1,
                                "each": "Q, E and plaquette (measuring stage 1)", "warmup": "one 3-step measured flow",
                                "seconds": ms_meas * 1e-3,
                                "site_steps_per_s": V * n_steps / (ms_meas * 1e-3)}
    return out


def flow_accuracy(qcb, src, n_steps):
    """|dQ|, dE/E and dP of FP32 flows against the FP64 flow of the same configuration."""
    ref = qcb.GradientFlow(src, 0.02, prec=64, store=0)
    t64, p64 = ref.measure(src, n_steps, 1, plaquette=True)
    ref.close()
    out = {}
    for store, tag in ((0, "fp32_18"), (1, "fp32_12")):
        fl = qcb.GradientFlow(src, 0.02, prec=32, store=store)
        t32, p32 = fl.measure(src, n_steps, 1, plaquette=True)
        fl.close()
        out[tag] = {"dQ_max": float(max(abs(t32[:, 1] - t64[:, 1]))),
                    "dE_rel_max": float(max(abs(t32[:, 2] - t64[:, 2]) / abs(t64[:, 2]))),
                    "dP_max": float(max(abs(p32 - p64))), "flow_steps": n_steps,
                    "Q_final_fp64": float(t64[-1, 1]), "E_final_fp64": float(t64[-1, 2])}
    return out


def run_precision(qcb, n_therm: int = 500, n_flow: int = 400):
    """The precision configuration at full size: 48^4, beta = 6.2, hot start from seed 99 and
    n_therm FP64 heatbath sweeps (N_hits = 2), then the flow eps = 0.02 for n_flow steps (t = 8.0)
    measured at every step in FP64 and in FP32 (18 and 12 reals); max |dQ(t)|, dE(t)/E(t) and
    dP(t) over all n_flow + 1 measurements against the FP64 flow."""
    Lp = (48, 48, 48, 48)
    f = qcb.GaugeField(Lp, qcb.PREC_F64, qcb.STORE_18)
    f.hot_start(99)
    for k in range(n_therm):
        f.hb_sweep(6.2, N_HITS, 99, k)
    plaq = f.plaquette()
    ref = qcb.GradientFlow(f, 0.02, prec=64, store=0)
    t64, p64 = ref.measure(f, n_flow + 1, 1, plaquette=True)
    ref.close()
    out = {"L": list(Lp), "beta": 6.2, "therm_sweeps": n_therm, "n_hits": N_HITS, "plaquette_therm": plaq,
           "flow_steps": n_flow, "t_final": float(t64[-1, 0]), "Q_final_fp64": float(t64[-1, 1]),
           "E_final_fp64": float(t64[-1, 2])}
    for store, tag in ((0, "fp32_18"), (1, "fp32_12")):
        fl = qcb.GradientFlow(f, 0.02, prec=32, store=store)
        t32, p32 = fl.measure(f, n_flow + 1, 1, plaquette=True)
        fl.close()
        out[tag] = {"dQ_max": float(max(abs(t32[:, 1] - t64[:, 1]))),
                    "dE_rel_max": float(max(abs(t32[:, 2] - t64[:, 2]) / abs(t64[:, 2]))),
                    "dP_max": float(max(abs(p32 - p64)))}
    f.close()
    return out


def run_batch(qcb, n_sweeps: int = 300):
    """Batched chains (the batching configuration): 96x8^4 + 96x12^4 + 48x16^4 + 16x24^4, beta ~
    U[5.7, 6.3], seeds 0..255, hot starts, FP64, N_hits = 1; launch shape and storage autotuned on
    the live batch, then n_sweeps CUDA-graph sweeps timed.  Per-chain <P> of one chain of each size
    is checked against a separate single-chain run of the same seed, storage and sweeps; the
    speed-up is against the same sweeps run chain by chain."""
    import numpy as np
    import torch

    rng = np.random.default_rng(0)
    Ls = [(8,) * 4] * 96 + [(12,) * 4] * 96 + [(16,) * 4] * 48 + [(24,) * 4] * 16
    betas = rng.uniform(5.7, 6.3, len(Ls))
    b = qcb.Batch(Ls, betas, list(range(len(Ls))))
    b.hot_start()
    variant, tune_ms = b.tune(1, 2, allow_store_change=True)
    k_tune = b.info()["sweep"]  # the tuning sweeps ran in the 18-real storage
    b.sweep(1, 2)
    b.sync()
    s = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    b.sweep(1, n_sweeps)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / n_sweeps
    info = b.info()
    plaq = b.plaquette()
    # per-chain check: the chain of each size against its own single-lattice run (same seed and
    # sweeps; 18-real storage for the tuning sweeps, then the storage the tuner chose)
    checked, dp = [], 0.0
    for i in (0, 96, 192, 240):
        f = qcb.GaugeField(Ls[i], qcb.PREC_F64, qcb.STORE_18)
        f.hot_start(i)
        for k in range(info["sweep"]):
            if k == k_tune and info["store"] != qcb.STORE_18:
                g = qcb.GaugeField(Ls[i], qcb.PREC_F64, info["store"])
                g.copy_from(f)
                f.close()
                f = g
            f.hb_sweep(float(betas[i]), 1, i, k)
        p1 = f.plaquette()
        f.close()
        checked.append(i)
        dp = max(dp, abs(p1 - float(plaq[i])))
    b.close()
    V = sum(L[0] ** 4 for L in Ls)
    serial = 0.0
    per = {}
    for Lc, cnt in (((8,) * 4, 96), ((12,) * 4, 96), ((16,) * 4, 48), ((24,) * 4, 16)):
        f = qcb.GaugeField(Lc)
        f.hot_start(1)
        for k in range(3):
            f.hb_sweep(6.0, 1, 1, k)
        f.sync()
        t0 = time.perf_counter()
        for k in range(10):
            f.hb_sweep(6.0, 1, 1, 3 + k)
        f.sync()
        one = (time.perf_counter() - t0) / 10 * 1e3
        per[f"{Lc[0]}^4"] = one
        serial += cnt * one
        f.close()
    return {"chains": len(Ls), "sites": V, "n_hits": 1, "timed_sweeps": n_sweeps, "total_sweeps": info["sweep"],
            "ms_per_sweep": ms, "link_upd_per_s": 4 * V / (ms * 1e-3),
            "serial_ms_per_sweep": serial, "serial_single_sweep_ms": per, "speedup_vs_serial": serial / ms,
            "tuned": {"variant": variant, "store": "12" if info["store"] == 1 else "18", "ms": tune_ms},
            "launches_per_sweep": 9, "graph": True,
            "per_chain_check": {"chains": checked, "max_abs_dP_vs_single_chain": dp}}


def serve_once(qcb, reqs, rate: float, store: int):
    """One server run: requests (L, input links, steps) submitted at Poisson arrival times of the
    given rate; returns latency (submit -> result), queue wait (submit -> admission) and rates."""
    import numpy as np

    arr = np.cumsum(np.random.default_rng(7).exponential(1.0 / rate, len(reqs)))
    site_steps = sum(int(L) ** 4 * (n - 1) for L, _, n in reqs)
    srv = qcb.Server(150 << 30, prec=qcb.PREC_F32, store=store)
    for L, U, _ in {int(L): (L, U, n) for L, U, n in reqs}.values():  # untimed warm-up, as in run_serve
        srv.submit(1_000_000 + int(L), (int(L),) * 4, U, 0.02, 4)
    srv.wait(300.0)
    while srv.poll() is not None:
        pass
    time.sleep(SERVE_COOL_S)  # every arm starts from an idle GPU
    start = srv.now()
    k, done = 0, {}
    while len(done) < len(reqs):
        now = srv.now() - start
        while k < len(reqs) and arr[k] <= now:
            L, U, n = reqs[k]
            srv.submit(k, (int(L),) * 4, U, 0.02, n)
            k += 1
        r = srv.poll()
        if r is None:
            time.sleep(0.0005)
            continue
        done[r[0]] = r
    lat = np.array([done[i][2][2] - (start + arr[i]) for i in range(len(reqs))])
    wait = np.array([done[i][2][1] - done[i][2][0] for i in range(len(reqs))])
    wall = max(done[i][2][2] for i in range(len(reqs))) - start
    st = srv.stats()
    srv.close()
    return {"rate_per_s": rate, "requests": len(reqs), "offered_site_steps_per_s": site_steps * rate / len(reqs),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "queue_wait_p50_s": float(np.percentile(wait, 50)), "queue_wait_p99_s": float(np.percentile(wait, 99)),
            "configs_per_s": len(reqs) / wall, "site_steps_per_s": site_steps / wall,
            "peak_resident": st["peak_resident"], "peak_bytes": st["peak_bytes"]}


def run_serve(qcb, n_req: int, stores=(0, 1), low_rates=(4.0, 2.0), n_low: int = 12):
    """Serving (the serving configuration): Poisson arrivals at 100 req/s, L in {8,12,16,20,24,32}
    with p = (.3,.25,.2,.1,.1,.05), beta ~ U[5.8, 6.3], inputs = 50 FP64 sweeps from seed = request
    id (excluded from latency), flow eps = 0.02 to t = L^2/32 in FP32 links with FP64 reprojection
    and Q/E every step; against one-at-a-time plain FP64 flow.  The saturated run is made in each
    FP32 storage of `stores`; the faster is reported at the top level (the other under
    "other_storage").  100 req/s offers several times what one GPU can flow, so that run measures a
    saturated queue; the first n_low requests are also offered at the lower rates, below saturation."""
    import numpy as np

    rng = np.random.default_rng(2026)
    sizes = rng.choice([8, 12, 16, 20, 24, 32], size=n_req, p=[.3, .25, .2, .1, .1, .05])
    betas = rng.uniform(5.8, 6.3, n_req)
    arr = np.cumsum(rng.exponential(1.0 / 100.0, n_req))
    b = qcb.Batch([(int(x),) * 4 for x in sizes], betas, list(range(n_req)))
    b.hot_start()
    b.sweep(1, 50)
    inputs = [b.download(i) for i in range(n_req)]
    b.close()
    steps = [int(round(x * x / 32 / 0.02)) + 1 for x in sizes]
    reqs = list(zip(sizes, inputs, steps))
    site_steps = sum(int(x) ** 4 * (n - 1) for x, n in zip(sizes, steps))
    arms = {}
    first_of = {int(x): i for i, x in reversed(list(enumerate(sizes)))}  # one input of each size
    for store in stores:
        srv = qcb.Server(150 << 30, prec=qcb.PREC_F32, store=store)
        # untimed warm-up: one 3-step request of each size grows the memory pool, allocates the
        # big requests' scratch and captures the shared launches' graphs
        for x, i in first_of.items():
            srv.submit(1_000_000 + x, (x,) * 4, inputs[i], 0.02, 4)
        srv.wait(300.0)
        while srv.poll() is not None:
            pass
        time.sleep(SERVE_COOL_S)  # every arm starts from an idle GPU
        start = srv.now()
        k, done = 0, {}
        while len(done) < n_req:
            now = srv.now() - start
            while k < n_req and arr[k] <= now:
                srv.submit(k, (int(sizes[k]),) * 4, inputs[k], 0.02, steps[k])
                k += 1
            r = srv.poll()
            if r is None:
                time.sleep(0.0005)
                continue
            done[r[0]] = r
        lat = np.array([done[i][2][2] - (start + arr[i]) for i in range(n_req)])
        wait = np.array([done[i][2][1] - done[i][2][0] for i in range(n_req)])
        wall = max(done[i][2][2] for i in range(n_req)) - start
        st = srv.stats()
        srv.close()
        arms[store] = {"prec": "fp32-12" if store == 1 else "fp32-18",
                       "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                       "queue_wait_p50_s": float(np.percentile(wait, 50)),
                       "queue_wait_p99_s": float(np.percentile(wait, 99)),
                       "configs_per_s": n_req / wall, "site_steps_per_s": site_steps / wall,
                       "peak_resident": st["peak_resident"], "peak_bytes": st["peak_bytes"]}
    store = max(arms, key=lambda s_: arms[s_]["configs_per_s"])
    # the serial FP64 arm: one field and one flow state per lattice size, allocated before the timed
    # loop (as the server's pool is), then one request at a time from its host configuration to its
    # results
    serial = {}
    for x in sorted(set(int(v) for v in sizes)):
        fx = qcb.GaugeField((x,) * 4, 64, 0)
        serial[x] = (fx, qcb.GradientFlow(fx, 0.02, prec=64, store=0))
        fx.upload(inputs[first_of[x]])
        serial[x][1].measure(fx, 4, 1)  # untimed warm-up: allocations and measurement graphs
    tq, lat2, busy = 0.0, [], 0.0
    time.sleep(SERVE_COOL_S)
    for i in range(n_req):
        t0 = time.perf_counter()
        f, fl = serial[int(sizes[i])]
        f.upload(inputs[i])
        fl.measure(f, steps[i], 1)
        dt = time.perf_counter() - t0
        busy += dt
        tq = max(tq, arr[i]) + dt
        lat2.append(tq - arr[i])
    for f, fl in serial.values():
        fl.close()
        f.close()
    lat2 = np.array(lat2)
    low = [serve_once(qcb, reqs[:n_low], r, store) for r in low_rates]
    out = {"requests": n_req, "rate_per_s": 100.0, "site_steps": site_steps,
           "offered_site_steps_per_s": site_steps * 100.0 / n_req, "saturated": True}
    out.update(arms[store])
    out.update({"serial_fp64": {"p50_s": float(np.percentile(lat2, 50)), "p99_s": float(np.percentile(lat2, 99)),
                                "configs_per_s": n_req / tq, "site_steps_per_s": site_steps / busy},
                "speedup_configs_per_s": arms[store]["configs_per_s"] / (n_req / tq),
                "other_storage": {a["prec"]: {"configs_per_s": a["configs_per_s"], "p50_s": a["p50_s"],
                                              "p99_s": a["p99_s"],
                                              "speedup_configs_per_s": a["configs_per_s"] / (n_req / tq)}
                                  for s_, a in arms.items() if s_ != store},
                "below_saturation": low})
    return out


def capture_batch(qcb, args):
    """A quarter of the batching configuration (same mix of 8^4 ... 24^4 chains and couplings,
    1.5 GB FP64) for ncu captures of the tiled heatbath: 12-real storage and launch shape 0 (the
    tuner's usual choice on the full batch), `warmup` untimed then `steps` CUDA-graph sweeps."""
    import numpy as np

    rng = np.random.default_rng(0)
    Ls = [(8,) * 4] * 24 + [(12,) * 4] * 24 + [(16,) * 4] * 12 + [(24,) * 4] * 4
    b = qcb.Batch(Ls, rng.uniform(5.7, 6.3, len(Ls)), list(range(len(Ls))), qcb.PREC_F64, qcb.STORE_12)
    b.hot_start()
    b.set_variant(0)
    b.sweep(1, args.warmup)
    b.sweep(1, args.steps)
    b.sync()
    b.close()


def capture_serve(qcb, args):
    """24 serving requests of 16^4 (FP32-18, 1.1 GB resident), all on the shared tiled path, each
    flowed `steps` RK3 steps, for ncu captures of the shared flow stage and clover pass.  The inputs
    are made before the server starts and submitted back to back, so with a few hundred steps all
    24 requests are resident together after the first ticks."""
    f = qcb.GaugeField((16,) * 4)
    inputs = []
    for rid in range(24):
        f.hot_start(1000 + rid)
        inputs.append(f.download())
    f.close()
    srv = qcb.Server(150 << 30, qcb.PREC_F32, qcb.STORE_18)
    for rid, U in enumerate(inputs):
        srv.submit(rid, (16,) * 4, U, 0.02, args.steps)
    srv.wait(600.0)
    while srv.poll() is not None:
        pass
    srv.close()


def run_ours(args, rank: int, world: int, local: int):
    import torch

    qcb = load_package()
    torch.cuda.set_device(local)
    if args.only in ("batch", "serve"):
        (capture_batch if args.only == "batch" else capture_serve)(qcb, args)
        return
    hbm_peak, peak_kind = peaks()
    V = L[0] * L[1] * L[2] * L[3]
    f = qcb.GaugeField(L, qcb.PREC_F64, qcb.STORE_18)
    f.hot_start(SEED_HOT)
    stream, e0, e1 = cuda_timer(qcb, f)

    if args.only == "obs":
        # observables and 12-real heatbath of every form on the configuration (for ncu captures):
        # per form `steps` plaquette and clover passes; then 2 FP64 12-real heatbath sweeps
        for i in range(args.warmup):
            f.hb_sweep(BETA, N_HITS, SEED_HB, i)
        for prec, store in ((64, 0), (64, 1), (32, 0), (32, 1)):
            g = qcb.GaugeField(L, prec, store)
            g.copy_from(f)
            for k in range(args.steps):
                g.plaquette()
                g.clover_qe()
            g.close()
        g = qcb.GaugeField(L, qcb.PREC_F64, qcb.STORE_12)
        g.copy_from(f)
        for k in range(2):
            g.hb_sweep(BETA, N_HITS, SEED_HB, 1000 + k)
        g.close()
        f.close()
        return

    if args.only in ("flow", "mflow"):
        for i in range(args.warmup):
            f.hb_sweep(BETA, N_HITS, SEED_HB, i)
        fma_peak = {64: qcb.fma_rate(64) / 1e12, 32: qcb.fma_rate(32) / 1e12}
        for prec, store in ((64, 0), (32, 0), (32, 1)):
            if args.only == "mflow":  # the measured flow alone (ncu captures of its kernels)
                fl = qcb.GradientFlow(f, 0.02, prec=prec, store=store)
                fl.measure(f, args.steps + 1, 1, plaquette=True)
                fl.close()
            else:
                flow_block(qcb, f, prec, store, args.steps, hbm_peak, fma_peak, local, measured=False)
        f.close()
        return

    # ---------------- device-resident heatbath: warm-up, then K timed sweeps
    # (--only hb --hb-hits n profiles the kernel at another N_hits; every bench line uses N_HITS)
    nh = args.hb_hits if args.only == "hb" else N_HITS
    for i in range(args.warmup):
        f.hb_sweep(BETA, nh, SEED_HB, i)
    f.sync()
    barrier(world)
    f.timing(True)
    f.timing_reset()
    n_launch0 = qcb.launch_count()
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(args.steps):
            f.hb_sweep(BETA, nh, SEED_HB, args.warmup + i)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
    n_launch = qcb.launch_count() - n_launch0
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    n_hb, hb_ms = f.timing_read(qcb.K_HB)
    f.timing(False)
    link_upd = 4 * V * args.steps
    value = replica_rate(link_upd, ms, world)
    per_launch_ms = hb_ms / n_hb
    bytes_launch = 9 * S_U[64] * (V // 2)  # 9 s_U per link-update, V/2 link-updates per (parity, mu) launch
    achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
    traffic = profile_traffic("hb_subsweep_fp64_32x4")
    plaq = f.plaquette()

    if args.only == "hb":
        f.close()
        return

    # ---------------- end to end through the C ABI with host buffers: every step uploads its
    # configuration from pinned host memory, sweeps, and reads the plaquette back.  Headline: the
    # pipelined upload (the next step's copy overlaps this step's sweep); beside it the
    # synchronous upload.
    U_host = torch.empty(V * 72, dtype=torch.float64, pin_memory=True)
    qcb._check(qcb.lib().qcb_field_download_aos(f.h, U_host.data_ptr()))
    e2e_f = qcb.GaugeField(L, qcb.PREC_F64, qcb.STORE_18)
    es, ea, eb = cuda_timer(qcb, e2e_f)
    n_e2e = max(3, min(args.steps, 10))

    def e2e_steps(n, sweep0, pipelined):
        if pipelined:
            e2e_f.prefetch_ptr(U_host.data_ptr())
        for i in range(n):
            if pipelined:
                e2e_f.commit_prefetch()
            else:
                qcb._check(qcb.lib().qcb_field_upload_aos(e2e_f.h, U_host.data_ptr()))
            e2e_f.hb_sweep(BETA, N_HITS, SEED_HB, sweep0 + i)
            if pipelined and i + 1 < n:
                e2e_f.prefetch_ptr(U_host.data_ptr())
            e2e_f.plaquette()  # device -> host read of the step's result

    def e2e_timed(pipelined, sweep0):
        e2e_steps(2, sweep0, pipelined)
        e2e_f.sync()
        barrier(world)
        ea.record(es)
        ea.synchronize()  # no copy of the timed steps starts before the start event
        e2e_steps(n_e2e, sweep0 + 100, pipelined)
        eb.record(es)
        eb.synchronize()
        return max_over_ranks(ea.elapsed_time(eb), world)

    e2e_ms = e2e_timed(True, 20_000)
    e2e_value = replica_rate(4 * V * n_e2e, e2e_ms, world)
    e2e_sync_value = replica_rate(4 * V * n_e2e, e2e_timed(False, 30_000), world)
    e2e_f.close()
    del U_host

    # ---------------- flow: FP64 vs FP32 (18 and 12 reals) on the heatbath configuration
    fma_peak = {64: qcb.fma_rate(64) / 1e12, 32: qcb.fma_rate(32) / 1e12}
    flow = {"fma_peak_tflops": fma_peak}
    flow["fp64"] = flow_block(qcb, f, 64, 0, FLOW_STEPS, hbm_peak, fma_peak, local)
    flow["fp32_18"] = flow_block(qcb, f, 32, 0, FLOW_STEPS, hbm_peak, fma_peak, local)
    flow["fp32_12"] = flow_block(qcb, f, 32, 1, FLOW_STEPS, hbm_peak, fma_peak, local)
    acc = flow_accuracy(qcb, f, 40)
    for k in ("fp32_18", "fp32_12"):
        flow[k].update(acc[k])
        flow[k]["speedup_vs_fp64"] = flow[k]["site_steps_per_s"] / flow["fp64"]["site_steps_per_s"]
        flow[k]["measured_flow"]["speedup_vs_fp64"] = (flow[k]["measured_flow"]["site_steps_per_s"] /
                                                       flow["fp64"]["measured_flow"]["site_steps_per_s"])

    # ---------------- heatbath variants on the same lattice: N_hits = 1, FP32 links
    hb_more = {}
    for tag, prec, nh in (("fp64_nhits1", 64, 1), ("fp32_nhits2", 32, 2)):
        g = qcb.GaugeField(L, prec, qcb.STORE_18)
        g.copy_from(f)
        for i in range(2):
            g.hb_sweep(BETA, nh, SEED_HB, 50_000 + i)
        g.timing(True)
        g.timing_reset()
        for i in range(5):
            g.hb_sweep(BETA, nh, SEED_HB, 50_100 + i)
        n, kms = g.timing_read(qcb.K_HB)
        su = S_U[prec]
        ach = 9 * su * (V // 2) / (kms / n * 1e-3) / 1e9
        hb_more[tag] = {"link_upd_per_s": (V // 2) / (kms / n * 1e-3), "per_launch_ms": kms / n,
                        "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                                     "frac": ach / hbm_peak}}
        g.close()

    precision = run_precision(qcb) if args.parts in ("all",) else None
    batch = run_batch(qcb) if args.parts in ("all",) else None
    serve = run_serve(qcb, args.serve_requests) if args.parts in ("all",) else None

    cpu = None
    if rank == 0 and args.cpu_seconds > 0:
        cpu = cpu_sample(seconds=args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "link-upd/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(CONFIG, parallelism=f"replicas x{world}"),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic,
                         "traffic_source": "ncu DRAM bytes per launch of this kernel, from the committed capture "
                                           "profiles/hb_subsweep_fp64_32x4.md (not measured in this run)",
                         "kernel": "k_hb_subsweep<double,9,mu>",
                         "per_launch_ms": per_launch_ms, "algorithmic_bytes_per_launch": bytes_launch,
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "link-upd/s", "h2d_bytes_per_step": V * 576,
                    "d2h_bytes_per_step": 8, "steps": n_e2e,
                    "step": "upload FP64 AoS config from pinned host (pipelined: the next step's copy overlaps "
                            "this step's sweep) + sweep + plaquette readback via the C ABI",
                    "synchronous_upload_value": e2e_sync_value},
            "hits_per_s": value * N_HITS,
            "gpu_launches": n_launch,
            "clocks": clk.summary(),
            "plaquette_after": plaq,
            "hb": hb_more,
            "flow": flow,
            "precision": precision,
            "batch": batch,
            "serve": serve,
        }
        print(json.dumps(line), flush=True)
    f.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="length of the CPU-baseline sample (0 skips it)")
    ap.add_argument("--only", default="all", choices=["all", "hb", "flow", "mflow", "obs", "batch", "serve"],
                    help="run one part (used for ncu captures of a single kernel family)")
    ap.add_argument("--parts", default="all", choices=["all", "core"],
                    help="core: skip the batch and serving sections")
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--hb-hits", type=int, default=N_HITS,
                    help="N_hits of the heatbath with --only hb (ncu captures at another N_hits)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_setup(args.gpus) if args.impl == "ours" else (
        int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()

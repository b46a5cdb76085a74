"""Benchmark of the B200 gauge-field hot path; prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the "plain FP64 at scale" configuration): a 32^4 periodic SU(3) lattice, FP64 links
(18 reals), hot start from seed 7, Wilson action beta = 6.0, N_hits = 2.  One step = one full
checkerboard heatbath sweep (8 (parity, mu) passes, every link updated once with N_hits hits).
`value` is link-updates/s over all ranks with the field resident in HBM; `e2e` is the same metric
through the C ABI with the configuration uploaded from pinned host memory each step and the
plaquette read back.  The flow part of the metric (site-steps/s of the Wilson flow, FP64 vs FP32
18- and 12-real with |dQ|, dE/E and dP against FP64) is measured on the same configuration and
reported under "flow".  Multi-GPU runs are independent replicas (weak scaling, no collective on the
data path).  The reference arm times the CPU restatement of the reference's heatbath on the host
cores.
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
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
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


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
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

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cuda_timer(qcb, field):
    """CUDA events on the field's own stream (the stream the kernels are launched on)."""
    import torch

    stream = torch.cuda.ExternalStream(field.stream)
    return stream, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def cpu_sample(orc, seconds: float = 12.0, threads: int = 0):
    """Times the oracle's heatbath with the reference's cost structure (staple per hit) on the host cores."""
    orc.set_threads(threads)
    U = orc.hot_start(L, SEED_HOT)
    V = U.shape[0]
    n, t0 = 0, time.perf_counter()
    while True:
        orc.hb_subsweep(U, L, BETA, N_HITS, SEED_HB, 0, n % 2, (n // 2) % 4, refcost=True)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": n * (V // 2) / el, "unit": "link-upd/s", "cores": orc.threads(), "kind": "port",
            "sample": f"{n} (parity,mu) sub-sweeps of 32^4 (V/2 links each, N_hits=2, staple recomputed per hit "
                      f"as heatbath_mpi.cpp:12), {el:.1f} s, 1 process x {orc.threads()} OpenMP threads"}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    orc = load_oracle()
    orc.set_threads(0)
    U = orc.hot_start(L, SEED_HOT)
    V = U.shape[0]
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        orc.hb_subsweep(U, L, BETA, N_HITS, SEED_HB, i, i % 2, (i // 2) % 4, refcost=True)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = args.steps * (V // 2) / tot
    sample = (f"each step one (parity,mu) sub-sweep of the 32^4 workload (V/2 = {V // 2} link-updates, N_hits=2, "
              f"staple recomputed per hit); CPU restatement of the reference, 1 process x {orc.threads()} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "link-upd/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "hb_fp64_32^4", "L": list(L), "beta": BETA, "n_hits": N_HITS, "start": "hot seed 7"},
        "cpu_baseline": {"value": value, "unit": "link-upd/s", "cores": orc.threads(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "link-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def flow_block(qcb, src, prec, store, n_steps, n_warm, hbm_peak):
    """Times n_steps RK3 steps (fused stages) and returns site-steps/s and stage-kernel roofline."""
    fl = qcb.GradientFlow(src, 0.02, prec=prec, store=store)
    f = fl.field
    stream, e0, e1 = cuda_timer(qcb, f)
    fl.rk3_step(n_warm)
    f.sync()
    f.timing(True)
    f.timing_reset()
    e0.record(stream)
    fl.rk3_step(n_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    nl, kms = f.timing_read(qcb.K_FLOW)
    f.timing(False)
    V = src.V
    s_u = (S_U12 if store == 1 else S_U)[prec]
    bytes_stage = V * 4 * (2 * s_u) + V * 4 * S_Z[prec] * (4 / 3)  # per stage: read+write U, Z traffic averaged
    achieved = bytes_stage / (kms / nl * 1e-3) / 1e9
    fl.close()
    return {"site_steps_per_s": V * n_steps / (ms * 1e-3), "ms_per_rk3": ms / n_steps,
            "stage_kernel_ms": kms / nl, "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                                                       "unit": "GB/s", "frac": achieved / hbm_peak}}


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


def run_ours(args, rank: int, world: int, local: int):
    import torch

    qcb = load_package()
    torch.cuda.set_device(local)
    hbm_peak, peak_kind = peaks()
    V = L[0] * L[1] * L[2] * L[3]
    f = qcb.GaugeField(L, qcb.PREC_F64, qcb.STORE_18)
    f.hot_start(SEED_HOT)
    stream, e0, e1 = cuda_timer(qcb, f)

    if args.only == "flow":
        for i in range(args.warmup):
            f.hb_sweep(BETA, N_HITS, SEED_HB, i)
        for prec, store in ((64, 0), (32, 0), (32, 1)):
            flow_block(qcb, f, prec, store, args.steps, 2, hbm_peak)
        f.close()
        return

    # ---------------- device-resident heatbath: warm-up, then K timed sweeps
    for i in range(args.warmup):
        f.hb_sweep(BETA, N_HITS, SEED_HB, i)
    f.sync()
    barrier(world)
    f.timing(True)
    f.timing_reset()
    n_launch0 = qcb.launch_count()
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(args.steps):
            f.hb_sweep(BETA, N_HITS, SEED_HB, args.warmup + i)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
    n_launch = qcb.launch_count() - n_launch0
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    n_hb, hb_ms = f.timing_read(qcb.K_HB)
    f.timing(False)
    link_upd = 4 * V * args.steps
    value = world * link_upd / (ms * 1e-3)
    per_launch_ms = hb_ms / n_hb
    bytes_launch = 9 * S_U[64] * (V // 2)  # 9 s_U per link-update, V/2 link-updates per (parity, mu) launch
    achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
    traffic = profile_traffic("hb_subsweep_fp64_32x4")
    plaq = f.plaquette()

    if args.only == "hb":
        f.close()
        return

    # ---------------- end to end through the C ABI with host buffers
    U_host = torch.empty(V * 72, dtype=torch.float64, pin_memory=True)
    qcb._check(qcb.lib().qcb_field_download_aos(f.h, U_host.data_ptr()))
    e2e_f = qcb.GaugeField(L, qcb.PREC_F64, qcb.STORE_18)
    es, ea, eb = cuda_timer(qcb, e2e_f)
    n_e2e = max(3, min(args.steps, 10))
    for i in range(2):
        qcb._check(qcb.lib().qcb_field_upload_aos(e2e_f.h, U_host.data_ptr()))
        e2e_f.hb_sweep(BETA, N_HITS, SEED_HB, 10_000 + i)
        e2e_f.plaquette()
    barrier(world)
    ea.record(es)
    for i in range(n_e2e):
        qcb._check(qcb.lib().qcb_field_upload_aos(e2e_f.h, U_host.data_ptr()))
        e2e_f.hb_sweep(BETA, N_HITS, SEED_HB, 20_000 + i)
        e2e_f.plaquette()  # device -> host read of the step's result
    eb.record(es)
    eb.synchronize()
    e2e_ms = max_over_ranks(ea.elapsed_time(eb), world)
    e2e_value = world * 4 * V * n_e2e / (e2e_ms * 1e-3)
    e2e_f.close()
    del U_host

    # ---------------- flow: FP64 vs FP32 (18 and 12 reals) on the heatbath configuration
    flow = {}
    n_flow = 20
    flow["fp64"] = flow_block(qcb, f, 64, 0, n_flow, 2, hbm_peak)
    flow["fp32_18"] = flow_block(qcb, f, 32, 0, n_flow, 2, hbm_peak)
    flow["fp32_12"] = flow_block(qcb, f, 32, 1, n_flow, 2, hbm_peak)
    acc = flow_accuracy(qcb, f, 40)
    for k in ("fp32_18", "fp32_12"):
        flow[k].update(acc[k])
        flow[k]["speedup_vs_fp64"] = flow[k]["site_steps_per_s"] / flow["fp64"]["site_steps_per_s"]

    cpu = None
    if rank == 0 and args.cpu_seconds > 0:
        orc = load_oracle()
        cpu = cpu_sample(orc, seconds=args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "link-upd/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "hb_fp64_32^4", "L": list(L), "beta": BETA, "n_hits": N_HITS,
                       "start": "hot seed 7", "step": "one full checkerboard sweep (8 (parity,mu) launches)",
                       "l2": "inputs larger than L2 (604 MB FP64 field vs 126 MB L2)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic, "kernel": "k_hb_subsweep<double,9,mu>",
                         "per_launch_ms": per_launch_ms, "algorithmic_bytes_per_launch": bytes_launch,
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "link-upd/s", "h2d_bytes_per_step": V * 576,
                    "d2h_bytes_per_step": 8, "steps": n_e2e,
                    "step": "upload FP64 AoS config from pinned host + sweep + plaquette readback via the C ABI"},
            "gpu_launches": n_launch,
            "clocks": clk.summary(),
            "plaquette_after": plaq,
            "flow": flow,
        }
        print(json.dumps(line), flush=True)
    f.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="length of the CPU-baseline sample (0 skips it)")
    ap.add_argument("--only", default="all", choices=["all", "hb", "flow"],
                    help="run one part (used for ncu captures of a single kernel family)")
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

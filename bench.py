"""Benchmark of the explicit RK3 residual-and-update path (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): 3-D sine-wave advection
on the perturbed curvilinear periodic grid of 256^3 intervals (257^3 nodes, 4 ghost
layers), WENO7 primitive reconstruction + AUSM+, 8th-order collocated viscous terms
(mu = 1e-4 constant, Pr = 0.72), SSP-RK3 at a fixed dt equal to the CFL-0.5 step of the
initial state.  One "step" = one full SSP-RK3 step (3 stages) of the whole block; one
cell-update = one interior node advanced through one step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cb200|reference] [--n 256]

--impl reference times the reference algorithm's CPU form on the host cores: the FP64
oracle (the reference has no CPU implementation of this path; its kernels are CUDA only),
on a bounded sample of the same workload.
Under torchrun each rank runs an independent replica of the workload on its own GPU
(weak scaling, no data-path collective); rank 0 prints the line.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "corefl-cpc_b200"))

METRIC = "RK3 cell-updates/s, mixed vs FP64 at equal L1 error; p50/p99 solve latency"
UNIT = "cell-updates/s"

# Compulsory HBM traffic of each kernel per interior node it processes (every array it reads or
# writes counted once), for the per-kernel rooflines.  Plain form: FP64 arrays.
KERNEL_BYTES_PER_NODE = {
    "pv_flux_x": 8 * (5 + 3 + 1 + 10), "pv_flux_y": 8 * (5 + 3 + 1 + 10), "pv_flux_z": 8 * (5 + 3 + 1 + 10),
    "weno_char_x": 8 * (5 + 2 + 3 + 1 + 10), "weno_char_y": 8 * (5 + 2 + 3 + 1 + 10),
    "weno_char_z": 8 * (5 + 2 + 3 + 1 + 10),
    # u, v, w, T + 9 metric + mu read, 12 node fluxes written
    "visc8_node_flux": 8 * (4 + 9 + 1 + 12),
    # 12 node fluxes + J read, dq (5) written: the divergence assigns dq
    "visc8_divergence": 8 * (12 + 1 + 5),
    "stage_update": 8 * (5 + 5 + 5 + 1 + 5 + 6),
}
# Mixed form: the sweeps and node fluxes read the FP32 copies of bv, the metric and J, the node
# fluxes live in FP32 scratch; dq, the state and mu stay FP64.
KERNEL_BYTES_PER_NODE_MIXED = dict(KERNEL_BYTES_PER_NODE, **{
    "pv_flux_x": 4 * (5 + 3 + 1) + 8 * 10, "pv_flux_y": 4 * (5 + 3 + 1) + 8 * 10,
    "pv_flux_z": 4 * (5 + 3 + 1) + 8 * 10,
    "visc8_node_flux": 4 * (4 + 9 + 12) + 8, "visc8_divergence": 4 * (12 + 1) + 8 * 5,
})
# Executed FP64 operations per interior node (an FMA counted as 2) of the FP64 sweeps, from ncu's
# sm__sass_thread_inst_executed_op_d{fma,mul,add}_pred_on on the 129^3 sine wave, per node of one
# launch; these kernels are bound by the FP64 pipe, not by HBM.  The FP64 peak is the B200's
# nominal (no measured FP64 figure is available).
KERNEL_FP64_FLOPS_PER_NODE = {"pv_flux_x": 1500, "pv_flux_y": 1500, "pv_flux_z": 1500}
FP64_NOMINAL_TFLOPS = 37.0
FLOPS_PER_CELL_UPDATE = 15000  # 3 stages x (3 sweeps x 1,500 + node fluxes 406 + divergence 144)
# per padded node (kernels that sweep the ghost layers too)
KERNEL_BYTES_PER_PADDED_NODE = {"bv_to_f32": 6 * (8 + 4), "store_qn": 5 * 16, "properties": 8 * (4 + 2)}


def kernel_rooflines(prof, nodes, padded, bytes_map, peak):
    """Achieved algorithmic GB/s of every profiled kernel whose compulsory bytes are known."""
    out = {}
    for name, (count, ms) in prof.items():
        per = bytes_map.get(name)
        n = nodes
        if per is None:
            per, n = KERNEL_BYTES_PER_PADDED_NODE.get(name), padded
        if per is None or ms <= 0:
            continue
        gbs = per * n * count / (ms * 1e-3) / 1e9
        out[name] = {"ms_per_step": ms, "launches": count, "bytes_per_node": per, "achieved_GBps": gbs,
                     "frac": gbs / peak}
    return out


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cb200", choices=["cb200", "reference"])
    ap.add_argument("--n", type=int, default=256, help="intervals per direction of the sine-wave grid")
    ap.add_argument("--cpu-n", type=int, default=48, help="intervals of the CPU-baseline sample grid")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form")
    ap.add_argument("--no-serve", action="store_true", help="skip the served reactor/shock-tube workload")
    ap.add_argument("--no-reacting", action="store_true", help="skip the reacting H2/air box")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-blocks form")
    ap.add_argument("--batch-blocks", type=int, default=296, help="blocks of the batched-blocks form")
    ap.add_argument("--batch-steps", type=int, default=5, help="steps of the batched-blocks form")
    ap.add_argument("--reacting-n", type=int, default=192, help="nodes per side of the reacting H2/air box")
    ap.add_argument("--no-c5", action="store_true", help="skip the two-temperature AIR5 square cylinder")
    ap.add_argument("--c5-side", type=int, default=256, help="nodes along the body side of each cylinder block")
    ap.add_argument("--c5-normal", type=int, default=512, help="wall-normal nodes of each cylinder block")
    ap.add_argument("--c5-steps", type=int, default=100, help="timed steps of the square cylinder")
    ap.add_argument("--c5-warmup", type=int, default=20, help="warm-up steps of the square cylinder")
    ap.add_argument("--c5-variants", type=int, default=16,
                    help="freestream-Mach variants of the cylinder batched in one context (0: skip)")
    ap.add_argument("--c5-variant-steps", type=int, default=20, help="timed steps of the batched variants")
    ap.add_argument("--reacting-steps", type=int, default=5, help="timed steps of the reacting H2/air box")
    ap.add_argument("--serve-seconds", type=float, default=0.05,
                    help="length of the seeded Poisson arrival window of the served workload")
    ap.add_argument("--serve-tube-t-end", type=float, default=1e-6,
                    help="physical end time of the served shock tubes (the workload's is 50e-6)")
    ap.add_argument("--serve-reactor-t-end", type=float, default=1e-3,
                    help="physical end time of the served 0-D reactors")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="mean arrivals per second")
    ap.add_argument("--reactor-sweep", action="store_true",
                    help="time one ROK4E attempt of the batched H2/air reactors at several batch sizes")
    ap.add_argument("--schedule", default=None,
                    help="use these tile widths instead of timing them: 'NI' for the y/z sweeps and the "
                         "batch, or 'NI,CS' to also fix the batch's cluster size (e.g. from an earlier run)")
    ap.add_argument("--accuracy-steps", type=int, default=100,
                    help="RK3 steps of the mixed-vs-FP64 accuracy run (the workload's 100 steps)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running (read-only query)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(args, samples=None, seconds=None):
    """FP64 oracle (all host threads) on the sine-wave workload at --cpu-n intervals, timed.

    With `samples` (the GPU's results on the same samples, from accuracy_samples) the oracle's
    results on those samples also check the GPU forms: the sine wave run the same number of steps
    at the same dt (L1 / Linf of rho), and the reacting-box sample (L1 / Linf of rho, T and Y_k),
    each relative to the mean magnitude of the oracle's field."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import numpy as np
    import oracle_py
    from cb200 import cases
    n = args.cpu_n
    case = cases.sine_wave(n=n)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    threads = os.cpu_count() or 1
    oracle_py.set_threads(threads)
    oracle_py.boundary(p, b, faces)
    oracle_py.properties(p, b)
    dt = samples["sine_dt"] if samples else oracle_py.cfl_dt(p, b)
    max_steps = samples["sine_steps"] if samples else 50
    budget = seconds if seconds is not None else args.cpu_seconds
    t0 = time.perf_counter()
    steps = 0
    while True:
        oracle_py.rk3_step(p, [b], [faces], dt, True)
        steps += 1
        el = time.perf_counter() - t0
        if steps >= max_steps or (not samples and el >= budget):
            break
    nodes = case.n_nodes
    out = {"value": nodes * steps / el, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"FP64 oracle, sine-wave WENO7+AUSM+/visc8 on {n}^3 intervals ({nodes} nodes), "
                     f"{steps} RK3 steps in {el:.1f} s", "steps": steps, "seconds": el}
    if samples:
        g = b.ngg
        rho_o = b.a["bv"][0, g:-g, g:-g, g:-g]
        mo = np.abs(rho_o).mean()
        acc = {"sample": f"sine wave {n}^3 intervals, {steps} steps at dt {dt:.6g}"}
        for form in ("fp64", "mixed"):
            d = np.abs(samples["sine_rho_" + form] - rho_o)
            acc["l1_rho_" + form] = float(d.mean() / mo)
            acc["linf_rho_" + form] = float(d.max() / mo)
        out["accuracy_vs_oracle"] = acc
        if "box" in samples:
            bx = samples["box"]
            from cb200 import mech as mechmod
            h2 = mechmod.load_json(os.path.join(REPO, "tests", "golden", "h2_li2004.json"))
            c = cases.h2_air_box(h2, n_nodes=bx["n"])
            pb, hb, fb = c.param, c.blocks[0], c.faces[0]
            oracle_py.boundary(pb, hb, fb)
            oracle_py.properties(pb, hb)
            for _ in range(bx["steps"]):
                oracle_py.rk3_step(pb, [hb], [fb], bx["dt"], True)
            gb = hb.ngg
            inner = (slice(gb, -gb), slice(gb, -gb), slice(gb, -gb))
            ref = {"rho": hb.a["bv"][0][inner], "T": hb.a["bv"][5][inner], "Y": hb.a["sv"][(slice(None),) + inner]}
            bacc = {"sample": f"reacting H2/air box {bx['n']}^3 nodes, {bx['steps']} steps at dt {bx['dt']:g}"}
            for form in ("fp64", "mixed"):
                for k in ("rho", "T", "Y"):
                    dd = np.abs(bx[form][k] - ref[k])
                    bacc[f"l1_{k}_{form}"] = float(dd.mean() / np.abs(ref[k]).mean())
                    bacc[f"linf_{k}_{form}"] = float(dd.max() / np.abs(ref[k]).mean())
            out["reacting_accuracy_vs_oracle"] = bacc
    return out


def accuracy_samples(args, local_rank):
    """The GPU forms on the accuracy samples the CPU-baseline leg checks against the oracle: the
    sine wave at --cpu-n intervals run --accuracy-steps steps at its CFL-0.5 dt, and a 24^3
    reacting H2/air box run 10 steps of 2e-9 s, each in the FP64 and the mixed form from the same
    initial state."""
    import numpy as np
    import torch
    import cb200
    from cb200 import abi, cases
    from cb200 import mech as mechmod
    from cb200.field import DeviceBlock
    sh = torch.cuda.current_stream().cuda_stream
    out = {"sine_steps": args.accuracy_steps}
    case = cases.sine_wave(n=args.cpu_n)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    g = hb.ngg
    dt = None
    for form, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        dev = DeviceBlock(hb, device=f"cuda:{local_rank}")
        pv = abi.ParamView.from_buffer_copy(p)
        pv.precision = prec
        ctx = cb200.Context(pv)
        ctx.bind(0, dev.view(), faces)
        ctx.boundary(0, sh)
        ctx.properties(0, sh)
        if dt is None:
            dt = ctx.cfl_dt(sh)
        for _ in range(args.accuracy_steps):
            ctx.rk3_step(dt, True, sh)
        torch.cuda.synchronize()
        out["sine_rho_" + form] = dev.t["bv"][0, g:-g, g:-g, g:-g].cpu().numpy()
        ctx.close()
        del dev
    out["sine_dt"] = dt
    h2 = mechmod.load_json(os.path.join(REPO, "tests", "golden", "h2_li2004.json"))
    c = cases.h2_air_box(h2, n_nodes=24)
    pb, hb2, fb = c.param, c.blocks[0], c.faces[0]
    gb = hb2.ngg
    inner = (slice(gb, -gb), slice(gb, -gb), slice(gb, -gb))
    box = {"n": 24, "steps": 10, "dt": 2e-9}
    for form, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        dev = DeviceBlock(hb2, device=f"cuda:{local_rank}")
        pv = abi.ParamView.from_buffer_copy(pb)
        pv.precision = prec
        ctx = cb200.Context(pv)
        ctx.bind(0, dev.view(), fb)
        ctx.boundary(0, sh)
        ctx.properties(0, sh)
        for _ in range(box["steps"]):
            ctx.rk3_step(box["dt"], True, sh)
        torch.cuda.synchronize()
        bv = dev.t["bv"].cpu().numpy()
        box[form] = {"rho": bv[0][inner], "T": bv[5][inner], "Y": dev.t["sv"].cpu().numpy()[(slice(None),) + inner]}
        ctx.close()
        del dev
    out["box"] = box
    return out


def reference_arm(args, rank):
    if rank != 0:
        return
    base = cpu_baseline(args)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": base["steps"], "warmup": 1, "ms_per_step": 1e3 * base["seconds"] / base["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"sine-wave 3-D curvilinear periodic, WENO7+AUSM+, 8th-order viscous, "
                                   f"sample {args.cpu_n}^3 intervals of the {args.n}^3 workload",
                       "l2": "n/a (CPU)"},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def load_traffic():
    """DRAM bytes per node of each kernel from the committed ncu summary, if present."""
    try:
        with open(os.path.join(REPO, "profiles", "traffic_per_node.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def tune_sweeps(ctx, args, stream):
    """The block's sweep tile widths: timed on the block (cb2_autotune), or fixed by --schedule."""
    if args.schedule:
        ni = int(args.schedule.split(",")[0])
        ctx.set_tile_widths(0, [0, ni, ni])
        return [0, ni, ni]
    return ctx.autotune(0, stream)


def gpu_arm(args, rank, world, local_rank):
    import torch
    import cb200
    from cb200 import cases
    from cb200.field import DeviceBlock

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    case = cases.sine_wave(n=args.n)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    dev = DeviceBlock(hb, device=f"cuda:{local_rank}")
    host_state = {n: hb.a[n] for n in ("cv", "bv")}
    gh = hb.ngg
    xyz = torch.from_numpy(case.meta["xyz_sum"][gh:-gh, gh:-gh, gh:-gh].copy())
    del case, hb
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    ctx.properties(0, sh)
    dt = ctx.cfl_dt(sh)
    tile_widths = tune_sweeps(ctx, args, sh)  # y/z sweep tile widths, timed on this block
    nodes = (args.n + 1) ** 3

    for _ in range(args.warmup):
        ctx.rk3_step(dt, True, sh)
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.5)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = ctx.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.rk3_step(dt, True, sh)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launch_count() - n0
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
        ms = float(t.item())
    clocks = sampler.stop() if sampler else None
    status = ctx.read_status(sh)

    # per-kernel durations of one profiled step (same stream, CUDA events)
    ctx.profile(True)
    ctx.rk3_step(dt, True, sh)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    total = sum(v[1] for v in prof.values())
    # the kernel with the largest share of the step among those whose compulsory bytes are known
    known = {k: v for k, v in prof.items() if k in KERNEL_BYTES_PER_NODE} or prof
    top = max(known.items(), key=lambda kv: kv[1][1])
    kname, (kcount, kms) = top
    avg_ms = kms / kcount
    bpn = KERNEL_BYTES_PER_NODE.get(kname)
    peak, peak_kind = measured_peaks()
    roof = None
    if bpn:
        achieved = bpn * nodes / (avg_ms * 1e-3) / 1e9
        traffic = load_traffic().get(kname)
        roof = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": (traffic * nodes if traffic else None),
                "algorithmic_bytes": bpn * nodes, "avg_launch_ms": avg_ms,
                "share": kms / total}
        fpn = KERNEL_FP64_FLOPS_PER_NODE.get(kname)
        if fpn:
            # the roof that binds this kernel: the FP64 pipe
            tf = fpn * nodes / (avg_ms * 1e-3) / 1e12
            roof["compute"] = {"pipe": "fp64", "achieved": tf, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                               "frac": tf / FP64_NOMINAL_TFLOPS, "peak_source": "nominal",
                               "flops_per_node": fpn, "flops_per_cell_update": FLOPS_PER_CELL_UPDATE}
    padded = (args.n + 1 + 8) ** 3
    kernel_roofs = kernel_rooflines(prof, nodes, padded, KERNEL_BYTES_PER_NODE, peak)

    e2e = None
    if not args.no_e2e:
        pin = {n: torch.from_numpy(a).pin_memory() for n, a in host_state.items()}
        out_cv = torch.empty_like(pin["cv"]).pin_memory()
        h2d = sum(t.numel() * 8 for t in pin.values())
        d2h = out_cv.numel() * 8
        k_e2e = max(1, min(args.steps, 10))
        # Every step copies its input state in from pinned host memory and its result out, as a
        # caller holding the state on the host would.  The transfers run on their own streams,
        # double-buffered through device staging arrays, so step k+1's input crosses PCIe while
        # step k computes and step k-1's result crosses back.
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        stage = {n: torch.empty_like(dev.t[n]) for n in ("cv", "bv")}
        outs = [torch.empty_like(dev.t["cv"]) for _ in range(2)]
        ev = lambda: torch.cuda.Event()  # noqa: E731
        ev_in = [ev() for _ in range(k_e2e)]
        ev_staged = [ev() for _ in range(k_e2e)]
        ev_done = [ev() for _ in range(k_e2e)]
        ev_out = [ev() for _ in range(k_e2e)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(s_in)
        with torch.cuda.stream(s_in):
            for n in ("cv", "bv"):
                stage[n].copy_(pin[n], non_blocking=True)
            ev_in[0].record(s_in)
        for k in range(k_e2e):
            stream.wait_event(ev_in[k])
            for n in ("cv", "bv"):
                dev.t[n].copy_(stage[n])
            ev_staged[k].record(stream)
            if k + 1 < k_e2e:
                s_in.wait_event(ev_staged[k])
                with torch.cuda.stream(s_in):
                    for n in ("cv", "bv"):
                        stage[n].copy_(pin[n], non_blocking=True)
                    ev_in[k + 1].record(s_in)
            ctx.rk3_step(dt, True, sh)
            if k >= 2:
                stream.wait_event(ev_out[k - 2])  # the transfer that last read this buffer
            outs[k % 2].copy_(dev.t["cv"])
            ev_done[k].record(stream)
            s_out.wait_event(ev_done[k])
            with torch.cuda.stream(s_out):
                out_cv.copy_(outs[k % 2], non_blocking=True)
                ev_out[k].record(s_out)
        s_out.wait_event(ev_done[k_e2e - 1])
        e3.record(s_out)
        torch.cuda.synchronize()
        ms_e = e2.elapsed_time(e3)
        del stage, outs
        if dist:
            t = torch.tensor([ms_e], device=f"cuda:{local_rank}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e = float(t.item())
        e2e = {"value": world * nodes * k_e2e / (ms_e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": k_e2e, "ms_per_step": ms_e / k_e2e,
               "transfers": "pinned host state in and result out every step, on their own streams, "
                            "overlapped with the neighbouring steps' compute"}

    mixed = None
    if not args.no_mixed:
        mixed = mixed_form(args, p, dev, faces, host_state, xyz, dt, ctx, stream, nodes, world, dist, local_rank)

    ctx.close()
    del dev, xyz
    torch.cuda.empty_cache()
    reacting = None if args.no_reacting else reacting_box(args, local_rank)
    batched = None if args.no_batch else batched_blocks(args, local_rank)
    c5 = None if args.no_c5 else square_cylinder(args, local_rank)
    c5v = None
    if not args.no_c5 and args.c5_variants > 0:
        c5v = square_cylinder_variants(args, local_rank, c5 and c5.get("value"))
    served = None if args.no_serve else serve_workload(args)
    reactors = reactor_sweep(args) if args.reactor_sweep else None
    samples = accuracy_samples(args, local_rank) if (rank == 0 and not args.no_cpu_baseline) else None
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    base = None if args.no_cpu_baseline else cpu_baseline(args, samples)
    value = world * nodes * args.steps / (ms * 1e-3)
    acc = (base or {}).get("accuracy_vs_oracle", {})
    racc = (base or {}).get("reacting_accuracy_vs_oracle", {})
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"sine-wave advection, 3-D curvilinear periodic grid {args.n}^3 intervals "
                                   f"({args.n + 1}^3 nodes, 4 ghost layers), WENO7 reconstruction + AUSM+, "
                                   f"8th-order collocated viscous (mu=1e-4, Pr=0.72), SSP-RK3 fixed dt",
                       "dt": dt, "precision": "plain FP64", "per_gpu_nodes": nodes,
                       "sweep_tile_widths": tile_widths,
                       "l2": "inputs larger than L2 (about 7 GB of field arrays per GPU)",
                       "parallelism": f"{world} independent replicas" if world > 1 else "single GPU"},
            "roofline": roof, "gpu_launches": launches, "clocks": clocks, "status_flags": status,
            "e2e": None if e2e is None else {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step",
                                                                 "d2h_bytes_per_step", "steps", "ms_per_step")},
            "cpu_baseline": None if base is None else {k: base[k] for k in ("value", "unit", "cores", "kind",
                                                                            "sample")},
            # the rest of the headline metric, kept at the top level
            "mixed_value": mixed and mixed["value"], "mixed_speedup_vs_fp64": mixed and mixed["speedup_vs_fp64"],
            "mixed_l1_rho_vs_fp64": mixed and mixed["l1_rho_vs_fp64"],
            "mixed_l1_rho_vs_oracle": acc.get("l1_rho_mixed"), "mixed_linf_rho_vs_oracle": acc.get("linf_rho_mixed"),
            "fp64_l1_rho_vs_oracle": acc.get("l1_rho_fp64"),
            "serve_p50_s": served and served["latency_all"]["p50_s"],
            "serve_p99_s": served and served["latency_all"]["p99_s"],
            "serve_requests_per_s": served and served["throughput_requests_per_s"],
            "reacting_box": reacting and {"fp64_value": reacting["fp64"]["value"],
                                          "mixed_value": reacting["mixed"]["value"],
                                          "speedup_mixed_vs_fp64": reacting["speedup_mixed_vs_fp64"],
                                          "mixed_l1_rho_vs_oracle": racc.get("l1_rho_mixed"),
                                          "mixed_l1_T_vs_oracle": racc.get("l1_T_mixed"),
                                          "mixed_l1_Y_vs_oracle": racc.get("l1_Y_mixed")},
            "square_cylinder_air5": c5 and {k: c5.get(k) for k in ("value", "ms_per_step", "steps", "nodes",
                                                                     "status_flags", "error") if k in c5},
            "square_cylinder_air5_variants": c5v and {k: c5v.get(k) for k in (
                "variants", "value", "ms_per_step", "steps", "nodes", "speedup_vs_one_case", "status_flags", "error")
                if k in c5v},
            "batched_blocks": batched and {"speedup_batched": batched["speedup_batched"],
                                           "batched_value": batched["batched"]["value"]},
            "details": "second JSON object on stderr"}
    details = {"mixed": mixed, "serve": served, "reacting_box": reacting, "batched_blocks": batched,
               "square_cylinder_air5": c5, "square_cylinder_air5_variants": c5v, "cpu_baseline": base, "e2e": e2e,
               "reactor_sweep": reactors,
               "kernel_ms_per_step": {k: v[1] for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
               "kernel_rooflines": kernel_roofs}
    print(json.dumps(details, default=float), file=sys.stderr, flush=True)
    print(json.dumps(line, default=float), flush=True)


def mixed_form(args, p, dev, faces, host_state, xyz, dt, ctx64, stream, nodes, world, dist, local_rank):
    """The mixed-precision form on the same workload: FP32 reconstruction, fluxes and viscous
    stencils, FP64 state and stage update.  Both forms run `accuracy_steps` RK3 steps from the
    same initial state; the mixed run is timed with CUDA events and its density is compared with
    the FP64 run (which the parity tests tie to the FP64 oracle) and with the exact advected
    profile."""
    import torch
    import cb200
    from cb200 import abi
    sh = stream.cuda_stream
    pm = abi.ParamView.from_buffer_copy(p)
    pm.precision = abi.PREC_MIXED
    ctx32 = cb200.Context(pm)
    ctx32.bind(0, dev.view(), faces)
    tune_sweeps(ctx32, args, sh)
    dev_init = {n: torch.from_numpy(a).to(dev.t[n].device) for n, a in host_state.items()}
    g = (dev.t["bv"].shape[-1] - int(round(xyz.shape[-1]))) // 2

    def reset():
        for n, t in dev_init.items():
            dev.t[n].copy_(t)
        ctx64.properties(0, sh)

    def rho():
        return dev.t["bv"][0, g:-g, g:-g, g:-g].clone()

    def run(ctx, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0.record(stream)
        for _ in range(steps):
            ctx.rk3_step(dt, True, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device=f"cuda:{local_rank}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    S = args.accuracy_steps
    for _ in range(args.warmup):
        ctx32.rk3_step(dt, True, sh)
    reset()
    ms32 = run(ctx32, S)
    r32 = rho()
    status32 = ctx32.read_status(sh)
    ctx32.profile(True)
    ctx32.rk3_step(dt, True, sh)
    torch.cuda.synchronize()
    prof32 = ctx32.profile_read()
    ctx32.profile(False)
    reset()
    ms64 = run(ctx64, S)
    r64 = rho()
    ctx32.close()
    t_end = S * dt
    ex = 1.0 + 0.2 * torch.sin(2 * math.pi * (xyz.to(r64.device) - 3.0 * t_end))
    mean64 = r64.abs().mean()
    d = (r32 - r64).abs()
    out = {"precision": "mixed: FP32 reconstruction/AUSM+/8th-order viscous stencils, FP64 state, "
                        "temperature and stage update",
           "steps": S, "value": world * nodes * S / (ms32 * 1e-3), "ms_per_step": ms32 / S,
           "fp64_value_same_run": world * nodes * S / (ms64 * 1e-3), "fp64_ms_per_step": ms64 / S,
           "speedup_vs_fp64": ms64 / ms32,
           "l1_rho_vs_fp64": float(d.mean() / mean64), "linf_rho_vs_fp64": float(d.max() / mean64),
           "l1_rho_vs_exact_mixed": float((r32 - ex).abs().mean() / ex.abs().mean()),
           "l1_rho_vs_exact_fp64": float((r64 - ex).abs().mean() / ex.abs().mean()),
           "t_end": t_end, "status_flags": status32,
           "accuracy_bound_l1": 1e-6,
           "kernel_ms_per_step": {k: v[1] for k, v in sorted(prof32.items(), key=lambda kv: -kv[1][1])}}
    peak, _ = measured_peaks()
    n_side = round(nodes ** (1.0 / 3.0))
    out["kernel_rooflines"] = kernel_rooflines(prof32, nodes, (n_side + 8) ** 3, KERNEL_BYTES_PER_NODE_MIXED, peak)
    out["meets_accuracy_bound"] = out["l1_rho_vs_fp64"] <= 1e-6
    return out


def reacting_box(args, local_rank):
    """The reacting H2/air box (3-D periodic, --reacting-n nodes per side, L = 1 mm, random-phase
    velocity with u_rms = 10 m/s, 1200 K with five 300 K hot spots, 1 atm, stoichiometric
    premixed H2/air, 9 species / 19 reactions): WENO5 + HLLC, 2nd-order mixture-averaged
    viscous terms, finite-rate chemistry, fixed dt = 2e-9 s, in the plain and the mixed form
    (FP32 sweeps; viscous, chemistry and transport FP64).  Timed with CUDA events over
    --reacting-steps steps after 2 warm-up steps, each form from the same initial state."""
    import torch
    import cb200
    from cb200 import abi, cases
    from cb200 import mech as mechmod
    from cb200.field import DeviceBlock
    h2 = mechmod.load_json(os.path.join(REPO, "tests", "golden", "h2_li2004.json"))
    case = cases.h2_air_box(h2, n_nodes=args.reacting_n)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    dev = DeviceBlock(hb, device=f"cuda:{local_rank}")
    init = {n: dev.t[n].clone() for n in ("cv", "bv", "sv")}
    del case, hb
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    nodes = args.reacting_n ** 3
    dt = 2e-9
    out = {"workload": f"reacting H2/air box {args.reacting_n}^3 nodes, WENO5 + HLLC, 2nd-order viscous, "
                       f"finite-rate chemistry (9 species, 19 reactions), fixed dt 2e-9 s",
           "steps": args.reacting_steps}
    for name, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        pv = abi.ParamView.from_buffer_copy(p)
        pv.precision = prec
        for n, t in init.items():
            dev.t[n].copy_(t)
        ctx = cb200.Context(pv)
        ctx.bind(0, dev.view(), faces)
        ctx.properties(0, sh)
        for _ in range(2):
            ctx.rk3_step(dt, True, sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.reacting_steps):
            ctx.rk3_step(dt, True, sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.reacting_steps
        ctx.profile(True)
        ctx.rk3_step(dt, True, sh)
        torch.cuda.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
        status = ctx.read_status(sh)
        ctx.close()
        top = sorted(prof.items(), key=lambda kv: -kv[1][1])[:8]
        out[name] = {"value": nodes / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "status_flags": status,
                     "kernel_ms_per_step": {k: v[1] for k, v in top}}
    out["speedup_mixed_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    del dev, init
    torch.cuda.empty_cache()
    return out


def square_cylinder(args, local_rank):
    """The two-temperature AIR5 Mach-10 square cylinder: four body-fitted blocks of
    --c5-side x --c5-normal nodes (1024 x 512 in all by default; tanh wall clustering, first cell
    1e-6 m; cb200.grid), freestream T = T_ve = 250 K, p = 500 Pa, Y_N2 = 0.767, Y_O2 = 0.233 on
    the box except its downstream side (outflow), isothermal 300 K wall; characteristic WENO5 with
    the rho e_ve row, positivity limiter, 2nd-order viscous terms with the e_ve conduction, Park's
    17 reactions with the AIR5 control temperatures and the e_ve source, VT relaxation, NASA9,
    limit_flow; FP64, CFL 0.3.  The inner faces are exchanged on the device after every stage
    (cb2_halo).  --c5-steps steps run inside one device-driven graph launch (cb2_rk3_run, CFL dt
    computed on the device every step), timed with CUDA events after --c5-warmup warm-up steps of
    the impulsive start."""
    import torch
    import cb200
    from cb200 import cases
    from cb200 import mech as mechmod
    from cb200.field import DeviceBlock
    gold = os.path.join(REPO, "tests", "golden", "air5_park.json")
    air5 = mechmod.load_json(gold)
    tt = mechmod.load_two_temperature_json(gold)
    case = cases.square_cylinder_air5(air5, tt, n_side=args.c5_side, n_normal=args.c5_normal)
    p = case.param
    p.positive_preserving = 1
    p.limit_flow = 1
    devs = [DeviceBlock(hb, device=f"cuda:{local_rank}") for hb in case.blocks]
    nodes = sum(hb.mx * hb.my * hb.mz for hb in case.blocks)
    ctx = cb200.Context(p)
    nb = len(devs)
    for b in range(nb):
        ctx.bind(b, devs[b].view(), case.faces[b])
        ctx.bind_inner_faces(b, case.meta["inner"][b])
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    # the reference's initialisation: properties, faces, inner faces, properties, cv from bv
    for b in range(nb):
        ctx.properties(b, sh)
    for b in range(nb):
        ctx.boundary(b, sh)
    ctx.halo(sh)
    for b in range(nb):
        ctx.properties(b, sh)
    for b in range(nb):
        ctx.cv_from_bv(b, sh)
    t = 0.0
    out = {"workload": f"two-temperature AIR5 Mach-10 square cylinder, 4 body-fitted blocks of "
                       f"{args.c5_side} x {args.c5_normal} nodes ({nodes} nodes), first cell 1e-6 m, WENO5-ch + "
                       f"positivity limiter, 2nd-order viscous, Park chemistry, VT relaxation, limit_flow, "
                       f"CFL 0.3, FP64", "nodes": nodes}
    try:
        t, n_w, _ = ctx.rk3_run(args.c5_warmup, time=t, fixed_dt=False, stream=sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t1, n_s, dt_last = ctx.rk3_run(args.c5_steps, time=t, fixed_dt=False, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(n_s, 1)
        ctx.profile(True)
        ctx.rk3_step(dt_last, True, sh)
        torch.cuda.synchronize()
        prof = ctx.profile_read()
        ctx.profile(False)
        out.update({"steps": n_s, "warmup": n_w, "value": nodes / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                    "dt_last": dt_last, "physical_time": t1, "status_flags": ctx.read_status(sh),
                    "kernel_ms_per_step": {k: v[1] for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:10]}})
    except cb200.CB2Error as e:
        out["error"] = str(e)
    ctx.close()
    del devs
    torch.cuda.empty_cache()
    return out


def square_cylinder_variants(args, local_rank, one_case_value=None):
    """The AIR5 cylinder's freestream-Mach variants batched in one context: --c5-variants copies of
    the four-block grid (64 blocks for 16 variants), Mach linspace(6, 14), each with its own inflow
    faces and inner faces, advanced together inside one device-driven graph launch per call
    (cb2_rk3_run), the blocks' work of every stage on concurrent branch streams.  All variants
    take the common CFL step (the minimum over the 64 blocks, set by the fastest freestream).
    Every variant starts from the Mach-10 impulsive start with its velocity scaled to its Mach
    number.  Timed with CUDA events after --c5-warmup steps."""
    import numpy as np
    import torch
    import cb200
    from cb200 import abi, cases
    from cb200 import mech as mechmod
    from cb200.field import DeviceBlock
    gold = os.path.join(REPO, "tests", "golden", "air5_park.json")
    air5 = mechmod.load_json(gold)
    tt = mechmod.load_two_temperature_json(gold)
    base = cases.square_cylinder_air5(air5, tt, n_side=args.c5_side, n_normal=args.c5_normal)
    p = base.param
    p.positive_preserving = 1
    p.limit_flow = 1
    fs = base.meta["freestream"]
    machs = np.linspace(6.0, 14.0, args.c5_variants)
    ctx = cb200.Context(p)
    devs = []
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    out = {"variants": len(machs), "machs": [float(m) for m in machs]}
    try:
        for v, mach in enumerate(machs):
            for b in range(4):
                dev = DeviceBlock(base.blocks[b], device=f"cuda:{local_rank}")
                dev.t["bv"][1] *= mach / 10.0
                devs.append(dev)
                fl = []
                for f in base.faces[b]:
                    f2 = abi.FaceBC.from_buffer_copy(f)
                    if f2.type == abi.BC_INFLOW:
                        f2.u = mach * fs["c"]
                    fl.append(f2)
                ctx.bind(4 * v + b, dev.view(), fl)
        for v in range(len(machs)):
            for b in range(4):
                inner = []
                for f in base.meta["inner"][b]:
                    f2 = abi.InnerFace.from_buffer_copy(f)
                    f2.target_block += 4 * v
                    inner.append(f2)
                ctx.bind_inner_faces(4 * v + b, inner)
        nb = 4 * len(machs)
        for fn in (ctx.properties, ctx.boundary):
            for b in range(nb):
                fn(b, sh)
        ctx.halo(sh)
        for fn in (ctx.properties, ctx.cv_from_bv):
            for b in range(nb):
                fn(b, sh)
        t, n_w, _ = ctx.rk3_run(args.c5_warmup, fixed_dt=False, stream=sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t1, n_s, dt_last = ctx.rk3_run(args.c5_variant_steps, time=t, fixed_dt=False, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(n_s, 1)
        nodes = nb * args.c5_side * args.c5_normal
        out.update({"blocks": nb, "nodes": nodes, "steps": n_s, "warmup": n_w, "ms_per_step": ms,
                    "value": nodes / (ms * 1e-3), "unit": UNIT, "dt_last": dt_last,
                    "status_flags": ctx.read_status(sh)})
        if one_case_value:
            out["speedup_vs_one_case"] = out["value"] / one_case_value
    except cb200.CB2Error as e:
        out["error"] = str(e)
    ctx.close()
    del devs
    torch.cuda.empty_cache()
    return out


def batched_blocks(args, local_rank):
    """Batched form: --batch-blocks closed periodic sine-wave blocks (WENO7 + AUSM+, inviscid,
    FP64) of seeded uneven sizes n^3 nodes, n ~ U{12..40}, advanced --batch-steps CFL steps
    (a) in one persistent launch (cb2_block_batch_advance, tile width and cluster size tuned first) and (b) one
    block after another through cb2_rk3_step, each from the same initial states.  Wall clock
    around each form (the batch call synchronises; the loop ends with a synchronise)."""
    import numpy as np
    import torch
    import cb200
    from cb200 import abi, cases
    from cb200.field import DeviceBlock
    rng = np.random.default_rng(2027)
    sizes = rng.integers(12, 41, args.batch_blocks)
    blocks = []
    for n in sizes:
        c = cases.sine_wave(n=int(n) - 1, viscous_order=0)
        blocks.append((c.param, c.blocks[0], c.faces[0]))
    p0 = blocks[0][0]
    nodes = int(sum(int(n) ** 3 for n in sizes))
    S = args.batch_steps
    out = {"workload": f"{args.batch_blocks} periodic sine-wave blocks of n^3 nodes, n ~ U{{12..40}} (seeded), "
                       f"WENO7 + AUSM+, inviscid, CFL 0.5 steps, FP64", "blocks": args.batch_blocks,
           "nodes": nodes, "steps": S}
    # (a) one persistent launch
    devs = [DeviceBlock(hb, device=f"cuda:{local_rank}") for _, hb, _ in blocks]
    ctx = cb200.Context(p0)
    cs = (abi.BlockCase * len(blocks))()
    for c, d in zip(cs, devs):
        c.zone = d.view()
        c.time, c.t_end, c.dt = 0.0, 1e30, 0.0
    if args.schedule:
        fixed = [int(v) for v in args.schedule.split(",")]
        ni, cl = fixed[0], fixed[1] if len(fixed) > 1 else 8
        ctx.block_batch_set_schedule(ni, cl)
    else:
        ni, cl = ctx.block_batch_autotune(cs)
    out["schedule"] = {"tile_width": ni, "cluster_ctas": cl}
    for d, (_, hb, _) in zip(devs, blocks):
        d.load(hb, ["cv", "bv"])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.block_batch_advance(cs, S)
    t_batch = time.perf_counter() - t0
    failed = sum(1 for c in cs if c.status & abi.BLOCK_FAILED)
    ctx.close()
    # (b) the same blocks one by one through the block path
    for d, (_, hb, _) in zip(devs, blocks):
        d.load(hb, ["cv", "bv"])
    ctxs = []
    for (p, _, faces), d in zip(blocks, devs):
        cx = cb200.Context(p)
        cx.bind(0, d.view(), faces)
        ctxs.append(cx)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for cx in ctxs:
        for _ in range(S):
            cx.rk3_step(0.0, fixed_dt=False)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    for cx in ctxs:
        cx.close()
    out["batched"] = {"value": nodes * S / t_batch, "unit": UNIT, "seconds": t_batch, "failed_blocks": failed}
    out["one_by_one"] = {"value": nodes * S / t_seq, "unit": UNIT, "seconds": t_seq}
    out["speedup_batched"] = t_seq / t_batch
    del devs
    torch.cuda.empty_cache()
    return out


def reactor_sweep(args):
    """us per ROK4E attempt of the batched 0-D H2/air reactors (one warp each) at batch sizes from a
    few warps to past the GPU's concurrency: latency where the batch is small, throughput where it
    saturates.  The reactors start from the reference's reactor runs (tests/golden) with their end
    times moved out of reach, so every reactor takes every attempt."""
    import ctypes as C
    import torch
    import cb200
    from cb200 import abi, cases, mech as mechmod
    runs = json.load(open(os.path.join(REPO, "tests", "golden", "h2_reactor_runs.json")))
    h2 = mechmod.load_json(os.path.join(REPO, "tests", "golden", "h2_li2004.json"))
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, dim=1, inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5, mech=h2.ptr())
    ctx = cb200.Context(p)
    out = {}
    attempts = 200
    for n in (32, 592, 4096, 16384):
        rr = [runs["runs"][i % len(runs["runs"])] for i in range(n)]
        dev = lambda a: torch.tensor(a, dtype=torch.float64, device="cuda")
        T0, p0 = dev([r["T0"] for r in rr]), dev([r["p0"] for r in rr])
        Y, t_end = dev([r["Y"] for r in rr]), dev([r["t_end"] * 1e3 for r in rr])
        st = torch.zeros(n * C.sizeof(abi.Reactor), dtype=torch.uint8, device="cuda")
        ctx.reactor_setup(st.data_ptr(), n, T0.data_ptr(), p0.data_ptr(), Y.data_ptr(), t_end.data_ptr(), runs["h0"])
        ctx.reactor_advance(st.data_ptr(), n, 20, runs["rtol"], runs["atol"])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.reactor_advance(st.data_ptr(), n, attempts, runs["rtol"], runs["atol"])
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[str(n)] = {"us_per_attempt": ms * 1e3 / attempts, "attempts_per_s": n * attempts / (ms * 1e-3)}
    ctx.close()
    return out


def serve_workload(args):
    """The served workload: seeded Poisson arrivals (mean --serve-rate per second over
    --serve-seconds) of 0-D H2/air reactors (T0 ~ U[1000, 1500] K, p0 ~ U[1, 10] atm,
    phi ~ U[0.5, 2], to 1 ms, ROK4E with RTol 1e-6, ATol 1e-12) and 1-D reactive shock tubes
    (N ~ U{200..4000} nodes over 0.1 m, (1500 K, 5 atm) | (300 K, 1 atm) stoichiometric H2/air,
    WENO5 + HLLC with chemistry, CFL 0.5, to 50 us), half each, served by cb2_serve_run on this
    GPU.  Latency = completion - arrival on the host clock."""
    import cb200
    from cb200 import abi, cases, serve
    from cb200 import mech as mechmod
    h2 = mechmod.load_json(os.path.join(REPO, "tests", "golden", "h2_li2004.json"))
    p = cases.make_param(n_var=5 + h2.ns, n_spec=h2.ns, dim=2, inviscid_scheme=abi.INV_HLLC,
                         reconstruction=abi.REC_WENO5, cfl=0.5, mech=h2.ptr())
    p.reaction = 1
    ctx = cb200.Context(p)
    reqs = serve.request_stream(h2, rate=args.serve_rate, duration=args.serve_seconds, seed=2026,
                                t_reactor=args.serve_reactor_t_end, t_tube=args.serve_tube_t_end)
    opt = serve.options(h2, hbm_budget=16 << 30, max_tubes=296, max_reactors=4096, tube_steps=20,
                        reactor_attempts=500, time_limit=900.0)
    res, st = serve.serve(ctx, ctx, reqs, opt)
    ctx.close()
    kinds = {"reactor": [r for q, r in zip(reqs, res) if q.kind == abi.REQ_REACTOR],
             "shock_tube": [r for q, r in zip(reqs, res) if q.kind == abi.REQ_TUBE]}
    tube_cu = sum(q.n_nodes * r.steps for q, r in zip(reqs, res) if q.kind == abi.REQ_TUBE)
    out = {"workload": f"seeded Poisson arrivals of 0-D H2/air reactors (to {args.serve_reactor_t_end:g} s) and "
                       f"1-D reactive shock tubes (200..4000 nodes, to {args.serve_tube_t_end:g} s; the served "
                       f"workload's tubes run to 5e-05 s), half each",
           "tube_time_step": "CFL 0.5 with the reference's reaction-time-scale limit (local_time_step)",
           "arrival_rate_per_s": args.serve_rate, "arrival_window_s": args.serve_seconds, "requests": len(reqs),
           "wall_s": st.wall_s, "throughput_requests_per_s": len(reqs) / st.wall_s,
           "tube_cell_updates_per_s": tube_cu / st.wall_s, "batched_iterations": st.iterations,
           "peak_pool_bytes": st.peak_pool_bytes,
           "failed": int(sum(1 for q, r in zip(reqs, res) if (q.kind == abi.REQ_TUBE and r.status & 2)
                             or (q.kind == abi.REQ_REACTOR and r.status & abi.REACTOR_NONPHYSICAL)))}
    for k, v in kinds.items():
        if v:
            out[f"latency_{k}"] = serve.latency_summary(v)
    out["latency_all"] = serve.latency_summary(res)
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()

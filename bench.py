#!/usr/bin/env python
"""Throughput of the spherical-transform cycle on B200.

One step = one full cycle (backward Legendre -> phi-FFT -> grid products ->
phi-FFT -> forward Legendre) of one transform instance at L=511, Nr=257,
Ntheta=768, Nphi=1536 with {u, omega, B} + {T} backward and
{omega x u, u x B, u T} + {u . omega} forward (synthetic seeded spectra).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--tier split|fp64|fp32acc]

Multi-GPU (torchrun, one rank per GPU): the cycle shards by radius with no
collective inside the path; each rank runs its own full instance (weak scaling),
value = all ranks' cycles / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "transform cycles/s at L=511 Nr=257: TC split-precision vs FP64 GPU, err≤1e-12"
UNIT = "cycles/s"
TIERS = {"fp64": 0, "split": 1, "fp32acc": 2}
DTYPES = {"fp64": "f64", "split": "s8 slices (int32 accumulate) + f64 recombination",
          "fp32acc": "s8 slices (int32 accumulate) + f64 recombination"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_slab_radii(cfg, threads: int) -> int:
    """Radii of the CPU sample: at least two per host thread (the oracle runs
    OpenMP over radial blocks, as the reference's flag-11 path does) and at
    least 16, never more than the shell."""
    return int(min(cfg.nr, max(16, 2 * threads)))


def cpu_cycle_rate(cfg, steps: int = 1, warmup: int = 1, budget_s: float = 150.0):
    """Times the CPU FP64 oracle (reference sym_dgemm path restated, OpenBLAS
    DGEMM, OpenMP over radial blocks on all host threads) on a radial slab of
    cpu_slab_radii radii spread over the shell.  Every stage is linear in Nr,
    so cycles/s of the full shell = slab cycles/s x nr_slab / Nr.  Up to
    `steps` cycles are timed, fewer when they would overrun `budget_s` (the
    slab size is kept, the repeat count shrinks).  Returns (cycles/s of the
    full shell, slab radii, threads, stage times of the last cycle, cycles
    timed)."""
    import numpy as np
    from oracle import oracle as om
    from kemorin_mhd_b200.config import SphConfig
    from kemorin_mhd_b200.synthetic import make_d_rj
    om.use_openblas()
    threads = os.cpu_count() or 1
    nr = cpu_slab_radii(cfg, threads)
    idx = np.linspace(0, cfg.nr - 1, nr).round().astype(int)
    c = SphConfig(cfg.ltr, cfg.nth, cfg.nph, nr, cfg.nvb, cfg.nsb, cfg.nvf, cfg.nsf, cfg.products)
    o = om.Oracle(c, nthreads=threads, radius=cfg.radius()[idx])
    d = make_d_rj(c)
    t_start = time.perf_counter()
    for _ in range(max(0, warmup)):
        o.cycle(d)
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        o.cycle(d)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start + times[-1] > budget_s:
            break
    t = statistics.median(times)
    rate = 1.0 / (t * cfg.nr / nr)
    return rate, nr, threads, o.last_timing(), len(times)


def bench_config(cfg, fields_bwd, fields_fwd, ws):
    """The `config` object of both arms' JSON lines."""
    return {"workload": cfg.name, "L": cfg.ltr, "Nr": cfg.nr, "Ntheta": cfg.nth, "Nphi": cfg.nph,
            "fields_bwd": fields_bwd, "fields_fwd": fields_fwd,
            "parallelism": f"radial-instance x{ws} (no collective)",
            "l2": "inputs larger than L2 (d_rj 5.4 GB, rtm 16 GB per direction)"}


def cpu_sample_text(nr, cfg, timed):
    return (f"radial slab of {nr}/{cfg.nr} radii spread over the shell, {timed} cycle(s) timed (median), "
            f"scaled x{cfg.nr / nr:.2f} to the full shell (every stage is linear in Nr)")


def run_reference(args, cfg):
    from kemorin_mhd_b200.config import FIELD_NAMES
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    rate, nr, threads, stages, timed = cpu_cycle_rate(cfg, steps=args.steps, warmup=min(args.warmup, 1))
    fb, ff = FIELD_NAMES[args.fields]
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded spectra N(0,1)(l+1)^-2 sin(pi(r-ri)/(ro-ri)), Chebyshev radii)",
        "config": bench_config(cfg, fb, ff, ws),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": cpu_sample_text(nr, cfg, timed), "slab_radii": nr,
                         "extrapolation_factor": cfg.nr / nr, "cycles_timed": timed,
                         "stages_ms": stages},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_slabs(args, cfg, fields_bwd, fields_fwd):
    """One instance spread over the N ranks by radius (kemorin_mhd_b200/slabs.py):
    rank i holds its owned radii plus one halo radius on each side; every step
    first refreshes the input halo from the neighbouring ranks (NCCL send/recv,
    one radius row per backward column and neighbour) and then runs its local
    cycle.  Strong scaling: `value` is the whole shell's cycles/s (one cycle of
    the instance per step, time = max over ranks).  With --check every rank
    also runs the whole shell on its GPU once (untimed) and compares its owned
    radii bit for bit."""
    import datetime
    import torch
    from kemorin_mhd_b200.slabs import SlabTransform, exchange_halo, radial_slab
    from kemorin_mhd_b200.synthetic import make_d_rj_torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    tier = "split" if args.tier == "auto" else args.tier
    slab = radial_slab(cfg.nr, ws, rank)
    J = cfg.J
    st = SlabTransform(cfg, slab, tier=TIERS[tier])
    stream = torch.cuda.current_stream()
    st.tr.set_stream(stream.cuda_stream)
    full = make_d_rj_torch(cfg, seed=1234)
    d_in = full[:, slab.lo * J:slab.hi * J].contiguous()
    d_out = torch.zeros((cfg.ncf, J * slab.nr_local), dtype=torch.float64, device="cuda")
    cols = list(range(cfg.ncb))

    def step():
        if dist is not None:
            exchange_halo(slab, J, d_in, cols)
        st.tr.nonlinear_cycle(d_in, d_out)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_step = float(ms.item()) / args.steps
    check = None
    if args.check:
        st_out = d_out[:, slab.owned_rows(J)].clone()
        st.close()
        from kemorin_mhd_b200 import sph_trans
        whole = sph_trans.SphTransform(cfg, tier=TIERS[tier], device=local)
        w_out = torch.zeros((cfg.ncf, J * cfg.nr), dtype=torch.float64, device="cuda")
        whole.nonlinear_cycle(full, w_out)
        torch.cuda.synchronize()
        same = torch.tensor([1.0 if torch.equal(st_out, w_out[:, slab.r0 * J:slab.r1 * J]) else 0.0],
                            dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(same, op=dist.ReduceOp.MIN)
        check = bool(same.item() == 1.0)
        whole.close()
    else:
        st.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": 1e3 / ms_step, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": DTYPES[tier], "tier": tier,
            "data": "synthetic (seeded spectra N(0,1)(l+1)^-2 sin(pi(r-ri)/(ro-ri)), Chebyshev radii)",
            "config": dict(bench_config(cfg, fields_bwd, fields_fwd, ws),
                           parallelism=f"radial slabs x{ws} (one instance; NCCL halo send/recv of one "
                                       "radius per backward column and neighbour each step)"),
            "slab_radii_rank0": [slab.r0, slab.r1], "bit_exact_vs_whole_shell": check,
            "gpu_launches": {"fp64": 4, "split": 6, "fp32acc": 6}[tier] * args.steps,
            "clocks": clk, "cpu_baseline": None,
            "e2e": None,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg3")
    ap.add_argument("--tier", default="auto", choices=["auto"] + list(TIERS))
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-tier comparison run")
    ap.add_argument("--no-tiers", action="store_true", help="split tier: skip the fp32acc comparison run")
    ap.add_argument("--nr", type=int, default=0, help="override the radius count (small profiling cases)")
    ap.add_argument("--fields", default="default", choices=["default", "dynamo", "full"],
                    help="field set: default u,omega,B + T; dynamo u,omega,B,J + T with the Lorentz force; "
                         "full u,omega,B,J + T,C with the Lorentz force and the composition flux")
    ap.add_argument("--slabs", action="store_true",
                    help="one instance over the N ranks by radius (strong scaling) instead of one instance per rank")
    ap.add_argument("--check", action="store_true", help="--slabs: compare every rank's radii with the whole shell")
    ap.add_argument("--p-on-the-fly", action="store_true",
                    help="FP64 tier: P_l^m generated inside the Legendre kernels (no stored tables); "
                         "also times the stored-table FP64 tier on the same input")
    args = ap.parse_args()

    if args.config == "cfg4":
        return run_batch(args)
    from kemorin_mhd_b200.config import NAMED, SphConfig
    cfg = NAMED[args.config]
    if args.nr > 0:
        cfg = SphConfig(cfg.ltr, cfg.nth, cfg.nph, args.nr, cfg.nvb, cfg.nsb, cfg.nvf, cfg.nsf, cfg.products,
                        name=f"L{cfg.ltr}_Nr{args.nr}")
    from kemorin_mhd_b200.config import FIELD_NAMES, with_fields
    cfg = with_fields(cfg, args.fields)
    fields_bwd, fields_fwd = FIELD_NAMES[args.fields]
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.slabs:
        return run_slabs(args, cfg, fields_bwd, fields_fwd)

    import numpy as np
    import torch
    from kemorin_mhd_b200 import sph_trans
    from kemorin_mhd_b200.synthetic import make_d_rj_torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    tier = args.tier
    if tier == "auto":
        tier = "split"
    lib = sph_trans.load_library()

    if args.p_on_the_fly and args.tier != "fp64":
        raise SystemExit("--p-on-the-fly needs --tier fp64")

    def make(tier_name, otf=False):
        return sph_trans.SphTransform(cfg, tier=TIERS[tier_name], device=local, p_on_the_fly=otf)

    try:
        tr = make(tier, otf=args.p_on_the_fly)
    except sph_trans.KmhdError:
        if args.tier != "auto":
            raise
        tier = "fp64"
        tr = make(tier)
    stream = torch.cuda.current_stream()
    tr.set_stream(stream.cuda_stream)
    d_in = make_d_rj_torch(cfg, seed=1234 + rank)
    d_out = torch.zeros((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, device="cuda")

    for _ in range(args.warmup):
        tr.nonlinear_cycle(d_in, d_out)
    torch.cuda.synchronize()

    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stage = {"leg_bwd": 0.0, "fft_nl": 0.0, "leg_fwd": 0.0}
    kern = {"slice_bwd": 0.0, "gemm_bwd": 0.0, "fft_nl": 0.0, "slice_fwd": 0.0, "gemm_fwd": 0.0}
    e0.record(stream)
    for _ in range(args.steps):
        tr.nonlinear_cycle(d_in, d_out)
        t = tr.last_timing()
        for k in stage:
            stage[k] += t[k]
        t = tr.kernel_timing()
        for k in kern:
            kern[k] += t[k]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms_total = max_over_ranks(e0.elapsed_time(e1))
    ms_step = ms_total / args.steps
    value = ws * args.steps / (ms_total * 1e-3)
    for k in stage:
        stage[k] /= args.steps
    for k in kern:
        kern[k] /= args.steps

    # FP64 GPU cycle on the same input: the bar of the split tier (speed and error)
    extra = {}
    if tier != "fp64" and not args.no_fp64:
        ref64 = make("fp64")
        ref64.set_stream(stream.cuda_stream)
        out64 = torch.zeros_like(d_out)
        for _ in range(2):
            ref64.nonlinear_cycle(d_in, out64)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        n64 = max(2, args.steps // 2)
        f0.record(stream)
        for _ in range(n64):
            ref64.nonlinear_cycle(d_in, out64)
        f1.record(stream)
        torch.cuda.synchronize()
        ms64 = max_over_ranks(f0.elapsed_time(f1) / n64)
        k64 = ref64.kernel_timing()
        den = out64.abs().amax(dim=1)
        err = ((d_out - out64).abs().amax(dim=1) / den).tolist()
        extra = {"fp64_gpu": {"value": ws * 1e3 / ms64, "unit": UNIT, "ms_per_step": ms64, "kernels_ms": k64,
                              "roofline": fp64_rooflines(cfg, k64, ctypes_probe(lib, local))},
                 "speedup_vs_fp64_gpu": ms64 / ms_step,
                 "rel_err_vs_fp64_per_field": err, "rel_err_max": max(err)}
        # release the FP64 handle (about 50 GB at L=511, Nr=257) before the next
        # tier's handle is made; its output stays for the error fields
        ref64.close()
        del ref64
        torch.cuda.synchronize()
        if tier == "split" and not args.no_tiers:
            # the third tier on the same input: fp32acc (4 slices, 10 products, bound 1e-6)
            t32 = make("fp32acc")
            t32.set_stream(stream.cuda_stream)
            out32 = torch.zeros_like(d_out)
            for _ in range(2):
                t32.nonlinear_cycle(d_in, out32)
            torch.cuda.synchronize()
            f0.record(stream)
            for _ in range(n64):
                t32.nonlinear_cycle(d_in, out32)
            f1.record(stream)
            torch.cuda.synchronize()
            ms32 = max_over_ranks(f0.elapsed_time(f1) / n64)
            err32 = ((out32 - out64).abs().amax(dim=1) / den).tolist()
            extra["fp32acc_gpu"] = {"value": ws * 1e3 / ms32, "unit": UNIT, "ms_per_step": ms32,
                                    "kernels_ms": t32.kernel_timing(), "speedup_vs_fp64_gpu": ms64 / ms32,
                                    "rel_err_vs_fp64_per_field": err32, "rel_err_max": max(err32)}
            t32.close()
            del out32
        del out64
    if args.p_on_the_fly:
        # the stored-table FP64 tier on the same input (one handle at a time:
        # at L=1023 each holds ~80 GB)
        tr_bytes = tr.device_bytes()
        tr.close()
        torch.cuda.synchronize()
        st = make("fp64")
        st.set_stream(stream.cuda_stream)
        out_st = torch.zeros_like(d_out)
        for _ in range(2):
            st.nonlinear_cycle(d_in, out_st)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        nst = max(2, args.steps // 2)
        f0.record(stream)
        for _ in range(nst):
            st.nonlinear_cycle(d_in, out_st)
        f1.record(stream)
        torch.cuda.synchronize()
        ms_st = max_over_ranks(f0.elapsed_time(f1) / nst)
        den = out_st.abs().amax(dim=1)
        err = ((d_out - out_st).abs().amax(dim=1) / den).tolist()
        extra = {"p_tables": "generated in the Legendre kernels (KMHD_FLAG_P_ON_THE_FLY)",
                 "device_bytes": tr_bytes,
                 "fp64_stored_tables": {"value": ws * 1e3 / ms_st, "unit": UNIT, "ms_per_step": ms_st,
                                        "device_bytes": st.device_bytes(), "kernels_ms": st.kernel_timing()},
                 "speed_vs_stored_tables": ms_st / ms_step,
                 "rel_err_vs_stored_per_field": err, "rel_err_vs_stored_max": max(err)}
        tr = st
        del out_st

    # roofline of the dominant kernel: the Legendre GEMM (split tiers: the one
    # tcgen05 kernel, launched once per direction; FP64: the slower of the two
    # DMMA kernels).  Durations are CUDA events on the launching stream.
    peaks, psrc = load_peaks()
    flops = 2.0 * cfg.nh * cfg.J * cfg.nr * (5 * cfg.nvb + cfg.nsb)  # per direction (bwd = fwd here)
    if tier == "fp64":
        which = "gemm_fwd" if kern["gemm_fwd"] >= kern["gemm_bwd"] else "gemm_bwd"
        dur = kern[which]
        pk = ctypes_probe(lib, local)
        roof = {"bound": "tensor", "achieved": flops / (dur * 1e-3) / 1e12, "peak": pk, "unit": "TFLOP/s",
                "peak_source": "FP64 tensor pipe measured in-process (DMMA chain probe); "
                               "MEASURED_PEAKS.json carries no FP64 figure",
                "kernel": "k_leg_fwd_f64" if which == "gemm_fwd" else "k_leg_bwd_f64"}
    else:
        dur = 0.5 * (kern["gemm_bwd"] + kern["gemm_fwd"])
        pk = 2.0 * peaks["bf16_tflops"]
        execd = split_executed_ops(cfg, 26 if tier == "split" else 10)
        roof = {"bound": "tensor", "achieved": flops / (dur * 1e-3) / 1e12, "peak": pk, "unit": "TFLOP/s",
                "peak_source": f"INT8 dense = 2 x bf16 burst of {psrc} MEASURED_PEAKS.json",
                "kernel": "k_split_gemm",
                "achieved_is": "useful FP64-equivalent flop/s (2*Nh*J*Nr*(5nv+ns) per launch)",
                "executed_int8_tops": execd / (dur * 1e-3) / 1e12,
                "executed_frac": execd / (dur * 1e-3) / 1e12 / pk,
                "overhead_factor": execd / flops,
                "executed_note": "counts every K chunk; the forward launch skips chunks whose data digits "
                                 "are all zero (about 19% of them at L=511), so the executed figures are "
                                 "upper bounds"}
    roof["frac"] = roof["achieved"] / roof["peak"] if roof["peak"] else None
    roof["traffic"] = read_traffic(roof["kernel"], cfg.name)
    roof["algorithmic_flops_per_launch"] = flops
    roof["ms_per_launch"] = dur

    # the largest single launch of the cycle: the fused FFT + products kernel,
    # bounded by HBM (it reads the backward rtm records and writes the forward
    # ones once: Nr*Ntheta*(L+1)*2*(ncb+ncf) doubles per launch)
    fft_bytes = 8.0 * cfg.nr * cfg.nth * (cfg.ltr + 1) * 2 * (cfg.ncb + cfg.ncf)
    dur_fft = kern["fft_nl"]
    roof_fft = {"bound": "hbm", "kernel": "k_fft_cycle_f", "unit": "GB/s",
                "achieved": fft_bytes / (dur_fft * 1e-3) / 1e9 if dur_fft > 0 else None,
                "peak": peaks["hbm_gbs"], "peak_source": f"hbm_gbs of {psrc} MEASURED_PEAKS.json",
                "algorithmic_bytes_per_launch": fft_bytes, "ms_per_launch": dur_fft,
                "traffic": read_traffic("k_fft_cycle_f", cfg.name)}
    roof_fft["frac"] = roof_fft["achieved"] / roof_fft["peak"] if roof_fft["achieved"] else None

    # end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e and not args.p_on_the_fly:  # (the on-the-fly handle is closed by now)
        h_in = torch.empty((cfg.ncb, cfg.J * cfg.nr), dtype=torch.float64, pin_memory=True)
        h_in.copy_(d_in)
        h_out = torch.empty((cfg.ncf, cfg.J * cfg.nr), dtype=torch.float64, pin_memory=True)
        tr.nonlinear_cycle(h_in, h_out)
        ke = max(2, min(args.steps, 4))
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            tr.nonlinear_cycle(h_in, h_out)
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": ws * ke / dt, "unit": UNIT, "h2d_bytes_per_step": h_in.numel() * 8,
               "d2h_bytes_per_step": h_out.numel() * 8, "steps": ke,
               "note": "host wall clock around kmhd_sph_cycle with pinned host d_rj in/out"}
        del h_in, h_out

    cpu = None
    if rank == 0 and not args.no_cpu:
        rate, nr, threads, stages, timed = cpu_cycle_rate(cfg, steps=1, warmup=1)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": cpu_sample_text(nr, cfg, timed), "slab_radii": nr,
               "extrapolation_factor": cfg.nr / nr, "stages_ms": stages}

    launches = {"fp64": 4, "split": 6, "fp32acc": 6}[tier]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPES[tier], "tier": tier,
        "data": "synthetic (seeded spectra N(0,1)(l+1)^-2 sin(pi(r-ri)/(ro-ri)), Chebyshev radii)",
        "config": bench_config(cfg, fields_bwd, fields_fwd, ws),
        "stages_ms": stage, "kernels_ms": kern, "roofline": roof, "roofline_fft": roof_fft,
        "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": launches * args.steps, "clocks": clk,
    }
    line.update(extra)
    if rank == 0:
        print(json.dumps(line), flush=True)
    tr.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """cfg4: 64 uneven instances.  Baseline: the 64 plain FP64 cycles run one
    after the other (each a synchronous call); then the split tier with the
    path autotuner as one batched call (captured CUDA graph, every instance on
    its own stream).  Host wall clock around whole synchronous calls."""
    import torch
    from kemorin_mhd_b200 import sph_trans
    from kemorin_mhd_b200.config import batch_configs
    from kemorin_mhd_b200.synthetic import make_d_rj_torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    cfgs = batch_configs()
    n = len(cfgs)
    d_in = [make_d_rj_torch(c, seed=500 + i) for i, c in enumerate(cfgs)]

    def outs():
        return [torch.zeros((c.ncf, c.J * c.nr), dtype=torch.float64, device="cuda") for c in cfgs]

    # baseline: sequential plain FP64 cycles
    trs = [sph_trans.SphTransform(c, tier=0, device=local) for c in cfgs]
    o64 = outs()
    for _ in range(max(1, args.warmup)):
        for tr, d, o in zip(trs, d_in, o64):
            tr.nonlinear_cycle(d, o)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for tr, d, o in zip(trs, d_in, o64):
            tr.nonlinear_cycle(d, o)
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    for tr in trs:
        tr.close()
    del trs
    torch.cuda.empty_cache()
    # batched split tier with the path autotuner
    trs = [sph_trans.SphTransform(c, tier=TIERS["split"], device=local, autotune=True) for c in cfgs]
    ob = outs()
    for _ in range(max(1, args.warmup)):
        sph_trans.batch_cycle(trs, d_in, ob)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sph_trans.batch_cycle(trs, d_in, ob)
    torch.cuda.synchronize()
    t_b = time.perf_counter() - t0
    clk = clocks.stop()
    err = max(float(((a - b).abs().amax(dim=1) / b.abs().amax(dim=1)).max()) for a, b in zip(ob, o64))
    nsplit = sum(1 for tr in trs if tr.uses_split())
    value = n * args.steps / t_b
    for tr in trs:
        tr.close()
    # every instance on the split path: their GEMMs run as one grouped launch per direction
    trs = [sph_trans.SphTransform(c, tier=TIERS["split"], device=local) for c in cfgs]
    og = outs()
    for _ in range(max(1, args.warmup)):
        sph_trans.batch_cycle(trs, d_in, og)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sph_trans.batch_cycle(trs, d_in, og)
    torch.cuda.synchronize()
    t_g = time.perf_counter() - t0
    err_g = max(float(((a - b).abs().amax(dim=1) / b.abs().amax(dim=1)).max()) for a, b in zip(og, o64))
    line = {
        "metric": "batched uneven instance cycles/s (cfg4: 64 instances, L in {63,127,255}, Nr in {33,65,129}, 2-4 fields)",
        "value": value, "unit": "instance cycles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_b / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES["split"], "data": "synthetic (seeded spectra, as cfg3)",
        "config": {"workload": "cfg4_batch64", "instances": n, "timing": "host wall clock around synchronous calls"},
        "fp64_sequential": {"value": n * args.steps / t_seq, "unit": "instance cycles/s",
                            "ms_per_step": 1e3 * t_seq / args.steps},
        "speedup_vs_fp64_sequential": t_seq / t_b,
        "autotuned_split_instances": nsplit, "autotuned_fp64_instances": n - nsplit,
        "rel_err_vs_fp64_max": err, "clocks": clk,
        "all_split_grouped_gemm": {"value": n * args.steps / t_g, "unit": "instance cycles/s",
                                   "ms_per_step": 1e3 * t_g / args.steps,
                                   "speedup_vs_fp64_sequential": t_seq / t_g, "rel_err_vs_fp64_max": err_g},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    for tr in trs:
        tr.close()
    return 0


def ctypes_probe(lib, dev):
    import ctypes
    try:
        f = lib.kmhd_probe_fp64_tflops
    except AttributeError:
        return None
    f.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    v = ctypes.c_double()
    return v.value if f(dev, ctypes.byref(v)) == 0 else None


def fp64_rooflines(cfg, kern, probe_tflops):
    """FP64-tier Legendre GEMMs (DMMA) against the FP64 tensor pipe measured
    in-process by the DMMA chain probe: useful flops per launch
    2*Nh*J*Nr*(5nv+ns) of each direction over its CUDA-event duration."""
    out = {}
    for key, name, nv, ns in (("gemm_bwd", "k_leg_bwd_f64", cfg.nvb, cfg.nsb),
                              ("gemm_fwd", "k_leg_fwd_f64", cfg.nvf, cfg.nsf)):
        fl = 2.0 * cfg.nh * cfg.J * cfg.nr * (5 * nv + ns)
        dur = kern.get(key, 0.0)
        ach = fl / (dur * 1e-3) / 1e12 if dur > 0 else None
        out[name] = {"bound": "tensor", "unit": "TFLOP/s", "achieved": ach, "peak": probe_tflops,
                     "frac": ach / probe_tflops if (ach and probe_tflops) else None, "ms_per_launch": dur,
                     "algorithmic_flops_per_launch": fl,
                     "peak_source": "FP64 tensor pipe measured in-process (DMMA chain probe)"}
    return out


def read_traffic(kernel, workload):
    """DRAM bytes (read + write) per launch of the kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}_dram.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def split_executed_ops(cfg, nprod):
    """INT8 ops (2 per MAC) one launch of the split GEMM would issue with every
    K chunk, averaged over the two directions: every (m, type, 128-row tile,
    64-column tile, 32-deep K chunk) runs nprod slice products of 128 x 64 x 32
    (the forward launch skips the chunks whose data digits are all zero)."""
    pad = lambda x, q: (x + q - 1) // q * q  # noqa: E731
    L, nh, nr = cfg.ltr, cfg.nh, cfg.nr
    nrT, nrR = pad(nr, 16), pad(nr, 8)
    tot = 0
    for m in range(L + 1):
        ke, ko = (L - m) // 2 + 1, (L - m + 1) // 2
        kep, kop, nhp = pad(ke, 32), pad(ko, 32), pad(nh, 32)
        gb, gf = (cfg.nvb + cfg.nsb + 3) // 4, (cfg.nvf + cfg.nsf + 3) // 4  # 8-column blocks per radius
        geo = {0: (nh, kop + kep, 4 * cfg.nvb * nrT), 1: (nh, kep + kop, 4 * cfg.nvb * nrT),
               2: (nh, kep, 8 * nrR * gb), 3: (nh, kop, 8 * nrR * gb),
               4: (ke, nhp, 8 * nrR * gf), 5: (ko, nhp, 8 * nrR * gf),
               6: (ke, 2 * nhp, 4 * cfg.nvf * nrT), 7: (ko, 2 * nhp, 4 * cfg.nvf * nrT)}
        for t, (rows, kp, ncol) in geo.items():
            if rows == 0 or ncol == 0:
                continue
            tot += (pad(rows, 128) // 128) * (pad(ncol, 64) // 64) * (kp // 32)
    return tot * nprod * 128 * 64 * 32 * 2 / 2.0


if __name__ == "__main__":
    sys.exit(main())

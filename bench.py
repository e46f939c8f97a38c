#!/usr/bin/env python
"""Benchmark of the batched training forward (srkTrainingForward drop-in).

Workload (one step): R_b = dx^2 (conv(E_b,Gx) dE_b/dx + conv(E_b,Gy) dE_b/dy)
for B = 5000 images of N = 512 (E = I, KW = 121, W = 392, dx = 4 nm, Green's
tensor gamma = 1/30 nm, R_w = erosion*dx), fp32, inputs already resident in
HBM (5.2 GB > L2, so no flush is needed between steps).  Inputs are seeded
Gaussian random fields (correlation length 8 px, min-max scaled to [0,1]).

Multi-GPU: one process per GPU, each rank runs its own B images (weak
scaling, no data-path collective); the step time is the max over ranks.

Extra keys: roofline (HBM, algorithmic (N^2+W^2)*4 bytes per image),
cpu_baseline (FP64 oracle on the host cores, rank 0 at N=1), e2e (host
buffers through the public API, copies inside the timed region), clocks,
gpu_launches, ops (per-operator throughput of the OaS derivatives).

--impl reference times the reference's CPU path restated by the oracle on
all host cores (the reference's own CPU code does not build on its own), and
adds the reference's own cuFFT srkTrainingForward built from its sources as
"gpu_reference".
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


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--B", type=int, default=5000)
    p.add_argument("--N", type=int, default=512)
    p.add_argument("--KW", type=int, default=121)
    p.add_argument("--dx", type=float, default=4.0)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-ops", action="store_true")
    p.add_argument("--no-extra", action="store_true", help="skip the fp16 and published-config lines")
    p.add_argument("--no-graph", action="store_true", help="time direct calls instead of the captured CUDA graph")
    p.add_argument("--no-grid", action="store_true", help="skip the per-op grid (Mpix/s and error per size)")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--large-slabs", action="store_true",
                   help="also time one N=32768 KW=121 image split by column slabs over the ranks "
                        "(halo exchange + slab forward / adjoint)")
    p.add_argument("--schedule", default="auto", choices=["auto", "persistent", "three_pass", "direct", "tensor_rows"],
                   help="override the autotuned kernel schedule (profiling)")
    p.add_argument("--dtype", default="f32", choices=["f32", "f16", "bf16"],
                   help="storage type of the main workload (profiling; the metric is quoted on f32)")
    p.add_argument("--tile-M", type=int, default=0,
                   help="fixed tile size instead of the autotuned one (profiling: no tuner launches)")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_per_image(N, KW, field):
    """A per-image figure (dram bytes, warp instructions) of the launch
    sequence from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    key = "N=%d KW=%d" % (N, KW)
    with open(path) as fh:
        for line in fh:
            if line.startswith(key) and field + "=" in line:
                return float(line.split(field + "=")[1].split()[0])
    return None


def profiled_traffic(N, KW, B):
    """dram bytes per launch sequence from the committed ncu summary, if any."""
    per_img = profiled_per_image(N, KW, "bytes_per_image")
    return None if per_img is None else per_img * B


def issue_bound(N, KW, B, ms, sm_mhz):
    """The instruction-issue bound of the step: warp instructions (committed
    ncu count) at one instruction per cycle on each of the 148 x 4 schedulers
    at the sampled SM clock, against the measured step time."""
    per_img = profiled_per_image(N, KW, "warp_instructions_per_image")
    if per_img is None or not sm_mhz:
        return None
    rate = 148 * 4 * sm_mhz * 1e6
    min_ms = per_img * B / rate * 1e3
    return {"warp_instructions_per_step": per_img * B, "issue_slots_per_s": rate, "min_ms": min_ms,
            "frac": min_ms / ms, "source": "profiles/traffic.txt (ncu smsp__inst_executed.sum)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

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
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def grf_batch(torch, B, N, seed0, ell=8.0):
    """Seeded Gaussian random fields generated on the device by the library
    (srk_grf: Philox noise, GpGenerator's filter, min-max scaled), [B][N][N]."""
    import shrinkage_full_tests_b200 as srk
    out = torch.empty((B, N, N), device="cuda", dtype=torch.float32)
    srk.grf(out, ell, seed0)
    torch.cuda.synchronize()
    return out


def make_spectra(torch, srk, KW, N, dx):
    e = (KW - 1) // 2
    Kx = torch.zeros((KW, KW), device="cuda")
    Ky = torch.zeros_like(Kx)
    srk.green_tensor(Kx, Ky, 1.0 / 30.0, e * dx, dx)
    GX = torch.zeros((N, N // 2 + 1), dtype=torch.complex64, device="cuda")
    GY = torch.zeros_like(GX)
    srk.srkPrecomputeKernelFreq(Kx, KW, KW, N, GX)
    srk.srkPrecomputeKernelFreq(Ky, KW, KW, N, GY)
    torch.cuda.synchronize()
    return Kx, Ky, GX, GY


def cpu_oracle_rate(N, KW, dx, seconds, nthreads):
    """Images/s of the FP64 oracle forward (direct valid convolution) on the host."""
    import numpy as np
    from oracle import oracle as O
    e = (KW - 1) // 2
    Kx, Ky = O.make_kernel(KW, dx, 1.0 / 30.0, e * dx)
    n, t0 = 0, time.perf_counter()
    while True:
        E = O.grf(N, 8.0, 1000 + n).astype(np.float64)
        O.forward(E, E, Kx, Ky, e, dx, nthreads=nthreads)
        n += 1
        el = time.perf_counter() - t0
        if (el >= seconds and n >= 2) or n >= 200:
            break
    return n / el, n, el


def time_steps(torch, fn, steps, warmup, dist):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    t = torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        fn()
    t.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(t) / steps
    if dist:
        dist.barrier()
    return ms


def max_over_ranks(torch, dist, x):
    if not dist:
        return x
    v = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v.item())


def e2e_pipeline(torch, srk, plan, GX, GY, N, W, e, dx, B, steps, warmup, dist, chunk=32):
    """Host-buffer end to end: pinned host E -> device, forward, device -> pinned
    host R, chunked over three streams so copies overlap compute."""
    Eh = torch.empty((B, N, N), dtype=torch.float32).pin_memory()
    Eh.uniform_()
    Rh = torch.empty((B, W, W), dtype=torch.float32).pin_memory()
    nslot = 3
    dE = [torch.empty((chunk, N, N), device="cuda") for _ in range(nslot)]
    dR = [torch.empty((chunk, W, W), device="cuda") for _ in range(nslot)]
    s_in, s_cmp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(nslot)]
    ev_cmp = [torch.cuda.Event() for _ in range(nslot)]
    ev_out = [torch.cuda.Event() for _ in range(nslot)]
    cur = torch.cuda.current_stream()

    def step():
        start = torch.cuda.Event()
        start.record(cur)
        for st in (s_in, s_cmp, s_out):
            st.wait_event(start)
        for i, b0 in enumerate(range(0, B, chunk)):
            b1 = min(B, b0 + chunk)
            k = i % nslot
            if i >= nslot:
                s_in.wait_event(ev_out[k])       # slot free again
            with torch.cuda.stream(s_in):
                dE[k][: b1 - b0].copy_(Eh[b0:b1], non_blocking=True)
                ev_in[k].record(s_in)
            s_cmp.wait_event(ev_in[k])
            srk.srkTrainingForward(dE[k], dE[k], GX, GY, N, W, e, dx, b1 - b0, s_cmp, dR[k], plan)
            ev_cmp[k].record(s_cmp)
            s_out.wait_event(ev_cmp[k])
            with torch.cuda.stream(s_out):
                Rh[b0:b1].copy_(dR[k][: b1 - b0], non_blocking=True)
                ev_out[k].record(s_out)
        for st in (s_in, s_cmp, s_out):
            end = torch.cuda.Event()
            end.record(st)
            cur.wait_event(end)

    ms = time_steps(torch, step, steps, warmup, dist)
    return ms, B * N * N * 4, B * W * W * 4


def run_ours(a):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        dist = td
    import shrinkage_full_tests_b200 as srk

    N, KW, B, dx = a.N, a.KW, a.B, a.dx
    e = (KW - 1) // 2
    W = N - 2 * e
    _, _, GX, GY = make_spectra(torch, srk, KW, N, dx)
    tdt, sdt = {"f32": (torch.float32, srk.SRK_F32), "f16": (torch.float16, srk.SRK_F16),
                "bf16": (torch.bfloat16, srk.SRK_BF16)}[a.dtype]
    E = grf_batch(torch, B, N, seed0=1_000_003 * rank + 17).to(tdt)
    R = torch.empty((B, W, W), device="cuda", dtype=tdt)
    plan = srk.SrkPlan(N, W, e, dx, B, dtype=sdt, tile_M=a.tile_M if a.tile_M else srk.SRK_TILE_AUTOTUNE)
    if a.schedule != "auto":
        plan.set_schedule({"persistent": srk.SRK_SCHEDULE_PERSISTENT, "three_pass": srk.SRK_SCHEDULE_THREE_PASS,
                           "direct": srk.SRK_SCHEDULE_DIRECT, "tensor_rows": srk.SRK_SCHEDULE_TENSOR_ROWS}[a.schedule])
    call = lambda: srk.srkTrainingForward(E, E, GX, GY, N, W, e, dx, B, None, R, plan)
    call()
    plan.sync()
    info = plan.info()
    # the step is one CUDA graph launch: the whole launch sequence of the
    # call (P1 / P2 / P3 per scratch chunk on three streams, forked from and
    # joined back into the capturing stream) captured once and replayed
    graph = None
    if not a.no_graph:
        cs = torch.cuda.Stream()
        cs.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(cs):
            call()
        cs.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=cs):
            call()
        torch.cuda.synchronize()
    step = graph.replay if graph is not None else call

    clk = ClockSampler(local)
    clk.start()
    ms = time_steps(torch, step, a.steps, a.warmup, dist)
    # the same K steps as direct calls (15 launches each): the value is the
    # faster of the two ways of issuing the identical work
    ms_direct = time_steps(torch, call, a.steps, a.warmup, dist) if graph is not None else None
    clocks = clk.stop()
    ms_graph = ms
    if ms_direct is not None:
        ms_direct = max_over_ranks(torch, dist, ms_direct)
        ms_graph = max_over_ranks(torch, dist, ms_graph)
        ms = min(ms_graph, ms_direct)
    ms = max_over_ranks(torch, dist, ms)
    imgs_per_s = world * B / (ms * 1e-3)
    mpix = world * B * W * W / (ms * 1e-3) / 1e6

    launches_per_step = info["last_launches"]
    peak, peak_kind = measured_peaks()
    alg_bytes = B * (N * N + W * W) * (4 if a.dtype == "f32" else 2)
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    traffic = profiled_traffic(N, KW, B)

    e2e = None
    if not a.no_e2e and a.dtype == "f32":
        ms_e2e, h2d, d2h = e2e_pipeline(torch, srk, plan, GX, GY, N, W, e, dx, B, max(2, a.steps // 2),
                                        1, dist)
        ms_e2e = max_over_ranks(torch, dist, ms_e2e)
        e2e = {"value": world * B / (ms_e2e * 1e-3), "unit": "img/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e, "pipeline": "3 streams, 32-image chunks"}

    ops = None
    if not a.no_ops and world == 1:
        ops = ops_throughput(torch, srk)
    grid = None
    if not a.no_grid and world == 1:
        grid = ops_grid(torch, srk)

    extra = {}
    if not a.no_extra and world == 1:
        extra["fp16_storage"] = half_storage_rate(torch, srk, E.float(), GX, GY, N, W, e, dx, B)
        extra["published_config"] = published_config_rate(torch, srk)
        # the large single image of the configurations: N = 32768, KW = 121, GRF ell = 32 px
        extra["large_image"] = ops_throughput(torch, srk, N=32768, KW=121, reps=1, spectra_M=2048, ell=32.0)
        torch.cuda.empty_cache()
        extra["direct_path"] = direct_path_rates(torch, srk)
        torch.cuda.empty_cache()

    if a.large_slabs:
        extra["large_image_slabs"] = large_image_slabs(torch, srk, rank, world, dist)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        nth = os.cpu_count() or 1
        rate, n, el = cpu_oracle_rate(N, KW, dx, a.cpu_seconds, nth)
        cpu = {"value": rate, "unit": "img/s", "cores": nth, "kind": "port",
               "sample": "%d images of N=%d KW=%d, FP64 direct valid convolution (oracle), %.1f s" % (n, N, KW, el)}

    graphed = graph is not None
    del graph
    if dist:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": "srkTrainingForward images/s (B=5000 per GPU, N=512, KW=121)",
            "value": imgs_per_s, "unit": "img/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": a.dtype, "data": "synthetic: seeded Gaussian random fields (ell=8 px, [0,1]), device-resident",
            "config": {"workload": "srkTrainingForward B=%d N=%d KW=%d W=%d dx=%g nm gamma=1/30 nm" % (B, N, KW, W, dx),
                       "B_per_gpu": B, "N": N, "KW": KW, "W": W, "tile_M": info["tile_M"],
                       "l2": "inputs (%.1f GB/GPU) larger than L2; no flush" % (B * N * N * 4 / 1e9),
                       "parallelism": "dp%d (batch shards, no collective)" % world},
            "output_mpix_per_s": mpix,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "srkTrainingForward launch sequence (P1+P2+P3 per chunk)",
                         "algorithmic_bytes_per_step": alg_bytes,
                         "issue_bound": issue_bound(N, KW, B, ms, (clocks or {}).get("sm_mhz"))},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches_per_step * a.steps,
            "ops": ops,
            "ops_grid": grid,
            "schedule": {"tile_M": info["tile_M"],
                         "schedule": ["persistent", "three_pass", "direct", "tensor_rows"][info["schedule"]],
                         "autotuned": a.schedule == "auto",
                         "step": ("one CUDA graph launch of the captured call" if graphed and ms == ms_graph
                                  else "direct call (%d launches)" % launches_per_step),
                         "ms_per_step_graph_replay": ms_graph if graphed else None,
                         "ms_per_step_direct_call": ms_direct},
        }
        line.update(extra)
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def half_storage_rate(torch, srk, E32, GX, GY, N, W, e, dx, B, steps=20):
    """Same workload with FP16 image storage (FP32 arithmetic)."""
    E = E32.half()
    R = torch.empty((B, W, W), device="cuda", dtype=torch.float16)
    plan = srk.SrkPlan(N, W, e, dx, B, dtype=srk.SRK_F16, tile_M=srk.SRK_TILE_AUTOTUNE)
    fn = lambda: srk.srkTrainingForward(E, E, GX, GY, N, W, e, dx, B, None, R, plan)
    ms = time_steps(torch, fn, steps, 3, None)
    peak, _ = measured_peaks()
    alg = B * (N * N + W * W) * 2
    info = plan.info()
    sched = ["persistent", "three_pass", "direct", "tensor_rows"][info["schedule"]]
    arith = ("f16 x f16 -> f32 column DFT and row convolution on the tensor cores, f32 inverse column FFT"
             if sched == "tensor_rows" else "f32 arithmetic")
    out = {"value": B / (ms * 1e-3), "unit": "img/s", "ms_per_step": ms, "dtype": "f16 storage, " + arith,
           "hbm_frac": alg / (ms * 1e-3) / 1e9 / peak, "tile_M": info["tile_M"], "schedule": sched}
    del E, R, plan
    torch.cuda.empty_cache()
    return out


def direct_path_rates(torch, srk, steps=10, bf16_peak=None):
    """The tensor-core direct schedule (SRK_SCHEDULE_DIRECT) against the FFT
    three-pass schedule on the training forward, B = 5000, N = 256, dx = 4 nm,
    KW = 15 and 31, FP16 storage (one MMA pass) and FP32 storage (three
    passes).  roofline: the MMA work the kernel executes (2 kernels x KW x
    (128 + KW - 1, rounded to 16) x 128 x 128 multiply-adds per 128 x 128
    output tile, x 3 passes for FP32) over the time, against the measured
    dense bf16 tensor peak; useful_tflops counts only the 2 x KW^2 taps per
    output pixel."""
    try:
        path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        peak = float(json.load(open(path))["bf16_tflops"]) if os.path.exists(path) else 1590.0
    except Exception:  # noqa: BLE001
        peak = 1590.0
    out = []
    B, N, dx = 5000, 256, 4.0
    E32 = grf_batch(torch, B, N, 41)
    for KW in (15, 31):
        e = (KW - 1) // 2
        W = N - 2 * e
        _, _, GX, GY = make_spectra(torch, srk, KW, N, dx)
        tiles = B * ((W + 127) // 128) ** 2
        KT = (128 + KW - 1 + 15) // 16 * 16
        mma_flop = tiles * 2 * KW * KT * 128 * 128 * 2
        useful = B * W * W * 2 * KW * KW * 2
        for dt, sdt, tdt, npass in (("f16", srk.SRK_F16, torch.float16, 1), ("f32", srk.SRK_F32, torch.float32, 3)):
            E = E32.to(tdt)
            R = torch.empty((B, W, W), device="cuda", dtype=tdt)
            row = {"N": N, "KW": KW, "B": B, "storage": dt}
            for name, sch in (("fft_three_pass", srk.SRK_SCHEDULE_THREE_PASS), ("direct", srk.SRK_SCHEDULE_DIRECT)):
                plan = srk.SrkPlan(N, W, e, dx, B, dtype=sdt)
                plan.set_schedule(sch)
                fn = lambda: srk.srkTrainingForward(E, E, GX, GY, N, W, e, dx, B, None, R, plan)
                ms = time_steps(torch, fn, steps, 3, None)
                plan.sync()
                row[name + "_ms"] = ms
                del plan
            tf = mma_flop * npass / (row["direct_ms"] * 1e-3) / 1e12
            row["direct_roofline"] = {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                                      "frac": tf / peak, "peak_source": "measured bf16 dense (burst)"}
            row["direct_useful_tflops"] = useful / (row["direct_ms"] * 1e-3) / 1e12
            row["faster"] = "direct" if row["direct_ms"] < row["fft_three_pass_ms"] else "fft_three_pass"
            out.append(row)
            del E, R
    del E32
    return out


def published_config_rate(torch, srk, steps=20):
    """The only published number of the reference: srkTrainingForward at
    B=3000, N=256, KW=121 took 55.39 ms on an sm_86-class GPU
    (notebooks/plot_compare_demo.ipynb cell 0)."""
    B, N, KW = 3000, 256, 121
    e = (KW - 1) // 2
    W = N - 2 * e
    _, _, GX, GY = make_spectra(torch, srk, KW, N, 1.0)
    E = grf_batch(torch, B, N, 99)
    R = torch.empty((B, W, W), device="cuda")
    plan = srk.SrkPlan(N, W, e, 1.0, B, tile_M=srk.SRK_TILE_AUTOTUNE)
    fn = lambda: srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
    ms = time_steps(torch, fn, steps, 3, None)
    out = {"config": "B=3000 N=256 KW=121", "ms_per_step": ms, "value": B / (ms * 1e-3), "unit": "img/s",
           "published_ms": 55.39, "speedup_vs_published": 55.39 / ms, "tile_M": plan.info()["tile_M"]}
    del E, R, plan
    torch.cuda.empty_cache()
    return out


def ops_throughput(torch, srk, N=4096, KW=61, reps=3, spectra_M=1024, ell=8.0):
    """Output Mpix/s of each OaS operator on one N x N image (one GPU)."""
    import numpy as np
    e = (KW - 1) // 2
    W = N - 2 * e
    _, _, GX, GY = make_spectra(torch, srk, KW, spectra_M, 1.0)
    f, g = grf_batch(torch, 2, N, 77, ell=ell)
    df, dg = (1e-2 * torch.randn((2, N, N), device="cuda")).unbind(0)
    lam, dlam = torch.randn((2, W, W), device="cuda").unbind(0)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=spectra_M, tile_M=srk.SRK_TILE_AUTOTUNE)
    R = torch.empty((W, W), device="cuda")
    ux, uy = torch.empty_like(R), torch.empty_like(R)
    o1, o2 = torch.empty((N, N), device="cuda"), torch.empty((N, N), device="cuda")
    runs = {
        "forward": lambda: srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan, ux, uy),
        "adjoint": lambda: srk.adjointSRK(lam, ux, uy, f, GX, GY, N, W, e, 1.0, None, o1, o2, plan),
        "tangent": lambda: srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, e, 1.0, None, R, plan),
        "tangent_adjoint": lambda: srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, GX, GY, N, W, e, 1.0,
                                                                   None, o1, o2, plan),
    }
    info = plan.info()
    out = {"config": "N=%d KW=%d B=1 fp32 tile_M=%d spectra_M=%d" % (N, KW, info["tile_M"], spectra_M),
           "library_workspace_bytes": info["scratch_bytes"] + 2 * W * W * 4 + 2 * info["tile_M"] ** 2 * 8}
    alg = {"forward": 2 * N * N + W * W, "adjoint": 3 * W * W + N * N + 2 * N * N,
           "tangent": 4 * N * N + W * W, "tangent_adjoint": 6 * N * N + 2 * W * W}
    peak, _ = measured_peaks()
    for k, fn in runs.items():
        ms = time_steps(torch, fn, reps * 4, 2, None)
        px = W * W if k in ("forward", "tangent") else N * N
        out[k] = {"ms": ms, "out_mpix_per_s": px / (ms * 1e-3) / 1e6,
                  "hbm_frac": alg[k] * 4 / (ms * 1e-3) / 1e9 / peak}
    return out


def ops_grid(torch, srk, reps=3):
    """Output Mpix/s of each operator over the benchmark grid, FP32 and FP16
    storage: forward and adjoint at N in {1k, 2k, 4k, 8k} x KW in {31, 61,
    121}; tangent and tangent-adjoint at N in {4k, 8k, 16k} x KW in {31, 121};
    one image per call, GRF inputs, spectra at the reference's OaS tile size
    (1024, 2048 from N = 8k).  hbm_frac: the operator's algorithmic bytes
    (forward 2N^2 + W^2, adjoint with v, ux, uy given 3W^2 + 3N^2, tangent
    4N^2 + W^2, tangent-adjoint 6N^2 + 2W^2; 4 or 2 bytes per value) over the
    time, against the measured HBM peak.  The errors of the same operators
    against the FP64 oracle come from the GPU parity tests
    (tests/test_gpu_configs.py), not from this timing run."""
    peak, _ = measured_peaks()
    cases = [(op, N, KW) for N in (1024, 2048, 4096, 8192) for KW in (31, 61, 121) for op in ("forward", "adjoint")]
    cases += [(op, N, KW) for N in (4096, 8192, 16384) for KW in (31, 121) for op in ("tangent", "tangent_adjoint")]
    out = []
    by_size = {}
    for op, N, KW in cases:
        by_size.setdefault((N, KW), []).append(op)
    for (N, KW), ops in sorted(by_size.items()):
        e = (KW - 1) // 2
        W = N - 2 * e
        Ms = 2048 if N >= 8192 else 1024
        _, _, GX, GY = make_spectra(torch, srk, KW, Ms, 1.0)
        f32 = grf_batch(torch, 2, N, 300 + N + KW)
        gen = torch.Generator(device="cuda").manual_seed(N + KW)
        for dt, tdt, sdt, bpv in (("f32", torch.float32, srk.SRK_F32, 4), ("f16", torch.float16, srk.SRK_F16, 2)):
            f, g = f32[0].to(tdt), f32[1].to(tdt)
            plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=Ms, dtype=sdt)
            R = torch.empty((W, W), device="cuda", dtype=tdt)
            ux, uy = torch.empty_like(R), torch.empty_like(R)
            o1 = torch.empty((N, N), device="cuda", dtype=tdt)
            o2 = torch.empty_like(o1)
            lam = torch.randn((W, W), device="cuda", generator=gen).to(tdt)
            runs, alg = {}, {}
            if "forward" in ops:
                runs["forward"] = lambda: srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan, ux, uy)
                alg["forward"] = 2 * N * N + W * W
            if "adjoint" in ops:
                runs["adjoint"] = lambda: srk.adjointSRK(lam, ux, uy, f, GX, GY, N, W, e, 1.0, None, o1, o2, plan)
                alg["adjoint"] = 3 * W * W + 3 * N * N
            if "tangent" in ops:
                df = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(tdt)
                dg = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(tdt)
                dlam = torch.randn((W, W), device="cuda", generator=gen).to(tdt)
                runs["tangent"] = lambda: srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, e, 1.0, None, R, plan)
                alg["tangent"] = 4 * N * N + W * W
                runs["tangent_adjoint"] = lambda: srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, GX, GY, N, W,
                                                                                 e, 1.0, None, o1, o2, plan)
                alg["tangent_adjoint"] = 6 * N * N + 2 * W * W
            srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan, ux, uy)  # ux, uy for the adjoint
            for op, fn in runs.items():
                ms = time_steps(torch, fn, reps, 1, None)
                px = W * W if op in ("forward", "tangent") else N * N
                out.append({"op": op, "N": N, "KW": KW, "storage": dt, "ms": ms,
                            "out_mpix_per_s": px / (ms * 1e-3) / 1e6,
                            "hbm_frac": alg[op] * bpv / (ms * 1e-3) / 1e9 / peak,
                            "tile_M": plan.info()["tile_M"]})
            del plan, R, ux, uy, o1, o2, lam
            runs.clear()
            torch.cuda.empty_cache()
        del f32
    return out


def large_image_slabs(torch, srk, rank, world, dist, N=32768, KW=121, reps=2, spectra_M=2048):
    """One N x N image split by column slabs over the ranks: each rank holds
    its own columns, exchanges the halos with its neighbours (NCCL
    point-to-point) and computes its output columns; the time of each op is
    the max over ranks of exchange + slab launch sequence."""
    from shrinkage_full_tests_b200 import shard
    e = (KW - 1) // 2
    W = N - 2 * e
    _, _, GX, GY = make_spectra(torch, srk, KW, spectra_M, 1.0)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=spectra_M, tile_M=512)
    S = plan.info()["tile_stride"]
    lo, hi = shard.slab_bounds(N, e, S, world)[rank]
    wlo, whi = min(lo, W), min(hi, W)
    gen = torch.Generator(device="cuda").manual_seed(5 + rank)
    f, g = (torch.rand((hi - lo, N), device="cuda", generator=gen) for _ in range(2))
    v, ux, uy = (torch.randn((whi - wlo, W), device="cuda", generator=gen) for _ in range(3))
    fwd, _, adj = shard.device_slab_ops(plan, GX, GY, N, e, 1.0)
    runs = {"forward": lambda: shard.forward_slabs(g, f, N, e, S, rank, world, dist, fwd),
            "adjoint": lambda: shard.adjoint_slabs(v, ux, uy, f, N, e, S, rank, world, dist, adj)}
    out = {"config": "N=%d KW=%d one image over %d GPU(s), column slabs of whole %d-column tiles" % (N, KW, world, S),
           "slab_columns_rank0": list(shard.slab_bounds(N, e, S, world)[0])}
    for k, fn in runs.items():
        ms = max_over_ranks(torch, dist, time_steps(torch, fn, reps, 1, dist))
        px = W * W if k == "forward" else N * N
        out[k] = {"ms": ms, "out_mpix_per_s": px / (ms * 1e-3) / 1e6}
    return out


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    N, KW, B, dx = a.N, a.KW, a.B, a.dx
    e = (KW - 1) // 2
    W = N - 2 * e
    nth = os.cpu_count() or 1
    import numpy as np
    from oracle import oracle as O
    Kx, Ky = O.make_kernel(KW, dx, 1.0 / 30.0, e * dx)
    sample = 4  # images per step
    imgs = [O.grf(N, 8.0, 2000 + i).astype(np.float64) for i in range(sample)]

    def step():
        for E in imgs:
            O.forward(E, E, Kx, Ky, e, dx, nthreads=nth)

    for _ in range(a.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        step()
    el = (time.perf_counter() - t0) / a.steps
    rate = sample / el
    line = {
        "impl": "reference", "metric": "srkTrainingForward images/s (B=5000 per GPU, N=512, KW=121)",
        "value": rate, "unit": "img/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": el * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded Gaussian random fields (ell=8 px, [0,1])",
        "config": {"workload": "srkTrainingForward B=%d N=%d KW=%d W=%d dx=%g nm gamma=1/30 nm" % (B, N, KW, W, dx),
                   "sample_per_step": "%d images (bounded sample of the B=%d workload)" % (sample, B)},
        "cpu_baseline": {"value": rate, "unit": "img/s", "cores": nth, "kind": "port",
                         "sample": "%d images per step, FP64 direct valid convolution (oracle restating "
                                   "cpu_conv_valid, adjoint/main_adjoint.cu:70-90)" % sample},
        "e2e": {"value": rate, "unit": "img/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["cpu_reference_f32_1thread"] = cpu_checker_f32_rate(N, KW, dx, Kx, Ky, imgs[0].astype(np.float32))
    line["gpu_reference"] = gpu_reference(a)
    line["gpu_reference_oas"] = gpu_reference_oas()
    line["gpu_reference_cudnn"] = gpu_reference_cudnn(a)
    print(json.dumps(line))


def cpu_checker_f32_rate(N, KW, dx, Kx, Ky, img, cols=16):
    """The reference's own CPU checker form (cpu_conv_valid + combine,
    adjoint/main_adjoint.cu:70-90, :321-333: float, one thread) timed on
    `cols` output columns of one image and scaled to whole images."""
    from oracle import oracle as O
    e = (KW - 1) // 2
    W = N - 2 * e
    t0 = time.perf_counter()
    O.forward_f32_cols(img, img, Kx, Ky, e, dx, W // 2, cols)
    el = time.perf_counter() - t0
    return {"value": cols / W / el, "unit": "img/s", "cores": 1, "kind": "port",
            "sample": "%d of %d output columns of one N=%d KW=%d image (%.2f s), scaled to a whole image"
                      % (cols, W, N, KW, el)}


def ref_inputs(torch, N, KW, dx, B, n_distinct=16):
    """Inputs of the reference arm, made without the product library: the
    kernel and its spectrum by the FP64 oracle on the host (make_kernel,
    srkPrecomputeKernelFreq restated), B images cycled from `n_distinct`
    host Gaussian random fields (the timed reference kernels do not depend
    on the data)."""
    import numpy as np
    from oracle import oracle as O
    e = (KW - 1) // 2
    Kx, Ky = O.make_kernel(KW, dx, 1.0 / 30.0, e * dx)
    imgs = np.stack([O.grf(N, 8.0, 17 + i).astype(np.float32) for i in range(min(B, n_distinct))])
    base = torch.from_numpy(imgs).cuda()
    reps = (B + base.shape[0] - 1) // base.shape[0]
    E = base.repeat(reps, 1, 1)[:B].contiguous()
    return Kx, Ky, E


def ref_spectra(torch, Kx, Ky, M):
    from oracle import oracle as O
    return (torch.from_numpy(O.kernel_freq(Kx, M)).cuda(), torch.from_numpy(O.kernel_freq(Ky, M)).cuda())


def gpu_reference_oas(N=4096, KW=61, M=1024, reps=5):
    """Stand-in for srkForwardOaS (srk_forward.cuh:354-501), whose cufftDX
    build is unavailable (MathDx is not installed): the same overlap-and-save
    decomposition — M x M tiles at stride M - 2e, 2-D R2C FFT, products with
    the Gx and Gy spectra, C2R, valid crop — with every tile of the image in
    ONE batched cuFFT plan (torch.fft over a [tiles, M, M] batch), then the
    central differences and the combine.  A fair lower bound for the
    per-tile cufftDX kernels (the same FFT work, batched).  Checked against
    the FP64 oracle on one output window; timed with CUDA events."""
    try:
        import numpy as np
        import torch
        if not torch.cuda.is_available():
            return None
        from oracle import oracle as O
        e = (KW - 1) // 2
        W = N - 2 * e
        S = M - 2 * e
        T = (W + S - 1) // S
        Kx, Ky, f3 = ref_inputs(torch, N, KW, 1.0, 1)
        f = f3[0]
        Kxt, Kyt = torch.from_numpy(Kx).cuda(), torch.from_numpy(Ky).cuda()

        def spec(K):
            # kernel centred at the origin of the tile frame (the reference's fftshift)
            P = torch.zeros((M, M), device="cuda")
            P[:KW, :KW] = K
            P = torch.roll(P, shifts=(-e, -e), dims=(0, 1))
            return torch.fft.rfft2(P)
        SX, SY = spec(Kxt), spec(Kyt)
        pad = torch.zeros((T * S + 2 * e, T * S + 2 * e), device="cuda")

        def step():
            pad[:N, :N] = f
            tiles = pad.unfold(0, M, S).unfold(1, M, S).reshape(T * T, M, M)
            F = torch.fft.rfft2(tiles)
            u = []
            for G in (SX, SY):
                c = torch.fft.irfft2(F * G, s=(M, M))[:, e:e + S, e:e + S]
                u.append(c.reshape(T, T, S, S).permute(0, 2, 1, 3).reshape(T * S, T * S)[:W, :W])
            fx = (f[e + 1:N - e + 1, e:N - e] - f[e - 1:N - e - 1, e:N - e]) * 0.5
            fy = (f[e:N - e, e + 1:N - e + 1] - f[e:N - e, e - 1:N - e - 1]) * 0.5
            return u[0] * fx + u[1] * fy

        for _ in range(2):
            step()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(reps):
            step()
        s1.record()
        torch.cuda.synchronize()
        ms = s0.elapsed_time(s1) / reps
        R = step().double().cpu().numpy()
        ox = oy = W // 2
        fh = f.double().cpu().numpy()
        ref = O.forward(fh, fh, Kx, Ky, e, 1.0, window=(ox, oy, 128, 128))
        diff = float(np.abs(R[ox:ox + 128, oy:oy + 128] - ref).max() / np.abs(ref).max())
        return {"what": "srkForwardOaS stand-in: every tile in one batched cuFFT plan (cufftDX build unavailable)",
                "config": "N=%d KW=%d M_TILE=%d, %d tiles per conv" % (N, KW, M, T * T), "ms": ms,
                "out_mpix_per_s": W * W / (ms * 1e-3) / 1e6, "max_rel_diff_vs_oracle_window": diff}
    except Exception as ex:  # noqa: BLE001
        return {"unavailable": "%s" % ex}


def gpu_reference_cudnn(a, B=20, reps=2):
    """The reference's cuDNN forward (training/srk_cudnn_forward.cuh:194-269,
    built from its sources) on a bounded batch of the same workload, scaled
    to images/s; None if unavailable."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from tests.gpu_util import ref_gpu
        L = ref_gpu()
        if L is None:
            return {"unavailable": "oracle/_ref/libref_gpu.so not built"}
        N, KW, dx = a.N, a.KW, a.dx
        e = (KW - 1) // 2
        W = N - 2 * e
        Kx, Ky, E = ref_inputs(torch, N, KW, dx, B)
        Kxt, Kyt = torch.from_numpy(Kx).cuda(), torch.from_numpy(Ky).cuda()
        R = torch.empty((B, W, W), device="cuda")
        st = torch.cuda.current_stream().cuda_stream
        ws = L.ref_cudnn_ws_create(N, W, KW, B, st)
        call = lambda: L.ref_cudnn_forward(E.data_ptr(), E.data_ptr(), Kxt.data_ptr(), Kyt.data_ptr(), N, W, e, dx,
                                           B, st, R.data_ptr(), ws)
        assert call() == 0
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(reps):
            call()
        s1.record()
        torch.cuda.synchronize()
        ms = s0.elapsed_time(s1) / reps
        L.ref_cudnn_ws_destroy(ws, st)
        return {"value": B / (ms * 1e-3), "unit": "img/s", "ms_per_step": ms, "B": B,
                "what": "reference srkCudnnForward (cuDNN heuristic algorithm) compiled for sm_100a from its sources, "
                        "bounded batch of the same workload"}
    except Exception as ex:  # noqa: BLE001
        return {"unavailable": "%s" % ex}


def gpu_reference(a):
    """The reference's own cuFFT srkTrainingForward (built from its sources into
    oracle/_ref) on this GPU, same workload; None if unavailable.  Its inputs
    and spectra are made without the product library (ref_inputs)."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from tests.gpu_util import ref_gpu
        L = ref_gpu()
        if L is None:
            return {"unavailable": "oracle/_ref/libref_gpu.so not built"}
        N, KW, B, dx = a.N, a.KW, a.B, a.dx
        e = (KW - 1) // 2
        W = N - 2 * e
        Kx, Ky, E = ref_inputs(torch, N, KW, dx, B)
        GX, GY = ref_spectra(torch, Kx, Ky, N)
        R = torch.empty((B, W, W), device="cuda")
        free0 = torch.cuda.mem_get_info()[0]
        st = torch.cuda.current_stream().cuda_stream
        ws = L.ref_train_ws_create(N, B, st)
        ws_bytes = free0 - torch.cuda.mem_get_info()[0]
        fn = lambda: L.ref_train_forward(E.data_ptr(), E.data_ptr(), GX.data_ptr(), GY.data_ptr(), N, W, e, dx, B,
                                         st, R.data_ptr(), ws)
        ms = time_steps(torch, fn, max(2, a.steps), 1, None)
        L.ref_train_ws_destroy(ws, st)
        return {"value": B / (ms * 1e-3), "unit": "img/s", "ms_per_step": ms, "workspace_bytes": ws_bytes,
                "what": "reference srkTrainingForward (cuFFT) compiled for sm_100a from its sources",
                "inputs": "16 host GRFs (FP64 oracle generator) cycled over B; spectra by the FP64 oracle"}
    except Exception as ex:  # the CPU line must still print
        return {"unavailable": "%s" % ex}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark: final-pass vectors/s of the multipass PIV analysis on B200.

Workload (default, `--workload c5`): a synthetic 4096x4096 uint16 (12-bit) particle-image pair
(0.05 particles/px, diameters 2-4 px, vortex of 10 px plus 0.01/px shear, spurious particle
clusters in 2 % of the final-pass cells of frame B), four passes 128 -> 64 -> 32 -> 16 px at 75 %
overlap (1,042,441 vectors in the final pass), FP32 plain path, no preprocessing beyond the
u16 -> f32 conversion, signal mask off, reference validation defaults.

One step = one frame pair: both frames prepared from device-resident u16 samples, all four
passes (placement, correlation, validation), final field in device memory. Inputs (2 x 32 MiB
samples, 2 x 64 MiB prepared images, two alternating pairs) exceed the 126 MB L2 between steps.

Printed JSON line (rank 0): value = whole-job final-pass vectors/s (device-resident inputs);
e2e = the same through the C ABI with pinned HOST buffers (H2D of both frames and D2H of the
final field inside the timed region); roofline of the correlation kernels; CPU baseline of the
oracle port; SM clocks sampled during the timed region.

`--impl reference` times the reference's CPU algorithm (the C++ restatement in oracle/, all host
threads) on a bounded sample of the same workload; rank 0 only.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "final-pass vectors/sec on 1 B200 at <=0.01 px RMS (plain vs batched TC); p99 latency"

WORKLOADS = {
    "c5": dict(
        name="4096x4096 u16 12-bit particle pair, 128->64->32->16 px at 75% overlap, FP32 plain",
        h=4096, w=4096, bits=12, windows=[128, 64, 32, 16], overlap=0.75, final_iterations=1, ppp=0.05,
        dmin=2.0, dmax=4.0, vmax=10.0, shear=0.01, outlier_frac=0.02, seed=5),
    "c3": dict(
        name="1280x800 u16 video stream, sequential pairs, 64->32 px at 50% overlap, 64 pairs per CUDA-graph replay",
        h=800, w=1280, bits=12, windows=[64, 32], overlap=0.5, final_iterations=1, ppp=0.04, dmin=2.0, dmax=5.0,
        amplitude=6.0, wavelength=320.0, phase_step=0.02, frames=65, stream=True, seed=3, outlier_frac=0.0),
    "c4": dict(
        name="serving: Poisson arrivals 400 pairs/s, u16 pairs of 512x512 / 1024x768 / 2048x2048, schedules "
             "[32] / [64,32] / [64,32,16] at 50% overlap, 60 GB admission budget, continuous batching",
        rate=400.0, duration=60.0, sizes=[(512, 512), (768, 1024), (2048, 2048)],
        schedules=[[32], [64, 32], [64, 32, 16]], pool=3, budget=60 << 30, max_in_flight=256, seed=4,
        serving=True, windows=[32], overlap=0.5, final_iterations=1, h=512, w=512, outlier_frac=0.0),
    "c2": dict(
        name="1024x1024 u16 12-bit Lamb-Oseen pair, min-background subtraction and 99th-percentile clip, "
             "64->32->16 px at 50% overlap, FP32 plain",
        h=1024, w=1024, bits=12, windows=[64, 32, 16], overlap=0.5, final_iterations=1, ppp=0.03,
        dmin=3.0, dmax=3.0, vmax=8.0, shear=0.0, outlier_frac=0.0, seed=2, core=80.0,
        clip_percentile=99.0, background="min", deform=True, batch_pairs=64),
    # the reference's default analysis (PivConfig / PreprocessConfig defaults, preprocess.rs:5-29,
    # multipass.rs:52-78) on a 1080p 8-bit pair: the frame shape its published timings use
    "r1080": dict(
        name="1920x1080 u8 particle pair, the reference's default analysis: blur 1 + local normalisation 4, "
             "96->64->64 px at 50% overlap, FP32 plain",
        h=1080, w=1920, bits=8, windows=[96, 64], overlap=0.5, final_iterations=2, ppp=0.03, dmin=2.0, dmax=4.0,
        vmax=6.0, shear=0.005, outlier_frac=0.0, seed=12, preprocess="default",
        # published: PIVKit (Metal, M5 Max) on this shape, about 200 pairs/s pipelined
        # (docs/phase3-plan.md:479-480,561 of the reference)
        published_pairs_per_s=200.0, batch_pairs=64),
}


def alg_flops(n):
    """Algorithmic FLOPs per window of side n: three real 2-D FFTs (r2c A, r2c B, c2r) at
    2.5 n^2 log2(n^2) each, the cross-spectrum multiply 6 n (n/2+1), the peak scan 2 n^2."""
    return 7.5 * n * n * math.log2(n * n) + 6 * n * (n // 2 + 1) + 2 * n * n


def product_grid(h, w, window, overlap):
    """Grid::new (grid.rs:20-44) through the library: (nx, ny, step, x0, y0)."""
    import piv_b200 as P
    g = P.Grid.new(h, w, window, overlap)
    return g.nx, g.ny, g.step, g.x0, g.y0


def oracle_grid(h, w, window, overlap):
    """Grid::new through the oracle, for the reference arm, which loads nothing of the product."""
    from oracle import oracle as O
    g = O.grid(h, w, window, overlap)
    return g.nx, g.ny, g.step, g.x0, g.y0


def make_inputs(wl, seed_offset=0, grid=product_grid):
    """The workload's synthetic u8/u16 pair (numpy only); `grid` places the outlier clusters on
    the final pass's cells."""
    from piv_b200 import synthetic as S
    h, w = wl["h"], wl["w"]
    field = S.vortex_shear_field(h, w, vmax=wl["vmax"], core=wl.get("core"), shear=wl["shear"])
    cells = None
    if wl["outlier_frac"] > 0:
        nx, ny, step, x0, y0 = grid(h, w, wl["windows"][-1], wl["overlap"])
        rng = np.random.default_rng(wl["seed"] + seed_offset)
        k = rng.choice(nx * ny, int(round(wl["outlier_frac"] * nx * ny)), replace=False)
        cells = np.stack([x0 + (k % nx) * step, y0 + (k // nx) * step], 1)
    return S.baseline_pair(h, w, wl["seed"] + seed_offset, field, ppp=wl["ppp"], dmin=wl["dmin"], dmax=wl["dmax"],
                           bits=wl["bits"], outlier_cells=cells, outlier_window=wl["windows"][-1])


def input_ring(a0, b0):
    """A ring of shifted copies of the pair holding at least 256 MiB of samples, taken in turn by
    the steps, so that a step's inputs come from HBM rather than from the 126 MB L2."""
    pair_bytes = a0.nbytes + b0.nbytes
    n_ring = max(2, -(-(256 << 20) // pair_bytes))
    return [(a0, b0)] + [(np.ascontiguousarray(np.roll(a0, (37 * k, 53 * k), (0, 1))),
                          np.ascontiguousarray(np.roll(b0, (37 * k, 53 * k), (0, 1)))) for k in range(1, n_ring)]


def workload_config(wl, ring, nvec, world):
    """The `config` object both arms print for a frame-pair workload."""
    a0 = ring[0][0]
    h, w = a0.shape
    pair_bytes = a0.nbytes + ring[0][1].nbytes
    cfg = {"workload": wl["name"], "image": f"{h}x{w} {a0.dtype.name} ({wl['bits']}-bit)", "windows": pass_windows(wl),
           "overlap": wl["overlap"], "final_pass_vectors": nvec, "parallelism": f"replicas x{world}",
           "inputs": f"{len(ring)} shifted copies of the pair taken in turn, {len(ring) * pair_bytes / 2**20:.0f} MiB "
                     f"of samples" + (" (+ one background image per pair)" if wl.get("background") else ""),
           "l2": "inputs > L2: a step's samples are not resident in the 126 MB L2 when it starts"}
    if wl.get("published_pairs_per_s"):
        cfg["baseline"] = (f"published {wl['published_pairs_per_s']:.0f} pairs/s (reference's Metal port, Apple M5 "
                           f"Max) x {nvec} final vectors")
    return cfg


class _DeviceBuffer:
    """A raw device allocation exposed to torch through __cuda_array_interface__."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def make_stream(wl):
    """A synthetic high-speed video: particles advected frame to frame by Taylor-Green vortices
    u = A sin(kx + phi_i) cos(ky), v = -A cos(kx + phi_i) sin(ky) whose phase drifts slowly.
    Returns [frames, H, W] u16 (12-bit)."""
    from piv_b200 import synthetic as S
    h, w, full = wl["h"], wl["w"], (1 << wl["bits"]) - 1
    x, y, s, a = S._blobs(h, w, wl["seed"], wl["ppp"], wl["dmin"], wl["dmax"], (120 / 255) * full, full)
    k = 2 * math.pi / wl["wavelength"]
    out = []
    for i in range(wl["frames"]):
        f = S.render(h, w, x, y, s, a)
        out.append(S.quantise(S.add_noise(f, (4 / 255) * full, wl["seed"] + 7 * i), full, np.uint16))
        phi = wl["phase_step"] * i
        amp = wl["amplitude"]

        def field(X, Y, phi=phi):
            X = np.asarray(X, np.float64)
            Y = np.asarray(Y, np.float64)
            return ((amp * np.sin(k * X + phi) * np.cos(k * Y)).astype(np.float32),
                    (-amp * np.cos(k * X + phi) * np.sin(k * Y)).astype(np.float32))
        x, y = S.displace(x, y, field)
    return np.stack(out)


def run_stream(args, wl):
    """The batching form on a video stream: all sequential pairs of wl['frames'] frames analysed by
    one CUDA-graph replay per step (prepare every frame, every pass of every pair)."""
    import torch

    import piv_b200 as P
    from piv_b200.replicas import Ranks
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(local)
    ranks = Ranks(backend="nccl", device=dev)
    # replicas: every rank analyses its own stream (weak scaling), nothing crosses GPUs
    frames = make_stream(dict(wl, seed=wl["seed"] + 101 * ranks.rank))
    nf, h, w = frames.shape
    k = nf - 1
    an = P.PivAnalyzer(piv_config(wl), device=local)
    fa, fb = an.prepare(frames[0], P.RAW), an.prepare(frames[1], P.RAW)
    tuned = an.autotune(fa, fb) if not args.no_autotune else {}
    batch = P.PivBatch(an, h, w, k, sequential=True)
    # the raw frames go once into the batch's device input slab (inputs resident in HBM)
    slab = torch.as_tensor(_DeviceBuffer(batch.input_device(), frames.nbytes // 2, "<i2"), device=dev)
    slab.copy_(torch.from_numpy(frames.reshape(-1).view(np.int16)).to(dev))
    torch.cuda.synchronize()
    bstream = torch.cuda.ExternalStream(batch.stream(), device=dev)
    nvec = k * final_vectors(wl)
    for _ in range(args.warmup):
        batch.run()
    batch.sync()
    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    sampler = ClockSampler(gpu_uuid if gpu_uuid.startswith("GPU-") else f"GPU-{gpu_uuid}")
    sampler.start()
    time.sleep(0.3)
    ranks.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(bstream)
    for _ in range(args.steps):
        batch.run()
    ev[1].record(bstream)
    ev[1].synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    ms = ranks.max(ev[0].elapsed_time(ev[1]))
    value = ranks.world * args.steps * nvec / (ms * 1e-3)
    # end to end: pinned host frames -> input slab -> graph -> results to host, every step
    pin = torch.from_numpy(frames.view(np.int16)).pin_memory().numpy().view(np.uint16)
    res = batch.run_host(pin)
    # two batches (each its own graph and copy streams, one shared compute stream) in turn: one's
    # upload and download overlap the other's graph; host clock with the device synchronised at
    # both ends
    batch2 = P.PivBatch(an, h, w, k, sequential=True)
    batch2.set_stream(batch.stream())
    batch2.run_host(pin)
    batch2.run_host(pin)
    g = batch.grid
    outs = [tuple(torch.empty(k * g.ny * g.nx, dtype=dt).pin_memory().numpy().reshape(k, g.ny, g.nx)
                  for dt in (torch.float32, torch.float32, torch.float32, torch.uint8)) for _ in range(2)]
    pair_of_batches = [batch, batch2]

    def e2e_run(n):
        last = None
        for i in range(n):
            b = pair_of_batches[i % 2]
            if i >= 2:
                last = b.wait_host()
            b.submit_host(pin, out=outs[i % 2])
        for i in range(max(0, n - 2), n):
            last = pair_of_batches[i % 2].wait_host()
        return last

    e2e_run(4)
    e2e_steps = max(8, args.steps // 2)
    ranks.barrier()
    torch.cuda.synchronize()
    t_e2e = time.perf_counter()
    res = e2e_run(e2e_steps)
    torch.cuda.synchronize()
    e2e_ms = ranks.max(1e3 * (time.perf_counter() - t_e2e))
    line = {"metric": METRIC, "value": value, "unit": "vectors/s", "n_gpus": ranks.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl["name"], "frames_per_step": nf, "pairs_per_step": k,
                       "final_pass_vectors_per_pair": final_vectors(wl), "windows": pass_windows(wl),
                       "l2": f"inputs > L2: {nf} frames = {frames.nbytes / 2**20:.0f} MiB of samples + "
                             f"{nf * h * w * 4 / 2**20:.0f} MiB prepared per step"},
            "e2e": {"value": ranks.world * e2e_steps * nvec / (e2e_ms * 1e-3), "unit": "vectors/s",
                    "h2d_bytes_per_step": int(pin.nbytes), "d2h_bytes_per_step": int(nvec * 13 + k * 40),
                    "ms_per_step": e2e_ms / e2e_steps,
                    "how": f"two PivBatch objects in turn sharing one compute stream (submit_host / wait_host "
                           f"over pinned frames): upload of {nf} frames, one graph replay and download of {k} "
                           f"fields per step; host clock, device synchronised at both ends"},
            "gpu_launches": int(batch.kernels() * args.steps), "graph_launches": args.steps,
            "clocks": clocks, "autotuned_variants": tuned, "wall_ms_per_step": 1e3 * wall / args.steps,
            "valid_fraction_last_pair": float(np.mean((res[-1].field.flags & P.flags.INVALID) == 0)),
            "parallelism": f"replicas x{ranks.world}"}
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)
    del batch, batch2
    ranks.close()
    return 0


def serving_block(wl, duration, local, ranks):
    """The serving form under a Poisson load: requests of mixed sizes and window schedules are
    submitted at their arrival times to one PivServer (continuous batching); latency is submit ->
    results in host memory. vectors/s counts the final-pass vectors of all completed requests
    over the span from the first submission to the last completion."""
    import threading as th

    import torch

    import piv_b200 as P
    from piv_b200 import synthetic as S
    # replicas: every rank serves its own Poisson stream on its own GPU
    rng = np.random.default_rng(wl["seed"] + 101 * ranks.rank)
    pool = {}
    for si, (h, w) in enumerate(wl["sizes"]):
        for j in range(wl["pool"]):
            shear, off = float(rng.uniform(0, 0.02)), float(rng.uniform(0, 4))
            f = (lambda sh, of, hh: (lambda X, Y: (np.float32(of) + sh * (np.asarray(Y, np.float32) - hh / 2),
                                                   np.float32(0.5 * of))))(shear, off, h)
            a, b = S.baseline_pair(h, w, 1000 * si + j, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)
            pool[(si, j)] = tuple(torch.from_numpy(x.view(np.int16)).pin_memory().numpy().view(np.uint16) for x in (a, b))
    cfgs = [P.PivConfig(windows=s, overlap=wl["overlap"], final_iterations=1) for s in wl["schedules"]]
    n = int(rng.poisson(wl["rate"] * duration))
    arrivals = np.cumsum(rng.exponential(1.0 / wl["rate"], n))
    kinds = [(int(rng.integers(0, len(wl["sizes"]))), int(rng.integers(0, len(cfgs))), int(rng.integers(0, wl["pool"])))
             for _ in range(n)]
    vec = {(si, ci): len(P.Grid.new(wl["sizes"][si][0], wl["sizes"][si][1], cfgs[ci].windows[-1], cfgs[ci].overlap))
           for si in range(len(wl["sizes"])) for ci in range(len(cfgs))}
    sv = P.PivServer(memory_budget_bytes=wl["budget"], max_in_flight=wl["max_in_flight"], device=local)
    # the server's pool is grown to its admission budget (within the free memory) before the
    # arrivals start, so that no admission waits on the driver to map new memory under load
    free = torch.cuda.mem_get_info(torch.device("cuda", local))[0]
    held0 = sv.reserve(int(max(0, min(wl["budget"], free - (16 << 30)))))
    # warm-up: one request of every kind
    for si in range(len(wl["sizes"])):
        for ci in range(len(cfgs)):
            sv.wait(sv.submit(*pool[(si, 0)], cfgs[ci]))
    tickets = []
    lat = []
    done = th.Event()

    def waiter():
        i = 0
        while i < n:
            while i >= len(tickets):
                if done.is_set() and i >= len(tickets):
                    return
                time.sleep(0.0002)
            _, l = sv.wait(tickets[i])
            lat.append(l)
            i += 1

    wt = th.Thread(target=waiter)
    wt.start()
    sampler = _clock_sampler(torch, torch.device("cuda", local))
    sampler.start()
    s0 = sv.stats()
    ranks.barrier()
    t0 = time.perf_counter()
    for i in range(n):
        now = time.perf_counter() - t0
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        si, ci, pj = kinds[i]
        tickets.append(sv.submit(*pool[(si, pj)], cfgs[ci]))
    done.set()
    wt.join()
    span = time.perf_counter() - t0
    clocks = sampler.stop()
    s1 = sv.stats()
    held1 = sv.reserve(0)
    # Capacity of the batching form on the same mix: the first requests of the stream submitted at
    # once (the scheduler then advances all of them together, one fused correlation launch per
    # step), against the plain path on the same requests one after another (PivAnalyzer.analyze
    # from the same pinned host frames, one analyzer per (size, schedule)).
    burst = kinds[:min(len(kinds), 1200)]
    burst_vec = sum(vec[(si, ci)] for si, ci, _ in burst)
    ranks.barrier()
    t1 = time.perf_counter()
    bt = [sv.submit(*pool[(si, pj)], cfgs[ci]) for si, ci, pj in burst]
    for t in bt:
        sv.wait(t)
    sat_s = ranks.max(time.perf_counter() - t1)
    sv.close()
    ans = {}  # (size, schedule) -> analyzer and its two frames, reused by every request of that kind
    for si in range(len(wl["sizes"])):
        for ci in range(len(cfgs)):
            an = P.PivAnalyzer(cfgs[ci], device=local)
            h, w = wl["sizes"][si]
            ans[(si, ci)] = (an, an.frame(h, w), an.frame(h, w))

    def plain(si, ci, pj):
        an, fa, fb = ans[(si, ci)]
        an.analyze(fa.prepare(pool[(si, pj)][0], P.RAW), fb.prepare(pool[(si, pj)][1], P.RAW))

    for key in ans:  # warm-up: first use of each analyzer (workspace, pass graph capture)
        for _ in range(3):
            plain(key[0], key[1], 0)
    ranks.barrier()
    t2 = time.perf_counter()
    for si, ci, pj in burst:
        plain(si, ci, pj)
    plain_s = ranks.max(time.perf_counter() - t2)
    for an, fa, fb in ans.values():
        fa.close()
        fb.close()
        an.close()
    total_vec = ranks.sum(sum(vec[(si, ci)] for si, ci, _ in kinds))
    span = ranks.max(span)
    n_all = int(ranks.sum(n))
    launches = ranks.sum(s1["kernel_launches"] - s0["kernel_launches"])
    lat_a = np.concatenate([np.asarray(x) for x in ranks.gather(lat)])
    return {"workload": wl["name"], "value": total_vec / span, "unit": "vectors/s", "requests": n_all,
            "duration_s": duration, "rate_per_s": wl["rate"] * ranks.world, "span_s": span,
            "latency_ms": {"p50": float(np.percentile(lat_a, 50)), "p90": float(np.percentile(lat_a, 90)),
                           "p99": float(np.percentile(lat_a, 99)), "max": float(lat_a.max()),
                           "mean": float(lat_a.mean())},
            "achieved_rate_per_s": n_all / span,
            "h2d_bytes_per_request": int(np.mean([pool[(si, pj)][0].nbytes * 2 for si, _, pj in kinds])),
            "d2h_bytes_per_request": int(np.mean([vec[(si, ci)] * 13 for si, ci, _ in kinds])),
            "gpu_launches": int(launches), "server_steps": int(s1["steps"] - s0["steps"]),
            "pool_reserved_bytes": int(held0), "pool_grew_bytes": int(held1 - held0),
            "saturated": {"requests": int(ranks.sum(len(burst))), "value": ranks.sum(burst_vec) / sat_s,
                          "unit": "vectors/s", "span_s": sat_s,
                          "how": "the first requests of the stream submitted at once to the same server, host to host"},
            "plain_one_at_a_time": {"value": ranks.sum(burst_vec) / plain_s, "unit": "vectors/s", "span_s": plain_s,
                                    "how": "the same requests through PivAnalyzer.prepare + analyze one after another "
                                           "(blocking, host to host), one analyzer per size and schedule"},
            "clocks": clocks}


def run_serving(args, wl):
    """The serving workload on its own: one JSON line whose value is the served vectors/s."""
    import torch

    from piv_b200.replicas import Ranks
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks(backend="nccl", device=torch.device("cuda", local))
    duration = args.duration if args.duration else wl["duration"]
    r = serving_block(wl, duration, local, ranks)
    line = {"metric": METRIC, "value": r["value"], "unit": "vectors/s", "n_gpus": ranks.world, "steps": r["requests"],
            "warmup": 9, "ms_per_step": 1e3 * r["span_s"] / max(r["requests"], 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl["name"], "requests": r["requests"], "duration_s": duration,
                       "rate_per_s": r["rate_per_s"], "parallelism": f"replicas x{ranks.world}"},
            "latency_ms": r["latency_ms"], "achieved_rate_per_s": r["achieved_rate_per_s"],
            "e2e": {"value": r["value"], "unit": "vectors/s", "h2d_bytes_per_step": r["h2d_bytes_per_request"],
                    "d2h_bytes_per_step": r["d2h_bytes_per_request"]},
            "gpu_launches": r["gpu_launches"], "server_steps": r["server_steps"],
            "pool_reserved_bytes": r["pool_reserved_bytes"], "pool_grew_bytes": r["pool_grew_bytes"],
            "saturated": r["saturated"], "plain_one_at_a_time": r["plain_one_at_a_time"], "clocks": r["clocks"]}
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def piv_config(wl):
    import piv_b200 as P
    return P.PivConfig(windows=list(wl["windows"]), overlap=wl["overlap"], final_iterations=wl["final_iterations"],
                       deform=bool(wl.get("deform", False)), precision=wl.get("precision", "fp32"))


def final_vectors(wl, h=None, w=None):
    import piv_b200 as P
    return len(P.Grid.new(h or wl["h"], w or wl["w"], wl["windows"][-1], wl["overlap"]))


def pass_windows(wl):
    return list(wl["windows"]) + [wl["windows"][-1]] * (wl["final_iterations"] - 1)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu_id)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
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
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def fp32_peak_tflops(dev):
    """Measured FP32 CUDA-core throughput: a cuBLAS SGEMM (TF32 off), best of 5, 8192^3."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, device=dev, dtype=torch.float32)
        b = torch.randn(n, n, device=dev, dtype=torch.float32)
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def load_traffic(workload):
    """Per-launch DRAM traffic of the correlation kernels from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"correlate_{workload}_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except OSError:
        return None


def _crop_background(wl, a, b, ch, cw):
    """The workload's background over the cropped pair (per-pixel minimum, decoded), or None."""
    if wl.get("background") != "min":
        return None
    top = np.float32(np.iinfo(a.dtype).max)
    return (np.minimum(a[:ch, :cw], b[:ch, :cw]).astype(np.float32) / top).astype(np.float32)


def oracle_config(wl):
    from oracle import oracle as O
    return O.OracleConfig(tuple(wl["windows"]), wl["overlap"], wl["final_iterations"],
                          deform=int(bool(wl.get("deform", False))))


def oracle_frames(wl, a, b, bg):
    """The oracle's prepared images and signal-mask intensities of a pair, with the workload's
    preprocessing: the percentile clip of each frame's codes (a3), decoding, the background
    subtraction base = max(raw - background, 0) and the default blur and local normalisation where
    the workload has them (preprocess.rs:138-158)."""
    from oracle import oracle as O
    dec = O.u16_to_f32 if a.dtype == np.uint16 else O.u8_to_f32
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    if wl.get("clip_percentile"):
        a, _ = O.percentile_clip_u16(a, wl["clip_percentile"])
        b, _ = O.percentile_clip_u16(b, wl["clip_percentile"])
    fa, fb = dec(a), dec(b)
    ba, bb = fa, fb
    blur, radius, eps = (1.0, 4, 0.02) if wl.get("preprocess") == "default" else (0.0, 0, 0.0)
    if bg is not None or radius:
        fa, ba = O.prepare(fa, blur, radius, eps, background=bg)
        fb, bb = O.prepare(fb, blur, radius, eps, background=bg)
    return fa, fb, ba, bb


def _oracle_inputs(wl, a, b, crop):
    from oracle import oracle as O
    ch, cw = min(crop, wl["h"]), min(crop, wl["w"])
    fa, fb, ba, bb = oracle_frames(wl, a[:ch, :cw], b[:ch, :cw], _crop_background(wl, a, b, ch, cw))
    return O, fa, fb, oracle_config(wl), ch, cw, ba, bb


def oracle_pair(wl, a, b, bg, nthreads):
    """One analysis of a pair by the oracle port, preparation included: the reference's
    PreparedFrame::new + PivAnalyzer::analyze (preprocess.rs:138-158, multipass.rs:136-192).
    Returns the number of final-pass vectors."""
    from oracle import oracle as O
    fa, fb, ba, bb = oracle_frames(wl, a, b, bg)
    fin, _, _ = O.analyze(oracle_config(wl), fa, fb, ba, bb, nthreads=nthreads)
    return int(fin["dx"].size)


def preprocess_config(wl):
    import piv_b200 as P
    clip = float(wl.get("clip_percentile", 0.0))
    if wl.get("preprocess") == "default":  # blur sigma 1, local normalisation radius 4, eps 0.02
        return P.PreprocessConfig(clip_percentile=clip)
    return P.PreprocessConfig(smooth_sigma=0.0, normalize_radius=0, normalize_eps=0.0, clip_percentile=clip)


def _torch_view(x):
    """A numpy frame as a torch-compatible array of the same bytes (torch has no uint16)."""
    return x.view(np.int16) if x.dtype == np.uint16 else x


def cpu_baseline(wl, a, b, budget_s=10.0, crop=1024, single_s=0.0):
    """Times the oracle port (reference operation order, OpenMP over windows, all host threads) on
    whole pairs of the workload, preparation included, until budget_s has passed (at least one
    pair); returns final-pass vectors/s and the sample used, plus a single-thread figure on a
    crop x crop corner of the pair with the same schedule when single_s > 0."""
    nthreads = os.cpu_count() or 1
    bg = _crop_background(wl, a, b, a.shape[0], a.shape[1])

    def timed(fa, fb, fbg, nt, budget):
        t0 = time.perf_counter()
        reps, vec = 0, 0
        while True:
            vec += oracle_pair(wl, fa, fb, fbg, nt)
            reps += 1
            if time.perf_counter() - t0 >= budget:
                break
        return reps, vec, time.perf_counter() - t0

    reps, vec, dt = timed(a, b, bg, nthreads, budget_s)
    out = {"value": vec / dt, "unit": "vectors/s", "cores": nthreads, "kind": "port",
           "sample": f"{reps} x the whole {a.shape[0]}x{a.shape[1]} pair, preparation and all "
                     f"{len(pass_windows(wl))} passes ({vec // reps} final vectors), oracle/piv_oracle.cpp, "
                     f"{nthreads} OpenMP threads, {dt:.1f} s"}
    if single_s > 0:
        ch, cw = min(crop, a.shape[0]), min(crop, a.shape[1])
        ca, cb = np.ascontiguousarray(a[:ch, :cw]), np.ascontiguousarray(b[:ch, :cw])
        r1, v1, d1 = timed(ca, cb, _crop_background(wl, a, b, ch, cw), 1, single_s)
        out["single_thread_value"] = v1 / d1
        out["single_thread_sample"] = f"{r1} x the same analysis of a {ch}x{cw} corner on 1 thread, {d1:.1f} s"
    return out


def accuracy_vs_fp64(wl, a, b, an, crop=1024, cache=None):
    """The GPU's final field on a crop of the pair against the FP64 oracle's (every correlation
    step in f64): RMS and max |d| over cells both mark valid, and the share of equal flags.
    `cache` (a dict) keeps the oracle's field for further calls on the same crop."""
    O, fa, fb, cfg, ch, cw, ba, bb = _oracle_inputs(wl, a, b, crop)
    if cache is not None and "fp64" in cache:
        ref = cache["fp64"]
    else:
        ref, _, _ = O.analyze(cfg, fa, fb, ba, bb, mode=O.FP64)
        if cache is not None:
            cache["fp64"] = ref
    pre, bg = preprocess_config(wl), _crop_background(wl, a, b, ch, cw)
    r = an.analyze(an.prepare(np.ascontiguousarray(a[:ch, :cw]), pre, background=bg),
                   an.prepare(np.ascontiguousarray(b[:ch, :cw]), pre, background=bg))
    ok = (ref["flags"] == 0) & (r.field.flags == 0)
    d = np.hypot(r.field.dx[ok] - ref["dx"][ok], r.field.dy[ok] - ref["dy"][ok])
    return {"rms_px_vs_fp64": float(np.sqrt(np.mean(d * d))) if d.size else None,
            "max_px_vs_fp64": float(d.max()) if d.size else None,
            "flag_agreement": float(np.mean(ref["flags"] == r.field.flags)),
            "sample": f"final field of a {ch}x{cw} crop ({ok.sum()} cells valid in both), FP64 oracle"}


def run_profile_case(args, wl):
    """An untimed run for profilers: one pair of the workload, prepared with the workload's
    preprocessing and analysed --steps times through the host C ABI with the default launch
    variants (inputs cached under /tmp between processes)."""
    import piv_b200 as P
    w = dict(wl)
    if args.profile_case != "all":
        w["windows"] = [int(x) for x in args.profile_case.split(",")]
    cache = f"/tmp/piv_b200_{args.workload}_pair.npz"
    if os.path.exists(cache):
        z = np.load(cache)
        a, b = z["a"], z["b"]
    else:
        a, b = make_inputs(wl)
        np.savez(cache, a=a, b=b)
    an = P.PivAnalyzer(piv_config(w), device=0)
    pre, bg = preprocess_config(wl), _crop_background(wl, a, b, a.shape[0], a.shape[1])
    fa, fb = an.prepare(a, pre, background=bg), an.prepare(b, pre, background=bg)
    for _ in range(max(args.steps, 1)):
        r = an.analyze(fa, fb)
    print(json.dumps({"profile_case": w["windows"], "vectors": int(r.field.dx.size), "summary": r.summary.as_dict(),
                      "launches": an.launches()}))
    return 0


# seconds of timed steps the reference arm aims at (whole pairs when the steps fit)
REF_TOTAL_S = 165.0


def run_reference(args, wl):
    """The reference's CPU algorithm (the oracle port of piv-core, all host threads) on this arm's
    workload: the same pair, the same ring of shifted copies taken in turn, the same preparation
    and pass schedule, one step = one pair. Nothing of the product library is loaded. Steps are
    timed one by one on the host clock; when whole pairs would take well over REF_TOTAL_S in all,
    every step analyses the same top band of rows of its pair instead, and the line says so."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if wl.get("serving"):
        return run_reference_serving(args, wl)
    nthreads = os.cpu_count() or 1
    if wl.get("stream"):
        fr = make_stream(dict(wl, frames=2))
        a0, b0 = fr[0], fr[1]
    else:
        a0, b0 = make_inputs(wl, grid=oracle_grid)
    ring = input_ring(a0, b0)
    h, w = a0.shape
    # the background of each pair (BackgroundEstimator, preprocess.rs:47-72), estimated before the
    # steps as the reference estimates it before its pair loop
    bgs = [_crop_background(wl, a, b, h, w) for a, b in ring]
    nx, ny, _, _, _ = oracle_grid(h, w, wl["windows"][-1], wl["overlap"])
    nvec = nx * ny
    # warm-up: the same analysis on a band of the top rows (the oracle keeps no state between
    # calls; this starts its thread pool and touches the inputs) and a size estimate for the steps
    band = min(h, max(256, max(wl["windows"]) * 2))
    t_band = 0.0
    for i in range(args.warmup):
        a, b = ring[i % len(ring)]
        t0 = time.perf_counter()
        v_band = oracle_pair(wl, a[:band], b[:band], None if bgs[i % len(ring)] is None else bgs[i % len(ring)][:band],
                             nthreads)
        t_band = time.perf_counter() - t0
    est_pair = t_band * nvec / max(v_band, 1)
    rows = h
    if args.steps * est_pair > 1.5 * REF_TOTAL_S:
        rows = max(band, int(h * REF_TOTAL_S / (args.steps * est_pair)))
    times, vecs = [], 0
    for i in range(args.steps):
        a, b = ring[i % len(ring)]
        bg = bgs[i % len(ring)]
        t0 = time.perf_counter()
        vecs += oracle_pair(wl, a[:rows], b[:rows], None if bg is None else bg[:rows], nthreads)
        times.append(time.perf_counter() - t0)
    total = float(sum(times))
    v = vecs / total
    sample = (f"{args.steps} whole {h}x{w} pair{'s' if args.steps != 1 else ''}" if rows == h else
              f"{args.steps} steps, each the top {rows} of {h} rows of its pair (whole pairs would take about "
              f"{args.steps * est_pair:.0f} s)") + (f", preparation and all {len(pass_windows(wl))} passes, "
                                                   f"oracle/piv_oracle.cpp (C++ restatement of piv-core), "
                                                   f"{nthreads} OpenMP threads, {total:.1f} s timed")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "vectors/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(wl, ring, nvec, args.gpus),
            "cpu_baseline": {"value": v, "unit": "vectors/s", "cores": nthreads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "vectors/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_ms": {"min": 1e3 * min(times), "median": 1e3 * float(np.median(times)), "max": 1e3 * max(times)}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_serving(args, wl):
    """The reference's CPU path on the serving mix: one request of every (size, schedule) kind in
    turn per step (the reference has no serving form; its analysis runs one pair at a time)."""
    from piv_b200 import synthetic as S
    nthreads = os.cpu_count() or 1
    reqs = []
    for si, (h, w) in enumerate(wl["sizes"]):
        f = (lambda X, Y: (np.float32(2.0) + 0.01 * (np.asarray(Y, np.float32) - h / 2), np.float32(1.0)))
        a, b = S.baseline_pair(h, w, 1000 * si, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)
        for sched in wl["schedules"]:
            reqs.append((dict(wl, windows=list(sched), final_iterations=1, h=h, w=w), a, b))
    for _ in range(args.warmup):
        pass  # the oracle keeps no state between calls
    times, vecs = [], 0
    for i in range(args.steps):
        t0 = time.perf_counter()
        for rwl, a, b in reqs:
            vecs += oracle_pair(rwl, a, b, None, nthreads)
        times.append(time.perf_counter() - t0)
    total = float(sum(times))
    v = vecs / total
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "vectors/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl["name"], "parallelism": f"replicas x{args.gpus}"},
            "cpu_baseline": {"value": v, "unit": "vectors/s", "cores": nthreads, "kind": "port",
                             "sample": f"{args.steps} x one request of each of the {len(reqs)} (size, schedule) kinds "
                                       f"in turn, {nthreads} OpenMP threads, {total:.1f} s"},
            "e2e": {"value": v, "unit": "vectors/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def batched_figure(args, P, torch, wl, an, pre, pairs_host, bg_ptr, dev, ranks):
    """The batching form: K independent pairs of the ring per CUDA-graph replay (PivBatch), inputs
    resident on the device; K pairs of samples exceed L2, so every replay reads them from HBM.
    One background image (that of the first pair) serves the whole batch."""
    a0 = pairs_host[0][0]
    h, w = a0.shape
    nvec = len(an.output_grid(h, w))
    K = int(wl["batch_pairs"])
    bt = P.PivBatch(an, h, w, K, sequential=False, dtype=a0.dtype, cfg=pre)
    bt.set_background(bg_ptr)
    frames = np.stack([x for k in range(K) for x in pairs_host[k % len(pairs_host)]])
    tview = _torch_view(frames.reshape(-1))
    slab = torch.as_tensor(_DeviceBuffer(bt.input_device(), tview.size, "<i2" if a0.dtype == np.uint16 else "|u1"),
                           device=dev)
    slab.copy_(torch.from_numpy(tview).to(dev))
    torch.cuda.synchronize()
    bstream = torch.cuda.ExternalStream(bt.stream(), device=dev)
    for _ in range(max(args.warmup, 3)):
        bt.run()
    bt.sync()
    runs = max(5, args.steps // 10)
    sampler = _clock_sampler(torch, dev)
    sampler.start()
    time.sleep(0.2)
    ranks.barrier()
    ev_start, ev_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev_start.record(bstream)
    for _ in range(runs):
        bt.run()
    ev_end.record(bstream)
    ev_end.synchronize()
    clocks = sampler.stop()
    bms = ranks.max(ev_start.elapsed_time(ev_end)) / runs
    out = {"workload": wl["name"], "pairs_per_graph": K, "value": ranks.world * K * nvec / (bms * 1e-3),
           "unit": "vectors/s", "ms_per_pair": bms / K, "runs": runs, "gpu_launches": int(bt.kernels() * runs),
           "clocks": clocks,
           "how": f"{K} independent pairs per CUDA-graph replay of PivBatch (preparation of all frames and every "
                  f"pass), {frames.nbytes / 2**20:.0f} MiB of samples resident on the device"}
    del slab
    bt.close()
    return out


def _clock_sampler(torch, dev):
    gpu_uuid = str(torch.cuda.get_device_properties(dev).uuid)
    return ClockSampler(gpu_uuid if gpu_uuid.startswith("GPU-") else f"GPU-{gpu_uuid}")


def device_background(P, torch, an, pairs_dev, dtype_code, h, w, dev):
    """The background of each pair, the per-pixel minimum over its two frames
    (BackgroundEstimator, preprocess.rs:47-72), estimated on the device before the timed steps as
    the reference estimates it before its pair loop. Returns the device images."""
    import ctypes
    lib = P.load_library()
    out = []
    for ta, tb in pairs_dev:
        stack = torch.stack([ta, tb])
        bgk = torch.empty((h, w), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        P.api._check(lib.piv_background_device(an._h, ctypes.c_void_p(stack.data_ptr()), dtype_code, 2, h, w, 0,
                                               ctypes.c_void_p(bgk.data_ptr())))
        torch.cuda.synchronize()
        out.append(bgk)
    return out


def c2_batched_block(args, P, torch, dev, local, ranks):
    """c2 as configured (1024x1024 u16 Lamb-Oseen pair, min background, 99th-percentile clip,
    deformed 64 -> 32 -> 16 px at 50 %) in the batching form, for the default run's line."""
    wl = dict(WORKLOADS["c2"])
    wl["name"] += ", deformed windows"
    a0, b0 = make_inputs(wl, seed_offset=ranks.rank)
    ring = input_ring(a0, b0)
    h, w = a0.shape
    dtype_code = P.api._dtype_code(a0)
    pairs_dev = [(torch.from_numpy(_torch_view(a)).to(dev), torch.from_numpy(_torch_view(b)).to(dev)) for a, b in ring]
    an = P.PivAnalyzer(piv_config(wl), device=local)
    pre = preprocess_config(wl)
    bgs = device_background(P, torch, an, pairs_dev[:1], dtype_code, h, w, dev)
    fa, fb = an.frame(h, w), an.frame(h, w)
    fa.prepare_device(pairs_dev[0][0].data_ptr(), dtype_code, pre, bgs[0].data_ptr())
    fb.prepare_device(pairs_dev[0][1].data_ptr(), dtype_code, pre, bgs[0].data_ptr())
    tuned = an.autotune(fa, fb) if not args.no_autotune else {}
    out = batched_figure(args, P, torch, wl, an, pre, ring, bgs[0].data_ptr(), dev, ranks)
    out["autotuned_variants"] = tuned
    an.close()
    return out


def tc_tiers_block(args, P, torch, wl, pre, pairs_dev, bg_ptrs, dtype_code, dev, local, h, w, a0, b0, ranks,
                   fp64_cache):
    """The split-precision tensor-core tiers on this workload, timed by the same device-resident
    step loop as the headline, with their error against the FP64 oracle."""
    out = {}
    for prec in ("bf16x3", "fp16x3"):
        wlp = dict(wl, precision=prec)
        loop = SlotLoop(P, torch, piv_config(wlp), pre, pairs_dev, bg_ptrs, dtype_code, dev, local, h, w)
        tuned = loop.autotune() if not args.no_autotune else {}
        for i in range(args.warmup):
            loop.step(i)
        torch.cuda.synchronize()
        steps = max(10, args.steps // 2)
        sampler = _clock_sampler(torch, dev)
        sampler.start()
        time.sleep(0.2)
        ranks.barrier()
        l0 = loop.launches()
        ms = ranks.max(loop.run(steps))
        launches = loop.launches() - l0
        clocks = sampler.stop()
        out[prec] = {"value": ranks.world * steps * loop.nvec / (ms * 1e-3), "unit": "vectors/s",
                     "ms_per_pair": ms / steps, "steps": steps, "gpu_launches": int(launches), "clocks": clocks,
                     "autotuned_variants": tuned,
                     "accuracy": accuracy_vs_fp64(wlp, a0, b0, loop.slots[0][0], cache=fp64_cache)}
        loop.close()
    return out


class SlotLoop:
    """The device-resident step loop. Two slots, each an analyzer (workspace and pass graph) with
    its own frames: the frames of step i+1 are prepared on a preparation stream while step i is
    analysed on the analysis stream, as PivPipeline does for host frames; analyses stay in order
    on one stream. Step i takes pair i % len(ring) of the device-resident ring, prepares both
    frames from its raw samples and analyses them into device buffers. Repeated calls on a slot's
    frames replay its captured pass graph."""

    def __init__(self, P, torch, cfg, pre, pairs_dev, bg_ptrs, dtype_code, dev, local, h, w):
        self.torch = torch
        self.pre, self.pairs_dev, self.bg_ptrs, self.dtype_code = pre, pairs_dev, bg_ptrs, dtype_code
        self.stream = torch.cuda.Stream(device=dev)
        self.prep_stream = torch.cuda.Stream(device=dev)
        self.slots = []
        for _ in range(2):
            an = P.PivAnalyzer(cfg, device=local)
            an.set_stream(self.stream.cuda_stream)
            self.slots.append((an, an.frame(h, w), an.frame(h, w)))
        self.prepared = [torch.cuda.Event() for _ in self.slots]
        self.analysed = [torch.cuda.Event() for _ in self.slots]
        for ev in self.analysed:
            ev.record(self.stream)
        self.nvec = len(self.slots[0][0].output_grid(h, w))
        self.out = ([torch.empty(self.nvec, device=dev, dtype=torch.float32) for _ in range(3)]
                    + [torch.empty(self.nvec, device=dev, dtype=torch.uint8),
                       torch.empty(8, device=dev, dtype=torch.int64)])

    def step(self, i):
        k = i % len(self.pairs_dev)
        ta, tb = self.pairs_dev[k]
        s_an, s_fa, s_fb = self.slots[i % 2]
        # the slot's frames are free once its previous pair has been analysed
        self.prep_stream.wait_event(self.analysed[i % 2])
        s_an.set_stream(self.prep_stream.cuda_stream)
        s_fa.prepare_device(ta.data_ptr(), self.dtype_code, self.pre, self.bg_ptrs[k])
        s_fb.prepare_device(tb.data_ptr(), self.dtype_code, self.pre, self.bg_ptrs[k])
        self.prepared[i % 2].record(self.prep_stream)
        self.stream.wait_event(self.prepared[i % 2])
        s_an.set_stream(self.stream.cuda_stream)
        s_an.analyze_device(s_fa, s_fb, *[t.data_ptr() for t in self.out])
        self.analysed[i % 2].record(self.stream)

    def autotune(self):
        """Launch-geometry (and, for the split precisions, FP32-or-tensor-core) autotuning of both
        slots on the first pair; results are identical across FP32 variants."""
        tuned = {}
        ta, tb = self.pairs_dev[0]
        for s_an, s_fa, s_fb in self.slots:
            s_fa.prepare_device(ta.data_ptr(), self.dtype_code, self.pre, self.bg_ptrs[0])
            s_fb.prepare_device(tb.data_ptr(), self.dtype_code, self.pre, self.bg_ptrs[0])
            tuned = s_an.autotune(s_fa, s_fb) or tuned
        return tuned

    def launches(self):
        return sum(s[0].launches() for s in self.slots)

    def run(self, steps):
        """`steps` steps between two events on the analysis stream (the preparation stream waits
        for the first); returns the elapsed milliseconds."""
        torch = self.torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        self.prep_stream.wait_event(e0)
        for i in range(steps):
            self.step(i)
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def pass_times(self, steps, npass):
        """The same steps with CUDA events around every correlation launch (eager launches):
        per pass, (total ms, launches) over both slots."""
        for s_an, _, _ in self.slots:
            s_an.set_profiling(True)
            for p in range(npass):
                s_an.profile(p)  # reset
        for i in range(steps):
            self.step(i)
        self.torch.cuda.synchronize()
        corr = [tuple(map(sum, zip(*(s[0].profile(p) for s in self.slots)))) for p in range(npass)]
        for s_an, _, _ in self.slots:
            s_an.set_profiling(False)
        return corr

    def close(self):
        for s_an, _, _ in self.slots:
            s_an.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c5", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="c5 at N=1: skip the tensor-core tiers, the c2 batched figure and the c4 serving run")
    ap.add_argument("--serving-s", type=float, default=10.0,
                    help="c5 at N=1: seconds of Poisson arrivals in the short c4 serving run")
    ap.add_argument("--precision", choices=["fp32", "bf16x3", "fp16x3"], default=None,
                    help="correlation arithmetic: FP32 FFTs, or split-BF16 tensor-core DFTs (16 and 32 px windows)")
    ap.add_argument("--deform", type=int, choices=[0, 1], default=None,
                    help="window deformation from the second pass on (default: the workload's setting)")
    ap.add_argument("--duration", type=float, default=None, help="serving workload: seconds of arrivals")
    ap.add_argument("--profile-case", default=None, metavar="WINDOWS",
                    help="profiler workload: analyse the workload's pair --steps times with the given comma-separated "
                         "window schedule (or 'all'), through the host API, untimed")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    wl = dict(WORKLOADS[args.workload])
    if args.deform is not None:
        wl["deform"] = bool(args.deform)
    if args.deform is not None or "deform" in WORKLOADS[args.workload]:
        wl["name"] = wl["name"] + (", deformed windows" if wl.get("deform") else ", uniform windows")
    if args.precision is not None:
        wl["precision"] = args.precision
        if args.precision != "fp32":
            wl["name"] = wl["name"].replace("FP32 plain", f"{args.precision.upper()} tensor cores where the autotuner "
                                            "finds them faster (16/32 px), FP32 elsewhere")
    if args.profile_case:
        return run_profile_case(args, wl)
    if args.impl == "reference":
        return run_reference(args, wl)
    if wl.get("stream"):
        return run_stream(args, wl)
    if wl.get("serving"):
        return run_serving(args, wl)

    import torch

    import piv_b200 as P

    from piv_b200.replicas import Ranks
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Ranks(backend="nccl", device=dev)
    rank, world = ranks.rank, ranks.world

    # ---------------------------------------------------------------- inputs (host, then device)
    a0, b0 = make_inputs(wl, seed_offset=rank)
    # a ring of shifted copies of the pair, at least 256 MiB of samples, so that the steps read
    # their inputs from HBM rather than from the 126 MB L2
    pairs_host = input_ring(a0, b0)
    n_ring = len(pairs_host)
    dtype_code = P.api._dtype_code(a0)
    h, w = a0.shape
    # raw u16 samples on the device (held as int16 tensors: same bytes)
    pairs_dev = [(torch.from_numpy(_torch_view(a)).to(dev), torch.from_numpy(_torch_view(b)).to(dev))
                 for a, b in pairs_host]

    pre = preprocess_config(wl)
    lib = P.load_library()
    import ctypes
    bg_devs, bg_ptrs, bg_hosts = [], [None] * n_ring, [None] * n_ring
    loop = SlotLoop(P, torch, piv_config(wl), pre, pairs_dev, bg_ptrs, dtype_code, dev, local, h, w)
    an, fa, fb = loop.slots[0]
    stream = loop.stream
    g = an.output_grid(h, w)
    nvec = len(g)
    if wl.get("background") == "min":
        # the background of each pair, the per-pixel minimum over its two frames
        # (BackgroundEstimator, preprocess.rs:47-72), estimated before the timed steps as the
        # reference estimates it before its pair loop
        for k, (ta, tb) in enumerate(pairs_dev):
            stack = torch.stack([ta, tb])
            bgk = torch.empty((h, w), dtype=torch.float32, device=dev)
            torch.cuda.synchronize()
            P.api._check(lib.piv_background_device(an._h, ctypes.c_void_p(stack.data_ptr()), dtype_code, 2, h, w, 0,
                                                   ctypes.c_void_p(bgk.data_ptr())))
            torch.cuda.synchronize()
            bg_devs.append(bgk)
            bg_ptrs[k] = bgk.data_ptr()
        bg_hosts = [b.cpu().numpy() for b in bg_devs[:2]] + [None] * (n_ring - 2)
    bg_ptr = bg_ptrs[0]
    tuned = loop.autotune() if not args.no_autotune else {}
    for i in range(args.warmup):
        loop.step(i)
    stream.synchronize()

    # ---------------------------------------------------------------- timed: device-resident
    npass = len(pass_windows(wl))
    ranks.barrier()
    torch.cuda.synchronize()
    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    sampler = ClockSampler(gpu_uuid if gpu_uuid.startswith("GPU-") else f"GPU-{gpu_uuid}")
    sampler.start()
    time.sleep(0.3)
    l0 = loop.launches()
    ms = loop.run(args.steps)
    torch.cuda.synchronize()
    launches = loop.launches() - l0
    clocks = sampler.stop()
    ms_max = ranks.max(ms)
    # per-pass kernel times for the roofline, from a second loop of the same steps
    corr = loop.pass_times(args.steps, npass)
    value = world * args.steps * nvec / (ms_max * 1e-3)

    # ---------------------------------------------------------------- timed: end to end (host buffers)
    pin = [(torch.from_numpy(_torch_view(a)).pin_memory().numpy().view(a.dtype),
            torch.from_numpy(_torch_view(b)).pin_memory().numpy().view(b.dtype)) for a, b in pairs_host[:2]]
    hdx = torch.empty(nvec, dtype=torch.float32).pin_memory().numpy().reshape(g.ny, g.nx)
    hdy = torch.empty(nvec, dtype=torch.float32).pin_memory().numpy().reshape(g.ny, g.nx)
    hppr = torch.empty(nvec, dtype=torch.float32).pin_memory().numpy().reshape(g.ny, g.nx)
    hfl = torch.empty(nvec, dtype=torch.uint8).pin_memory().numpy().reshape(g.ny, g.nx)
    summ = P._lib.PivSummaryC()
    pc = pre._c()
    bg_args = [None if x is None else ctypes.c_void_p(x.ctypes.data) for x in bg_hosts[:2]]

    def e2e_step(i):
        ha, hb = pin[i % len(pin)]
        for fr, hx in ((fa, ha), (fb, hb)):
            P.api._check(lib.piv_frame_prepare(an._h, fr._h, ctypes.c_void_p(hx.ctypes.data), dtype_code,
                                               ctypes.byref(pc), bg_args[i % len(pin)]))
        P.api._check(lib.piv_analyze(an._h, fa._h, fb._h, ctypes.c_void_p(hdx.ctypes.data),
                                     ctypes.c_void_p(hdy.ctypes.data), ctypes.c_void_p(hppr.ctypes.data),
                                     ctypes.c_void_p(hfl.ctypes.data), ctypes.byref(summ)))

    for i in range(args.warmup):
        e2e_step(i)
    e2e_steps = max(3, args.steps // 4)
    ranks.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    t_wall = time.perf_counter()
    for i in range(e2e_steps):
        e2e_step(i)
    e3.record(stream)
    e3.synchronize()
    t_wall = time.perf_counter() - t_wall
    ms_serial = ranks.max(e2.elapsed_time(e3))

    # pipelined: the same calls through PivPipeline (depth 3), so one pair's uploads and downloads
    # overlap the others' kernels; host clock with the device synchronised at both ends
    depth = 3
    pl = P.PivPipeline(an, h, w, dtype=a0.dtype, cfg=pre, depth=depth)
    pl.set_background(bg_ptr)  # one background image for the pipelined run (that of the first pair)
    outs = [tuple(torch.empty(nvec, dtype=dt).pin_memory().numpy().reshape(g.ny, g.nx)
                  for dt in (torch.float32, torch.float32, torch.float32, torch.uint8)) for _ in range(depth)]

    def e2e_run(n):
        tickets = []
        for i in range(n):
            if len(tickets) == depth:
                pl.wait(tickets.pop(0))
            ha, hb = pin[i % len(pin)]
            tickets.append(pl.submit(ha, hb, out=outs[i % depth]))
        for t in tickets:
            pl.wait(t)

    e2e_run(max(args.warmup, depth))
    # host-clocked: enough pairs for about half a second, so that clock jitter stays small
    pipe_steps = int(min(20000, max(12, args.steps // 2, 500.0 / max(ms_max / args.steps, 1e-3))))
    ranks.barrier()
    torch.cuda.synchronize()
    t_pipe = time.perf_counter()
    e2e_run(pipe_steps)
    torch.cuda.synchronize()
    t_pipe = time.perf_counter() - t_pipe
    ms2 = ranks.max(1e3 * t_pipe)
    pl.close()
    e2e_value = world * pipe_steps * nvec / (ms2 * 1e-3)
    h2d = sum(x.nbytes for x in pin[0])
    d2h = hdx.nbytes + hdy.nbytes + hppr.nbytes + hfl.nbytes + 5 * 8

    # ---------------------------------------------------------------- batched form (optional)
    batched = None
    if wl.get("batch_pairs"):
        batched = batched_figure(args, P, torch, wl, an, pre, pairs_host, bg_ptr, dev, ranks)

    # ---------------------------------------------------------------- roofline (correlation kernels)
    pw = pass_windows(wl)
    flops = 0.0
    kms = 0.0
    klaunch = 0
    per_pass = []
    for p, n in enumerate(pw):
        cells = len(an.pass_grid(h, w, p))
        t_ms, cnt = corr[p]
        f = cells * alg_flops(n)
        per_pass.append({"window": n, "cells": cells, "ms_per_launch": t_ms / max(cnt, 1),
                         "tflops": f / (t_ms / max(cnt, 1) * 1e-3) / 1e12 if cnt else None})
        flops += f * cnt
        kms += t_ms
        klaunch += cnt
    achieved = flops / (kms * 1e-3) / 1e12 if kms > 0 else 0.0
    peaks = measured_peaks()
    sgemm = fp32_peak_tflops(dev) if rank == 0 else None
    traffic = load_traffic(args.workload)
    roof = {"bound": "fp32", "achieved": achieved, "peak": sgemm, "unit": "TFLOP/s",
            "frac": (achieved / sgemm) if sgemm else None,
            "traffic": (traffic or {}).get("bytes_per_pair"),
            "kernel": "correlate_kernel (all passes of one pair)",
            "source": "CUDA events around each correlation launch on the analyzer's stream, over a second "
                      "loop of the same steps (the timed loop replays the pass graph)",
            "peak_source": "measured cuBLAS SGEMM (FP32 CUDA cores, TF32 off), 8192^3, in this run",
            "per_pass": per_pass,
            "hbm_peak_gbs": peaks.get("hbm_gbs")}

    vs_baseline = None
    if wl.get("published_pairs_per_s"):
        vs_baseline = value / (wl["published_pairs_per_s"] * nvec)
    line = {"metric": METRIC, "value": value, "unit": "vectors/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": vs_baseline, "dtype": "f32" if wl.get("precision", "fp32") == "fp32" else wl["precision"] + "+f32", "data": "synthetic",
            "config": workload_config(wl, pairs_host, nvec, world),
            "schedule": "two analyzer slots: the frames of pair i+1 are prepared on a second stream while pair i is "
                        "analysed; analyses in order on one stream",
            "e2e": {"value": e2e_value, "unit": "vectors/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": pipe_steps,
                    "ms_per_step": ms2 / pipe_steps,
                    "how": "PivPipeline (3 slots) over pinned host frames: upload, preparation, all passes and "
                           "download of the final field per pair; host clock, device synchronised at both ends",
                    "serial_value": world * e2e_steps * nvec / (ms_serial * 1e-3),
                    "serial_ms_per_step": ms_serial / e2e_steps,
                    "serial_wall_ms_per_step": 1e3 * t_wall / e2e_steps},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clocks, "autotuned_variants": tuned}
    if batched:
        line["batched"] = batched
    if world == 1 and not args.no_extras and args.workload == "c5":
        # the forms the metric names beside the plain FP32 path: the split-precision tensor-core
        # tiers of this workload, c2 in the batching form, and a short c4 serving run
        fp64_cache = {}
        line["accuracy"] = accuracy_vs_fp64(wl, a0, b0, an, cache=fp64_cache)
        line["tc"] = tc_tiers_block(args, P, torch, wl, pre, pairs_dev, bg_ptrs, dtype_code, dev, local, h, w, a0, b0,
                                    ranks, fp64_cache)
        line["batched"] = c2_batched_block(args, P, torch, dev, local, ranks)
        line["serving"] = serving_block(dict(WORKLOADS["c4"]), args.serving_s, local, ranks)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, a0, b0, single_s=4.0)
        if "accuracy" not in line:
            line["accuracy"] = accuracy_vs_fp64(wl, a0, b0, an)
    if rank == 0:
        print(json.dumps(line), flush=True)
    loop.close()
    ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

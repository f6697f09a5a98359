#!/usr/bin/env python
"""Benchmark: Mrays/s of the ray-casting hot path on the large plain scene.

Workload (the largest single-GPU configuration of the benchmark set):
16x16 jittered grid of UV spheres (64 rings x 128 segments, 4,128,770
triangles with the ground plane, 257 objects), four area lights with 16
samples each, path-traced GI with 2 bounces (pathlight, 1 path per camera
sample), 1920x1080, 16 camera samples per pixel, seeded synthetic geometry.
One step = one full render of that frame.  Mrays/s counts every traced ray
(primary + shadow + bounce) over the device time of the render.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun), every rank renders its own frame
replica (the path shards by frame/tile with no exchange): weak scaling,
value = all rays of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import csv
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from yafray_b200 import abi, replicas, scenes  # noqa: E402

METRIC = "Mrays/s"
HARNESS = os.path.join(ROOT, "oracle", "_ref", "yr_ref_harness")


def workload(args):
    if args.config == "small":
        sc = scenes.config_small()
        name = "small: UV sphere 16,128 tris + plane, point light, 320x240, 1 spp"
    else:
        sc = scenes.config_large(seed=args.seed, resx=args.resx, resy=args.resy, spp=args.spp, grid=args.grid)
        name = (f"large: {args.grid}x{args.grid} spheres + plane ({sc.ntris:,} tris, {len(sc.meshes)} objects), "
                f"4 area lights x16, path GI depth 2, {args.resx}x{args.resy}, {args.spp} spp")
    return sc, name


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for r in csv.reader(fh):
                if len(r) >= 9:
                    rows.append([x.strip() for x in r])
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------- CPU legs
BLOCK = 64  # threadedscene_t's block size (blockSpliter_t(resx, resy, 64))


def sample_blocks(sc, cores, target_s=15.0):
    """A stratified sample of the frame's 64x64 blocks for the CPU timing:
    the first distinct blocks of the R2 low-discrepancy sequence over the
    block grid (spread over the whole frame), about `target_s` seconds of
    work for `cores` threads (~0.9 Mrays/s per core, ~74 rays per camera
    sample on the large frame), at least one block per thread."""
    bw, bh = (sc.resx + BLOCK - 1) // BLOCK, (sc.resy + BLOCK - 1) // BLOCK
    spp = max(1, sc.render.spp)
    rays_per_block = BLOCK * BLOCK * spp * 74.0
    n = int(target_s * cores * 0.9e6 / rays_per_block)
    n = max(min(cores, bw * bh), min(n, bw * bh))
    a1, a2 = 0.7548776662466927, 0.5698402909980532   # R2 sequence (plastic number)
    seen, out, k = set(), [], 0
    while len(out) < n:
        bx = int(((0.5 + k * a1) % 1.0) * bw)
        by = int(((0.5 + k * a2) % 1.0) * bh)
        k += 1
        if (bx, by) not in seen:
            seen.add((bx, by))
            out.append((bx, by))
    return out


def reference_blocks(sc, threads, blocks, reps, timeout=1800):
    """Run the unmodified reference (oracle/_ref) on the listed 64x64 blocks
    with `threads` workers (threadedscene_t's worker loop over the block
    list); returns per-render dicts (render_s, primary, shadow, bounce)."""
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.yrs"), os.path.join(d, "o.bin")
        scenes.write_yrs(sc, sp)
        spec = ",".join(f"{bx}.{by}" for bx, by in blocks)
        cmd = [HARNESS, "render_blocks", sp, op, str(threads), spec, str(reps)]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-2000:])
        return [json.loads(line) for line in r.stdout.splitlines() if line.startswith("{")]


def sample_text(sc, blocks, thr, res):
    nb = ((sc.resx + BLOCK - 1) // BLOCK) * ((sc.resy + BLOCK - 1) // BLOCK)
    rps = (res["shadow"] + res["bounce"] + res["primary"]) / max(1, res["primary"])
    return (f"unmodified reference, {thr} worker threads running threadedscene_t's per-block render "
            f"(scene_t::render(renderArea_t&)) over {len(blocks)} of the frame's {nb} 64x64 blocks "
            f"({100.0 * len(blocks) / nb:.1f}% of the frame, stratified by the R2 sequence over the block grid, "
            f"{sc.render.spp} spp, {rps:.1f} rays per camera sample); rays counted at "
            f"scene_t::isShadowed/firstHit + camera rays in per-thread counters; render phase timed, kd build "
            f"excluded")


def cpu_baseline(sc):
    threads = host_cores()
    if os.path.exists(HARNESS):
        blocks = sample_blocks(sc, threads)
        res = reference_blocks(sc, threads, blocks, 1)[-1]
        rays = res["primary"] + res["shadow"] + res["bounce"]
        return {"value": rays / res["render_s"] / 1e6, "unit": METRIC, "cores": threads, "kind": "reference",
                "sample": sample_text(sc, blocks, threads, res),
                "blocks": [list(b) for b in blocks],
                "rays_per_sample": rays / max(1, res["primary"])}
    import yrtest as T
    O = T.OracleScene(sc)
    t0 = time.perf_counter()
    _, st = O.render(0, min(sc.resx, 64), 0, 8)
    dt = time.perf_counter() - t0
    rays = int(st[0] + st[1] + st[2])
    return {"value": rays / dt / 1e6, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"oracle port, 1 thread, pixels 64x8 of the frame ({rays:,} rays)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc, name = workload(args)
    if not os.path.exists(HARNESS):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/yr_ref_harness was not built"}))
        return
    threads = host_cores()
    blocks = sample_blocks(sc, threads, target_s=10.0)
    res = reference_blocks(sc, threads, blocks, args.warmup + args.steps)
    timed = res[args.warmup:]
    rays = sum(r["primary"] + r["shadow"] + r["bounce"] for r in timed)
    secs = sum(r["render_s"] for r in timed)
    value = rays / secs / 1e6
    sample = sample_text(sc, blocks, threads, timed[-1])
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * secs / max(1, len(timed)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "sample_blocks": len(blocks)},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ------------------------------------------------------------------ GPU leg
def load_traffic():
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return {}
    return {}


def run_diff(args, api, torch, local, fd_params=16, steps=None, warmup=None):
    """Adjoint workload: the small scene at 512x512, 64 spp, 64 material
    groups (diffuse RGB + specular weight) and 8 area lights = 264
    parameters; target rendered from hidden parameters.  One step = one
    forward render + one yr_backward.  Reports the adjoint / forward time
    ratio and a check of the gradient against FP64-accumulated central
    differences (step 1e-3) on `fd_params` sampled parameters."""
    sc = scenes.config_diff(res=args.diff_res, spp=args.diff_spp)
    hid = scenes.config_diff(res=args.diff_res, spp=args.diff_spp, hidden=True)
    ds = api.DeviceScene(sc, device=local)
    n = ds.param_count()
    theta = ds.params_get()
    dh = api.DeviceScene(hid, device=local)
    target = torch.empty((sc.resy, sc.resx, 4), dtype=torch.float32, device="cuda")
    dh.render_into(target.data_ptr())
    dh.close()
    img = torch.empty_like(target)
    grad = torch.empty(n, dtype=torch.float32, device="cuda")
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    for _ in range(warmup):
        ds.render_into(img.data_ptr())
        ds.backward(img.data_ptr(), target.data_ptr(), grad.data_ptr())
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd_ms = bwd_ms = 0.0
    rays = 0
    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(steps):
        ev[0].record()
        st = ds.render_into(img.data_ptr())
        ev[1].record()
        loss = ds.backward(img.data_ptr(), target.data_ptr(), grad.data_ptr())
        ev[2].record()
        torch.cuda.synchronize()
        fwd_ms += ev[0].elapsed_time(ev[1])
        bwd_ms += ev[1].elapsed_time(ev[2])
        rays += st.rays_primary + st.rays_shadow + st.rays_bounce
    clk = clocks.stop()
    g = grad.cpu().numpy().astype(np.float64)
    tgt = target.cpu().numpy()

    def loss64(t):
        d = t.cpu().numpy()[..., :3].astype(np.float64) - tgt[..., :3].astype(np.float64)
        return float((d * d).sum())

    rng = np.random.default_rng(0)
    idx = rng.choice(n, size=min(fd_params, n), replace=False)
    rel, fds = [], []
    for k in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[k] = np.float32(theta[k] + 1e-3)
        tm[k] = np.float32(theta[k] - 1e-3)
        ds.params_set(tp)
        ds.render_into(img.data_ptr())
        lp = loss64(img)
        ds.params_set(tm)
        ds.render_into(img.data_ptr())
        lm = loss64(img)
        fd = (lp - lm) / (float(tp[k]) - float(tm[k]))
        fds.append(fd)
        rel.append(abs(g[k] - fd) / max(abs(fd), 1e-30))
    # parameters whose gradient is ~0 (a material group the camera does not
    # see) have no meaningful relative error: report them by absolute error
    fmax = max(abs(f) for f in fds)
    big = [r for r, f in zip(rel, fds) if abs(f) > 1e-6 * fmax]
    tiny_abs = max([abs(g[k] - f) for k, f in zip(idx, fds) if abs(f) <= 1e-6 * fmax] or [0.0])
    ds.params_set(theta)
    ds.close()
    value = rays / ((fwd_ms + bwd_ms) / 1000.0) / 1e6 if fwd_ms + bwd_ms > 0 else 0.0
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": steps,
        "warmup": warmup, "ms_per_step": (fwd_ms + bwd_ms) / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": f"adjoint: small scene {args.diff_res}x{args.diff_res}, {args.diff_spp} spp, 64 "
                               f"material groups, 8 area lights, {n} parameters", "parameters": n},
        "forward_ms": fwd_ms / steps, "adjoint_ms": bwd_ms / steps,
        "adjoint_over_forward": bwd_ms / fwd_ms if fwd_ms else None, "loss": loss,
        "fd_check": {"params": [int(k) for k in idx], "max_rel_err": float(max(big)),
                     "median_rel_err": float(np.median(big)), "params_with_zero_gradient": len(rel) - len(big),
                     "max_abs_err_zero_gradient": float(tiny_abs), "max_abs_gradient": float(fmax),
                     "step": 1e-3, "accumulation": "fp64"},
        "gpu_launches": None, "clocks": clk,
    }


def run_inverse(args, api, torch, local):
    """Batched inverse problems: `inverse_count` scenes (UV sphere of 20k-500k
    triangles with an fBm-modulated albedo - 6 octaves, lacunarity 2, gain
    0.5, size U(1,8) - on a plane, one area light; 256x256, 32 spp).  Target
    images come from hidden material parameters (every shader parameter -
    albedo, specular weight, fBm amplitude and base colour - scaled by
    U(0.7,1.3)); the light is known (its power is not optimised, since only
    the product of power and albedo is visible).  Adam (lr 1e-2) runs
    `inverse_steps` steps per problem from the scene's own parameters, once
    through yr_backward_batch (all problems' forward + adjoint as one CUDA
    graph per step) and once through yr_render + yr_backward per scene.
    Reports the parameter error (over optimised parameters with a non-zero
    gradient at the start) and the wall time of both."""
    from yafray_b200 import optim
    scs = scenes.config_diffnoise(count=args.inverse_count)
    t0 = time.perf_counter()
    dss = [api.DeviceScene(sc, device=local) for sc in scs]
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(77)
    start, hidden, targets = [], [], []
    masks = []
    for d in dss:
        th = d.params_get()
        m = np.ones(th.size, bool)
        m[th.size - len(d.sc.lights):] = False  # light powers come last
        masks.append(m)
        hd = np.where(m, th * rng.uniform(0.7, 1.3, th.size), th).astype(np.float32)
        d.params_set(hd)
        t = torch.empty((d.sc.resy, d.sc.resx, 4), dtype=torch.float32, device="cuda")
        d.render_into(t.data_ptr())
        targets.append(t)
        d.params_set(th)
        start.append(th)
        hidden.append(hd)
    # identifiable parameters: non-zero gradient at the start
    ident = []
    for d, t in zip(dss, targets):
        img = torch.empty_like(t)
        d.render_into(img.data_ptr())
        g = torch.zeros(max(1, d.param_count()), dtype=torch.float32, device="cuda")
        d.backward(img.data_ptr(), t.data_ptr(), g.data_ptr())
        ident.append((g.cpu().numpy()[:d.param_count()] != 0) & masks[len(ident)])
    rays_per_step = 0
    for d in dss:
        st = d.render_into(torch.empty((d.sc.resy, d.sc.resx, 4), device="cuda").data_ptr())
        rays_per_step += 2 * (st.rays_primary + st.rays_shadow + st.rays_bounce)  # forward + adjoint recompute
    res = {}
    for mode in ("batched", "plain"):
        for d, th in zip(dss, start):
            d.params_set(th)
        params, hist, secs = optim.fit(dss, targets, steps=args.inverse_steps, lr=1e-2, batched=(mode == "batched"),
                                       masks=masks)
        errs = []
        for x, th, hd, m in zip(params, start, hidden, ident):
            e0 = np.linalg.norm((th - hd)[m])
            errs.append(float(np.linalg.norm((x - hd)[m]) / e0) if e0 > 0 else 0.0)
        res[mode] = {"seconds": secs, "ms_per_step": 1000 * secs / args.inverse_steps,
                     "param_err_rel_median": float(np.median(errs)), "param_err_rel_max": float(np.max(errs)),
                     "loss_ratio_median": float(np.median(hist[-1] / hist[0]))}
    b = res["batched"]
    value = rays_per_step * args.inverse_steps / b["seconds"] / 1e6
    h2d = sum(len(d.sc.shaders) * C.sizeof(abi.YrShaderDesc) + len(d.sc.lights) * C.sizeof(abi.YrLightDesc)
              for d in dss)
    d2h = sum(4 * (max(1, d.param_count()) + 1) for d in dss)
    ntris = sum(int(d.info().ntriangles) for d in dss)
    for d in dss:
        d.close()
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.inverse_steps,
        "warmup": 0, "ms_per_step": b["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": f"inverse: {len(dss)} problems, {ntris:,} triangles, 256x256, 32 spp, fBm albedo, "
                               f"Adam lr 1e-2 x {args.inverse_steps} steps", "scene_setup_s": round(setup_s, 2)},
        "batched": b, "plain_gpu": res["plain"],
        "speedup_vs_plain": res["plain"]["seconds"] / b["seconds"],
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "wall time of the host Adam loop: parameters up, gradients and losses down every step"},
        "gpu_launches": args.inverse_steps,
    }))


def run_batch(args, api, torch, local, barrier, steps=None, warmup=None, count=None):
    """Uneven batch: `batch_count` independent scenes (1k-200k triangles,
    1-32 objects, 64^2-512^2, 4-64 spp, 1-4 lights, GI 1-3 bounces) rendered
    as one launch (yr_render_batch: autotuned schedule, CUDA graph), with
    the plain one-scene-per-call path (yr_render per scene) timed beside it
    on the same scenes; images of both paths are compared bit for bit."""
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    scs = scenes.config_batch(count=args.batch_count if count is None else count)
    t0 = time.perf_counter()
    dss = [api.DeviceScene(sc, device=local) for sc in scs]
    setup_s = time.perf_counter() - t0
    ntris = sum(int(d.info().ntriangles) for d in dss)
    outs = [torch.empty((d.sc.resy, d.sc.resx, 4), dtype=torch.float32, device="cuda") for d in dss]
    plain = [torch.empty_like(o) for o in outs]
    ptrs = [o.data_ptr() for o in outs]
    t0 = time.perf_counter()
    st, prm = api.render_batch(dss, ptrs)   # first call autotunes and captures the graph
    tune_s = time.perf_counter() - t0
    for _ in range(max(0, warmup - 1)):
        api.render_batch(dss, ptrs)
        for d, o in zip(dss, plain):
            d.render_into(o.data_ptr())
    torch.cuda.synchronize()

    def timed(fn):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rays = 0
        for _ in range(steps):
            rays += fn()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1), rays

    def batched():
        s, _ = api.render_batch(dss, ptrs)
        return s.rays_primary + s.rays_shadow + s.rays_bounce

    def per_scene():
        r = 0
        for d, o in zip(dss, plain):
            s = d.render_into(o.data_ptr())
            r += s.rays_primary + s.rays_shadow + s.rays_bounce
        return r

    clocks = ClockSampler(local)
    clocks.start()
    ms_b, rays_b = timed(batched)
    ms_p, rays_p = timed(per_scene)
    clk = clocks.stop()
    identical = all(bool(torch.equal(a, b)) for a, b in zip(outs, plain))
    # what the batch would take if every scene ran at the rate that the
    # fastest scene reaches alone (its own device time, CUDA events inside
    # yr_render), summed over the batch
    rates, srays, sms = [], [], []
    for d, o in zip(dss, plain):
        st1 = d.render_into(o.data_ptr())
        r1 = st1.rays_primary + st1.rays_shadow + st1.rays_bounce
        srays.append(r1)
        sms.append(st1.ms)
        rates.append(r1 / max(st1.ms, 1e-6) / 1e3)  # Mrays/s
    best = max(rates)
    ideal_ms = sum(srays) / best / 1e3 * steps
    # where the per-scene path's time goes: the scenes' own device time
    # (each render alone, CUDA events inside yr_render) and what the calls
    # add around it; and how much of the device time the largest quarter
    # of the scenes (by rays) takes
    dev_ms = float(sum(sms))
    order = sorted(range(len(srays)), key=lambda i: -srays[i])
    top = order[:max(1, len(order) // 4)]
    ceiling = {"best_single_scene_value": best, "ideal_ms_per_step": ideal_ms / steps,
               "max_ratio_vs_plain": ms_p / ideal_ms,
               "note": "the batch's time if every scene ran at the rate that the fastest scene reaches alone",
               "scenes_device_ms": dev_ms, "plain_call_overhead_ms": ms_p / steps - dev_ms,
               "largest_quarter_device_share": float(sum(sms[i] for i in top)) / max(dev_ms, 1e-9),
               "largest_quarter_rays_share": float(sum(srays[i] for i in top)) / max(1.0, float(sum(srays)))}
    value = rays_b / (ms_b / 1000.0) / 1e6
    plain_value = rays_p / (ms_p / 1000.0) / 1e6
    # end to end: parameters host -> device and every image back to pinned host memory
    host = [torch.empty(o.shape, dtype=torch.float32).pin_memory() for o in outs]
    h2d = sum(len(d.sc.shaders) * C.sizeof(abi.YrShaderDesc) + len(d.sc.lights) * C.sizeof(abi.YrLightDesc)
              for d in dss)
    d2h = sum(h.numel() * 4 for h in host)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_rays = 0
    for _ in range(steps):
        for d in dss:
            d.set_params(d.sc.shaders, d.sc.lights)
        e2e_rays += batched()
        for h, o in zip(host, outs):
            h.copy_(o, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": steps,
        "warmup": warmup, "ms_per_step": ms_b / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": f"batch: {len(dss)} scenes, {ntris:,} triangles, one graph launch",
                   "schedule": {1: "tiles", 2: "waves"}.get(prm.mode, prm.mode), "streams": prm.streams,
                   "block_size": prm.block_size, "queue_tile": prm.queue_tile,
                   "stack_entries": prm.stack_entries, "autotune_s": round(tune_s, 3),
                   "scene_setup_s": round(setup_s, 3), "l2": "scene arrays and images larger than L2"},
        "plain_gpu": {"value": plain_value, "unit": METRIC, "ms_per_step": ms_p / steps,
                      "launch": "yr_render per scene"},
        "speedup_vs_plain": value / plain_value if plain_value else None,
        "identical_images": identical,
        "ceiling": ceiling,
        "e2e": {"value": e2e_rays / e2e_s / 1e6, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": steps,
        "clocks": clk,
    }
    for d in dss:
        d.close()
    return line


def run_kdbuild(args, api, local):
    """kd-trees of every mesh of the large scene (kdTree_t, kdtree.cc:57-582):
    yr_kdtree_build_gpu (host meshes in, host trees out, one call) against
    the host build on all host cores (yr_kdtree_build_ex per mesh, meshes
    spread over threads, as scene creation does); trees compared node for
    node."""
    import concurrent.futures as cf
    import ctypes as C
    import numpy as np
    from yafray_b200 import abi, scenes
    sc = scenes.config_large(seed=args.seed, resx=64, resy=64, spp=1, grid=args.grid)
    meshes = [m for m in sc.meshes if not m.is_instance]
    ntris = sum(int(m.tris.shape[0]) for m in meshes)
    for _ in range(args.warmup):
        api.kdtrees_gpu(meshes, device=local)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        g = api.kdtrees_gpu(meshes, device=local)
        times.append(time.perf_counter() - t0)
    lib = abi.load()

    def host(m):
        v = np.ascontiguousarray(m.verts, np.float32)
        t = np.ascontiguousarray(m.tris, np.uint32)
        p = C.POINTER(abi.YrKdTree)()
        abi.check(lib.yr_kdtree_build_ex(v.ctypes.data_as(C.POINTER(C.c_float)), v.shape[0],
                                         t.ctypes.data_as(C.POINTER(C.c_uint32)), t.shape[0], None, 1,
                                         C.byref(p)), "yr_kdtree_build_ex")
        tr = p.contents
        nodes = np.ctypeslib.as_array(C.cast(tr.nodes, C.POINTER(C.c_uint32)), (2 * tr.nnodes,)).copy()
        prims = np.ctypeslib.as_array(tr.prims, (max(tr.nprims, 1),))[:tr.nprims].copy()
        lib.yr_kdtree_free(p)
        return nodes, prims

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(cores) as ex:
        h = list(ex.map(host, meshes))
    host_s = time.perf_counter() - t0
    same = all(np.array_equal(a["nodes"].reshape(-1), b[0]) and np.array_equal(a["prims"], b[1])
               for a, b in zip(g, h))
    best = min(times)
    line = {
        "metric": "kd-tree build Mtriangles/s", "value": ntris / best / 1e6, "unit": "Mtriangles/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * best,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic (seeded scene generator)",
        "config": {"workload": f"kd build of the large scene's {len(meshes)} meshes ({ntris} triangles), "
                               "host meshes in, host trees out (yr_kdtree_build_gpu)",
                   "timing": "wall clock around the call (host copies, device build, trees back)"},
        "host_build": {"value": ntris / host_s / 1e6, "unit": "Mtriangles/s", "seconds": host_s, "cores": cores},
        "trees_identical": bool(same),
        "gpu_seconds": [round(t, 4) for t in times],
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="large", choices=["large", "small", "batch", "diff", "inverse", "kdbuild"])
    ap.add_argument("--inverse-count", type=int, default=32, help="problems in the inverse workload")
    ap.add_argument("--inverse-steps", type=int, default=200, help="Adam steps per problem")
    ap.add_argument("--batch-count", type=int, default=256, help="scenes in the batch workload")
    ap.add_argument("--diff-res", type=int, default=512, help="image size of the adjoint workload")
    ap.add_argument("--diff-spp", type=int, default=64, help="samples per pixel of the adjoint workload")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--resx", type=int, default=1920)
    ap.add_argument("--resy", type=int, default=1080)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--grid", type=int, default=16)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch and adjoint ratios that the default line carries")
    ap.add_argument("--exact-order", action="store_true",
                    help="exact slab tests in the object tree (reference visiting order)")
    ap.add_argument("--shadow-tree", action="store_true", help="answer shadow rays with the shadow-ray tree")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    from yafray_b200 import api
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    if args.config == "kdbuild":
        if rank == 0:
            run_kdbuild(args, api, local)
        return
    if args.config == "batch":
        print(json.dumps(run_batch(args, api, torch, local, barrier)))
        return
    if args.config == "diff":
        print(json.dumps(run_diff(args, api, torch, local)))
        return
    if args.config == "inverse":
        run_inverse(args, api, torch, local)
        return
    sc, name = workload(args)
    if args.exact_order:
        sc.render.flags |= 2
        name += ", exact object-tree order"
    if args.shadow_tree:
        sc.render.flags |= 1
        name += ", shadow-ray tree"
    t0 = time.perf_counter()
    ds = api.DeviceScene(sc, device=local)
    info = ds.info()
    build_s = time.perf_counter() - t0
    # the same kd-trees built on the GPU (yr_kdtree_build_gpu): the process's
    # first build (cold: module load, first device allocations) and a second
    # one (warm)
    meshes = [m for m in sc.meshes if not m.is_instance]
    kd_s = []
    for _ in range(2):
        t0 = time.perf_counter()
        gtrees = api.kdtrees_gpu(meshes, device=local)
        kd_s.append(time.perf_counter() - t0)
    gpu_kd_nodes = int(sum(t["nodes"].shape[0] for t in gtrees))
    del gtrees
    out = torch.empty((sc.resy, sc.resx, 4), dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        ds.render_into(out.data_ptr())
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    agg = {"rays": 0, "kms": np.zeros(abi.YR_K_COUNT), "launch": np.zeros(abi.YR_K_COUNT),
           "krays": np.zeros(abi.YR_K_COUNT), "knodes": np.zeros(abi.YR_K_COUNT), "ktests": np.zeros(abi.YR_K_COUNT)}
    for _ in range(args.steps):
        st = abi.YrRenderStats()
        st.want_kernel_stats = 1
        abi.check(ds.lib.yr_render(ds.handle, C.c_void_p(out.data_ptr()), 0, C.byref(st), C.c_void_p(0)), "yr_render")
        agg["rays"] += st.rays_primary + st.rays_shadow + st.rays_bounce
        agg["kms"] += np.array(st.kernel_ms[:])
        agg["launch"] += np.array(st.kernel_launches[:])
        agg["krays"] += np.array(st.kernel_rays[:], dtype=np.float64)
        agg["knodes"] += np.array(st.kernel_nodes[:], dtype=np.float64)
        agg["ktests"] += np.array(st.kernel_tests[:], dtype=np.float64)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max, rays_all = replicas.combine(ms, float(agg["rays"]), device="cuda")
    value = rays_all / (ms_max / 1000.0) / 1e6
    gpu_launches = int(agg["launch"].sum())

    # end to end through the C ABI: per step the shader/light parameters go
    # host -> device (yr_scene_set_params) and the image comes back to a
    # pinned host buffer (yr_render with a host destination)
    host_img = torch.empty((sc.resy, sc.resx, 4), dtype=torch.float32).pin_memory()
    h2d = len(sc.shaders) * C.sizeof(abi.YrShaderDesc) + len(sc.lights) * C.sizeof(abi.YrLightDesc)
    d2h = host_img.numel() * 4
    e2e_rays = 0
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ds.set_params(sc.shaders, sc.lights)
        st = ds.render_into(host_img.data_ptr(), on_host=True)
        e2e_rays += st.rays_primary + st.rays_shadow + st.rays_bounce
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_t, e2e_r = replicas.combine(e2e_s, float(e2e_rays), device="cuda")
    e2e_value = e2e_r / e2e_t / 1e6

    # roofline of the dominant kernel class: algorithmic bytes per ray =
    # 32 (ray) + 16 (hit / occlusion record) + 16 per node visited (the
    # reference's kdTreeNode) + 48 per triangle tested (triangle_t a,b,c,N)
    kms = agg["kms"]
    dom = int(np.argmax(kms))
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    alg_bytes = 48.0 * agg["krays"][dom] + 16.0 * agg["knodes"][dom] + 48.0 * agg["ktests"][dom]
    achieved = alg_bytes / (kms[dom] / 1000.0) / 1e9 if kms[dom] > 0 else 0.0
    launches = max(1.0, agg["launch"][dom])
    # DRAM bytes per ray of this kernel class from an ncu capture of the same
    # kernel on a smaller frame of the same scene (profiles/ncu_traffic.json),
    # scaled to the rays of an average launch here
    tinfo = load_traffic().get(abi.KERNEL_CLASSES[dom])
    traffic = (float(tinfo["dram_bytes_per_ray"]) * agg["krays"][dom] / launches
               if isinstance(tinfo, dict) and "dram_bytes_per_ray" in tinfo else None)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "traffic_source": (tinfo or {}).get("source") if isinstance(tinfo, dict) else None,
                "kernel": abi.KERNEL_CLASSES[dom],
                "bytes_per_launch": alg_bytes / launches, "ms_per_launch": kms[dom] / launches,
                "rays_per_launch": agg["krays"][dom] / launches,
                "peak_source": peak_src,
                "nodes_per_ray": agg["knodes"][dom] / max(1.0, agg["krays"][dom]),
                "tests_per_ray": agg["ktests"][dom] / max(1.0, agg["krays"][dom])}
    # the traversal is bound by instruction issue, not by HBM: the same
    # kernel against the SMs' issue rate (one warp instruction per clock per
    # sub-partition, 4 per SM), with warp instructions per ray and lanes per
    # warp instruction from the ncu capture of the kernel (profiles/)
    if isinstance(tinfo, dict) and "warp_inst_per_ray" in tinfo:
        props = __import__("torch").cuda.get_device_properties(local)
        mhz = clk.get("sm_mhz") or 1965.0
        issue_peak = props.multi_processor_count * 4 * mhz * 1e6 / 1e9   # G warp instructions/s
        rays_s = agg["krays"][dom] / (kms[dom] / 1000.0) if kms[dom] > 0 else 0.0
        achieved_issue = float(tinfo["warp_inst_per_ray"]) * rays_s / 1e9
        roofline["issue"] = {"achieved": achieved_issue, "peak": issue_peak, "unit": "G warp inst/s",
                             "frac": achieved_issue / issue_peak, "warp_inst_per_ray": tinfo["warp_inst_per_ray"],
                             "threads_per_warp_inst": tinfo.get("threads_per_warp_inst"),
                             "source": tinfo.get("issue_source")}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": name, "triangles": int(info.ntriangles), "objects": int(info.nobjects),
                   "kd_nodes": int(info.nnodes), "l2": "inputs larger than L2 (scene arrays "
                   f"{info.device_bytes / 1e6:.0f} MB on the device)",
                   "host_build_s": round(info.build_seconds, 3), "scene_setup_s": round(build_s, 3),
                   "gpu_kd_build_cold_s": round(kd_s[0], 3), "gpu_kd_build_warm_s": round(kd_s[1], 3),
                   "gpu_kd_nodes_equal": gpu_kd_nodes == int(info.nnodes),
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": gpu_launches,
        "roofline": roofline,
        "kernels_ms": {abi.KERNEL_CLASSES[k]: round(float(kms[k]), 3) for k in range(abi.YR_K_COUNT) if kms[k] > 0},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline(sc)
            line["cpu_baseline"]["frame_rays_per_sample"] = rays_all / (world * args.steps * sc.resx * sc.resy *
                                                                         sc.render.spp)
        except Exception as ex:  # the GPU number stands without it
            line["cpu_baseline"] = {"value": None, "error": str(ex)[:300]}
    ds.close()
    if world == 1 and not args.no_extras:
        # the metric's other two ratios, on their own workloads
        b = run_batch(args, api, torch, local, barrier, steps=2, warmup=2)
        line["batch"] = {"workload": b["config"]["workload"], "schedule": b["config"]["schedule"],
                         "streams": b["config"]["streams"], "value": b["value"], "unit": METRIC,
                         "plain_gpu_value": b["plain_gpu"]["value"], "ratio": b["speedup_vs_plain"],
                         "identical_images": b["identical_images"], "ms_per_step": b["ms_per_step"],
                         "plain_ms_per_step": b["plain_gpu"]["ms_per_step"], "steps": b["steps"],
                         "ceiling_ratio_vs_plain": b["ceiling"]["max_ratio_vs_plain"],
                         "ceiling": {k: b["ceiling"][k] for k in ("scenes_device_ms", "plain_call_overhead_ms",
                                                                  "largest_quarter_device_share",
                                                                  "largest_quarter_rays_share", "note")}}
        d = run_diff(args, api, torch, local, steps=3, warmup=2)
        line["adjoint"] = {"workload": d["config"]["workload"], "forward_ms": d["forward_ms"],
                           "adjoint_ms": d["adjoint_ms"], "ratio": d["adjoint_over_forward"],
                           "fd_check": d["fd_check"], "steps": d["steps"]}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

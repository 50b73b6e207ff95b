#!/usr/bin/env python
"""Render-path benchmark: panorama output Mpix/s of the B200 backend.

Workload (one step): the full-size plain-method panorama - 24 RGGB frames of
6000x4000 at 14 bits (black 512, gain U(0.7, 1.4), sigma_read 3 DN) in a 3x8
grid with 30% overlap and focal length 4500 px, giving a 35400x9600 output in
2048x2048 tiles with a 6-level seam blend.  A step demosaics the 24 CFA frames
(device resident) and renders every tile: warp + gain + coverage, exact chamfer
distance, ownership, seam DP and the multi-band compose.  Inputs (1.15 GB of
CFA) and outputs (2 GB) are far larger than the 126 MB L2, so no flush is
needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank renders its own seeded panorama (independent
objects, no data-path collective): weak scaling, value = all ranks' output
pixels / max-over-ranks time.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

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

METRIC = "Panorama output Mpix/s on 1 B200: learned vs plain blend at ≥45 dB PSNR"
UNIT = "Mpix/s"
# Used when the driver's measured peaks are absent: an earlier measurement on
# B200s of the same pool (burst GEMM 1.59 PFLOP/s; about 1.4 sustained under
# the 1 kW power cap at about 1.3 GHz).
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
        return False

    def summary(self):
        rows = []
        for ln in (self.out or "").splitlines():
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]) if parts[3] not in ("[N/A]", "") else 0.0,
                             parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        load = [r for r in rows if r[2] > 200.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i, v in enumerate(r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median([r[0] for r in load])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows), "power_w_max": max(r[2] for r in rows)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def setup_ours(cfg, rank, device, world=1, sharded=False):
    """The rank's render: with `sharded`, its share of one panorama (a
    contiguous band of tile columns balanced by area x contributors, only
    the frames its tiles need, tiles renumbered to them); otherwise a whole
    panorama of its own seed."""
    import torch

    from image360_b200 import COORDS_REFERENCE, B200ComputeBackend, RenderPlan, shard, synth
    t0 = time.time()
    if sharded:
        geo = synth.make_panorama(cfg, with_cfa=False)
        mine, need = shard.shard(geo.tiles, rank, world)
        full = synth.make_panorama(cfg, device=device, frames=need)
        pano = synth.Panorama(cfg=cfg, canvas_w=full.canvas_w, canvas_h=full.canvas_h,
                              to_canvas=full.to_canvas[need], gains=full.gains[need],
                              cfa=[full.cfa[f] for f in need], tiles=shard.local_view(geo.tiles, mine, need))
        del full
    else:
        cfg = synth.PanoConfig(**{**cfg.__dict__, "seed": cfg.seed + 1000 * rank})
        pano = synth.make_panorama(cfg, device=device)
    torch.cuda.synchronize()
    log(f"[rank {rank}] synthetic panorama {pano.canvas_w}x{pano.canvas_h}, {len(pano.cfa)} frames, "
        f"{len(pano.tiles)} tiles in {time.time() - t0:.1f}s")
    be = B200ComputeBackend()
    assert be.initialize() == 0, be.get_last_error()
    black, cm, rc, filt = synth.demosaic_params(cfg)
    cfa = [c.view(torch.int16).contiguous() for c in pano.cfa]
    rgb = [torch.empty((cfg.frame_h, cfg.frame_w, 3), dtype=torch.int16, device=device) for _ in cfa]
    outs = [torch.empty((t[3], t[2], 3), dtype=torch.int16, device=device) for t in pano.tiles]
    gains = (1.0 / pano.gains).astype(np.float32)
    frames = [(r.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for r, H, g in zip(rgb, pano.to_canvas, gains)]
    tiles = [(x, y, w, h, cs, o.data_ptr()) for (x, y, w, h, cs), o in zip(pano.tiles, outs)]
    plan = RenderPlan(frames, tiles, cfg.bands, COORDS_REFERENCE)
    return dict(cfg=cfg, pano=pano, be=be, cfa=cfa, rgb=rgb, outs=outs, plan=plan, demosaic=(black, cm, rc, filt))


def make_step(S, stream_ptr, overlap=False):
    """One step: demosaic every frame, then render the panorama.  With
    overlap=True the demosaic runs on a stream of its own and the render is
    split after its warp stage (the only stage that reads the demosaiced
    frames): step k+1's demosaic waits for step k's warp and then runs beside
    step k's remaining stages; step k+1's render waits for that demosaic."""
    import torch
    be, plan = S["be"], S["plan"]
    black, cm, rc, filt = S["demosaic"]
    w, h = S["cfg"].frame_w, S["cfg"].frame_h
    pairs = [(c.data_ptr(), r.data_ptr()) for c, r in zip(S["cfa"], S["rgb"])]

    def demosaic(sp):
        for c, r in pairs:
            if be.launch_demosaic(c, w, h, black, cm, rc, filt, r, sp) != 0:
                raise RuntimeError(be.get_last_error())

    if not overlap:
        def step():
            demosaic(stream_ptr)
            if plan.execute(stream_ptr) != 0:
                raise RuntimeError(be.get_last_error())
        return step
    dstream = torch.cuda.Stream()
    render = torch.cuda.ExternalStream(stream_ptr)
    ev_dem, ev_warp = torch.cuda.Event(), torch.cuda.Event()
    ev_warp.record(render)

    def step():
        dstream.wait_event(ev_warp)
        demosaic(dstream.cuda_stream)
        ev_dem.record(dstream)
        render.wait_event(ev_dem)
        if plan.execute_stages(0, 0, stream_ptr) != 0:
            raise RuntimeError(be.get_last_error())
        ev_warp.record(render)
        if plan.execute_stages(1, 9, stream_ptr) != 0:
            raise RuntimeError(be.get_last_error())
    return step


def _levels(w, h, bands):
    """Level dims of a tile after the band clamp of SeamBlend.cpp:457-459."""
    mb, ww, hh = 1, w, h
    while ww > 1 and hh > 1 and mb < bands:
        ww, hh, mb = (ww + 1) // 2, (hh + 1) // 2, mb + 1
    b = min(bands, max(1, mb))
    dims = [(w, h)]
    for _ in range(1, b):
        dims.append(((dims[-1][0] + 1) // 2, (dims[-1][1] + 1) // 2))
    return dims


def _sum_over_ranks(v, world, device):
    """Sum of a per-rank count over the ranks (control plane, outside the
    timed regions)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], device=device, dtype=torch.float64)
    dist.all_reduce(t)
    return int(t.item())


def _seam_tile_ms(cyc, clocks):
    mhz = clocks.get("sm_mhz") or 1965.0
    ms = cyc[cyc > 0] / (mhz * 1e3)
    if not len(ms):
        return None
    return {"tiles": int(len(ms)), "max": round(float(ms[0]), 3), "p90": round(float(np.percentile(ms, 90)), 3),
            "median": round(float(np.median(ms)), 3), "sum": round(float(ms.sum()), 2),
            "slowest": [round(float(v), 3) for v in ms[:12]]}


def stage_bytes(stats, S, fused_levels=2):
    """Algorithmic bytes per stage: the bytes each stage must move over the
    workload's tiles and contributors (item pixels, covered pixels, pyramid
    levels), counted over every item pixel.  With the fused pyramid
    (fused_levels 2) the base stage reads level 0 and writes level 2, the
    materialised stages start at level 2, and the fine stage reads the
    owners' pixels and writes the output.  With fused_levels 1 the base
    stage writes level 1, the down steps start there, the blend and collapse
    start at level 2, and the fine stage also reads level 1."""
    cfg = S["cfg"]
    npx_in = len(S["cfa"]) * cfg.frame_w * cfg.frame_h
    cov = stats["coveredItemPixels"]
    out = stats["outputPixels"]
    tiles = S["pano"].tiles
    item_px = sum(t[2] * t[3] * len(t[4]) for t in tiles)
    lo = 2 if fused_levels >= 1 else 1
    lo_down = 2 if fused_levels == 2 else 1
    base = down = bands_b = collapse = level1 = 0
    for (_, _, w, h, cs) in tiles:
        d = _levels(w, h, cfg.bands)
        n = [a * b for a, b in d]
        k = len(cs)
        if len(n) > lo_down:
            base += k * (7 * n[0] + 20 * n[lo_down])
        if fused_levels == 1 and len(n) > 1:
            level1 += k * 20 * n[1]
        for l in range(lo_down, len(n) - 1):
            down += k * 20 * (n[l] + n[l + 1])
        for l in range(lo, len(n)):
            bands_b += (k * 20 + 12) * n[l]
        for l in range(lo, len(n) - 1):
            collapse += 24 * n[l]
    return {
        "demosaic": npx_in * (2 + 6),
        # 6 B of source read and 6 B written per covered item pixel (bilinear
        # taps at about 1:1 scale read each source texel about once)
        "warp_gain_coverage": cov * 12,
        "chamfer_forward": item_px // 8 + item_px * 4,
        "chamfer_backward": item_px * 8,
        "ownership": item_px * 4 + out,
        "pyramid_base": base,
        "pyramid_down": down,
        "blend_bands": bands_b,
        "collapse": collapse,
        "fine_output": out * 13 + level1,
        "blend_total": cov * 6 + out * 6,
    }


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from image360_b200 import synth
    device = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    cfg = synth.C1 if args.scale == 1.0 else synth.scaled(synth.C1, args.scale, tile=synth.C1.tile)
    sharded = world > 1 and args.mode == "sharded"
    if sharded:
        # one panorama of 8 frame columns per rank, its tiles split into
        # contiguous column bands balanced by cost
        cfg = synth.PanoConfig(**{**cfg.__dict__, "cols": cfg.cols * world})
    net = untrained = train_info = None
    if not args.no_learned and world == 1:
        net, untrained, train_info = prepare_network(args, cfg, rank)
    S = setup_ours(cfg, rank, device, world, sharded)
    stream = torch.cuda.Stream(device=device)
    sp = stream.cuda_stream
    step = make_step(S, sp, overlap=True)
    plan = S["plan"]
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        assert plan.wait(sp) == 0, S["be"].get_last_error()
    torch.cuda.synchronize()
    # The plan's autotuner picks the band height and chamfer ring depth on
    # this workload (untimed; every setting renders the same bits).
    tuned = plan.autotune(sp) if not args.no_autotune else None
    if args.fusion is not None or args.warp_shape is not None:
        t = plan.tuning()
        assert plan.set_tuning(t["band_rows"], t["dt_slots"],
                               t["fused_levels"] if args.fusion is None else args.fusion,
                               t["warp_shape"] if args.warp_shape is None else args.warp_shape, sp) == 0
        tuned = {**(tuned or {}), **plan.tuning(), "forced": True}
    if args.chain_lag is not None:
        assert plan.set_chain_lag(args.chain_lag, sp) == 0
        tuned = {**(tuned or {}), "chain_lag": plan.chain_lag(), "forced": True}
    if args.chain_split is not None:
        assert plan.set_chain_split(args.chain_split, sp) == 0
        tuned = {**(tuned or {}), "chain_split": plan.chain_split(), "forced": True}
    torch.cuda.synchronize()
    stats = plan.stats(sp)
    stages = plan.profile(sp)
    seam_cyc = np.sort(plan.seam_tile_cycles(sp).astype(np.float64))[::-1]
    # demosaic stage timed alone with events on the launching stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    be, (black, cm, rc, filt) = S["be"], S["demosaic"]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for c, r in zip(S["cfa"], S["rgb"]):
            be.launch_demosaic(c.data_ptr(), cfg.frame_w, cfg.frame_h, black, cm, rc, filt, r.data_ptr(), sp)
        ev[1].record(stream)
    torch.cuda.synchronize()
    stages = {"demosaic": ev[0].elapsed_time(ev[1]), **stages}
    # timed region
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            t0.record(stream)
            for _ in range(args.steps):
                step()
            t1.record(stream)
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    assert plan.wait(sp) == 0, S["be"].get_last_error()
    if world > 1:
        tt = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        dist.barrier()
    out_px = stats["outputPixels"]
    ms_step = ms / args.steps
    px_total = _sum_over_ranks(out_px, world, device)
    value = px_total / 1e6 / (ms_step / 1e3)
    e2e = run_e2e(args, S, stream, world, device, tuned) if not args.no_e2e else None
    shard_loads = None
    if world > 1:
        mine = {"rank": rank, "tiles": len(S["pano"].tiles), "frames": len(S["pano"].cfa),
                "output_mpix": round(out_px / 1e6, 2), "ms_per_step": round(ms_step, 3),
                "tile_cost": sum(t[2] * t[3] * max(1, len(t[4])) for t in S["pano"].tiles)}
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        shard_loads = gathered
    if rank != 0:
        return None
    peaks, peak_kind = measured_peaks()
    sb = stage_bytes(stats, S, plan.tuning()["fused_levels"])
    blend_stages = ["chamfer_forward", "chamfer_backward", "ownership", "seam_dp", "pyramid_base", "pyramid_down",
                    "blend_bands", "collapse", "fine_output"]
    blend_ms = sum(stages[s] for s in blend_stages)
    # Dominant memory-bound kernel: the tile warp in the form the plan runs
    # (one launch per chain and execute; the seam step is a sequential
    # dynamic program, not bandwidth-bound).  Traffic per step: the ncu DRAM
    # bytes of a smaller capture of that form (profiles/<kernel>_traffic.json),
    # read bytes scaled by covered item pixels and written bytes by item pixels.
    dom = "warp_gain_coverage"
    kname = "k_warp_tiles" if plan.tuning()["warp_shape"] == 1 else "k_warp_rows"
    ach = sb[dom] / (stages[dom] / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", kname + "_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            tj = json.load(f)
        item_px = sum(t[2] * t[3] * len(t[4]) for t in S["pano"].tiles)
        traffic = int(tj["read_bytes_per_covered_item_px"] * stats["coveredItemPixels"] +
                      tj["write_bytes_per_item_px"] * item_px)
    roof = {"kernel": kname + " (" + dom + ")", "bound": "hbm", "achieved": round(ach, 1), "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": round(ach / peaks["hbm_gbs"], 4), "traffic": traffic,
            "algorithmic_bytes": sb[dom], "ms": round(stages[dom], 3),
            "peak_source": peak_kind + " (hbm_gbs, burst copy)"}
    per_stage = {}
    for k, v in stages.items():
        d = {"ms": round(v, 3)}
        if k in sb:
            d["GBps"] = round(sb[k] / (v / 1e3) / 1e9, 1)
            d["frac"] = round(d["GBps"] / peaks["hbm_gbs"], 4)
        per_stage[k] = d
    per_stage["blend_total"] = {"ms": round(blend_ms, 3), "GBps": round(sb["blend_total"] / (blend_ms / 1e3) / 1e9, 1),
                                "frac": round(sb["blend_total"] / (blend_ms / 1e3) / 1e9 / peaks["hbm_gbs"], 4)}
    launches = (len(S["cfa"]) + stats["kernelsPerExecute"]) * args.steps
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16 storage / fp32 arithmetic", "data": "synthetic (seeded scene, 14-bit RGGB)",
        "config": {"workload": f"plain seam blend, 24 x {cfg.frame_w}x{cfg.frame_h} RGGB -> "
                               f"{S['pano'].canvas_w}x{S['pano'].canvas_h} in {cfg.tile}^2 tiles, {cfg.bands} bands",
                   "tiles": stats["numTiles"], "tile_contributors": stats["numItems"],
                   "item_pixels": sum(t[2] * t[3] * len(t[4]) for t in S["pano"].tiles),
                   "covered_item_pixels": stats["coveredItemPixels"],
                   "output_mpix": round(out_px / 1e6, 2), "coords": "reference (bit-exact vs CPU backend)",
                   "l2": "inputs and outputs larger than L2 (no flush)",
                   "blend": "plain seam blend (--no-learned: learned blend not measured in this run)",
                   "parallelism": (f"{world} ranks, one panorama of {cfg.rows}x{cfg.cols} frames, tiles split by "
                                   f"contiguous tile-column bands balanced on area x contributors, no data-path collective" if sharded else
                                   f"{world} independent panoramas" if world > 1 else "1 GPU"),
                   "schedule": "steps back to back: step k+1's demosaic (own stream) overlaps stages 1-9 of step "
                               "k's render, after its warp stage has read the frames",
                   "autotuned": tuned},
        "roofline": roof, "stages": per_stage, "gpu_launches": launches,
        # SM cycles of the seam kernel's five phases (crossover scan, colour
        # cost, DP, backtrack, reassign), summed over tiles, pairs and every
        # execution of the plan since it was built (autotuning included).
        "seam_phase_cycles_cumulative": stats["seamPhaseCycles"],
        "clocks": clk.summary(),
        # the seam step's SM cycles per tile (last execution), slowest first,
        # as ms at the sampled SM clock: the stage lasts as long as its
        # slowest tile, which the chain split schedules first
        "seam_tile_ms": _seam_tile_ms(seam_cyc, clk.summary()),
        "e2e": e2e,
    }
    if shard_loads is not None:
        line["shards"] = shard_loads
    if net is not None:
        lr = run_learned(args, S, stream, net, untrained, train_info)
        lr["speedup_vs_plain"] = round(lr["value"] / value * world, 3)
        lr["speedup_vs_plain_with_fallback"] = round(lr["with_fallback"]["value"] / value * world, 3)
        lr["speedup_vs_plain_with_judge"] = round(lr["with_judge"]["value"] / value, 3)
        line["learned"] = lr
        line["config"]["blend"] = ("plain seam blend (value); learned blend measured in 'learned' "
                                   "(same frames, 256x256 overlap windows, judged per window at 45 dB)")
    if world > 1:
        return line  # the secondary legs and the CPU checks run at N = 1 only
    if not args.no_color:
        line["color_correct"] = run_color(args, S, stream)
    if not args.no_export:
        line["export_preview"] = run_export(args, S, stream)
    if not args.no_uneven:
        line["uneven_tiles"] = run_uneven(args, S, stream)
    if not args.no_stack:
        line["median_stack"] = run_stack(args, device, stream)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(S, args)
    if not args.no_parity:
        line["parity"] = parity_check(S, sp)
    if not args.no_native:
        line["native_fp16"] = run_native(args, S, stream, step)
    return line


def run_native(args, S, stream, step):
    """The native mode of the same step: the render's stored pyramid levels in
    FP16 (FP32 arithmetic), timed like the headline, and its error against
    the FP64 restatement of the blend (the oracle's compose in FP64 on the
    same warped contributors and owner map) on two seeded tiles with several
    contributors.  The plan goes back to the exact mode afterwards."""
    import torch

    import oracle
    from image360_b200 import PRECISION_EXACT, PRECISION_FP16, synth
    plan, pano, cfg = S["plan"], S["pano"], S["cfg"]
    sp = stream.cuda_stream
    exact_tuning = plan.tuning()
    assert plan.set_precision(PRECISION_FP16, sp) == 0
    # the autotuner again in this mode (untimed): FP16 storage changes the
    # stored levels' traffic, so the fastest fusion depth may differ
    tuned = plan.autotune(sp) if not args.no_autotune else plan.tuning()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
    torch.cuda.synchronize()
    assert plan.wait(sp) == 0
    ms = t0.elapsed_time(t1) / args.steps
    stages = plan.profile(sp)
    O = oracle.oracle()
    rng = np.random.default_rng(9)
    multi = [i for i, t in enumerate(pano.tiles) if len(t[4]) >= 3] or list(range(len(pano.tiles)))
    pick = sorted(int(i) for i in rng.permutation(multi)[:2])
    gains = (1.0 / pano.gains).astype(np.float32)
    errs = []
    for i in pick:
        x, y, w, h, cs = pano.tiles[i]
        got = S["outs"][i].cpu().numpy().view(np.uint16)
        bufs = [O.gain(O.warp(S["rgb"][k].cpu().numpy().view(np.uint16), w, h,
                              synth.inverse_homography_f32(pano.to_canvas[k]), x, y), gains[k]) for k in cs]
        _, owner = O.blend(bufs, cfg.bands, return_owner=True)
        ref = O.compose(bufs, None, owner, cfg.bands, f64=True)
        d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
        errs.append((int(d.max()), float(d.mean())))
    assert plan.set_precision(PRECISION_EXACT, sp) == 0
    t = exact_tuning
    assert plan.set_tuning(t["band_rows"], t["dt_slots"], t["fused_levels"], t["warp_shape"], sp) == 0
    with torch.cuda.stream(stream):
        assert plan.execute(sp) == 0 and plan.wait(sp) == 0
    torch.cuda.synchronize()
    out_px = sum(t[2] * t[3] for t in pano.tiles)
    lo = 2 if tuned["fused_levels"] == 2 else 1
    return {"value": round(out_px / 1e6 / (ms / 1e3), 2), "unit": UNIT, "ms_per_step": round(ms, 3),
            "autotuned": tuned,
            "storage": f"pyramid levels >= {lo} in FP16 (num / 256, den, weight), FP32 arithmetic; warped pixels u16",
            "stages_ms": {k: round(v, 3) for k, v in stages.items()},
            "error_vs_fp64": {"tiles": [pano.tiles[i][:4] for i in pick], "max_dn": max(e[0] for e in errs),
                              "mean_dn": round(float(np.mean([e[1] for e in errs])), 5),
                              "reference": "oracle FP64 compose on the same warped contributors and owner map"}}


def parity_check(S, sp):
    """Every tile of the benchmarked panorama (the plan's own outputs after
    the timed steps) against the reference's CPU code run here on the same
    demosaiced frames: warp + gain + seam blend of each tile as
    RenderExecutor does it (RenderExecutor.cpp:101-140), scalar tier, on the
    host threads.  Outside the timed region."""
    import torch

    from image360_b200 import synth
    plan, pano, cfg = S["plan"], S["pano"], S["cfg"]
    with torch.cuda.stream(torch.cuda.ExternalStream(sp)):
        assert plan.execute(sp) == 0 and plan.wait(sp) == 0
    torch.cuda.synchronize()
    impl, kind = _cpu_impl()
    threads = _cpu_threads()
    frames = [r.cpu().numpy().view(np.uint16) for r in S["rgb"]]
    gains = (1.0 / pano.gains).astype(np.float32)
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    t0 = time.time()
    if kind == "reference":
        _, ref = impl.render_tiles(threads, frames, inv, gains, pano.tiles, cfg.bands, tier=0)
    else:
        _, ref = impl.render_tiles(threads, frames, inv, gains, pano.tiles, cfg.bands)
    secs = time.time() - t0
    bad, worst = 0, 0
    for o, r in zip(S["outs"], ref):
        got = o.cpu().numpy().view(np.uint16)
        if not np.array_equal(got, r):
            bad += 1
            worst = max(worst, int(np.abs(got.astype(np.int32) - r.astype(np.int32)).max()))
    return {"checked": f"all {len(ref)} tiles vs the reference's CPU code ({kind}, scalar tier) on the same frames",
            "exact": bad == 0, "tiles_differing": bad, "max_abs_diff": worst, "cpu_seconds": round(secs, 1)}


def prepare_network(args, cfg, rank):
    """Trains the blend network on the GPU (own kernels) on seeded panoramas
    of the benchmark's configuration other than the benchmarked one, or loads
    weights given with --weights; also makes the untrained network."""
    import torch

    from image360_b200 import blendnet as bn, learned
    t0 = time.time()
    if args.weights:
        net = bn.BlendNet(seed=1)
        net.set_params(np.fromfile(args.weights, np.float32))
        info = {"weights": os.path.basename(args.weights)}
    else:
        base = synth_cfg_for_training(cfg, rank)
        net = learned.train_on_scenes(base, args.train_scenes, args.train_steps, args.train_batch, 1e-3, seed=1 + rank,
                                      log=log)
        info = {"scenes": args.train_scenes, "steps": args.train_steps, "batch": args.train_batch, "lr": 1e-3,
                "windows": args.train_steps * args.train_batch, "optimizer": "adam",
                "target": "plain 6-level seam blend of the same window", "seconds": round(time.time() - t0, 1)}
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return net, bn.BlendNet(seed=2), info


def synth_cfg_for_training(cfg, rank):
    from image360_b200 import synth
    return synth.PanoConfig(**{**cfg.__dict__, "seed": cfg.seed + 1000 * rank})


def network_flops_per_px() -> float:
    """Algorithmic FLOPs of the blend network per window pixel (2 * 9 * cin *
    cout per layer, half-resolution layers at a quarter of the pixels)."""
    from image360_b200 import blendnet as bn
    area = [1, 1, 0.25, 0.25, 0.25, 1, 1, 1]
    return sum(2.0 * 9 * ci * co * a for (ci, co), a in zip(bn.LAYERS, area))


def run_learned(args, S, stream, net, untrained, train_info):
    """The learned form of the same step (demosaic + warp + per-window network
    or copy), its per-window judge against the plain blend just rendered, the
    cost of the fallback, and the same judge for the untrained network (the
    coverage-weighted mean, i.e. the method without learning)."""
    import torch

    from image360_b200 import RenderPlan, COORDS_REFERENCE, learned
    sp = stream.cuda_stream
    cfg, be, plan = S["cfg"], S["be"], S["plan"]
    black, cm, rc, filt = S["demosaic"]
    render = learned.PanoramaRender.__new__(learned.PanoramaRender)  # view over the bench's own scene
    render.cfg, render.pano, render.be, render.plan = cfg, S["pano"], be, plan
    render.cfa, render.rgb, render.outs, render.demosaic_args, render._items = S["cfa"], S["rgb"], S["outs"], \
        S["demosaic"], None
    louts = [torch.empty_like(o) for o in S["outs"]]

    def step():
        for c, r in zip(S["cfa"], S["rgb"]):
            be.launch_demosaic(c.data_ptr(), cfg.frame_w, cfg.frame_h, black, cm, rc, filt, r.data_ptr(), sp)
        render.learned(net, louts, args.learned_batch, stream=sp)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
    torch.cuda.synchronize()
    ms_step = t0.elapsed_time(t1) / args.steps
    stages = render.learned(net, louts, args.learned_batch, stream=sp)
    # the plan's own outputs hold the plain blend of the same frames
    with torch.cuda.stream(stream):
        assert plan.execute(sp) == 0 and plan.wait(sp) == 0
    torch.cuda.synchronize()
    peak = learned.white_level(cfg)
    st, ps = render.judge(louts, 45.0, peak, stream=sp)
    fin = ps[np.isfinite(ps)]
    # The complete learned form: the step above, the plain blend of the same
    # warped frames (stages 1-9 of the plan: the judge's reference) and the
    # judge, which replaces every window below 45 dB with the plain blend.
    with torch.cuda.stream(stream):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            step()
            assert plan.execute_stages(1, 9, sp) == 0
            render.judge(louts, 45.0, peak, stream=sp)
        b.record(stream)
    torch.cuda.synchronize()
    ms_judged = a.elapsed_time(b) / args.steps
    win = render.windows()
    kind = win[:, 3]
    # fallback cost: the plain blend of every tile holding a failing window
    fb_tiles = sorted({int(t) for t, ok in zip(win[:, 0], ps >= 45.0) if not ok})
    fb_ms = 0.0
    if fb_tiles:
        sub_outs = [torch.empty_like(S["outs"][t]) for t in fb_tiles]
        frames = [(r.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g))
                  for r, H, g in zip(S["rgb"], S["pano"].to_canvas, (1.0 / S["pano"].gains).astype(np.float32))]
        tiles = [(*S["pano"].tiles[t][:5], o.data_ptr()) for t, o in zip(fb_tiles, sub_outs)]
        sub = RenderPlan(frames, tiles, cfg.bands, COORDS_REFERENCE)
        with torch.cuda.stream(stream):
            for _ in range(2):
                sub.execute(sp)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                sub.execute(sp)
            b.record(stream)
        torch.cuda.synchronize()
        assert sub.wait(sp) == 0
        fb_ms = a.elapsed_time(b) / args.steps
        sub.close()
    # the method without learning: the untrained network's head
    untr = None
    if untrained is not None:
        uouts = [torch.empty_like(o) for o in S["outs"]]
        render.learned(untrained, uouts, args.learned_batch, stream=sp)
        ust, ups = render.judge(uouts, 45.0, peak, stream=sp)
        untr = {"fallback_windows": ust["fallbackSubTiles"], **_by_kind(ups, kind, "network_windows")}
        del uouts
    out_px = sum(t[2] * t[3] for t in S["pano"].tiles)
    net_px = st["netSubTiles"] * learned.WINDOW * learned.WINDOW
    flops = net_px * network_flops_per_px()
    tfl = flops / (stages["network"] / 1e3) / 1e12
    peaks, peak_kind = measured_peaks()
    res = {
        "value": round(out_px / 1e6 / (ms_step / 1e3), 2), "unit": UNIT, "ms_per_step": round(ms_step, 3),
        "with_judge": {"value": round(out_px / 1e6 / (ms_judged / 1e3), 2), "ms_per_step": round(ms_judged, 3),
                       "what": "network step + plain blend of every tile (the judge's reference) + judge and "
                               "per-window fallback"},
        "with_fallback": {"value": round(out_px / 1e6 / ((ms_step + fb_ms) / 1e3), 2),
                          "ms_per_step": round(ms_step + fb_ms, 3), "fallback_ms": round(fb_ms, 3),
                          "fallback_tiles": len(fb_tiles)},
        "stages_ms": {k: round(v, 3) for k, v in stages.items()},
        "network": {"windows": st["netSubTiles"], "window": learned.WINDOW, "gflop": round(flops / 1e9, 1),
                    "tflops": round(tfl, 1), "bound": "tensor",
                    "peak": peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"]), "unit": "TFLOP/s",
                    "frac": round(tfl / peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"]), 4),
                    "peak_source": peak_kind + " (bf16_tflops_sustained: the network runs inside a long step)"},
        "windows": {k: st[k] for k in ("subTiles", "netSubTiles", "copySubTiles", "emptySubTiles", "overflowSubTiles")},
        "judge": {"threshold_db": 45.0, "peak_dn": peak, "fallback_windows": st["fallbackSubTiles"],
                  "min_psnr_db": round(st["minPsnr"], 2), "mean_psnr_db": round(st["meanPsnr"], 2),
                  "p1_psnr_db": round(float(np.percentile(fin, 1)), 2), "p5_psnr_db": round(float(np.percentile(fin, 5)), 2),
                  "median_psnr_db": round(float(np.median(fin)), 2), "max_abs_error": st["maxAbsError"],
                  "windows_at_or_above_45db": round(float(np.mean(ps >= 45.0)), 4),
                  "network_windows": _by_kind(ps, kind, None)["network_windows"],
                  "copy_windows": _by_kind(ps, kind, None, 1)["copy_windows"]},
        "untrained_head": untr, "train": train_info,
    }
    del louts
    return res


def _by_kind(ps, kind, key, k=2):
    """PSNR summary of the windows of one kind (2 network, 1 copy)."""
    name = {2: "network_windows", 1: "copy_windows"}[k]
    sel = ps[kind == k]
    fin = sel[np.isfinite(sel)]
    d = {"count": int(sel.size), "below_45db": int(np.sum(sel < 45.0)),
         "mean_psnr_db": round(float(fin.mean()), 2) if fin.size else None,
         "p1_psnr_db": round(float(np.percentile(fin, 1)), 2) if fin.size else None,
         "p5_psnr_db": round(float(np.percentile(fin, 5)), 2) if fin.size else None,
         "median_psnr_db": round(float(np.median(fin)), 2) if fin.size else None}
    return {name: d} if key is None else {key: d}


def run_e2e(args, S, stream, world, device, tuned=None):
    """The step end to end through the public API with HOST buffers: the
    pipelined render executor (i360b_pipeline_*) takes each step's pinned CFA
    frames, uploads them, demosaics, renders every tile and downloads every
    tile output into pinned host memory; two device slots let one step's
    download, the next step's render and the one after's upload overlap.
    Timed on the device from the first upload to the last download of K
    steps.  The serial form (copies and compute on one stream, no overlap) is
    reported beside it."""
    import torch

    from image360_b200 import COORDS_REFERENCE, RenderPipeline
    cfg, pano = S["cfg"], S["pano"]
    host_cfa = [c.cpu().pin_memory() for c in S["cfa"]]
    host_out = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in S["outs"]]
    h2d = sum(c.numel() * 2 for c in host_cfa)
    d2h = sum(o.numel() * 2 for o in host_out)
    px = sum(o.shape[0] * o.shape[1] for o in S["outs"])
    gains = (1.0 / pano.gains).astype(np.float32)
    pipe = RenderPipeline(cfg.frame_w, cfg.frame_h, pano.to_canvas, gains, S["demosaic"], pano.tiles, cfg.bands,
                          COORDS_REFERENCE, depth=2)
    cfa_ptrs = [c.data_ptr() for c in host_cfa]
    out_ptrs = [o.data_ptr() for o in host_out]
    for _ in range(max(2, args.warmup)):
        assert pipe.submit(cfa_ptrs, out_ptrs) == 0, S["be"].get_last_error()
    assert pipe.wait()[0] == 0, S["be"].get_last_error()
    pipe_tuned = pipe.autotune() if tuned is not None else None
    for _ in range(2):
        assert pipe.submit(cfa_ptrs, out_ptrs) == 0
    assert pipe.wait()[0] == 0
    # at least 10 steps: the first upload and the last download cannot overlap
    # anything, and this amortises them as a stream of panoramas would
    k = max(args.steps, 10)
    with ClockSampler(int(str(device).split(":")[-1]) if ":" in str(device) else 0) as clk:
        for _ in range(k):
            assert pipe.submit(cfa_ptrs, out_ptrs) == 0, S["be"].get_last_error()
        rc, ms_total = pipe.wait()
    assert rc == 0, S["be"].get_last_error()
    pipe.close()
    ms = ms_total / k
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    serial = run_e2e_serial(args, S, stream, world, device, host_cfa, host_out)
    px_total = _sum_over_ranks(px, world, device)
    return {"value": round(px_total / 1e6 / (ms / 1e3), 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": round(ms, 3), "steps": k,
            "api": "i360b_pipeline_submit/wait, 2 device slots, pinned host buffers", "autotuned": pipe_tuned,
            "clocks": clk.summary(), "serial": serial}


def run_e2e_serial(args, S, stream, world, device, host_cfa, host_out):
    """Copies in, demosaic + render, copies out, all on one stream (no overlap)."""
    import torch
    sp = stream.cuda_stream
    step = make_step(S, sp)

    def e2e_step():
        for hc, dc in zip(host_cfa, S["cfa"]):
            dc.copy_(hc, non_blocking=True)
        step()
        for ho, do in zip(host_out, S["outs"]):
            ho.copy_(do, non_blocking=True)

    with torch.cuda.stream(stream):
        for _ in range(max(1, args.warmup // 2)):
            e2e_step()
    torch.cuda.synchronize()
    k = max(1, min(args.steps, 3))
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        t0.record(stream)
        for _ in range(k):
            e2e_step()
        t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / k
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], device=device, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    px = _sum_over_ranks(sum(o.shape[0] * o.shape[1] for o in S["outs"]), world, device)
    return {"value": round(px / 1e6 / (ms / 1e3), 2), "unit": UNIT, "ms_per_step": round(ms, 3)}


# ---------------------------------------------------------------------------
# CPU side: the reference's own CPU code (oracle/_ref) or the C restatement
# ---------------------------------------------------------------------------
def _cpu_impl():
    import oracle
    oracle.build()
    r = oracle.reference()
    if r is not None:
        return r, "reference"
    return oracle.oracle(), "port"


def cpu_demosaic_all(impl, kind, cfa_host, cfg, threads):
    from image360_b200 import synth
    black, cm, rc, filt = synth.demosaic_params(cfg)
    if kind != "reference":
        return [impl.demosaic(c, black, cm, rc, filt) for c in cfa_host]
    import ctypes as ct
    import oracle
    outs = [np.zeros((cfg.frame_h, cfg.frame_w, 3), np.uint16) for _ in cfa_host]
    impl.lib.ref_demosaic_frames(threads, impl.tier, len(cfa_host), oracle._ptr_array(cfa_host, ct.c_uint16),
                                 cfg.frame_w, cfg.frame_h, ct.c_uint16(black), cm.ctypes.data_as(oracle._f32p),
                                 rc.reshape(12).ctypes.data_as(oracle._f32p), ct.c_uint32(filt),
                                 oracle._ptr_array(outs, ct.c_uint16))
    return outs


def cpu_sample(impl, kind, frames_host, pano, cfg, threads, n_tiles, cfa_host, gains, seed=7):
    """One bounded sample of the job on the host cores, timed as it runs (no
    extrapolation): the demosaic of the frames in proportion to the sampled
    tiles (frames / tiles of the panorama), then n_tiles tiles chosen with
    `seed`, rendered as the reference's CPU backend does (one chunk task per
    worker thread: warp + gain of every contributor, seam blend).  Returns
    (output pixels of the sampled tiles, seconds, description)."""
    from image360_b200 import synth
    black, cm, rc, filt = synth.demosaic_params(cfg)
    rng = np.random.default_rng(seed)
    n_dem = max(1, int(round(len(cfa_host) * n_tiles / len(pano.tiles))))
    idx = [int(i) for i in rng.permutation(len(cfa_host))[:n_dem]]
    order = rng.permutation(len(pano.tiles))[:n_tiles]
    sample = [pano.tiles[i] for i in order]
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    t0 = time.time()
    if kind == "reference":
        import ctypes as ct
        import oracle
        outs = [np.zeros((cfg.frame_h, cfg.frame_w, 3), np.uint16) for _ in idx]
        cptr = oracle._ptr_array([cfa_host[i] for i in idx], ct.c_uint16)
        optr = oracle._ptr_array(outs, ct.c_uint16)
        impl.lib.ref_demosaic_frames(threads, impl.tier, len(idx), cptr, cfg.frame_w, cfg.frame_h, ct.c_uint16(black),
                                     cm.ctypes.data_as(oracle._f32p), rc.reshape(12).ctypes.data_as(oracle._f32p),
                                     ct.c_uint32(filt), optr)
    else:
        for i in idx:
            impl.demosaic(cfa_host[i], black, cm, rc, filt)
    t_dem = time.time() - t0
    secs, _ = impl.render_tiles(threads, frames_host, inv, gains, sample, cfg.bands, want_out=False)
    px = sum(t[2] * t[3] for t in sample)
    return px, t_dem + secs, (f"{len(idx)} of {len(cfa_host)} frames demosaiced + {len(sample)} of {len(pano.tiles)} "
                              f"tiles rendered on {threads} threads (frames in proportion to the tiles), timed as run")


def _cpu_threads():
    """hardware_concurrency()-1 worker threads: the reference's CPU-backend
    task window (ComputeBackendFactory.cpp:99-100)."""
    return max(1, (os.cpu_count() or 2) - 1)


def cpu_baseline(S, args):
    impl, kind = _cpu_impl()
    threads = _cpu_threads()
    cfg, pano = S["cfg"], S["pano"]
    frames_host = [r.cpu().numpy().view(np.uint16) for r in S["rgb"]]
    cfa_host = [c.cpu().numpy().view(np.uint16) for c in S["cfa"]]
    gains = (1.0 / pano.gains).astype(np.float32)
    n_tiles = max(threads, args.cpu_tiles)
    px, secs, desc = cpu_sample(impl, kind, frames_host, pano, cfg, threads, n_tiles, cfa_host, gains)
    return {"value": round(px / 1e6 / secs, 3), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": desc, "sample_seconds": round(secs, 1), "threads_model": "hardware_concurrency()-1 tasks"}


def run_uneven(args, S, stream):
    """The batched uneven-tile workload: 256 output tiles with sides drawn from
    {512, 768, 1024, 1536, 2048}, each overlapped by 1-7 placements of frames
    from the step's pool of 24 demosaiced 6000x4000 frames, 6 bands, rendered
    by one plan (every stage one launch over all tiles, replayed as a CUDA
    graph) with the autotuned band height, ring depth and level-fusion depth.
    Timed with CUDA events on the stream; a seeded sample of 16 tiles is
    checked bit for bit against the reference's CPU code."""
    import torch

    from image360_b200 import COORDS_REFERENCE, RenderPlan, synth
    cfg, pano = S["cfg"], S["pano"]
    sp = stream.cuda_stream
    n = 256 if args.scale == 1.0 else max(8, int(256 * args.scale))
    sides = synth.C3_SIDES if args.scale == 1.0 else tuple(max(16, int(v * args.scale)) for v in synth.C3_SIDES)
    ut = synth.uneven_tiles(n, len(S["rgb"]), cfg.frame_w, cfg.frame_h, cfg.focal, seed=20260711, sides=sides)
    gains = (1.0 / pano.gains[ut.frame_of]).astype(np.float32)
    outs = [torch.empty((t[3], t[2], 3), dtype=torch.int16, device=S["rgb"][0].device) for t in ut.tiles]
    frames = [(S["rgb"][f].data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g))
              for f, H, g in zip(ut.frame_of, ut.to_canvas, gains)]
    plan = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(ut.tiles, outs)], 6, COORDS_REFERENCE)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            assert plan.execute(sp) == 0
        assert plan.wait(sp) == 0
    tuned = plan.autotune(sp) if not args.no_autotune else plan.tuning()
    stats = plan.stats(sp)
    stages = plan.profile(sp)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for _ in range(args.steps):
            assert plan.execute(sp) == 0
        ev[1].record(stream)
    torch.cuda.synchronize()
    assert plan.wait(sp) == 0
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    px = stats["outputPixels"]
    peaks, kind = measured_peaks()
    blend_ms = sum(v for k, v in stages.items() if k != "warp_gain_coverage")
    blend_bytes = stats["coveredItemPixels"] * 6 + px * 6
    res = {"value": round(px / 1e6 / (ms / 1e3), 1), "unit": "output Mpix/s", "ms_per_step": round(ms, 3),
           "steps": args.steps, "tiles": len(ut.tiles), "tile_contributors": stats["numItems"],
           "output_mpix": round(px / 1e6, 1), "covered_item_pixels": stats["coveredItemPixels"],
           "gpu_launches_per_step": stats["kernelsPerExecute"], "autotuned": tuned,
           "stages_ms": {k: round(v, 3) for k, v in stages.items()},
           "blend_roofline": {"achieved": round(blend_bytes / (blend_ms / 1e3) / 1e9, 1), "peak": peaks["hbm_gbs"],
                              "unit": "GB/s", "frac": round(blend_bytes / (blend_ms / 1e3) / 1e9 / peaks["hbm_gbs"], 4),
                              "algorithmic_bytes": blend_bytes,
                              "bytes_formula": "sum of covered item pixels * 6 + output pixels * 6",
                              "peak_source": kind + " (hbm_gbs, burst copy)"}}
    if not args.no_parity:
        impl, ikind = _cpu_impl()
        rng = np.random.default_rng(5)
        pick = sorted(int(i) for i in rng.permutation(len(ut.tiles))[:16])
        host = {f: S["rgb"][f].cpu().numpy().view(np.uint16) for f in sorted(set(int(f) for f in ut.frame_of))}
        fr = [host[int(f)] for f in ut.frame_of]
        inv = np.stack([synth.inverse_homography_f32(H) for H in ut.to_canvas])
        sub = [ut.tiles[i] for i in pick]
        if ikind == "reference":
            _, ref = impl.render_tiles(_cpu_threads(), fr, inv, gains, sub, 6, tier=0)
        else:
            _, ref = impl.render_tiles(_cpu_threads(), fr, inv, gains, sub, 6)
        bad = sum(not np.array_equal(outs[i].cpu().numpy().view(np.uint16), r) for i, r in zip(pick, ref))
        res["parity"] = {"checked": f"{len(pick)} seeded tiles vs the reference's CPU code ({ikind}, scalar tier)",
                         "exact": bad == 0, "tiles_differing": int(bad)}
    plan.close()
    return res


def run_stack(args, device, stream):
    """The median-stack workload: 16 RGGB frames of 4000x3000 (14-bit, one
    scene, near-identity homographies: translation U(-3, 3) px, rotation
    +-0.2 degrees, 5% of each frame's pixels under white outlier rectangles).
    A step demosaics the 16 frames and makes the per-pixel sigma-clipped
    median of the frames warped onto the reference grid, with the fused
    warp + median kernel (the warped frames are never written).  Timed with
    CUDA events; the result is checked outside the timed region against the
    reference's CPU code on the full stack (demosaic, WarpPerspective of
    every frame, MedianStack), which is also timed as the CPU baseline."""
    import torch

    from image360_b200 import synth
    cfg = synth.C2 if args.scale == 1.0 else synth.scaled_stack(synth.C2, args.scale)
    t0 = time.time()
    st = synth.make_stack(cfg, device=device)
    torch.cuda.synchronize()
    log(f"burst of {cfg.frames} frames {cfg.frame_w}x{cfg.frame_h} in {time.time() - t0:.1f}s, "
        f"outliers {np.mean(st.outlier_frac):.3f}")
    be = _backend()
    black, cm, rc, filt = synth.demosaic_params(cfg)
    w, h, n = cfg.frame_w, cfg.frame_h, cfg.frames
    cfa = [c.view(torch.int16).contiguous() for c in st.cfa]
    rgb = [torch.empty((h, w, 3), dtype=torch.int16, device=device) for _ in cfa]
    out = torch.empty((h, w, 3), dtype=torch.int16, device=device)
    Hs = np.stack([synth.inverse_homography_f32(H) for H in st.to_ref])
    sp = stream.cuda_stream
    rptr = [r.data_ptr() for r in rgb]

    def demosaic():
        for c, r in zip(cfa, rgb):
            if be.launch_demosaic(c.data_ptr(), w, h, black, cm, rc, filt, r.data_ptr(), sp) != 0:
                raise RuntimeError(be.get_last_error())

    def median():
        if be.launch_warp_median(rptr, w, h, Hs, out.data_ptr(), w, h, 0, 0, 2.0, sp) != 0:
            raise RuntimeError(be.get_last_error())

    ev = []
    with torch.cuda.stream(stream):
        for i in range(args.warmup + args.steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record(stream)
            demosaic()
            e[1].record(stream)
            median()
            e[2].record(stream)
            if i >= args.warmup:
                ev.append(e)
    torch.cuda.synchronize()
    ms_step = float(np.mean([a.elapsed_time(c) for a, _, c in ev]))
    ms_dem = float(np.mean([a.elapsed_time(b) for a, b, _ in ev]))
    ms_med = float(np.mean([b.elapsed_time(c) for _, b, c in ev]))
    npx = w * h
    med_bytes = npx * 3 * (n * 2 + 2)
    dem_bytes = n * npx * (2 + 6)
    peaks, kind = measured_peaks()
    gbps = med_bytes / (ms_med / 1e3) / 1e9
    res = {"value": round(npx / 1e6 / (ms_step / 1e3), 1), "unit": "stack output Mpix/s",
           "ms_per_step": round(ms_step, 3), "steps": args.steps,
           "workload": f"{n} x {w}x{h} RGGB {cfg.bits}-bit, translation +-{cfg.max_shift} px, rotation "
                       f"+-{cfg.max_rot_deg} deg, outliers {np.mean(st.outlier_frac):.3f} of pixels; demosaic + "
                       f"fused warp/median (sigma 2)",
           "gpu_launches_per_step": n + 1,
           "stages_ms": {"demosaic": round(ms_dem, 3), "warp_median": round(ms_med, 3)},
           "demosaic_GBps": round(dem_bytes / (ms_dem / 1e3) / 1e9, 1),
           "roofline": {"kernel": "k_warp_median", "bound": "hbm", "achieved": round(gbps, 1),
                        "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(gbps / peaks["hbm_gbs"], 4),
                        "algorithmic_bytes": med_bytes,
                        "bytes_formula": "Npx * 3 * (N * 2 + 2): every frame's texels read once, the median written",
                        "peak_source": kind + " (hbm_gbs, burst copy)"}}
    if not args.no_cpu_baseline:
        res["cpu_check"] = cpu_stack_check(st, cfg, Hs, out.cpu().numpy().view(np.uint16))
    return res


def _backend():
    from image360_b200 import B200ComputeBackend
    be = B200ComputeBackend()
    assert be.initialize() == 0, be.get_last_error()
    return be


def cpu_stack_check(st, cfg, Hs, got):
    """The reference's CPU code on the full stack, in row strips on
    hardware_concurrency()-1 threads: demosaic of every frame, WarpPerspective
    of every frame onto the reference grid, MedianStack.  Run with the
    reference's scalar tier (the algorithm as written, which the GPU
    reproduces: bit-exact expected) and timed with its run-time tier (what
    the CPU backend picks on this host; its FMA-contracted statistics may
    clip a different value set at a few scalars)."""
    from concurrent.futures import ThreadPoolExecutor

    from image360_b200 import synth
    impl, kind = _cpu_impl()
    threads = _cpu_threads()
    black, cm, rc, filt = synth.demosaic_params(cfg)
    w, h = cfg.frame_w, cfg.frame_h
    cfa = [c.cpu().numpy().view(np.uint16) for c in st.cfa]
    strips = [(y0, min(h, y0 + max(8, h // (4 * threads)))) for y0 in range(0, h, max(8, h // (4 * threads)))]

    def run(tier):
        kw = {} if tier is None else {"tier": tier}
        t0 = time.time()
        with ThreadPoolExecutor(threads) as ex:
            # whole-frame demosaic tasks (the 3x3 stencil needs neighbouring rows)
            rgb = list(ex.map(lambda c: impl.demosaic(c, black, cm, rc, filt, **kw), cfa))
            warped = [np.zeros((h, w, 3), np.uint16) for _ in rgb]

            def warp_strip(args):
                k, (y0, y1) = args
                warped[k][y0:y1] = impl.warp(rgb[k], w, y1 - y0, Hs[k], 0, y0, **kw)
            list(ex.map(warp_strip, [(k, s) for k in range(len(rgb)) for s in strips]))
            med = np.zeros((h, w, 3), np.uint16)

            def med_strip(s):
                y0, y1 = s
                med[y0:y1] = impl.median([wp[y0:y1] for wp in warped], 2.0, **kw)
            list(ex.map(med_strip, strips))
        return med, time.time() - t0

    exact_tier = 0 if kind == "reference" else None
    ref_exact, secs_exact = run(exact_tier)
    out = {"kind": kind, "cores": threads, "exact_vs_scalar_tier": bool(np.array_equal(got, ref_exact))}
    if kind == "reference":
        ref_auto, secs = run(impl.tier)
        diff = np.abs(got.astype(np.int32) - ref_auto.astype(np.int32))
        out.update({"auto_tier": int(impl.tier), "values_differing_from_auto_tier": int((diff > 0).sum()),
                    "max_diff_vs_auto_tier": int(diff.max())})
    else:
        secs = secs_exact
    out.update({"value": round(w * h / 1e6 / secs, 2), "unit": "stack output Mpix/s", "seconds": round(secs, 2),
                "sample": f"full stack: {len(cfa)} frames demosaiced (one task each), warped and median-stacked in "
                          f"{len(strips)} row strips per frame on {threads} threads"})
    return out


def run_export(args, S, stream):
    """The panorama export that follows the render: the preview composite of
    PanoramaExporter::ExportPreviewJpeg at the size the reference's CLI asks
    for (cli/main.cpp: maxDimension = canvas width, so scale 1 on a wide
    panorama) from the plan's tile outputs, timed alone with CUDA events."""
    import torch
    plan, pano = S["plan"], S["pano"]
    sp = stream.cuda_stream
    W, H = pano.canvas_w, pano.canvas_h
    cap = W * H * 3
    out = torch.empty(cap, dtype=torch.uint8, device=S["outs"][0].device)
    times = []
    with torch.cuda.stream(stream):
        for i in range(args.warmup + args.steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            e[0].record(stream)
            r, ow, oh = plan.export_preview(W, H, W, out.data_ptr(), cap, sp)
            e[1].record(stream)
            assert r == 0, S["be"].get_last_error()
            if i >= args.warmup:
                times.append(e)
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in times]))
    px = ow * oh
    alg = px * (6 + 3)  # one RGB48 source sample read, one RGB8 pixel written
    peaks, kind = measured_peaks()
    gbps = alg / (ms / 1e3) / 1e9
    return {"value": round(px / 1e6 / (ms / 1e3), 1), "unit": "preview Mpix/s", "ms_per_step": round(ms, 3),
            "preview": f"{ow}x{oh} RGB8 (maxDimension {W})", "gpu_launches_per_step": 2,
            "roofline": {"kernel": "k_export_place (zero fill included)", "bound": "hbm", "achieved": round(gbps, 1),
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(gbps / peaks["hbm_gbs"], 4),
                         "algorithmic_bytes": alg, "peak_source": kind + " (hbm_gbs, burst copy)"}}


def run_color(args, S, stream):
    """Optimize-stage colour correction of the step's 24 frames, timed alone
    (OptimizeExecutor.cpp:283-330: Lab statistics of the reference and each
    target frame, then the Reinhard transfer of every target in place):
    i360b_launch_color_correct on copies of the demosaiced frames, restored
    before every step outside the timed events (inputs far larger than L2),
    with frame 0 as the reference."""
    import torch
    be, cfg = S["be"], S["cfg"]
    sp = stream.cuda_stream
    n, w, h = len(S["rgb"]), cfg.frame_w, cfg.frame_h
    work = [torch.empty_like(r) for r in S["rgb"]]
    ptrs = [t.data_ptr() for t in work]
    stats = torch.zeros(n * 6, dtype=torch.float64, device=work[0].device)
    times, stat_times = [], []
    with torch.cuda.stream(stream):
        for i in range(args.warmup + args.steps):
            for a, b in zip(work, S["rgb"]):
                a.copy_(b)
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(stream)
            assert be.launch_lab_stats(ptrs, [w] * n, [h] * n, stats.data_ptr(), sp) == 0, be.get_last_error()
            e[1].record(stream)
            e[2].record(stream)
            assert be.launch_color_correct(ptrs, [w] * n, [h] * n, 0, stats.data_ptr(), sp) == 0, be.get_last_error()
            e[3].record(stream)
            if i >= args.warmup:
                times.append(e[2:])
                stat_times.append(e[:2])
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in times]))
    ms_stats = float(np.mean([a.elapsed_time(b) for a, b in stat_times]))
    px = n * w * h
    alg = px * 6 + (n - 1) * w * h * 12  # statistics read every frame; transfer reads and writes each target
    peaks, kind = measured_peaks()
    gbps = alg / (ms / 1e3) / 1e9
    tr_ms = ms - ms_stats
    tr_gbps = (n - 1) * w * h * 12 / (tr_ms / 1e3) / 1e9
    out = {"value": round(px / 1e6 / (ms / 1e3), 1), "unit": "frame Mpix/s", "ms_per_step": round(ms, 3),
           "frames": n, "frame": f"{w}x{h}", "reference_frame": 0, "gpu_launches_per_step": 3,
           "stats_ms": round(ms_stats, 3), "transfer_ms": round(tr_ms, 3),
           "roofline": {"kernel": "k_lab_partials + k_reinhard", "bound": "issue (correctly rounded FP32 powers and cube roots)",
                        "achieved": round(gbps, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": round(gbps / peaks["hbm_gbs"], 4), "algorithmic_bytes": alg,
                        "transfer_GBps": round(tr_gbps, 1), "peak_source": kind + " (hbm_gbs, burst copy)"}}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_color_baseline(S, n, w, h)
    return out


def cpu_color_baseline(S, n, w, h):
    """The reference's per-image colour task (OptimizeExecutor.cpp:308-327:
    ComputeLabStats of the reference, of the target, ApplyReinhardColorTransfer
    of the target) on hardware_concurrency()-1 host threads, on row strips of
    the frames, extrapolated to the n-1 targets of the frame set."""
    import ctypes as ct
    from concurrent.futures import ThreadPoolExecutor

    import oracle
    impl, kind = _cpu_impl()
    stats_fn = impl.lib.ref_lab_stats if kind == "reference" else impl.lib.or_lab_stats
    tr_fn = impl.lib.ref_reinhard if kind == "reference" else impl.lib.or_reinhard
    threads = max(1, (os.cpu_count() or 2) - 1)
    rows = max(1, h // 16)
    ref = np.ascontiguousarray(S["rgb"][0][:rows].cpu().numpy().view(np.uint16))
    tgts = [np.ascontiguousarray(S["rgb"][1 + k % (n - 1)][rows * (k // (n - 1)):][:rows].cpu().numpy().view(np.uint16))
            for k in range(threads)]
    d = lambda a: a.ctypes.data_as(oracle._f64p)

    def task(t):
        rm, rs, tm, ts = (np.zeros(3) for _ in range(4))
        stats_fn(ref.ctypes.data_as(oracle._u16p), w, rows, d(rm), d(rs))
        stats_fn(t.ctypes.data_as(oracle._u16p), w, t.shape[0], d(tm), d(ts))
        tr_fn(t.ctypes.data_as(oracle._u16p), w, t.shape[0], d(tm), d(ts), d(rm), d(rs))

    t0 = time.time()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(task, tgts))
    spent = time.time() - t0
    px_s = sum(t.shape[0] * w for t in tgts) / spent  # target pixels colour-corrected per second
    job_s = (n - 1) * w * h / px_s
    return {"value": round(n * w * h / 1e6 / job_s, 2), "unit": "frame Mpix/s", "cores": threads, "kind": kind,
            "sample": f"{threads} per-image tasks on {w}x{rows} strips (reference strip stats, target strip stats, "
                      f"target transfer), extrapolated to {n - 1} targets of {w}x{h}",
            "sample_seconds": round(spent, 2), "job_seconds": round(job_s, 2)}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path on this host's
    cores, on the same workload; rank 0 only.  Each step is one bounded
    sample of the job (a proportional share of the frames demosaiced and
    `--cpu-tiles` tiles rendered, a new seeded choice every step), timed as
    it runs: value = the sampled tiles' output pixels / the steps' seconds."""
    if rank != 0:
        return None
    from image360_b200 import synth
    impl, kind = _cpu_impl()
    threads = _cpu_threads()
    cfg = synth.C1 if args.scale == 1.0 else synth.scaled(synth.C1, args.scale, tile=synth.C1.tile)
    if world > 1 and args.mode == "sharded":
        cfg = synth.PanoConfig(**{**cfg.__dict__, "cols": cfg.cols * world})
    pano = synth.make_panorama(cfg, device="cpu")
    cfa_host = [c.numpy().view(np.uint16) for c in pano.cfa]
    gains = (1.0 / pano.gains).astype(np.float32)
    # every frame demosaiced once by the CPU code itself (untimed setup: the
    # render of a sampled tile needs all of its contributors)
    frames_host = cpu_demosaic_all(impl, kind, cfa_host, cfg, threads)
    n_tiles = max(1, min(args.cpu_tiles, len(pano.tiles)))
    px_tot = secs_tot = 0.0
    desc = ""
    t_wall = time.time()
    for s in range(args.warmup + args.steps):
        if s == args.warmup:
            t_wall = time.time()
        px, secs, desc = cpu_sample(impl, kind, frames_host, pano, cfg, threads, n_tiles, cfa_host, gains, seed=100 + s)
        if s >= args.warmup:
            px_tot += px
            secs_tot += secs
    wall = time.time() - t_wall
    value = px_tot / 1e6 / secs_tot
    return {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(secs_tot / args.steps * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16 storage / fp32 arithmetic",
            "data": "synthetic (seeded scene, 14-bit RGGB)", "impl": "reference",
            "config": {"workload": f"plain seam blend, 24 x {cfg.frame_w}x{cfg.frame_h} RGGB -> "
                                   f"{pano.canvas_w}x{pano.canvas_h} in {cfg.tile}^2 tiles, {cfg.bands} bands",
                       "step": f"one sample per step: {desc}", "parallelism": f"{threads} host threads",
                       "timed_wall_seconds": round(wall, 1)},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": kind, "sample": desc},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["sharded", "replicas"], default="sharded",
                    help="N > 1: one panorama of 8N frame columns split over the ranks (sharded), or one "
                         "panorama per rank (replicas)")
    ap.add_argument("--scale", type=float, default=1.0, help="geometry scale of the workload (1.0 = full size)")
    ap.add_argument("--cpu-tiles", type=int, default=15, help="tiles per CPU sample (one per host thread)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned blend")
    ap.add_argument("--no-color", action="store_true", help="skip the colour-correction leg")
    ap.add_argument("--no-export", action="store_true", help="skip the preview-export leg")
    ap.add_argument("--no-stack", action="store_true", help="skip the median-stack leg")
    ap.add_argument("--no-uneven", action="store_true", help="skip the 256 uneven-tile leg")
    ap.add_argument("--no-parity", action="store_true", help="skip the full-panorama check against the CPU code")
    ap.add_argument("--no-native", action="store_true", help="skip the FP16-storage (native mode) leg")
    ap.add_argument("--fusion", type=int, choices=[0, 1, 2], default=None,
                    help="force the level-fusion depth after autotuning (measurement of one form)")
    ap.add_argument("--warp-shape", type=int, choices=[0, 1], default=None,
                    help="force the tile-warp form after autotuning")
    ap.add_argument("--chain-lag", type=int, default=None,
                    help="force the chain stagger after autotuning (-1: chains together; L: the other chains "
                         "start after the first finishes stage L)")
    ap.add_argument("--chain-split", type=int, default=None,
                    help="force the chain split after autotuning (0: balanced; p: the p%% of tiles with the "
                         "slowest seam step in the first chain)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the plan's default band height and ring depth")
    ap.add_argument("--train-steps", type=int, default=782, help="Adam steps (782 x 64 = 50k windows)")
    ap.add_argument("--train-batch", type=int, default=64)
    ap.add_argument("--train-scenes", type=int, default=4)
    ap.add_argument("--learned-batch", type=int, default=256, help="network windows per pass")
    ap.add_argument("--weights", default="", help="trained parameters (fp32) instead of training")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        log("note: warmup raised to 3")
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        else:
            line = run_ours(args, rank, world, local_rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

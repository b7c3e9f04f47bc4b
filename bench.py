"""Benchmark of the B200 render path on the sky-lit 2.6M-triangle scene.

One step = one full render of the workload (1920x1080 pixels x 64 samples,
depth 8, 32 subdivision-6 icospheres under a Hosek-Wilkie sky) with the scene
resident in HBM.  Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--integrator megakernel|wavefront] [--spp S] [--scale F]

`value` is device-timed Mpaths/s (CUDA events on the render stream, max over
ranks); `e2e` is the same metric through the reference-facing C-ABI with the
camera uploaded from host memory and the film read back to host memory every
step.  --impl reference times the CPU restatement of the reference routines
(oracle) on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "sky-lit 32 icospheres (2,621,440 tris), 1920x1080, 64 spp, depth 8, Hosek sky T=3 elev 30deg"
# the single-frame workloads: scene generator, full-size image, description
SCENES = {
    "sky": ("sky_scene", (1920, 1080), WORKLOAD),
    "room": ("room_scene", (256, 256), "closed room, 36 tris (5 walls, ceiling light quad, 2 boxes), 256x256, "
                                       "16 spp, depth 5"),
    "env": ("env_scene", (1920, 1080), "32 icospheres (2,621,440 tris) lit by a 2048x1024 log-normal + 3 lobes "
                                       "env map, MIS, FP64 CDF, 1920x1080, 128 spp, depth 8"),
}
METRIC = "Mpaths/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 5; 800 for the room, whose step is ~2 ms, so that the timed "
                         "region spans the clock sampler's interval)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--integrator", default="wavefront", choices=["megakernel", "wavefront"])
    ap.add_argument("--no-compare", action="store_true",
                    help="skip timing the other integrator on the same scene and samples")
    ap.add_argument("--spp", type=int, default=None, help="samples per pixel (default: the workload's)")
    ap.add_argument("--scale", type=float, default=1.0, help="image size scale (1 = the workload's full size)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="wavefront: fixed launch parameters")
    ap.add_argument("--no-rmse", action="store_true", help="skip the RMSE of both integrators against the FP64 oracle")
    ap.add_argument("--wf-block", type=int, default=128)
    ap.add_argument("--wf-slots", type=int, default=1 << 21)
    ap.add_argument("--wf-sort", type=int, default=0)
    ap.add_argument("--wf-graph", type=int, default=1, help="wavefront: 1 CUDA-graph while loop, 0 host loop")
    ap.add_argument("--wf-tree", type=int, default=0,
                    help="wavefront (without autotuning): 0 auto, 1 binary tree, 2 four-wide tree, "
                         "3 four-wide tree for shadow rays only")
    ap.add_argument("--workload", default="sky", choices=["sky", "room", "env", "batched", "adjoint"],
                    help="sky: the headline sky-lit scene; room: the 36-triangle room; env: the env-map MIS "
                         "scene; batched: 64 uneven frames in one wavefront launch against 64 sequential "
                         "megakernel renders; adjoint: forward+backward of the differentiable-rendering "
                         "configuration")
    a = ap.parse_args()
    if a.steps is None:
        a.steps = 800 if a.workload == "room" else 5
    return a


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x: float) -> float:
    """the largest value of x over all ranks (a replicated job's step takes
    as long as its slowest rank); x itself without a process group"""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, ms_per_step: float, world: int) -> float:
    """whole-job rate in millions of units per second: every rank renders
    the full workload (replicas), so world x units in the slowest rank's
    step time"""
    return world * units_per_rank / (ms_per_step / 1000) / 1e6


class Clocks:
    """nvidia-smi sampler during the timed region"""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.path = Path(tempfile.gettempdir()) / f"noor_b200_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if not self.p or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [l.split(",") for l in self.path.read_text().splitlines() if l.strip()]
        self.path.unlink(missing_ok=True)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, n in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_scene(args):
    """the workload's scene at --scale of its image size; fills args.spp
    with the workload's sample count when not given"""
    from noor_b200 import scenes
    fn, (w0, h0), _ = SCENES[args.workload]
    w, h = int(round(w0 * args.scale)), int(round(h0 * args.scale))
    kw = dict(width=w, height=h)
    if args.spp:
        kw["spp"] = args.spp
    s = getattr(scenes, fn)(**kw)
    args.spp = s.render["spp"]
    t = time.time()
    built = scenes.BuiltPayload(s)
    return s, built, time.time() - t


def algorithmic_bytes(orc, cam, spp, isect, sample_pixels=20000, seed=0):
    """Bytes the path reads by the traversal/shading model: per traversal step
    32 B per node, per tested triangle 48 B (watertight: three vertices) or
    32 B (Wald: first sector) + 16 B per in-range triangle (Wald second
    record), per extension hit 16 B attributes + 3 x (16+16+8) B vertex data.
    Counted by the oracle on a pixel subsample with 2 samples each.  Returns
    bytes per path and the counts per path, with the traversal of extension
    rays and of shadow rays apart."""
    n = cam.w * cam.h
    rng = np.random.default_rng(seed)
    px = np.sort(rng.choice(n, size=min(sample_pixels, n), replace=False))
    tot = np.zeros(8, np.uint64)
    paths = 0
    # contiguous runs keep the oracle call simple: sample blocks of 64 pixels
    for b in px[:: 64]:
        p1 = min(int(b) + 64, n)
        _, c = orc.render(cam, 1, 2, p0=int(b), p1=p1, isect=isect, threads=1, counters=True)
        tot += c
        paths += 2 * (p1 - int(b))
    ext, shadow, nodes, tris, inrange, sh_nodes, sh_tris, sh_inrange = [float(x) / paths for x in tot]
    tri_b = 32.0 if isect == 1 else 48.0

    def trav(nd, tr, ir):
        return 32.0 * nd + tri_b * tr + (16.0 * ir if isect == 1 else 0.0)

    per_path = trav(nodes, tris, inrange) + ext * (16 + 3 * 40)
    return per_path, dict(ext_rays_per_path=ext, shadow_rays_per_path=shadow, nodes_per_path=nodes,
                          tris_per_path=tris, ext_nodes_per_path=nodes - sh_nodes, ext_tris_per_path=tris - sh_tris,
                          ext_traversal_bytes_per_path=trav(nodes - sh_nodes, tris - sh_tris, inrange - sh_inrange),
                          shadow_traversal_bytes_per_path=trav(sh_nodes, sh_tris, sh_inrange), sample_paths=paths)


# slot state the extend kernel moves per ray besides the traversal: reads
# origin + direction (32 B) and the queue entry (4 B); writes the hit record
# (16 B + 8 B) and one queue entry (4 B)
EXTEND_SLOT_BYTES = 64.0
# queue state the shadow kernel moves per ray besides the traversal: the
# queue entry (4 B), its ray (32 B), the slot's frame word (16 B in a
# multi-scene launch, counted always) and the pending contribution it may
# cancel (16 B), rounded to the sector-aligned 72 B
SHADOW_QUEUE_BYTES = 72.0
# ncu DRAM bytes per extension ray of wf_extend, from the capture summarised
# in profiles/wf_extend_sky.md (the line "dram_bytes_per_ext_ray: X")
TRAFFIC_PROFILE = ROOT / "profiles" / "wf_extend_sky.md"


def profiled_traffic_per_ray():
    import re
    if not TRAFFIC_PROFILE.exists():
        return None
    m = re.search(r"dram_bytes_per_ext_ray:\s*([0-9.eE+]+)", TRAFFIC_PROFILE.read_text())
    return float(m.group(1)) if m else None


# issue-slot use and SIMT efficiency of wf_extend, from the ncu capture
# summarised in profiles/wf_extend_sky.md (lines "issue_slots_busy_pct: X",
# "lanes_active_per_inst: X", "dram_pct_of_peak: X")
def profiled_issue():
    import re
    if not TRAFFIC_PROFILE.exists():
        return None
    text = TRAFFIC_PROFILE.read_text()
    out = {}
    for k in ("issue_slots_busy_pct", "lanes_active_per_inst", "dram_pct_of_peak", "achieved_occupancy_pct"):
        m = re.search(k + r":\s*([0-9.eE+]+)", text)
        if m:
            out[k] = float(m.group(1))
    return out or None


def rmse_vs_fp64(r, imgs, spp, rows, mult=16):
    """RMSE of each integrator's image against the FP64 oracle on `rows`
    (full image rows): on the same seeds (precision: FP32 arithmetic and
    compensated accumulation) and at mult x the samples (estimator)"""
    from oracle.oracle import Oracle
    W = r.w
    threads = os.cpu_count() or 1
    orc = Oracle(r.built.payload, r.spec, r.hosek)
    same, high = [], []
    for y in rows:
        same.append(orc.render(r.camera, 1, spp, p0=y * W, p1=(y + 1) * W, fp64=True, threads=threads))
        high.append(orc.render(r.camera, 1, spp * mult, p0=y * W, p1=(y + 1) * W, fp64=True, threads=threads))
    orc.close()
    same, high = np.concatenate(same), np.concatenate(high)
    sel = lambda img: np.concatenate([img[y] for y in rows])
    rm = lambda a, b: float(np.sqrt(np.mean((a - b) ** 2)))
    out = {"rows": rows, "pixels": len(rows) * W, "spp": spp, "reference_spp": spp * mult,
           "same_seeds": {k: rm(sel(v), same) for k, v in imgs.items()},
           "at_reference_spp": {k: rm(sel(v), high) for k, v in imgs.items()}}
    e = out["at_reference_spp"]
    if len(e) == 2:
        a, b = e.values()
        out["estimator_rmse_rel_diff"] = abs(a - b) / max(b, 1e-30)
    return out


def calibrate_pixels(orc, cam, spp, threads, target_s):
    """pixels of a centre block the oracle renders in about target_s seconds
    (growing blocks until one takes >= 1 s, then scaled)"""
    n = cam.w * cam.h
    npx = 1024
    while True:
        p0 = max(0, n // 2 - npx // 2)
        t = time.time()
        orc.render(cam, 1, spp, p0=p0, p1=min(n, p0 + npx), threads=threads)
        dt = time.time() - t
        if dt >= 1.0 or npx >= n:
            break
        npx = min(n, npx * 4)
    return int(max(1024, min(n, npx / max(dt, 1e-3) * target_s)))


def cpu_baseline(args, s, built, spec, hosek, cam, budget_s):
    """oracle FP32 on all host threads over a pixel subsample of the workload"""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    orc = Oracle(built.payload, spec, hosek)
    n = cam.w * cam.h
    npx = calibrate_pixels(orc, cam, args.spp, threads, budget_s)
    p0 = max(0, n // 2 - npx // 2)
    t = time.time()
    orc.render(cam, 1, args.spp, p0=p0, p1=p0 + npx, threads=threads)
    dt = time.time() - t
    orc.close()
    return {"value": npx * args.spp / dt / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{npx} contiguous pixels around the image centre x {args.spp} spp of the workload "
                      f"({npx * args.spp} paths, {dt:.1f} s), FP32 transcription of the reference routines"}


def run_reference(args):
    """The reference arm: the oracle's transcription of the reference's render
    routines on the host cores, over a payload from the reference's own BVH
    builder (oracle/_ref/libnoor_ref.so).  The workload's scene generators
    and struct layouts are loaded without the product package, so the
    product library is never loaded on this arm."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle.oracle import Oracle, RefPayload, camera_lookat, host_modules, ref_available
    if args.workload not in SCENES:
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm times the single-frame "
                          f"workloads ({', '.join(SCENES)}); the reference has no {args.workload} path"}))
        return
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libnoor_ref.so (the reference's own "
                          "builder) was not built: the reference tree was absent at build time"}))
        return
    capi, scenes = host_modules()
    fn, (w0, h0), _ = SCENES[args.workload]
    kw = dict(width=int(round(w0 * args.scale)), height=int(round(h0 * args.scale)))
    if args.spp:
        kw["spp"] = args.spp
    s = getattr(scenes, fn)(**kw)
    args.spp = s.render["spp"]
    built = RefPayload(s, capi, scenes)
    spec = built.default_spec(s.render["bounces"], s.render.get("rr", 1))
    spec.mis = int(s.render.get("mis", 0))
    cam = camera_lookat(capi, s.camera)
    hosek = reference_hosek(capi, s.hosek) if s.hosek is not None else capi.HosekSky()
    orc = Oracle(built.payload, spec, hosek)
    threads = os.cpu_count() or 1
    n = cam.w * cam.h
    # up to ~3 s of CPU work per step, the whole run within about 2.5 minutes
    npx = calibrate_pixels(orc, cam, args.spp, threads, max(0.05, min(3.0, 150.0 / (args.steps + args.warmup))))
    times = []
    for i in range(args.warmup + args.steps):
        p0 = (n // 2 + i * npx) % max(1, n - npx)
        t = time.time()
        orc.render(cam, 1, args.spp, p0=p0, p1=p0 + npx, threads=threads)
        if i >= args.warmup:
            times.append(time.time() - t)
    orc.close()
    built.free()
    ms = 1000 * statistics.mean(times)
    v = npx * args.spp / (ms / 1000) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": SCENES[args.workload][2], "sample_per_step": f"{npx} pixels x {args.spp} spp",
                       "payload": "the reference's own BVH builder and Wald records (oracle/_ref)"},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                             "sample": f"{npx} pixels x {args.spp} spp per step, FP32 transcription of the "
                                       "reference's device routines (the reference has no CPU render path)"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_hosek(capi, h):
    """Hosek sky for the reference arm as HosekSky::update sets it
    (noor/header/hosek.h:61-83): the reference's own fit,
    arhosek_rgb_skymodelstate_alloc_update, per colour channel's ground
    albedo (oracle/_ref/libnoor_ref.so), and the sun fields."""
    from oracle.oracle import ref_hosek_state
    elev = float(np.pi / 2 - h["sun_lat"])
    out = capi.HosekSky()
    for i in range(3):
        st = ref_hosek_state(float(h["turbidity"]), float(h["albedo"]), elev)
        for c in range(3):
            for j in range(9):
                out.state[i].configs[c][j] = float(st[9 * c + j])
            out.state[i].radiances[c] = float(st[27 + c])
        out.state[i].solar_radius = float(np.radians(0.51) / 2)
    d = np.array([np.sin(h["sun_lat"]) * np.cos(h["sun_lon"]), np.cos(h["sun_lat"]),
                  np.sin(h["sun_lat"]) * np.sin(h["sun_lon"])], np.float32)
    out.solar_dir[:] = [float(x) for x in d / np.linalg.norm(d)]
    out.ground_albedo[:] = [h["albedo"]] * 3
    out.solar_scale = h["solar_scale"]
    out.solar_radius = float(h["solar_radius_scale"] * np.radians(0.51) / 2)
    return out


class MegakernelPath:
    """reference-facing path: noor_render_frames (the megakernel) into the
    context film; e2e adds update_cuda_camera and noor_get_framebuffer"""

    name = "megakernel"

    def __init__(self, args, s, r):
        self.args = args
        self.r = r
        self.w, self.h = self.r.w, self.r.h
        self.host_film = np.zeros((self.h, self.w, 4), np.float32)

    def step(self):
        self.r.frame = C.c_uint(1)
        self.r.render(self.args.spp)

    def e2e_step(self):
        from noor_b200 import _capi
        _capi.call("update_cuda_camera")
        self.step()
        _capi.call("noor_get_framebuffer", self.host_film.ctypes.data_as(C.POINTER(C.c_float)), self.w * self.h)

    def e2e_bytes(self):
        from noor_b200 import _capi
        return C.sizeof(_capi.Camera), int(self.host_film.nbytes)

    def counters(self, reset=False):
        return self.r.counters(reset)

    def warm(self):
        pass

    def describe(self):
        return {"entry_point": "noor_render_frames"}

    def profile(self):
        """(kernel, device ms, launches) of the dominant kernel of one step"""
        return "megakernel", device_timed(self.step, 1), 1, {}

    def image(self):
        return self.r.framebuffer()[..., :3]


class WavefrontPath:
    """persistent wavefront integrator through noor_wavefront_render (CUDA
    graph while loop, parameters from noor_wavefront_autotune during warm-up);
    e2e adds the frame description from host memory and the film copied back
    to pinned host memory"""

    name = "wavefront"

    def __init__(self, args, s, r):
        import torch
        from noor_b200 import scenes, _capi
        self.args = args
        self.r = r
        self.w, self.h = self.r.w, self.r.h
        self.film = torch.zeros((self.h, self.w, 4), dtype=torch.float32, device="cuda")
        self.host_film = torch.zeros((self.h, self.w, 4), dtype=torch.float32).pin_memory()
        self.frames = (_capi.WfFrame * 1)(scenes.wf_frame(0, s.camera, args.spp, s.render["bounces"],
                                                          d_film=self.film.data_ptr()))
        self.params = scenes.wf_params(args.wf_block, args.wf_slots, args.wf_sort, args.wf_graph,
                                       traversal=args.wf_tree)
        self.tuned_ms = None

    def warm(self):
        from noor_b200 import _capi
        if self.args.no_autotune:
            return
        best = _capi.WfParams(0, 0, 0, self.args.wf_graph)
        ms = C.c_float()
        _capi.call("noor_wavefront_autotune", self.frames, 1, C.byref(best), C.byref(ms))
        self.params, self.tuned_ms = best, ms.value

    def step(self):
        from noor_b200 import _capi
        _capi.call("noor_wavefront_render", self.frames, 1, C.byref(self.params))

    def e2e_step(self):
        self.step()
        self.host_film.copy_(self.film)

    def e2e_bytes(self):
        from noor_b200 import _capi
        return C.sizeof(_capi.WfFrame), int(self.host_film.numel() * 4)

    def counters(self, reset=False):
        from noor_b200 import _capi
        c = (C.c_uint64 * 3)()
        _capi.call("noor_wavefront_counters", c, int(reset))
        return tuple(int(x) for x in c)

    def describe(self):
        p = self.params
        return {"entry_point": "noor_wavefront_render",
                "wavefront": {"block": p.block_size, "slots": p.queue_capacity, "material_sort": p.sort_granularity,
                              "graph": p.use_graph,
                              "tree": ["auto", "binary", "four-wide", "four-wide shadow rays"][p.traversal],
                              "shade_regs": p.shade_regs or 80,
                              "autotune_best_ms": self.tuned_ms}}

    def image(self):
        import torch
        torch.cuda.synchronize()
        return self.film.cpu().numpy()[..., :3]

    def profile(self):
        """one render with CUDA events around every stage launch
        (noor_wavefront_profile): (dominant kernel, its device ms summed over
        its launches, launches, ms per stage)"""
        from noor_b200 import _capi
        prof = _capi.WfProfile()
        _capi.call("noor_wavefront_profile", self.frames, 1, C.byref(self.params), C.byref(prof))
        names = ["wf_regen", "extension_ordering", "wf_extend", "wf_shade", "shadow_ordering", "wf_shadow",
                 "wf_check"]
        stages = {n: {"ms": float(prof.ms[i]), "launches": int(prof.launches[i])} for i, n in enumerate(names)}
        top = max(range(len(names)), key=lambda i: prof.ms[i])
        return names[top], float(prof.ms[top]), int(prof.launches[top]), stages


def device_timed(fn, steps):
    """device time of `steps` calls of fn on the library's stream (ms per call)"""
    from noor_b200 import _capi
    _capi.call("noor_event_record", 0)
    for _ in range(steps):
        fn()
    _capi.call("noor_event_record", 1)
    ms = C.c_float()
    _capi.call("noor_event_elapsed", 0, 1, C.byref(ms))
    return ms.value / steps


def run_batched(args):
    """C4: 64 frames of uneven resolution, scene size and spp (sky or env map)
    rendered in one wavefront launch (CUDA-graph device loop, launch
    parameters from the autotuner), against the same 64 frames rendered one
    after another by the plain megakernel."""
    import torch
    from noor_b200 import scenes, _capi
    sc, frames = scenes.batched_workload()
    keys = list(sc.keys())
    t = time.time()
    r = scenes.Renderer(sc[keys[0]])
    ids, keep = {keys[0]: 0}, []
    for k in keys[1:]:
        # the other scenes' payloads on the GPU (the same bytes as the host
        # builder's, noor_build_payload_gpu) now that the context is up
        sid, kp = scenes.upload_scene(sc[k], built=scenes.BuiltPayload(sc[k], gpu=True))
        ids[k] = sid
        keep.append(kp)
    setup_s = time.time() - t
    films = [torch.zeros((f["camera"]["h"], f["camera"]["w"], 4), dtype=torch.float32, device="cuda") for f in frames]
    desc = (_capi.WfFrame * len(frames))(*[scenes.wf_frame(ids[f["key"]], f["camera"], f["spp"], f["bounces"],
                                                           d_film=t_.data_ptr()) for f, t_ in zip(frames, films)])
    npaths = sum(f["camera"]["w"] * f["camera"]["h"] * f["spp"] for f in frames)
    best = _capi.WfParams(0, 0, 0, 1)
    tms = C.c_float()
    _capi.call("noor_wavefront_autotune", desc, len(frames), C.byref(best), C.byref(tms))
    wf = lambda: _capi.call("noor_wavefront_render", desc, len(frames), C.byref(best))
    mk = lambda: _capi.call("noor_megakernel_batch", desc, len(frames), None)
    for _ in range(max(3, args.warmup)):
        wf()
    l0 = C.c_uint64()
    _capi.call("noor_launch_count", C.byref(l0))
    with Clocks(0) as clk:
        wf_ms = device_timed(wf, args.steps)
    l1 = C.c_uint64()
    _capi.call("noor_launch_count", C.byref(l1))
    img_wf = [f_.cpu().numpy()[..., :3] for f_ in films]
    for _ in range(2):
        mk()
    mk_ms = device_timed(mk, max(2, args.steps // 2))
    img_mk = [f_.cpu().numpy()[..., :3] for f_ in films]
    rel = np.concatenate([(np.abs(a - b) / np.maximum(np.abs(b), 1e-2)).ravel() for a, b in zip(img_wf, img_mk)])
    # end to end: frame descriptions from host memory, films back to pinned host memory
    host = [torch.zeros(f_.shape, dtype=torch.float32).pin_memory() for f_ in films]
    e2e_t = []
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        wf()
        for h_, f_ in zip(host, films):
            h_.copy_(f_)
        if i >= args.warmup:
            e2e_t.append(time.perf_counter() - t)
    e2e_ms = statistics.mean(e2e_t) * 1000
    line = {"metric": METRIC, "value": npaths / (wf_ms / 1000) / 1e6, "unit": METRIC, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wf_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": "64 uneven frames (sides 128-1024, 5k-2.6M triangles, 4-64 spp, depth 6, "
                                   "sky or env map) in one wavefront launch",
                       "frames": len(frames), "scenes": len(keys), "paths_per_step": npaths,
                       "triangles_uploaded": int(sum(x.num_triangles for x in sc.values())),
                       "setup_s": round(setup_s, 1), "payload_builder": "host for the first scene, GPU for the rest",
                       "wavefront": {"block": best.block_size, "slots": best.queue_capacity,
                                     "material_sort": best.sort_granularity, "graph": best.use_graph}},
            "other_integrator": {"integrator": "megakernel, 64 sequential renders (noor_megakernel_batch)",
                                 "value": npaths / (mk_ms / 1000) / 1e6, "ms_per_step": mk_ms,
                                 "speedup_of_headline": mk_ms / wf_ms,
                                 "same_samples_image_check": {"median_rel_diff": float(np.median(rel)),
                                                              "frac_pixels_rel_diff_gt_1e-3": float((rel > 1e-3).mean())}},
            "e2e": {"value": npaths / (e2e_ms / 1000) / 1e6, "unit": METRIC,
                    "h2d_bytes_per_step": C.sizeof(_capi.WfFrame) * len(frames),
                    "d2h_bytes_per_step": int(sum(f_.numel() * 4 for f_ in films))},
            "gpu_launches": int(l1.value - l0.value) // max(1, args.steps) * args.steps, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    r.close()


def run_adjoint(args):
    """C5: forward + backward of the path-replay adjoint on the
    differentiable-rendering configuration (512x512, 16 spp, depth 4,
    204,800 triangles, 64 materials, 512x256 env map), L2 loss against a
    seeded target render."""
    import torch
    from noor_b200 import scenes, _capi
    from noor_b200.adjoint import render, scene_parameters
    kw = dict(width=int(round(512 * args.scale)), height=int(round(512 * args.scale)))
    if args.spp:
        kw["spp"] = args.spp
    s = scenes.adjoint_scene(**kw)
    r = scenes.Renderer(s)
    W, H, spp = s.camera["w"], s.camera["h"], s.render["spp"]
    alb, rough, env = scene_parameters(s)
    rng = np.random.default_rng(11)
    with torch.no_grad():
        target = render((alb * torch.from_numpy(rng.uniform(0.8, 1.2, alb.shape).astype(np.float32)).cuda()).contiguous(),
                        rough, (env * 1.1).contiguous(), W, H, spp, first_frame=1000)
    params = [t.clone().requires_grad_(True) for t in (alb, rough, env)]

    def step():
        for p in params:
            p.grad = None
        img = render(*params, W, H, spp)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        return loss

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    l0 = C.c_uint64()
    _capi.call("noor_launch_count", C.byref(l0))
    fwd, bwd = [], []
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for p in params:
                p.grad = None
            a = time.perf_counter()
            img = render(*params, W, H, spp)
            loss = ((img - target) ** 2).sum()
            torch.cuda.synchronize()
            b = time.perf_counter()
            loss.backward()
            torch.cuda.synchronize()
            c = time.perf_counter()
            fwd.append(b - a)
            bwd.append(c - b)
        total = (time.perf_counter() - t0) / args.steps
    l1 = C.c_uint64()
    _capi.call("noor_launch_count", C.byref(l1))
    ms = total * 1000
    npaths = W * H * spp
    # the plain megakernel rendering the same image at the loaded parameters
    for _ in range(2):
        r.frame = C.c_uint(1)
        r.render(spp)
    mk_ms = device_timed(lambda: (setattr(r, "frame", C.c_uint(1)), r.render(spp)), max(1, args.steps))
    line = {"metric": "ms per forward+backward iteration", "value": ms, "unit": "ms", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": f"differentiable rendering: 10 subdivision-5 icospheres (204,800 tris), 64 "
                                   f"materials, 512x256 env map, {W}x{H}, {spp} spp, depth 4, L2 loss",
                       "params": int(sum(p.numel() for p in params))},
            "forward_ms": 1000 * statistics.mean(fwd), "backward_ms": 1000 * statistics.mean(bwd),
            "forward_mpaths_per_s": npaths / statistics.mean(fwd) / 1e6,
            "megakernel_render_ms": mk_ms, "megakernel_mpaths_per_s": npaths / (mk_ms / 1000) / 1e6,
            "backward_mpaths_per_s": npaths / statistics.mean(bwd) / 1e6,
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 4},
            "gpu_launches": int(l1.value - l0.value), "clocks": clk.summary(),
            "timing": "host wall clock around synchronised calls (the adjoint entry points synchronise)"}
    print(json.dumps(line), flush=True)
    r.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    if args.workload in ("batched", "adjoint"):
        # one-GPU configurations: under a multi-rank launch rank 0 runs them
        # (its line says n_gpus 1) and the other ranks exit without work
        if rank == 0:
            (run_batched if args.workload == "batched" else run_adjoint)(args)
        return
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from noor_b200 import scenes, _capi
    s, built, build_s = build_scene(args)
    r = scenes.Renderer(s, built=built)
    # the same payload with the bottom-level trees built on the GPU (context
    # up): its timings beside the host build's, and a byte check of the nodes
    gb = scenes.BuiltPayload(s, gpu=True)
    bvh_build = {"host_payload_s": round(built.stat.build_seconds, 3), "host_tree_s": round(built.stat.tree_seconds, 3),
                 "gpu_payload_s": round(gb.stat.build_seconds, 3), "gpu_tree_s": round(gb.stat.tree_seconds, 3),
                 "gpu_tree_device_ms": round(gb.stat.tree_device_ms, 1),
                 "identical_nodes": bool(np.array_equal(gb.nodes(), built.nodes()) and
                                         np.array_equal(gb.triangle_order(), built.triangle_order()))}
    gb.free()
    paths_ = {"megakernel": MegakernelPath(args, s, r), "wavefront": WavefrontPath(args, s, r)}
    path = paths_[args.integrator]
    other = None if args.no_compare else paths_["megakernel" if args.integrator == "wavefront" else "wavefront"]

    def timed(p, clocks_index=None):
        """warm-up, then K device-timed steps: (ms per step, launches, ext, shadow, clocks)"""
        p.warm()   # the wavefront path autotunes its launch parameters here
        for _ in range(max(3, args.warmup)):
            p.step()
        p.counters(reset=True)
        l0 = C.c_uint64()
        _capi.call("noor_launch_count", C.byref(l0))
        if world > 1:
            torch.distributed.barrier()
        with Clocks(local if clocks_index is None else clocks_index) as clk:
            _capi.call("noor_event_record", 0)
            for _ in range(args.steps):
                p.step()
            _capi.call("noor_event_record", 1)
            ms = C.c_float()
            _capi.call("noor_event_elapsed", 0, 1, C.byref(ms))
        l1 = C.c_uint64()
        _capi.call("noor_launch_count", C.byref(l1))
        ext, shadow, _ = p.counters()
        ms_step = max_over_ranks(ms.value / args.steps)
        return ms_step, int(l1.value - l0.value), ext, shadow, clk.summary()

    ms_step, launches, ext, shadow, clocks = timed(path)
    npaths = path.w * path.h * args.spp
    value = job_rate(npaths, ms_step, world)
    mrays = job_rate((ext + shadow) / args.steps, ms_step, world)
    compare = None
    img = path.image()
    imgs = {path.name: img}
    if other is not None:
        oms, olaunch, oext, oshadow, oclk = timed(other)
        oimg = other.image()
        imgs[other.name] = oimg
        rel = np.abs(img - oimg) / np.maximum(np.abs(oimg), 1e-2)
        compare = {"integrator": other.name, "value": job_rate(npaths, oms, world), "ms_per_step": oms,
                   "mrays_per_s": job_rate((oext + oshadow) / args.steps, oms, world),
                   "gpu_launches": olaunch, "clocks": oclk,
                   "speedup_of_headline": oms / ms_step,
                   "same_samples_image_check": {"median_rel_diff": float(np.median(rel)),
                                                "frac_pixels_rel_diff_gt_1e-3": float((rel > 1e-3).mean()),
                                                "mean_ratio": float(img.mean() / max(oimg.mean(), 1e-30))}}

    # the dominant kernel's device time, for the roofline (one extra render
    # with events around every stage launch, outside the timed region)
    top_kernel, top_ms, top_launches, stages = path.profile()

    # end to end through the public C-ABI with host buffers
    e2e_t = []
    for i in range(args.warmup + args.steps):
        if world > 1:
            torch.distributed.barrier()
        t = time.perf_counter()
        path.e2e_step()
        if i >= args.warmup:
            e2e_t.append(time.perf_counter() - t)
    e2e_ms = max_over_ranks(statistics.mean(e2e_t) * 1000)
    h2d, d2h = path.e2e_bytes()
    e2e = {"value": job_rate(npaths, e2e_ms, world), "unit": METRIC, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h}

    if rank == 0:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
        hbm = peaks.get("hbm_gbs", 6650.0)
        roof = {"bound": "hbm", "limiter": "issue and divergence: the traversal's node reads hit L1/L2 and DRAM "
                                           "runs at a few per cent of peak (issue block)",
                "kernel": top_kernel, "achieved": None, "peak": hbm, "unit": "GB/s", "frac": None,
                "traffic": None, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "kernel_ms_per_step": top_ms, "kernel_launches_per_step": top_launches,
                "kernel_share_of_step": top_ms / sum(v["ms"] for v in stages.values()) if stages else 1.0,
                "stages": stages}
        cpu = None
        if not args.no_cpu_baseline:
            from oracle.oracle import Oracle
            orc = Oracle(built.payload, r.spec, r.hosek)
            per_path, counts = algorithmic_bytes(orc, r.camera, args.spp, r.spec.intersector)
            orc.close()
            if top_kernel == "wf_extend":
                # traversal bytes of the extension rays + the slot state of every ray
                alg = counts["ext_traversal_bytes_per_path"] * npaths + EXTEND_SLOT_BYTES * ext / args.steps
                # the ncu capture is of the sky-lit scene
                tr = profiled_traffic_per_ray() if args.workload == "sky" else None
                traffic = tr * ext / args.steps / top_launches if tr else None
            elif top_kernel == "wf_shadow":
                # traversal bytes of the shadow rays + the queue state of every one
                alg = counts["shadow_traversal_bytes_per_path"] * npaths + SHADOW_QUEUE_BYTES * shadow / args.steps
                traffic = None
            else:
                alg = per_path * npaths
                traffic = None
            achieved = alg / (top_ms / 1000) / 1e9
            if top_kernel == "wf_extend" and args.workload == "sky":
                roof["issue"] = profiled_issue()
            roof.update(achieved=achieved, frac=achieved / hbm, traffic=traffic,
                        algorithmic_bytes_per_launch=alg / top_launches, algorithmic_bytes_per_path=per_path,
                        **counts)
            cpu = cpu_baseline(args, s, built, r.spec, r.hosek, r.camera, args.cpu_seconds)
        rmse = None
        if not args.no_rmse:
            h = path.h
            rows = list(range(h)) if args.workload == "room" else [int(h * (k + 1) / 5) for k in range(4)]
            rmse = rmse_vs_fp64(r, imgs, args.spp, rows)
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator, random-init sky)",
                "config": {"workload": SCENES[args.workload][2], "integrator": args.integrator, "width": path.w,
                           "height": path.h, "spp": args.spp, "bounces": s.render["bounces"],
                           "triangles": s.num_triangles,
                           "intersector": "watertight", "film": "kahan",
                           "l2": "inputs larger than L2 (scene ~0.5 GB resident)",
                           "parallelism": f"replicas{world}", "bvh_build_s": round(build_s, 2), "bvh_build": bvh_build,
                           **path.describe()},
                "mrays_per_s": mrays, "rays_per_step": (ext + shadow) / args.steps, "ext_rays_per_step": ext / args.steps,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "rmse_vs_fp64": rmse,
                "gpu_launches": launches, "clocks": clocks, "other_integrator": compare}
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

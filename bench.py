"""Benchmark of the B200 path-tracing core (one JSON line on rank 0).

Workload: the reference's throughput configuration — 64 fBm-displaced
icospheres (1 310 722 triangles) on a ground plane, area light + sun, Disney
materials, 1920x1080, 256 spp, max depth 12 (synthetic, seeded). One step is
one full frame render (530 841 600 camera samples). The scene (~95 MB of
nodes and triangles) is resident in HBM before the timed region; L2 is
flushed between steps by writing a 256 MiB buffer.

  value  : Msamples/s over the K timed steps, device time from CUDA events on
           the library's launching stream (max over ranks; whole-job total).
  e2e    : the same metric through rt_render with a HOST film buffer: the
           per-step render parameters go in, the 24.9 MB linear-HDR film comes
           back to pinned host memory, both inside the timed region.
  roofline: algorithmic bytes per sample (reference BVH2 traversal: 32 B per
           node visit, 36 B per triangle test, 64 B per quad/sphere test,
           96 B per path segment), counted on the GPU by the counting build
           over a fixed pixel subsample, times samples per launch, divided by
           the render kernel's average launch time, against measured HBM.
  cpu_baseline: the oracle (C++ restatement of 3d-ray's C# loop) on all host
           cores over a bounded pixel window of the same frame.

Multi-GPU: rendering does not shard in the reference (one process, one
frame); `--gpus N` runs N independent replicas, one full frame per rank per
step ("scaling": "weak"), with only a barrier and a max-reduce of the timings.

`--impl reference` times the reference's CPU path (the oracle port: 3d-ray's
C# cannot run here) on the same configuration and metric.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Msamples/s and time to relMSE 1e-3 on 1 B200: batched wavefront vs plain kernel"
UNIT = "Msamples/s"
W, H, SPP, DEPTH = 1920, 1080, 256, 12


def load_package():
    import importlib.util
    if "rt3d_b200" in sys.modules:
        return sys.modules["rt3d_b200"]
    d = os.path.join(ROOT, "3d-ray_b200")
    spec = importlib.util.spec_from_file_location("rt3d_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    m = importlib.util.module_from_spec(spec)
    sys.modules["rt3d_b200"] = m
    spec.loader.exec_module(m)
    return m


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) >= 9:
                for k, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_setup(n_gpus, backend=None):
    """One process per GPU (torchrun): replicas that meet only at a barrier and
    a max-reduce of their timings. NCCL on GPUs; gloo when there is no GPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return dist.get_rank(), world, dist


def max_over_ranks(x: float, dist) -> float:
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world_size: int, units_per_step: float, steps: int, total_ms: float) -> float:
    """Whole-job throughput in millions of units per second: every rank renders
    the same frame, and the job takes as long as its slowest rank (total_ms is
    the max over ranks)."""
    return world_size * units_per_step * steps / (total_ms / 1e3) / 1e6


def barrier(dist):
    if dist is not None:
        dist.barrier()


def build_world():
    rt = load_package()
    return rt, rt.scenes.throughput_scene()


def oracle_scene(rt, world):
    from oracle import binding
    binding.build()
    return binding.OracleScene(rt.abi.PackedWorld(world))


def cpu_baseline(rt, world, budget_s=12.0, osc=None, runs=5):
    """Times the oracle on a bounded sample of the same frame (the scene build,
    like the reference's, is outside the timing): full-width pixel rows spread
    evenly over the frame's height, so the sample has the frame's mix of cheap
    and expensive pixels. An untimed warm-up, then the median of `runs` timed
    passes, sized so the passes take about budget_s together."""
    own = osc is None
    if own:
        osc = oracle_scene(rt, world)
    cores = os.cpu_count() or 1

    def row(y):
        return rt.abi.render_params(W, H, SPP, DEPTH, pixel_x0=0, pixel_y0=y, window_w=W, window_h=1)

    # warm-up and calibration on two rows
    cal = [row(H // 3), row(2 * H // 3)]
    t = time.perf_counter()
    for p in cal:
        osc.render(p, threads=cores)
    rate = 2 * W * SPP / (time.perf_counter() - t)
    nrows = int(max(2, min(64, budget_s / runs * rate / (W * SPP))))
    rows = [row(int((k + 0.5) * H / nrows)) for k in range(nrows)]
    times = []
    for _ in range(runs):
        t = time.perf_counter()
        for p in rows:
            osc.render(p, threads=cores)
        times.append(time.perf_counter() - t)
    dt = statistics.median(times)
    samples = nrows * W * SPP
    if own:
        osc.close()
    try:
        import cpuinfo
        model = cpuinfo.get_cpu_info().get("brand_raw", "")
    except Exception:
        model = ""
    return {"value": samples / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port", "cpu": model,
            "sample": f"{nrows} full-width rows evenly spread over the 1920x1080 frame at {SPP} spp, depth {DEPTH} "
                      f"({samples} samples per pass; median of {runs} passes after a warm-up, {dt:.2f} s each)"}


def run_reference(args):
    # The reference path is a CPU renderer: rank 0 alone runs it, other ranks exit.
    if int(os.environ.get("RANK", "0")) != 0:
        return
    rt, world = build_world()
    osc = oracle_scene(rt, world)
    per = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(rt, world, budget_s=8.0, osc=osc)
        if i >= args.warmup:
            per.append(b["value"])
            base = b
    v = float(np.mean(per))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "icospheres-64x20480 1920x1080 256spp depth12 (CPU sample window)",
                       "triangles": world.num_tris},
            "cpu_baseline": dict(base, value=v),
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def flush_l2(torch_mod, buf):
    buf.fill_(1)


def rel_mse(x, r):
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


def time_to_relmse_on(lib, abi, h, width, height, depth, window=None, target=1e-3,
                      kernels=("wavefront", "megakernel")):
    """Seconds of device time until a render reaches relMSE <= target against
    a 65 536-spp wavefront reference of the same frame (or window), rendered
    from a disjoint Sobol range so that it is uncorrelated with the test
    images; spp doubles from 16. For the two frames measured here (the Cornell
    box and the icosphere window), tests/test_image_parity.py renders this
    reference and holds it to a committed 4096-sample oracle render of the
    frame at the oracle's noise floor."""
    import torch
    x0, y0, ww, wh = window or (0, 0, width, height)
    win = dict(pixel_x0=x0, pixel_y0=y0, window_w=ww, window_h=wh) if window else {}
    film = torch.empty((3, height, width), dtype=torch.float32, device="cuda")
    st = abi.RtStats()
    ref_spp = 65536
    p = abi.render_params(width, height, ref_spp, depth, kernel=abi.KERNEL_WAVEFRONT, spp_offset=1 << 20, **win)
    abi.check(lib.rt_render_device(h, C.byref(p), C.c_void_p(film.data_ptr()), C.byref(st)), "reference")
    ref = film[:, y0:y0 + wh, x0:x0 + ww].cpu().numpy().copy()
    out = {"reference_spp": ref_spp, "reference_seconds": st.kernel_ms / 1e3, "target": target}
    for kname in kernels:
        kid = abi.KERNEL_WAVEFRONT if kname == "wavefront" else abi.KERNEL_MEGAKERNEL
        spp = 16
        while spp <= 16384:
            p = abi.render_params(width, height, spp, depth, kernel=kid, **win)
            abi.check(lib.rt_render_device(h, C.byref(p), C.c_void_p(film.data_ptr()), C.byref(st)), kname)
            e = rel_mse(film[:, y0:y0 + wh, x0:x0 + ww].cpu().numpy(), ref)
            if e <= target:
                out[kname] = {"seconds": st.kernel_ms / 1e3, "spp": spp, "rel_mse": e}
                break
            spp *= 2
    if "wavefront" in out and "megakernel" in out:
        out["speedup_wavefront"] = out["megakernel"]["seconds"] / out["wavefront"]["seconds"]
    return out


def time_to_relmse(rt, lib, abi):
    """Cornell box 256x256, depth 8 (the C1 frame at the configuration's size)."""
    pw = abi.PackedWorld(rt.scenes.cornell())
    h = C.c_void_p()
    abi.check(lib.rt_scene_create(pw.ref(), C.byref(h)), "rt_scene_create")
    try:
        out = {"workload": "cornell 256x256 depth 8"}
        out.update(time_to_relmse_on(lib, abi, h, 256, 256, 8))
    finally:
        lib.rt_scene_destroy(h)
    return out


def profile_frame(args):
    """One warm-up and one measured frame with fixed wavefront settings (4M
    slots, block 256, material sort) or the megakernel: the workload the ncu
    summaries under profiles/ were captured on."""
    rt, world = build_world()
    abi = rt.abi
    lib = abi.load()
    pw = abi.PackedWorld(world)
    scene = C.c_void_p()
    abi.check(lib.rt_scene_create(pw.ref(), C.byref(scene)), "rt_scene_create")
    kern = abi.KERNEL_WAVEFRONT if args.kernel == "wavefront" else abi.KERNEL_MEGAKERNEL
    p = abi.render_params(W, H, args.spp, DEPTH, kernel=kern, wavefront_size=1 << 22, block_size=256,
                          trace_block_size=args.block,
                          sort_materials=1, node_layout=args.node_layout, ray_fetch=args.ray_fetch,
                          ray_groups=args.ray_groups, profile_kernels=int(args.split))
    film = np.zeros((3, H, W), np.float32)
    st = abi.RtStats()
    for i in range(2):
        abi.check(lib.rt_render(scene, C.byref(p), film.ctypes.data_as(C.c_void_p), C.byref(st)), "rt_render")
        line = {"frame": i, "kernel": args.kernel, "node_layout": args.node_layout, "ray_fetch": args.ray_fetch,
                "ray_groups": args.ray_groups,
                "spp": args.spp,
                "kernel_ms": st.kernel_ms, "Msamples_per_s": W * H * args.spp / st.kernel_ms / 1e3,
                "iterations": st.iterations, "launches": st.kernel_launches}
        if args.split:
            line.update(regen_ms=st.regen_ms, extend_ms=st.extend_ms, sort_ms=st.sort_ms, shade_ms=st.shade_ms,
                        occlude_ms=st.occlude_ms)
        print(json.dumps(line), flush=True)
    lib.rt_scene_destroy(scene)


def profile_adjoint(args):
    """The C4 fit's adjoint call (256x256, 32 spp, depth 8, the sphere's
    seven BSDF slots) twice, in the --adjoint-kernel form: the workload the
    adjoint's ncu summaries under profiles/ were captured on."""
    rt = load_package()
    abi = rt.abi
    sphere = dict(base_color=(0.6, 0.3, 0.2), roughness=0.4, metallic=0.2, specular=0.6, sheen=0.3)
    ds = rt.DiffScene(rt.scenes.cornell_sphere(sphere))
    slots = [ds.slot("fit_sphere", "base_color", c) for c in range(3)]
    slots += [ds.slot("fit_sphere", n) for n in ("roughness", "metallic", "specular", "sheen")]
    res, spp = 256, 32
    wimg = np.random.default_rng(2).uniform(0, 1, (3, res, res)).astype(np.float32)
    rp = abi.render_params(res, res, spp, 8, kernel=adjoint_kernel(args))
    for i in range(2):
        g = ds.adjoint(rp, wimg, slots)
        st = ds.last_stats
        print(json.dumps({"call": i, "adjoint_kernel": args.adjoint_kernel, "kernel_ms": st.kernel_ms,
                          "Msamples_per_s": res * res * spp / st.kernel_ms / 1e3, "launches": st.kernel_launches,
                          "finite": bool(np.isfinite(g).all())}), flush=True)
    ds.close()


def c1_side(rt, lib, abi):
    """C1: the Cornell box at 256x256, 64 spp, depth 8: the plain megakernel
    and the autotuned wavefront (device time, third of three renders), and the
    oracle on all host cores over a 256x64 band (median of 3)."""
    world = rt.scenes.cornell()
    pw = abi.PackedWorld(world)
    h = C.c_void_p()
    abi.check(lib.rt_scene_create(pw.ref(), C.byref(h)), "rt_scene_create")
    film = np.zeros((3, 256, 256), np.float32)
    out = {"workload": "cornell 256x256 64spp depth 8"}
    base = abi.render_params(256, 256, 64, 8, kernel=abi.KERNEL_WAVEFRONT)
    best = abi.RtRenderParams()
    abi.check(lib.rt_autotune(h, C.byref(base), C.byref(best)), "rt_autotune")
    for name, kern in (("megakernel", abi.KERNEL_MEGAKERNEL), ("wavefront", abi.KERNEL_WAVEFRONT)):
        p = abi.render_params(256, 256, 64, 8, kernel=kern)
        st = abi.RtStats()
        for _ in range(3):
            abi.check(lib.rt_render(h, C.byref(p), film.ctypes.data_as(C.c_void_p), C.byref(st)), "c1")
        out[name] = 256 * 256 * 64 / st.kernel_ms / 1e3
    lib.rt_scene_destroy(h)
    osc = oracle_scene(rt, world)
    p = abi.render_params(256, 256, 64, 8, pixel_x0=0, pixel_y0=96, window_w=256, window_h=64)
    cores = os.cpu_count() or 1
    osc.render(p, threads=cores)
    ts = []
    for _ in range(3):
        t = time.perf_counter()
        osc.render(p, threads=cores)
        ts.append(time.perf_counter() - t)
    osc.close()
    out["cpu_port"] = 256 * 64 * 64 / statistics.median(ts) / 1e6
    out["unit"] = UNIT
    out["cores"] = cores
    return out


def bvh_build_side(lib, abi, pw):
    """The bench scene's mesh BVHs: the device build against the host build on
    every host thread (wall time of the mesh-BVH phase of scene creation,
    triangle upload and node download included), and whether the two trees are
    the same bit for bit."""
    def export(h, info):
        nodes = np.zeros((info.num_nodes, 8), np.int32)
        order = np.zeros(info.num_tris, np.int32)
        abi.check(lib.rt_scene_export_bvh(h, abi.ptr(nodes), nodes.shape[0], None, 0, abi.ptr(order), order.size))
        return nodes, order

    hinfo = abi.RtSceneInfo()
    abi.check(lib.rt_world_inspect(pw.ref(), C.byref(hinfo), None, 0, None, 0, None, 0), "rt_world_inspect")
    hn = np.zeros((hinfo.num_nodes, 8), np.int32)
    ho = np.zeros(hinfo.num_tris, np.int32)
    abi.check(lib.rt_world_inspect(pw.ref(), C.byref(hinfo), abi.ptr(hn), hn.shape[0], None, 0, abi.ptr(ho), ho.size))
    runs = []
    same = True
    for _ in range(2):   # the first build in a process also loads its kernels
        opt = abi.RtSceneOptions()
        opt.bvh_build = abi.BVH_DEVICE
        h = C.c_void_p()
        abi.check(lib.rt_scene_create_ex(pw.ref(), C.byref(opt), C.byref(h)), "rt_scene_create_ex")
        info = abi.RtSceneInfo()
        abi.check(lib.rt_scene_info(h, C.byref(info)))
        dn, do = export(h, info)
        lib.rt_scene_destroy(h)
        same = same and bool(info.bvh_on_device) and np.array_equal(dn, hn) and np.array_equal(do, ho)
        runs.append(info.bvh_build_ms)
    return {"triangles": int(hinfo.num_tris), "nodes": int(hinfo.num_nodes), "device_ms": runs[-1],
            "device_first_ms": runs[0], "host_ms": hinfo.bvh_build_ms, "host_threads": os.cpu_count(),
            "speedup": hinfo.bvh_build_ms / runs[-1], "identical": same}


def batched_side(rt):
    """C3 (32 requests of uneven resolution, spp and depth over the icosphere
    field and the Cornell box) and C5 (eight 512x512 views of the box with the
    medium and the glass sphere, 512 spp, depth 16), each as one persistent
    batched wavefront launch; device time."""
    out = {}
    reqs = rt.scenes.batch_requests()
    films, st = rt.render_batch(reqs, [rt.scenes.throughput_scene(), rt.scenes.cornell()])
    n = sum(r["width"] * r["height"] * r["spp"] for r in reqs)
    out["c3_batch"] = {"requests": len(reqs), "samples": n, "seconds": st.kernel_ms / 1e3,
                       "msamples_per_s": n / st.kernel_ms / 1e3, "launches": st.kernel_launches}
    reqs5 = [dict(scene=0, width=512, height=512, spp=512, max_depth=16, camera=c)
             for c in rt.scenes.volume_views()]
    films, st = rt.render_batch(reqs5, [rt.scenes.cornell_volume()])
    n = sum(r["width"] * r["height"] * r["spp"] for r in reqs5)
    out["c5_views"] = {"views": len(reqs5), "samples": n, "seconds": st.kernel_ms / 1e3,
                       "msamples_per_s": n / st.kernel_ms / 1e3,
                       "finite": bool(all(np.isfinite(f).all() for f in films))}
    out["adjoint"] = adjoint_side(rt)
    return out


def adjoint_side(rt):
    """The path-replay adjoint (rt_adjoint) in both forms, device time of
    both passes: C4 at the fit's call (256x256, 32 spp, depth 8, the sphere's
    seven BSDF slots) and C5 at 64x64, 256 spp, depth 16 (the medium's six
    slots), the second of two calls each."""
    abi = rt.abi
    out = {}
    sphere = dict(base_color=(0.6, 0.3, 0.2), roughness=0.4, metallic=0.2, specular=0.6, sheen=0.3)
    for name, world, res, spp, depth in (("c4_256x256_32spp_bsdf7", rt.scenes.cornell_sphere(sphere), 256, 32, 8),
                                         ("c5_64x64_256spp_medium6", rt.scenes.cornell_volume(), 64, 256, 16)):
        ds = rt.DiffScene(world)
        if name.startswith("c4"):
            slots = [ds.slot("fit_sphere", "base_color", c) for c in range(3)]
            slots += [ds.slot("fit_sphere", n) for n in ("roughness", "metallic", "specular", "sheen")]
        else:
            slots = [ds.medium_slot(k, c) for k in ("sigma_a", "sigma_s") for c in range(3)]
        wimg = np.random.default_rng(2).uniform(0, 1, (3, res, res)).astype(np.float32)
        row = {}
        for kname, kern in (("megakernel", abi.KERNEL_MEGAKERNEL), ("wavefront", abi.KERNEL_WAVEFRONT)):
            rp = abi.render_params(res, res, spp, depth, kernel=kern)
            for _ in range(2):
                ds.adjoint(rp, wimg, slots)
            row[kname] = res * res * spp / ds.last_stats.kernel_ms / 1e3
        row["unit"] = "Msamples/s"
        row["speedup_wavefront"] = row["wavefront"] / row["megakernel"]
        out[name] = row
        ds.close()
    return out


def adjoint_kernel(args):
    """The rt_adjoint form --adjoint-kernel names."""
    abi = load_package().abi
    return abi.KERNEL_WAVEFRONT if args.adjoint_kernel == "wavefront" else abi.KERNEL_MEGAKERNEL


def gradcheck(args):
    """The path-replay adjoint against central finite differences under common
    random numbers: C4 (the Cornell box with a Disney sphere: the sphere's
    baseColor, roughness, metallic, specular and sheen, and the emitter's
    radiance, with the reference's luminance clamps), C5 (the medium's
    sigma_a and sigma_s and the glass sphere's absorption) and the absorption
    of a glass sphere of optical depth ~1 under the flat sky (C5's glass, 90
    units of radius at sigma_a (0.1, 0.3, 0.5), passes e^-18 of the light or
    less, so its absorption gradient is close to zero).

    Each parameter gets its own linear loss L = sum(w * film), with w the sign
    of that parameter's finite-difference image from an independent pilot
    render: every pixel's change then adds to the gradient instead of partly
    cancelling, so the gradient stands well above the sampling noise (a fixed
    weighting: the pilot's samples are disjoint from the check's). The check's
    samples are split into 8 independent Sobol batches; in each, the adjoint
    (rt_adjoint) and the central difference of two wavefront renders of the
    same samples at theta +- eps estimate dL/dtheta. Per parameter the line
    gives both means, their relative difference, the standard error of the
    per-batch difference and of each estimate, all relative to the
    finite-difference mean."""
    rt = load_package()
    abi = rt.abi
    spp = args.spp if args.spp != SPP else 16384
    nb = 8
    only = [x for x in args.gc_params.split(",") if x] if args.gc_params else []
    sphere = dict(base_color=(0.6, 0.3, 0.2), roughness=0.4, metallic=0.2, specular=0.6, sheen=0.3)
    for name in ("c4", "c5", "glass"):
        if only and not any(o.startswith(name + ":") for o in only):
            continue
        if name == "c4":
            w = rt.scenes.cornell_sphere(sphere)
            res, depth = 64, 8
        elif name == "c5":
            w = rt.scenes.cornell_volume()
            res, depth = 48, 16
        else:   # a glass sphere of optical depth ~1 under the sky (C5's glass transmits e^-18 and less)
            w = rt.scenes.sky_scene()
            res, depth = 48, 8
        ds = rt.DiffScene(w)
        kw = dict(max_sample_radiance=1e30, indirect_clamp_factor=1.0) if args.gc_no_clamps else {}
        if args.gc_no_rr:   # Russian roulette never starts within the depth
            kw["rr_min_bounces"] = 1000
        per = max(spp // nb, 1)
        # the finite differences may take more samples per batch than the
        # adjoint (the adjoint's are the first of them), and a larger eps
        fper = max(per, args.gc_fd_spp // nb) if args.gc_fd_spp else per
        rp = abi.render_params(res, res, per, depth, kernel=adjoint_kernel(args), **kw)
        rw = abi.render_params(res, res, fper, depth, kernel=abi.KERNEL_WAVEFRONT, **kw)
        pilot = abi.render_params(res, res, 2048, depth, kernel=abi.KERNEL_WAVEFRONT, spp_offset=1 << 24, **kw)
        theta = ds.get_params()
        if name == "c4":
            slots = {f"sphere.base_color[{c}]": (ds.slot("fit_sphere", "base_color", c), 1e-3) for c in range(3)}
            for n in ("roughness", "metallic", "specular", "sheen"):
                slots[f"sphere.{n}"] = (ds.slot("fit_sphere", n), 1e-2)
            for c in range(3):
                i = ds.slot("light", "radiance", c)
                slots[f"light.radiance[{c}]"] = (i, 1e-3 * float(theta[i]))
        elif name == "c5":
            slots = {}
            for c in range(3):
                for nm in ("sigma_a", "sigma_s"):
                    i = ds.medium_slot(nm, c)
                    slots[f"medium.{nm}[{c}]"] = (i, 1e-2 * float(theta[i]))
                i = ds.slot("glass", "absorption", c)
                slots[f"glass.absorption[{c}]"] = (i, 1e-2 * float(theta[i]))
                # the single-scattering albedo at a fixed sigma_t: sigma_s = albedo * sigma_t,
                # sigma_a = (1 - albedo) * sigma_t, a direction in the parameter vector
                dirs = ds.medium_albedo_direction(theta, c)
                isc = ds.medium_slot("sigma_s", c)
                slots[f"medium.albedo[{c}]"] = (list(dirs.items()), 1e-2 * float(theta[isc]) / dirs[isc])
        else:
            slots = {f"glass.absorption[{c}]": (ds.slot("glass", "absorption", c),
                                                1e-2 * float(theta[ds.slot("glass", "absorption", c)]))
                     for c in range(3)}

        if only:
            slots = {k: (i, e * args.gc_eps) for k, (i, e) in slots.items()
                     if any(o == f"{name}:{k}" for o in only)}

        def film_at(dirs, h, p):   # the film at theta + h * (the direction dirs)
            th = theta.copy()
            for j, c in dirs:
                th[j] = np.float32(float(theta[j]) + h * c)
            ds.set_params(th)
            return ds.render(p).astype(np.float64)

        rows = {}
        adj_ms, t0 = 0.0, time.time()
        for key, (i, eps) in slots.items():
            dirs = i if isinstance(i, list) else [(i, 1.0)]
            if args.gc_loss == "sum":   # L = the sum of the film: one loss for every setting of the renderer
                wimg = np.ones((3, res, res), np.float32)
            else:
                d = film_at(dirs, eps, pilot) - film_at(dirs, -eps, pilot)
                wimg = np.sign(d).astype(np.float32)
            adj = np.zeros(nb)
            fd = np.zeros(nb)
            for b in range(nb):
                rp.spp_offset = rw.spp_offset = b * fper
                ds.set_params(theta)
                g = ds.adjoint(rp, wimg, [j for j, _ in dirs])
                adj[b] = sum(c * float(g[j]) for j, c in dirs)
                adj_ms += ds.last_stats.kernel_ms
                lp = float((film_at(dirs, eps, rw) * wimg).sum())
                lm = float((film_at(dirs, -eps, rw) * wimg).sum())
                fd[b] = (lp - lm) / (2.0 * eps)
                if args.gc_richardson:   # (4 D(eps) - D(2 eps)) / 3 cancels the eps^2 term
                    lp2 = float((film_at(dirs, 2 * eps, rw) * wimg).sum())
                    lm2 = float((film_at(dirs, -2 * eps, rw) * wimg).sum())
                    fd[b] = (4.0 * fd[b] - (lp2 - lm2) / (4.0 * eps)) / 3.0
            ds.set_params(theta)
            diff = adj - fd
            ma, mf = float(adj.mean()), float(fd.mean())
            den = max(abs(mf), 1e-30)
            se = float(diff.std(ddof=1) / np.sqrt(nb))
            rows[key] = {"adjoint": ma, "fd": mf, "eps": eps, "rel_err": abs(ma - mf) / den,
                         "diff_stderr_rel": se / den, "z": float(diff.mean() / se) if se > 0 else 0.0,
                         "adjoint_stderr_rel": float(adj.std(ddof=1) / np.sqrt(nb)) / den,
                         "fd_stderr_rel": float(fd.std(ddof=1) / np.sqrt(nb)) / den}
        n = res * res * per * nb
        print(json.dumps({"gradcheck": name, "clamps": not args.gc_no_clamps, "roulette": not args.gc_no_rr,
                          "image": f"{res}x{res}", "loss_kind": args.gc_loss, "adjoint_kernel": args.adjoint_kernel,
                          "samples_per_param": n,
                          "richardson": bool(args.gc_richardson),
                          "fd_samples_per_param": res * res * fper * nb,
                          "batches": nb, "loss": "sign of the pilot finite-difference image, per parameter",
                          "adjoint_msamples_per_s": n * len(slots) / adj_ms / 1e3, "seconds": time.time() - t0,
                          "params": rows}), flush=True)
        ds.close()


def fit(args):
    """C4: recover the sphere's Disney parameters (baseColor, roughness,
    metallic, specular, sheen) and the emitter radiance from a 1024-spp target
    rendered with seeded ground truth drawn uniformly in valid ranges. Adam,
    lr 1e-2, 200 steps of 32 spp, L2 loss on the 256x256 HDR film; gradients
    from rt_adjoint. The radiance is optimised as its logarithm (Adam moves a
    parameter by about lr per step, and radiance is O(10)). Each step uses a
    fresh Sobol range (spp_offset), so the fit sees independent samples."""
    import torch
    rt = load_package()
    abi = rt.abi
    steps = args.steps if args.steps != 3 else 200
    rng = np.random.default_rng(2024)
    names = ["base_color", "base_color", "base_color", "roughness", "metallic", "specular", "sheen"]
    chans = [0, 1, 2, 0, 0, 0, 0]

    def draw():
        return np.concatenate([rng.uniform(0.05, 0.95, 3), rng.uniform(0.05, 1.0, 1), rng.uniform(0.0, 1.0, 1),
                               rng.uniform(0.0, 1.0, 1), rng.uniform(0.0, 1.0, 1)]).astype(np.float32), \
            (np.array([17.0, 12.0, 4.0]) * rng.uniform(0.6, 1.4, 3)).astype(np.float32)

    truth_s, truth_e = draw()
    init_s, init_e = draw()
    ds = rt.DiffScene(rt.scenes.cornell_sphere())
    theta0 = ds.get_params()
    s_idx = [ds.slot("fit_sphere", n, c) for n, c in zip(names, chans)]
    e_idx = [ds.slot("light", "radiance", c) for c in range(3)]

    def vec(sv, ev):
        th = theta0.copy()
        th[s_idx] = sv
        th[e_idx] = ev
        return th

    res = args.res
    ds.set_params(vec(truth_s, truth_e))
    tp = abi.render_params(res, res, 1024, 8, kernel=abi.KERNEL_WAVEFRONT, spp_offset=1 << 24)
    target = ds.render(tp)
    x_s = torch.tensor(init_s, dtype=torch.float64, requires_grad=True)
    x_le = torch.tensor(np.log(init_e), dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([x_s, x_le], lr=1e-2)
    mask = s_idx + e_idx
    hist, hist_truth, traj = [], [], []
    keys = ["base_r", "base_g", "base_b", "roughness", "metallic", "specular", "sheen"]
    t0 = time.perf_counter()
    adj_ms = 0.0
    for it in range(steps):
        if it >= steps - 10:   # the loss the ground truth gets on the same samples
            ds.set_params(vec(truth_s, truth_e))
            rp = abi.render_params(res, res, 32, 8, kernel=adjoint_kernel(args), spp_offset=it * 32)
            hist_truth.append(float(((ds.render(rp).astype(np.float64) - target) ** 2).mean()))
        sv = x_s.detach().numpy().astype(np.float32)
        ev = np.exp(x_le.detach().numpy()).astype(np.float32)
        if it % 20 == 0:   # the trajectory: every parameter's error before step it
            traj.append({"step": it, **{k: round(float(abs(a - b)), 4) for k, a, b in zip(keys, sv, truth_s)},
                         **{f"radiance_{c}": round(float(abs(ev[c] / truth_e[c] - 1)), 4) for c in range(3)}})
        ds.set_params(vec(sv, ev))
        # the forward film on the wavefront, the adjoint on the same samples
        rw = abi.render_params(res, res, 32, 8, kernel=abi.KERNEL_WAVEFRONT, spp_offset=it * 32)
        rp = abi.render_params(res, res, 32, 8, kernel=adjoint_kernel(args), spp_offset=it * 32)
        img = ds.render(rw)
        diff = img.astype(np.float64) - target
        loss = float((diff ** 2).mean())
        g = ds.adjoint(rp, (2.0 * diff / diff.size).astype(np.float32), mask)
        adj_ms += ds.last_stats.kernel_ms
        opt.zero_grad()
        x_s.grad = torch.from_numpy(g[s_idx].astype(np.float64))
        x_le.grad = torch.from_numpy(g[e_idx].astype(np.float64) * ev)   # d/dlog e = e d/de
        opt.step()
        with torch.no_grad():
            x_s.clamp_(0.0, 1.0)
        hist.append(loss)
    wall = time.perf_counter() - t0
    final_s = x_s.detach().numpy()
    final_e = np.exp(x_le.detach().numpy())
    print(json.dumps({
        "fit": "c4", "image": f"{res}x{res}", "steps": steps, "spp_per_step": 32, "lr": 1e-2, "target_spp": 1024,
        "adjoint_kernel": args.adjoint_kernel,
        "loss_first": hist[0], "loss_last10_mean": float(np.mean(hist[-10:])),
        "loss_at_truth_last10_mean": float(np.mean(hist_truth)),
        "param_abs_err_init": dict(zip(keys, map(float, np.abs(init_s - truth_s)))),
        "param_abs_err_final": dict(zip(keys, map(float, np.abs(final_s - truth_s)))),
        "radiance_rel_err_init": list(map(float, np.abs(init_e / truth_e - 1))),
        "radiance_rel_err_final": list(map(float, np.abs(final_e / truth_e - 1))),
        "seconds": wall, "adjoint_ms_per_step": adj_ms / steps,
        "loss_curve": [float(h) for h in hist[::max(1, steps // 10)]], "trajectory": traj}), flush=True)
    ds.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--kernel", default="wavefront", choices=["megakernel", "wavefront"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-kernel and relMSE side measurements")
    ap.add_argument("--spp", type=int, default=SPP)
    ap.add_argument("--node-layout", type=int, default=2, choices=[2, 4],
                    help="BVH records for --profile-frame: two-wide or four-wide")
    ap.add_argument("--split", action="store_true", help="--profile-frame: per-kernel event times")
    ap.add_argument("--block", type=int, default=256, choices=[64, 128, 256],
                    help="--profile-frame: block size of extend/occlude (the others use 256)")
    ap.add_argument("--ray-fetch", type=int, default=1, choices=[1, 2],
                    help="--profile-frame: one ray per thread (1) or persistent dynamic fetch (2)")
    ap.add_argument("--ray-groups", type=int, default=1, choices=[1, 2, 3, 4],
                    help="--profile-frame: rays in slot order (1), regrouped by kind in each block (2), bounce rays sorted by origin and direction (3), bounce and shadow rays sorted (4)")
    ap.add_argument("--fit", action="store_true", help="the C4 inverse-rendering fit (Adam on rt_adjoint) and exit")
    ap.add_argument("--adjoint-kernel", default="wavefront", choices=["megakernel", "wavefront"],
                    help="--fit / --gradcheck: the rt_adjoint form (the same gradient; the wavefront form is 7-16x faster)")
    ap.add_argument("--res", type=int, default=256, help="--fit: square image size")
    ap.add_argument("--gradcheck", action="store_true",
                    help="adjoint gradients against central finite differences (C4, C5) and exit")
    ap.add_argument("--gc-params", default="",
                    help="--gradcheck: only these parameters, e.g. c4:sphere.roughness,c5:medium.sigma_s[0]")
    ap.add_argument("--gc-fd-spp", type=int, default=0,
                    help="--gradcheck: samples per pixel of the finite differences over all batches (default --spp)")
    ap.add_argument("--gc-eps", type=float, default=1.0, help="--gradcheck with --gc-params: eps multiplier")
    ap.add_argument("--gc-no-clamps", action="store_true",
                    help="--gradcheck: without the luminance clamps (maximum sample radiance, indirect clamp)")
    ap.add_argument("--gc-no-rr", action="store_true", help="--gradcheck: Russian roulette off")
    ap.add_argument("--gc-loss", default="sign", choices=["sign", "sum"],
                    help="--gradcheck: per-parameter sign-weighted loss, or the plain sum of the film")
    ap.add_argument("--gc-richardson", action="store_true",
                    help="--gradcheck: Richardson-extrapolated differences (4 D(eps) - D(2 eps)) / 3")
    ap.add_argument("--bvh-build", action="store_true",
                    help="build the bench scene's mesh BVHs on the host and twice on the device, print the timings "
                         "and exit (the command profiled by ncu for the device build)")
    ap.add_argument("--profile-frame", action="store_true",
                    help="render the frame twice with fixed settings and exit (the command profiled by ncu)")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="the C4 fit's adjoint call twice (--adjoint-kernel form) and exit (the command profiled by ncu)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_frame:
        return profile_frame(args)
    if args.profile_adjoint:
        return profile_adjoint(args)
    if args.bvh_build:
        rt, world = build_world()
        lib = rt.abi.load()
        print(json.dumps(bvh_build_side(lib, rt.abi, rt.abi.PackedWorld(world))), flush=True)
        return
    if args.gradcheck:
        return gradcheck(args)
    if args.fit:
        return fit(args)

    import torch
    rank, world_size, dist = dist_setup(args.gpus)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    rt, world = build_world()
    abi = rt.abi
    lib = abi.load()
    pw = abi.PackedWorld(world)
    scene = C.c_void_p()
    abi.check(lib.rt_scene_create(pw.ref(), C.byref(scene)), "rt_scene_create")
    spp = args.spp
    kern = abi.KERNEL_WAVEFRONT if args.kernel == "wavefront" else abi.KERNEL_MEGAKERNEL
    params = abi.render_params(W, H, spp, DEPTH, kernel=kern)
    tuned = None
    if kern == abi.KERNEL_WAVEFRONT:   # setup, outside the timed region (like the BVH build)
        best = abi.RtRenderParams()
        abi.check(lib.rt_autotune(scene, C.byref(params), C.byref(best)), "rt_autotune")
        tuned = {"wavefront_size": best.wavefront_size, "block_size": best.block_size,
                 "sort_materials": best.sort_materials, "node_layout": best.node_layout,
                 "ray_fetch": best.ray_fetch, "trace_block_size": best.trace_block_size,
                 "ray_groups": best.ray_groups}
    film = torch.empty((3, H, W), dtype=torch.float32, device="cuda")
    l2 = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(p, steps, warmup):
        st = abi.RtStats()
        for _ in range(warmup):
            abi.check(lib.rt_render_device(scene, C.byref(p), C.c_void_p(film.data_ptr()), C.byref(st)), "warmup")
            flush_l2(torch, l2)
        torch.cuda.synchronize()
        barrier(dist)
        torch.cuda.synchronize()
        times, launches = [], 0
        for _ in range(steps):
            abi.check(lib.rt_render_device(scene, C.byref(p), C.c_void_p(film.data_ptr()), C.byref(st)), "step")
            times.append(st.kernel_ms)
            launches += st.kernel_launches
            flush_l2(torch, l2)
        torch.cuda.synchronize()
        barrier(dist)
        torch.cuda.synchronize()
        return max_over_ranks(float(sum(times)), dist), launches

    with ClockSampler(dev) as clk:
        total_ms, launches = timed(params, args.steps, args.warmup)
    samples_per_step = W * H * spp
    value = aggregate_rate(world_size, samples_per_step, args.steps, total_ms)
    ms_per_step = total_ms / args.steps

    # e2e: public API with host buffers (film read back to pinned memory).
    host_film = torch.empty((3, H, W), dtype=torch.float32).pin_memory()
    e2e_times, e2e_dev = [], []
    st2 = abi.RtStats()
    with ClockSampler(dev) as clk2:
        for i in range(args.steps + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            abi.check(lib.rt_render(scene, C.byref(params), C.c_void_p(host_film.data_ptr()), C.byref(st2)),
                      "rt_render")
            dt = time.perf_counter() - t0
            if i > 0:
                e2e_times.append(dt)
                e2e_dev.append(st2.kernel_ms)
            flush_l2(torch, l2)   # outside the host-timed call
    e2e_total = max_over_ranks(float(sum(e2e_times)), dist)
    e2e_value = aggregate_rate(world_size, samples_per_step, args.steps, e2e_total * 1e3)

    # Algorithmic work per sample of the reference algorithm (counting build
    # over four fixed 64x32 windows of the frame).
    cp = abi.render_params(W, H, spp, DEPTH, kernel=abi.KERNEL_MEGAKERNEL, count_work=1)
    keys = ["node_visits", "prim_tests", "other_tests", "closest_rays", "shadow_rays", "shadow_node_visits",
            "shadow_prim_tests", "shadow_other_tests", "samples"]
    work = dict.fromkeys(keys, 0)
    stc = abi.RtStats()
    for (x0, y0) in [(0, 0), (W // 2, H // 2), (W // 4, H // 3), (3 * W // 4, 2 * H // 3)]:
        cp.pixel_x0, cp.pixel_y0, cp.window_w, cp.window_h = min(x0, W - 64), min(y0, H - 32), 64, 32
        abi.check(lib.rt_render_device(scene, C.byref(cp), C.c_void_p(film.data_ptr()), C.byref(stc)), "count")
        for k in keys:
            work[k] += getattr(stc, k)
    ns = max(work["samples"], 1)
    per = {k: work[k] / ns for k in keys if k != "samples"}
    closest_b = 32 * per["node_visits"] + 36 * per["prim_tests"] + 64 * per["other_tests"]
    shadow_b = 32 * per["shadow_node_visits"] + 36 * per["shadow_prim_tests"] + 64 * per["shadow_other_tests"]
    bytes_per_sample = closest_b + shadow_b + 96 * per["closest_rays"]
    # Per-kernel algorithmic bytes per sample (wavefront form):
    #   extend : closest-ray traversal + 48 B ray in / hit out per closest ray
    #   occlude: shadow-ray traversal + 60 B (48 B record in, 12 B accumulate) per shadow ray
    #   shade  : 304 B path state + hit per vertex + 48 B per shadow record written
    #   regen  : 144 B path state written per sample + 48 B resolve
    kb = {"extend": closest_b + 48 * per["closest_rays"],
          "occlude": shadow_b + 60 * per["shadow_rays"],
          "shade": 304 * per["closest_rays"] + 48 * per["shadow_rays"],
          "regen": 192.0}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    roof = {"bound": "hbm", "peak": hbm, "unit": "GB/s",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6.65 TB/s",
            "algorithmic_bytes_per_sample": bytes_per_sample, "work_per_sample": per}
    if kern == abi.KERNEL_WAVEFRONT:
        pp = abi.render_params(W, H, spp, DEPTH, kernel=kern, profile_kernels=1)
        stp = abi.RtStats()
        abi.check(lib.rt_render_device(scene, C.byref(pp), C.c_void_p(film.data_ptr()), C.byref(stp)), "profile")
        kt = {"regen": stp.regen_ms, "extend": stp.extend_ms, "shade": stp.shade_ms, "occlude": stp.occlude_ms,
              "sort": stp.sort_ms}
        dom = max(["regen", "extend", "shade", "occlude"], key=lambda k: kt[k])
        # scale the profiled (ungraphed) split onto the timed per-step device time
        tot = sum(kt.values())
        k_s = ms_per_step / 1e3 * kt[dom] / tot
        achieved = kb[dom] * samples_per_step / k_s / 1e9
        roof.update({"kernel": f"k_wf_{dom}", "achieved": achieved, "frac": achieved / hbm,
                     "kernel_ms_per_step": {k: v * ms_per_step / tot for k, v in kt.items()},
                     "launches_per_step": stp.iterations, "algorithmic_bytes_per_launch": kb[dom] *
                     samples_per_step / max(stp.iterations, 1)})
    else:
        achieved = bytes_per_sample * samples_per_step / (ms_per_step / 1e3) / 1e9
        roof.update({"kernel": "k_render_mega", "achieved": achieved, "frac": achieved / hbm})
    traffic, l2_bytes = None, None
    prof = os.path.join(ROOT, "profiles", f"{roof['kernel']}_icospheres.md")
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":")[1])
            if line.startswith("l2_bytes_per_launch:"):
                l2_bytes = float(line.split(":")[1])
    roof["traffic"] = traffic
    roof["traffic_source"] = (f"profiles/{roof['kernel']}_icospheres.md: ncu DRAM read + write of a steady-state "
                              "launch (all 4 M slots busy), measured on the same kernels") if traffic else None
    # L2 roofline beside the HBM one: the scene is largely L2-resident, so the
    # traversal kernels are compared against L2 bandwidth too. The peak is a
    # project micro-benchmark (L2-only float4 streams over a 32 MiB buffer).
    l2_peak = C.c_double(0.0)
    if lib.rt_probe_l2_bandwidth(dev, 32 << 20, 64, C.byref(l2_peak)) == abi.RT_OK:
        l2r = {"peak": l2_peak.value, "unit": "GB/s", "peak_source": "rt_probe_l2_bandwidth (32 MiB, 64 passes)",
               "bytes_per_launch": l2_bytes}
        if l2_bytes and "kernel_ms_per_step" in roof:
            per_launch_s = roof["kernel_ms_per_step"][roof["kernel"][5:]] / 1e3 / max(roof["launches_per_step"], 1)
            l2r["achieved"] = l2_bytes / per_launch_s / 1e9
            l2r["frac"] = l2r["achieved"] / l2_peak.value
        roof["l2"] = l2r

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": f"icospheres-64x20480 ({world.num_tris} tris) {W}x{H} {spp}spp depth{DEPTH}",
                       "kernel": args.kernel, "autotuned": tuned, "parallelism": f"replicas{world_size}",
                       "l2": "flushed between steps (256 MiB write)", "spp": spp},
            "roofline": roof,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": C.sizeof(params),
                    "d2h_bytes_per_step": 3 * W * H * 4, "ms_per_step": e2e_total * 1e3 / args.steps,
                    "device_ms_per_step": sum(e2e_dev) / max(len(e2e_dev), 1), "clocks": clk2.summary()},
            "gpu_launches": launches, "clocks": clk.summary()}
    if not args.no_extras and kern == abi.KERNEL_WAVEFRONT:
        pm = abi.render_params(W, H, spp, DEPTH, kernel=abi.KERNEL_MEGAKERNEL)
        mt, _ = timed(pm, 1, 1)
        mv = world_size * samples_per_step / (mt / 1e3) / 1e6
        line["plain_kernel"] = {"value": mv, "unit": UNIT, "ms_per_step": mt, "speedup_wavefront": value / mv}
        if rank == 0:
            line["time_to_relmse_1e-3"] = time_to_relmse(rt, lib, abi)
            # the bench frame itself: a 256x256 window at its centre (a 65 536-spp
            # reference of the whole 1080p frame would take minutes)
            win = ((W - 256) // 2, (H - 256) // 2, 256, 256)
            t2 = {"workload": f"icospheres {W}x{H} depth {DEPTH}, window {win}"}
            t2.update(time_to_relmse_on(lib, abi, scene, W, H, DEPTH, window=win))
            line["time_to_relmse_1e-3_icospheres"] = t2
            line.update(batched_side(rt))
            line["c1"] = c1_side(rt, lib, abi)
            line["bvh_build"] = bvh_build_side(lib, abi, pw)
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(rt, world)
    lib.rt_scene_destroy(scene)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Throughput benchmark of the B200 path tracer.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]
                    [--config procedural|cornell|many_light] [--spp S]
    python bench.py --workload serving [--serving-jobs J] [--serving-scenes S] [--serving-rate R]
    python bench.py --workload viewports

Workload (default): the procedural mesh scene -- 64 seeded affine instances
of 8 geodesic spheres (997,920 instanced fp32 triangles, smooth normals), 32
random closure graphs over diffuse / emission / transparent / add / mix,
point / spot / sun lights, constant world colour -- rendered at 1920x1080,
64 spp, max 8 bounces.  One step renders that whole frame
(RenderSession.render_samples over all 64 samples).  The metric is
samples/s (pixels x spp / render seconds) with rays/s beside it.

`value` is device time (CUDA events on the session stream around each
render_samples call, max over ranks); `e2e` is the public API per step:
compile_scene from host arrays (geometry upload + BVH build), create_session,
render_samples, and the read of every pass back to host memory.  Under
torchrun each rank renders its own frame (seed = rank) on its own GPU: the
work shards by frame with no data-path collective (weak scaling).

--impl reference times the reference path's CPU restatement (the oracle,
all host threads) on a bounded row band of the same workload.

The headline line also carries two secondary measurements on the same GPU:
`viewports` (64 concurrent viewport renders, batched against sequential,
after a one-knob-at-a-time tuning sweep) and `serving` (a Poisson job
stream through the render server against one session per job; 64 jobs over
16 resident scenes by default).  `--workload serving` / `--workload
viewports` run only that measurement, at the --serving-* sizes or over the
full 27-point tuning grid.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    "procedural": dict(width=1920, height=1080, spp=64, bounces=8),
    "cornell": dict(width=256, height=256, spp=16, bounces=4),
    "many_light": dict(width=1280, height=720, spp=32, bounces=6, light_tree=1),
}


def make_scene(name: str, seed: int = 0):
    from psycles_b200 import scenes
    if name == "procedural":
        return scenes.procedural_scene(seed=0)
    if name == "cornell":
        return scenes.cornell_box()
    return scenes.many_light_scene(seed=0)


def workload_config(args, scene) -> dict:
    c = CONFIGS[args.config]
    return {"workload": f"{args.config} scene {c['width']}x{c['height']} {args.spp} spp max {c['bounces']} bounces",
            "width": c["width"], "height": c["height"], "spp": args.spp, "max_bounces": c["bounces"],
            "instanced_triangles": scene.instanced_triangles, "instances": len(scene.instances),
            "materials": len(scene.materials), "analytic_lights": len(scene.lights),
            "light_selection": "light tree" if c.get("light_tree") else "flat distribution",
            "l2_policy": "scene geometry + BVH (~150 MB) and per-path state (~400 MB) exceed the 126 MB L2"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "fallback": True}


class CpuBaseline:
    """The oracle (CPU restatement of the reference path) on all host cores.

    The scene is prepared once (BVH build, emitter tables), outside every
    timed region; its time is reported as `setup_s`.  A timed sample renders
    ALL spp of every `stride`-th row of the full frame (rows 0, stride,
    2*stride, ...), so it sees the frame's mix of sky, geometry and path
    lengths rather than one band, and is scaled to the frame by the stated
    factor (frame samples / sampled samples)."""

    def __init__(self, args, scene):
        from oracle.oracle import OracleScene
        c = CONFIGS[args.config]
        self.args, self.c = args, c
        self.cores = os.cpu_count() or 1
        self.desc = scene.to_desc()
        t0 = time.perf_counter()
        self.prepared = OracleScene(self.desc)
        self.setup_s = time.perf_counter() - t0

    def render(self, stride: int) -> tuple[int, float]:
        """Renders the rows of one stride; returns (samples, seconds)."""
        from oracle.oracle import OracleFilm
        from psycles_b200 import scenes
        c = self.c
        st = scenes.render_settings(c["width"], c["height"], max_bounces=c["bounces"],
                                    use_light_tree=c.get("light_tree", 0))
        film = OracleFilm(st)
        t0 = time.perf_counter()
        film.render_prepared(self.prepared, 0, self.args.spp, self.args.spp, row_stride=stride, threads=self.cores)
        dt = time.perf_counter() - t0
        rows = (c["height"] + stride - 1) // stride
        return c["width"] * rows * self.args.spp, dt

    def stride_for(self, seconds: float) -> int:
        """The row stride whose sample takes about `seconds`, from a short
        calibration render (every 540th row of the frame)."""
        c = self.c
        probe = max(1, c["height"] // 2)
        samples, dt = self.render(probe)
        rate = samples / max(dt, 1e-6)
        rows = max(1, int(seconds * rate / (c["width"] * self.args.spp)))
        return max(1, min(c["height"], c["height"] // rows))

    NOTE = ("the repo's scalar C++ restatement of the reference path (median-split BVH, std::thread per core), "
            "not the reference's Embree-backed Luisa fallback, which cannot be built here (LuisaCompute, LLVM and "
            "Embree absent); the reference publishes about 3.59 M samples/s for that fallback on a 16-core/32-thread "
            "host, on a different scene (Lone Monk 640x480, 64 spp)")

    def describe(self, stride: int, samples: int, dt: float) -> str:
        c = self.c
        rows = (c["height"] + stride - 1) // stride
        frame = c["width"] * c["height"] * self.args.spp
        return (f"every {stride}th row of the {c['width']}x{c['height']} frame ({rows} rows), all {self.args.spp} spp: "
                f"{samples} samples in {dt:.2f} s; frame = {frame / samples:.1f}x this sample; scene preparation "
                f"(BVH build, emitter tables) {self.setup_s:.2f} s outside the timed region")


def cpu_baseline(args, scene, seconds_budget: float = 15.0) -> dict:
    """The oracle on all host cores, on a bounded stratified row sample."""
    base = CpuBaseline(args, scene)
    stride = base.stride_for(seconds_budget)
    samples, dt = base.render(stride)
    return {"value": samples / dt, "unit": "samples/s", "cores": base.cores, "kind": "port",
            "sample": base.describe(stride, samples, dt), "setup_s": base.setup_s, "note": CpuBaseline.NOTE}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene = make_scene(args.config)
    base = CpuBaseline(args, scene)
    # each step renders the same stratified row sample; sized so that the
    # whole --warmup + --steps run takes about two minutes
    per_step = min(15.0, max(2.0, 120.0 / max(args.steps + args.warmup, 1)))
    stride = base.stride_for(per_step)
    times, samples = [], 0
    for _ in range(args.warmup + args.steps):
        samples, dt = base.render(stride)
        times.append(dt)
    timed = times[args.warmup:]
    step_s = statistics.mean(timed)
    value = samples / step_s
    c = CONFIGS[args.config]
    line = {"impl": "reference", "metric": "samples/s", "value": value, "unit": "samples/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, scene),
            "step": "one step renders the stratified row sample below (not the whole frame); ms_per_step is that "
                    "sample's measured time",
            "frame_extrapolation": c["width"] * c["height"] * args.spp / samples,
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": base.cores, "kind": "port",
                             "sample": base.describe(stride, samples, step_s), "note": CpuBaseline.NOTE},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def scene_bytes(scene) -> int:
    total = 0
    for m in scene.meshes:
        total += m.positions.nbytes + m.indices.nbytes
        total += 0 if m.normals is None else m.normals.nbytes
        total += 0 if m.materials is None else m.materials.nbytes
    total += len(scene.instances) * 80
    for cm in scene.materials:
        total += cm.program.closures.nbytes + cm.parameters.scalars.nbytes + cm.parameters.vectors.nbytes
    return total


def run_cuda(args) -> None:
    from psycles_b200 import dist as pdist
    rank, world, local = pdist.rank_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = dist_mod
    from psycles_b200 import _abi, scenes
    from psycles_b200.backend import CudaPathTracerBackend, SampleRange

    c = CONFIGS[args.config]
    scene = make_scene(args.config)
    backend = CudaPathTracerBackend(local)
    settings = lambda: scenes.render_settings(c["width"], c["height"], max_bounces=c["bounces"],
                                              seed=pdist.frame_seed(rank), use_light_tree=c.get("light_tree", 0))
    comp = backend.compile_scene(scene)
    if not comp.ok():
        raise SystemExit(f"compile_scene failed: {comp.diagnostics}")
    session = backend.create_session(comp.scene, settings())
    pixels = c["width"] * c["height"]
    samples_per_step = pixels * args.spp

    def step():
        session.reset(settings())
        ok = session.render_samples(SampleRange(0, args.spp, 0, args.spp))
        if not ok:
            raise SystemExit(f"render failed: {session.diagnostics}")
        return session.stats()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        return pdist.max_over_ranks(v, device=f"cuda:{local}")

    for _ in range(args.warmup):
        step()
    barrier()
    ms, rays, launches, seg = [], 0, 0, 0
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            s = step()
            ms.append(s.ms_total)
            rays += s.closest_rays + s.shadow_rays
            launches += s.kernel_launches
            seg += s.path_segments
        wall = time.perf_counter() - t0
    barrier()
    device_s = max_over_ranks(sum(ms) / 1e3)
    value = samples_per_step * args.steps * world / device_s
    rays_per_s = max_over_ranks(rays / (sum(ms) / 1e3)) * world if rays else 0.0

    # roofline of the dominant kernel (closest-hit traversal): algorithmic
    # bytes per ray = ray 32 B + path state 32 B + queue index 4 B read,
    # hit 20 B written, plus the scene's unique geometry once per launch.
    peaks = measured_peaks()
    kernel = {}
    if args.kernel_timing:
        kernel = kernel_profile(args, backend, comp.scene, settings())

    # e2e: host arrays -> compile_scene -> render -> passes in host memory;
    # one untimed warm-up iteration (its time is reported as `cold_ms`: the
    # device pool and the pinned readback staging grow on it), then up to
    # three timed ones
    e2e_ms = []
    d2h = 0
    phases = {}
    cold_ms = None
    for it in range(1 + max(1, min(args.steps, 3))):
        barrier()
        t0 = time.perf_counter()
        comp2 = backend.compile_scene(scene)
        t1 = time.perf_counter()
        sess2 = backend.create_session(comp2.scene, settings())
        assert sess2.render_samples(SampleRange(0, args.spp, 0, args.spp))
        t2 = time.perf_counter()
        d2h = 0
        for p in sess2.passes:
            d2h += sess2.read_pass(p.kind).nbytes
        t3 = time.perf_counter()
        if it == 0:
            cold_ms = (t3 - t0) * 1e3
        else:
            e2e_ms.append((t3 - t0) * 1e3)
        bs = comp2.scene.build_stats()
        # host -> device: every scene buffer compile_scene uploads (BVH
        # nodes, triangle records, meshes, instances, materials, emitters),
        # plus the session's Sobol table and pixel-filter table
        h2d_scene = int(bs.upload_bytes)
        h2d = h2d_scene + 256 * _abi.load().psy_sobol_sequence_size_for_samples(args.spp) * 16 + 1024 * 4
        phases = {"compile_ms": (t1 - t0) * 1e3, "session_render_ms": (t2 - t1) * 1e3,
                  "render_device_ms": sess2.stats().ms_total, "readback_ms": (t3 - t2) * 1e3,
                  "build": {n: (round(getattr(bs, n), 3) if isinstance(getattr(bs, n), float) else getattr(bs, n))
                            for n, _ in bs._fields_}}
        sess2.close()
        comp2.scene.close()
    e2e_s = max_over_ranks(statistics.mean(e2e_ms) / 1e3)
    e2e_value = samples_per_step * world / e2e_s

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    line = {
        "metric": "samples/s", "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": device_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, scene),
        "rays_per_s": rays_per_s, "wall_s": wall,
        "e2e": {"value": e2e_value, "unit": "samples/s", "h2d_bytes_per_step": h2d,
                "h2d_detail": {"scene_upload_bytes": h2d_scene, "session_tables_bytes": h2d - h2d_scene,
                               "host_scene_arrays_bytes": scene_bytes(scene)},
                "d2h_bytes_per_step": d2h, "includes": "compile_scene (upload + BVH build), render, pass readback",
                "steps": len(e2e_ms), "cold_ms": cold_ms, "phases": phases},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
        "tuning": __import__("psycles_b200.autotune", fromlist=["get_tuning"]).get_tuning(backend),
    }
    if kernel:
        line["roofline"] = kernel["roofline"]
        line["kernels"] = kernel["kernels"]
    if args.serving and args.config == "procedural":
        line["viewports"] = run_viewports(backend, comp.scene)
        line["serving"] = run_serving(backend, jobs=args.serving_jobs, rate=args.serving_rate,
                                      scene_count=args.serving_scenes)
    if args.cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, scene)
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


# ------------------------------------------------------------------ serving

SERVING_SIZES = [(256, 256), (512, 512), (1024, 768), (1920, 1080)]


def _random_camera(rng):
    import math
    from psycles_b200 import scenes
    eye = (float(rng.uniform(-14, 14)), float(rng.uniform(2, 10)), float(rng.uniform(12, 24)))
    target = (float(rng.uniform(-3, 3)), 2.0, float(rng.uniform(-3, 3)))
    return scenes.Camera(scenes.look_at(eye, target), math.radians(45), math.radians(45), 0)


def _parameter_edit(rng, material):
    """Same-structure edit of a compiled material: random RGB slots and
    mix factors (a parameter-only rebind)."""
    import numpy as np
    sc = material.parameters.scalars.copy()
    vc = rng.uniform(0.05, 0.95, material.parameters.vectors.shape).astype(np.float32)
    if sc.size:
        sc = rng.uniform(0.0, 1.0, sc.shape).astype(np.float32)
    return sc, vc


def serving_scenes(count: int):
    """The serving stream's resident scenes: procedural scenes built like the
    headline one with 8..64 instances of the 8 base meshes (125k-1M
    triangles), seeds 0..count-1."""
    from psycles_b200 import scenes
    return [scenes.procedural_scene(seed=k, instances_per_mesh=1 + k % 8) for k in range(count)]


def serving_workload(seed: int, jobs: int, rate: float, scene_count: int = 16):
    """The serving stream: Poisson arrivals at `rate` jobs/s over
    `scene_count` resident procedural scenes, resolution drawn from
    {256^2, 512^2, 1024x768, 1920x1080}, spp uniform in 1-64, random camera
    poses; 30 % of jobs preceded by a parameter-only material edit and 5 % by
    a structural graph edit (a recompiled material)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(jobs):
        t += float(rng.exponential(1.0 / rate))
        w, h = SERVING_SIZES[int(rng.integers(0, len(SERVING_SIZES)))]
        u = float(rng.random())
        out.append({"arrival": t, "scene": int(rng.integers(0, scene_count)), "width": w, "height": h,
                    "spp": int(rng.integers(1, 65)), "camera": _random_camera(rng),
                    "edit": "structural" if u < 0.05 else ("parameters" if u < 0.35 else None),
                    "edit_seed": int(rng.integers(0, 1 << 30)), "seed": k})
    return out


def _latency_summary(latencies, stream) -> dict:
    """p50 / p99 latency over all jobs and per resolution class."""
    import numpy as np
    lat = np.array(latencies)
    out = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)), "per_class": {}}
    for w, h in SERVING_SIZES:
        sel = np.array([j["width"] == w and j["height"] == h for j in stream])
        if sel.any():
            out["per_class"][f"{w}x{h}"] = {"jobs": int(sel.sum()), "p50_ms": float(np.percentile(lat[sel], 50)),
                                            "p99_ms": float(np.percentile(lat[sel], 99))}
    return out


def run_serving(backend, jobs: int = 64, rate: float = 200.0, scene_count: int = 16, capacity: int = 0) -> dict:
    """The same job stream through the render server (continuous batching)
    and through plain one-session-per-job renders; both arms read every pass
    back.  Latency is arrival -> passes in host memory."""
    import numpy as np
    from psycles_b200 import _abi, scenes
    from psycles_b200.backend import RenderServer, SampleRange
    from psycles_b200.materials import random_material

    base = serving_scenes(scene_count)
    stream = serving_workload(7, jobs, rate, scene_count)
    passes = (_abi.PASS_COMBINED, _abi.PASS_NORMAL, _abi.PASS_ALBEDO, _abi.PASS_SAMPLE_COUNT)
    total_samples = sum(j["width"] * j["height"] * j["spp"] for j in stream)
    structural = {}  # job index -> recompiled scene (built before the clock starts: the same for both arms)
    for i, j in enumerate(stream):
        if j["edit"] == "structural":
            rng = np.random.default_rng(j["edit_seed"])
            db = scenes.SceneDatabase(base[j["scene"]])
            m = int(rng.integers(0, len(base[j["scene"]].materials)))
            structural[i] = db.apply(material_graphs={m: random_material(rng, emission_probability=0.0)})

    def settings(j):
        return scenes.render_settings(j["width"], j["height"], max_bounces=8, seed=j["seed"])

    def arm(serve: bool) -> dict:
        compiled = [backend.compile_scene(sc).scene for sc in base]
        recompiled = {i: backend.compile_scene(sc).scene for i, sc in structural.items()}
        current = list(compiled)
        current_desc = list(base)  # the host scene each resident scene was compiled from
        latencies, t_done = [None] * len(stream), 0.0
        server = RenderServer(backend.context, path_capacity=capacity) if serve else None
        ids = [None] * len(stream)
        edits = [(i, j) for i, j in enumerate(stream)]

        def apply_edit(i, j):
            if j["edit"] == "structural":
                current[j["scene"]] = recompiled[i]
                current_desc[j["scene"]] = structural[i]
            elif j["edit"] == "parameters":
                rng = np.random.default_rng(j["edit_seed"])
                sc = current_desc[j["scene"]]
                m = int(rng.integers(0, len(sc.materials)))
                scal, vec = _parameter_edit(rng, sc.materials[m])
                if serve:
                    server.rebind_parameters(current[j["scene"]], m, scal, vec)
                else:
                    current[j["scene"]].rebind_parameters(m, scal, vec)

        t0 = time.perf_counter()
        if serve:
            def submitter():
                for i, j in edits:
                    delay = j["arrival"] - (time.perf_counter() - t0)
                    if delay > 0:
                        time.sleep(delay)
                    apply_edit(i, j)
                    ids[i] = server.submit(current[j["scene"]], settings(j), j["spp"], camera=j["camera"])
            th = threading.Thread(target=submitter)
            th.start()
            for i, j in enumerate(stream):
                while ids[i] is None:
                    time.sleep(0.0005)
                assert server.wait(ids[i], 600000) == _abi.PSY_OK
                for k in passes:
                    server.read_pass(ids[i], k, j["width"], j["height"])
                server.release(ids[i])
                now = time.perf_counter() - t0
                latencies[i] = (now - j["arrival"]) * 1e3
                t_done = now
            th.join()
            st = server.stats()
            extra = {"wavefronts": int(st.wavefronts), "server_p50_ms": st.latency_p50_ms,
                     "server_p99_ms": st.latency_p99_ms, "bytes_peak": int(st.bytes_peak),
                     "loop_busy_s": st.busy_ms / 1e3, "device_s": st.device_ms / 1e3,
                     "device_samples_per_s": total_samples / (st.device_ms / 1e3)}
            server.close()
        else:
            device_ms = 0.0
            for i, j in edits:
                delay = j["arrival"] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                apply_edit(i, j)
                sess = backend.create_session(current[j["scene"]], settings(j))
                sess.set_camera(j["camera"])
                assert sess.render_samples(SampleRange(0, j["spp"], 0, j["spp"])), sess.diagnostics
                device_ms += sess.stats().ms_total
                for k in passes:
                    sess.read_pass(k)
                sess.close()
                now = time.perf_counter() - t0
                latencies[i] = (now - j["arrival"]) * 1e3
                t_done = now
            extra = {"device_s": device_ms / 1e3, "device_samples_per_s": total_samples / (device_ms / 1e3)}
        for c in list(compiled) + list(recompiled.values()):
            c.close()
        return dict({"samples_per_s": total_samples / t_done, "wall_s": t_done},
                    **_latency_summary(latencies, stream), **extra)

    plain = arm(False)
    served = arm(True)
    arrival_span = stream[-1]["arrival"]
    offered = total_samples / arrival_span
    cut = f"; {jobs} of the stated 10,000 jobs" if jobs < 10000 else ""
    return {"workload": f"{jobs} jobs, Poisson arrivals at {rate:g}/s over {scene_count} resident procedural scenes "
                        "(125k-1M triangles); sizes 256^2..1920x1080, spp U[1,64], 8 bounces; 30% parameter "
                        f"edits, 5% structural edits; HBM admission budget 120 GB; every pass read back{cut}",
            "jobs": jobs, "rate_jobs_per_s": rate, "scenes": scene_count, "samples": total_samples,
            "path_capacity": capacity,
            "load": {"arrival_span_s": arrival_span, "offered_samples_per_s": offered,
                     "server_device_samples_per_s": served["device_samples_per_s"],
                     "utilisation": offered / served["device_samples_per_s"],
                     "note": ("the stream offers more samples per second than the GPU renders (utilisation above 1), "
                              "so jobs queue and latency measures the drain of that queue, not admission under "
                              "steady load") if offered > served["device_samples_per_s"]
                     else "the GPU keeps up with the offered load: latency is admission under steady load"},
            "server": served, "plain": plain,
            "server_vs_plain": served["samples_per_s"] / plain["samples_per_s"]}


VIEWPORT_SWEEP = {"path_capacity": (1 << 20, 1 << 22, 1 << 24), "sort_threshold": (0, 1 << 16, 1 << 20),
                  "stream_block_size": (128, 256, 512)}


def run_viewports(backend, compiled, count: int = 64, sweep: str = "descent") -> dict:
    """64 concurrent viewport renders of the procedural scene from random
    camera poses (128^2 .. 1920x1080, 1-16 spp) in one batched call (shared
    wavefronts, each replayed as a captured CUDA graph), after a tuning sweep
    over queue capacity {1M, 4M, 16M} paths, sort-by-material threshold
    {never, 64Ki, 1Mi} and block size {128, 256, 512} of the camera-ray and
    film kernels (`sweep`: "grid" = all 27 points, "descent" = one knob at a
    time from the defaults, "none" = the defaults only), against the same 64 sessions rendered one after
    another at the chosen tuning.  Both arms check out bit-identical."""
    import itertools
    import numpy as np
    from psycles_b200 import _abi, autotune, scenes
    from psycles_b200.backend import BatchRenderer, SampleRange
    rng = np.random.default_rng(11)
    sizes = [(128, 128), (256, 256), (512, 512), (1024, 768), (1920, 1080)]
    views = []
    for _ in range(count):
        w, h = sizes[int(rng.integers(0, len(sizes)))]
        views.append((w, h, int(rng.integers(1, 17)), _random_camera(rng)))
    total = sum(w * h * spp for w, h, spp, _ in views)

    def sessions():
        out = []
        for w, h, spp, cam in views:
            s = backend.create_session(compiled, scenes.render_settings(w, h, max_bounces=8))
            s.set_camera(cam)
            out.append((s, spp))
        return out

    default = autotune.get_tuning(backend)

    def batched(point: dict, keep: bool = False):
        autotune.set_tuning(backend, dict(default, sort_threshold=point["sort_threshold"],
                                          stream_block_size=point["stream_block_size"]))
        batch = BatchRenderer(backend.context, path_capacity=point["path_capacity"], use_graph=True)
        warm = sessions()  # the first call captures the wavefront graph and sizes the path state
        assert batch.render([(s, SampleRange(0, spp, 0, spp)) for s, spp in warm])
        for s, _ in warm:
            s.close()
        bs = sessions()
        t0 = time.perf_counter()
        assert batch.render([(s, SampleRange(0, spp, 0, spp)) for s, spp in bs])
        wall = time.perf_counter() - t0
        st = batch.stats()
        result = {"samples_per_s": total / wall, "device_samples_per_s": total / (st.ms_total / 1e3), "wall_s": wall,
                  "wavefronts": int(st.wavefronts), "graph_launches": int(st.graph_launches),
                  "kernel_launches": int(st.kernel_launches)}
        batch.close()
        if keep:
            return result, bs
        for s, _ in bs:
            s.close()
        return result, None

    start = {"path_capacity": 1 << 24, "sort_threshold": default["sort_threshold"],
             "stream_block_size": default["stream_block_size"]}
    trials = []
    if sweep == "grid":
        for vals in itertools.product(*VIEWPORT_SWEEP.values()):
            point = dict(zip(VIEWPORT_SWEEP, vals))
            trials.append((point, batched(point)[0]))
        best = max(trials, key=lambda t: t[1]["device_samples_per_s"])[0]
    elif sweep == "none":
        best = dict(start)
    else:
        best = dict(start)
        trials.append((dict(best), batched(best)[0]))
        rate = trials[-1][1]["device_samples_per_s"]
        for knob, values in VIEWPORT_SWEEP.items():
            for v in values:
                if v == best[knob]:
                    continue
                point = dict(best, **{knob: v})
                trials.append((point, batched(point)[0]))
                if trials[-1][1]["device_samples_per_s"] > rate:
                    rate, best = trials[-1][1]["device_samples_per_s"], point
    # the two arms at the chosen tuning
    batch_result, bs = batched(best, keep=True)
    autotune.set_tuning(backend, dict(default, sort_threshold=best["sort_threshold"],
                                      stream_block_size=best["stream_block_size"]))
    ss = sessions()
    t0 = time.perf_counter()
    dev = 0.0
    for s, spp in ss:
        assert s.render_samples(SampleRange(0, spp, 0, spp))
        dev += s.stats().ms_total
    plain_wall = time.perf_counter() - t0
    same = all(np.array_equal(a.read_pass(_abi.PASS_COMBINED).view(np.uint32),
                              b.read_pass(_abi.PASS_COMBINED).view(np.uint32)) for (a, _), (b, _) in zip(bs, ss))
    for s, _ in list(ss) + list(bs):
        s.close()
    # Upper bound of what graph replay leaves between kernels: a batch of
    # one 16x16 1-spp view runs the same captured wavefront (same launch
    # count per step) with almost no work, so its device time per launch
    # bounds the per-launch gap (launch latency + the kernel's own minimum
    # duration); times the batched call's launch count, it bounds what a
    # single fused persistent kernel could save over graph replay.
    tiny_batch = BatchRenderer(backend.context, path_capacity=best["path_capacity"], use_graph=True)
    tiny = []
    for _ in range(2):  # the first call captures the graph
        t = backend.create_session(compiled, scenes.render_settings(16, 16, max_bounces=8))
        assert tiny_batch.render([(t, SampleRange(0, 1, 0, 1))])
        tiny.append(t)
    tst = tiny_batch.stats()
    for t in tiny:
        t.close()
    tiny_batch.close()
    per_launch_us = tst.ms_total * 1e3 / max(int(tst.kernel_launches), 1)
    launch_bound_ms = per_launch_us * batch_result["kernel_launches"] / 1e3
    batch_device_ms = total / batch_result["device_samples_per_s"] * 1e3
    autotune.set_tuning(backend, default)
    return {"workload": f"{count} viewports of the procedural scene, random poses, 128^2..1920x1080, 1-16 spp, "
                        "8 bounces",
            "samples": total, "sweep": sweep,
            "trials": [dict(point, device_samples_per_s=r["device_samples_per_s"], samples_per_s=r["samples_per_s"])
                       for point, r in trials],
            "chosen": best, "batched": batch_result,
            "plain": {"samples_per_s": total / plain_wall, "device_samples_per_s": total / (dev / 1e3),
                      "wall_s": plain_wall},
            "batched_vs_plain": plain_wall / batch_result["wall_s"], "identical": bool(same),
            "graph_gaps": {"tiny_batch_launches": int(tst.kernel_launches), "tiny_batch_device_ms": tst.ms_total,
                           "device_us_per_launch_bound": per_launch_us,
                           "batched_launches": batch_result["kernel_launches"],
                           "launch_bound_ms": launch_bound_ms, "batched_device_ms": batch_device_ms,
                           "launch_share_bound": launch_bound_ms / batch_device_ms}}


# DRAM bytes per second of device time of the traversal and shading kernels,
# from one `ncu --set full` capture of each (the third launch of the 4-spp
# procedural render: DRAM read + write of the launch over its duration).
# The traffic of a bench launch is this rate times the launch's mean
# event-timed duration (the procedural workload only).
NCU_DRAM_GBS = {"intersect": (319.3 + 65.7) / 2.150, "shadow": (109.0 + 13.2) / 1.775,
                "shade": (713.4 + 424.1) / 1.202}


def kernel_profile(args, backend, compiled, settings) -> dict:
    """Per-kernel device time of one render with CUDA events around each
    launch class (psy_session profile mode)."""
    from psycles_b200 import _abi
    from psycles_b200.backend import SampleRange
    lib = backend.context.lib
    if not hasattr(lib, "psy_session_profile"):
        return {}
    sess = backend.create_session(compiled, settings)
    prof = _abi.KernelProfile()
    _abi.check(lib.psy_session_set_profiling(sess.handle, 1))
    assert sess.render_samples(SampleRange(0, args.spp, 0, args.spp))
    _abi.check(lib.psy_session_profile(sess.handle, __import__("ctypes").byref(prof)))
    sess.close()
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    kernels = {}
    for name in ("raygen", "intersect", "shade", "shadow", "film"):
        launches = getattr(prof, f"{name}_launches")
        ms = getattr(prof, f"{name}_ms")
        nbytes = getattr(prof, f"{name}_bytes")
        kernels[name] = {"launches": launches, "ms": ms,
                         "gbs": (nbytes / (ms / 1e3) / 1e9) if ms > 0 else 0.0, "algorithmic_bytes": nbytes}
    top = max(kernels, key=lambda k: kernels[k]["ms"])
    k = kernels[top]
    achieved = k["gbs"]
    traffic = None
    if args.config == "procedural" and top in NCU_DRAM_GBS and k["launches"]:
        traffic = NCU_DRAM_GBS[top] * 1e9 * (k["ms"] / 1e3) / k["launches"]
    for name, rec in kernels.items():
        rec["frac_of_hbm"] = rec["gbs"] / hbm
        rec["algorithmic_bytes_per_launch"] = rec["algorithmic_bytes"] / rec["launches"] if rec["launches"] else 0.0
        if args.config == "procedural" and name in NCU_DRAM_GBS and rec["launches"]:
            # DRAM bytes per launch (read + write), from the ncu rate above
            rec["traffic_per_launch"] = NCU_DRAM_GBS[name] * 1e9 * (rec["ms"] / 1e3) / rec["launches"]
    return {"kernels": kernels,
            "roofline": {"kernel": f"k_{top}", "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic,
                         "algorithmic_bytes_per_launch": k["algorithmic_bytes"] / k["launches"] if k["launches"] else 0.0,
                         "traffic_source": "ncu DRAM bytes per device-second of this kernel x mean launch duration"
                         if traffic is not None else None,
                         "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if not peaks.get("fallback")
                         else "fallback 6.65 TB/s"}}


def run_workload(args) -> None:
    """One serving-stream or viewport-batch measurement on one GPU (rank 0
    of a torchrun launch; the other ranks exit without work)."""
    from psycles_b200 import dist as pdist
    rank, _, local = pdist.rank_env()
    if rank != 0:
        return
    from psycles_b200.backend import CudaPathTracerBackend
    backend = CudaPathTracerBackend(local)
    line = {"workload": args.workload, "n_gpus": 1, "data": "synthetic"}
    with ClockSampler(local) as clocks:
        if args.workload == "serving":
            line["serving"] = run_serving(backend, jobs=args.serving_jobs, rate=args.serving_rate,
                                          scene_count=args.serving_scenes)
        else:
            comp = backend.compile_scene(make_scene("procedural"))
            line["viewports"] = run_viewports(backend, comp.scene, sweep=args.viewport_sweep)
            comp.scene.close()
    line["clocks"] = clocks.summary()
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--config", default="procedural", choices=sorted(CONFIGS))
    ap.add_argument("--spp", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-kernel-timing", dest="kernel_timing", action="store_false")
    ap.add_argument("--no-serving", dest="serving", action="store_false",
                    help="skip the batched-viewport and serving-stream measurements")
    ap.add_argument("--workload", default="frame", choices=["frame", "serving", "viewports"],
                    help="frame: the headline line (default); serving / viewports: only that measurement, "
                         "one JSON line, at the sizes of the --serving-* options or with the full tuning grid")
    ap.add_argument("--serving-jobs", type=int, default=64)
    ap.add_argument("--serving-scenes", type=int, default=16)
    ap.add_argument("--serving-rate", type=float, default=200.0)
    ap.add_argument("--viewport-sweep", default="grid", choices=["grid", "descent", "none"],
                    help="tuning sweep of --workload viewports (none: the defaults only)")
    args = ap.parse_args()
    if args.spp is None:
        args.spp = CONFIGS[args.config]["spp"]
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "frame":
        run_workload(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()

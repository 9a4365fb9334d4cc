#!/usr/bin/env python
"""Benchmark of the B200 form-factor path (one JSON line on rank 0).

Workload (the closed enclosure): an inward icosphere of 20 480 FP32 triangles
(subdivision 5, radius 1) holding two perpendicular 1x1 plates of 20x20 cells
(800 triangles each), N = 22 080 faces, 1000 front-side Malley rays per face
(R = 22 080 000 rays per step), per-(source face, hit face) uint32 counts in
an N x N matrix (1.95 GB) resident on the device.  Synthetic and seeded; each
step draws fresh rays (Philox epoch = step index).

A step is one ffb_form_factor_counts call: zero the count matrix, fused
emission + grid trace + one global reduction per hit (matrices this large
take no shared-memory histogram).  The 1.95 GB zeroing
writes more than the 126 MB L2 every step, so no step starts with the previous
step's lines in L2.

  value  rays/s with the scene, grid and matrix resident (CUDA events on the
         context stream around K steps, max over ranks)
  e2e    rays/s through the C ABI with host buffers: host ray counts in, the
         count matrix in pinned host memory every step (row blocks packed on
         the device to the (column, count) pairs of their nonzero entries,
         which cross PCIe and are expanded into the host rows by host threads
         while the next block traces)
  --impl reference  the reference's own CPU path (zgrid_cpu caster + malley_cpu
         emission, compiled from its sources into oracle/_ref) on a bounded
         sample of the same workload, all host cores
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = ("enclosure: inward icosphere s5 (20480 tri) + 2 perpendicular 20x20 plates (1600 tri), "
            "N=22080, 1000 front rays/face, N^2 uint32 counts")
METRIC = "rays/s"
FLOPS_PER_TEST = 42  # math/triangle.cpp:40-78 with u, v, n, uu, uv, vv, D precomputed per face
SEED = 0x5EED


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rays-per-face", type=int, default=1000)
    ap.add_argument("--cpu-sample-every", type=int, default=0, help="reference sample: every k-th source face")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default="", help="grid dims nx,ny,nz (default: automatic)")
    ap.add_argument("--cells-per-face", type=float, default=0.0,
                    help="fixed grid sizing target (0: the autotuner chooses the grid among 128, 192 and 256 cells "
                         "per face and the kernel's launch shape; the library default is 32)")
    ap.add_argument("--no-skip", action="store_true", help="plain DDA without empty-space jumps")
    ap.add_argument("--trace-shape", type=int, default=-1,
                    help="launch shape of the fused kernel with a fixed grid (-1: shape 0, or the autotuner's)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-scenes section")
    ap.add_argument("--no-served", action="store_true", help="skip the served-requests section")
    ap.add_argument("--no-csv", action="store_true", help="skip the CSV-export section")
    ap.add_argument("--no-thermal", action="store_true", help="skip the radiance / distant-source section")
    ap.add_argument("--no-obj", action="store_true", help="skip the OBJ-import section")
    ap.add_argument("--grid-build-only", type=int, default=0,
                    help="build the workload's grid this many times, print one JSON line of build times and exit "
                         "(a small command for profiling the grid-build kernels)")
    ap.add_argument("--served-requests", type=int, default=256)
    ap.add_argument("--served-slots", type=int, default=16, help="requests prepared and traced at once")
    ap.add_argument("--served-slice-rays", type=int, default=0,
                    help="rays per trace slice of the serving loop (0: the library default, 64 Mi)")
    ap.add_argument("--served-max-wait", type=float, default=30.0,
                    help="age limit of the shortest-first served run, s (0: skip that run)")
    ap.add_argument("--served-rate", type=float, default=200.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--served-sub-rate", type=float, default=0.5,
                    help="arrival rate of the sub-saturation run, requests/s (0: skip it)")
    ap.add_argument("--served-sub-requests", type=int, default=8)
    return ap.parse_args()


def workload(rays_per_face):
    from form_factors_b200 import scenes
    faces = scenes.enclosure(5, 20)
    n = len(faces)
    front = np.full(n, rays_per_face, np.int32)
    rear = np.zeros(n, np.int32)
    return faces, front, rear


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    """SM clock and clock-event reasons sampled while the timed region runs.
    NVML is polled from a thread every 2 ms (read-only queries), so a timed
    region of a tenth of a second still gets tens of samples; without NVML,
    nvidia-smi -lms 200 is the fallback."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device):
        self.device = device
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.proc = None
        self.nvml = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.device)
        bus = getattr(props, "pci_bus_id", None)
        if bus is not None:
            pci = "%08x:%02x:%02x.0" % (getattr(props, "pci_domain_id", 0), bus, getattr(props, "pci_device_id", 0))
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(pci)
        return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(props.uuid))

    def _sample(self):
        nv, h = self.nvml
        return (nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), nv.nvmlDeviceGetCurrentClocksEventReasons(h))

    def _poll(self):
        while not self.stop_flag.is_set():
            try:
                self.rows.append(self._sample())
            except Exception:  # a failed query ends sampling, not the run
                return
            self.stop_flag.wait(0.002)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            # the first queries after nvmlInit pay NVML's own set-up: take
            # them here, before the timed region, and keep their latency
            t0 = time.perf_counter()
            self._sample()
            self.first_query_ms = (time.perf_counter() - t0) * 1e3
            t0 = time.perf_counter()
            self._sample()
            self.query_ms = (time.perf_counter() - t0) * 1e3
            nv, h = self.nvml
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None
        if self.nvml:
            import threading
            self.stop_flag = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.thread:
            self.stop_flag.set()
            self.thread.join(2)
            rows, self.thread = self.rows, None
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            sm = [float(r[0]) for r in rows]
            loaded = [s for s in sm if s > 0.5 * max(sm)]
            reasons = sorted({name for r in rows for name, bit in self.REASON_BITS if r[1] & bit})
            return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": self.max_mhz,
                    "sm_min_mhz": min(sm), "reasons": reasons, "samples": len(rows),
                    "source": "nvml polled every 2 ms (one query round %.2f ms; the first after init %.1f ms, "
                              "taken before the timed region)" % (self.query_ms, self.first_query_ms)}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1])]
        mx = [num(r[2]) for r in rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# the reference CPU path (oracle/_ref), bounded sample
# ---------------------------------------------------------------------------
def reference_sampler(faces, rays_per_face, every, threads=0, target_rays_per_s=0.25e6):
    """Returns (run_step, describe, threads): run_step() casts one bounded
    sample with the reference's malley_cpu emission and zgrid_cpu caster
    (ray_caster/zgrid_cpu.cpp:115-132 cast over `threads` host threads on
    disjoint ray slices; emission/malley_cpu.cpp:195-211 single-threaded, as
    the reference's emitter is stateful) and returns (rays, seconds,
    emit_seconds, cast_seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ctypes as C
    from oracle_lib import Reference
    if not Reference.available():
        return None, "oracle/_ref/libffref.so not built (reference sources absent when the tree was built)", 0
    ref = Reference()
    n = len(faces)
    cores = threads if threads > 0 else (os.cpu_count() or 1)
    if every <= 0:
        every = max(1, int(round(n * rays_per_face / (target_rays_per_s * cores))))  # ~1-4 s per step
    mask = np.zeros(n, np.uint8)
    mask[::every] = 1
    # front weight 1, rear 0, total 1, n_rays = rays_per_face: exactly
    # rays_per_face front rays per sampled face (malley_emission.cpp:50-54)
    w = np.zeros(2 * n, np.float32)
    w[0::2] = 1.0
    prep = C.c_double()
    h = ref.lib.ffref_step_open(Reference.ZGRID_CPU, n, np.ascontiguousarray(faces, np.float32), C.byref(prep))
    if not h:
        return None, "reference zgrid_cpu prepare failed", 0
    hist = np.zeros(n, np.uint32)

    def run():
        te, tc = C.c_double(), C.c_double()
        t0 = time.perf_counter()
        k = ref.lib.ffref_step_run(h, rays_per_face, w, 1.0, mask, cores, hist.ctypes.data, C.byref(te),
                                   C.byref(tc))
        return k, time.perf_counter() - t0, te.value, tc.value

    desc = ("reference zgrid_cpu cast + malley_cpu emission (oracle/_ref) of every %d-th source face "
            "(%d faces, %d rays) against the full %d-face scene, cast on %d threads" %
            (every, int(mask.sum()), int(mask.sum()) * rays_per_face, n, cores))
    return run, desc, cores


def cpu_baseline(faces, rays_per_face, every):
    """The reference's zgrid_cpu path on the host cores: all threads (the
    reported value: rays per second of emission + cast) and one thread, each
    with its emission and cast seconds apart."""
    out = reference_sampler(faces, rays_per_face, every)
    if out[0] is None:
        return {"value": None, "unit": "rays/s", "cores": 0, "kind": "reference", "sample": out[1]}
    run, desc, cores = out
    run()
    k, s, te, tc = run()
    line = {"value": k / s, "unit": "rays/s", "cores": cores, "kind": "reference", "sample": desc,
            "emit_s": te, "cast_s": tc, "cast_rays_per_s": k / tc if tc > 0 else None,
            "emit_rays_per_s": k / te if te > 0 else None}
    one = reference_sampler(faces, rays_per_face, 0, threads=1)
    if one[0] is not None:
        run1, desc1, _ = one
        k1, s1, te1, tc1 = run1()
        line["one_thread"] = {"value": k1 / s1, "cast_rays_per_s": k1 / tc1 if tc1 > 0 else None,
                              "emit_s": te1, "cast_s": tc1, "sample": desc1}
    return line


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    faces, front, rear = workload(args.rays_per_face)
    out = reference_sampler(faces, args.rays_per_face, args.cpu_sample_every)
    if out[0] is None:
        print(json.dumps({"impl": "reference", "unavailable": out[1]}))
        return
    run, desc, cores = out
    for _ in range(args.warmup):
        run()
    rays = 0
    secs = emit_s = cast_s = 0.0
    for _ in range(args.steps):
        k, s, te, tc = run()
        rays += k
        secs += s
        emit_s += te
        cast_s += tc
    v = rays / secs
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": desc},
        "cpu_baseline": {"value": v, "unit": "rays/s", "cores": cores, "kind": "reference", "sample": desc,
                         "emit_s": emit_s / args.steps, "cast_s": cast_s / args.steps,
                         "cast_rays_per_s": rays / cast_s if cast_s > 0 else None},
        "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------------------
# batched scenes (resident grids, one CUDA graph) vs the plain path
# ---------------------------------------------------------------------------
def batched_section(ctx, stream, args):
    """256 scenes, triangle counts log-uniform 200-20k (plate pairs, inward UV
    spheres, clutter in a box), 1k-10k front rays per face.

    batched: grids and the 256 count matrices resident, all scenes launched
      from one CUDA graph replay (zeroing included).
    plain: the same scenes one at a time through the single-scene path
      (scene upload, grid build, zeroing and trace per scene), device matrices.
    plain_dropin: the same through the reference-facing call with a host
      float matrix per scene (ffb_form_factors: counts, normalisation and the
      copy to the host), as a FORM_FACTORS_B200 calculate delivers it.
    A second plain pass records CUDA events around each phase of each scene:
    upload, grid build, and the counts call (zeroing + trace, of which the
    trace kernel alone is also timed).  ceiling = plain_s / sum(trace): the
    speed-up a batched form could reach if everything but the traces went
    away."""
    import torch
    from form_factors_b200 import scenes
    sl, rpf = scenes.batch_workload(256, 200, 20000, 1000, 10000, seed=4)
    sizes = np.array([len(f) for f in sl])
    fronts = [np.full(len(f), int(r), np.int32) for f, r in zip(sl, rpf)]
    rears = [np.zeros(len(f), np.int32) for f in sl]
    seeds = np.arange(1, len(sl) + 1, dtype=np.uint64) * np.uint64(7919)
    rays = int(sum(int(f.sum()) for f in fronts))
    skip = not args.no_skip
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tuned = args.cells_per_face <= 0
    all_front, all_rear = np.concatenate(fronts), np.concatenate(rears)
    ctx.batch_set(sl, cells_per_face=args.cells_per_face if not tuned else 32.0, skip_empty=skip)
    tune_s = 0.0
    shapes = None
    if tuned:
        # the autotuner's choices for the batch's scene classes (a one-time
        # cost: the plain arm below takes the same choices from the cache)
        t0 = time.perf_counter()
        shapes = ctx.batch_autotune(all_front, all_rear)
        torch.cuda.synchronize()
        tune_s = time.perf_counter() - t0
    # the batch's grids built with those choices, and its chunk tables
    t0 = time.perf_counter()
    ev0.record(stream)
    if tuned:
        ctx.batch_autotune(all_front, all_rear)  # every scene's choice from the cache: grid builds only
    else:
        ctx.batch_set(sl, cells_per_face=args.cells_per_face, skip_empty=skip)
    ctx.batch_prepare(all_front, all_rear, seeds)
    ev1.record(stream)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    build_dev_s = ev0.elapsed_time(ev1) / 1e3
    offs, words = ctx.batch_counts_layout()
    counts = torch.empty(words, dtype=torch.int32, device="cuda")
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        ctx.batch_launch(counts, offs, advance_epoch=True)
    graph.replay()  # warm-up
    torch.cuda.synchronize()
    ev0.record(stream)
    graph.replay()
    ev1.record(stream)
    torch.cuda.synchronize()
    batched_s = ev0.elapsed_time(ev1) / 1e3
    del graph

    def grid(i):
        # the batch's choice for the scene (a cache hit of the autotuner), or the fixed grid
        if tuned:
            ctx.autotune(fronts[i], rears[i], int(seeds[i]))
        else:
            ctx.grid_build(cells_per_face=args.cells_per_face, skip_empty=skip)

    def plain_scene(i, out=None):
        n = len(sl[i])
        ctx.scene_set(sl[i])
        grid(i)
        ctx.form_factor_counts(fronts[i], rears[i], int(seeds[i]), epoch=2,
                               out=counts[int(offs[i]):int(offs[i]) + n * n], n_rows=n)

    # plain: one scene at a time, grid built per scene
    t0 = time.perf_counter()
    ev0.record(stream)
    for i in range(len(sl)):
        plain_scene(i)
    ev1.record(stream)
    torch.cuda.synchronize()
    plain_s = ev0.elapsed_time(ev1) / 1e3
    plain_wall = time.perf_counter() - t0
    # phase breakdown of the plain path (a second pass, events per phase)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in sl]
    trace_ms = []
    for i, f in enumerate(sl):
        n = len(f)
        e = evs[i]
        e[0].record(stream)
        ctx.scene_set(f)
        e[1].record(stream)
        grid(i)
        e[2].record(stream)
        ctx.form_factor_counts(fronts[i], rears[i], int(seeds[i]), epoch=2,
                               out=counts[int(offs[i]):int(offs[i]) + n * n], n_rows=n)
        e[3].record(stream)
        trace_ms.append(ctx.stats().kernel_ms)
    torch.cuda.synchronize()
    upload_s = sum(e[0].elapsed_time(e[1]) for e in evs) / 1e3
    grid_s = sum(e[1].elapsed_time(e[2]) for e in evs) / 1e3
    counts_s = sum(e[2].elapsed_time(e[3]) for e in evs) / 1e3
    gaps_s = sum(evs[i][3].elapsed_time(evs[i + 1][0]) for i in range(len(evs) - 1)) / 1e3
    # the zeroing alone, per scene (the counts call zeroes, then traces)
    z0, z1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    z0.record(stream)
    for i, f in enumerate(sl):
        n = len(f)
        counts[int(offs[i]):int(offs[i]) + n * n].zero_()
    z1.record(stream)
    torch.cuda.synchronize()
    zero_s = z0.elapsed_time(z1) / 1e3
    # stats().kernel_ms brackets the zeroing and the trace launch of a call
    trace_s = max(sum(trace_ms) / 1e3 - zero_s, 1e-9)
    del counts
    torch.cuda.empty_cache()
    # plain through the reference-facing call: a host float matrix per scene
    host = torch.empty(int(sizes.max()) ** 2, dtype=torch.float32, pin_memory=True)
    # warm-up: the eight largest scenes once, untimed, so that the call's
    # scratch buffers have reached their sizes before the timed pass
    for i in np.argsort(sizes)[-8:]:
        n = len(sl[i])
        ctx.scene_set(sl[i])
        grid(i)
        ctx.form_factors(fronts[i], rears[i], int(seeds[i]), epoch=1, n_rows=n,
                         out=host[:n * n].numpy().reshape(n, n))
    t0 = time.perf_counter()
    for i, f in enumerate(sl):
        n = len(f)
        ctx.scene_set(f)
        grid(i)
        ctx.form_factors(fronts[i], rears[i], int(seeds[i]), epoch=2, n_rows=n,
                         out=host[:n * n].numpy().reshape(n, n))
    dropin_s = time.perf_counter() - t0
    del host
    return {"workload": "256 scenes, faces log-uniform 200-20000 (plates/UV spheres/clutter), "
                        "1k-10k front rays/face, per-scene N^2 uint32 counts resident",
            "faces_total": int(sizes.sum()), "rays": rays,
            "counts_gb": round(4 * float((sizes.astype(float) ** 2).sum()) / 1e9, 2),
            "batched_s": batched_s, "batched_grid_build_s": build_s, "batched_grid_build_device_s": build_dev_s,
            "autotune_s": tune_s,
            "plain_s": plain_s, "plain_wall_s": plain_wall, "plain_dropin_host_float_s": dropin_s,
            "plain_breakdown_s": {"upload": upload_s, "grid_build": grid_s, "counts_call": counts_s,
                                  "zeroing": zero_s, "trace": trace_s, "host_gaps": gaps_s},
            "batched_scenes_per_s": len(sl) / batched_s, "plain_scenes_per_s": len(sl) / plain_s,
            "plain_dropin_scenes_per_s": len(sl) / dropin_s,
            "batched_rays_per_s": rays / batched_s, "plain_rays_per_s": rays / plain_s,
            "speedup_trace_resident": plain_s / batched_s,
            "speedup_grid_build_in_both": plain_s / (batched_s + build_s),
            "speedup_vs_dropin": dropin_s / batched_s,
            "ceiling": plain_s / trace_s,
            "launches": "one fused launch per scene over 4 side streams, replayed as one CUDA graph",
            "autotuned": bool(tuned),
            "shapes_used": sorted(set(int(v) for v in shapes)) if shapes is not None else [0]}


# ---------------------------------------------------------------------------
# served requests (Poisson arrivals, admission by memory budget)
# ---------------------------------------------------------------------------
def served_section(args, ctx, stream):
    """Requests of scenes with faces log-uniform 500-50k (the three
    families), 1k-100k front rays per face, Poisson arrivals at
    args.served_rate/s.

    served: the C++ serving loop -- admission by an 80 GB device budget into
      args.served_slots slots, preparation on the slots' threads, traces in
      16 Mi-ray slices round-robin over the prepared requests with two slices
      in flight; results resident until released.
    plain: the single-scene path, one request at a time in arrival order
      (scene upload, grid build, zeroing and trace into a resident device
      matrix), each request's latency from its arrival to its result.
    ceiling = plain_s / sum(trace): the speed-up left if everything but the
    traces (timed per request with CUDA events in the plain arm) went away."""
    import torch
    from form_factors_b200 import native, scenes
    rng = np.random.default_rng(9)
    n = args.served_requests
    fams = ("plates", "sphere", "clutter")
    sizes = np.exp(rng.uniform(np.log(500), np.log(50000), n))
    reqs = [(scenes.family_scene(fams[i % 3], sizes[i], rng), int(rng.integers(1000, 100001)), 100 + i)
            for i in range(n)]
    gaps = rng.exponential(1.0 / args.served_rate, n)
    arrivals = np.cumsum(gaps)
    rays = sum(len(f) * r for f, r, _ in reqs)

    def served(slots, arrivals, reqs, shortest_first=False):
        server = native.Server(0, budget_bytes=int(80e9), slots=slots)
        if args.served_slice_rays > 0:
            server.set_slicing(args.served_slice_rays)
        if shortest_first:
            server.set_admission(shortest_first=True, max_wait_s=args.served_max_wait)
        t0 = time.perf_counter()
        ids = []
        for (f, r, sd), at in zip(reqs, arrivals):
            delay = t0 + at - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(server.submit(f, r, sd, cells_per_face=0.0))
        # results in completion order, each released at once: a finished
        # result keeps its budget reservation until it is released
        infos = []
        pending = list(ids)
        while pending:
            rid, inf = server.wait_any(pending, timeout_s=1200)
            infos.append(inf)
            server.release(rid)
            pending.remove(rid)
        wall = time.perf_counter() - t0
        st = server.stats()
        server.close()
        lat = np.array([inf.latency_s for inf in infos])
        spans = [(inf.trace_start_ns, inf.trace_end_ns) for inf in infos]
        return wall, lat, st, spans, [inf.slices for inf in infos]

    def plain(arrivals, reqs):
        nmax = max(len(f) for f, _, _ in reqs)
        out = torch.empty(nmax * nmax, dtype=torch.int32, device="cuda")
        lat, trace = [], []
        ctx.set_stats(False)
        t0 = time.perf_counter()
        for (f, r, sd), at in zip(reqs, arrivals):
            delay = t0 + at - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            k = len(f)
            fr, re = np.full(k, r, np.int32), np.zeros(k, np.int32)
            ctx.scene_set(f)
            ctx.autotune(fr, re, sd)  # the cached choice: the grid and shape the server uses
            ctx.form_factor_counts(fr, re, sd, epoch=0, out=out[:k * k], n_rows=k)
            trace.append(ctx.stats().kernel_ms * 1e-3)  # synchronises: the result is resident
            lat.append(time.perf_counter() - t0 - at)
        wall = time.perf_counter() - t0
        del out
        torch.cuda.empty_cache()
        return wall, np.array(lat), np.array(trace)

    # both arms take the autotuner's cached choices: tune every request's
    # scene class once, before either arm is timed
    t0 = time.perf_counter()
    for f, r, sd in reqs:
        k = len(f)
        ctx.scene_set(f)
        ctx.autotune(np.full(k, r, np.int32), np.zeros(k, np.int32), sd)
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t0
    plain_wall, plain_lat, plain_trace = plain(arrivals, reqs)
    served_wall, lat, st, spans, slices = served(args.served_slots, arrivals, reqs)
    sjf = None
    if args.served_max_wait > 0:
        sjf_wall, sjf_lat, _, _, _ = served(args.served_slots, arrivals, reqs, shortest_first=True)
        sjf = {"admission": "least work first, the oldest first after %.0f s of waiting" % args.served_max_wait,
               "scenes_per_s": n / sjf_wall, "speedup_scenes_per_s": plain_wall / sjf_wall,
               "p50_latency_s": float(np.percentile(sjf_lat, 50)),
               "p99_latency_s": float(np.percentile(sjf_lat, 99)),
               "mean_latency_s": float(sjf_lat.mean()), "wall_s": sjf_wall}
    # device overlap: pairs of requests whose trace spans intersect
    ordered = sorted((a, b) for a, b in spans if b > a)
    overlaps = sum(1 for i in range(1, len(ordered)) if ordered[i][0] < max(e for _, e in ordered[:i]))
    sub = None
    if args.served_sub_rate > 0:
        # the same kind of requests at a rate the server keeps up with:
        # latency is then service time, not queueing
        m = args.served_sub_requests
        sub_reqs = [(scenes.family_scene(fams[i % 3], sizes[i % n], rng), int(rng.integers(1000, 100001)), 500 + i)
                    for i in range(m)]
        for f, r, sd in sub_reqs:
            ctx.scene_set(f)
            ctx.autotune(np.full(len(f), r, np.int32), np.zeros(len(f), np.int32), sd)
        sub_arr = np.cumsum(rng.exponential(1.0 / args.served_sub_rate, m))
        sub_wall, sub_lat, sub_st, _, _ = served(args.served_slots, sub_arr, sub_reqs)
        sub_rays = sum(len(f) * r for f, r, _ in sub_reqs)
        sub = {"rate_per_s": args.served_sub_rate, "requests": m, "rays": int(sub_rays),
               "offered_rays_per_s": sub_rays / max(float(sub_arr[-1]), 1e-9),
               "p50_latency_s": float(np.percentile(sub_lat, 50)),
               "p99_latency_s": float(np.percentile(sub_lat, 99)),
               "max_latency_s": float(sub_lat.max()), "wall_s": sub_wall, "peak_concurrent": int(sub_st.peak_running)}
    return {"workload": "%d requests, faces log-uniform 500-50000 (plates/UV spheres/clutter), 1k-100k front "
                        "rays/face, Poisson %.0f req/s, 80 GB budget, %d slots" % (n, args.served_rate,
                                                                                  args.served_slots),
            "requests": n, "rays": int(rays), "served_scenes_per_s": n / served_wall,
            "plain_scenes_per_s": n / plain_wall, "speedup_scenes_per_s": plain_wall / served_wall,
            "served_rays_per_s": rays / served_wall, "plain_rays_per_s": rays / plain_wall,
            "served_wall_s": served_wall, "plain_wall_s": plain_wall, "plain_trace_s": float(plain_trace.sum()),
            "ceiling": plain_wall / float(plain_trace.sum()),
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "plain_p50_latency_s": float(np.percentile(plain_lat, 50)),
            "plain_p99_latency_s": float(np.percentile(plain_lat, 99)),
            "latency_samples": int(len(lat)),
            "offered_rays_per_s": rays / max(float(arrivals[-1]), 1e-9), "peak_concurrent": int(st.peak_running),
            "peak_tracing": int(st.peak_tracing), "trace_slices": int(sum(slices)),
            "requests_overlapping_on_device": int(overlaps),
            "note": "offered load far above capacity: latency is queueing under saturation",
            "mean_latency_s": float(lat.mean()), "plain_mean_latency_s": float(plain_lat.mean()),
            "shortest_first": sjf,
            "autotune_warmup_s": tune_s,
            "sub_saturation": sub}


# ---------------------------------------------------------------------------
# CSV export of the step's matrix (csv_export::export_csv)
# ---------------------------------------------------------------------------
def csv_section(ctx, stream, counts, front, rear, n):
    """Formatting on the device from the resident counts (normalised on the
    fly), and the reference-facing export of a host float matrix to a file,
    against the reference's csv_export on a block of the same matrix."""
    import shutil
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Reference
    outgoing = (front.astype(np.int64) + rear).astype(np.int32)
    d_out = torch.from_numpy(outgoing).cuda()
    nonzero = int(torch.count_nonzero(counts).item())
    n_text = ctx.csv_length(counts=counts, outgoing=d_out)
    text = torch.empty(n_text, dtype=torch.uint8, device="cuda")
    ctx.csv_format(counts=counts, outgoing=d_out, out=text)  # warm-up
    reps = 3
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(reps):
        ctx.csv_format(counts=counts, outgoing=d_out, out=text)
    ev1.record(stream)
    torch.cuda.synchronize()
    fmt_s = ev0.elapsed_time(ev1) * 1e-3 / reps
    entries = n * n
    alg_bytes = 4 * entries + n_text  # each count read once, the text written once
    del text
    # end to end: host float matrix -> file, as csv_export::export_csv takes it
    ff = ctx.normalise(counts, outgoing)
    shm = "/dev/shm"
    where = shm if os.path.isdir(shm) and shutil.disk_usage(shm).free > 3 * n_text else tempfile.gettempdir()
    path = os.path.join(where, "ffb_bench_%d.csv" % os.getpid())
    times = []
    for _ in range(3):  # median: a new file's pages make single runs noisy
        t0 = time.perf_counter()
        ctx.csv_export(path, ff=ff)
        times.append(time.perf_counter() - t0)
        size = os.path.getsize(path)
        os.remove(path)
    exp_s = statistics.median(times)
    ref = None
    if Reference.available():
        k = 2048  # a k x k block of the same matrix: the reference's export is single-threaded
        block = np.ascontiguousarray(ff[:k, :k])
        rpath = os.path.join(where, "ffb_bench_ref_%d.csv" % os.getpid())
        r = Reference()
        t0 = time.perf_counter()
        rc = r.export_csv(rpath, block)
        ref_s = time.perf_counter() - t0
        os.remove(rpath)
        if rc == 0:
            ref = {"entries_per_s": k * k / ref_s, "cores": 1, "kind": "reference",
                   "sample": "csv_export::export_csv (oracle/_ref) of the top-left %dx%d block of the same matrix "
                             "to the same file system" % (k, k)}
    return {
        "workload": "CSV text of the %dx%d matrix of this step (csv_export::export_csv format)" % (n, n),
        "entries": entries, "nonzero_entries": nonzero, "text_bytes": int(n_text),
        "format_ms": fmt_s * 1e3, "format_entries_per_s": entries / fmt_s,
        "roofline": {"bound": "hbm", "achieved": alg_bytes / fmt_s / 1e9, "peak": measured_hbm_gbs(),
                     "peak_source": hbm_peak()[1], "unit": "GB/s",
                     "frac": alg_bytes / fmt_s / 1e9 / measured_hbm_gbs(),
                     "work": "4 B count read + text bytes written per entry (algorithmic)"},
        "export_s": exp_s, "export_entries_per_s": entries / exp_s, "export_bytes": size, "export_dir": where,
        "export_path": "host float matrix -> H2D -> format -> D2H (pipelined) -> fwrite; median of 3",
        "cpu_baseline": ref,
    }


# ---------------------------------------------------------------------------
# ray-traced thermal equations on the same scene and grid
# ---------------------------------------------------------------------------
def thermal_section(ctx, faces, rays_per_face):
    """One radiance-equation step (per-face meshes, temperature-weighted
    Malley emission, absorbed power scattered to the hit meshes) and one
    distant-source step (a disc of parallel rays) through the C ABI, against
    the reference's radiance_cpu over its zgrid_cpu caster on a bounded ray
    budget."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Reference
    n = len(faces)
    n_sphere = n - 1600  # the two 20 x 20 plates come last
    # one mesh per face as (first face, face count, material), built once as
    # the ffb_mesh layout: the scene is fixed across the controller's steps
    meshes = np.stack([np.arange(n), np.ones(n, np.int64), (np.arange(n) >= n_sphere).astype(np.int64)],
                      axis=1).astype(np.int32)
    # sphere: inward emitter only, so that every ray starts inside the scene
    materials = np.array([(0.9, 0.0, 0.8, 0.8), (0.7, 0.6, 0.5, 0.4)], np.float32)
    temps = (300.0 + 100.0 * np.random.default_rng(5).random(n)).astype(np.float32)
    n_rays = rays_per_face * n
    ctx.radiance_step(faces, meshes, materials, temps, n_rays, seed=1, epoch=0)  # warm-up
    reps = 3
    t0 = time.perf_counter()
    for e in range(reps):
        em, ab = ctx.radiance_step(faces, meshes, materials, temps, n_rays, seed=1, epoch=1 + e)
    rad_s = (time.perf_counter() - t0) / reps
    rad_ms_kernel = ctx.stats().kernel_ms
    sun_rays = 10_000_000
    ctx.distant_source_step(faces, meshes, materials, sun_rays, 1361.0, [0.3, -0.4, -0.8], seed=2)
    t0 = time.perf_counter()
    for e in range(reps):
        sun = ctx.distant_source_step(faces, meshes, materials, sun_rays, 1361.0, [0.3, -0.4, -0.8], seed=2,
                                      epoch=1 + e)
    sun_s = (time.perf_counter() - t0) / reps
    sun_ms_kernel = ctx.stats().kernel_ms
    ref = None
    if Reference.available():
        sample = 200_000
        r = Reference()
        m3 = np.array(meshes, np.int32)
        t0 = time.perf_counter()
        rc, _, _ = r.radiance(faces, m3, materials, temps, sample, caster=Reference.ZGRID_CPU)
        ref_s = time.perf_counter() - t0
        if rc == 0:
            ref = {"rays_per_s": sample / ref_s, "cores": 1, "kind": "reference",
                   "sample": "radiance_cpu + malley_cpu + zgrid_cpu (oracle/_ref), one calculate() of %d rays on "
                             "the same scene and meshes (the reference's equation is single-threaded)" % sample}
    return {
        "workload": "enclosure, %d per-face meshes, two materials, temperatures 300-400 K" % n,
        "radiance": {"rays": n_rays, "step_s": rad_s, "rays_per_s": n_rays / rad_s, "kernel_ms": rad_ms_kernel,
                     "emitted_w": float(em.sum()), "absorbed_w": float(ab.sum()),
                     "path": "host weights and powers -> fused emit/trace/fixed-point scatter -> host sums"},
        "distant_source": {"rays": sun_rays, "step_s": sun_s, "rays_per_s": sun_rays / sun_s,
                           "kernel_ms": sun_ms_kernel, "absorbed_w": float(sun.sum())},
        "cpu_baseline": ref,
    }


# ---------------------------------------------------------------------------
# OBJ scene import, then the scene and grid rebuilt on the device
# ---------------------------------------------------------------------------
def obj_section(device):
    """A 250 000-face scene written as OBJ text (%.9g coordinates, one object
    per 1 000 faces), imported through the C ABI (file read, upload, GPU
    parse and gather), set as the scene from the device and gridded; the
    reference's obj_import::scene timed on the same file."""
    import io
    import shutil
    from form_factors_b200 import native, scenes
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Reference
    faces = scenes.clutter(240000, 0.004, seed=3, enclosure_cells=65)[:250000]
    n = len(faces)
    buf = io.StringIO()
    v = faces.reshape(-1, 3)
    for k in range(0, n, 1000):
        buf.write("o part_%d\n" % (k // 1000))
        np.savetxt(buf, v[3 * k:3 * min(n, k + 1000)], fmt="v %.9g %.9g %.9g")
        idx = np.arange(3 * k + 1, 3 * min(n, k + 1000) + 1).reshape(-1, 3)
        np.savetxt(buf, idx, fmt="f %d %d %d")
    text = buf.getvalue().encode()
    shm = "/dev/shm"
    where = shm if os.path.isdir(shm) and shutil.disk_usage(shm).free > 4 * len(text) else tempfile.gettempdir()
    path = os.path.join(where, "ffb_bench_%d.obj" % os.getpid())
    with open(path, "wb") as f:
        f.write(text)
    ctx = native.Context(device)
    ctx.obj_load(path)  # warm-up
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        info = ctx.obj_load(path)
        times.append(time.perf_counter() - t0)
    load_s = statistics.median(times)
    # scene from the parsed faces and grid rebuild (a dynamic scene's update):
    # the first one allocates the context's buffers, the median of three
    # more is the steady state
    rebuilds = []
    for _ in range(4):
        t0 = time.perf_counter()
        ctx.obj_scene_set(info["n_faces"])
        ctx.grid_build()
        ctx.synchronize()
        rebuilds.append(time.perf_counter() - t0)
    rebuild_s = statistics.median(rebuilds[1:])
    ctx.close()
    ref = None
    if Reference.available():
        t0 = time.perf_counter()
        rc, _, _, _ = Reference().obj_scene(path)
        ref_s = time.perf_counter() - t0
        if rc == 0:
            ref = {"s": ref_s, "mb_per_s": len(text) / ref_s / 1e6, "cores": 1, "kind": "reference",
                   "sample": "obj_import::scene (oracle/_ref) on the same file"}
    os.remove(path)
    return {"workload": "%d faces, %d objects, %.1f MB of OBJ text" % (n, (n + 999) // 1000, len(text) / 1e6),
            "status": info["status"], "load_s": load_s, "mb_per_s": len(text) / load_s / 1e6,
            "faces_per_s": n / load_s, "scene_and_grid_rebuild_s": rebuild_s, "first_rebuild_s": rebuilds[0],
            "path": "file read -> one upload -> GPU line split, parse, gather -> host object/material lines",
            "cpu_baseline": ref}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def fp32_peak(device):
    import ctypes as C
    from form_factors_b200 import build
    lib = C.CDLL(build.PROBE_LIB)
    lib.ffb_probe_fp32_ops.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    v = C.c_double()
    best = 0.0
    for _ in range(3):
        if lib.ffb_probe_fp32_ops(device, 20, C.byref(v)) == 0:
            best = max(best, v.value)
    return best


def measured_hbm_gbs():
    """Measured copy bandwidth of these B200s (GB/s), MEASURED_PEAKS.json or the fallback."""
    return hbm_peak()[0]


def hbm_peak():
    """(GB/s, source): MEASURED_PEAKS.json's copy bandwidth, else the
    fallback from an earlier measurement of the same GPUs."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def traffic_per_launch():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(p))
        return d.get("k_form_factors_bytes_per_launch")
    except (OSError, ValueError):
        return None


def issue_roofline(k_ms, rays_per_launch, sm_mhz, n_sm, shape=0):
    """The bound the fused kernel meets: instruction issue.  Warp
    instructions per ray from the committed ncu summary (profiles/
    traffic.json) x rays per launch / kernel time, against 4 issue slots per
    SM per cycle at the SM clock sampled during the timed region.  None when
    an input is missing."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        ipr = float(d.get("warp_inst_per_ray_by_shape", {}).get(str(shape), d["k_form_factors_warp_inst_per_ray"]))
        if not sm_mhz or not k_ms or not n_sm:
            return None
        achieved = ipr * rays_per_launch / (k_ms * 1e-3)
        peak = 4.0 * n_sm * float(sm_mhz) * 1e6
        return {"achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "G warp instructions/s",
                "frac": achieved / peak, "warp_inst_per_ray": ipr,
                "note": "instructions per ray from the committed ncu capture (profiles/traffic.json); peak = 4 x SMs x "
                        "sampled SM clock"}
    except (OSError, ValueError, KeyError, TypeError):
        return None


def ours(args):
    import torch
    import torch.distributed as dist
    from form_factors_b200 import build, native, shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    build.build()
    faces, front, rear = workload(args.rays_per_face)
    n = len(faces)
    rays_per_step = int(front.sum() + rear.sum())
    ctx = native.Context(local)
    # a real (non-default) stream shared by the library and the timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    assert ctx.stream_ptr() == stream.cuda_stream
    ctx.scene_set(faces)
    ctx.set_stats(False)  # timed launches run the kernel without counters
    dims = tuple(int(x) for x in args.grid.split(",")) if args.grid else None
    tune = None
    if dims is None and args.cells_per_face <= 0:
        # grid and launch shape chosen by the autotuner, timed on the whole
        # step (every face emits: the launch tails weigh as in the real run;
        # rank 0's choice on every rank)
        t0 = time.perf_counter()
        tune = ctx.autotune(front, rear, SEED, candidates=[dict(cells_per_face=c, skip_empty=not args.no_skip)
                                                           for c in (128.0, 192.0, 256.0)], sample_every=1,
                            force=True)
        tune["tuning_s"] = time.perf_counter() - t0
        if world > 1:
            pick = torch.tensor([tune["cells_per_face"], float(tune["shape"])], device="cuda")
            dist.broadcast(pick, 0)
            tune["cells_per_face"], tune["shape"] = float(pick[0].item()), int(pick[1].item())
            ctx.set_trace_shape(tune["shape"])
        tune["shape_params"] = native.trace_shapes()[tune["shape"]]
        ctx.set_stats(False)
    if tune is None and args.trace_shape >= 0:
        ctx.set_trace_shape(args.trace_shape)
    t0 = time.perf_counter()
    if tune is None:
        ctx.grid_build(dims=dims, cells_per_face=args.cells_per_face, skip_empty=not args.no_skip)
    else:
        ctx.grid_build(cells_per_face=tune["cells_per_face"], skip_empty=tune["skip_empty"])
    torch.cuda.synchronize()
    grid_s = time.perf_counter() - t0
    info = ctx.grid_info()
    timed_shape = ctx.trace_shape()
    # source rows of this rank (all of them on one GPU): ranks split the rows
    # of the one solve, balanced by rays, and exchange nothing while tracing
    row_b, row_e = shard.rank_rows(front, rear, rank, world)
    rows = row_e - row_b
    counts = torch.empty(rows * n, dtype=torch.int32, device="cuda")  # uint32 bit patterns

    def step(i, out=counts):
        # every rank draws the rays of its own rows of the same solve (epoch i)
        ctx.form_factor_counts_rows(front, rear, SEED, row_b, row_e, epoch=i, out=out)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    if not clocks.thread:
        time.sleep(0.2)  # nvidia-smi's first sample
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    value = rays_per_step / (ms_step * 1e-3)  # all ranks' rays of one solve per step

    # kernel-only time of the fused kernel (one launch per step), then one
    # untimed launch of the variant with counters for the work per launch
    kms = []
    for i in range(3):
        step(10_000 + i)
        kms.append(ctx.stats().kernel_ms)
    k_ms = statistics.median(kms)
    ctx.set_stats(True)
    step(10_003)
    s = ctx.stats()
    ctx.set_stats(False)
    work = torch.tensor([s.tests, s.cells, s.hits, s.jumps], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(work)
        t = torch.tensor([k_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        k_ms = float(t.item())
    tests, cells, hits, jumps = [float(x) for x in work.tolist()]
    # the zeroing of the count rows alone: a counts call in which no face
    # emits does only that (its stats time brackets the memset)
    no_rays = np.zeros_like(front)
    zms = []
    for _ in range(3):
        ctx.form_factor_counts_rows(no_rays, no_rays, SEED, row_b, row_e, epoch=0, out=counts)
        zms.append(ctx.stats().kernel_ms)
    zero_ms = statistics.median(zms)
    zero_bytes = 4 * rows * n
    step(10_004)  # counts of a real step again: the sections below format and gather them
    tests_per_launch = tests
    achieved = tests_per_launch * FLOPS_PER_TEST / (k_ms * 1e-3)
    peak = fp32_peak(local)

    # end to end through the C ABI with host buffers
    host_counts = torch.empty(rows * n, dtype=torch.int32, pin_memory=True)
    if world > 1:  # ranks on one node share its cores between their host threads
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        ctx.set_host_threads(max(1, min(12, cores // world)))
    e2e_steps = max(2, min(args.steps, 5))
    step(20_000, out=host_counts)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        step(20_001 + i, out=host_counts)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    d2h_rank = ctx.stats().d2h_bytes  # the last step's device -> host bytes
    # the same steps with every row block copied dense (no host threads)
    host_threads = ctx.host_threads()
    ctx.set_host_threads(0)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        step(20_001 + i, out=host_counts)
    e2e_dense_s = (time.perf_counter() - t0) / e2e_steps
    ctx.set_host_threads(host_threads)
    t = torch.tensor([e2e_s, e2e_dense_s], device="cuda")
    d2h_t = torch.tensor([d2h_rank], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(d2h_t)
    e2e_s, e2e_dense_s = [float(x) for x in t.tolist()]
    # host -> device per step (all ranks): one 16-byte record per emitting
    # face (face, its ray counts, its first work chunk), the chunks built on
    # the GPU; device -> host: every rank's row blocks as the (column, count)
    # pairs of their nonzero entries plus a header per block
    h2d = 16 * int(np.count_nonzero(front.astype(np.int64) + rear))
    d2h = int(d2h_t.item())
    gather = None
    if world > 1:
        # the full matrix on every rank: one NCCL all_gather of the row
        # blocks, after the timed region
        torch.cuda.synchronize()
        g0 = time.perf_counter()
        full = shard.gather_rows(counts.view(rows, n), row_b, row_e, n)
        torch.cuda.synchronize()
        ok = torch.equal(full[row_b:row_e], counts.view(rows, n))
        gather = {"s": time.perf_counter() - g0, "bytes": 4 * n * n, "own_rows_equal": bool(ok),
                  "rows": [row_b, row_e]}
        del full

    batched = served = csv = thermal = None
    if rank == 0 and world == 1 and not args.no_csv:
        csv = csv_section(ctx, stream, counts, front, rear, n)
    if rank == 0 and world == 1 and not args.no_thermal:
        thermal = thermal_section(ctx, faces, args.rays_per_face)
    obj = None
    if rank == 0 and world == 1 and not args.no_obj:
        obj = obj_section(local)
    if rank == 0 and world == 1 and not args.no_batched:
        batched = batched_section(ctx, stream, args)
    if rank == 0 and world == 1 and not args.no_served:
        served = served_section(args, ctx, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(faces, args.rays_per_face, args.cpu_sample_every)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "faces": n, "rays_per_step": rays_per_step,
                       "grid": [info.nx, info.ny, info.nz],
                       "cells_per_face": tune["cells_per_face"] if tune else args.cells_per_face,
                       "autotune": tune, "trace_shape": timed_shape,
                       "grid_refs": int(info.n_refs),
                       "grid_build_ms": 1e3 * grid_s,
                       "parallelism": "source rows split over %d ranks (one solve)" % world if world > 1 else "single",
                       "gather": gather,
                       "l2": "flushed each step by zeroing the 1.95 GB count matrix"},
            "e2e": {"value": world * rays_per_step / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3, "host_threads": host_threads,
                    "output": "the N x N uint32 counts in pinned host memory, every step",
                    "transfer": "each row block packed on the device to (column, count) pairs of its nonzero "
                                "entries; the pairs cross PCIe and host threads expand them into the host "
                                "matrix with streaming stores while the next block traces",
                    "dense_copy": {"value": world * rays_per_step / e2e_dense_s, "ms_per_step": e2e_dense_s * 1e3,
                                   "d2h_bytes_per_step": 4 * n * n,
                                   "note": "the same steps with every row block copied dense (host threads 0)"}},
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "GFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic_per_launch(),
                         "kernel": "k_form_factors", "kernel_ms": k_ms,
                         "work": "%d FP32 ops per ray/triangle test x %.4g tests per launch" % (
                             FLOPS_PER_TEST, tests_per_launch),
                         "peak_source": "measured live: FMUL+FADD issue probe (libffb200_probe.so)",
                         "hbm": {"achieved_gbs": (traffic_per_launch() or 0) / (k_ms * 1e-3) / 1e9,
                                 "peak_gbs": measured_hbm_gbs(),
                                 "frac": (traffic_per_launch() or 0) / (k_ms * 1e-3) / 1e9 / measured_hbm_gbs(),
                                 "peak_source": hbm_peak()[1],
                                 "note": "DRAM bytes per launch (ncu) / kernel time, of the copy bandwidth"},
                         "issue": issue_roofline(k_ms, rays_per_step / world, clk.get("sm_mhz"), shape=timed_shape,
                                                 n_sm=
                                                 torch.cuda.get_device_properties(local).multi_processor_count)},
            "zeroing": {"ms": zero_ms, "bytes": zero_bytes, "gbs": zero_bytes / (zero_ms * 1e-3) / 1e9,
                        "frac": zero_bytes / (zero_ms * 1e-3) / 1e9 / measured_hbm_gbs(),
                        "note": "cudaMemsetAsync of the step's count rows before the trace, CUDA events"},
            "tests_per_ray": tests / rays_per_step, "cells_per_ray": cells / rays_per_step,
            "jumps_per_ray": jumps / rays_per_step,
            "hit_fraction": hits / rays_per_step,
            "clocks": clk,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        for key, sec in (("csv", csv), ("thermal", thermal), ("obj", obj), ("batched", batched),
                         ("served", served)):
            if sec is not None:
                line[key] = sec
        # last, so that a reader of the line's tail sees the headline ratios
        summary = {"value_g_rays_per_s": value / 1e9, "e2e_g_rays_per_s": line["e2e"]["value"] / 1e9}
        if cpu is not None and cpu.get("value"):
            summary["cpu_rays_per_s"] = cpu["value"]
            summary["cpu_one_thread_rays_per_s"] = (cpu.get("one_thread") or {}).get("value")
        if batched is not None:
            summary["batched_vs_plain"] = batched["speedup_trace_resident"]
            summary["batched_vs_plain_grid_build_in_both"] = batched["speedup_grid_build_in_both"]
            summary["batched_ceiling"] = batched["ceiling"]
        if served is not None:
            summary["served_vs_plain"] = served["speedup_scenes_per_s"]
            summary["served_requests"] = served["requests"]
            summary["served_p50_s"] = served["p50_latency_s"]
            summary["served_p99_s"] = served["p99_latency_s"]
            summary["served_ceiling"] = served.get("ceiling")
            if served.get("shortest_first"):
                summary["served_shortest_first_p50_s"] = served["shortest_first"]["p50_latency_s"]
                summary["served_shortest_first_vs_plain"] = served["shortest_first"]["speedup_scenes_per_s"]
            summary["plain_p50_s"] = served["plain_p50_latency_s"]
        line["summary"] = summary
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def grid_build_only(args):
    """Builds the workload's grid args.grid_build_only times (192 cells per
    face unless --cells-per-face or --grid says otherwise) and prints the
    device time of each build: the grid-build kernels alone, for profiling."""
    import torch
    from form_factors_b200 import build, native
    build.build()
    faces, _, _ = workload(args.rays_per_face)
    ctx = native.Context(0)
    ctx.scene_set(faces)
    dims = tuple(int(x) for x in args.grid.split(",")) if args.grid else None
    cpf = args.cells_per_face if args.cells_per_face > 0 else 192.0
    times = []
    for _ in range(args.grid_build_only):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.grid_build(dims=dims, cells_per_face=cpf, skip_empty=not args.no_skip)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    info = ctx.grid_info()
    ctx.close()
    print(json.dumps({"grid_build_ms": [1e3 * t for t in times], "grid": [info.nx, info.ny, info.nz],
                      "refs": int(info.n_refs), "faces": len(faces)}))


def main():
    args = parse()
    if args.grid_build_only > 0:
        grid_build_only(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()

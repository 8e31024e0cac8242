#!/usr/bin/env python3
"""Benchmark of the diffuse benchmark path: closest + shadow rays per second (Grays/s) on B200, one JSON line.

Workloads (synthetic box-field scenes standing in for the reference's unreleased 116,855-triangle scene):
  frame512  117,002 triangles, 512 x 512, 256 spp, depth 4, batch 256 (one wavefront pass), CUDA-graph frame  [default]
  frame720  the same at 1280 x 720
  frame256  12,290 triangles, 256 x 256, 16 spp, depth 4, batch 16
  trace16m  117,002 triangles, 2^24 incoherent rays traced closest-hit and any-hit
  precision1m  12,290 triangles, 2^20 incoherent rays, precision form (f16 conservative slabs + watertight FP32
            triangles) closest + any, checked against the FP64 oracle (lost hits, ties, max relative t error)
  serving   32 resident two-level scenes (animated instances, OpenPBR materials), a Poisson stream of requests
            (256^2..1080p, 1..256 spp, depth 8) served with continuous batching and, on the same stream, by the plain
            form (one request at a time); request throughput, p50 / p95 / p99 latency, Grays/s of both
  batched64  64 two-level scenes (TLAS over 1-4,096 instances of 1-8 box-field BLAS of 1k-500k triangles each, all
            BLAS built on the GPU by one H-PLOC launch), 4M rays per scene in one scene-tagged queue, closest + any
            in one persistent launch each, launch shape chosen by the autotuner
A step is one frame (frame*) or one closest + one any-hit pass over the batch (trace16m). `value` counts the rays of
all ranks over the max over ranks of the device-timed steps (CUDA events on the renderer's stream). `e2e` is the same
metric through the C ABI with host buffers: each frame's accumulation buffer (trace16m: rays in, hits out) crosses
PCIe inside the timed region. Multi-GPU runs are independent replicas (weak scaling): the path needs no exchange.
On one GPU the frame workloads also run trace16m and precision1m (config 2's ray batch and config 3) as child
processes after the frame, and carry their measured lines, shortened, under `companions` (--companions 0: not).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload frame512] [--impl ours|reference]
"""
import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # config 2 (the 117k scene) names no SAH bin count: 128 bins build the better tree there (measured 2-6% faster on
    # both frames and the incoherent batch); config 1 and its precision form keep the 32 bins their spec names
    "frame512": dict(scene="boxes117k", w=512, h=512, spp=256, batch=256, bounces=4, bins=128),
    "frame720": dict(scene="boxes117k", w=1280, h=720, spp=256, batch=256, bounces=4, bins=128),
    "frame256": dict(scene="boxes12k", w=256, h=256, spp=16, batch=16, bounces=4, bins=32),
    "trace16m": dict(scene="boxes117k", rays=1 << 24, bins=128),
    "precision1m": dict(scene="boxes12k", rays=1 << 20, precision=True, bins=32),
    "serving": dict(serving=True, scenes=32, requests=48, rate=100.0, small_requests=400, small_rate=400.0, max_paths=16 << 20, max_requests=64, seed=7,
                    builder=1),
    "batched64": dict(batched=True, scenes=64, rays_per_scene=4 << 20, tris=(1000, 500000), instances=(1, 4096), blas=(1, 8), seed=5),
}
STATE_BYTES = 40          # path state per queued ray: (o, id) + (d, T.r) + (T.g, T.b); shadow entries the same size
LAYOUT_NAMES = {2: "bvh2", 4: "bvh4", 8: "cwbvh"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """SM clock and clock-event reasons while the timed region runs: NVML read every 10 ms from a thread (read-only
    queries), or nvidia-smi at 200 ms where NVML is unavailable."""
    Q = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    BITS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, dev_id):
        self.samples, self.p, self.t, self.mx = [], None, None, None
        self.done = threading.Event()
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByUUID(dev_id) if dev_id.startswith("GPU-") else N.nvmlDeviceGetHandleByIndex(int(dev_id))
            reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or N.nvmlDeviceGetCurrentClocksThrottleReasons
            self.mx = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))

            def run():
                while not self.done.is_set():
                    try:
                        self.samples.append((float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)), int(reasons(h))))
                    except Exception:
                        pass
                    self.done.wait(0.01)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self.t = None
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            try:
                self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200", "-i", dev_id],
                                          stdout=self.f, stderr=subprocess.DEVNULL)
            except Exception:
                self.p = None

    def stop(self):
        if self.t is not None:
            self.done.set(); self.t.join(timeout=5)
            sm = [c for c, _ in self.samples]
            reasons = sorted({n for _, r in self.samples for bit, n in self.BITS.items() if r & bit})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.mx, "reasons": reasons, "samples": len(sm),
                    "source": "nvml, 10 ms"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate(); self.p.wait(timeout=10); self.f.flush(); self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1])); mx.append(float(c[2]))
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi, 200 ms"}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0")); local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reference_lib():
    import ctypes as C
    path = os.path.join(ROOT, "oracle", "_ref", "libcwpref.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.ref_render_cpu.restype = C.c_double
    L.ref_render_cpu.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_long, C.c_long, C.c_void_p, C.c_void_p, C.c_int]
    L.ref_trace.restype = C.c_double
    L.ref_trace.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_int]
    L.ref_build.restype = C.c_long
    L.ref_build.argtypes = [C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                            C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    if hasattr(L, "ref_frame_params"):
        L.ref_params_size.restype = C.c_int
        L.ref_frame_params.restype = None
        L.ref_frame_params.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int, C.c_uint,
                                       C.c_float, C.c_float, C.c_void_p]
    if hasattr(L, "ref_trace_inst"):
        L.ref_trace_inst.restype = C.c_double
        L.ref_trace_inst.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4 + [C.c_long, C.c_void_p, C.c_void_p, C.c_int]
    return L


class RefScene:
    """A workload's scene as the reference's own host code builds it, with no part of this library loaded: the box
    field in plain Python (workloads.box_field_arrays, bit-identical to the library's generator), the reference's
    BVHBuilder (16 SAH bins, one thread, accel/bvh_builder.cpp) with its CWBVH collapse or BVH2 layout and triangle
    packing (ref_build, oracle/_ref/libcwpref.so), and the frame parameters from its camera code (ref_frame_params:
    lookAtC2W / focalFromHfov / makeCamera and setupScene's sun, eps and filter arithmetic). Attributes: p (a Params
    record), nodes, woop, tris, albedo, order, n_tris, build_ms."""

    def __init__(self, L, wl, variant, w=512, h=512, bounces=4):
        import ctypes as C
        import numpy as np
        wk = importlib.import_module("cuda-wavefront-pathtracer_b200.workloads")
        pkg = sys.modules["cuda-wavefront-pathtracer_b200"]
        v, f, fm = wk.box_field_arrays(wk.SCENES[wl["scene"]], wk.SCENE_SEED)
        nt = len(f)
        cap = 5 * 2 * nt + 64
        nodes = np.zeros((cap, 4), np.float32); order = np.zeros(nt, np.int32)
        tris = np.zeros((3 * nt, 4), np.float32); woop = np.zeros((3 * nt, 4), np.float32)
        md, sah, ms = C.c_int(), C.c_double(), C.c_double()
        n = L.ref_build(v.ctypes.data, len(v), f.ctypes.data, fm.ctypes.data, nt, variant, 4, 0, nodes.ctypes.data, cap, order.ctypes.data,
                        tris.ctypes.data, woop.ctypes.data, C.byref(md), C.byref(sah), C.byref(ms))
        assert n > 0, "ref_build failed"
        self.nodes, self.order, self.tris, self.woop = nodes[:n].copy(), order, tris, woop
        self.albedo = np.full((1, 3), wk.ALBEDO, np.float32)
        self.n_tris, self.build_ms, self.sah = nt, ms.value, sah.value
        p = pkg.Params()
        assert L.ref_params_size() == C.sizeof(p), "cwp_params and the reference harness's RefParams differ in size"
        f3 = C.c_float * 3
        ext = float(np.max(v.max(0) - v.min(0)))
        L.ref_frame_params(f3(*wk.CAM_POS), f3(*wk.CAM_TARGET), f3(*wk.CAM_UP), wk.HFOV, w, h, f3(*wk.SUN_TO), f3(*(wk.SUN_E,) * 3), f3(*wk.SKY),
                           float(np.float32(wk.SUN_ANGLE_RAD * 180.0 / math.pi)), bounces, wk.SEED, wk.EPS_SCALE, ext, C.byref(p))
        self.p = p


def cpu_frame_sample(wl, rs, variant, seconds=12.0):
    """The frame on the host cores: the reference's own host code (oracle/_ref) over the reference-built scene rs
    (RefScene), else the oracle port. Pixels are taken as a contiguous band from the middle of the image, grown until
    about `seconds` of work."""
    import ctypes as C
    import numpy as np
    p = rs.p
    threads = os.cpu_count() or 1
    L = reference_lib()
    alb = np.ascontiguousarray(rs.albedo, np.float32)
    N = wl["w"] * wl["h"]
    npix, spent, rays = 64, 0.0, 0
    while True:
        pix0 = N // 2 - npix // 2
        acc = np.zeros((N, 4), np.float32); cnt = np.zeros(2, np.int64)
        if L is not None:
            kind = "reference"
            sec = L.ref_render_cpu(C.addressof(p), variant, 1, rs.nodes.ctypes.data, rs.woop.ctypes.data, rs.tris.ctypes.data, alb.ctypes.data,
                                   wl["bounces"], wl["spp"], 0, pix0, pix0 + npix, acc.ctypes.data, cnt.ctypes.data, threads)
        else:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            from conftest import Oracle
            kind, threads = "port", 1
            t0 = time.perf_counter()
            acc, cnt = Oracle().render(p, variant, 1, rs, wl["bounces"], wl["spp"], 0, pix0, pix0 + npix)
            sec = time.perf_counter() - t0
        rays = int(cnt.sum()); spent = sec
        if sec >= seconds / 4 or npix >= N:
            break
        npix = min(N, int(npix * max(2.0, min(16.0, seconds / 4 / max(sec, 1e-3)))))
    return dict(value=rays / spent / 1e9, unit="Grays/s", cores=threads, kind=kind,
                sample=f"{npix} pixels x {wl['spp']} spp of the {wl['w']}x{wl['h']} frame ({rays} closest+shadow rays in {spent:.2f} s)",
                host_build_ms=getattr(rs, "build_ms", None),
                host_build=("the reference's BVHBuilder (16 SAH bins, one thread) and " + ("CWBVH collapse" if variant == 8 else f"BVH{variant} layout")
                            + f" of the {rs.n_tris}-triangle scene") if getattr(rs, "build_ms", None) is not None else None)


def port_scene(cwp, wl, variant, w=512, h=512, bounces=4):
    """Where oracle/_ref is not built: the scene from the library's byte-identical 16-bin build, timed as a port."""
    from types import SimpleNamespace
    mesh, bvh = cwp.scene(wl["scene"], variant=variant, bins=16)
    return SimpleNamespace(p=cwp.frame_params(mesh, w, h, bounces=bounces), nodes=bvh.nodes, woop=bvh.woop, tris=bvh.tris, albedo=bvh.albedo,
                           order=bvh.order, n_tris=mesh.n_tris, build_ms=None, stride=bvh.stride)


# DRAM bytes per launch of the frame kernels at the frame512 defaults, from a small-case capture scaled to the full
# frame: the same frame at 16 spp (batch 16, 4.2 M paths per pass, path state 0.5 GB > L2), dram__bytes_read.sum +
# dram__bytes_write.sum of every launch of one frame (one pass), per closest ray (k_trace_shade) or shadow ray
# (k_shadow), times the full frame's rays over its 6 launches (summary and command in profiles/frame512_dram_traffic.txt).
# Valid only for the configuration it was derived for.
FRAME512_TRAFFIC = {"k_trace_shade": 1930e6, "k_shadow": 628e6}
FRAME512_TRAFFIC_BINS = 128   # the build the capture ran on


def frame_traffic(args, wl, variant, kernel):
    captured = (args.workload == "frame512" and variant == 8 and args.spatial == 1e-3 and not args.spp and not args.batch and args.sort == 0
                and args.graph == 1 and args.traversal == 0 and args.bins == FRAME512_TRAFFIC_BINS and args.stage_levels <= 0)
    if not captured or kernel not in FRAME512_TRAFFIC:
        return {"traffic": None}
    return {"traffic": FRAME512_TRAFFIC[kernel], "traffic_unit": "bytes per launch",
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the 16-spp frame (one pass, every launch), scaled by rays to the full frame (profiles/frame512_dram_traffic.txt)"}


NODE_BYTES = {2: 64, 4: 128, 8: 80}
TRI_BYTES = 48   # Woop rows, an upper bound (the test reads row 2 first and rows 0/1 only past the t check)


def onchip_bytes_frame(cwp, wl, mesh, bvh, variant, npix=1024):
    """Algorithmic on-chip bytes per ray of the frame (node visits x node size + triangle tests x 48 B), counted by
    the oracle's traversal of the same tree over a band of pixels (part of the CPU-baseline leg)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import Oracle
    p = cwp.frame_params(mesh, wl["w"], wl["h"], bounces=wl["bounces"])
    N = wl["w"] * wl["h"]; pix0 = N // 2 - npix // 2
    rc, st = Oracle().render_work(p, variant, 1, bvh, wl["bounces"], min(wl["spp"], 16), pix0, pix0 + npix)
    nb = NODE_BYTES[variant]
    return dict(closest=(st[0] * nb + st[1] * TRI_BYTES) / max(rc[0], 1), shadow=(st[2] * nb + st[3] * TRI_BYTES) / max(rc[1], 1),
                nodes_per_closest=st[0] / max(rc[0], 1), tris_per_closest=st[1] / max(rc[0], 1),
                nodes_per_shadow=st[2] / max(rc[1], 1), tris_per_shadow=st[3] / max(rc[1], 1),
                sample=f"oracle traversal of {npix} pixels x {min(wl['spp'], 16)} spp ({int(rc[0])} closest, {int(rc[1])} shadow rays) on the same tree")


def onchip_bytes_trace(cwp, bvh, variant, o, d, n=1 << 15):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import Oracle
    orc = Oracle(); nb = NODE_BYTES[variant]
    _, sc = orc.trace(variant, 1, False, bvh.nodes, bvh.woop, o[:n], d[:n], stats=True)
    _, sa = orc.trace(variant, 1, True, bvh.nodes, bvh.woop, o[:n], d[:n], stats=True)
    return dict(closest=(sc[0] * nb + sc[1] * TRI_BYTES) / n, shadow=(sa[0] * nb + sa[1] * TRI_BYTES) / n,
                nodes_per_closest=sc[0] / n, tris_per_closest=sc[1] / n, nodes_per_shadow=sa[0] / n, tris_per_shadow=sa[1] / n,
                sample=f"oracle traversal of {n} of the batch's rays on the same tree")


def cpu_trace_sample(bvh, variant, o, d, seconds=12.0):
    """Closest-hit and any-hit traversal of a sample of the batch on the host cores with the reference's own trav<>
    (oracle/_ref), else the oracle port. bvh: anything with nodes, woop (RefScene)."""
    import numpy as np
    L = reference_lib(); threads = os.cpu_count() or 1
    n, spent = 1 << 14, 0.0
    while True:
        hits = np.zeros((n, 4), np.float32); occ = np.zeros(n, np.int32)
        if L is not None:
            kind = "reference"
            spent = L.ref_trace(variant, 0, 1, bvh.nodes.ctypes.data, bvh.woop.ctypes.data, o[:n].ctypes.data, d[:n].ctypes.data, n, hits.ctypes.data, None, threads)
            spent += L.ref_trace(variant, 1, 1, bvh.nodes.ctypes.data, bvh.woop.ctypes.data, o[:n].ctypes.data, d[:n].ctypes.data, n, None, occ.ctypes.data, threads)
        else:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            from conftest import Oracle
            kind, threads = "port", 1
            t0 = time.perf_counter(); orc = Oracle()
            orc.trace(variant, 1, False, bvh.nodes, bvh.woop, o[:n], d[:n]); orc.trace(variant, 1, True, bvh.nodes, bvh.woop, o[:n], d[:n])
            spent = time.perf_counter() - t0
        if spent >= seconds / 4 or n >= len(o):
            break
        n = min(len(o), int(n * max(2.0, min(16.0, seconds / 4 / max(spent, 1e-3)))))
    return dict(value=2 * n / spent / 1e9, unit="Grays/s", cores=threads, kind=kind,
                sample=f"{n} of the {len(o)} incoherent rays, closest-hit and any-hit ({2 * n} rays in {spent:.2f} s)",
                host_build_ms=getattr(bvh, "build_ms", None),
                host_build=(f"the reference's BVHBuilder (16 SAH bins, one thread) and " + ("CWBVH collapse" if variant == 8 else f"BVH{variant} layout")
                            + f" of the {bvh.n_tris}-triangle scene") if getattr(bvh, "build_ms", None) is not None else None)


METRIC_FRAME = "closest+shadow rays per second, diffuse frame"
METRIC_BATCH = "closest+any rays per second, incoherent ray batch"
METRIC_BATCHED = "closest+any rays per second, batched two-level scenes"
METRIC_SERVING = "serving request throughput (continuous batching), Poisson stream of config-5 requests"


def run_reference(args, wl, rank):
    """--impl reference: the reference's CPU implementation of the path on this host's cores (rank 0 only), with the
    product arm's metric, unit and workload."""
    if rank != 0:
        return
    if wl.get("batched") or wl.get("serving"):
        why = ("the reference has no host path for many two-level scenes in one queue (its travInst on the host cores is the "
               "batched64 line's cpu_baseline)" if wl.get("batched") else "the reference has no serving loop")
        print(json.dumps({"impl": "reference", "metric": METRIC_BATCHED if wl.get("batched") else METRIC_SERVING, "unavailable": why}), flush=True)
        return
    # nothing of this library is loaded on this arm: the scene, the BVH, the frame parameters and the rays come from
    # the reference's own host code (oracle/_ref/libcwpref.so) and plain Python
    variant = args.variant
    L = reference_lib()
    if L is None or not hasattr(L, "ref_frame_params"):
        print(json.dumps({"impl": "reference", "metric": METRIC_FRAME if "rays" not in wl else METRIC_BATCH,
                          "unavailable": "oracle/_ref/libcwpref.so (the reference's host code compiled from its sources) is not built"}), flush=True)
        return
    importlib.import_module("cuda-wavefront-pathtracer_b200")   # ctypes records and workloads only; the CUDA library is not loaded
    wk = importlib.import_module("cuda-wavefront-pathtracer_b200.workloads")
    rs = RefScene(L, wl, variant, w=wl.get("w", 512), h=wl.get("h", 512), bounces=wl.get("bounces", 4))
    vals = []
    for i in range(args.warmup + args.steps):
        if "rays" in wl:
            import numpy as np

            def tr(o, d):   # the reference's host traversal finds the surface points of the incoherent batch
                h = np.zeros((len(o), 4), np.float32)
                L.ref_trace(variant, 0, 1, rs.nodes.ctypes.data, rs.woop.ctypes.data, o.ctypes.data, d.ctypes.data, len(o), h.ctypes.data, None, 0)
                return h
            if i == 0:
                ro, rd = wk.incoherent_rays(1 << 20, rs.p, rs.tris, tr, seed=41)
            cb = cpu_trace_sample(rs, variant, ro, rd, seconds=args.ref_seconds)
        else:
            cb = cpu_frame_sample(wl, rs, variant, seconds=args.ref_seconds)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    if "rays" not in wl:
        config = {"workload": args.workload, "scene": f"{wl['scene']} ({rs.n_tris} triangles, box field seed 1)", "resolution": f"{wl['w']}x{wl['h']}",
                  "spp": wl["spp"], "batch": wl["batch"], "depth": wl["bounces"], "layout": LAYOUT_NAMES[variant], "sah_bins": 16, "tri": "woop",
                  "bvh": "binned SAH (the reference's BVHBuilder, 16 bins)"}
    else:
        config = {"workload": args.workload, "scene": f"{wl['scene']} ({rs.n_tris} triangles)", "rays": wl["rays"], "layout": LAYOUT_NAMES[variant],
                  "sah_bins": 16, "tri": "woop", "bvh": "binned SAH (the reference's BVHBuilder, 16 bins)"}
    assert sys.modules["cuda-wavefront-pathtracer_b200"]._lib is None, "the reference arm loaded this library"
    print(json.dumps({"impl": "reference", "metric": METRIC_FRAME if "rays" not in wl else METRIC_BATCH,
                      "value": v, "unit": "Grays/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "config": config,
                      "cpu_baseline": cb, "e2e": {"value": v, "unit": "Grays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def reference_cuda_frame(cwp, wl, mesh, p, ours_ms, ours_img, device, reps=2):
    """The same frame rendered by the reference's own CUDA build on this GPU (oracle/_ref/pt, compiled from its
    sources for sm_100 with its own flags), outside the timed region, from the same scene written as PLY with the
    camera and lighting files (its binned-SAH BVHBuilder at 16 bins builds its tree). Records its frame time on BVH2
    and BVH8 (best of `reps` after its warm-up), this library's frame time on the same 16-bin trees and on the
    benchmark's own tree (ours_ms, the bench's timed frames), the ratios, and the PSNR of every image against the
    reference's BVH2 image."""
    import tempfile as tf
    pt = os.path.join(ROOT, "oracle", "_ref", "pt")
    if not os.path.exists(pt):
        return {"unavailable": "oracle/_ref/pt (the reference's CUDA build) is not built"}
    w, h, spp, K, B = wl["w"], wl["h"], wl["spp"], wl["batch"], wl["bounces"]
    rec = {"command": "oracle/_ref/pt --mesh scene.ply --camera camera.json --lighting lighting.json --albedo 0.7 0.7 0.7 --filter box "
                      f"--hfov 45 --width {w} --height {h} --spp {spp} --bounces {B} --variant bvh2|bvh8 --tri woop --fuse 1 --batch {K} --leaf 4 --reps {reps}"}
    ref_img = None
    with tf.TemporaryDirectory() as tmp:
        for rv in ("bvh2", "bvh8"):
            a = cwp.reference_inputs(mesh, p, tmp, w, h, spp, K, variant=rv)
            out = os.path.join(tmp, f"ref_{rv}")
            res = subprocess.run([pt] + a + ["--out", out, "--reps", str(reps)], capture_output=True, text=True, timeout=900)   # one-GPU runs: its device 0 is ours
            if res.returncode != 0:
                return {"unavailable": f"oracle/_ref/pt exited {res.returncode}: {res.stderr.strip().splitlines()[-1:] }"}
            lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
            best = min(lines, key=lambda l: l["t_frame_ms"])
            img = cwp.imageio.read_pfm(out + ".pfm")
            ref_img = img if ref_img is None else ref_img
            rec[f"reference_{rv}"] = {"t_frame_ms": best["t_frame_ms"], "rays_total": best["rays_total"], "grays_s": best["rays_total"] / best["t_frame_ms"] / 1e6,
                                      "psnr_vs_reference_bvh2_db": cwp.imageio.psnr(img, ref_img) if rv != "bvh2" else None}
    for variant in (2, 8):
        _, bvh = cwp.scene(wl["scene"], variant=variant, bins=16)
        r = cwp.Renderer(); r.init(p, bvh, variant=variant, batch=K, bounces=B, device=device)
        r.render(spp)   # graph capture
        best = min((r.render(spp) for _ in range(reps)), key=lambda st: st.frame_ms)
        img = cwp.imageio.accum_to_image(r.read_accum(), w, h, spp)
        r.close()
        rec[f"ours_same_tree_{LAYOUT_NAMES[variant]}"] = {"t_frame_ms": best.frame_ms, "grays_s": (best.rays + best.shadow_rays) / best.frame_ms / 1e6,
                                                          "psnr_vs_reference_bvh2_db": cwp.imageio.psnr(img, ref_img)}
    # binned SAH at the 32 bins BASELINE's config 1 names (the reference's split rule; its own builder has 16 bins)
    _, bvh = cwp.scene(wl["scene"], variant=8, bins=32)
    r = cwp.Renderer(); r.init(p, bvh, variant=8, batch=K, bounces=B, device=device)
    r.render(spp)
    best = min((r.render(spp) for _ in range(reps)), key=lambda st: st.frame_ms)
    img = cwp.imageio.accum_to_image(r.read_accum(), w, h, spp)
    r.close()
    rec["ours_binned32_cwbvh"] = {"t_frame_ms": best.frame_ms, "grays_s": (best.rays + best.shadow_rays) / best.frame_ms / 1e6,
                                  "psnr_vs_reference_bvh2_db": cwp.imageio.psnr(img, ref_img)}
    rec["ours_benchmark_tree"] = {"t_frame_ms": ours_ms, "psnr_vs_reference_bvh2_db": cwp.imageio.psnr(ours_img, ref_img)}
    ref_best = min(rec["reference_bvh2"]["t_frame_ms"], rec["reference_bvh8"]["t_frame_ms"])
    same_best = min(rec["ours_same_tree_bvh2"]["t_frame_ms"], rec["ours_same_tree_cwbvh"]["t_frame_ms"])
    rec["speedup_same_tree"] = ref_best / same_best
    rec["speedup_binned32_tree"] = ref_best / rec["ours_binned32_cwbvh"]["t_frame_ms"]
    rec["speedup_benchmark_tree"] = ref_best / ours_ms
    rec["note"] = ("ratios are the reference's best frame time (BVH2 or BVH8) over ours: on the same 16-bin binned-SAH trees (kernels alone), "
                   "on a 32-bin binned-SAH CWBVH built by this library with the reference's split rule (kernels and bin count), "
                   "and on the benchmark's own tree (kernels and tree); frame times are CUDA-event frame times of each build's own frame loop")
    return rec


def batched_setup(cwp, wl):
    meshes, xf, mesh_of, first = cwp.batch_scenes(n_scenes=wl["scenes"], seed=wl["seed"], tris=wl["tris"], instances=wl["instances"], blas_per_scene=wl["blas"])
    return meshes, xf, mesh_of, first


def batched_rays(torch, xf, first, per, seed=9, extent=40.0):
    """The queue on the device, scene-major: origins uniform in each scene's instance-translation box grown by the
    mesh extent, directions uniform on the sphere (tmin 0, tmax 1e30), int32 scene id per ray."""
    import numpy as np
    n_s = len(first) - 1
    g = torch.Generator(device="cuda"); g.manual_seed(seed)
    o = torch.empty((n_s * per, 4), dtype=torch.float32, device="cuda"); d = torch.empty_like(o)
    for s in range(n_s):
        a, b = int(first[s]), int(first[s + 1])
        t = xf[a:b].reshape(-1, 3, 4)[:, :, 3] if b > a else np.zeros((1, 3), np.float32)
        lo = torch.tensor(t.min(0) - extent, device="cuda"); hi = torch.tensor(t.max(0) + extent, device="cuda")
        sl = slice(s * per, (s + 1) * per)
        o[sl, :3] = lo + torch.rand((per, 3), generator=g, device="cuda") * (hi - lo); o[sl, 3] = 0.0
        v = torch.randn((per, 3), generator=g, device="cuda"); v /= v.norm(dim=1, keepdim=True)
        d[sl, :3] = v; d[sl, 3] = 1e30
    sc = torch.arange(n_s, dtype=torch.int32, device="cuda").repeat_interleave(per)
    return o, d, sc


def cpu_batched_sample(b, tuning_width, n_scenes, n_inst, o, d, sc, seconds=12.0):
    """The reference's two-level traversal (travInst, accel/traverse_inst.cuh, via oracle/_ref) on the host cores over
    a strided sample of the queue on the GPU-built buffers; the oracle restatement when the reference is absent."""
    import numpy as np
    nodes, tris = b.download(tuning_width)
    b.set_tlas_width(2)   # the reference's travInst reads a BVH2 TLAS (both forms are built)
    tlas, roots, inst = b.download_tlas(n_scenes, n_inst)
    b.set_tlas_width(4)
    L = reference_lib(); threads = os.cpu_count() or 1
    n = 1 << 12
    while True:
        step = max(1, len(o) // n)
        oo = np.ascontiguousarray(o[::step][:n]); dd = np.ascontiguousarray(d[::step][:n]); ss = np.ascontiguousarray(sc[::step][:n])
        m = len(oo)
        hits = np.zeros((m, 4), np.float32); hi = np.zeros(m, np.int32)
        if L is not None and hasattr(L, "ref_trace_inst"):
            kind = "reference"
            spent = L.ref_trace_inst(tuning_width, 0, 0, nodes.ctypes.data, tris.ctypes.data, tlas.ctypes.data, roots.ctypes.data, n_scenes, inst.ctypes.data,
                                     oo.ctypes.data, dd.ctypes.data, ss.ctypes.data, m, hits.ctypes.data, hi.ctypes.data, threads)
            spent += L.ref_trace_inst(tuning_width, 1, 0, nodes.ctypes.data, tris.ctypes.data, tlas.ctypes.data, roots.ctypes.data, n_scenes, inst.ctypes.data,
                                      oo.ctypes.data, dd.ctypes.data, ss.ctypes.data, m, None, hi.ctypes.data, threads)
        else:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            from conftest import Oracle
            kind, threads = "port", 1
            orc = Oracle(); t0 = time.perf_counter()
            orc.trace_inst(tuning_width, False, nodes, tris, tlas, roots, inst, oo, dd, ss); orc.trace_inst(tuning_width, True, nodes, tris, tlas, roots, inst, oo, dd, ss)
            spent = time.perf_counter() - t0
        if spent >= seconds / 4 or m >= len(o):
            break
        n = min(len(o), int(n * max(2.0, min(16.0, seconds / 4 / max(spent, 1e-3)))))
    return dict(value=2 * m / spent / 1e9, unit="Grays/s", cores=threads, kind=kind,
                sample=f"every {step}th ray of the {len(o)}-ray queue ({m} rays, closest-hit and any-hit, {2 * m} rays in {spent:.2f} s)")


def bench_batched(args, wl, cwp, torch, ws, rank, barrier, reduce, dev_id, hbm_peak, peak_kind, out):
    import numpy as np
    t0 = time.perf_counter()
    meshes, xf, mesh_of, first = batched_setup(cwp, wl)
    gen_s = time.perf_counter() - t0
    b = cwp.Batch(meshes, device=torch.cuda.current_device(), builder=args.builder, spatial=args.spatial if args.builder == 1 else 0.0,
                  tlas_width=args.tlas_width)
    inst = cwp.instances(xf, mesh_of)
    b.set_scenes(inst, first)
    info = b.info()
    n_s = len(first) - 1
    per = args.rays if args.rays else wl["rays_per_scene"]
    o, d, sc = batched_rays(torch, xf, first, per)
    n = len(o)
    hits = torch.empty((n, 4), dtype=torch.float32, device="cuda"); hi = torch.empty(n, dtype=torch.int32, device="cuda"); oi = torch.empty(n, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    # autotuner on a strided sample (every 32nd ray, all scenes represented)
    samp = torch.arange(0, n, 32, device="cuda")
    so, sd, ss = o[samp].contiguous(), d[samp].contiguous(), sc[samp].contiguous()
    sh = torch.empty((len(samp), 4), dtype=torch.float32, device="cuda"); si = torch.empty(len(samp), dtype=torch.int32, device="cuda")
    t1 = time.perf_counter()
    if args.tuning:
        blk, wd, fe, sm = (int(x) for x in args.tuning.split(","))
        b.set_tuning(blk, wd, fe, sm); tun = b.tuning()
    else:
        tun = b.autotune(so.data_ptr(), sd.data_ptr(), ss.data_ptr(), sh.data_ptr(), si.data_ptr(), len(samp))
    tune_s = time.perf_counter() - t1
    del so, sd, ss, sh, si

    def step(ev=None):
        if ev: ev[0].record(st)
        b.trace(o.data_ptr(), d.data_ptr(), sc.data_ptr(), hits.data_ptr(), hi.data_ptr(), n, stream=st.cuda_stream)
        if ev: ev[1].record(st)
        b.trace(o.data_ptr(), d.data_ptr(), sc.data_ptr(), 0, oi.data_ptr(), n, any_hit=True, stream=st.cuda_stream)
        if ev: ev[2].record(st)
    for _ in range(args.warmup):
        step()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    clk = Clocks(dev_id)
    barrier()
    torch.cuda.nvtx.range_push("timed")
    for i in range(args.steps):
        step(ev[i])
    torch.cuda.nvtx.range_pop()
    barrier()
    clocks = clk.stop()
    b.status()
    c_ms = sum(e[0].elapsed_time(e[1]) for e in ev); a_ms = sum(e[1].elapsed_time(e[2]) for e in ev)
    max_ms = reduce(c_ms + a_ms, "max")
    value = 2 * n * args.steps * ws / (max_ms * 1e-3) / 1e9
    hit_rate = float((hi >= 0).float().mean().item())
    # e2e: pinned host queue in, hits + instances out, every step, through the C ABI. The queue goes in 8 chunks:
    # chunk c's rays are copied in on one stream while chunk c - 1 is traced on the batch's stream and chunk c - 2's
    # results are copied out on a third (the traversal launches stay on one stream: they share the batch's cursor).
    ho, hd, hs = o.cpu().pin_memory(), d.cpu().pin_memory(), sc.cpu().pin_memory()
    hh = torch.empty((n, 4), dtype=torch.float32, pin_memory=True); hhi = torch.empty(n, dtype=torch.int32, pin_memory=True); hoi = torch.empty(n, dtype=torch.int32, pin_memory=True)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    nch = 8 if n >= 8 << 20 else 1
    cut = [n * i // nch for i in range(nch + 1)]

    def e2e_step():
        for c in range(nch):
            lo, hi_ = cut[c], cut[c + 1]
            with torch.cuda.stream(s_in):
                o[lo:hi_].copy_(ho[lo:hi_], non_blocking=True); d[lo:hi_].copy_(hd[lo:hi_], non_blocking=True); sc[lo:hi_].copy_(hs[lo:hi_], non_blocking=True)
            st.wait_stream(s_in)
            b.trace(o[lo].data_ptr(), d[lo].data_ptr(), sc[lo:].data_ptr(), hits[lo].data_ptr(), hi[lo:].data_ptr(), hi_ - lo, stream=st.cuda_stream)
            b.trace(o[lo].data_ptr(), d[lo].data_ptr(), sc[lo:].data_ptr(), 0, oi[lo:].data_ptr(), hi_ - lo, any_hit=True, stream=st.cuda_stream)
            s_out.wait_stream(st)
            with torch.cuda.stream(s_out):
                hh[lo:hi_].copy_(hits[lo:hi_], non_blocking=True); hhi[lo:hi_].copy_(hi[lo:hi_], non_blocking=True); hoi[lo:hi_].copy_(oi[lo:hi_], non_blocking=True)
        torch.cuda.current_stream().wait_stream(s_out)
    ref_h, ref_i, ref_o = hits.cpu(), hi.cpu(), oi.cpu()   # the whole-queue launches of the device-timed steps
    e2e_step(); barrier(); t2 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    barrier(); e_s = reduce(time.perf_counter() - t2, "max")
    # the chunked calls give the whole-queue launches' results (rays are independent)
    assert torch.equal(hhi, ref_i) and torch.equal(hoi, ref_o) and torch.equal(hh.view(torch.int32), ref_h.view(torch.int32))
    del ref_h, ref_i, ref_o
    dom_ms, dom_b, dom = (c_ms, 56.0, "k_batch_trace (closest)") if c_ms >= a_ms else (a_ms, 40.0, "k_batch_trace (any)")
    achieved = dom_b * n * args.steps / (dom_ms * 1e-3) / 1e9
    out.update(metric=METRIC_BATCHED, value=value, ms_per_step=max_ms / args.steps,
               config={"workload": args.workload, "scenes": n_s, "blas": info.n_blas, "tris": int(info.n_tris), "instances": int(info.n_instances),
                       "rays": n, "rays_per_scene": per, "hit_rate": hit_rate,
                       "tuning": {"block": tun.block, "width": tun.width, "fetch": tun.fetch, "smem_stack": tun.smem_stack, "sample_ms": tun.ms},
                       "tlas_width": args.tlas_width,
                       "autotune_s": tune_s, "blas_builder": ["gpu h-ploc (one launch)", "host binned SAH" + (f", spatial splits at {args.spatial:g}" if args.spatial > 0 else "")][args.builder], "blas_build_ms": info.blas_build_ms,
                       "blas_hploc_launches": info.blas_hploc_launches if args.builder == 0 else 0,
                       "tlas_build_ms": info.tlas_build_ms, "node_bytes": {"bvh2": int(info.node_bytes[0]), "bvh4": int(info.node_bytes[1]), "cwbvh": int(info.node_bytes[2])},
                       "scene_generation_s": gen_s, "l2": f"ray queue {n * 36 / 1e9:.1f} GB > L2 (126 MB)",
                       "closest_ms": c_ms / args.steps, "any_ms": a_ms / args.steps, "tri": "moller-trumbore"},
               clocks=clocks,
               e2e={"value": 2 * n * args.steps * ws / e_s / 1e9, "unit": "Grays/s", "h2d_bytes_per_step": n * 36, "d2h_bytes_per_step": n * 24},
               gpu_launches=2 * args.steps,
               roofline={"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "peak_kind": peak_kind, "traffic": None,
                         "algorithmic": "closest: 32 B ray + 4 B scene id in, 16 B hit + 4 B instance out; any: 36 B in + 4 B out"})
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        oh, dh, sh_ = o.cpu().numpy(), d.cpu().numpy(), sc.cpu().numpy()
        out["cpu_baseline"] = cpu_batched_sample(b, tun.width, n_s, len(mesh_of), oh, dh, sh_, seconds=args.ref_seconds)


def serve_stream(cwp, s, stream):
    """Feeds (arrival_s, request) pairs at their arrival times and steps the server until all are done: per request
    (latency ms, rays, shadow rays); throughput over the span from the first arrival to the last completion."""
    t0 = s.clock_ms(); todo = list(stream); ids = {}; done = {}
    while len(done) < len(stream):
        if s.clock_ms() - t0 > 900e3:
            raise RuntimeError(f"serving stream did not finish in 900 s ({len(done)} of {len(stream)} done)")
        now = (s.clock_ms() - t0) / 1e3
        while todo and todo[0][0] <= now:
            arr, r = todo.pop(0); ids[s.submit(r)] = arr
        a, p = s.step()
        for i in s.poll():
            _, st = s.result(i)
            done[i] = (st.done_ms - st.submit_ms, st.rays, st.shadow_rays, st.done_ms - t0)
        if a == 0 and p == 0 and todo and len(done) < len(stream):
            time.sleep(max(0.0, min(0.002, todo[0][0] - (s.clock_ms() - t0) / 1e3)))
    lat = sorted(v[0] for v in done.values())
    span = max(v[3] for v in done.values()) / 1e3 - stream[0][0]
    rays = sum(v[1] + v[2] for v in done.values())
    q = lambda f: lat[min(len(lat) - 1, int(f * len(lat)))]
    return {"requests": len(lat), "throughput_req_s": len(lat) / span, "grays_s": rays / span / 1e9, "p50_ms": q(0.50), "p95_ms": q(0.95), "p99_ms": q(0.99),
            "span_s": span, "rays": rays}


def equal_p99(cont, plain):
    """Throughput at equal p99 latency from two (arrival rate -> throughput, p99) sweeps: for each latency bound L
    (every p99 either form reached), the highest throughput each form sustained with p99 <= L, and their ratio."""
    bounds = sorted({pt["p99_ms"] for pt in cont + plain})
    best = lambda pts, L: max([pt["throughput_req_s"] for pt in pts if pt["p99_ms"] <= L] or [0.0])
    rows = []
    for L in bounds:
        c, p = best(cont, L), best(plain, L)
        rows.append({"p99_bound_ms": L, "continuous_req_s": c, "plain_req_s": p, "ratio": c / p if p > 0 else None})
    ratios = [r["ratio"] for r in rows if r["ratio"] is not None]
    # the bound at which the plain form reaches its best throughput (its capacity within any bound it meets)
    pmax = max(pt["throughput_req_s"] for pt in plain)
    Lp = min(pt["p99_ms"] for pt in plain if pt["throughput_req_s"] >= pmax * 0.999)
    at = next(r for r in rows if r["p99_bound_ms"] == Lp)
    return {"rows": rows, "max_ratio": max(ratios) if ratios else None, "median_ratio": statistics.median(ratios) if ratios else None,
            "at_plain_capacity": at}


def slo_sweep(cwp, b, mats, base, descs, first, wl, maxr, args, boxes, name, rates, n_req, resolutions=None, spps=None):
    """Each form fed Poisson streams of n_req requests at each arrival rate: (rate, throughput, p50, p99) points."""
    pts = {"continuous": [], "plain": []}
    for rate in rates:
        stream = cwp.serving_requests(n_req, rate, boxes, seed=wl["seed"] + 100 + int(rate * 10), resolutions=resolutions, spps=spps)
        for mode, m in (("continuous", maxr), ("plain", 1)):
            s = cwp.Server(b, mats, base, max_paths=args.paths or wl["max_paths"], max_requests=m, regroup=bool(args.regroup), policy=args.policy, overlap=bool(args.overlap))
            s.set_scenes(descs, first)
            r = serve_stream(cwp, s, stream)
            pts[mode].append({"rate_req_s": rate, "throughput_req_s": r["throughput_req_s"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"]})
            del s
    return {"stream": name, "requests_per_point": n_req, "points": pts, "equal_p99": equal_p99(pts["continuous"], pts["plain"])}


def bench_serving(args, wl, cwp, torch, out, barrier=lambda: None, reduce=lambda x, op: x):
    """Two request streams, each served by continuous batching and by the plain form (one request at a time, the same
    kernels): `mix` draws config 5's distribution (256^2..1080p, 1..256 spp), where single large requests already
    fill the GPU; `small` draws 256^2 / 512^2 at 1 / 4 spp, where one request alone leaves the GPU mostly idle."""
    import numpy as np
    t0 = time.perf_counter()
    meshes, descs, first, mats, base, boxes = cwp.serving_scenes(n_scenes=wl["scenes"], seed=wl["seed"])
    # BLAS on the host cores, binned SAH (spatial splits only with --serve-spatial: measured 2.3x slower here)
    b = cwp.Batch(meshes, device=torch.cuda.current_device(), builder=wl["builder"], spatial=args.serve_spatial, tlas_width=args.tlas_width)
    if args.tuning:
        blk, wd, fe, sm = (int(x) for x in args.tuning.split(","))
        b.set_tuning(blk, wd, fe, sm)
    gen_s = time.perf_counter() - t0
    n_req = args.rays if args.rays else wl["requests"]
    streams = {"mix": cwp.serving_requests(n_req, wl["rate"], boxes, seed=wl["seed"] + 1),
               "small": cwp.serving_requests(wl["small_requests"], wl["small_rate"], boxes, seed=wl["seed"] + 2, resolutions=[(256, 256), (512, 512)], spps=[1, 4])}
    res = {}
    maxr_c = args.max_requests or wl["max_requests"]
    for name, stream in streams.items():
        for mode, maxr in (("continuous", maxr_c), ("plain", 1)):
            s = cwp.Server(b, mats, base, max_paths=args.paths or wl["max_paths"], max_requests=maxr, regroup=bool(args.regroup), policy=args.policy, overlap=bool(args.overlap))
            s.set_scenes(descs, first)
            barrier()
            clk = Clocks(str(torch.cuda.current_device()))
            r = serve_stream(cwp, s, stream)
            r["clocks"] = clk.stop(); r["breakdown"] = s.info()
            # replicas: every rank serves its own copy of the stream; the job's throughput is all requests over the
            # slowest rank's span
            r["job_throughput_req_s"] = reduce(r["requests"], "sum") / reduce(r["span_s"], "max")
            res[(name, mode)] = r
            del s
    sweeps = {}
    if args.slo_sweep:
        sweeps["small"] = slo_sweep(cwp, b, mats, base, descs, first, wl, maxr_c, args, boxes, "small", [25.0, 50.0, 75.0, 100.0, 150.0], 200,
                                    resolutions=[(256, 256), (512, 512)], spps=[1, 4])
        sweeps["mix"] = slo_sweep(cwp, b, mats, base, descs, first, wl, maxr_c, args, boxes, "mix", [0.75, 1.5, 3.0], 64)
    info = b.info()
    c, p = res[("mix", "continuous")], res[("mix", "plain")]
    cs, ps = res[("small", "continuous")], res[("small", "plain")]
    strip = lambda r: {k: v for k, v in r.items() if k != "clocks"}
    out.update(metric=METRIC_SERVING, value=c["job_throughput_req_s"], unit="req/s",
               ms_per_step=1e3 / c["job_throughput_req_s"], higher_is_better=True, dtype="f32",
               config={"workload": args.workload, "scenes": wl["scenes"], "blas": info.n_blas, "tris": int(info.n_tris), "blas_builder": ["gpu h-ploc", "host binned SAH, 32 bins" + (f", spatial splits at {args.serve_spatial:g}" if args.serve_spatial > 0 else "")][wl["builder"]],
                       "blas_build_ms": info.blas_build_ms, "scene_generation_s": gen_s, "depth": 8, "max_paths": wl["max_paths"], "max_requests": maxr_c,
                       "tlas_width": args.tlas_width, "regroup": bool(args.regroup), "policy": ["even share", "oldest first with backfill"][args.policy],
                       "overlap": bool(args.overlap),
                       "materials": "OpenPBR subset: roughness U[0.05,1], metallic Bernoulli(0.3), 10% glass IOR 1.5",
                       "mix": {"requests": n_req, "arrival_rate_req_s": wl["rate"], "resolutions": "256^2, 512^2, 1280x720, 1920x1080", "spp": "1, 4, 16, 64, 256",
                               "continuous": strip(c), "plain": strip(p), "throughput_vs_plain": c["throughput_req_s"] / p["throughput_req_s"],
                               "p99_vs_plain": c["p99_ms"] / p["p99_ms"], "p50_vs_plain": c["p50_ms"] / p["p50_ms"]},
                       "small": {"requests": wl["small_requests"], "arrival_rate_req_s": wl["small_rate"], "resolutions": "256^2, 512^2", "spp": "1, 4",
                                 "continuous": strip(cs), "plain": strip(ps), "throughput_vs_plain": cs["throughput_req_s"] / ps["throughput_req_s"],
                                 "p99_vs_plain": cs["p99_ms"] / ps["p99_ms"], "p50_vs_plain": cs["p50_ms"] / ps["p50_ms"]},
                       "throughput_at_equal_p99": sweeps or None},
               clocks=c["clocks"],
               e2e={"value": c["job_throughput_req_s"], "unit": "req/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": None,
                    "note": "requests enter through the C ABI with host descriptors; images stay on the device until cwp_server_result"},
               gpu_launches=None)


COMPANION_KEYS = ("closest_ms", "any_ms", "references", "rays", "bvh", "lost_hits", "tie_mismatches", "extra_hits", "max_t_error", "plain_grays_s", "vs_plain")


def companions(args):
    """trace16m and precision1m, each in a child process on this GPU (its own context, run after the frame): their
    JSON lines with the config shortened to the figures that describe the result."""
    res = {}
    for name in ("trace16m", "precision1m"):
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", name, "--steps", str(max(args.steps, 3)), "--warmup", str(max(args.warmup, 3)),
               "--no-cpu-baseline", "--companions", "0"]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=dict(os.environ))
            line = [l for l in r.stdout.splitlines() if l.startswith("{")]
            if r.returncode != 0 or not line:
                res[name] = {"error": f"exit {r.returncode}: {r.stderr.strip().splitlines()[-1] if r.stderr.strip() else 'no output'}"}
                continue
            d = json.loads(line[-1])
            res[name] = {"metric": d["metric"], "value": d["value"], "unit": d["unit"], "steps": d["steps"], "warmup": d["warmup"], "ms_per_step": d["ms_per_step"],
                         "e2e": d.get("e2e"), "clocks": d.get("clocks"), "config": {k: d["config"][k] for k in COMPANION_KEYS if k in d["config"]}}
        except subprocess.TimeoutExpired:
            res[name] = {"error": "timed out after 900 s"}
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="frame512", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", type=int, default=8, choices=[2, 4, 8])
    ap.add_argument("--bins", type=int, default=0, help="SAH bins of the host build (default: the workload's)")
    ap.add_argument("--graph", type=int, default=1)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-cuda", type=int, default=1, help="frames: also render the frame with the reference's CUDA build (oracle/_ref/pt), outside the timed region")
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--spp", type=int, default=0, help="override the frame's samples per pixel (profiling cases)")
    ap.add_argument("--rays", type=int, default=0, help="override the batch size of trace16m / rays per scene of batched64 (profiling cases)")
    ap.add_argument("--scenes", type=int, default=0, help="override the scene count of batched64 (profiling cases)")
    ap.add_argument("--tuning", default="", help="batched64 / serving: fixed launch shape block,width,fetch,smem (batched64: instead of the autotuner)")
    ap.add_argument("--builder", type=int, default=0, help="batched64: 0 every BLAS on the GPU (H-PLOC, one launch), 1 on the host cores (binned SAH)")
    ap.add_argument("--precision", action="store_true", help="ray-batch workloads: use the precision form")
    ap.add_argument("--traversal", type=int, default=0, help="0 auto (persistent refill for BVH2/CWBVH), 1 refill, 2 one 32-ray fetch per warp")
    ap.add_argument("--spatial", type=float, default=1e-3, help="host BVH: spatial-split overlap threshold (1e-3 = SBVH, the default; 0 = the reference binned SAH only)")
    ap.add_argument("--paths", type=int, default=0, help="serving: paths in flight over all requests (default: the workload's; profiling cases)")
    ap.add_argument("--max-requests", type=int, default=0, help="serving: requests admitted at once by the continuous form (default: the workload's)")
    ap.add_argument("--tlas-width", type=int, default=4, choices=[2, 4], help="batched / serving: TLAS node width the traversal reads")
    ap.add_argument("--policy", type=int, default=0, help="serving: new paths by even share (0) or oldest first with backfill (1)")
    ap.add_argument("--slo-sweep", type=int, default=1, help="serving: also sweep arrival rates for throughput at equal p99 (1) or not (0)")
    ap.add_argument("--regroup", type=int, default=1, help="serving: sort each step's continuations by request (1) or not (0)")
    ap.add_argument("--serve-spatial", type=float, default=0.0, help="serving: spatial-split threshold of the host-built BLAS (0: binned SAH)")
    ap.add_argument("--overlap", type=int, default=1, help="serving: a step returns with its launches queued (1) or waits for them (0)")
    ap.add_argument("--sort", type=int, default=0, help="frames: regroup continuation rays before each bounce (0 off, 1 octant, 2 octant + origin cell)")
    ap.add_argument("--companions", type=int, default=1, help="frames at one GPU: also run trace16m and precision1m in child processes and carry their lines (1) or not (0)")
    ap.add_argument("--stage-levels", type=int, default=0, help="frames (CWBVH): top tree levels staged in shared memory per block (0 library default, -1 none, 1..3)")
    args = ap.parse_args()
    wl = dict(WORKLOADS[args.workload])
    if args.batch:
        wl["batch"] = args.batch
    if args.spp and "spp" in wl:
        wl["spp"] = args.spp
    if args.rays and "rays" in wl:
        wl["rays"] = args.rays
    if args.scenes and wl.get("batched"):
        wl["scenes"] = args.scenes
    if args.precision and "rays" in wl:
        wl["precision"] = True
    if not args.bins:
        args.bins = wl.get("bins", 32)
    ws, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, wl, rank)
        return
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    rep = importlib.import_module("cuda-wavefront-pathtracer_b200.replicas").Replicas()   # NCCL between the GPUs when ws > 1
    cwp = importlib.import_module("cuda-wavefront-pathtracer_b200")
    variant = args.variant
    if not wl.get("batched") and not wl.get("serving"):
        mesh, bvh = cwp.scene(wl["scene"], variant=variant, bins=args.bins, spatial=args.spatial)

    def barrier():
        rep.barrier()
        torch.cuda.synchronize()

    def reduce(x, op):
        return rep.max(x) if op == "max" else rep.sum(x)

    props = torch.cuda.get_device_properties(local)
    try:
        dev_id = "GPU-" + str(props.uuid)
    except Exception:
        dev_id = str(local)
    hbm_peak, peak_kind = peaks()
    out = {"metric": "", "value": 0.0, "unit": "Grays/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 0.0,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    if wl.get("serving"):
        bench_serving(args, wl, cwp, torch, out, barrier, reduce)
    elif wl.get("batched"):
        bench_batched(args, wl, cwp, torch, ws, rank, barrier, reduce, dev_id, hbm_peak, peak_kind, out)
    elif "rays" not in wl:
        # ------------------------------------------------------------------ frames
        w, h, spp, K, B = wl["w"], wl["h"], wl["spp"], wl["batch"], wl["bounces"]
        p = cwp.frame_params(mesh, w, h, bounces=B)
        r = cwp.Renderer()
        r.init(p, bvh, variant=variant, tri=1, batch=K, bounces=B, graph=args.graph, device=local, profile=1, traversal=args.traversal, sort=args.sort,
               stage_levels=args.stage_levels)
        for _ in range(args.warmup):
            r.render(spp)
        depths = B + 2
        rays = shadow = 0.0; ms = 0.0
        c_tot = np.zeros(depths); s_tot = np.zeros(depths); tms = np.zeros(depths); sms = np.zeros(depths)
        clk = Clocks(dev_id)
        barrier()
        torch.cuda.nvtx.range_push("timed")
        for _ in range(args.steps):
            st = r.render(spp)
            rays += st.rays; shadow += st.shadow_rays; ms += st.frame_ms
            c, s, tm, sm = r.depth_stats()
            c_tot += c; s_tot += s; tms += tm; sms += sm
        torch.cuda.nvtx.range_pop()
        barrier()
        clocks = clk.stop()
        max_ms = reduce(ms, "max")
        all_rays = reduce(rays + shadow, "sum")
        value = all_rays / (max_ms * 1e-3) / 1e9
        # end to end through the C ABI with host buffers: frame + read of the accumulation buffer into pinned memory
        host = torch.empty((w * h, 4), dtype=torch.float32, pin_memory=True)
        barrier(); t0 = time.perf_counter(); e_rays = 0.0
        for _ in range(args.steps):
            st = r.render(spp)
            cwp._check(cwp.lib().cwp_renderer_read_accum(r._h, host.data_ptr()))
            e_rays += st.rays + st.shadow_rays
        barrier(); e_s = time.perf_counter() - t0
        e_s = reduce(e_s, "max")
        e_rays = reduce(e_rays, "sum")
        # roofline of the dominant kernel (HBM: algorithmic path-state bytes per launch / its event-timed duration)
        tr_bytes = sum(STATE_BYTES * ((c_tot[d] if d > 0 else 0) + (c_tot[d + 1] if d + 1 < depths else 0) + s_tot[d]) for d in range(depths))
        sh_bytes = sum(STATE_BYTES * s_tot[d] for d in range(depths))
        dom = "k_trace_shade" if tms.sum() >= sms.sum() else "k_shadow"
        b, t = (tr_bytes, tms.sum()) if dom == "k_trace_shade" else (sh_bytes, sms.sum())
        achieved = b / (t * 1e-3) / 1e9 if t > 0 else 0.0
        out.update(metric=METRIC_FRAME, value=value, ms_per_step=max_ms / args.steps,
                   config={"workload": args.workload, "scene": f"{wl['scene']} ({mesh.n_tris} triangles, box field seed 1)", "references": len(bvh.order), "resolution": f"{w}x{h}",
                           "spp": spp, "batch": K, "depth": B, "layout": LAYOUT_NAMES[variant], "sah_bins": args.bins, "tri": "woop",
                           "bvh": (f"sbvh (spatial splits at overlap > {args.spatial:g} of the root area, {len(bvh.order) / mesh.n_tris:.2f} references per triangle)" if args.spatial > 0 else "binned SAH"),
                           "graph": args.graph, "traversal": ["auto", "refill", "batch"][args.traversal], "sort": ["off", "octant", "octant+cell"][args.sort],
                           "stage_levels": args.stage_levels,
                           "l2": f"path state {STATE_BYTES * 3 * w * h * K / 1e9:.1f} GB > L2 (126 MB); scene BVH resident",
                           "rays_per_frame": (rays + shadow) / args.steps, "closest_per_frame": rays / args.steps, "shadow_per_frame": shadow / args.steps,
                           "rays_per_sample": (rays + shadow) / args.steps / (w * h * spp), "trace_shade_ms": float(tms.sum() / args.steps),
                           "shadow_ms": float(sms.sum() / args.steps)},
                   clocks=clocks,
                   e2e={"value": e_rays / e_s / 1e9, "unit": "Grays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": w * h * 16,
                        "note": "scene uploaded once at init; each step renders and reads the w*h float4 accumulation buffer back into pinned host memory"},
                   gpu_launches=args.steps * (spp // K) * (2 + 2 * depths),
                   roofline={"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                             "peak_kind": peak_kind, **frame_traffic(args, wl, variant, dom),
                             "algorithmic": f"{STATE_BYTES} B of path state per queued ray read and per continuation/shadow ray written"})
        onchip = dict(kind="frame", closest=float(c_tot.sum()), shadow=float(s_tot.sum()), closest_ms=float(tms.sum()), shadow_ms=float(sms.sum()))
        ours_img = cwp.imageio.accum_to_image(r.read_accum(), w, h, spp)
        r.close()
        if rank == 0 and ws == 1 and args.reference_cuda:
            out["reference_cuda"] = reference_cuda_frame(cwp, wl, mesh, p, max_ms / args.steps, ours_img, local)
        if rank == 0 and ws == 1 and args.companions:
            out["companions"] = companions(args)
    else:
        # ------------------------------------------------------------------ ray batches
        n = wl["rays"]
        acc = cwp.Accel(bvh, tri=1, device=local)
        acc.set_traversal(args.traversal)
        p = cwp.frame_params(mesh, 512, 512)
        st = torch.cuda.current_stream()

        def tr(o, d):
            to, td = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
            hh = torch.empty((len(o), 4), dtype=torch.float32, device="cuda")
            acc.trace_closest(to.data_ptr(), td.data_ptr(), hh.data_ptr(), len(o), st.cuda_stream)
            torch.cuda.synchronize()
            return hh.cpu().numpy()
        o, d = cwp.incoherent_rays(n, p, bvh.tris, tr, seed=41)
        do, dd = torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()
        hits = torch.empty((n, 4), dtype=torch.float32, device="cuda"); occ = torch.empty(n, dtype=torch.int32, device="cuda")
        plain = None
        if wl.get("precision"):
            # the plain form on the same batch (the "vs plain" figure), then switch to the precision form
            for _ in range(2):
                acc.trace_closest(do.data_ptr(), dd.data_ptr(), hits.data_ptr(), n, st.cuda_stream); acc.trace_any(do.data_ptr(), dd.data_ptr(), occ.data_ptr(), n, st.cuda_stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(args.steps):
                acc.trace_closest(do.data_ptr(), dd.data_ptr(), hits.data_ptr(), n, st.cuda_stream); acc.trace_any(do.data_ptr(), dd.data_ptr(), occ.data_ptr(), n, st.cuda_stream)
            e1.record(st); torch.cuda.synchronize()
            plain = 2 * n * args.steps / (e0.elapsed_time(e1) * 1e-3) / 1e9
            acc.set_precision(1)
        for _ in range(args.warmup):
            acc.trace_closest(do.data_ptr(), dd.data_ptr(), hits.data_ptr(), n, st.cuda_stream)
            acc.trace_any(do.data_ptr(), dd.data_ptr(), occ.data_ptr(), n, st.cuda_stream)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps)]
        clk = Clocks(dev_id)
        barrier()
        torch.cuda.nvtx.range_push("timed")
        for i in range(args.steps):
            ev[3 * i].record(st)
            acc.trace_closest(do.data_ptr(), dd.data_ptr(), hits.data_ptr(), n, st.cuda_stream)
            ev[3 * i + 1].record(st)
            acc.trace_any(do.data_ptr(), dd.data_ptr(), occ.data_ptr(), n, st.cuda_stream)
            ev[3 * i + 2].record(st)
        torch.cuda.nvtx.range_pop()
        barrier()
        clocks = clk.stop()
        acc.status()
        c_ms = sum(ev[3 * i].elapsed_time(ev[3 * i + 1]) for i in range(args.steps))
        a_ms = sum(ev[3 * i + 1].elapsed_time(ev[3 * i + 2]) for i in range(args.steps))
        max_ms = reduce(c_ms + a_ms, "max")
        value = 2 * n * args.steps * ws / (max_ms * 1e-3) / 1e9
        # e2e: pinned host rays in, hits / occluders out, every step
        ho = torch.from_numpy(o).pin_memory(); hd = torch.from_numpy(d).pin_memory()
        hh = torch.empty((n, 4), dtype=torch.float32, pin_memory=True); hoc = torch.empty(n, dtype=torch.int32, pin_memory=True)

        def e2e_step():
            cwp._check(cwp.lib().cwp_trace_closest_host(acc._h, ho.data_ptr(), hd.data_ptr(), hh.data_ptr(), n, None))
            cwp._check(cwp.lib().cwp_trace_any_host(acc._h, ho.data_ptr(), hd.data_ptr(), hoc.data_ptr(), n, None))
        for _ in range(args.warmup):   # (the first call also allocates the library's staging buffers)
            e2e_step()
        barrier(); t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        barrier(); e_s = reduce(time.perf_counter() - t0, "max")
        dom_ms, dom_b, dom = (c_ms, 48.0, "k_trace_closest") if c_ms >= a_ms else (a_ms, 36.0, "k_trace_any")
        check = {}
        if wl.get("precision"):
            # FP64 oracle on the same batch: lost hits (must be 0), ties, max relative t error of the closest hits
            acc.trace_closest(do.data_ptr(), dd.data_ptr(), hits.data_ptr(), n, st.cuda_stream)
            t64 = torch.empty(n, dtype=torch.float64, device="cuda"); i64 = torch.empty(n, dtype=torch.int32, device="cuda")
            acc.trace_fp64(do.data_ptr(), dd.data_ptr(), t64.data_ptr(), i64.data_ptr(), n, stream=st.cuda_stream)
            torch.cuda.synchronize()
            h = hits.cpu().numpy(); t64n = t64.cpu().numpy(); i64n = i64.cpu().numpy(); ih = h[:, 3].view(np.int32)
            ext = float(np.ptp(mesh.arrays()[0], axis=0).max())
            pc = importlib.import_module("cuda-wavefront-pathtracer_b200.precision_check")
            c = pc.classify_vs_fp64(h, t64n, i64n, ext, o=o, d=d, verts=bvh.verts)
            ex = c["extra_mask"]
            excess = pc.edge_excess(o[ex], d[ex], bvh.verts, h[ex, 3].view(np.int32)) if ex.any() else np.zeros(1)
            check = {"fp64_rays": n, "lost_hits": c["lost"], "tie_mismatches": c["tie"], "extra_hits": c["extra"],
                     "extra_hits_max_edge_excess": float(excess.max()),
                     "max_t_error": c["max_t_error"], "t_error_unit": "max(t, scene extent)",
                     "plain_grays_s": plain, "vs_plain": value / plain if plain else None}
        achieved = dom_b * n * args.steps / (dom_ms * 1e-3) / 1e9
        onchip = dict(kind="batch", closest=float(n * args.steps), shadow=float(n * args.steps), closest_ms=c_ms, shadow_ms=a_ms)
        out.update(metric=METRIC_BATCH, value=value, ms_per_step=max_ms / args.steps,
                   config={"workload": args.workload, "scene": f"{wl['scene']} ({mesh.n_tris} triangles)", "references": len(bvh.order), "rays": n,
                           "layout": LAYOUT_NAMES[variant] + (" precision form (f16 conservative slabs, watertight fp32 triangles)" if wl.get("precision") else ""), **check,
                           "sah_bins": args.bins, "tri": "woop", "traversal": ["auto", "refill", "batch"][args.traversal],
                           "bvh": (f"sbvh ({len(bvh.order) / mesh.n_tris:.2f} references per triangle)" if args.spatial > 0 else "binned SAH"), "l2": f"ray batch {n * 32 / 1e9:.2f} GB > L2 (126 MB)",
                           "closest_ms": c_ms / args.steps, "any_ms": a_ms / args.steps},
                   clocks=clocks,
                   e2e={"value": 2 * n * args.steps * ws / e_s / 1e9, "unit": "Grays/s", "h2d_bytes_per_step": 2 * 2 * n * 16, "d2h_bytes_per_step": n * 16 + n * 4},
                   gpu_launches=2 * args.steps,
                   roofline={"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                             "peak_kind": peak_kind, "traffic": None,
                             "algorithmic": "closest: 32 B ray in + 16 B hit out; any: 32 B in + 4 B out"})
        acc.close()
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and not wl.get("batched") and not wl.get("serving"):
        # the reference's own host build (its BVHBuilder, 16 bins, timed) and its own traversal code on the host cores
        L = reference_lib()
        rs = (RefScene(L, wl, variant, w=wl.get("w", 512), h=wl.get("h", 512), bounces=wl.get("bounces", 4)) if L is not None and hasattr(L, "ref_frame_params")
              else port_scene(cwp, wl, variant, w=wl.get("w", 512), h=wl.get("h", 512), bounces=wl.get("bounces", 4)))
        if "rays" not in wl:
            out["cpu_baseline"] = cpu_frame_sample(wl, rs, variant)
        else:
            out["cpu_baseline"] = cpu_trace_sample(rs, variant, o, d)
        # on-chip roofline: oracle-counted node + triangle bytes per ray on the GPU's own tree, over the kernels' event
        # times, against the measured L2 read bandwidth (the scene is L2-resident, so this is the traversal's bound)
        if not wl.get("precision"):
            ob = onchip_bytes_frame(cwp, wl, mesh, bvh, variant) if "rays" not in wl else onchip_bytes_trace(cwp, bvh, variant, o, d)
            l2 = cwp.measure_l2_read(device=local)
            cb, sb = onchip["closest"] * ob["closest"], onchip["shadow"] * ob["shadow"]
            kern = ("k_trace_shade", "k_shadow") if onchip["kind"] == "frame" else ("k_trace_closest", "k_trace_any")
            big = 0 if onchip["closest_ms"] >= onchip["shadow_ms"] else 1
            ach = [cb / (onchip["closest_ms"] * 1e-3) / 1e9, sb / (onchip["shadow_ms"] * 1e-3) / 1e9]
            out["roofline_onchip"] = {"bound": "l2", "kernel": kern[big], "achieved": ach[big], "peak": l2, "unit": "GB/s", "frac": ach[big] / l2,
                                      "other_kernel": {"kernel": kern[1 - big], "achieved": ach[1 - big], "frac": ach[1 - big] / l2},
                                      "peak_kind": "measured: cwp_measure_l2_read, 32 MiB read 50 times per launch with 16-byte L2-cached loads",
                                      "bytes_per_closest_ray": ob["closest"], "bytes_per_shadow_ray": ob["shadow"],
                                      "nodes_per_closest_ray": ob["nodes_per_closest"], "tris_per_closest_ray": ob["tris_per_closest"],
                                      "nodes_per_shadow_ray": ob["nodes_per_shadow"], "tris_per_shadow_ray": ob["tris_per_shadow"],
                                      "algorithmic": f"node visits x {NODE_BYTES[variant]} B + triangle tests x {TRI_BYTES} B per ray ({ob['sample']})"}
    rep.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()

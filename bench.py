"""Benchmark of the pik reconstruction path on B200.

Workload (config 2 of the benchmark definition): a 3840x2160 generator image
(12 sinusoids, 20 rectangles, noise sigma 3, seed 0) encoded by the
reference encoder at butteraugli distance 1.0 -- mixed AcStrategy blocks,
adaptive quant field, chroma-from-luma, gaborish and EPF on -- decoded to
the reconstruction boundary by the reference's own decoding functions
(tests/golden/c2_4k_d1_frame.npz, made by tests/golden/make_fixtures.py).
One step = one full reconstruction of that frame (integer coefficients ->
FP32 linear RGB), the reference's Dequant::DoAC + ReconOpsinImage over all
groups + FinalizeFrameDecoding.

  value  decoded MP/s with the inputs resident in device memory, in the
         form chosen by --form (default: split-BF16 tensor-core transforms);
         "forms" gives every form's throughput on the same frame
  e2e    the same through the C ABI with host buffers: each step uploads the
         frame's side information and int16 coefficients from pinned host
         memory and reads the FP32 linear planes back; three contexts take
         the frames in turn with the non-blocking call, so one frame's
         copies overlap the other's kernels (the blocking one-context figure
         is "e2e_blocking"; "e2e_srgb8" reads back the 8-bit sRGB output
         instead).

`--impl reference` times the reference's own CPU implementation (built from
its sources into oracle/_ref/, AVX2 flavour, all host threads) on the same
frame. Multi-GPU: independent replicas (one frame per rank per step).
"""

from __future__ import annotations

import argparse
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

FRAME = os.path.join(ROOT, "tests", "golden", "c2_4k_d1_frame.npz")
BITSTREAM = os.path.join(ROOT, "tests", "golden", "c2_4k_d1.pik")
METRIC = ("decoded MP/s at 4K, split-BF16 vs FP32 form @<=2e-5 err; "
          "% of HBM peak")
# Algorithmic bytes per pixel of the path: int16 AC in (6), DC (0.1875),
# side info (0.094), CfL maps (~0.002), FP32 linear RGB out (12).
PATH_BYTES_PER_PX = 18.28
# Measured with ncu on one reconstruction of the 4K frame in the split-BF16
# form: warp instructions of the frame EPF launch (smsp__inst_executed.sum,
# profiles/k_epf_box_c2_4k.md) and the DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) of all the frame's 17 launches, run one after
# another with the caches kept between them (profiles/traffic_c2_4k.md).
EPF_WARP_INSTR_4K = 175.5e6
PATH_TRAFFIC_4K = 835.2e6
# Algorithmic bytes per pixel of each kernel group (PIKGPU_OPT_PROFILE
# groups), with 4-byte floats.
GROUP_BYTES = {
    # in + out: the guide is recomputed from the staged input tile
    "epf": 3 * 4 + 3 * 4,
    # filtered + original in, clamped out
    "ar_clamp": 3 * 4 + 3 * 4 + 3 * 4,
    # float coefficients in, pixels out
    "hf_idct": 3 * 4 + 3 * 4,
    "gaborish1_minmax": 3 * 4,
    "gaborish2_opsin_srgb": 3 * 4 + 3 * 4,
    # int16 AC in, float AC out
    "dequant_ac": 3 * 2 + 3 * 4,
    # DC read; per cell and channel the corner's 4 floats read and written
    # and 4 pred2x2 floats written
    "lf_prediction_update": 12 / 64 + 3 * 4 * (4 + 4 + 4) / 64,
    "dc_dequant_epf": 0.2,
}
# Arithmetic forms of the reconstruction (PIKGPU_OPT_FORM). The headline is
# the split-BF16 form; every form is timed on the same frame. Their errors
# against the FP64 oracle are checked by tests/test_split_bf16.py.
FORM_NAMES = {
    "fp32": "plain FP32 on CUDA cores (bit-exact to the FP32 oracle)",
    "split_bf16": "16x16 and 32x32 transforms on tcgen05 tensor cores, "
                  "split-BF16 with FP32 accumulate (16-point: hi+lo, 3 "
                  "products; 32-point: hi+mid+lo, 6 products)",
    "split_bf16x3": "16x16 and 32x32 transforms on tcgen05 tensor cores, "
                    "split-BF16 (hi+mid+lo, 6 products, FP32 accumulate)",
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (every 100 ms) during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.path = f"/tmp/pik_b200_clocks_{os.getpid()}.csv"
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "100", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
            os.remove(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None,
                    "reasons": ["no samples"]}

        def num(v):
            try:
                return float(v.split()[0])
            except (ValueError, IndexError):
                return None
        sm = [x for x in (num(r[0]) for r in rows) if x is not None]
        mx = [x for x in (num(r[1]) for r in rows) if x is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(value: float, device) -> float:
    """The maximum of a per-rank time over all ranks of the process group
    (the value itself with one rank or no group). Every rank must call it at
    the same point."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return value
    if dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reference_arm(args):
    """The reference's CPU reconstruction on the same frame."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import refpy
    if not refpy.available("avx2"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference build oracle/_ref is "
                          "missing (build() compiles it from the checkout)"}))
        return
    bs = open(BITSTREAM, "rb").read()
    fz = refpy.Frozen(bs, flavour="avx2")
    threads = os.cpu_count() or 1
    px = fz.xsize * fz.ysize
    for _ in range(args.warmup):
        fz.run_stages(threads=threads, want=())
    times = []
    for _ in range(args.steps):
        _, secs = fz.run_stages(threads=threads, want=())
        times.append(secs)
    t = sum(times)
    value = px * args.steps / t / 1e6
    sample = (f"{args.steps} full 3840x2160 reconstructions (DequantImageAC +"
              f" ReconOpsinImage per group + FinalizeFrameDecoding stages)")
    # The reference's whole decode of the same bitstream (PikToPixels:
    # headers, entropy decoding, reconstruction and the copy out) on the
    # same threads, a few frames; the difference to the reconstruction is
    # what a decoder pays outside this path.
    reps = max(1, min(args.steps, 3))
    refpy.decode(bs, fz.xsize, fz.ysize, threads=threads, flavour="avx2")
    t0 = time.perf_counter()
    for _ in range(reps):
        refpy.decode(bs, fz.xsize, fz.ysize, threads=threads,
                     flavour="avx2")
    full_ms = (time.perf_counter() - t0) * 1e3 / reps
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3),
        "unit": "MP/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "c2: 3840x2160 generator image, reference-"
                   "encoded at distance 1.0 (mixed blocks, EPF on)",
                   "impl": "reference C++ (AVX2 build, ThreadPool)"},
        "cpu_baseline": {"value": round(value, 3), "unit": "MP/s",
                         "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "MP/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_decode": {"value": round(px / (full_ms * 1e-3) / 1e6, 3),
                        "unit": "MP/s", "ms_per_frame": round(full_ms, 3),
                        "outside_reconstruction_ms": round(
                            full_ms - 1e3 * t / args.steps, 3),
                        "sample": f"{reps} PikToPixels decodes of the same "
                                  "bitstream"},
    }))


def cpu_baseline(frame_px):
    """Reference CPU path on a bounded sample: 2 reconstructions of the frame
    with all host threads."""
    try:
        from oracle import refpy
    except Exception as e:  # noqa: BLE001
        return {"value": None, "unit": "MP/s", "cores": 0,
                "kind": "reference", "sample": f"unavailable: {e}"}
    if not refpy.available("avx2"):
        return {"value": None, "unit": "MP/s", "cores": 0,
                "kind": "reference", "sample": "unavailable: no oracle/_ref"}
    bs = open(BITSTREAM, "rb").read()
    fz = refpy.Frozen(bs, flavour="avx2")
    threads = os.cpu_count() or 1
    fz.run_stages(threads=threads, want=())
    t = 0.0
    n = 2
    for _ in range(n):
        _, s = fz.run_stages(threads=threads, want=())
        t += s
    return {"value": round(frame_px * n / t / 1e6, 3), "unit": "MP/s",
            "cores": threads, "kind": "reference",
            "sample": f"{n} full 4K reconstructions, AVX2 build"}


def batch_frames(n=64):
    """The 64-image batch: image sides drawn uniformly from 256..2048 px
    (independently per axis) and distances from 0.5..3.0, seeds 0..63.
    Synthetic frames of those sizes (pik_b200.synthetic: scalars and quant
    field set from the reference encoder's frames at distance 1, the quant
    field scaled with 1 / distance, a broad transform mix) stand in for
    reference-encoded images."""
    from pik_b200 import synthetic
    rng = np.random.default_rng(2024)
    frames = []
    for i in range(n):
        w, h = (int(v) for v in rng.integers(256, 2049, size=2))
        d = float(rng.uniform(0.5, 3.0))
        frames.append(synthetic.make_frame(w, h, seed=i,
                                           qf_median=18.0 / d))
    return frames


def batch_main(args):
    """Total MP/s of 64 frames of uneven sizes: one replay of the batch's
    captured CUDA graph per step, against the same 64 frames reconstructed
    by per-image calls (each a synchronous sequence of 17 or so launches)."""
    import torch
    from pik_b200 import native
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    frames = batch_frames()
    px = sum(f.xsize * f.ysize for f in frames)
    b = native.Batch(len(frames), local, form=args.form)
    for c, f in zip(b.frames, frames):
        c.begin(f)
        c.set_ac()
    outs = [torch.empty((3, f.ysize, f.xsize), device=dev) for f in frames]
    ptrs = [o.data_ptr() for o in outs]
    strides = [f.xsize for f in frames]
    stream = torch.cuda.Stream(device=dev)
    for c in b.frames:
        c.L.pikgpu_set_stream(c.h, stream.cuda_stream)

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    def graph_step():
        b.reconstruct_device(ptrs, strides, stream.cuda_stream)

    def per_image_step():
        for c, o, f in zip(b.frames, outs, frames):
            c.reconstruct_device(o.data_ptr(), f.xsize)

    ms_untuned = timed(graph_step)
    shape = b.autotune(ptrs, strides, stream.cuda_stream)
    with ClockSampler(local) as clk:
        ms_graph = timed(graph_step)
    ms_single = timed(per_image_step)
    print(json.dumps({
        "metric": "total decoded MP/s, 64 images of uneven sizes: one CUDA "
                  "graph (one branch per image) vs per-image launches",
        "value": round(px / (ms_graph * 1e-3) / 1e6, 2), "unit": "MP/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_graph, 4), "higher_is_better": True,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch64: 64 synthetic frames, sides "
                   "U[256,2048] per axis, distance U[0.5,3.0]",
                   "total_megapixels": round(px / 1e6, 2),
                   "form": FORM_NAMES[args.form]},
        "per_image": {"value": round(px / (ms_single * 1e-3) / 1e6, 2),
                      "ms_per_step": round(ms_single, 4)},
        "speedup_vs_per_image": round(ms_single / ms_graph, 3),
        "untuned_graph": {"value": round(px / (ms_untuned * 1e-3) / 1e6, 2),
                          "ms_per_step": round(ms_untuned, 4),
                          "chains": len(frames), "tc_ctas_per_sm": 4},
        "autotuned": shape,
        "gpu_launches": b.launch_count() * args.steps,
        "graph_captures": b.capture_count(),
        "clocks": clk.summary(),
    }))
    b.close()


# Contexts that take the frames of the streaming end-to-end run in turn:
# with three, the read-back of one frame (the bound: 100 MB at ~57 GB/s)
# overlaps the upload and kernels of the next two.
STREAM_CONTEXTS = 3

def adjoint_main(args):
    """Gradient evaluations of sum((pre_opsin - target)^2) with respect to
    the dequantised AC and the quant field (pikgpu_adjoint: forward pass
    with the clamp tape, then the backward kernels) on a 1024x1024 frame
    encoded by the reference encoder at distance 1.5
    (tests/golden/c4_1k_d15_frame.npz; EPF on, the encoder's transform mix).
    The target is the XYB of the frame's source image (the generator image
    synthetic.ADJOINT_SOURCE through pik_b200.xyb.linear_to_xyb, the
    encoder's own opsin transform), i.e. the loss an encoder minimises."""
    import ctypes
    import torch
    from pik_b200 import layout, native, synthetic, xyb
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    frame = layout.Frame.load(os.path.join(ROOT, "tests", "golden",
                                           "c4_1k_d15_frame.npz"))
    px = frame.xsize * frame.ysize
    by, bx = frame.blocks
    src = dict(synthetic.ADJOINT_SOURCE)
    img = synthetic.make_image(src.pop("xsize"), src.pop("ysize"), **src)
    target = xyb.linear_to_xyb(synthetic.srgb8_to_linear255(img))
    stream = torch.cuda.Stream(device=dev)
    ctx = native.Context(local, form=args.form)
    ctx.begin(frame)
    ctx.set_ac()
    ctx.L.pikgpu_set_stream(ctx.h, stream.cuda_stream)
    t_dev = torch.from_numpy(target).to(dev)
    g_ac = torch.empty((3, by, bx * 64), dtype=torch.float32, device=dev)
    g_qf = torch.empty((by, bx), dtype=torch.float32, device=dev)
    loss = torch.empty(1, dtype=torch.float64, device=dev)
    lin = torch.empty((3, frame.ysize, frame.xsize), device=dev)

    def adj_step():
        ctx._check(ctx.L.pikgpu_adjoint(ctx.h, t_dev.data_ptr(),
                                        loss.data_ptr(), g_ac.data_ptr(),
                                        g_qf.data_ptr(), 1))

    def fwd_step():
        ctx.reconstruct_device(lin.data_ptr(), frame.xsize)

    def timed(fn, clk=None):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if clk:
            clk.__enter__()
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        return e0.elapsed_time(e1) / args.steps

    clk = ClockSampler(local)
    ms_adj = timed(adj_step, clk)
    launches = ctx.L.pikgpu_last_launch_count(ctx.h)
    ms_fwd = timed(fwd_step)
    # End to end with host buffers: target up, gradients and loss down.
    pin_t = torch.from_numpy(target).pin_memory()
    pin_ac = torch.empty(g_ac.shape, dtype=torch.float32).pin_memory()
    pin_qf = torch.empty(g_qf.shape, dtype=torch.float32).pin_memory()
    pin_l = torch.empty(1, dtype=torch.float64).pin_memory()

    def e2e_step():
        ctx._check(ctx.L.pikgpu_adjoint(ctx.h, pin_t.data_ptr(),
                                        pin_l.data_ptr(), pin_ac.data_ptr(),
                                        pin_qf.data_ptr(), 0))

    for _ in range(max(3, args.warmup)):
        e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    ctx.close()
    # FP64 oracle adjoint on the host (one thread), a bounded sample: one
    # gradient evaluation of the same frame.
    cpu = None
    try:
        from oracle import decisions as odec, oraclepy
        dg, ds = odec.dc_decisions(frame)
        t0 = time.perf_counter()
        oraclepy.adjoint(frame, target.astype(np.float64), dc_guide=dg,
                         dc_sigma=ds)
        cpu_s = time.perf_counter() - t0
        cpu = {"value": round(px / cpu_s / 1e6, 4), "unit": "MP/s",
               "cores": 1, "kind": "port",
               "sample": "one FP64 oracle gradient evaluation of the same "
                         "1024x1024 frame"}
    except Exception as e:  # oracle library not built on this host
        cpu = {"unavailable": str(e)[:200]}
    if rank == 0:
        print(json.dumps({
            "metric": "adjoint gradient evaluations of a 1024x1024 frame "
                      "(forward + backward), MP/s",
            "value": round(px / (ms_adj * 1e-3) / 1e6, 2), "unit": "MP/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_adj, 4), "higher_is_better": True,
            "dtype": "f32",
            "data": "generator image (seeded, synthetic) encoded by the "
                    "reference encoder; target = the source's XYB",
            "config": {"workload": "adjoint1k: 1024x1024 generator image "
                       "reference-encoded at distance 1.5 (63% DCT16X16, "
                       "30% DCT32X32, 6% DCT8; gaborish + EPF on), loss "
                       "sum((pre_opsin - XYB(source))^2)",
                       "form": FORM_NAMES[args.form]},
            "forward_only": {"value": round(px / (ms_fwd * 1e-3) / 1e6, 2),
                             "ms_per_step": round(ms_fwd, 4)},
            "backward_over_forward": round((ms_adj - ms_fwd) / ms_fwd, 3),
            "e2e": {"value": round(px / (e2e_ms * 1e-3) / 1e6, 2),
                    "unit": "MP/s",
                    "h2d_bytes_per_step": int(target.nbytes),
                    "d2h_bytes_per_step": int(pin_ac.numel() * 4 +
                                              pin_qf.numel() * 4 + 8)},
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }))


C5_MIXES = {
    "broad": "every transform type (36% DCT8, 22% DCT16X16, 18% DCT32X32, "
             "the rest small types)",
    "encoder": "the reference encoder's mix at distance 0.5 (72% DCT16X16, "
               "22% DCT32X32, 5% DCT8)",
}


def c5_frame(xsize=8192, ysize=8192, seed=5, mix="broad"):
    """The memory-bound roofline case: an 8192x8192 frame at distance 0.5
    with gaborish and EPF on, and 1% of the area in highlights at 4x linear
    light (pik_b200.synthetic.make_highlight_frame). `mix` "broad" gives
    every block type a real share; "encoder" takes the shares the reference
    encoder picks at distance 0.5. A synthetic frame stands in for the
    reference encoder's output: encoding 67 MP with butteraugli iterations
    takes hours on the host."""
    from pik_b200 import synthetic
    shares = synthetic.ENCODER_SHARES_D05 if mix == "encoder" else None
    return synthetic.make_highlight_frame(xsize, ysize, seed=seed,
                                          shares=shares)


def c5_summary(local, steps, warmup, mix="encoder"):
    """Device time per frame of the 8192x8192 workload (`mix`) in the plain
    FP32 and split-BF16 forms, inputs resident and outputs into device
    planes, with the achieved HBM GB/s of 18.28 algorithmic B/px. Reported
    in the default line beside the 4K figures."""
    import ctypes
    import torch
    from pik_b200 import native
    dev = torch.device("cuda", local)
    frame = c5_frame(mix=mix)
    px = frame.xsize * frame.ysize
    by, bx = frame.blocks
    ac_dev = torch.from_numpy(frame.quantized_ac).to(dev)
    planes = (ctypes.c_void_p * 3)(*[ac_dev[c].data_ptr() for c in range(3)])
    lin = torch.empty((3, frame.ysize, frame.xsize), dtype=torch.float32,
                      device=dev)
    stream = torch.cuda.Stream(device=dev)
    out = {"workload": "c5_8k: 8192x8192 synthetic highlight frame, "
                       "distance 0.5, gaborish + EPF on, FP32 planes out",
           "mix": C5_MIXES[mix]}
    for form in ("fp32", "split_bf16"):
        ctx = native.Context(local, form=form)
        ctx.begin(frame)
        ctx.L.pikgpu_set_stream(ctx.h, stream.cuda_stream)

        def step():
            ctx._check(ctx.L.pikgpu_frame_set_ac_device(ctx.h, planes,
                                                        bx * 64))
            ctx.reconstruct_device(lin.data_ptr(), frame.xsize)

        for _ in range(max(3, warmup)):
            step()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        ctx.close()
        out[form] = {"ms_per_frame": round(ms, 4),
                     "megapixels_per_s": round(px / (ms * 1e-3) / 1e6, 1),
                     "hbm_gbs": round(PATH_BYTES_PER_PX * px / (ms * 1e-3)
                                      / 1e9, 1)}
    out["split_over_fp32"] = round(out["fp32"]["ms_per_frame"] /
                                   out["split_bf16"]["ms_per_frame"], 3)
    return out


def c5_main(args):
    """Achieved HBM GB/s of the 8192x8192 reconstruction (FP32 linear planes
    out, 805 MB) in the split-BF16 and plain FP32 forms: 18.28 algorithmic
    bytes per pixel x pixels / device time per frame, inputs resident."""
    import torch
    import torch.distributed as dist
    from pik_b200 import native
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    frame = c5_frame(mix=args.mix)
    px = frame.xsize * frame.ysize
    by, bx = frame.blocks
    import ctypes
    ac_dev = torch.from_numpy(frame.quantized_ac).to(dev)
    planes = (ctypes.c_void_p * 3)(*[ac_dev[c].data_ptr() for c in range(3)])
    stream = torch.cuda.Stream(device=dev)
    outs = {}

    def time_form(form, sample_clocks=False):
        ctx = native.Context(local, form=form)
        ctx.begin(frame)
        ctx.L.pikgpu_set_stream(ctx.h, stream.cuda_stream)
        lin = torch.empty((3, frame.ysize, frame.xsize), dtype=torch.float32,
                          device=dev)

        def step():
            ctx._check(ctx.L.pikgpu_frame_set_ac_device(ctx.h, planes,
                                                        bx * 64))
            ctx.reconstruct_device(lin.data_ptr(), frame.xsize)

        for _ in range(max(3, args.warmup)):
            step()
        n_launch = ctx.L.pikgpu_last_launch_count(ctx.h)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.__enter__()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        t = e0.elapsed_time(e1) / args.steps
        t = max_over_ranks(t, dev)
        ctx.close()
        outs[form] = lin
        return t, n_launch, clk

    ms, launches, clk = time_form(args.form, sample_clocks=True)
    forms = {args.form: ms}
    for form in ("fp32", "split_bf16"):
        if form not in forms:
            forms[form] = time_form(form)[0]
    # The forms against each other on the [0, 1] scale (value / 255).
    diff = None
    if "fp32" in outs and args.form != "fp32":
        d = (outs[args.form] - outs["fp32"]).abs_() / 255.0
        diff = {"max_abs": float(d.max().item()),
                "frac_above_2e-5": float((d > 2e-5).float().mean().item())}
        del d
    outs.clear()

    # Per-kernel-group device times of the headline form.
    pctx = native.Context(local, profile=True, form=args.form)
    pctx.begin(frame)
    pctx.L.pikgpu_set_stream(pctx.h, stream.cuda_stream)
    pctx._check(pctx.L.pikgpu_frame_set_ac_device(pctx.h, planes, bx * 64))
    lin = torch.empty((3, frame.ysize, frame.xsize), dtype=torch.float32,
                      device=dev)
    acc = {}
    for i in range(3 + args.steps):
        pctx.reconstruct_device(lin.data_ptr(), frame.xsize)
        if i >= 3:
            for k, v in pctx.kernel_times().items():
                acc[k] = acc.get(k, 0.0) + v / args.steps
    pctx.close()
    del lin

    # End to end through the C ABI: one context, blocking calls, int16 AC
    # and side information up from pinned host memory, FP32 planes back.
    from pik_b200 import abi
    ctx = native.Context(local, form=args.form)
    ctx.L.pikgpu_set_stream(ctx.h, stream.cuda_stream)
    pin_ac = torch.from_numpy(frame.quantized_ac).pin_memory()
    pin_lin = torch.empty((3, frame.ysize, frame.xsize),
                          dtype=torch.float32).pin_memory()
    ac_planes = (ctypes.c_void_p * 3)(*[pin_ac[c].data_ptr()
                                        for c in range(3)])
    lin_planes = (ctypes.c_void_p * 3)(*[pin_lin[c].data_ptr()
                                         for c in range(3)])
    packed = abi.PackedFrame(frame)
    h2d = frame.quantized_ac.nbytes + sum(a.nbytes for a in
                                          packed.arrays.values())
    d2h = pin_lin.numel() * 4

    def e2e_step():
        ctx._check(ctx.L.pikgpu_frame_begin(ctx.h, packed.ref))
        ctx._check(ctx.L.pikgpu_frame_set_ac(ctx.h, ac_planes, bx * 64))
        ctx._check(ctx.L.pikgpu_reconstruct(ctx.h, lin_planes, frame.xsize,
                                            None, 0, 0))

    for _ in range(max(3, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    e2e_ms = max_over_ranks(e2e_ms, dev)
    ctx.close()

    # CPU: the FP32 oracle restatement (one host thread) on a bounded
    # sample, a 4096x4096 frame from the same generator settings.
    cpu = None
    if rank == 0:
        try:
            from oracle import oraclepy
            sample = c5_frame(4096, 4096, mix=args.mix)
            t0 = time.perf_counter()
            oraclepy.run(sample, want=("linear",))
            cpu_s = time.perf_counter() - t0
            cpu = {"value": round(sample.xsize * sample.ysize / cpu_s / 1e6,
                                  3),
                   "unit": "MP/s", "cores": 1, "kind": "port",
                   "sample": "one FP32 oracle reconstruction of a 4096x4096 "
                             "frame with the same generator settings"}
        except Exception as e:  # oracle library not built on this host
            cpu = {"unavailable": str(e)[:200]}

    peak, peak_kind = load_peaks()
    gbs = {f: PATH_BYTES_PER_PX * px / (t * 1e-3) / 1e9
           for f, t in forms.items()}
    top = max(acc, key=acc.get)
    achieved = GROUP_BYTES.get(top, 12) * px / (acc[top] * 1e-3) / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": "achieved HBM GB/s of the 8192x8192 reconstruction "
                      "(18.28 algorithmic B/px x px / frame time)",
            "value": round(ws * gbs[args.form], 1), "unit": "GB/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "c5_8k: 8192x8192 synthetic frame, "
                       "distance 0.5, 1% highlights at 4x, gaborish + EPF "
                       "on, FP32 linear planes out (805 MB)",
                       "mix": C5_MIXES[args.mix],
                       "form": FORM_NAMES[args.form],
                       "l2": "working set > L2 (inputs 403 MB, planes "
                             "805 MB each)",
                       "parallelism": f"replicas x{ws}"},
            "megapixels_per_s": round(ws * px / (ms * 1e-3) / 1e6, 1),
            "roofline": {"bound": "hbm", "kernel": top,
                         "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": None, "peak_kind": peak_kind,
                         "path_achieved": round(gbs[args.form], 1),
                         "path_frac": round(gbs[args.form] / peak, 4)},
            "forms": {f: {"GB/s": round(gbs[f], 1),
                          "MP/s": round(px / (t * 1e-3) / 1e6, 1),
                          "ms_per_step": round(t, 4)}
                      for f, t in forms.items()},
            "speedup_vs_fp32": round(forms["fp32"] / ms, 3),
            "form_vs_fp32": diff,
            "kernel_ms": {k: round(v, 4) for k, v in acc.items()},
            "e2e": {"value": round(ws * PATH_BYTES_PER_PX * px /
                                   (e2e_ms * 1e-3) / 1e9, 1),
                    "unit": "GB/s",
                    "megapixels_per_s": round(ws * px / (e2e_ms * 1e-3)
                                              / 1e6, 1),
                    "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "mode": "one context, blocking pikgpu_reconstruct"},
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours")
    ap.add_argument("--form", default="split_bf16",
                    choices=sorted(FORM_NAMES))
    ap.add_argument("--workload", default="c2_4k",
                    choices=["c2_4k", "batch64", "adjoint1k", "c5_8k"])
    ap.add_argument("--mix", default="broad", choices=sorted(C5_MIXES),
                    help="transform mix of the c5_8k frame")
    ap.add_argument("--no-c5", action="store_true",
                    help="leave the 8192x8192 summary out of the 4K line")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch64":
        return batch_main(args)
    if args.workload == "adjoint1k":
        return adjoint_main(args)
    if args.workload == "c5_8k":
        return c5_main(args)

    import torch
    import torch.distributed as dist
    from pik_b200 import layout, native

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    frame = layout.Frame.load(FRAME)
    px = frame.xsize * frame.ysize
    by, bx = frame.blocks
    dev = torch.device("cuda", local)

    # Device-resident runs: AC already in HBM, outputs into device buffers.
    ac_dev = torch.from_numpy(frame.quantized_ac).to(dev)
    lin_dev = torch.empty((3, frame.ysize, frame.xsize), dtype=torch.float32,
                          device=dev)
    stream = torch.cuda.Stream(device=dev)
    import ctypes
    planes = (ctypes.c_void_p * 3)(*[ac_dev[c].data_ptr() for c in range(3)])

    def time_device(form, sample_clocks=False, graphs=True):
        ctx = native.Context(local, form=form, graphs=graphs)
        ctx.begin(frame)
        ctx.L.pikgpu_set_stream(ctx.h, stream.cuda_stream)

        def step():
            ctx._check(ctx.L.pikgpu_frame_set_ac_device(ctx.h, planes,
                                                        bx * 64))
            ctx.reconstruct_device(lin_dev.data_ptr(), frame.xsize)

        for _ in range(max(3, args.warmup)):
            step()
        n_launch = ctx.L.pikgpu_last_launch_count(ctx.h)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.__enter__()
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__()
        t = start.elapsed_time(end) / args.steps
        t = max_over_ranks(t, dev)
        ctx.close()
        return t, n_launch, clk

    ms, launches, clk = time_device(args.form, sample_clocks=True)
    value = ws * px / (ms * 1e-3) / 1e6
    # The same without graph replay: every step launches its 17 kernels.
    ms_direct = time_device(args.form, graphs=False)[0]
    # The other forms on the same frame, for the form comparison.
    forms = {args.form: ms}
    for form in native.FORMS:
        if form not in forms:
            forms[form] = time_device(form)[0]

    # Per-kernel-group device times (CUDA events on the launching stream).
    pctx = native.Context(local, profile=True, form=args.form)
    pctx.begin(frame)
    pctx.L.pikgpu_set_stream(pctx.h, stream.cuda_stream)
    pctx._check(pctx.L.pikgpu_frame_set_ac_device(pctx.h, planes, bx * 64))
    acc = {}
    for i in range(3 + args.steps):
        pctx.reconstruct_device(lin_dev.data_ptr(), frame.xsize)
        if i >= 3:
            for k, v in pctx.kernel_times().items():
                acc[k] = acc.get(k, 0.0) + v / args.steps
    pctx.close()

    # End to end through the C ABI with pinned host buffers.
    ctx = native.Context(local, form=args.form)
    ctx.L.pikgpu_set_stream(ctx.h, stream.cuda_stream)
    pin = {
        "ac": torch.from_numpy(frame.quantized_ac).pin_memory(),
        "lin": torch.empty((3, frame.ysize, frame.xsize),
                           dtype=torch.float32).pin_memory(),
    }
    ac_planes = (ctypes.c_void_p * 3)(
        *[pin["ac"][c].data_ptr() for c in range(3)])
    lin_planes = (ctypes.c_void_p * 3)(
        *[pin["lin"][c].data_ptr() for c in range(3)])
    from pik_b200 import abi
    packed = abi.PackedFrame(frame)
    h2d = frame.quantized_ac.nbytes + sum(a.nbytes for a in
                                          packed.arrays.values())
    d2h = pin["lin"].numel() * 4

    def e2e_step():
        ctx._check(ctx.L.pikgpu_frame_begin(ctx.h, packed.ref))
        ctx._check(ctx.L.pikgpu_frame_set_ac(ctx.h, ac_planes, bx * 64))
        ctx._check(ctx.L.pikgpu_reconstruct(ctx.h, lin_planes, frame.xsize,
                                            None, 0, 0))

    for _ in range(max(3, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    # Host wall clock: the region includes host-side validation and uploads.
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    e2e_ms = max_over_ranks(e2e_ms, dev)
    e2e_blocking = ws * px / (e2e_ms * 1e-3) / 1e6
    ctx.close()

    # Streaming end to end: three contexts in turn with the non-blocking call,
    # so one frame's uploads, kernels and read-back overlap the other's.
    # Every step still uploads its side information and int16 AC from
    # pinned host memory and reads its linear planes back into pinned host
    # memory; the region ends when the last frame is read back.
    ctxs = [native.Context(local, form=args.form)
            for _ in range(STREAM_CONTEXTS)]
    pin_lins = [pin["lin"]] + [torch.empty_like(pin["lin"]).pin_memory()
                               for _ in range(STREAM_CONTEXTS - 1)]
    lin_ptrs = [[p[c].data_ptr() for c in range(3)] for p in pin_lins]

    def stream_step(i):
        c = ctxs[i % STREAM_CONTEXTS]
        c.wait()
        c._check(c.L.pikgpu_frame_begin(c.h, packed.ref))
        c._check(c.L.pikgpu_frame_set_ac(c.h, ac_planes, bx * 64))
        c.reconstruct_async(lin_ptrs[i % STREAM_CONTEXTS], frame.xsize)

    for i in range(max(3, args.warmup)):
        stream_step(i)
    for c in ctxs:
        c.wait()
    if ws > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        stream_step(i)
    for c in ctxs:
        c.wait()
    stream_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    stream_ms = max_over_ranks(stream_ms, dev)
    e2e = ws * px / (stream_ms * 1e-3) / 1e6

    # The same streaming run with the 8-bit sRGB output only (interleaved
    # RGB bytes, ExternalImage::CopyTo's rounding: what dpik writes to an
    # 8-bit PPM) read back instead of the linear float planes.
    pin_rgbs = [torch.empty((frame.ysize, frame.xsize, 3),
                            dtype=torch.uint8).pin_memory()
                for _ in range(STREAM_CONTEXTS)]

    def stream_step8(i):
        c = ctxs[i % STREAM_CONTEXTS]
        c.wait()
        c._check(c.L.pikgpu_frame_begin(c.h, packed.ref))
        c._check(c.L.pikgpu_frame_set_ac(c.h, ac_planes, bx * 64))
        c.reconstruct_async(None, 0, pin_rgbs[i % STREAM_CONTEXTS].data_ptr(),
                            3 * frame.xsize)

    for i in range(max(3, args.warmup)):
        stream_step8(i)
    for c in ctxs:
        c.wait()
    if ws > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(args.steps):
        stream_step8(i)
    for c in ctxs:
        c.wait()
    stream8_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    stream8_ms = max_over_ranks(stream8_ms, dev)
    e2e8 = ws * px / (stream8_ms * 1e-3) / 1e6
    for c in ctxs:
        c.close()

    peak, peak_kind = load_peaks()
    top = max(acc, key=acc.get)
    # DRAM bytes per launch of the 4K workload measured with ncu
    # (dram__bytes_read.sum + dram__bytes_write.sum, one cold launch each).
    ncu_traffic_4k = {
        "epf": 100.38e6 + 63.28e6,
        "gaborish1_minmax": 99.54e6 + 64.64e6,
        "gaborish2_opsin_srgb": 99.55e6 + 63.85e6,
    }
    traffic = ncu_traffic_4k.get(top) if px == 3840 * 2160 else None
    top_bytes = GROUP_BYTES.get(top, 12) * px
    achieved = top_bytes / (acc[top] * 1e-3) / 1e9
    # The EPF is bound by instruction issue, not HBM: its warp instructions
    # per launch (ncu smsp__inst_executed.sum, one launch of the 4K frame)
    # against the issue rate of 4 schedulers per SM at the sampled clock.
    clocks = clk.summary()
    issue = None
    if top == "epf" and px == 3840 * 2160 and clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        rate = sms * 4 * clocks["sm_mhz"] * 1e6  # warp instructions / s
        floor_ms = EPF_WARP_INSTR_4K / rate * 1e3
        issue = {"warp_instructions": EPF_WARP_INSTR_4K,
                 "per_pixel": round(EPF_WARP_INSTR_4K / px, 2),
                 "sm_mhz": clocks["sm_mhz"], "sms": sms,
                 "floor_ms": round(floor_ms, 4),
                 "frac": round(floor_ms / acc[top], 4)}
    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 2), "unit": "MP/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": "c2: 3840x2160 generator image, reference-encoded"
                            " at distance 1.0 (mixed blocks, adaptive qf, CfL,"
                            " gaborish + EPF on)",
                "form": FORM_NAMES[args.form],
                "l2": "working set > L2 (inputs 50 MB, planes 100 MB each)",
                "parallelism": f"replicas x{ws}"},
            "roofline": {"bound": "hbm", "kernel": top,
                         "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind,
                         "path_achieved": round(
                             PATH_BYTES_PER_PX * px / (ms * 1e-3) / 1e9, 1),
                         "path_frac": round(PATH_BYTES_PER_PX * px /
                                            (ms * 1e-3) / 1e9 / peak, 4),
                         "path_traffic": (PATH_TRAFFIC_4K
                                          if px == 3840 * 2160 else None),
                         "path_algorithmic_bytes": round(
                             PATH_BYTES_PER_PX * px),
                         "issue": issue},
            "kernel_ms": {k: round(v, 4) for k, v in acc.items()},
            "forms": {f: {"value": round(ws * px / (t * 1e-3) / 1e6, 2),
                          "ms_per_step": round(t, 4)}
                      for f, t in forms.items()},
            "speedup_vs_fp32": round(forms["fp32"] / ms, 3),
            "launch_mode": "CUDA graph replay of the frame's launch "
                           "sequence (PIKGPU_OPT_GRAPHS), one graph launch "
                           "per step",
            "direct_launches": {
                "value": round(ws * px / (ms_direct * 1e-3) / 1e6, 2),
                "ms_per_step": round(ms_direct, 4)},
            "e2e": {"value": round(e2e, 2), "unit": "MP/s",
                    "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "mode": f"{STREAM_CONTEXTS} contexts in turn, "
                            "pikgpu_reconstruct_async + pikgpu_wait (copies "
                            "of one frame overlap another's kernels)"},
            "e2e_blocking": {"value": round(e2e_blocking, 2), "unit": "MP/s",
                             "mode": "one context, blocking "
                                     "pikgpu_reconstruct per frame"},
            "e2e_srgb8": {"value": round(e2e8, 2), "unit": "MP/s",
                          "h2d_bytes_per_step": int(h2d),
                          "d2h_bytes_per_step": int(3 * px),
                          "mode": "as e2e, with the 8-bit sRGB output (what "
                                  "dpik writes to an 8-bit PPM) read back "
                                  "instead of the linear planes"},
            "gpu_launches": launches * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu_baseline(px) if ws == 1 else None,
        }
        if ws == 1 and not args.no_c5:
            out["c5_8k"] = c5_summary(local, min(args.steps, 10),
                                      args.warmup)
        print(json.dumps(out))
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

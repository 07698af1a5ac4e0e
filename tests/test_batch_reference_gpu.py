"""The batched form on reference-encoded frames: eight generator images
with the batch workload's distribution (seeds 0..7, distances drawn from
U[0.5, 3.0]; sides drawn from U[256, 512] per axis, smaller than the
workload's 256..2048 so that the reference encoder, run here at test time,
takes seconds), encoded by the reference encoder compiled from its sources
and decoded to the reconstruction boundary by its own decoding functions.
In the FP32 form every frame of the batch must equal the FP32 oracle bit
for bit. In the split-BF16 form every frame must equal its single-frame
result bit for bit, and, given the FP32 form's discrete decisions (EPF
guide and sigma, clamp branches), be within max-abs 2e-5 of the FP64
oracle on the [0, 1] scale."""

import numpy as np
import pytest

from oracle import decisions, oraclepy, refpy
from pik_b200 import native, synthetic

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not refpy.available("scalar"),
                       reason="reference build (oracle/_ref) not present"),
]


def reference_frames(n=8):
    rng = np.random.default_rng(2024)
    frames = []
    for i in range(n):
        w, h = (int(v) for v in rng.integers(256, 513, size=2))
        d = float(rng.uniform(0.5, 3.0))
        img = synthetic.make_image(w, h, seed=i, sinusoids=12, rectangles=20,
                                   noise_sigma=3)
        bs = refpy.encode(synthetic.srgb8_to_linear255(img), d, threads=8)
        frames.append(refpy.Frozen(bs, flavour="scalar").frame())
    return frames


def batch_run(frames, form, dec=None):
    import torch
    b = native.Batch(len(frames), form=form)
    try:
        for i, (c, f) in enumerate(zip(b.frames, frames)):
            c.begin(f)
            c.set_ac()
            if dec is not None and f.have_ar:
                c.set_decisions(dec[i][0], dec[i][1])
                c.set_clamp_decisions(dec[i][2])
        outs = [torch.empty((3, f.ysize, f.xsize), device="cuda")
                for f in frames]
        b.reconstruct_device([o.data_ptr() for o in outs],
                             [f.xsize for f in frames])
        return [o.cpu().numpy() for o in outs]
    finally:
        b.close()


def single(frame, form):
    ctx = native.Context(0, form=form)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        return ctx.reconstruct(linear=True)[0]
    finally:
        ctx.close()


def fp32_decisions(frame):
    ctx = native.Context(0, keep_stages=True)
    try:
        ctx.begin(frame)
        ctx.set_ac()
        ctx.reconstruct(linear=True)
        if not frame.have_ar:
            return None, None, None
        g, s = ctx.decisions()
        return g, s, ctx.clamp_decisions()
    finally:
        ctx.close()


def test_reference_encoded_batch():
    frames = reference_frames()
    fp32 = batch_run(frames, "fp32")
    for f, got in zip(frames, fp32):
        want = oraclepy.run(f, precision=32, want=("linear",))["linear"]
        np.testing.assert_array_equal(got, want)
    split = batch_run(frames, "split_bf16")
    for f, got in zip(frames, split):
        np.testing.assert_array_equal(got, single(f, "split_bf16"))
    dec = [fp32_decisions(f) for f in frames]
    shared = batch_run(frames, "split_bf16", dec)
    for f, got, (g, s, tape) in zip(frames, shared, dec):
        dg, ds = decisions.dc_decisions(f)
        o64 = oraclepy.run(f, precision=64, want=("linear",), guide=g,
                           sigma=s, dc_guide=dg, dc_sigma=ds,
                           clamp_tape=tape)["linear"]
        err = float(np.abs(got - o64).max()) / 255
        print(f"{f.xsize}x{f.ysize}: split-BF16 vs FP64 {err:.3g}")
        assert err <= 2e-5

"""The CUDA adjoint (pikgpu_adjoint) against the FP64 reference gradient of
the oracle (oracle/pik_adjoint.inc, itself checked against finite
differences in test_adjoint_oracle.py) and against central finite
differences (oracle/finite_diff.py: step 1e-3 of a coefficient's
quantisation step, a relative 1e-3 on the quant field).

Both sides hold every discrete decision at the CUDA forward's values: the
EPF's guide and sigma and the clamp's branch per coefficient (the clamp
tape). The oracle gets them as inputs and the finite differences set them
as overrides. Without the tape the FP32 and FP64 forwards can take
different clamp branches on identical inputs: a correction that cancels to
exactly +0.0 in one precision (ratio 0, the coefficient dropped in all
channels) is a residue of ~1e-17 in the other (ratio 1, kept), which leaves
the outputs equal but changes the gradient of the block
(test_own_branches_differ_only_by_branch_flips). Tolerances: relative L2
error 1e-3, every entry within 1e-3 of the largest gradient."""

import numpy as np
import pytest

from oracle import decisions, finite_diff, oraclepy
from pik_b200 import native, synthetic

pytestmark = pytest.mark.gpu

SHARES = {"DCT": 0.3, "DCT16X16": 0.3, "DCT32X32": 0.2, "DCT4X4": 0.05,
          "DCT2X2": 0.05, "IDENTITY": 0.04, "LINES": 0.03, "DCT_NOHF": 0.02,
          "DCT4X4_NOHF": 0.01}

REL_L2 = 1e-3      # ||g - g_ref|| / ||g_ref||
ELEM_REL = 1e-3    # |g - g_ref| <= ELEM_REL * max|g_ref| for every entry


def forward(frame, form="fp32"):
    """A context after one forward pass; dec = (guide, sigma, clamp tape)."""
    ctx = native.Context(0, keep_stages=True, form=form)
    ctx.begin(frame)
    ctx.set_ac()
    ctx.reconstruct(linear=True)
    if frame.have_ar:
        dec = ctx.decisions() + (ctx.clamp_decisions(),)
    else:
        dec = (None, None, None)
    return ctx, dec, ctx.stage("pre_opsin")


def make_target(pre, seed):
    rng = np.random.default_rng(seed)
    return (pre + rng.normal(0, 0.01, pre.shape)).astype(np.float32)


def reference(frame, target, dec, tape=True):
    dg, ds = decisions.dc_decisions(frame)
    kw = dict(dc_guide=dg, dc_sigma=ds)
    if frame.have_ar:
        kw.update(guide=dec[0], sigma=dec[1],
                  clamp_tape=dec[2] if tape else None)
    return oraclepy.adjoint(frame, target.astype(np.float64), **kw)


def compare(name, g, ref):
    g = g.astype(np.float64)
    d = np.abs(g - ref)
    scale = np.abs(ref).max()
    rel = np.linalg.norm(g - ref) / max(np.linalg.norm(ref), 1e-30)
    print(f"{name}: rel_l2 {rel:.3g} max_abs {d.max():.3g} "
          f"(scale {scale:.3g})")
    assert rel <= REL_L2, (name, rel)
    assert d.max() <= ELEM_REL * scale, (name, d.max(), scale)


def check_against_reference(frame, seed=0, form="fp32"):
    ctx, dec, pre = forward(frame, form)
    try:
        target = make_target(pre, seed)
        loss, g_ac, g_qf = ctx.adjoint(target)
    finally:
        ctx.close()
    loss_r, g_ac_r, g_qf_r = reference(frame, target, dec)
    print(f"loss {loss:.9g} ref {loss_r:.9g}")
    assert abs(loss - loss_r) <= 1e-4 * loss_r
    compare("grad_ac", g_ac, g_ac_r)
    compare("grad_qf", g_qf, g_qf_r)


@pytest.mark.parametrize("variant", ["all_types", "no_hf", "no_gaborish",
                                     "epf_off", "sharpened", "no_lf"])
def test_adjoint_matches_fp64_reference(variant):
    frame = synthetic.make_frame(261, 203, seed=11, qf_median=10.0,
                                 shares=SHARES)
    if variant == "no_hf":
        frame.predict_hf = 0
    if variant == "no_gaborish":
        frame.gaborish = 0
    if variant == "epf_off":
        frame.have_ar = 0
    if variant == "sharpened":
        frame.epf_use_sharpened = 1
    if variant == "no_lf":
        frame.predict_lf = 0
    check_against_reference(frame)


@pytest.mark.parametrize("size", [(8, 8), (13, 7), (600, 70), (70, 600)])
def test_adjoint_small_and_ragged(size):
    frame = synthetic.make_frame(*size, seed=21, qf_median=9.0)
    check_against_reference(frame)


def test_adjoint_split_bf16_forward():
    frame = synthetic.make_frame(261, 203, seed=12, qf_median=10.0,
                                 shares=SHARES)
    check_against_reference(frame, form="split_bf16")


def check_fd(name, fd, g, scale):
    """Every entry within 1e-3 of itself plus 1e-4 of the gradient's largest
    entry (the FP32 gradient's own rounding, ~5e-5 of it), and the sampled
    vector within 1e-3 in relative L2."""
    fd, g = np.asarray(fd), np.asarray(g, np.float64)
    err = np.abs(fd - g)
    rel = np.linalg.norm(fd - g) / np.linalg.norm(fd)
    print(f"{name}: {len(g)} entries, rel_l2 {rel:.3g}, max_abs {err.max():.3g}"
          f" (scale {scale:.3g})")
    bad = np.nonzero(err > 1e-3 * np.abs(fd) + 1e-4 * scale)[0]
    assert len(bad) == 0, list(zip(fd[bad], g[bad]))[:5]
    assert rel <= 1e-3


def finite_differences(frame, n_ac, n_qf, seed):
    """The CUDA gradient at sampled entries against central differences of
    the FP64 forward (oracle/finite_diff.py) with every discrete decision --
    EPF guide and sigma, DC EPF, clamp branches -- taken from the CUDA
    forward pass: step 1e-3 of each coefficient's quantisation step, and a
    relative 1e-3 on the quant field. (Differences of the FP32 forward
    itself resolve such steps only to its rounding, and a larger step
    crosses the curvature of the clamp's 1 / |correction|.)"""
    ctx, dec, pre = forward(frame)
    try:
        target = make_target(pre, seed)
        _, g_ac, g_qf = ctx.adjoint(target)
    finally:
        ctx.close()
    dg, ds = decisions.dc_decisions(frame)
    kw = dict(dc_guide=dg, dc_sigma=ds)
    if frame.have_ar:
        kw.update(guide=dec[0], sigma=dec[1], clamp_tape=dec[2])
    rng = np.random.default_rng(seed)
    idx = rng.choice(g_ac.size, n_ac, replace=False)
    by, bx = frame.blocks
    cells = [divmod(int(c), bx) for c in rng.choice(by * bx, n_qf,
                                                    replace=False)]
    fd_ac, fd_qf = finite_diff.gradients(frame, target, kw, idx, cells)
    check_fd("grad_ac", fd_ac, g_ac.ravel()[idx], np.abs(g_ac).max())
    check_fd("grad_qf", fd_qf, [g_qf[y, x] for y, x in cells],
             np.abs(g_qf).max())


def test_adjoint_matches_finite_differences():
    frame = synthetic.make_frame(261, 203, seed=13, qf_median=10.0,
                                 shares=SHARES)
    finite_differences(frame, n_ac=256, n_qf=64, seed=5)


def test_adjoint_1024_distance_1_5():
    """1024 x 1024 at distance 1.5 (quant field ~ 18 / 1.5), every block
    size, EPF on: the full gradient against the FP64 reference, and 256 AC
    entries + 64 quant-field cells against finite differences."""
    frame = synthetic.make_frame(1024, 1024, seed=4, qf_median=12.0,
                                 shares=SHARES)
    check_against_reference(frame, seed=1)
    finite_differences(frame, n_ac=256, n_qf=64, seed=6)


def test_adjoint_reference_encoded_frame_source_target():
    """The adjoint workload itself: the 1024 x 1024 generator image encoded
    by the reference encoder at distance 1.5 (tests/golden/
    c4_1k_d15_frame.npz), with the source image's XYB as the target (the
    loss an encoder minimises). Full gradient against the FP64 reference."""
    import os
    from pik_b200 import layout, xyb
    from tests import golden_cases
    frame = layout.Frame.load(os.path.join(golden_cases.GOLDEN,
                                           "c4_1k_d15_frame.npz"))
    src = dict(synthetic.ADJOINT_SOURCE)
    img = synthetic.make_image(src.pop("xsize"), src.pop("ysize"), **src)
    target = xyb.linear_to_xyb(synthetic.srgb8_to_linear255(img))
    ctx, dec, pre = forward(frame)
    try:
        loss, g_ac, g_qf = ctx.adjoint(target)
    finally:
        ctx.close()
    loss_r, g_ac_r, g_qf_r = reference(frame, target, dec)
    print(f"loss {loss:.9g} ref {loss_r:.9g} (per pixel "
          f"{loss / pre[0].size:.3g})")
    assert abs(loss - loss_r) <= 1e-4 * loss_r
    compare("grad_ac", g_ac, g_ac_r)
    compare("grad_qf", g_qf, g_qf_r)


def test_own_branches_differ_only_by_branch_flips():
    """With its own clamp branches the FP64 reference gradient differs from
    the CUDA one only on blocks where the two precisions' clamp branches
    differ (checked here against the shared-branch reference): the shared
    tape is what makes the comparison exact, not a tolerance."""
    frame = synthetic.make_frame(261, 203, seed=11, qf_median=10.0,
                                 shares=SHARES)
    ctx, dec, pre = forward(frame)
    try:
        target = make_target(pre, 0)
        _, g_ac, _ = ctx.adjoint(target)
    finally:
        ctx.close()
    _, shared, _ = reference(frame, target, dec)
    _, own, _ = reference(frame, target, dec, tape=False)
    by, bx = frame.blocks
    blk = lambda a: np.abs(a).reshape(3, by, bx, 64).max(axis=(0, 3))
    scale = np.abs(shared).max()
    flipped = blk(own - shared) > 1e-6 * scale
    print(f"blocks whose FP64 gradient moves with the branches: "
          f"{flipped.sum()} of {by * bx}")
    assert flipped.mean() < 0.05
    compare("grad_ac (shared branches)", g_ac, shared)


def test_clamp_tape_replay_reproduces_the_pass():
    """Following its own recorded branches reproduces a forward pass bit for
    bit; an invalid code is rejected."""
    frame = synthetic.make_frame(261, 203, seed=14, qf_median=10.0,
                                 shares=SHARES)
    for form in ("fp32", "split_bf16"):
        ctx, dec, _ = forward(frame, form)
        try:
            want = ctx.reconstruct(linear=True)[0]
            tape = dec[2]
            assert tape.shape == (frame.blocks[0], frame.blocks[1] * 64)
            assert set(np.unique(tape)) <= {0, 1, 2, 3, 4}
            ctx.set_clamp_decisions(tape)
            got = ctx.reconstruct(linear=True)[0]
            np.testing.assert_array_equal(got, want)
            np.testing.assert_array_equal(ctx.clamp_decisions(), tape)
            bad = tape.copy()
            bad[0, 0] = 5
            with pytest.raises(native.PikGpuError) as e:
                ctx.set_clamp_decisions(bad)
            assert e.value.code == -1
        finally:
            ctx.close()


def test_adjoint_errors():
    ctx = native.Context(0)
    try:
        with pytest.raises(native.PikGpuError) as e:
            ctx.adjoint(np.zeros((3, 8, 8), np.float32))
        assert e.value.code == -4
        f = synthetic.make_frame(16, 16, seed=2)
        ctx.begin(f)
        with pytest.raises(native.PikGpuError) as e:  # no AC yet
            ctx.adjoint(np.zeros((3, 16, 16), np.float32))
        assert e.value.code == -4
        with pytest.raises(ValueError):
            ctx.adjoint(np.zeros((3, 8, 16), np.float32))
    finally:
        ctx.close()

"""The FP64 adjoint of the oracle (oracle/pik_adjoint.inc) against FP64
central finite differences of its own forward pass, with the EPF decisions
held at the base point. This pins the reference gradient that the CUDA
adjoint is checked against. Tolerances: AC coefficients within 1e-5
absolute (gradients up to ~3) and the quant field within 1e-3 relative."""

import numpy as np
import pytest

from oracle import decisions, finite_diff, oraclepy
from pik_b200 import synthetic

SHARES = {"DCT": 0.3, "DCT16X16": 0.3, "DCT32X32": 0.2, "DCT4X4": 0.05,
          "DCT2X2": 0.05, "IDENTITY": 0.04, "LINES": 0.03, "DCT_NOHF": 0.02,
          "DCT4X4_NOHF": 0.01}


def fd_check(frame, n_ac=24, n_qf=8, seed=0):
    base = oraclepy.run(frame, precision=64, want=("dequant_ac", "pre_opsin"),
                        export_decisions=bool(frame.have_ar))
    kw = {}
    if frame.have_ar:
        kw.update(guide=base["guide"], sigma=base["sigma"])
    dg, ds = decisions.dc_decisions(frame)
    kw.update(dc_guide=dg, dc_sigma=ds)
    rng = np.random.default_rng(seed)
    target = base["pre_opsin"] + rng.normal(0, 0.01, base["pre_opsin"].shape)
    _, g_ac, g_qf = oraclepy.adjoint(frame, target, **kw)
    ac0 = base["dequant_ac"]
    h = 1e-4
    for i in rng.integers(0, ac0.size, n_ac):
        a = ac0.copy().ravel()
        a[i] += h
        lp = oraclepy.adjoint(frame, target, ac_dequant=a.reshape(ac0.shape),
                              grads=False, **kw)[0]
        a[i] -= 2 * h
        lm = oraclepy.adjoint(frame, target, ac_dequant=a.reshape(ac0.shape),
                              grads=False, **kw)[0]
        assert abs((lp - lm) / (2 * h) - g_ac.ravel()[i]) <= 1e-5
    by, bx = frame.blocks
    qf = frame.raw_quant_field.astype(np.float64)
    for ci in rng.integers(0, by * bx, n_qf):
        yb, xb = divmod(int(ci), bx)
        loss = []
        for sgn in (1, -1):
            qn = qf[yb, xb] * (1 + sgn * 1e-3)
            scale = np.ones((by, bx))
            scale[yb, xb] = qf[yb, xb] / qn
            a = ac0.copy()
            a[:, yb, xb * 64:(xb + 1) * 64] *= qf[yb, xb] / qn
            loss.append(oraclepy.adjoint(frame, target, ac_dequant=a,
                                         ar_scale=scale, grads=False,
                                         **kw)[0])
        fd = (loss[0] - loss[1]) / (2e-3 * qf[yb, xb])
        assert abs(fd - g_qf[yb, xb]) <= 1e-3 * abs(fd) + 1e-7


@pytest.mark.parametrize("variant", ["all_types", "no_hf", "no_gaborish",
                                     "epf_off"])
def test_oracle_adjoint_matches_finite_differences(variant):
    frame = synthetic.make_frame(136, 104, seed=8, qf_median=10.0,
                                 shares=SHARES)
    if variant == "no_hf":
        frame.predict_hf = 0
    if variant == "no_gaborish":
        frame.gaborish = 0
    if variant == "epf_off":
        frame.have_ar = 0
    fd_check(frame)


def test_finite_diff_module_matches_the_adjoint():
    """oracle/finite_diff.py (the pool-based differences the CUDA adjoint is
    checked with) against the FP64 adjoint, decisions held at the base
    point's."""
    frame = synthetic.make_frame(72, 64, seed=3, qf_median=10.0,
                                 shares=SHARES)
    base = oraclepy.run(frame, precision=64, want=("pre_opsin",),
                        export_decisions=True)
    dg, ds = decisions.dc_decisions(frame)
    kw = dict(guide=base["guide"], sigma=base["sigma"], dc_guide=dg,
              dc_sigma=ds)
    rng = np.random.default_rng(2)
    target = base["pre_opsin"] + rng.normal(0, 0.01, base["pre_opsin"].shape)
    _, g_ac, g_qf = oraclepy.adjoint(frame, target, **kw)
    idx = rng.choice(g_ac.size, 16, replace=False)
    cells = [(1, 2), (5, 7)]
    fd_ac, fd_qf = finite_diff.gradients(frame, target, kw, idx, cells,
                                         workers=2)
    np.testing.assert_allclose(fd_ac, g_ac.ravel()[idx], rtol=1e-3,
                               atol=1e-7)
    np.testing.assert_allclose(fd_qf, [g_qf[y, x] for y, x in cells],
                               rtol=1e-3, atol=1e-9)

"""Central finite differences of the FP64 oracle's forward pass (test
infrastructure, like the rest of oracle/).

The function is the loss of oracle/pik_adjoint.inc,
L = sum((pre_opsin - target)^2), of one dequantised AC coefficient or of one
cell's quant field (a real number: the cell's coefficients scale with
qf / qf' and its clamp intervals with the same factor), every discrete
decision -- the EPF's guide and sigma, the DC EPF's, the clamp's branch per
coefficient -- held at the values given in `decisions` (keyword arguments of
oraclepy.adjoint). A coefficient moves by `step` of its quantisation step
(DequantMatrix * InvGlobalScale / qf, pik/compressed_image.cc:586-707), the
unit the integer AC lives on; the quant field by a relative `step`.

The evaluations (two FP64 forward passes each) run in a pool of spawned
processes, each holding the frame, target and base coefficients."""

from __future__ import annotations

import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np

from oracle import oraclepy

_state: dict = {}


def _init(frame, target, ac0, decisions):
    _state.update(frame=frame, target=target, ac0=ac0, decisions=decisions)


def _loss(ac, scale=None):
    s = _state
    return oraclepy.adjoint(s["frame"], s["target"], ac_dequant=ac,
                            ar_scale=scale, grads=False,
                            **s["decisions"])[0]


def _ac_task(i: int, h: float) -> float:
    ac = _state["ac0"].copy()
    flat = ac.reshape(-1)
    x = flat[i]
    flat[i] = x + h
    lp = _loss(ac)
    flat[i] = x - h
    lm = _loss(ac)
    return (lp - lm) / (2 * h)


def _qf_task(yb: int, xb: int, rel: float) -> float:
    frame, ac0 = _state["frame"], _state["ac0"]
    by, bx = frame.blocks
    q = float(frame.raw_quant_field[yb, xb])
    out = []
    for sgn in (1, -1):
        qn = q * (1 + sgn * rel)
        scale = np.ones((by, bx))
        scale[yb, xb] = q / qn
        a = ac0.copy()
        a[:, yb, xb * 64:(xb + 1) * 64] *= q / qn
        out.append(_loss(a, scale))
    return (out[0] - out[1]) / (2 * rel * q)


def quant_step(frame, flat_index: int) -> float:
    """Quantisation step of the dequantised AC entry `flat_index` of the
    (3, By, Bx*64) frame layout: the dequant matrix entry of its cell, kind
    and channel times InvGlobalScale / qf."""
    by, bx = frame.blocks
    c, y, xk = np.unravel_index(flat_index, (3, by, bx * 64))
    x, k = divmod(int(xk), 64)
    a = int(frame.ac_strategy[y, x])
    typ, blk = a >> 4, a & 0xF
    kind = {7: 0, 8: 3}.get(typ, typ)  # DCT_NOHF, DCT4X4_NOHF
    qf = int(frame.raw_quant_field[y, x])
    cf = int(frame.dequant_control_field[y // 8, x // 8])
    table = int(frame.dequant_map[cf, qf - 1])
    off = int(frame.dequant_offsets.reshape(-1)[(table * 7 + kind) * 3 + c])
    dm = float(frame.dequant_table.reshape(-1)[off + blk * 64 + k])
    return dm * (65536.0 / frame.global_scale) / qf


def gradients(frame, target: np.ndarray, decisions: dict, ac_entries,
              qf_cells, *, step: float = 1e-3, workers: int | None = None):
    """Finite-difference gradients at the given flat AC indices and
    (yb, xb) quant-field cells. Returns (fd_ac, fd_qf) as float64 arrays."""
    base = oraclepy.run(frame, precision=64, want=("dequant_ac",),
                        **{k: v for k, v in decisions.items()
                           if k in ("guide", "sigma", "dc_guide", "dc_sigma",
                                    "clamp_tape")})
    ac0 = base["dequant_ac"]
    t = np.ascontiguousarray(target, np.float64)
    n = workers or max(1, min(16, os.cpu_count() or 1))
    with ProcessPoolExecutor(max_workers=n,
                             mp_context=mp.get_context("spawn"),
                             initializer=_init,
                             initargs=(frame, t, ac0, decisions)) as pool:
        fa = [pool.submit(_ac_task, int(i), step * quant_step(frame, int(i)))
              for i in ac_entries]
        fq = [pool.submit(_qf_task, int(y), int(x), step) for y, x in qf_cells]
        return (np.array([f.result() for f in fa]),
                np.array([f.result() for f in fq]))

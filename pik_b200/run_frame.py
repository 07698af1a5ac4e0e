"""Reconstructs a frozen frame file (layout.Frame .npz) on the GPU.

    python -m pik_b200.run_frame FRAME.npz [--crop W H] [--reps N]
           [--form fp32|split_bf16|split_bf16x3] [--out linear.npy]
    python -m pik_b200.run_frame --highlight W H [--mix broad|encoder] ...

`--crop` keeps the top-left W x H pixels (multiples of 64 keep the colour
tiles and transform placement intact), which makes small cases of a large
frame for profiling. `--highlight W H` generates a frame of the 8192x8192
workload's kind at any size instead.
"""

from __future__ import annotations

import argparse
import dataclasses
import sys
import time

import numpy as np

from . import layout, native, synthetic


def crop(frame: layout.Frame, w: int, h: int) -> layout.Frame:
    w, h = min(w, frame.xsize), min(h, frame.ysize)
    bx, by = -(-w // 8), -(-h // 8)
    tx, ty = -(-w // 64), -(-h // 64)
    acs = frame.ac_strategy[:by, :bx].copy()
    # A multi-block transform cut by the crop edge becomes DCT8 blocks.
    for y in range(by):
        for x in range(bx):
            a = int(acs[y, x])
            cov = layout.ACS_COVER[a >> 4]
            if cov > 1:
                y0, x0 = y - (a & 0xF) // cov, x - (a & 0xF) % cov
                if y0 + cov > by or x0 + cov > bx:
                    acs[y, x] = 0
    return dataclasses.replace(
        frame, xsize=w, ysize=h, ac_strategy=acs,
        raw_quant_field=frame.raw_quant_field[:by, :bx].copy(),
        ar_sigma_lut_ids=frame.ar_sigma_lut_ids[:by, :bx].copy(),
        quantized_dc=frame.quantized_dc[:, :by, :bx].copy(),
        quantized_ac=frame.quantized_ac[:, :by, :bx * 64].copy(),
        ytox_map=frame.ytox_map[:ty, :tx].copy(),
        ytob_map=frame.ytob_map[:ty, :tx].copy(),
        dequant_control_field=frame.dequant_control_field[:ty, :tx].copy())


def parse_args(argv=None) -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("frame", nargs="?", help="frozen frame (.npz)")
    ap.add_argument("--highlight", nargs=2, type=int, metavar=("W", "H"),
                    help="instead of a file: a W x H frame from the "
                         "8192x8192 workload's generator (seed 5)")
    ap.add_argument("--mix", default="broad", choices=["broad", "encoder"],
                    help="transform mix of --highlight frames")
    ap.add_argument("--crop", nargs=2, type=int)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--out")
    ap.add_argument("--form", default="fp32", choices=sorted(native.FORMS))
    args = ap.parse_args(argv)
    if (args.frame is None) == (args.highlight is None):
        ap.error("give either a frame file or --highlight W H")
    return args


def load_frame(args: argparse.Namespace) -> layout.Frame:
    if args.highlight:
        shares = (synthetic.ENCODER_SHARES_D05 if args.mix == "encoder"
                  else None)
        frame = synthetic.make_highlight_frame(*args.highlight, seed=5,
                                               shares=shares)
    else:
        frame = layout.Frame.load(args.frame)
    if args.crop:
        frame = crop(frame, *args.crop)
    return frame


def main(argv=None) -> int:
    args = parse_args(argv)
    frame = load_frame(args)
    ctx = native.Context(0, form=args.form)
    ctx.begin(frame)
    ctx.set_ac()
    t = time.perf_counter()
    for _ in range(args.reps):
        lin, _ = ctx.reconstruct(linear=True)
    dt = (time.perf_counter() - t) / args.reps
    ctx.close()
    print(f"{frame.xsize}x{frame.ysize}: {dt * 1e3:.3f} ms per frame "
          f"(host wall, including copies)")
    if args.out:
        np.save(args.out, lin)
    return 0


if __name__ == "__main__":
    sys.exit(main())

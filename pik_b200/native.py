"""Python access to the native library (pik_b200/libpikgpu.so, the C ABI of
include/pikgpu.h). Fails loudly when the library is missing: there is no
fallback implementation."""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import abi, layout

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        "libpikgpu.so")

OK = 0
ERRORS = {-1: "INVALID_ARG", -2: "UNSUPPORTED", -3: "CUDA", -4: "STATE",
          -5: "NO_MEMORY"}
STAGES = {"dc": 0, "idct": 1, "smoothed": 2, "epf": 3, "ar": 4,
          "pre_opsin": 5, "dequant_ac": 6}
OPT_KEEP_STAGES = 1
OPT_PROFILE = 2
OPT_FORM = 3
OPT_GRAPHS = 4
OPT_TC_WAIT_POLLS = 5
FORMS = {"fp32": 0, "split_bf16": 1, "split_bf16x3": 2}

_lib = None


class PikGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -c 'import "
            f"__graft_entry__ as g; g.build()'` (no fallback exists)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    S = ctypes.c_size_t
    L.pikgpu_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
    L.pikgpu_ctx_destroy.argtypes = [P]
    L.pikgpu_last_error.restype = ctypes.c_char_p
    L.pikgpu_last_error.argtypes = [P]
    L.pikgpu_validate.argtypes = [P, ctypes.c_char_p, S]
    L.pikgpu_set_option.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.pikgpu_frame_begin.argtypes = [P, P]
    L.pikgpu_frame_set_ac.argtypes = [P, ctypes.POINTER(P), S]
    L.pikgpu_frame_set_group_ac.argtypes = [P, ctypes.c_uint32,
                                            ctypes.POINTER(P), S]
    L.pikgpu_frame_set_ac_device.argtypes = [P, ctypes.POINTER(P), S]
    L.pikgpu_reconstruct.argtypes = [P, ctypes.POINTER(P), S, P, S,
                                     ctypes.c_int]
    L.pikgpu_get_stage.argtypes = [P, ctypes.c_int, ctypes.POINTER(P), S, S,
                                   S]
    L.pikgpu_set_epf_decisions.argtypes = [P, P, P]
    L.pikgpu_get_epf_decisions.argtypes = [P, P, P]
    L.pikgpu_last_kernel_times.argtypes = [P, P, ctypes.c_int]
    L.pikgpu_kernel_name.restype = ctypes.c_char_p
    L.pikgpu_kernel_name.argtypes = [ctypes.c_int]
    L.pikgpu_set_stream.argtypes = [P, P]
    L.pikgpu_last_launch_count.argtypes = [P]
    L.pikgpu_dc_reconstruct_noalloc.argtypes = [
        P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32,
        P, ctypes.c_int32, ctypes.c_int32, P, P, ctypes.c_char_p, S]
    L.pikgpu_adjoint.argtypes = [P, P, P, P, P, ctypes.c_int]
    L.pikgpu_graph_stats.argtypes = [P, P, P]
    L.pikgpu_encode_pnm.argtypes = [P, ctypes.c_int, ctypes.c_int, P, S,
                                    ctypes.POINTER(S), ctypes.c_int]
    L.pikgpu_reconstruct_async.argtypes = [P, ctypes.POINTER(P), S, P, S,
                                           ctypes.c_int]
    L.pikgpu_wait.argtypes = [P]
    L.pikgpu_frame_set_dequantized_ac.argtypes = [P, P, ctypes.c_int]
    L.pikgpu_frame_set_clamp_scale.argtypes = [P, P, ctypes.c_int]
    L.pikgpu_set_clamp_decisions.argtypes = [P, P]
    L.pikgpu_get_clamp_decisions.argtypes = [P, P]
    L.pikgpu_batch_create.argtypes = [ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(P)]
    L.pikgpu_batch_destroy.argtypes = [P]
    L.pikgpu_batch_frame.restype = P
    L.pikgpu_batch_frame.argtypes = [P, ctypes.c_int]
    L.pikgpu_batch_reconstruct.argtypes = [P, ctypes.POINTER(P),
                                           ctypes.POINTER(S), P]
    L.pikgpu_batch_last_error.restype = ctypes.c_char_p
    L.pikgpu_batch_last_error.argtypes = [P]
    L.pikgpu_batch_launch_count.argtypes = [P]
    L.pikgpu_batch_capture_count.argtypes = [P]
    L.pikgpu_batch_autotune.argtypes = [P, ctypes.POINTER(P),
                                        ctypes.POINTER(S), P,
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
    _lib = L
    return L


def validate(frame: layout.Frame) -> tuple[int, str]:
    """Host-only validation (no device needed)."""
    packed = abi.PackedFrame(frame)
    buf = ctypes.create_string_buffer(512)
    rc = lib().pikgpu_validate(packed.ref, buf, 512)
    return rc, buf.value.decode()


def dc_reconstruct_noalloc(qdc_ptr: int, xsize_blocks: int,
                           ysize_blocks: int, global_scale: int,
                           quant_dc: int, dc_dequant, ytox_dc: int,
                           ytob_dc: int, dc_ptr: int, stream: int = 0) -> None:
    """pikgpu_dc_reconstruct_noalloc on device buffers (3 contiguous int16
    planes in, 3 contiguous float planes out) on the current device."""
    mul = np.ascontiguousarray(dc_dequant, np.float32)
    assert mul.shape == (3,)
    buf = ctypes.create_string_buffer(512)
    rc = lib().pikgpu_dc_reconstruct_noalloc(
        qdc_ptr or None, xsize_blocks, ysize_blocks, global_scale, quant_dc,
        mul.ctypes.data, ytox_dc, ytob_dc, dc_ptr or None, stream or None,
        buf, 512)
    if rc != OK:
        raise PikGpuError(rc, buf.value.decode())


def _planes(arrs) -> ctypes.Array:
    return (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])


class Context:
    """One pikgpu context (device memory + stream)."""

    def __init__(self, device: int = 0, *, keep_stages: bool = False,
                 profile: bool = False, form: str = "fp32",
                 graphs: bool = True):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.pikgpu_ctx_create(device, ctypes.byref(h))
        if rc != OK:
            raise PikGpuError(rc, "pikgpu_ctx_create failed")
        self.h = h
        self._check(self.L.pikgpu_set_option(h, OPT_KEEP_STAGES,
                                             int(keep_stages)))
        self._check(self.L.pikgpu_set_option(h, OPT_PROFILE, int(profile)))
        self._check(self.L.pikgpu_set_option(h, OPT_FORM, FORMS[form]))
        self._check(self.L.pikgpu_set_option(h, OPT_GRAPHS, int(graphs)))
        self.frame = None
        self._packed = None

    @classmethod
    def borrowed(cls, handle: int) -> "Context":
        """A view of a context owned by something else (a batch frame)."""
        self = cls.__new__(cls)
        self.L = lib()
        self.h = ctypes.c_void_p(handle)
        self._owned = False
        self.frame = None
        self._packed = None
        return self

    def close(self) -> None:
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.L.pikgpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int) -> None:
        if rc < 0:
            raise PikGpuError(rc, self.L.pikgpu_last_error(self.h).decode())

    def set_option(self, option: int, value: int) -> None:
        self._check(self.L.pikgpu_set_option(self.h, option, value))

    def begin(self, frame: layout.Frame) -> None:
        self._packed = abi.PackedFrame(frame)
        self.frame = frame
        self._check(self.L.pikgpu_frame_begin(self.h, self._packed.ref))

    def set_ac(self, ac: np.ndarray | None = None) -> None:
        a = self._packed.ac if ac is None else np.ascontiguousarray(ac,
                                                                    np.int16)
        self._ac_keep = a
        self._check(self.L.pikgpu_frame_set_ac(self.h, _planes(a),
                                               a.shape[-1]))

    def set_ac_device(self, plane_ptrs, stride: int) -> None:
        """pikgpu_frame_set_ac_device: three device pointers (int16 planes
        of By rows, `stride` elements apart). The context's own layout is
        read in place by later reconstructions; others are copied."""
        planes = (ctypes.c_void_p * 3)(*plane_ptrs)
        self._check(self.L.pikgpu_frame_set_ac_device(self.h, planes, stride))

    def set_group_ac(self, group: int, planes: np.ndarray) -> None:
        a = np.ascontiguousarray(planes, np.int16)
        self._check(self.L.pikgpu_frame_set_group_ac(self.h, group,
                                                     _planes(a), a.shape[-1]))

    def reconstruct(self, *, linear: bool = True, srgb8: bool = False):
        f = self.frame
        if f is None:  # let the library report the state error
            self._check(self.L.pikgpu_reconstruct(self.h, None, 0, None, 0,
                                                  0))
        lin = np.zeros((3, f.ysize, f.xsize), np.float32) if linear else None
        rgb = np.zeros((f.ysize, f.xsize, 3), np.uint8) if srgb8 else None
        self._check(self.L.pikgpu_reconstruct(
            self.h, _planes(lin) if lin is not None else None, f.xsize,
            rgb.ctypes.data if rgb is not None else None, 3 * f.xsize, 0))
        return lin, rgb

    def reconstruct_device(self, lin_ptr: int, lin_stride: int,
                           rgb_ptr: int = 0, rgb_stride: int = 0) -> None:
        """Outputs into device memory (three consecutive planes)."""
        f = self.frame
        planes = None
        if lin_ptr:
            plane = lin_stride * f.ysize * 4
            planes = (ctypes.c_void_p * 3)(lin_ptr, lin_ptr + plane,
                                           lin_ptr + 2 * plane)
        self._check(self.L.pikgpu_reconstruct(self.h, planes, lin_stride,
                                              rgb_ptr or None, rgb_stride, 1))

    def reconstruct_async(self, lin_planes, lin_stride: int,
                          rgb_ptr: int = 0, rgb_stride: int = 0,
                          on_device: bool = False) -> None:
        """pikgpu_reconstruct_async: `lin_planes` are 3 pointers (host
        pinned memory, or device); complete after wait()."""
        planes = None
        if lin_planes is not None:
            planes = (ctypes.c_void_p * 3)(*lin_planes)
        self._check(self.L.pikgpu_reconstruct_async(
            self.h, planes, lin_stride, rgb_ptr or None, rgb_stride,
            int(on_device)))

    def wait(self) -> None:
        self._check(self.L.pikgpu_wait(self.h))

    def stage(self, name: str) -> np.ndarray:
        f = self.frame
        by, bx = f.blocks
        shape = {"dc": (by, bx), "dequant_ac": (by, bx * 64),
                 "pre_opsin": (f.ysize, f.xsize)}.get(name, (by * 8, bx * 8))
        out = np.zeros((3,) + shape, np.float32)
        self._check(self.L.pikgpu_get_stage(self.h, STAGES[name],
                                            _planes(out), shape[1], shape[1],
                                            shape[0]))
        return out

    def set_decisions(self, guide: np.ndarray | None,
                      sigma: np.ndarray | None) -> None:
        g = None if guide is None else np.ascontiguousarray(guide, np.uint8)
        s = None if sigma is None else np.ascontiguousarray(sigma, np.int32)
        self._keep_dec = (g, s)
        self._check(self.L.pikgpu_set_epf_decisions(
            self.h, g.ctypes.data if g is not None else None,
            s.ctypes.data if s is not None else None))

    def decisions(self):
        f = self.frame
        by, bx = f.blocks
        g = np.zeros((3, by * 8 + 12, bx * 8 + 12), np.uint8)
        s = np.zeros((by, bx), np.int32)
        self._check(self.L.pikgpu_get_epf_decisions(self.h, g.ctypes.data,
                                                    s.ctypes.data))
        return g, s

    def adjoint(self, target: np.ndarray, *, grads: bool = True):
        """pikgpu_adjoint with host buffers: (loss, grad_ac (3, By, Bx*64),
        grad_qf (By, Bx)) of sum((pre_opsin - target)^2), `target` being
        (3, ysize, xsize) XYB."""
        f = self.frame
        if f is None:
            self._check(self.L.pikgpu_adjoint(self.h, None, None, None, None,
                                              0))
        by, bx = f.blocks
        t = np.ascontiguousarray(target, np.float32)
        if t.shape != (3, f.ysize, f.xsize):
            raise ValueError(f"target shape {t.shape}")
        loss = np.zeros(1, np.float64)
        g_ac = np.zeros((3, by, bx * 64), np.float32) if grads else None
        g_qf = np.zeros((by, bx), np.float32) if grads else None
        self._check(self.L.pikgpu_adjoint(
            self.h, t.ctypes.data, loss.ctypes.data,
            g_ac.ctypes.data if grads else None,
            g_qf.ctypes.data if grads else None, 0))
        return float(loss[0]), g_ac, g_qf

    def encode_pnm(self, bits: int = 8, srgb: bool = True) -> bytes:
        """pikgpu_encode_pnm of the last reconstruction: the bytes of a PPM
        (8 or 16 bits) or PFM (32) file."""
        n = ctypes.c_size_t()
        self._check(self.L.pikgpu_encode_pnm(self.h, bits, int(srgb), None,
                                             0, ctypes.byref(n), 0))
        buf = np.zeros(n.value, np.uint8)
        self._check(self.L.pikgpu_encode_pnm(self.h, bits, int(srgb),
                                             buf.ctypes.data, n.value,
                                             ctypes.byref(n), 0))
        return buf.tobytes()

    def clamp_decisions(self) -> np.ndarray:
        """The clamp tape of the last recording forward pass, (By, Bx*64)
        uint8."""
        by, bx = self.frame.blocks
        t = np.zeros((by, bx * 64), np.uint8)
        self._check(self.L.pikgpu_get_clamp_decisions(self.h, t.ctypes.data))
        return t

    def set_clamp_decisions(self, tape: np.ndarray | None) -> None:
        t = None if tape is None else np.ascontiguousarray(tape, np.uint8)
        self._keep_tape = t
        self._check(self.L.pikgpu_set_clamp_decisions(
            self.h, t.ctypes.data if t is not None else None))

    def set_dequantized_ac(self, ac: np.ndarray | None) -> None:
        """Dequantised AC (3, By, Bx*64) used instead of Dequant::DoAC's;
        None restores dequantising the int16 AC."""
        a = None if ac is None else np.ascontiguousarray(ac, np.float32)
        self._check(self.L.pikgpu_frame_set_dequantized_ac(
            self.h, a.ctypes.data if a is not None else None, 0))

    def set_clamp_scale(self, scale: np.ndarray | None) -> None:
        """Per-cell multiplier (By, Bx) of the clamp's non-LLF intervals."""
        a = None if scale is None else np.ascontiguousarray(scale,
                                                            np.float32)
        self._check(self.L.pikgpu_frame_set_clamp_scale(
            self.h, a.ctypes.data if a is not None else None, 0))

    def graph_stats(self) -> dict:
        cap, rep = ctypes.c_int(), ctypes.c_int()
        self._check(self.L.pikgpu_graph_stats(self.h, ctypes.byref(cap),
                                              ctypes.byref(rep)))
        return {"captures": cap.value, "last_replayed": bool(rep.value)}

    def kernel_times(self) -> dict:
        ms = np.zeros(16, np.float32)
        n = self.L.pikgpu_last_kernel_times(self.h, ms.ctypes.data, 16)
        self._check(n)
        return {self.L.pikgpu_kernel_name(i).decode(): float(ms[i])
                for i in range(n)}


class Batch:
    """pikgpu_batch: frames of uneven sizes reconstructed together by one
    captured CUDA graph (one branch per frame). Frame i is configured through
    `self.frames[i]` (a Context view: begin, set_ac, set_decisions)."""

    def __init__(self, num_frames: int, device: int = 0, *,
                 form: str = "fp32"):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.pikgpu_batch_create(device, num_frames, ctypes.byref(h))
        if rc != OK:
            raise PikGpuError(rc, "pikgpu_batch_create failed")
        self.h = h
        self.frames = [Context.borrowed(self.L.pikgpu_batch_frame(h, i))
                       for i in range(num_frames)]
        for c in self.frames:
            c._check(self.L.pikgpu_set_option(c.h, OPT_FORM, FORMS[form]))

    def close(self) -> None:
        if getattr(self, "h", None):
            for c in self.frames:
                c.h = None
            self.L.pikgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def reconstruct_device(self, out_ptrs, strides, stream: int = 0) -> None:
        """Frame i writes 3 consecutive planes (strides[i] x ysize floats)
        at device address out_ptrs[i]."""
        n = len(self.frames)
        outs = (ctypes.c_void_p * n)(*out_ptrs)
        st = (ctypes.c_size_t * n)(*strides)
        rc = self.L.pikgpu_batch_reconstruct(self.h, outs, st, stream or None)
        if rc != OK:
            raise PikGpuError(rc,
                              self.L.pikgpu_batch_last_error(self.h).decode())

    def autotune(self, out_ptrs, strides, stream: int = 0) -> dict:
        """Times the batch's launch shapes and keeps the fastest."""
        n = len(self.frames)
        outs = (ctypes.c_void_p * n)(*out_ptrs)
        st = (ctypes.c_size_t * n)(*strides)
        chains, tc = ctypes.c_int(), ctypes.c_int()
        rc = self.L.pikgpu_batch_autotune(self.h, outs, st, stream or None,
                                          ctypes.byref(chains),
                                          ctypes.byref(tc))
        if rc != OK:
            raise PikGpuError(rc,
                              self.L.pikgpu_batch_last_error(self.h).decode())
        return {"chains": chains.value, "tc_ctas_per_sm": tc.value}

    def launch_count(self) -> int:
        return self.L.pikgpu_batch_launch_count(self.h)

    def capture_count(self) -> int:
        return self.L.pikgpu_batch_capture_count(self.h)

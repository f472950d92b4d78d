"""Learned multilevel convolutional preconditioner (host wrapper of the C ABI).

The network, its tensor-core kernels and its training step live in the CUDA
library (csrc/precond.cu); this module packs batches of node grids into the
flat FP32 arrays the ABI takes and keeps the parameter blob (save / load).
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, lib


def _stream(stream):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)


def pack_samples(shapes):
    """ctypes sample array for [(nx, ny), ...] laid out back to back; returns (array, total nodes, offsets)."""
    arr = (_native.SilPrecondSample * len(shapes))()
    off = 0
    offsets = []
    for k, (nx, ny) in enumerate(shapes):
        arr[k].nx, arr[k].ny, arr[k].offset = int(nx), int(ny), off
        offsets.append(off)
        off += int(nx) * int(ny)
    return arr, off, offsets


class LearnedPreconditioner:
    def __init__(self, seed=0, stream=None):
        self._h = ctypes.c_void_p()
        check(lib().sil_precond_create(ctypes.byref(self._h), seed, _stream(stream)), "precond_create")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _native is not None and _native._lib is not None:
            try:
                _native._lib.sil_precond_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self._h = ctypes.c_void_p()

    @staticmethod
    def num_params():
        return int(lib().sil_precond_num_params())

    def get_params(self):
        out = np.zeros(self.num_params(), dtype=np.float32)
        check(lib().sil_precond_get_params(self._h, out.ctypes.data), "precond_get_params")
        return out

    def set_params(self, params, stream=None):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.num_params()
        check(lib().sil_precond_set_params(self._h, p.ctypes.data, _stream(stream)), "precond_set_params")

    def save(self, path):
        np.save(path, self.get_params())

    def load(self, path):
        self.set_params(np.load(path))

    def apply(self, shapes, nu, r, out, stream=None, active=None):
        """out = M(r); nu, r, out: flat torch CUDA float32 tensors laid out as pack_samples(shapes).
        active: optional torch CUDA int32 tensor, one entry per sample; samples
        whose entry is 0 are skipped (their part of out is left as it was)."""
        arr, n, _ = pack_samples(shapes)
        if active is None:
            check(lib().sil_precond_apply(self._h, _stream(stream), arr, len(shapes), nu.data_ptr(), r.data_ptr(),
                                          out.data_ptr()), "precond_apply")
        else:
            check(lib().sil_precond_apply_active(self._h, _stream(stream), arr, len(shapes), nu.data_ptr(),
                                                 r.data_ptr(), active.data_ptr(), out.data_ptr()),
                  "precond_apply_active")
        return out

    def loss_grad(self, shapes, nu, b, x, want_grad=True, stream=None):
        arr, n, _ = pack_samples(shapes)
        loss = ctypes.c_double()
        per = np.zeros(len(shapes))
        g = np.zeros(self.num_params(), dtype=np.float32) if want_grad else None
        check(lib().sil_precond_loss_grad(self._h, _stream(stream), arr, len(shapes), nu.data_ptr(), b.data_ptr(),
                                          x.data_ptr(), ctypes.byref(loss), per.ctypes.data,
                                          g.ctypes.data if want_grad else None), "precond_loss_grad")
        return loss.value, per, g

    def train_step(self, shapes, nu, b, x, lr, stream=None):
        arr, n, _ = pack_samples(shapes)
        loss = ctypes.c_double()
        check(lib().sil_precond_train_step(self._h, _stream(stream), arr, len(shapes), nu.data_ptr(), b.data_ptr(),
                                           x.data_ptr(), ctypes.c_float(lr), ctypes.byref(loss)), "precond_train_step")
        return loss.value

    def debug_fetch(self, which, level, count):
        out = np.zeros(count, dtype=np.float32)
        check(lib().sil_precond_debug_fetch(self._h, which, level, out.ctypes.data, count), "precond_debug_fetch")
        return out

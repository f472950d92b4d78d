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

    def get_optimizer_state(self):
        """(m, v, steps) of the library's Adam."""
        m = np.zeros(self.num_params(), dtype=np.float32)
        v = np.zeros(self.num_params(), dtype=np.float32)
        t = ctypes.c_int64(0)
        check(lib().sil_precond_get_optimizer_state(self._h, m.ctypes.data, v.ctypes.data, ctypes.byref(t)),
              "precond_get_optimizer_state")
        return m, v, t.value

    def set_optimizer_state(self, m, v, steps, stream=None):
        m = np.ascontiguousarray(m, dtype=np.float32)
        v = np.ascontiguousarray(v, dtype=np.float32)
        check(lib().sil_precond_set_optimizer_state(self._h, m.ctypes.data, v.ctypes.data, int(steps), _stream(stream)),
              "precond_set_optimizer_state")

    def save_checkpoint(self, path, step, seed, extra=None):
        """A training checkpoint: header, parameters and the Adam state."""
        m, v, t = self.get_optimizer_state()
        write_checkpoint(path, self.get_params(), step, seed, dict(extra or {}, adam_steps=t), m=m, v=v)

    def load_checkpoint(self, path):
        """Restores the parameters (and the Adam state when the checkpoint has
        it) of a checkpoint; returns its (step, seed, extra)."""
        params, step, seed, extra, m, v = read_checkpoint(path, with_optimizer=True)
        self.set_params(params)
        if m is not None:
            self.set_optimizer_state(m, v, extra.get("adam_steps", step))
        return step, seed, extra

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


# ----------------------------------------------------------------- checkpoints
#
# Flat binary: 8-byte magic, then little-endian uint32 version, uint32 dtype
# code (1 = float32), uint64 parameter count, uint64 step, uint64 seed,
# uint64 length of a UTF-8 JSON block of extra fields, the JSON, then the
# parameters; version 2 adds the Adam moments m and v after them, so a
# resumed run continues exactly.

_MAGIC = b"SILPCKPT"


def write_checkpoint(path, params, step, seed, extra=None, m=None, v=None):
    """Writes the checkpoint to `path` + '.tmp', flushes it to disk and then
    renames it over `path`, so a crash or kill during the write leaves the
    previous checkpoint intact."""
    import json
    import os
    import struct
    p = np.ascontiguousarray(params, dtype=np.float32)
    blob = json.dumps(extra or {}, sort_keys=True).encode()
    version = 1 if m is None else 2
    tmp = str(path) + ".tmp"
    with open(tmp, "wb") as f:
        f.write(_MAGIC)
        f.write(struct.pack("<IIQQQQ", version, 1, p.size, int(step), int(seed), len(blob)))
        f.write(blob)
        f.write(p.tobytes())
        if m is not None:
            f.write(np.ascontiguousarray(m, dtype=np.float32).tobytes())
            f.write(np.ascontiguousarray(v, dtype=np.float32).tobytes())
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


def read_checkpoint(path, with_optimizer=False):
    """(params, step, seed, extra[, m, v]) of a checkpoint (m, v None for a
    version-1 file); ValueError on a malformed file."""
    import json
    import struct
    with open(path, "rb") as f:
        data = f.read()
    head = 8 + struct.calcsize("<IIQQQQ")
    if len(data) < head or data[:8] != _MAGIC:
        raise ValueError("not a preconditioner checkpoint")
    version, dtype, count, step, seed, nblob = struct.unpack("<IIQQQQ", data[8:head])
    if version not in (1, 2) or dtype != 1:
        raise ValueError(f"unsupported checkpoint version {version} / dtype {dtype}")
    arrays = 1 if version == 1 else 3
    if len(data) != head + nblob + 4 * count * arrays:
        raise ValueError("truncated or padded checkpoint")
    extra = json.loads(data[head:head + nblob].decode())
    off = head + nblob
    params = np.frombuffer(data, dtype="<f4", count=count, offset=off).copy()
    m = v = None
    if version == 2:
        m = np.frombuffer(data, dtype="<f4", count=count, offset=off + 4 * count).copy()
        v = np.frombuffer(data, dtype="<f4", count=count, offset=off + 8 * count).copy()
    return (params, step, seed, extra, m, v) if with_optimizer else (params, step, seed, extra)

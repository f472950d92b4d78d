"""similie_b200 -- B200 (sm_100a) discrete-exterior-calculus operators.

Python mirror of SimiLie's operator API for the DEC hot path, over the C ABI
in include/sil_b200.h (libsil_b200.so).  Fields are torch CUDA tensors used
purely as device buffers; every operator runs as a hand-written sm_100a
kernel.  Names, argument meaning and the (out, in) order follow the
reference:

  deriv / coboundary         src/similie/exterior/coboundary.hpp:614-709
  transposed_coboundary      src/similie/exterior/coboundary.hpp:656-696
  fill_discrete_hodge_star   src/similie/exterior/hodge_star.hpp:453-494
  hodge_star (tensor_prod with the stored star)   hodge_star.hpp:227-273
  codifferential, make_staged_codifferential      codifferential.hpp:510-656
  laplacian, make_staged_laplacian                laplacian.hpp:327-358, 814-951

A field tensor holds its lattice axes plus one form-component axis (last by
default, SimiLie's component-fastest "coalescent" layout; pass comp_axis=0
for the component-first layout).  `front` gives the absolute discrete
coordinate of element 0 per lattice axis (DDC domain front).
"""
import ctypes
from math import comb

import numpy as np

from . import _native
from ._native import SilError, check, lib

__all__ = [
    "Geometry", "MetricGeometry", "deriv", "coboundary", "transposed_coboundary", "hodge_star", "fill_discrete_hodge_star",
    "codifferential", "make_staged_codifferential", "laplacian", "make_staged_laplacian", "StagedLaplacian",
    "SilError", "field_struct",
]


def _torch():
    import torch
    return torch


def _dtype_code(t):
    torch = _torch()
    if t.dtype == torch.float64:
        return _native.SIL_F64
    if t.dtype == torch.float32:
        return _native.SIL_F32
    raise TypeError(f"similie_b200 fields are float64 or float32, got {t.dtype}")


def field_struct(t, comp_axis=-1, front=None):
    """sil_field describing a CUDA tensor (no copy)."""
    if not t.is_cuda:
        raise ValueError("similie_b200 operators take CUDA tensors (device buffers)")
    nd = t.dim()
    comp_axis = comp_axis % nd
    axes = [a for a in range(nd) if a != comp_axis]
    if len(axes) > _native.SIL_MAX_DIMS:
        raise ValueError("too many lattice dimensions")
    f = _native.SilField()
    f.data = t.data_ptr()
    f.dtype = _dtype_code(t)
    f.ndims = len(axes)
    f.ncomp = t.shape[comp_axis]
    for i, a in enumerate(axes):
        f.front[i] = 0 if front is None else int(front[i])
        f.extent[i] = t.shape[a]
        f.stride[i] = t.stride(a)
    f.comp_stride = t.stride(comp_axis)
    return f


def _stream(stream):
    if stream is None:
        return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _mask(form_dims, ndims):
    if form_dims is None:
        return (1 << ndims) - 1
    m = 0
    for d in form_dims:
        m |= 1 << int(d)
    return m


def deriv(out, inp, k, form_dims=None, comp_axis=-1, in_front=None, out_front=None, stream=None):
    """Coboundary d of a k-form (clamped sampling), bit-exact in FP64."""
    fi = field_struct(inp, comp_axis, in_front)
    fo = field_struct(out, comp_axis, out_front)
    check(lib().sil_deriv(_stream(stream), _mask(form_dims, fi.ndims), k, ctypes.byref(fi), ctypes.byref(fo)),
          "deriv")
    return out


coboundary = deriv


def transposed_coboundary(out, inp, k, form_dims=None, comp_axis=-1, in_front=None, out_front=None, stream=None):
    """Transposed coboundary (zero-outside sampling, backward shift, negated sum)."""
    fi = field_struct(inp, comp_axis, in_front)
    fo = field_struct(out, comp_axis, out_front)
    check(lib().sil_transposed_coboundary(_stream(stream), _mask(form_dims, fi.ndims), k, ctypes.byref(fi),
                                          ctypes.byref(fo)), "transposed_coboundary")
    return out


class Geometry:
    """Rectilinear grid with the identity metric: per-axis node coordinates.

    Stands for the (position, metric) tensor-field pair SimiLie passes to its
    staged operators when position(i, j, ...) = (x_i, y_j, ...) and the metric
    is the identity."""

    def __init__(self, coords, front=None):
        self.n = len(coords)
        self._coords = [np.ascontiguousarray(c, dtype=np.float64) for c in coords]
        ptrs = (ctypes.c_void_p * self.n)(*[c.ctypes.data for c in self._coords])
        npts = (ctypes.c_int64 * self.n)(*[len(c) for c in self._coords])
        fr = (ctypes.c_int64 * self.n)(*(front if front is not None else [0] * self.n))
        self._h = ctypes.c_void_p()
        check(lib().sil_geometry_create(ctypes.byref(self._h), self.n, ptrs, npts, fr), "Geometry")

    @classmethod
    def from_position(cls, position, metric=None, front=None, atol=0.0):
        """Build from SimiLie-style position (and optional metric) fields given
        as host arrays shaped (*lattice, n) / (*lattice, n*n).  Only the
        rectilinear identity-metric case is accepted."""
        pos = np.asarray(position, dtype=np.float64)
        n = pos.shape[-1]
        coords = []
        for a in range(n):
            idx = [0] * n
            idx[a] = slice(None)
            c = pos[tuple(idx) + (a,)]
            expect = np.expand_dims(c, tuple(d for d in range(n) if d != a))
            if np.max(np.abs(pos[..., a] - expect)) > atol:
                raise NotImplementedError("position field is not a tensor product of per-axis coordinates")
            coords.append(c)
        if metric is not None:
            m = np.asarray(metric, dtype=np.float64).reshape(pos.shape[:-1] + (n, n))
            if np.max(np.abs(m - np.eye(n))) > atol:
                raise NotImplementedError("only the identity metric has a diagonal Hodge star here")
        return cls(coords, front=front)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value is not None and _native._lib is not None:
            _native._lib.sil_geometry_destroy(h)
            self._h = None


def hodge_star(geometry, out, inp, k, form_dims=None, comp_axis=-1, in_front=None, out_front=None, stream=None):
    """Hodge star of a k-form into an (n-k)-form at every node of `out`."""
    fi = field_struct(inp, comp_axis, in_front)
    fo = field_struct(out, comp_axis, out_front)
    check(lib().sil_hodge_star(geometry.handle, _stream(stream), _mask(form_dims, fi.ndims), k, ctypes.byref(fi),
                               ctypes.byref(fo)), "hodge_star")
    return out


def fill_discrete_hodge_star_metric(hodge, position, k_in, metric=None, fronts=None, stream=None):
    """Stored Hodge tensor of a general metric: hodge (*lattice, n**k_in * C(n, n-k_in)),
    position (*lattice, n), metric (*lattice, n*n) or None for the identity (FP64 CUDA tensors).
    fronts: optional dict of lattice fronts for 'hodge', 'position', 'metric'."""
    fronts = fronts or {}
    n = position.shape[-1]
    fh = field_struct(hodge, -1, fronts.get("hodge"))
    fp = field_struct(position, -1, fronts.get("position"))
    fm = field_struct(metric, -1, fronts.get("metric")) if metric is not None else None
    check(lib().sil_fill_discrete_hodge_star_metric(_stream(stream), n, k_in, ctypes.byref(fp),
                                                     ctypes.byref(fm) if fm is not None else None,
                                                     ctypes.byref(fh)), "fill_discrete_hodge_star_metric")
    return hodge


def hodge_star_stored(hodge, out, inp, n, k_in, fronts=None, stream=None):
    """out = tensor_prod(inp, hodge): apply a stored Hodge tensor to a k-form (FP64 CUDA tensors)."""
    fronts = fronts or {}
    fh = field_struct(hodge, -1, fronts.get("hodge"))
    fi = field_struct(inp, -1, fronts.get("in"))
    fo = field_struct(out, -1, fronts.get("out"))
    check(lib().sil_hodge_star_stored(_stream(stream), n, k_in, ctypes.byref(fh), ctypes.byref(fi),
                                      ctypes.byref(fo)), "hodge_star_stored")
    return out


def fill_discrete_hodge_star(geometry, hodge, k_in, front=None, stream=None):
    """Stored per-node Hodge tensor, shape (*lattice, n**k_in * C(n, n-k_in))."""
    fh = field_struct(hodge, -1, front)
    check(lib().sil_fill_discrete_hodge_star(geometry.handle, _stream(stream), k_in, ctypes.byref(fh)),
          "fill_discrete_hodge_star")
    return hodge


def codifferential(geometry, out, inp, k, form_dims=None, comp_axis=-1, in_front=None, out_front=None, stream=None):
    """Codifferential of a k-form (single fused kernel)."""
    fi = field_struct(inp, comp_axis, in_front)
    fo = field_struct(out, comp_axis, out_front)
    check(lib().sil_codifferential(geometry.handle, _stream(stream), _mask(form_dims, fi.ndims), k, ctypes.byref(fi),
                                   ctypes.byref(fo)), "codifferential")
    return out


class StagedCodifferential:
    """make_staged_codifferential(...).run(out, in) with nothing to precompute:
    the Hodge factors come from the geometry inside the kernel."""

    def __init__(self, geometry, k, form_dims=None, comp_axis=-1):
        self.geometry, self.k, self.form_dims, self.comp_axis = geometry, k, form_dims, comp_axis

    def run(self, out, inp, in_front=None, out_front=None, stream=None):
        return codifferential(self.geometry, out, inp, self.k, self.form_dims, self.comp_axis, in_front, out_front,
                              stream)


def make_staged_codifferential(geometry, k, form_dims=None, comp_axis=-1):
    """Staged codifferential of a k-form: over a Geometry (rectilinear grid,
    identity metric; the Hodge factors come from the coordinates inside the
    kernel) or a MetricGeometry (the stored general-metric stars are filled
    once here)."""
    if isinstance(geometry, MetricGeometry):
        return MetricStagedCodifferential(geometry, k)
    return StagedCodifferential(geometry, k, form_dims, comp_axis)


class MetricGeometry:
    """The (position, metric) tensor-field pair of SimiLie's staged operators
    in the general case: position (*lattice, n) and metric (*lattice, n*n,
    row-major; None for the identity) as FP64 CUDA tensors over the n <= 3
    form dims, with optional lattice fronts.  Operators built on it store the
    per-node Hodge tensors fill_discrete_hodge_star computes from them."""

    def __init__(self, position, metric=None, position_front=None, metric_front=None):
        self.position = position.contiguous()
        self.metric = metric.contiguous() if metric is not None else None
        self.n = self.position.shape[-1]
        self._fp = field_struct(self.position, -1, position_front)
        self._fm = field_struct(self.metric, -1, metric_front) if self.metric is not None else None

    def fields(self):
        return ctypes.byref(self._fp), (ctypes.byref(self._fm) if self._fm is not None else None)


class MetricStagedCodifferential:
    """make_staged_codifferential(exec, tensor, metric, position): the k-form
    and (n-k+1)-form Hodge tensors are filled at construction over the
    position lattice; run(out, inp) is one fused kernel (FP64, fields over
    exactly the n form dims, inside the position lattice)."""

    def __init__(self, geometry, k, stream=None):
        self.geometry, self.k = geometry, k
        self._p = ctypes.c_void_p()
        fp, fm = geometry.fields()
        check(lib().sil_codifferential_plan_create(ctypes.byref(self._p), _stream(stream), geometry.n, k, fp, fm),
              "make_staged_codifferential")

    def run(self, out, inp, in_front=None, out_front=None, stream=None):
        fi = field_struct(inp, -1, in_front)
        fo = field_struct(out, -1, out_front)
        check(lib().sil_codifferential_run(self._p, _stream(stream), ctypes.byref(fi), ctypes.byref(fo)),
              "codifferential")
        return out

    def __del__(self):
        p = getattr(self, "_p", None)
        if p is not None and p.value is not None and _native._lib is not None:
            _native._lib.sil_codifferential_plan_destroy(p)
            self._p = None


class StagedLaplacian:
    """Hodge Laplacian plan.  mode 'fused' runs one pass over the fields;
    'unfused' runs the reference's kernel chain with intermediate buffers."""

    def __init__(self, geometry, out_like, inp_like, k, mode="fused", form_dims=None, comp_axis=-1, in_front=None,
                 out_front=None):
        self.geometry = geometry
        self.k = k
        self.comp_axis = comp_axis
        self.in_front, self.out_front = in_front, out_front
        fi = field_struct(inp_like, comp_axis, in_front)
        fo = field_struct(out_like, comp_axis, out_front)
        self.mask = _mask(form_dims, fi.ndims)
        self._p = ctypes.c_void_p()
        m = {"fused": 0, "unfused": 1}[mode]
        if isinstance(geometry, MetricGeometry):
            # stored general-metric Hodge tensors, filled here (fused only)
            if mode != "fused" or comp_axis % inp_like.dim() != inp_like.dim() - 1:
                raise ValueError("a MetricGeometry Laplacian is fused, component-last")
            fp, fm = geometry.fields()
            check(lib().sil_laplacian_plan_create_metric(ctypes.byref(self._p), _stream(None), geometry.n, k, fp, fm,
                                                         ctypes.byref(fi), ctypes.byref(fo)), "make_staged_laplacian")
            return
        check(lib().sil_laplacian_plan_create(ctypes.byref(self._p), geometry.handle, self.mask, k, ctypes.byref(fi),
                                              ctypes.byref(fo), m), "make_staged_laplacian")

    @property
    def kernel(self):
        return lib().sil_laplacian_plan_kernel(self._p)

    @property
    def variant(self):
        return lib().sil_laplacian_plan_variant(self._p)

    @property
    def scratch_bytes(self):
        return lib().sil_laplacian_plan_scratch_bytes(self._p)

    def run(self, out, inp, stream=None):
        fi = field_struct(inp, self.comp_axis, self.in_front)
        fo = field_struct(out, self.comp_axis, self.out_front)
        check(lib().sil_laplacian_run(self._p, _stream(stream), ctypes.byref(fi), ctypes.byref(fo)), "laplacian")
        return out

    def status(self):
        check(lib().sil_laplacian_plan_status(self._p), "laplacian status")

    def set_wait_bound(self, tries):
        """Bound of each pipeline wait of the TMA kernel in mbarrier polls (-1:
        the default; 0: every wait runs out at once, which the failure-path
        tests use)."""
        check(lib().sil_laplacian_plan_set_wait_bound(self._p, int(tries)), "laplacian wait bound")

    def __del__(self):
        p = getattr(self, "_p", None)
        if p is not None and p.value is not None and _native._lib is not None:
            _native._lib.sil_laplacian_plan_destroy(p)
            self._p = None


def make_staged_laplacian(geometry, out_like, inp_like, k, mode="fused", **kw):
    return StagedLaplacian(geometry, out_like, inp_like, k, mode, **kw)


def laplacian(geometry, out, inp, k, form_dims=None, comp_axis=-1, in_front=None, out_front=None, stream=None):
    """Plan-less Hodge Laplacian (table-driven fused kernel, or the 2D 0-form kernel)."""
    fi = field_struct(inp, comp_axis, in_front)
    fo = field_struct(out, comp_axis, out_front)
    check(lib().sil_laplacian(geometry.handle, _stream(stream), _mask(form_dims, fi.ndims), k, ctypes.byref(fi),
                              ctypes.byref(fo)), "laplacian")
    return out


def ncomp(n, k):
    return comb(n, k)

"""Host-side handles over the C ABI: context, basis and Hamiltonian.

Device memory is held in torch CUDA tensors and passed to the library as raw
pointers; all library work runs on the torch stream that is current when a
method is called.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

from . import _lib
from ._lib import check


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError('CUDA 不可用')
    return torch


def el_dtype(x):
    """Library dtype code of a torch tensor (EL_F32/F64/C64/C128)."""
    import torch
    dt = {torch.float32: _lib.EL_F32, torch.float64: _lib.EL_F64,
          torch.complex64: _lib.EL_C64, torch.complex128: _lib.EL_C128}.get(getattr(x, 'dtype', None))
    if dt is None:
        raise ValueError('设备向量须为 float32/float64/complex64/complex128 张量')
    return dt


def check_device_vector(ctx, x, numel, name='psi', complex_only=False):
    """Refuse, before its address reaches a kernel, any tensor that is not a
    contiguous CUDA tensor on the context's device holding exactly ``numel``
    elements of a library dtype; returns its dtype code.  The C ABI carries
    device addresses without lengths, so this is where a short vector or a
    host tensor is caught."""
    import torch
    if not isinstance(x, torch.Tensor):
        raise ValueError('%s 须为 torch 张量' % name)
    dt = el_dtype(x)
    if complex_only and dt not in (_lib.EL_C64, _lib.EL_C128):
        raise ValueError('%s must be complex64 or complex128' % name)
    if x.numel() != int(numel):
        raise ValueError('%s 元素数 %d ≠ %d（基维度 × 向量数）' % (name, x.numel(), int(numel)))
    if not x.is_contiguous():
        raise ValueError('%s must be contiguous' % name)
    if not x.is_cuda or x.device.index != ctx.device.index:
        raise ValueError('%s 须在 %s 上（实为 %s）' % (name, ctx.device, x.device))
    return dt


class Context:
    """One library context per (thread, device).  Mirrors the per-run device
    setup of matrix_free.py:177-185."""

    def __init__(self, device=0):
        torch = _torch()
        self.lib = _lib.load()
        self.device = torch.device('cuda', int(device) if not isinstance(device, torch.device)
                                   else (device.index or 0))
        h = C.c_void_p()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        rc = self.lib.el_ctx_create(self.device.index, C.c_void_p(stream), C.byref(h))
        if rc != _lib.EL_OK:
            raise RuntimeError('el_ctx_create failed (status %d): CUDA 不可用' % rc)
        self.handle = h
        self._cancel = None

    def sync_stream(self):
        torch = _torch()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        self.lib.el_ctx_set_stream(self.handle, C.c_void_p(stream))

    def set_cancel(self, flag_array):
        """flag_array: a numpy int32 array of length >= 1 polled by the library."""
        if flag_array is None:
            self._cancel = None
            self.lib.el_ctx_set_cancel(self.handle, None)
            return
        arr = np.ascontiguousarray(flag_array, dtype=np.int32)
        self._cancel = arr
        self.lib.el_ctx_set_cancel(self.handle, C.c_void_p(arr.ctypes.data))

    @property
    def launches(self) -> int:
        return int(self.lib.el_ctx_launches(self.handle))

    @property
    def copied_bytes(self):
        """(host->device, device->host) bytes copied by the library so far."""
        a = C.c_int64()
        b = C.c_int64()
        check(self.lib.el_ctx_bytes(self.handle, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def call(self, name, *args):
        self.sync_stream()
        rc = getattr(self.lib, name)(self.handle, *args)
        check(rc, self.handle, name)

    def close(self):
        if getattr(self, 'handle', None):
            self.lib.el_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts = {}


def default_context(device=0) -> Context:
    import threading
    key = (threading.get_ident(), int(device))
    ctx = _contexts.get(key)
    if ctx is None:
        ctx = Context(device)
        _contexts[key] = ctx
    return ctx


def _edges_array(edges):
    e = np.asarray([[int(a), int(b)] for a, b in (edges or [])], dtype=np.int32).reshape(-1, 2)
    return np.ascontiguousarray(e)


class Basis:
    """Full, blockade or fixed-excitation basis (ascending codes, site 0 = MSB).

    kind='blockade' with edges follows basis.py:24-47; kind='charge' with k
    follows matrix_free.py:12-38; kind='full' is the 2^N basis."""

    def __init__(self, ctx: Context, n: int, kind='full', edges=None, k=None, max_states=None):
        self.ctx = ctx
        self.n = int(n)
        kinds = {'full': _lib.EL_BASIS_FULL, 'blockade': _lib.EL_BASIS_BLOCKADE,
                 'charge': _lib.EL_BASIS_CHARGE}
        if kind not in kinds:
            raise ValueError('unknown basis kind %r' % (kind,))
        self.kind = kind
        e = _edges_array(edges)
        self.edges = e
        h = C.c_void_p()
        ctx.call('el_basis_build', C.c_int(self.n), C.c_void_p(e.ctypes.data) if e.size else None,
                 C.c_int(len(e)), C.c_int(kinds[kind]), C.c_int(int(k or 0)),
                 C.c_int64(int(max_states) if max_states else 0), C.byref(h))
        self.handle = h
        dim = C.c_int64()
        lay = C.c_int()
        check(ctx.lib.el_basis_info(h, C.byref(dim), C.byref(lay)))
        self.dim = int(dim.value)
        self.layout = int(lay.value)

    def codes(self):
        torch = _torch()
        out = torch.empty(self.dim, dtype=torch.int64, device=self.ctx.device)
        self.ctx.call('el_basis_codes', self.handle, C.c_void_p(out.data_ptr()))
        return out

    def rank(self, codes):
        torch = _torch()
        c = torch.as_tensor(codes, dtype=torch.int64, device=self.ctx.device).contiguous()
        out = torch.empty(c.numel(), dtype=torch.int64, device=self.ctx.device)
        self.ctx.call('el_basis_rank', self.handle, C.c_void_p(c.data_ptr()),
                      C.c_int64(c.numel()), C.c_void_p(out.data_ptr()))
        return out

    def close(self):
        if getattr(self, 'handle', None):
            self.ctx.lib.el_basis_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Hamiltonian:
    """H = sum delta_i n_i + (Omega_i/2) sigma^x_i + sum V_ij n_i n_j on a basis,
    plus optional exchange channels ``exchange`` = [(i, j, J, A), ...]
    (I2 hopping J and I3 pair creation A, channels.py:119-131)."""

    def __init__(self, ctx: Context, basis: Basis, omega, delta, pairs, exchange=None):
        self.ctx = ctx
        self.basis = basis
        n = basis.n
        om = np.asarray(omega, complex).reshape(-1)
        de = np.asarray(delta, float).reshape(-1)
        if om.shape != (n,) or de.shape != (n,) or not np.isfinite(om).all() or not np.isfinite(de).all():
            raise ValueError('Om/delta 须为有限、长度为 N 的数组')
        pi = np.ascontiguousarray([int(p[0]) for p in pairs], dtype=np.int32)
        pj = np.ascontiguousarray([int(p[1]) for p in pairs], dtype=np.int32)
        V = np.ascontiguousarray([float(p[2]) for p in pairs], dtype=np.float64)
        ore = np.ascontiguousarray(om.real, dtype=np.float64)
        oim = np.ascontiguousarray(om.imag, dtype=np.float64)
        de = np.ascontiguousarray(de, dtype=np.float64)
        h = C.c_void_p()
        ctx.call('el_ham_create', basis.handle, _lib.dptr(ore), _lib.dptr(oim), _lib.dptr(de),
                 C.c_int(len(V)), C.c_void_p(pi.ctypes.data) if len(V) else None,
                 C.c_void_p(pj.ctypes.data) if len(V) else None,
                 _lib.dptr(V) if len(V) else None, C.byref(h))
        self.handle = h
        self.n = n
        self.dim = basis.dim
        self.omega = om
        self.delta = de
        self.pairs = list(zip(pi.tolist(), pj.tolist(), V.tolist()))
        self.gamma = np.zeros(n)
        self.exchange = []
        if exchange:
            self.set_exchange(exchange)

    def set_exchange(self, exchange):
        """Replace the exchange channels: [(i, j, J, A), ...] (complex J, A)."""
        ex = [(int(e[0]), int(e[1]), complex(e[2]), complex(e[3])) for e in (exchange or [])]
        pi = np.ascontiguousarray([e[0] for e in ex], dtype=np.int32)
        pj = np.ascontiguousarray([e[1] for e in ex], dtype=np.int32)
        amp = [np.ascontiguousarray([f(e) for e in ex], dtype=np.float64)
               for f in (lambda e: e[2].real, lambda e: e[2].imag, lambda e: e[3].real, lambda e: e[3].imag)]
        k = len(ex)
        self.ctx.call('el_ham_set_exchange', self.handle, C.c_int(k),
                      C.c_void_p(pi.ctypes.data) if k else None, C.c_void_p(pj.ctypes.data) if k else None,
                      *[_lib.dptr(a) if k else None for a in amp])
        self.exchange = ex

    def set_loss(self, gamma):
        """Loss rates per site (gamma_mhz): non-Hermitian diagonal
        -0.5 i gamma 1e-3 / CONV per excited site; None or zeros clear it."""
        g = np.zeros(self.n) if gamma is None else np.asarray(gamma, float).reshape(-1)
        if g.shape != (self.n,) or not np.isfinite(g).all():
            raise ValueError('gamma 须为有限、长度为 N 的数组')
        g = np.ascontiguousarray(g, dtype=np.float64)
        self.ctx.call('el_ham_set_loss', self.handle, _lib.dptr(g))
        self.gamma = g

    @property
    def lossy(self) -> bool:
        return bool(np.any(getattr(self, 'gamma', np.zeros(1)) != 0))

    @property
    def complex_drive(self) -> bool:
        """H is complex: a complex Omega, J or A, or a loss diagonal."""
        return bool(np.any(self.omega.imag != 0)) or self.lossy or any(
            e[2].imag != 0 or e[3].imag != 0 for e in getattr(self, 'exchange', ()))

    def set_drive(self, omega, delta):
        om = np.asarray(omega, complex).reshape(-1)
        de = np.asarray(delta, float).reshape(-1)
        if om.shape != (self.n,) or de.shape != (self.n,):
            raise ValueError('Om/delta 须为有限、长度为 N 的数组')
        ore = np.ascontiguousarray(om.real, dtype=np.float64)
        oim = np.ascontiguousarray(om.imag, dtype=np.float64)
        de = np.ascontiguousarray(de, dtype=np.float64)
        self.ctx.call('el_ham_set_drive', self.handle, _lib.dptr(ore), _lib.dptr(oim), _lib.dptr(de))
        self.omega = om
        self.delta = de

    def diag(self, dtype='float64'):
        torch = _torch()
        td = torch.float64 if dtype == 'float64' else torch.float32
        out = torch.empty(self.dim, dtype=td, device=self.ctx.device)
        self.ctx.call('el_ham_diag', self.handle, C.c_int(_lib.DTYPES[dtype]), C.c_void_p(out.data_ptr()))
        return out

    def hv(self, x):
        """y = H x for x of shape (dim,) or (dim, nvec) on the device."""
        import torch
        if not isinstance(x, torch.Tensor) or x.dim() not in (1, 2):
            raise ValueError('x 须为 (dim,) 或 (dim, nvec) 的 torch 张量')
        nvec = 1 if x.dim() == 1 else int(x.shape[1])
        if x.shape[0] != self.dim:
            raise ValueError('通道内核：向量长度 %d ≠ 基维度 %d' % (x.shape[0], self.dim))
        x = x.contiguous()
        dt = check_device_vector(self.ctx, x, self.dim * nvec, name='x')
        y = torch.empty_like(x)
        self.ctx.call('el_hv', self.handle, C.c_int(dt), C.c_int(nvec),
                      C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))
        return y

    def close(self):
        if getattr(self, 'handle', None):
            self.ctx.lib.el_ham_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

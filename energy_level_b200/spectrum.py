"""Source-state Lanczos spectra on the B200 path.

S(w) = -1/pi Im <phi|(w + shift + i eta - H)^{-1}|phi> for one source state
phi (typically O|0>), as in the reference's spectrum.py:

- ``lanczos`` runs the tridiagonalisation on the device (el_lanczos_tridiag:
  three-term recurrence, FP64 alpha/beta, full reorthogonalisation twice per
  step) and returns the keys of spectrum.py:34-103 (alphas, betas, norm2, n,
  converged, ortho_loss, reortho, note, seconds);
- ``quadrature`` and ``lorentz_spectrum`` are the host post-processing of
  spectrum.py:106-135 (Ritz nodes / weights sum to |phi|^2, continued
  fraction);
- ``source_spectrum`` is spectrum.py:138-180 with the same result dict;
- ``resolve_source`` builds phi from a ``system['source']`` mapping as
  eq_route.py:160-257 does (vector, psi0/state, diagonal, site_weights with
  subtract_mean, sparse, full_sparse).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .core import _torch

__all__ = ['lanczos', 'quadrature', 'lorentz_spectrum', 'source_spectrum', 'resolve_source']


def _device_vector(ham, phi, dtype):
    torch = _torch()
    td = getattr(torch, dtype)
    if hasattr(phi, 'data_ptr'):
        v = phi.to(device=ham.ctx.device, dtype=td).contiguous()
    else:
        arr = np.asarray(phi).reshape(-1)
        if not dtype.startswith('complex') and np.iscomplexobj(arr) and np.any(arr.imag != 0):
            raise ValueError('complex source state needs a complex dtype')
        if not dtype.startswith('complex'):
            arr = arr.real
        v = torch.as_tensor(np.ascontiguousarray(arr), dtype=td, device=ham.ctx.device)
    if v.numel() != ham.dim:
        raise ValueError('源态长度 %d ≠ 当前基维度 %d' % (v.numel(), ham.dim))
    return v


def lanczos(ham, phi, n_krylov=200, *, reortho=True, memory_budget_mb=512.0, dtype=None):
    """Device Lanczos from phi; same result keys as spectrum.py:34-103."""
    if dtype is None:
        if hasattr(phi, 'data_ptr'):
            cplx = ham.complex_drive or phi.is_complex()
        else:
            cplx = ham.complex_drive or np.iscomplexobj(np.asarray(phi))
        dtype = 'complex128' if cplx else 'float64'
    if dtype not in ('float32', 'float64', 'complex64', 'complex128'):
        raise ValueError('dtype 必须为 float32/float64/complex64/complex128')
    k = int(n_krylov)
    if k < 1:
        raise ValueError('n_krylov 须为正')
    dim = ham.dim
    if dim == 0:
        raise ValueError('源态为空')
    k = min(k, dim)
    note = ''
    if reortho and memory_budget_mb is not None:
        need = dim * k * 16 * 2
        if need > float(memory_budget_mb) * 1024 ** 2:
            reortho = False
            note = ('全重正交工作区约 %.0f MiB > 预算 %.0f MiB ⇒ 降级为不重正交'
                    % (need / 2 ** 20, float(memory_budget_mb)))
    v = _device_vector(ham, phi, dtype)
    al = np.zeros(k)
    be = np.zeros(max(k - 1, 1))
    n = C.c_int()
    norm2 = C.c_double()
    ol = C.c_double()
    conv = C.c_int()
    t0 = time.perf_counter()
    ham.ctx.call('el_lanczos_tridiag', ham.handle, C.c_int(_lib.DTYPES[dtype]), C.c_void_p(v.data_ptr()),
                 C.c_int(k), C.c_int(1 if reortho else 0), _lib.dptr(al), _lib.dptr(be), C.byref(n),
                 C.byref(norm2), C.byref(ol), C.byref(conv))
    nn = int(n.value)
    return {'alphas': al[:nn].copy(), 'betas': be[:max(nn - 1, 0)].copy(),
            'norm2': float(norm2.value), 'n': nn, 'converged': bool(conv.value),
            'ortho_loss': float(ol.value), 'reortho': bool(reortho), 'note': note,
            'seconds': round(time.perf_counter() - t0, 3)}


def quadrature(alphas, betas, norm2, shift=0.0):
    """Ritz nodes (relative to shift) and weights norm2 |u_0|^2 (spectrum.py:106-121)."""
    alphas = np.asarray(alphas, float)
    betas = np.asarray(betas, float)
    if alphas.size == 0:
        return np.zeros(0), np.zeros(0)
    if betas.size:
        evals, evecs = np.linalg.eigh(np.diag(alphas) + np.diag(betas, 1) + np.diag(betas, -1))
    else:
        evals, evecs = alphas.copy(), np.ones((1, 1))
    weights = float(norm2) * np.abs(evecs[0, :]) ** 2
    return evals - float(shift), weights


def lorentz_spectrum(alphas, betas, norm2, omega, eta, shift=0.0):
    """Continued fraction for -1/pi Im <phi|(w + shift + i eta - H)^{-1}|phi>
    (spectrum.py:124-135)."""
    alphas = np.asarray(alphas, float)
    betas = np.asarray(betas, float)
    omega = np.asarray(omega, float)
    if alphas.size == 0:
        return np.zeros_like(omega)
    z = omega + float(shift) + 1j * float(eta)
    g = z - alphas[-1]
    for j in range(alphas.size - 2, -1, -1):
        g = z - alphas[j] - (betas[j] ** 2) / g
    return -float(norm2) * np.imag(1.0 / g) / np.pi


def source_spectrum(ham, phi, *, shift=0.0, eta=0.05, n_krylov=None, omega_min=None, omega_max=None,
                    n_omega=800, reortho=True, memory_budget_mb=512.0, dtype=None):
    """Lanczos -> quadrature + broadened spectrum + diagnostics
    (spectrum.py:138-180, same result dict)."""
    k = int(n_krylov) if n_krylov else min(ham.dim, 200)
    lz = lanczos(ham, phi, k, reortho=reortho, memory_budget_mb=memory_budget_mb, dtype=dtype)
    nodes, weights = quadrature(lz['alphas'], lz['betas'], lz['norm2'], shift)
    if omega_min is None or omega_max is None:
        if nodes.size:
            lo, hi = float(nodes.min()), float(nodes.max())
        else:
            lo, hi = 0.0, 1.0
        pad = max(0.05 * (hi - lo), 4.0 * float(eta))
        omega_min = lo - pad if omega_min is None else float(omega_min)
        omega_max = hi + pad if omega_max is None else float(omega_max)
    omega = np.linspace(float(omega_min), float(omega_max), int(n_omega))
    eta = float(eta)
    spectral = lorentz_spectrum(lz['alphas'], lz['betas'], lz['norm2'], omega, eta, shift)
    integral = float(np.trapezoid(spectral, omega)) if omega.size > 1 else 0.0
    return {
        'omega': omega, 'spectral': spectral,
        'evals': nodes, 'spectrum_weights': weights,
        'source_norm': float(lz['norm2']), 'eta': eta, 'shift': float(shift),
        'krylov': {'n': lz['n'], 'n_requested': k, 'converged': lz['converged'],
                   'ortho_loss': lz['ortho_loss'], 'reortho': lz['reortho'],
                   'note': lz['note'], 'seconds': lz['seconds']},
        'error_report': {'source_norm': float(lz['norm2']),
                         'spectral_integral': integral,
                         'integral_ratio': (integral / lz['norm2']) if lz['norm2'] else None,
                         'eta_mhz': eta,
                         'krylov_n': lz['n'],
                         'ortho_loss': lz['ortho_loss'],
                         'reortho': lz['reortho']},
    }


def resolve_source(source, psi0, n_sites, codes=None):
    """phi and diagnostics from a source mapping and |0> on the basis `codes`
    (None = full 2^N basis); the kinds and checks of eq_route.py:160-257."""
    import scipy.sparse as sp
    if not isinstance(source, dict):
        raise ValueError('manybody.source 须是映射（kind=vector/diagonal/sparse/full_sparse）')
    kind = str(source.get('kind') or '')
    n_sites = int(n_sites)
    dim = len(codes) if codes is not None else (1 << n_sites)
    psi = np.asarray(psi0, dtype=complex).reshape(-1)
    if psi.size != dim:
        raise ValueError('初态维度 %d 与当前基维度 %d 不一致' % (psi.size, dim))

    def _coo(block):
        rows = np.asarray(block.get('rows', ()), dtype=int).ravel()
        cols = np.asarray(block.get('cols', ()), dtype=int).ravel()
        vals = np.asarray(block.get('values', ()), dtype=complex).ravel()
        if not (len(rows) == len(cols) == len(vals)):
            raise ValueError('source 的 rows/cols/values 长度不一致')
        if len(rows) == 0:
            raise ValueError('source 的稀疏结构为空')
        size = int(block.get('dim') or (max(rows.max(), cols.max()) + 1))
        return sp.coo_matrix((vals, (rows, cols)), shape=(size, size)).tocsr()

    if kind == 'vector':
        v = np.asarray(source.get('values', ()), dtype=complex).reshape(-1)
        if v.size != dim:
            raise ValueError('source vector 长度 %d ≠ 当前基维度 %d' % (v.size, dim))
        return v, {'kind': kind, 'dim': dim}
    if kind in ('psi0', 'state'):
        return psi.copy(), {'kind': 'psi0', 'dim': dim}
    if kind == 'diagonal':
        d = np.asarray(source.get('values', ()), dtype=complex).reshape(-1)
        if d.size != dim:
            raise ValueError('source diagonal 长度 %d ≠ 当前基维度 %d' % (d.size, dim))
        return d * psi, {'kind': kind, 'dim': dim}
    if kind in ('site_weights', 'weights'):
        w = np.asarray(source.get('weights', ()), dtype=float).reshape(-1)
        if w.size != n_sites:
            raise ValueError('source site_weights 长度 %d ≠ 原子数 %d' % (w.size, n_sites))
        cc = np.arange(1 << n_sites, dtype=np.int64) if codes is None else np.asarray(codes, np.int64)
        bits = np.asarray([((cc >> (n_sites - 1 - i)) & 1) for i in range(n_sites)], dtype=float)
        d = (bits.T @ w).astype(complex)
        info = {'kind': 'site_weights', 'dim': dim, 'sum_weights': float(w.sum()),
                'weight_sq': float((w * w).sum())}
        if source.get('subtract_mean'):
            mean = complex(np.vdot(psi, d * psi))
            d = d - mean
            info['subtracted_mean'] = mean.real
        return d * psi, info
    if kind == 'sparse':
        O = _coo(source)
        if O.shape != (dim, dim):
            raise ValueError('source sparse 形状 %r ≠ 当前基 (%d,%d)' % (O.shape, dim, dim))
        return O @ psi, {'kind': kind, 'dim': dim}
    if kind == 'full_sparse':
        full = 1 << n_sites
        if full > (1 << 16):
            raise ValueError('full_sparse 需要 2^N ≤ 65536；大系统请给当前基（扇区）的 source')
        O = _coo(source)
        if O.shape != (full, full):
            raise ValueError('source full_sparse 形状 %r ≠ (%d,%d)' % (O.shape, full, full))
        if codes is None:
            return O @ psi, {'kind': kind, 'dim': full}
        expand = np.zeros(full, dtype=complex)
        expand[np.asarray(codes, int)] = psi
        phi_full = O @ expand
        phi = phi_full[np.asarray(codes, int)]
        norm_full = float(np.linalg.norm(phi_full))
        leak = 0.0 if norm_full == 0 else 1.0 - float(np.linalg.norm(phi)) ** 2 / norm_full ** 2
        return phi, {'kind': kind, 'dim': dim, 'projected_leak': max(0.0, leak)}
    raise ValueError('未知 source.kind=%r（可选 vector/psi0/diagonal/sparse/full_sparse）' % kind)

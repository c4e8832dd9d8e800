"""Source-state Lanczos spectra on the B200 path.

S(w) = -1/pi Im <phi|(w + shift + i eta - H)^{-1}|phi> for one source state
phi (typically O|0>), as in the reference's spectrum.py:

- ``lanczos`` runs the tridiagonalisation on the device (el_lanczos_tridiag:
  three-term recurrence, FP64 alpha/beta, full reorthogonalisation twice per
  step) and returns the keys of spectrum.py:34-103 (alphas, betas, norm2, n,
  converged, ortho_loss, reortho, note, seconds);
- ``quadrature`` and ``lorentz_spectrum`` give the outputs of the host
  post-processing of spectrum.py:106-135: Gauss nodes / weights of phi's
  spectral measure (summing to |phi|^2) from a tridiagonal eigensolver, and
  the broadened spectrum as a Lorentzian sum over those nodes;
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
    """Gauss quadrature of phi's spectral measure (Golub-Welsch): nodes are
    the eigenvalues of the Jacobi matrix J = tridiag(betas, alphas, betas)
    less ``shift``; weights are norm2 times the squared first components of
    J's unit eigenvectors, so they sum to |phi|^2 (the outputs of
    spectrum.py:106-121).  J is handed to a symmetric tridiagonal solver
    (LAPACK stemr through scipy) and never formed as a dense matrix."""
    from scipy.linalg import eigh_tridiagonal
    a = np.asarray(alphas, float).reshape(-1)
    if a.size == 0:
        return np.zeros(0), np.zeros(0)
    b = np.asarray(betas, float).reshape(-1)[:a.size - 1]
    if a.size == 1:
        return a - float(shift), np.array([float(norm2)])
    lam, u = eigh_tridiagonal(a, b)
    return lam - float(shift), float(norm2) * u[0] ** 2


def lorentz_spectrum(alphas, betas, norm2, omega, eta, shift=0.0):
    """S(w) = -1/pi Im <phi|(w + shift + i eta - H)^{-1}|phi> in the Krylov
    model (spectrum.py:124-135).  The (0,0) element of J's resolvent is the
    Stieltjes transform of the quadrature measure, sum_k w_k / (z - x_k), so
    S is a sum of Lorentzians of half-width eta centred on the Ritz nodes --
    the value of the continued fraction, evaluated here from the eigen-
    decomposition in blocks of frequencies."""
    omega = np.asarray(omega, float)
    x, w = quadrature(alphas, betas, norm2, shift)
    eta = float(eta)
    out = np.zeros(omega.size)
    if x.size == 0 or eta == 0.0:
        return out.reshape(omega.shape)
    flat = omega.reshape(-1)
    scale = w * (eta / np.pi)
    for lo in range(0, flat.size, 4096):
        d = flat[lo:lo + 4096, None] - x[None, :]
        out[lo:lo + 4096] = (scale / (d * d + eta * eta)).sum(axis=1)
    return out.reshape(omega.shape)


def _display_window(nodes, eta, lo, hi):
    """Frequency window: any bound the caller gave, else the Ritz nodes' span
    widened on each side by the larger of 5 % of the span and four
    half-widths (the default grid of spectrum.py:155-162, so that a default
    call lands on the same frequencies)."""
    first, last = (float(nodes.min()), float(nodes.max())) if nodes.size else (0.0, 1.0)
    margin = max(0.05 * (last - first), 4.0 * float(eta))
    return (first - margin if lo is None else float(lo)), (last + margin if hi is None else float(hi))


def source_spectrum(ham, phi, *, shift=0.0, eta=0.05, n_krylov=None, omega_min=None, omega_max=None,
                    n_omega=800, reortho=True, memory_budget_mb=512.0, dtype=None):
    """Device Lanczos from phi, then the quadrature, the broadened spectrum on
    a frequency grid and diagnostics; result keys of spectrum.py:138-180
    (omega, spectral, evals, spectrum_weights, source_norm, eta, shift,
    krylov, error_report)."""
    requested = int(n_krylov) if n_krylov else min(ham.dim, 200)
    lz = lanczos(ham, phi, requested, reortho=reortho, memory_budget_mb=memory_budget_mb, dtype=dtype)
    norm2, eta = float(lz['norm2']), float(eta)
    nodes, weights = quadrature(lz['alphas'], lz['betas'], norm2, shift)
    grid = np.linspace(*_display_window(nodes, eta, omega_min, omega_max), int(n_omega))
    spectral = lorentz_spectrum(lz['alphas'], lz['betas'], norm2, grid, eta, shift)
    # the broadened weight inside the window (trapezoid rule); close to
    # |phi|^2 when the window holds the spectrum
    inside = 0.5 * float(np.sum((spectral[1:] + spectral[:-1]) * np.diff(grid))) if grid.size > 1 else 0.0
    health = {key: lz[key] for key in ('ortho_loss', 'reortho')}
    krylov = dict(health, n=lz['n'], n_requested=requested, converged=lz['converged'], note=lz['note'],
                  seconds=lz['seconds'])
    report = dict(health, source_norm=norm2, spectral_integral=inside,
                  integral_ratio=inside / norm2 if norm2 else None, eta_mhz=eta, krylov_n=lz['n'])
    return dict(omega=grid, spectral=spectral, evals=nodes, spectrum_weights=weights, source_norm=norm2,
                eta=eta, shift=float(shift), krylov=krylov, error_report=report)


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

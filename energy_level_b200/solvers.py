"""Thin wrappers of the native drivers (Lanczos, bounds, KPM, Chebyshev step).

Each function queues work on the current torch stream through the C ABI and
returns host results; device vectors are torch tensors.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

from . import _lib
from .core import Hamiltonian, _torch, check_device_vector

_TORCH_DT = {"float32": "float32", "float64": "float64", "complex64": "complex64",
             "complex128": "complex128"}
REORTH = {"none": 0, "partial": 1, "full": 2}


def _tdtype(dtype):
    torch = _torch()
    return getattr(torch, _TORCH_DT[dtype])


def bounds(ham: Hamiltonian, max_iter=300, tol=1e-12, seed=0):
    """Extremal eigenvalues (emin, emax) by FP64 Lanczos (kpm.py:82-97 role)."""
    lo = C.c_double()
    hi = C.c_double()
    ham.ctx.call('el_bounds', ham.handle, C.c_int(int(max_iter)), C.c_double(float(tol)),
                 C.c_uint64(int(seed)), C.byref(lo), C.byref(hi))
    return float(lo.value), float(hi.value)


def kpm_scale(emin, emax):
    """Centre/radius with the reference padding (kpm.py:95-96)."""
    c = 0.5 * (emin + emax)
    r = 0.5 * (emax - emin) * (1.0 + 1e-3) + 1e-12
    return c, r


def kpm_moments(ham: Hamiltonian, num, nvec, c, r, dtype="float32", chunk=32, seed=0,
                probes=None, mode="doubling", generic=False):
    """mu[0..num] of Htil = (H - c)/r from nvec Rademacher probes.

    probes: None (counter-based, from seed) or an int8/float array [nvec, dim]
    of +-1 entries (e.g. the reference's own numpy draws).  generic=True
    forces the row-parallel kernel where the tiled full-basis one applies."""
    if dtype not in ("float32", "float64"):
        raise ValueError('dtype 必须为 float32/float64')
    mu = np.zeros(int(num) + 1)
    pb = None
    if probes is not None:
        p = np.asarray(probes)
        if p.shape != (int(nvec), ham.dim):
            raise ValueError('probes must have shape (nvec, dim)')
        if not np.all(np.abs(p) == 1):
            raise ValueError('probes must be +-1')
        pb = np.ascontiguousarray(p, dtype=np.int8)
    md = {"direct": _lib.EL_KPM_DIRECT, "doubling": _lib.EL_KPM_DOUBLING}[mode]
    if generic:
        md |= _lib.EL_KPM_GENERIC_KERNEL
    ham.ctx.call('el_kpm_moments', ham.handle, C.c_int(_lib.DTYPES[dtype]), C.c_int(int(num)),
                 C.c_int(int(nvec)), C.c_int(int(chunk)), C.c_uint64(int(seed)),
                 C.c_void_p(pb.ctypes.data) if pb is not None else None, C.c_int(md),
                 C.c_double(float(c)), C.c_double(float(r)), _lib.dptr(mu))
    return mu


def lanczos_ground(ham: Hamiltonian, dtype="float64", v0=None, seed=0, max_iter=300,
                   max_restarts=8, tol=1e-9, nev=2, reorth="partial", return_vec=False):
    """Lowest eigenpairs with Ritz-residual certification.

    Returns dict(evals, residuals, iters, converged[, vec])."""
    torch = _torch()
    if ham.complex_drive and not dtype.startswith("complex"):
        dtype = "complex128" if dtype == "float64" else "complex64"
    td = _tdtype(dtype)
    nev = min(int(nev), ham.dim)
    ev = np.zeros(max(nev, 1))
    res = np.zeros(max(nev, 1))
    it = C.c_int()
    conv = C.c_int()
    v0p = None
    if v0 is not None:
        v0t = torch.as_tensor(v0, dtype=td, device=ham.ctx.device).contiguous()
        if v0t.numel() != ham.dim:
            raise ValueError('v0 length must equal the basis dimension')
        check_device_vector(ham.ctx, v0t, ham.dim, name='v0')
        v0p = C.c_void_p(v0t.data_ptr())
    vec = torch.empty(ham.dim, dtype=td, device=ham.ctx.device) if return_vec else None
    ham.ctx.call('el_lanczos_ground', ham.handle, C.c_int(_lib.DTYPES[dtype]), v0p,
                 C.c_uint64(int(seed)), C.c_int(int(max_iter)), C.c_int(int(max_restarts)),
                 C.c_double(float(tol)), C.c_int(nev), C.c_int(REORTH[reorth]),
                 _lib.dptr(ev), _lib.dptr(res), C.byref(it), C.byref(conv),
                 C.c_void_p(vec.data_ptr()) if vec is not None else None)
    out = dict(evals=ev[:nev], residuals=res[:nev], iters=int(it.value), converged=bool(conv.value),
               dtype=dtype)
    if vec is not None:
        out["vec"] = vec
    return out


def cheb_step(ham: Hamiltonian, psi, tau_ns, tol=1e-12):
    """psi <- exp(-i CONV H tau) psi in place (complex64/complex128 tensor)."""
    dt = check_device_vector(ham.ctx, psi, ham.dim, complex_only=True)
    nt = C.c_int()
    ham.ctx.call('el_cheb_step', ham.handle, C.c_int(dt), C.c_void_p(psi.data_ptr()),
                 C.c_double(float(tau_ns)), C.c_double(float(tol)), C.byref(nt))
    return int(nt.value)


def observables(ham: Hamiltonian, psi):
    """(<n_i> per site, squared norm) of a device state."""
    psi_c = psi.contiguous() if hasattr(psi, 'contiguous') else psi   # kept alive across the call
    dt = check_device_vector(ham.ctx, psi_c, ham.dim)
    ns = np.zeros(ham.n)
    nrm = C.c_double()
    ham.ctx.call('el_observables', ham.handle, C.c_int(dt), C.c_void_p(psi_c.data_ptr()),
                 _lib.dptr(ns), C.byref(nrm))
    return ns, float(nrm.value)


def taylor_step(ham: Hamiltonian, psi, tau_ns, tol=1e-13):
    """psi <- exp(-i CONV H tau) psi for any H (loss diagonal included):
    scaled Taylor polynomial (el_taylor_step); returns the H applications."""
    dt = check_device_vector(ham.ctx, psi, ham.dim, complex_only=True)
    nt = C.c_int()
    ham.ctx.call('el_taylor_step', ham.handle, C.c_int(dt), C.c_void_p(psi.data_ptr()), C.c_double(float(tau_ns)),
                 C.c_double(float(tol)), C.byref(nt))
    return int(nt.value)


def spin_observables(ham: Hamiltonian, psi, pairs=()):
    """Device spin observables of a state (el_spin_observables).

    Returns dict(n, norm, sm, nn, xy): <n_i>, squared norm, <sigma-_i>
    (complex) per site, and for each (i, j) of ``pairs`` <n_i n_j> and
    <sigma+_i sigma-_j> (complex)."""
    psi = psi.contiguous() if hasattr(psi, 'contiguous') else psi
    dt = check_device_vector(ham.ctx, psi, ham.dim)
    n = ham.n
    pr = np.asarray(list(pairs), dtype=np.int32).reshape(-1, 2)
    pi = np.ascontiguousarray(pr[:, 0])
    pj = np.ascontiguousarray(pr[:, 1])
    k = len(pr)
    ns = np.zeros(n)
    sm = np.zeros(2 * n)
    nn = np.zeros(max(k, 1))
    xy = np.zeros(2 * max(k, 1))
    nrm = C.c_double()
    ham.ctx.call('el_spin_observables', ham.handle, C.c_int(dt), C.c_void_p(psi.data_ptr()), C.c_int(k),
                 C.c_void_p(pi.ctypes.data) if k else None, C.c_void_p(pj.ctypes.data) if k else None,
                 _lib.dptr(ns), C.byref(nrm), _lib.dptr(sm), _lib.dptr(nn) if k else None,
                 _lib.dptr(xy) if k else None)
    return dict(n=ns, norm=float(nrm.value), sm=sm[0::2] + 1j * sm[1::2],
                nn=nn[:k], xy=xy[0:2 * k:2] + 1j * xy[1:2 * k:2])


def pauli_expect(ham: Hamiltonian, psi, specs):
    """<psi|P|psi> (complex) of each Pauli string in ``specs``
    ([{'label', 'terms': [(site, axis), ...]}], axes 'x'/'y'/'z'), on the device
    (el_pauli_expect)."""
    psi = psi.contiguous() if hasattr(psi, 'contiguous') else psi
    dt = check_device_vector(ham.ctx, psi, ham.dim)
    specs = list(specs or [])
    if not specs:
        return np.zeros(0, complex)
    offs, sites, axes = [0], [], []
    for sp in specs:
        for site, ax in sp['terms']:
            sites.append(int(site))
            axes.append(str(ax))
        offs.append(len(sites))
    offs = np.ascontiguousarray(offs, dtype=np.int32)
    sites = np.ascontiguousarray(sites, dtype=np.int32)
    out = np.zeros(2 * len(specs))
    ham.ctx.call('el_pauli_expect', ham.handle, C.c_int(dt), C.c_void_p(psi.data_ptr()), C.c_int(len(specs)),
                 C.c_void_p(offs.ctypes.data), C.c_void_p(sites.ctypes.data),
                 ''.join(axes).encode('ascii'), _lib.dptr(out))
    return out[0::2] + 1j * out[1::2]


def observables_noalloc(ham: Hamiltonian, psi):
    """observables() through el_observables_noalloc: no device allocation,
    static scratch shared per device (at most 40 sites; calls on one device
    must not overlap in time)."""
    dt = check_device_vector(ham.ctx, psi, ham.dim)   # contiguous: no copy is made
    ns = np.zeros(ham.n)
    nrm = C.c_double()
    ham.ctx.call('el_observables_noalloc', ham.handle, C.c_int(dt), C.c_void_p(psi.data_ptr()),
                 _lib.dptr(ns), C.byref(nrm))
    return ns, float(nrm.value)

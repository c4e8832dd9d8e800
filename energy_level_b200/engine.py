"""Exact quench / ramp evolution on the B200 path (Chebyshev propagator).

``evolve_manybody`` takes the reference engine's arguments
(engine_ed.py:154-161) and returns the same result contract
(engine_ed.py:348-372): t, pops, states, method, backend, pops_atom, S, corr,
loss, norms, basis_probabilities, basis_states, basis, error_report, diag,
observables[, psi_amp].  Propagation follows the segment rule of
engine_ed.py:130-147 exactly: every output interval is split at the drive
boundaries (runtime.py:56-60), the drive of each piece is resolved at its
midpoint with the 'left' or 'midpoint' rule (runtime.py:90-114), and each
piece is one exp(-i CONV H dt) applied by el_cheb_step instead of
expm_multiply.  Static drives (no segments) are one piece per output
interval.  Cooperative cancellation polls progress_arr[1] between pieces
(runtime.py:12-14).
"""
from __future__ import annotations

import numpy as np

from . import model, solvers
from .state import state_vector

CONV = 2 * np.pi * 1e-3


def time_grid(t):
    t = np.asarray(t, float)
    if t.ndim != 1 or len(t) < 2 or not np.isfinite(t).all() or np.any(np.diff(t) < 0):
        raise ValueError('t_grid 必须包含至少两个有限、单调不减的时间点')
    return t


def check_cancel(progress_arr):
    if progress_arr is not None and float(progress_arr[1]) != 0:
        raise RuntimeError('用户取消')


def segment_intervals(a, b, segments):
    """Split [a, b] at every drive boundary inside it (runtime.py:56-60)."""
    bounds = [float(a)] + sorted({float(s['t0']) for s in segments or []
                                  if a < float(s['t0']) < b}) + [float(b)]
    return list(zip(bounds[:-1], bounds[1:]))


def _segment_arrays(segment, n):
    om = np.asarray(segment.get('Om', np.zeros(n)), float).reshape(-1)
    ph = np.asarray(segment.get('phase', np.zeros(n)), float).reshape(-1)
    de = np.asarray(segment.get('delta', np.zeros(n)), float).reshape(-1)
    if om.size != n or ph.size != n or de.size != n:
        raise ValueError('segment_drive: 每段的 Om/phase/delta 长度必须等于 n')
    return om * np.exp(1j * ph), de


def segment_drive(t, segments, n, interp='left'):
    """Drive in force at time t (runtime.py:90-114)."""
    if not segments:
        return None
    if interp not in ('left', 'midpoint'):
        raise ValueError('drive_interp 须为 left/midpoint，得到 %r' % (interp,))
    ordered = sorted(segments, key=lambda s: float(s['t0']))
    idx = 0
    for k, s in enumerate(ordered):
        if float(s['t0']) <= t:
            idx = k
    om, de = _segment_arrays(ordered[idx], n)
    if interp == 'midpoint' and idx < len(ordered) - 1:
        om2, de2 = _segment_arrays(ordered[idx + 1], n)
        om, de = 0.5 * (om + om2), 0.5 * (de + de2)
    return om, de


def _entropy_mid(psi, codes, n, cut):
    """Half-chain von Neumann entropy (nat) for n <= 20 (else None)."""
    if n > 20:
        return None
    full = np.zeros(1 << n, complex)
    if codes is None:
        full[:] = psi
    else:
        full[codes] = psi
    nrm = np.linalg.norm(full)
    if nrm == 0:
        return None
    s = np.linalg.svd((full / nrm).reshape(1 << cut, 1 << (n - cut)), compute_uv=False)
    p = s * s
    p = p[p > 1e-300]
    return float(-np.sum(p * np.log(p)))


def evolve_manybody(calib, psi0=None, t_grid=None, Om=None, delta=None, gamma=None, terms=None,
                    segments=None, progress_arr=None, log=None, want_corr=True, want_entropy=True,
                    max_dim=None, entropy_cut=None, record_psi=False, diag=False, plan=None,
                    want_observables=True, memory_budget_mb=None, drive_interp='left',
                    dtype='complex128', tol=None, device='cuda', **unused):
    """Many-body evolution on the GPU; see the module docstring for the contract."""
    import torch
    log = log or (lambda *a: None)
    if progress_arr is None:
        progress_arr = np.zeros(2)
    if dtype not in ('complex64', 'complex128'):
        raise ValueError('dtype 必须为 complex64/complex128')
    atoms = (calib or {}).get('atoms') or []
    n = len(atoms)
    if n == 0:
        raise ValueError('多体演化：calib 没有原子（先 assemble.calibrate）')
    projected = plan is not None and plan.get('projected')
    if projected:
        Om = plan.get('Om') if Om is None else Om
        delta = plan.get('delta') if delta is None else delta
        gamma = plan.get('gamma') if gamma is None else gamma
        terms = plan.get('terms') if terms is None else terms
    t = time_grid(t_grid)
    check_cancel(progress_arr)
    ctx, basis, ham, perm = model.build(calib, Om, delta, gamma, terms, plan=plan, device=device)
    dim = basis.dim
    if max_dim is not None and dim > int(max_dim):
        raise ValueError('多体 ED 有效维度 %d 超上限 %d；请调整系统或后端' % (dim, int(max_dim)))
    es = 16 if dtype == 'complex128' else 8
    need = dim * es * 5 + len(t) * n * 8 * 4
    if memory_budget_mb is not None and need > float(memory_budget_mb) * 1024 ** 2:
        raise ValueError('ED 基空间、观测量和传播向量 预计至少 %.2f MiB，超过预算 %.2f MiB'
                         % (need / 1024 ** 2, float(memory_budget_mb)))
    if segments:
        for s in segments:
            g = np.asarray(s.get('gamma', np.zeros(n)), float)
            if np.any(g != 0):
                raise model.ConfigConflict('b200-cheb needs gamma = 0', keys=('manybody.gamma_mhz',))
    codes = basis.codes().cpu().numpy() if projected else None
    if isinstance(psi0, str) and psi0 == 'ground':
        raise ValueError('ground 初态请先由 b200_lanczos_ground_state 准备')
    psi0v = state_vector(psi0, n, codes)
    tol = float(tol if tol is not None else (1e-13 if dtype == 'complex128' else 1e-7))
    cut = int(entropy_cut if entropy_cut is not None else max(1, n // 2))
    if want_entropy and n >= 2 and not (1 <= cut <= n - 1):
        raise ValueError('多体：entropy_cut=%d 越界（n_atoms=%d 时须 ∈[1,%d]）' % (cut, n, n - 1))
    tdt = getattr(torch, dtype)
    psi = torch.as_tensor(psi0v, dtype=tdt, device=ctx.device).contiguous()
    n_t = len(t)
    pops_atom = np.zeros((n_t, n))
    norms = np.zeros(n_t)
    S_mid = np.full(n_t, np.nan) if want_entropy else None
    terms_used = 0
    pieces = 0

    def reduce(k):
        ns, nrm = solvers.observables(ham, psi)
        pops_atom[k] = ns
        norms[k] = nrm
        if want_entropy and n >= 2 and dim <= (1 << 20):
            S_mid[k] = np.nan if (v := _entropy_mid(psi.cpu().numpy(), codes, n, cut)) is None else v

    base_om = np.zeros(n, complex) if Om is None else np.asarray(Om, complex)
    base_de = np.zeros(n) if delta is None else np.asarray(delta, float)
    reduce(0)
    current = None
    for k in range(1, n_t):
        for a, b in (segment_intervals(t[k - 1], t[k], segments) if segments else [(t[k - 1], t[k])]):
            check_cancel(progress_arr)
            if segments:
                om, de = segment_drive(0.5 * (a + b), segments, n, interp=drive_interp)
            else:
                om, de = base_om, base_de
            key = (tuple(np.round(om, 15)), tuple(np.round(de, 15)))
            if key != current:
                ham.set_drive(om, de)
                current = key
            if b > a:
                terms_used += solvers.cheb_step(ham, psi, b - a, tol=tol)
                pieces += 1
        reduce(k)
        progress_arr[0] = (k + 1) / n_t
    final = psi.cpu().numpy().astype(np.complex128)
    corr = None
    if want_corr:
        cc = codes if codes is not None else np.arange(dim, dtype=np.int64)
        if dim <= (1 << 24):
            p = np.abs(final) ** 2
            bits = np.asarray([((cc >> (n - 1 - i)) & 1) for i in range(n)], dtype=np.float64)
            ni = bits @ p
            corr = (bits * p) @ bits.T - np.outer(ni, ni)
    loss = 1.0 - norms
    backend = 'b200-cheb-plan-%s' % plan['constraint']['kind'] if projected else 'b200-cheb'
    states = [{'label': 'atom%d' % a.get('id', i), 'atom_id': a.get('id', i)} for i, a in enumerate(atoms)]
    out = dict(
        t=t, pops=pops_atom, states=states, method='manybody', backend=backend,
        pops_atom=pops_atom, S=S_mid, corr=corr, loss=loss, norms=norms,
        basis_probabilities=None, basis_states=(codes if projected else None),
        basis=dict(kind='projected' if projected else 'full', bit_order='site0-msb',
                   n_atoms=n, dim=dim, full_dim=1 << n),
        error_report=dict(backend=backend, solver='chebyshev', dim=dim, n_atoms=n, n_t=n_t,
                          hermitian=True, used_sectors=False, full_pops=False,
                          projected=bool(projected), entropy_cut=(cut if want_entropy else None),
                          entropy_note=(None if dim <= (1 << 20) and n <= 20 else
                                        'entropy computed only for n <= 20'),
                          max_norm_dev=float(np.max(np.abs(norms - 1.0))),
                          chebyshev_terms=int(terms_used), pieces=int(pieces), tol=tol, dtype=dtype),
        diag=({'dim': dim, 'n_atoms': n, 'backend': backend, 'launches': ctx.launches} if diag else None),
        observables=None)
    if record_psi:
        out['psi_amp'] = final
    return out

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

Observables at every output time (engine_ed.py:259-281) are device sums
(el_spin_observables, el_pauli_expect): <n_i>, norm, sx/sy/sz/sp/sm/phase,
the selected link correlations and the Pauli strings; at the last time also
<n_i n_j> for ``corr`` and <sigma+_i sigma-_j> for ``xy_corr``.  The
bipartite entropy is the SVD (cuSOLVER through torch) of the state's Schmidt
matrix built on the device: the reshaped state on the full basis, the
occupied prefix x suffix matrix on a restricted basis (at most 2^20 entries,
else NaN, as observables.py:89-114).  Joint basis probabilities are kept
when dim <= fullpop_max (65536), as the reference does.
"""
from __future__ import annotations

import bisect

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


class SegmentTable:
    """segment_drive over one fixed segment list: the segments are sorted
    once and each one's arrays built once, so resolving the drive of many
    intervals costs a bisection each (same values as segment_drive).  The
    returned arrays are shared: callers copy before changing them."""

    def __init__(self, segments, n):
        self.ordered = sorted(segments, key=lambda s: float(s['t0']))
        self.t0 = [float(s['t0']) for s in self.ordered]
        self.n = n
        self._arrays = {}

    def _at(self, i):
        a = self._arrays.get(i)
        if a is None:
            a = self._arrays[i] = _segment_arrays(self.ordered[i], self.n)
        return a

    def drive(self, t, interp='left'):
        if interp not in ('left', 'midpoint'):
            raise ValueError('drive_interp 须为 left/midpoint，得到 %r' % (interp,))
        # the last segment with t0 <= t in t0 order (the first one if none)
        idx = max(bisect.bisect_right(self.t0, t) - 1, 0)
        om, de = self._at(idx)
        if interp == 'midpoint' and idx < len(self.ordered) - 1:
            om2, de2 = self._at(idx + 1)
            om, de = 0.5 * (om + om2), 0.5 * (de + de2)
        return om, de


SCHMIDT_MAX_ENTRIES = 1 << 20
FULLPOP_MAX = 65536


class _Schmidt:
    """Device Schmidt matrix of a state for the cut after `cut` sites."""

    def __init__(self, basis, n, cut, device):
        import torch
        self.n, self.cut = n, cut
        self.restricted = basis.kind != 'full'
        self.ok = True
        if not self.restricted:
            self.shape = (1 << cut, 1 << (n - cut))
            self.ok = n <= 20
            return
        codes = basis.codes()
        _, li = torch.unique(codes >> (n - cut), return_inverse=True)
        _, ri = torch.unique(codes & ((1 << (n - cut)) - 1), return_inverse=True)
        self.shape = (int(li.max()) + 1, int(ri.max()) + 1)
        self.ok = self.shape[0] * self.shape[1] <= SCHMIDT_MAX_ENTRIES
        self.flat = (li * self.shape[1] + ri) if self.ok else None

    def entropy(self, psi):
        import torch
        from .observables import entropy_from_schmidt
        if not self.ok:
            return None
        if self.restricted:
            M = torch.zeros(self.shape[0] * self.shape[1], dtype=psi.dtype, device=psi.device)
            M[self.flat] = psi
            M = M.view(self.shape)
        else:
            M = psi.view(self.shape)
        sv = torch.linalg.svdvals(M).double().cpu().numpy()
        return entropy_from_schmidt(sv, self.restricted)


def evolve_manybody(calib, psi0=None, t_grid=None, Om=None, delta=None, gamma=None, terms=None,
                    segments=None, progress_arr=None, log=None, want_corr=True, want_entropy=True,
                    max_dim=None, entropy_cut=None, record_psi=False, diag=False, plan=None,
                    want_observables=True, memory_budget_mb=None, drive_interp='left',
                    dtype='complex128', tol=None, device='cuda', fullpop_max=None, loops=None,
                    want_xy_corr=True, link_pairs=None, pauli_strings=None, **unused):
    """Many-body evolution on the GPU; see the module docstring for the contract."""
    import torch
    log = log or (lambda *a: None)
    if progress_arr is None:
        progress_arr = np.zeros(2)
    if dtype not in ('complex64', 'complex128'):
        raise ValueError('dtype 必须为 complex64/complex128')
    from . import observables as obsmod
    atoms = (calib or {}).get('atoms') or []
    n = len(atoms)
    if n == 0:
        raise ValueError('多体演化：calib 没有原子（先 assemble.calibrate）')
    if link_pairs is not None:
        link_pairs = [(int(a), int(b)) for a, b in link_pairs]
        if any(a < 0 or a >= n or b < 0 or b >= n or a == b for a, b in link_pairs):
            raise ValueError('link_pairs 含越界原子下标')
    pauli_specs = obsmod.normalize_pauli_strings(pauli_strings, n) if pauli_strings else None
    if pauli_specs and not want_observables:
        raise ValueError('manybody.pauli_strings 需要 want_observables=true'
                         '（它挂在公共观测契约的 observables 下，不会单独开一份结果）')
    projected = plan is not None and plan.get('projected')
    if projected:
        Om = plan.get('Om') if Om is None else Om
        delta = plan.get('delta') if delta is None else delta
        gamma = plan.get('gamma') if gamma is None else gamma
        terms = plan.get('terms') if terms is None else terms
    t = time_grid(t_grid)
    check_cancel(progress_arr)
    ctx, basis, ham, perm = model.build(calib, Om, delta, gamma, terms, plan=plan, device=device,
                                        allow_loss=True)
    hermitian = not ham.lossy
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
    fullpop = int(FULLPOP_MAX if fullpop_max is None else fullpop_max)
    if memory_budget_mb is not None:
        fullpop = min(fullpop, int(float(memory_budget_mb) * 1024 ** 2) // max(1, n_t * 8 * 4))
    pops_atom = np.zeros((n_t, n))
    norms = np.zeros(n_t)
    S_mid = np.full(n_t, np.nan) if want_entropy else None
    sx = np.zeros((n_t, n)); sy = np.zeros((n_t, n)); sz = np.zeros((n_t, n))
    spv = np.zeros((n_t, n), complex); smv = np.zeros((n_t, n), complex)
    phase = np.full((n_t, n), np.nan)
    link_series = (np.full((n_t, len(link_pairs)), np.nan + 0j, complex)
                   if link_pairs is not None else None)
    pauli_series = np.zeros((n_t, len(pauli_specs)), complex) if pauli_specs else None
    joint = np.zeros((n_t, dim)) if dim <= fullpop else None
    all_pairs = [(i, j) for i in range(n) for j in range(i + 1, n)]
    schmidt = _Schmidt(basis, n, cut, ctx.device) if (want_entropy and n >= 2) else None
    final_pairs = {}
    terms_used = 0
    pieces = 0

    def reduce(k):
        last = k == n_t - 1
        need_all = last and (want_corr or (want_observables and want_xy_corr))
        links = link_pairs if (link_pairs is not None and want_observables) else []
        ob = solvers.spin_observables(ham, psi, list(links) + (all_pairs if need_all else []))
        pops_atom[k] = ob['n']
        norms[k] = ob['norm']
        sm = ob['sm']
        sx[k], sy[k], sz[k] = 2.0 * sm.real, 2.0 * sm.imag, ob['norm'] - 2.0 * ob['n']
        spv[k], smv[k] = np.conj(sm), sm
        ph = np.angle(sm)
        ph[np.abs(sm) < 1e-14] = np.nan
        phase[k] = ph
        if link_series is not None and want_observables:
            link_series[k] = ob['xy'][:len(links)]
        if need_all:
            final_pairs['nn'] = ob['nn'][len(links):]
            final_pairs['xy'] = ob['xy'][len(links):]
            final_pairs['n'] = ob['n']
        if pauli_series is not None:
            pauli_series[k] = solvers.pauli_expect(ham, psi, pauli_specs)
        if schmidt is not None:
            v = schmidt.entropy(psi)
            S_mid[k] = np.nan if v is None else v
        elif want_entropy:
            S_mid[k] = 0.0          # n < 2: no bipartition, S = 0
        if joint is not None:
            joint[k] = (psi.abs() ** 2).double().cpu().numpy()

    base_om = np.zeros(n, complex) if Om is None else np.asarray(Om, complex)
    base_de = np.zeros(n) if delta is None else np.asarray(delta, float)
    reduce(0)
    current = None
    table = SegmentTable(segments, n) if segments else None
    for k in range(1, n_t):
        for a, b in (segment_intervals(t[k - 1], t[k], segments) if segments else [(t[k - 1], t[k])]):
            check_cancel(progress_arr)
            if segments:
                om, de = table.drive(0.5 * (a + b), interp=drive_interp)
            else:
                om, de = base_om, base_de
            key = (tuple(np.round(om, 15)), tuple(np.round(de, 15)))
            if key != current:
                ham.set_drive(om, de)
                current = key
            if b > a:
                step = solvers.cheb_step if hermitian else solvers.taylor_step
                terms_used += step(ham, psi, b - a, tol=tol)
                pieces += 1
        reduce(k)
        progress_arr[0] = (k + 1) / n_t
    final = psi.cpu().numpy().astype(np.complex128)
    corr = None
    xy_last = None
    if final_pairs:
        ni = final_pairs['n']
        NN = np.diag(ni).astype(float)
        XY = np.diag(ni).astype(complex)
        for q, (i, j) in enumerate(all_pairs):
            NN[i, j] = NN[j, i] = final_pairs['nn'][q]
            XY[i, j] = final_pairs['xy'][q]
            XY[j, i] = np.conj(final_pairs['xy'][q])
        if want_corr:
            corr = NN - np.outer(ni, ni)
        if want_observables and want_xy_corr:
            xy_last = XY
    loss = 1.0 - norms
    backend = ('b200-cheb-plan-%s' % plan['constraint']['kind'] if projected else
               'b200-cheb' if hermitian else 'b200-cheb-nonhermitian')
    capped = joint is None or projected
    if not capped:
        pops = joint
        states = [{'label': obsmod.product_label(n, s), 'index': s} for s in range(dim)]
    else:
        pops = pops_atom
        states = [{'label': 'atom%d' % a.get('id', i), 'atom_id': a.get('id', i)} for i, a in enumerate(atoms)]
    S_note = None
    if want_entropy and S_mid is not None and np.isnan(S_mid).any():
        S_note = ('部分输出时刻未计算纠缠熵（Schmidt 矩阵超过 2^20 个元素或全空间 n > 20）；缺失值为 NaN')
    obs = None
    if want_observables:
        loop_phase, loop_winding = (obsmod.loop_observables(xy_last, loops)
                                    if (xy_last is not None and loops is not None) else ([], []))
        lps, lws = (obsmod.link_loop_observables(link_series, link_pairs, loops)
                    if (link_series is not None and loops is not None)
                    else (np.empty((0, 0), float), np.empty((0, 0), float)))
        obs = dict(sx=sx, sy=sy, sz=sz, sp=spv, sm=smv, phase=phase, xy_corr=xy_last,
                   loop_phase=loop_phase, loop_winding=loop_winding, loop_phase_series=lps,
                   loop_winding_series=lws, link_corr=link_series, link_pairs=link_pairs,
                   pauli_strings=pauli_series,
                   pauli_string_labels=[d['label'] for d in pauli_specs] if pauli_specs else [])
    out = dict(
        t=t, pops=pops, states=states, method='manybody', backend=backend,
        pops_atom=pops_atom, S=S_mid, corr=corr, loss=loss, norms=norms,
        basis_probabilities=joint, basis_states=(codes if projected else None),
        basis=dict(kind='projected' if projected else 'full', bit_order='site0-msb',
                   n_atoms=n, dim=dim, full_dim=1 << n),
        error_report=dict(backend=backend, solver='chebyshev' if hermitian else 'taylor', dim=dim,
                          n_atoms=n, n_t=n_t, hermitian=hermitian, used_sectors=False, full_pops=(not capped),
                          projected=bool(projected), entropy_cut=(cut if want_entropy else None),
                          entropy_note=S_note,
                          max_norm_dev=float(np.max(np.abs(norms - 1.0))) if hermitian else 0.0,
                          chebyshev_terms=int(terms_used), pieces=int(pieces), tol=tol, dtype=dtype),
        diag=({'dim': dim, 'n_atoms': n, 'backend': backend, 'launches': ctx.launches} if diag else None),
        observables=obs)
    if record_psi:
        out['psi_amp'] = final
    return out

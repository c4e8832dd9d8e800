"""calib / plan -> native basis and Hamiltonian, with the reference's checks.

Accepts the reference engine's inputs unchanged: a ``calib`` dict
(atoms + pairs with V/J/A), per-site ``Om``/``delta``/``gamma`` arrays,
``terms`` and an optional HamiltonianPlan or ``basis_indices``.
The B200 path implements Omega, delta, the I1 density interaction V and the
I2 / I3 exchange channels J / A (channels.py:91-132); non-Hermitian gamma is
refused with ConfigConflict, never silently dropped (backends.py:9-18
semantics).  The batched persistent solver implements the Omega/delta/V model
only and refuses J/A the same way.
"""
from __future__ import annotations

import numpy as np

from .core import Basis, Context, Hamiltonian, default_context


class ConfigConflict(ValueError):
    """A configuration key is refused by the selected backend; ``keys`` lists
    the offending ``manybody.*`` keys (same contract as backends.py:9-18)."""

    def __init__(self, message, *, keys=()):
        super().__init__(message)
        self.keys = tuple(keys)


def active_terms(calib):
    """Channels present in a calib (couplings.py:26-40 semantics)."""
    given = (calib or {}).get('terms')
    if given is not None:
        return list(given)
    pairs = (calib or {}).get('pairs') or []
    out = []
    for name, key in (('I1', 'V'), ('I2', 'J'), ('I3', 'A')):
        if any(abs(complex(p.get(key) or 0.0)) > 0.0 for p in pairs):
            out.append(name)
    return out


def model_arrays(calib, Om=None, delta=None, gamma=None, terms=None, exchange=None, allow_loss=False):
    """Validate and flatten a calib to (n, Om complex[n], delta[n], pairs).

    ``exchange``: a list that receives the (i, j, J, A) exchange channels of
    the terms in use; None refuses a nonzero J or A with ConfigConflict.
    ``allow_loss``: accept gamma != 0 (the caller sets the loss diagonal);
    otherwise it is refused with ConfigConflict."""
    n, Om, delta, (pi, pj, V) = model_columns(calib, Om, delta, gamma, terms, exchange, allow_loss)
    return n, Om, delta, list(zip(pi.tolist(), pj.tolist(), V.tolist()))


def model_columns(calib, Om=None, delta=None, gamma=None, terms=None, exchange=None, allow_loss=False):
    """model_arrays with the density pairs as columns: (n, Om, delta,
    (i int32[m], j int32[m], V float64[m])) for the pairs with V != 0, in
    calib order.  Same checks and errors as model_arrays."""
    atoms = (calib or {}).get('atoms') or []
    n = len(atoms)
    if n == 0:
        raise ValueError('通道声明需要至少一个原子')
    Om = np.zeros(n, complex) if Om is None else np.asarray(Om, complex).reshape(-1)
    delta = np.zeros(n) if delta is None else np.asarray(delta, float).reshape(-1)
    gamma = np.zeros(n) if gamma is None else np.asarray(gamma, float).reshape(-1)
    if any(x.shape != (n,) or not np.isfinite(x).all() for x in (Om, delta, gamma)):
        raise ValueError('Om/delta/gamma 须为有限、长度为 N 的数组')
    if np.any(gamma != 0) and not allow_loss:
        raise ConfigConflict('b200 backends need a Hermitian H (gamma = 0)', keys=('manybody.gamma_mhz',))
    raw = calib.get('pairs') or []
    m = len(raw)
    none = (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0))
    if m == 0:
        return n, Om, delta, none

    def column(key):
        # complex from the start: a float column would drop the imaginary
        # part of numpy complex scalars with only a warning
        return np.fromiter((p.get(key) or 0.0 for p in raw), dtype=complex, count=m)
    if terms is None:
        terms = (calib or {}).get('terms')
    if terms is None:
        # the terms a calib carries (active_terms): a channel is on when any
        # of its pair values has a nonzero magnitude
        cols = {key: column(key) for key in ('V', 'J', 'A')}
        use = {name for name, key in (('I1', 'V'), ('I2', 'J'), ('I3', 'A'))
               if np.any(np.abs(cols[key]) > 0.0)}
    else:
        use = set(terms)
        cols = {key: column(key) for name, key in (('I1', 'V'), ('I2', 'J'), ('I3', 'A')) if name in use}
    # columns of the pair list; the checks below raise, for the first pair
    # that fails any of them, the error that pair's own checks would raise
    # first (range, J, A, V, in that order)
    ii = np.fromiter((p['i'] for p in raw), dtype=np.int64, count=m)
    jj = np.fromiter((p['j'] for p in raw), dtype=np.int64, count=m)
    zero = np.zeros(m, complex)
    V = cols['V'] if 'I1' in use else zero
    J = cols['J'] if 'I2' in use else zero
    A = cols['A'] if 'I3' in use else zero
    checks = [
        ((ii < 0) | (ii >= n) | (jj < 0) | (jj >= n) | (ii == jj),
         lambda k: ValueError('pair (%d, %d) out of range' % (ii[k], jj[k]))),
        (~np.isfinite(J), lambda k: ValueError('pair (%d, %d): J must be finite' % (ii[k], jj[k]))),
        ((J != 0) if exchange is None else np.zeros(m, bool),
         lambda k: ConfigConflict('this b200 solver implements the Omega/delta/V model only '
                                  '(I2 channel J != 0)', keys=('manybody.calib',))),
        (~np.isfinite(A), lambda k: ValueError('pair (%d, %d): A must be finite' % (ii[k], jj[k]))),
        ((A != 0) if exchange is None else np.zeros(m, bool),
         lambda k: ConfigConflict('this b200 solver implements the Omega/delta/V model only '
                                  '(I3 channel A != 0)', keys=('manybody.calib',))),
        (V.imag != 0, lambda k: ValueError('V must be real')),
    ]
    first = None
    for order, (mask, err) in enumerate(checks):
        if mask.any():
            k = int(np.argmax(mask))
            if first is None or (k, order) < first[:2]:
                first = (k, order, err)
    if first is not None:
        raise first[2](first[0])
    if exchange is not None:
        for k in np.flatnonzero((J != 0) | (A != 0)):
            exchange.append((int(ii[k]), int(jj[k]), complex(J[k]), complex(A[k])))
    keep = np.flatnonzero(V.real != 0)
    return n, Om, delta, (ii[keep].astype(np.int32), jj[keep].astype(np.int32),
                          np.ascontiguousarray(V.real[keep], dtype=np.float64))


def _is_chain_or_ring(n, edges):
    es = sorted({tuple(sorted((int(a), int(b)))) for a, b in edges})
    chain = [(i, i + 1) for i in range(n - 1)]
    return es == chain or es == sorted(chain + [(0, n - 1)])


_PROJECTING = ('blockade', 'pxp')


def resolve_constraint(calib, constraint):
    """A reference constraint spec -> (projected, edges, spec).

    Same meaning as hamiltonian_plan.py:15-50: the spec is None, a kind
    string or a dict with kind none/blockade/pxp (default none), mode
    full/project (default project for blockade and pxp, else full),
    threshold_mhz >= 0 and edges (an integer pair list, 'auto' or absent).
    A blockade or pxp spec in project mode restricts the basis to the
    independent sets of its graph: the explicit edges, else every pair of
    the calib whose |V| reaches threshold_mhz; with neither, ValueError (no
    spec ever yields a silently unconstrained basis).  Edges come back as
    sorted (i < j) pairs without repeats."""
    spec = {'kind': constraint} if isinstance(constraint, str) else constraint
    if spec is None:
        spec = {}
    if not isinstance(spec, dict):
        raise ValueError('manybody.constraint 须为 dict 或字符串')
    kind = str(spec.get('kind', 'none')).lower()
    if kind not in ('none',) + _PROJECTING:
        raise ValueError('constraint.kind 只支持 none/blockade/pxp')
    mode = str(spec.get('mode', 'project' if kind in _PROJECTING else 'full')).lower()
    if mode not in ('full', 'project'):
        raise ValueError('constraint.mode 只支持 full/project')
    thr = float(spec.get('threshold_mhz', 0.0) or 0.0)
    if not (np.isfinite(thr) and thr >= 0):
        raise ValueError('constraint.threshold_mhz 必须是有限非负数')
    given = spec.get('edges')
    norm = dict(kind=kind, mode=mode, threshold_mhz=thr, edges=given)
    if not (kind in _PROJECTING and mode == 'project'):
        return False, [], norm
    n = len(calib.get('atoms') or [])
    if given is not None and not isinstance(given, str):
        edges = set()
        for e in given:
            ok = len(e) == 2 and all(not isinstance(v, (bool, np.bool_)) and int(v) == v for v in e)
            if not ok:
                raise ValueError('blockade edge 必须是两个整数下标')
            a, b = int(e[0]), int(e[1])
            if a == b or min(a, b) < 0 or max(a, b) >= n:
                raise ValueError('blockade edge 越界或自环：%r' % (e,))
            edges.add((min(a, b), max(a, b)))
        return True, [list(e) for e in sorted(edges)], norm
    if given not in (None, 'auto'):
        raise ValueError('constraint.edges 只支持 auto 或整数边列表')
    if thr <= 0:
        raise ValueError('blockade/PXP project 模式需要 threshold_mhz>0 或显式 edges')
    pairs = calib.get('pairs') or []
    strong = {(min(int(p['i']), int(p['j'])), max(int(p['i']), int(p['j'])))
              for p in pairs if abs(complex(p.get('V', 0.0))) >= thr}
    return True, [list(e) for e in sorted(strong)], norm


def plan_edges(plan, calib=None):
    """Blockade edges of a projected plan: its own 'blockade_edges' when the
    plan carries them (build_plan output), else derived from its constraint
    spec and calib by resolve_constraint."""
    if plan.get('blockade_edges') is not None:
        return [list(map(int, e)) for e in plan['blockade_edges']]
    calib = plan.get('calib', calib)
    if calib is None or plan.get('constraint') is None:
        raise ValueError('projected plan 缺少 blockade_edges（也无 constraint + calib 可推导）')
    projected, edges, _ = resolve_constraint(calib, plan['constraint'])
    if not projected:
        raise ValueError('plan 声明 projected，但其 constraint 不投影')
    return edges


def basis_for(ctx: Context, n, plan=None, basis_indices=None, constraint=None, max_states=None,
              calib=None):
    """Native basis for the reference's basis descriptions.

    plan: HamiltonianPlan dict (hamiltonian_plan.py:129-148) -> its blockade
    edges when projected; basis_indices: an explicit code list, accepted when
    it is a blockade sector of its plan, a fixed-excitation sector or the full
    basis (checked code by code); returns (Basis, permutation or None) where the
    permutation maps the caller's order to ascending order."""
    if plan is not None and plan.get('projected'):
        edges = plan_edges(plan, calib)
        b = Basis(ctx, n, kind='blockade', edges=edges, max_states=max_states)
        if plan.get('states') is not None and len(plan['states']) != b.dim:
            raise ValueError('plan states do not match its blockade edges')
        return b, None
    if constraint is not None:
        if isinstance(constraint, dict) and constraint.get('kind') == 'charge':
            return Basis(ctx, n, kind='charge', k=int(constraint['k'])), None
        if calib is None:
            raise ValueError('a blockade/pxp constraint needs the calib (threshold edges)')
        projected, edges, _ = resolve_constraint(calib, constraint)
        if projected:
            return Basis(ctx, n, kind='blockade', edges=edges, max_states=max_states), None
    if basis_indices is None:
        return Basis(ctx, n, kind='full'), None
    codes = np.asarray(basis_indices, np.int64).reshape(-1)
    if codes.size == 0 or np.any(codes < 0) or np.any(codes >= (1 << n)):
        raise ValueError('basis_indices 须为非空有效位编码')
    order = np.argsort(codes, kind='stable')
    srt = codes[order]
    if np.any(np.diff(srt) == 0):
        raise ValueError('basis_indices 不能重复')
    perm = None if np.array_equal(order, np.arange(codes.size)) else order
    pc = np.array([int(c).bit_count() for c in srt])
    if codes.size == (1 << n):
        return Basis(ctx, n, kind='full'), perm
    if np.all(pc == pc[0]):
        b = Basis(ctx, n, kind='charge', k=int(pc[0]))
        if b.dim == codes.size and np.array_equal(b.codes().cpu().numpy(), srt):
            return b, perm
    # a blockade sector: the graph of pairs never jointly excited
    bits = np.array([[(int(c) >> (n - 1 - i)) & 1 for i in range(n)] for c in srt], dtype=np.int64)
    co = bits.T @ bits
    edges = [[i, j] for i in range(n) for j in range(i + 1, n) if co[i, j] == 0]
    b = Basis(ctx, n, kind='blockade', edges=edges)
    if b.dim == codes.size and np.array_equal(b.codes().cpu().numpy(), srt):
        return b, perm
    raise ValueError('basis_indices is not a full, fixed-excitation or blockade basis; '
                     'the b200 backends need one of those')


def check_number_conserving(calib, Om=None, terms=None):
    """Refuse a fixed-excitation basis for a model that leaves it: Omega != 0
    or a nonzero I3 pair creation A (matrix_free.py:41-48)."""
    use = set(calib.get('terms', ()) if terms is None else terms)
    if Om is not None and np.any(np.asarray(Om, complex) != 0):
        raise ValueError('固定 charge_sector 要求 Omega=0')
    if 'I3' in use and any(complex(p.get('A', 0)) != 0 for p in calib.get('pairs', ())):
        raise ValueError('固定 charge_sector 不支持 I3 双激发项')


def build(calib, Om=None, delta=None, gamma=None, terms=None, plan=None, basis_indices=None,
          constraint=None, device=0, ctx=None, max_states=None, allow_loss=False):
    """(ctx, basis, hamiltonian, permutation) for a reference-style model.
    ``allow_loss``: the caller propagates in time and accepts gamma != 0 (a
    non-Hermitian loss diagonal, channels.py:69-76)."""
    exchange = []
    n, Om, delta, pairs = model_arrays(calib, Om, delta, gamma, terms, exchange=exchange,
                                       allow_loss=allow_loss)
    dev = device
    if isinstance(dev, str):
        if dev.startswith('cpu'):
            raise RuntimeError('CUDA 不可用')
        dev = int(dev.split(':')[1]) if ':' in dev else 0
    ctx = ctx or default_context(int(dev))
    b, perm = basis_for(ctx, n, plan=plan, basis_indices=basis_indices, constraint=constraint,
                        max_states=max_states, calib=calib)
    h = Hamiltonian(ctx, b, Om, delta, pairs, exchange=exchange)
    if gamma is not None and np.any(np.asarray(gamma, float) != 0):
        h.set_loss(gamma)
    return ctx, b, h, perm

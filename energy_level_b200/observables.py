"""Host post-processing of the device observables (small n x n arrays).

The per-state sums (<n_i>, <sigma-_i>, <n_i n_j>, <sigma+_i sigma-_j>,
Pauli strings) run on the device (el_spin_observables, el_pauli_expect);
this module holds what the reference does with them afterwards:

- ``normalize_pauli_strings``: the accepted forms and checks of
  observables.py:315-375 (list of [site, axis] pairs or dicts with label and
  terms; distinct integer sites; x/y/z axes and their aliases);
- ``loop_observables`` / ``link_loop_observables``: bond-phase sums around
  closed loops (observables.py:206-278);
- ``product_label``: '|g r ...>' labels of basis states (observables.py:83-86);
- ``entropy_from_schmidt``: von Neumann entropy of Schmidt weights, with the
  full-basis (observables.py:50-80) and restricted-basis (:89-114) rules.
"""
from __future__ import annotations

import numpy as np

_AXES = {'x': 'x', 'y': 'y', 'z': 'z', 'sx': 'x', 'sy': 'y', 'sz': 'z',
         'σx': 'x', 'σy': 'y', 'σz': 'z', 'sigmax': 'x', 'sigmay': 'y', 'sigmaz': 'z'}


def _axis(raw):
    a = _AXES.get(str(raw).strip().lower())
    if a is None:
        raise ValueError('Pauli 字符串的轴须为 x/y/z（可写 σx 等），得到 %r' % (raw,))
    return a


def normalize_pauli_strings(spec, n_atoms=None, err=None):
    """Pauli string specs -> [{'label', 'terms': [(site, axis), ...]}]."""
    if spec is None:
        return None
    err = err or ValueError
    if not isinstance(spec, (list, tuple)):
        raise err('manybody.pauli_strings 须是 list（得到 %s）' % type(spec).__name__)
    n = None if n_atoms is None else int(n_atoms)
    out = []
    for k, item in enumerate(spec):
        tag = 'pauli_strings[%d]' % k
        if isinstance(item, dict):
            raw, label = item.get('terms', item.get('sites')), item.get('label')
        else:
            raw, label = item, None
        if raw is None:
            raise err('%s 缺 terms（形如 [[0,"x"],[1,"y"]]）' % tag)
        if not isinstance(raw, (list, tuple)) or not raw:
            raise err('%s.terms 须是非空序列' % tag)
        terms, seen = [], set()
        for t in raw:
            if not isinstance(t, (list, tuple)) or len(t) != 2:
                raise err('%s.terms 的每一项须为 [site, axis]，得到 %r' % (tag, t))
            site = t[0]
            if isinstance(site, bool) or not isinstance(site, (int, np.integer)):
                raise err('%s.terms 的站点须为整数，得到 %r' % (tag, site))
            site = int(site)
            if n is not None and not 0 <= site < n:
                raise err('%s.terms 的站点 %d 越界（原子数 %d）' % (tag, site, n))
            if site in seen:
                raise err('%s 在同一站点 %d 上放了两个算符；Pauli 字符串要求站点互不相同' % (tag, site))
            seen.add(site)
            terms.append((site, _axis(t[1])))
        if label is None:
            label = ' '.join('%s@%d' % (ax, s) for s, ax in terms)
        out.append({'label': str(label), 'terms': terms})
    return out


def loop_observables(xy_corr, loops):
    """Phase sum arg<sigma+_a sigma-_b> around each loop (closing edge added)
    and its winding (sum / 2 pi); NaN when an edge amplitude vanishes."""
    if loops is None:
        return [], []
    xy = np.asarray(xy_corr, complex)
    phases, wind = [], []
    for loop in loops:
        q = [int(x) for x in loop]
        if len(q) < 2 or any(x < 0 or x >= xy.shape[0] for x in q):
            raise ValueError('loop 必须包含至少两个合法原子下标')
        vals = []
        for a, b in zip(q, q[1:] + q[:1]):
            z = xy[a, b]
            vals.append(float(np.angle(z)) if abs(z) > 1e-14 else np.nan)
        total = float(np.sum(vals)) if np.all(np.isfinite(vals)) else np.nan
        phases.append(total)
        wind.append(float(total / (2.0 * np.pi)) if np.isfinite(total) else np.nan)
    return phases, wind


def link_loop_observables(link_corr, link_pairs, loops):
    """Loop phase / winding time series from the selected links (either
    orientation; the reverse one is the complex conjugate)."""
    if loops is None:
        return np.empty((0, 0), float), np.empty((0, 0), float)
    lookup = {}
    for q, (a, b) in enumerate([(int(a), int(b)) for a, b in (link_pairs or [])]):
        lookup.setdefault((a, b), []).append((q, 1))
        lookup.setdefault((b, a), []).append((q, -1))
    arr = np.asarray(link_corr, complex)
    if arr.ndim == 1:
        arr = arr[None, :]
    phase = np.full((arr.shape[0], len(loops)), np.nan, float)
    winding = np.full_like(phase, np.nan)
    for ell, raw in enumerate(loops):
        loop = [int(x) for x in raw]
        if len(loop) < 2:
            raise ValueError('loop 必须包含至少两个合法原子下标')
        cols = []
        for a, b in zip(loop, loop[1:] + loop[:1]):
            choice = lookup.get((a, b))
            if not choice:
                cols = None
                break
            cols.append(choice[0])
        if cols is None:
            continue
        vals = np.zeros((arr.shape[0], len(cols)))
        valid = np.ones(arr.shape[0], bool)
        for j, (q, sign) in enumerate(cols):
            z = arr[:, q] if sign > 0 else np.conj(arr[:, q])
            valid &= np.abs(z) > 1e-14
            vals[:, j] = np.angle(z)
        total = vals.sum(axis=1)
        phase[valid, ell] = total[valid]
        winding[valid, ell] = total[valid] / (2.0 * np.pi)
    return phase, winding


def product_label(n, s):
    bits = ''.join('r' if ((int(s) >> (n - 1 - i)) & 1) else 'g' for i in range(n))
    return '|%s>' % bits if n else '|>'


def entropy_from_schmidt(sv, restricted):
    """S = -sum w ln w of the Schmidt weights w = sv^2: full basis drops
    w <= 1e-15 (no renormalisation); a restricted basis renormalises the
    weights and drops zeros (None for a zero state)."""
    w = np.asarray(sv, float) ** 2
    if restricted:
        tot = w.sum()
        if tot <= 0:
            return None
        w = w / tot
        w = w[w > 0]
    else:
        w = w[w > 1e-15]
        if w.size == 0:
            return 0.0
    return float(-np.sum(w * np.log(w)))

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


_NO_PHASE = 1e-14   # a bond amplitude at or below this has no defined phase


def _closed_loop(loop, n_sites=None):
    """Sites of a loop given without its closing repeat, and the site each
    one links to (the next, the last back to the first)."""
    q = np.asarray([int(x) for x in loop], dtype=np.int64)
    if q.size < 2 or (n_sites is not None and (q.min() < 0 or q.max() >= n_sites)):
        raise ValueError('loop 必须包含至少两个合法原子下标')
    return q, np.roll(q, -1)


def _phase_sum(z):
    """z[..., e]: the complex amplitudes of a loop's directed bonds.  Returns
    (sum_e arg z, that sum / 2 pi) over the last axis, NaN wherever a bond has
    no defined phase (the gauge-invariant flux of observables.py:206-231)."""
    z = np.asarray(z, complex)
    defined = np.all(np.abs(z) > _NO_PHASE, axis=-1)
    flux = np.where(defined, np.angle(z).sum(axis=-1), np.nan)
    return flux, flux / (2.0 * np.pi)


def loop_observables(xy_corr, loops):
    """Flux arg<sigma+_a sigma-_b> summed around each loop of sites and its
    winding (flux / 2 pi), from one <sigma+ sigma-> matrix; NaN for a loop
    with a vanishing bond.  Returns two lists (one entry per loop)."""
    if loops is None:
        return [], []
    xy = np.asarray(xy_corr, complex)
    flux, wind = [], []
    for loop in loops:
        a, b = _closed_loop(loop, xy.shape[0])
        f, w = _phase_sum(xy[a, b])
        flux.append(float(f))
        wind.append(float(w))
    return flux, wind


def link_loop_observables(link_corr, link_pairs, loops):
    """The same flux and winding as time series, from the selected links only:
    link_corr[t, q] = <sigma+_a sigma-_b> for link_pairs[q] = (a, b).  A bond
    of a loop is the first link joining its two sites, read conjugated when
    the link runs the other way; a loop with a bond no link covers stays NaN
    (observables.py:234-278 semantics).  Returns (flux, winding), each of
    shape (times, loops)."""
    if loops is None:
        return np.empty((0, 0), float), np.empty((0, 0), float)
    links = np.asarray([(int(a), int(b)) for a, b in (link_pairs or [])], dtype=np.int64).reshape(-1, 2)
    series = np.asarray(link_corr, complex)
    series = series[None, :] if series.ndim == 1 else series
    flux = np.full((series.shape[0], len(loops)), np.nan)
    wind = np.full_like(flux, np.nan)
    for ell, loop in enumerate(loops):
        a, b = _closed_loop(loop)
        fwd = (links[:, None, 0] == a) & (links[:, None, 1] == b)      # [link, bond]
        rev = (links[:, None, 0] == b) & (links[:, None, 1] == a)
        hit = fwd | rev
        if not hit.any(axis=0).all():
            continue
        col = np.argmax(hit, axis=0)                                   # first link per bond
        z = series[:, col]
        flip = ~fwd[col, np.arange(col.size)]
        z[:, flip] = np.conj(z[:, flip])
        flux[:, ell], wind[:, ell] = _phase_sum(z)
    return flux, wind


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

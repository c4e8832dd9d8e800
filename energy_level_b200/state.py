"""Initial states in the MSB basis, full or projected.

The reference's state grammar (state.py:112-208) is accepted unchanged: None
(every site |g>), a 'g'/'r' pattern ('|grg>' style decorations allowed), a
basis index, a list of N local states (each 'g', 'r', 0, 1 or an [a_g, a_r]
pair), a {'kind': 'product', 'amplitudes' | 'local_states': [...]} dict, a
full 2^N vector (array or list), or ('sup', [...]) -- a superposition of
specs or of (pattern, amplitude) pairs.  The spec is classified once by an
ordered rule table; amplitudes are evaluated directly on the basis codes, and
in a projected basis any weight outside the basis is an error, never a
silent projection (state.py:160-163).  Error texts are the reference's, so a
caller sees the same messages from either engine.
"""
from __future__ import annotations

import numpy as np

_NAMED = {'g': (1.0, 0.0), 'r': (0.0, 1.0)}   # local states by letter (and by index 0 / 1)


def _is_index(x):
    return isinstance(x, (int, np.integer)) and not isinstance(x, bool)


def _scalar(x):
    """A complex amplitude, also from a [re, im] pair."""
    if isinstance(x, (list, tuple)) and len(x) == 2:
        return complex(float(x[0]), float(x[1]))
    return complex(x)


def _local(x):
    """Unit local state [a_g, a_r] of one site."""
    if isinstance(x, str):
        if x not in _NAMED:
            raise ValueError('局部二能级态字符串只接受 g 或 r')
        return np.asarray(_NAMED[x], complex)
    if _is_index(x):
        if int(x) not in (0, 1):
            raise ValueError('局部二能级态索引只接受 0 或 1')
        return np.asarray(_NAMED['gr'[int(x)]], complex)
    pair = np.asarray([_scalar(v) for v in x], complex) if hasattr(x, '__len__') else None
    if pair is None or pair.shape != (2,):
        raise ValueError('局部态必须是 [a_g, a_r]，形状为 (2,)')
    size = float(np.linalg.norm(pair))
    if not (np.isfinite(size) and size > 0):
        raise ValueError('局部态不能是零向量或含非有限数值')
    return pair / size


def _product_sites(spec, n):
    """The N local states of a product spec (None for 'ground')."""
    if spec is None:
        return [_local('g')] * n
    if _is_index(spec):
        if not 0 <= int(spec) < (1 << n):
            raise ValueError('多体初态索引越界')
        return [_local((int(spec) >> (n - 1 - i)) & 1) for i in range(n)]
    if isinstance(spec, str):
        if spec == 'ground':
            return None
        letters = ''.join(ch for ch in spec if ch not in '|> ')
        if len(letters) != n or set(letters) - set('gr'):
            raise ValueError('模式串须由长度为 N 的 g/r 组成')
        return [_local(ch) for ch in letters]
    if isinstance(spec, dict):
        if spec.get('kind', 'product') != 'product':
            raise ValueError('未知乘积态 kind=%r；请使用 kind=product + amplitudes' % spec.get('kind'))
        spec = spec.get('amplitudes', spec.get('local_states'))
        if spec is None:
            raise ValueError('product 初态需要 amplitudes 或 local_states')
    if isinstance(spec, (list, tuple)) and len(spec) == n:
        return [_local(x) for x in spec]
    raise ValueError('无法解析多体乘积初态')


def product_vectors(spec, n):
    """Local states [a_g, a_r] of every site for a product spec, or None for
    'ground' (prepared by a solver, not by the grammar)."""
    return _product_sites(spec, int(n))


# grammar forms, tested in this order (the first match decides)
def _looks_full_list(spec, n):
    return (isinstance(spec, (list, tuple)) and len(spec) == (1 << n)
            and not (len(spec) == n and all(isinstance(x, (str, int, np.integer)) for x in spec)))


_FORMS = (
    ('array', lambda spec, n: isinstance(spec, np.ndarray)),
    ('superposition', lambda spec, n: isinstance(spec, (list, tuple)) and len(spec) > 0
     and isinstance(spec[0], str) and spec[0] == 'sup'),
    ('index', lambda spec, n: _is_index(spec)),
    ('full_list', _looks_full_list),
)


def _form(spec, n):
    return next((name for name, test in _FORMS if test(spec, n)), 'product')


def _on_basis(spec, n, codes, projected):
    """Amplitudes of `spec` on the basis codes, and whether they are already
    normalised (the superposition form normalises its sum itself)."""
    form = _form(spec, n)
    if form == 'array':
        full = np.asarray(spec, complex)
        if full.shape != (1 << n,):
            raise ValueError('初态向量形状必须是 (2**N,)；受限态需携带完整基身份')
        size = np.linalg.norm(full)
        return (full[codes] / size if size > 0 else full[codes]), False
    if form == 'full_list':
        return _on_basis(np.asarray(spec, complex), n, codes, projected)
    if form == 'index':
        if not 0 <= int(spec) < (1 << n):
            raise ValueError('多体初态索引越界')
        return (codes == int(spec)).astype(complex), False
    if form == 'superposition':
        total = np.zeros(codes.size, complex)
        for part in spec[1]:
            weighted = (isinstance(part, (list, tuple)) and len(part) == 2
                        and not isinstance(part[0], (list, tuple, dict)))
            sub, amp = (part[0], _scalar(part[1])) if weighted else (part, 1.0)
            total += amp * _normalised(sub, n, codes, projected)
        size = np.linalg.norm(total)
        if not (np.isfinite(size) and size > 0):
            raise ValueError('多体初态零范数或包含非有限数值')
        return total / size, True
    sites = _product_sites(spec, n)
    if sites is None:
        raise ValueError('ground 初态必须由求解器从当前 Hamiltonian 准备')
    occupied = [np.flatnonzero(loc) for loc in sites]
    if all(o.size == 1 for o in occupied):
        # every site exactly |g> or |r> (up to a phase): a single basis code
        bits = [int(o[0]) for o in occupied]
        code = sum(b << (n - 1 - i) for i, b in enumerate(bits))
        amp = complex(np.prod([loc[b] for loc, b in zip(sites, bits)]))
        return np.where(codes == code, amp, 0.0).astype(complex), False
    amps = np.ones(codes.size, complex)
    for i, loc in enumerate(sites):
        amps *= loc[(codes >> (n - 1 - i)) & 1]
    return amps, False


def _normalised(spec, n, codes, projected):
    amps, done = _on_basis(spec, n, codes, projected)
    if done:
        return amps
    size = float(np.linalg.norm(amps))
    if not (np.isfinite(size) and size > 0):
        raise ValueError('多体初态零范数或不在受限子空间')
    if projected and abs(size - 1.0) > 1e-10:
        raise ValueError('初态含受限子空间之外的幅度；不会静默投影')
    return amps / size


def state_vector(spec, n, codes=None):
    """Normalised state on the basis `codes` (ascending int64 codes; None =
    the full 2^N basis)."""
    n = int(n)
    if codes is None:
        return _normalised(spec, n, np.arange(1 << n, dtype=np.int64), False)
    return _normalised(spec, n, np.asarray(codes, np.int64), True)

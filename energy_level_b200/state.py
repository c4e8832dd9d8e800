"""Initial states in the MSB basis, full or projected.

Restates the state grammar of the reference (state.py:112-208): None (all
|g>), a 'g'/'r' pattern, a basis index, a list of local [a_g, a_r] vectors, a
{'kind': 'product', 'amplitudes': ...} dict, a full 2^N vector, or a
('sup', [...]) superposition.  In a projected basis the amplitudes are
evaluated directly on the basis codes, and weight outside the basis is an
error, never a silent projection (state.py:160-163).
"""
from __future__ import annotations

import numpy as np


def _scalar(x):
    if isinstance(x, (list, tuple)) and len(x) == 2:
        return complex(float(x[0]), float(x[1]))
    return complex(x)


def _local(x):
    if isinstance(x, str):
        if x == 'g':
            return np.array([1.0, 0.0], complex)
        if x == 'r':
            return np.array([0.0, 1.0], complex)
        raise ValueError('局部二能级态字符串只接受 g 或 r')
    if isinstance(x, (int, np.integer)) and not isinstance(x, bool):
        if int(x) not in (0, 1):
            raise ValueError('局部二能级态索引只接受 0 或 1')
        return np.eye(2, dtype=complex)[:, int(x)]
    a = np.asarray([_scalar(v) for v in x], complex) if hasattr(x, '__len__') else None
    if a is None or a.shape != (2,):
        raise ValueError('局部态必须是 [a_g, a_r]，形状为 (2,)')
    nrm = float(np.linalg.norm(a))
    if not np.isfinite(nrm) or nrm <= 0:
        raise ValueError('局部态不能是零向量或含非有限数值')
    return a / nrm


def product_vectors(spec, n):
    if spec is None:
        return [np.array([1.0, 0.0], complex) for _ in range(n)]
    if isinstance(spec, (int, np.integer)) and not isinstance(spec, bool):
        if not 0 <= int(spec) < (1 << n):
            raise ValueError('多体初态索引越界')
        return [_local((int(spec) >> (n - 1 - i)) & 1) for i in range(n)]
    if isinstance(spec, str):
        if spec == 'ground':
            return None
        s = spec.replace('|', '').replace('>', '').replace(' ', '')
        if len(s) != n or any(c not in 'gr' for c in s):
            raise ValueError('模式串须由长度为 N 的 g/r 组成')
        return [_local(c) for c in s]
    if isinstance(spec, dict):
        if spec.get('kind', 'product') != 'product':
            raise ValueError('未知乘积态 kind=%r；请使用 kind=product + amplitudes' % spec.get('kind'))
        raw = spec.get('amplitudes', spec.get('local_states'))
        if raw is None:
            raise ValueError('product 初态需要 amplitudes 或 local_states')
        spec = raw
    if isinstance(spec, (list, tuple)) and len(spec) == n:
        return [_local(x) for x in spec]
    raise ValueError('无法解析多体乘积初态')


def state_vector(spec, n, codes=None):
    """Normalised state on the basis `codes` (None = full 2^N basis)."""
    n = int(n)
    basis = np.arange(1 << n, dtype=np.int64) if codes is None else np.asarray(codes, np.int64)
    projected = codes is not None
    if isinstance(spec, np.ndarray):
        full = np.asarray(spec, complex)
        if full.shape != (1 << n,):
            raise ValueError('初态向量形状必须是 (2**N,)；受限态需携带完整基身份')
        nrm = np.linalg.norm(full)
        vec = full[basis] / nrm if nrm > 0 else full[basis]
    elif isinstance(spec, (list, tuple)) and spec and isinstance(spec[0], str) and spec[0] == 'sup':
        vec = np.zeros(len(basis), complex)
        for comp in spec[1]:
            if (isinstance(comp, (list, tuple)) and len(comp) == 2
                    and not isinstance(comp[0], (list, tuple, dict))):
                pattern, amp = comp
                vec += _scalar(amp) * state_vector(pattern, n, codes)
            else:
                vec += state_vector(comp, n, codes)
        nrm = np.linalg.norm(vec)
        if not np.isfinite(nrm) or nrm <= 0:
            raise ValueError('多体初态零范数或包含非有限数值')
        return vec / nrm
    elif isinstance(spec, (int, np.integer)) and not isinstance(spec, bool):
        if not 0 <= int(spec) < (1 << n):
            raise ValueError('多体初态索引越界')
        vec = (basis == int(spec)).astype(complex)
    elif (isinstance(spec, (list, tuple)) and len(spec) == (1 << n)
          and not (len(spec) == n and all(isinstance(x, (str, int, np.integer)) for x in spec))):
        return state_vector(np.asarray(spec, complex), n, codes)
    else:
        vecs = product_vectors(spec, n)
        if vecs is None:
            raise ValueError('ground 初态必须由求解器从当前 Hamiltonian 准备')
        if all(np.count_nonzero(loc) == 1 for loc in vecs):
            # every site in |g> or |r> (up to a phase): one basis code
            bits = [int(np.flatnonzero(loc)[0]) for loc in vecs]
            c0 = sum(b << (n - 1 - i) for i, b in enumerate(bits))
            amp = complex(np.prod([loc[b] for loc, b in zip(vecs, bits)]))
            vec = np.zeros(len(basis), complex)
            vec[np.flatnonzero(basis == c0)] = amp
        else:
            vec = np.ones(len(basis), complex)
            for i, loc in enumerate(vecs):
                vec *= loc[(basis >> (n - 1 - i)) & 1]
    nrm = float(np.linalg.norm(vec))
    if not np.isfinite(nrm) or nrm <= 0:
        raise ValueError('多体初态零范数或不在受限子空间')
    if projected and abs(nrm - 1.0) > 1e-10:
        raise ValueError('初态含受限子空间之外的幅度；不会静默投影')
    return vec / nrm

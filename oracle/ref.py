"""numpy restatement of the reference's ED algorithms -- TEST INFRASTRUCTURE ONLY.

Used by tests, ``__graft_entry__.smoke()`` and the CPU baseline of
``bench.py`` as the checker; never imported by the product package.
Conventions (reference src/core/manybody/basis.py:1-9, channels.py:12-14):
site 0 is the most significant bit of a code, bit 1 means |r>, H[t, s] =
<t|H|s>, energies in cyclic MHz, CONV = 2 pi 1e-3 (evolve_util.py:12).
Pinned by tests/golden (fixtures written by the reference itself).
"""
from __future__ import annotations

import numpy as np

CONV = 2 * np.pi * 1e-3


# ------------------------------------------------------------------ basis

def basis_bits(n, states):
    """(n, dim) int8 bits, row i = site i (basis.py:6-9)."""
    states = np.asarray(states, dtype=np.int64)
    return np.asarray([((states >> (int(n) - 1 - i)) & 1) for i in range(int(n))], dtype=np.int8)


def validate_edges(n, edges):
    """Sorted unique (i<j) edges; errors as basis.py:12-21."""
    out = set()
    for e in edges or []:
        if len(e) != 2 or any(isinstance(i, (bool, np.bool_)) or int(i) != i for i in e):
            raise ValueError('blockade edge must be two integers')
        i, j = map(int, e)
        if not 0 <= i < n or not 0 <= j < n or i == j:
            raise ValueError('blockade edge out of range or self loop: %r' % (e,))
        out.add(tuple(sorted((i, j))))
    return sorted(out)


def independent_states(n, edges, max_states=1 << 20):
    """Ascending codes of the independent sets (basis.py:24-47).

    The reference walks a DFS that tries 'site empty' before 'site occupied';
    with site 0 as the most significant bit its leaves come out in ascending
    code order, which is what this site-by-site numpy expansion plus a sort
    produces."""
    n = int(n)
    edges = validate_edges(n, edges)
    earlier = [0] * n   # code bits of already placed neighbours of site i
    for i, j in edges:
        a, b = min(i, j), max(i, j)
        earlier[b] |= 1 << (n - 1 - a)
    codes = np.zeros(1, np.int64)
    for i in range(n):
        bit = np.int64(1) << (n - 1 - i)
        ok = (codes & np.int64(earlier[i])) == 0
        codes = np.concatenate((codes, codes[ok] | bit))
    codes.sort()
    if max_states and codes.size > int(max_states):
        raise ValueError('restricted basis dimension exceeds max_states=%d' % max_states)
    return codes


def number_sector_basis(n, k):
    """Ascending codes with popcount k (matrix_free.py:12-38)."""
    n, k = int(n), int(k)
    if not 0 <= n <= 63 or not 0 <= k <= n:
        raise ValueError('charge_sector out of range')
    codes = np.zeros(1, np.int64)
    counts = np.zeros(1, np.int8)
    for i in range(n):
        new = codes | (np.int64(1) << i)
        cnew = counts + 1
        keep = cnew <= k
        codes = np.concatenate((codes, new[keep]))
        counts = np.concatenate((counts, cnew[keep]))
    out = codes[counts == k]
    out.sort()
    return out


def fib(i):
    a, b = 0, 1
    for _ in range(i):
        a, b = b, a + b
    return a


# ------------------------------------------------------------ Hamiltonian

def diagonal(n, codes, delta, pairs):
    """d(s) = sum delta_i n_i + sum V_ij n_i n_j (channels.py:58-77, real case)."""
    bits = basis_bits(n, codes).astype(np.float64)
    d = np.zeros(bits.shape[1])
    for i in range(n):
        d += float(delta[i]) * bits[i]
    for i, j, V in pairs:
        d += float(V) * bits[int(i)] * bits[int(j)]
    return d


def loss_diagonal(n, codes, gamma):
    """Imaginary diagonal -0.5 i sum gamma_i 1e-3 / CONV n_i (channels.py:69-76)."""
    bits = basis_bits(n, codes).astype(np.float64)
    g = np.asarray(gamma, float)
    return -0.5j * (g * 1e-3 / CONV) @ bits


def channel_list(n, omega, exchange=None):
    """(selector, mask, amp) channels as channel_spec builds them
    (channels.py:114-131): per site with Omega != 0 a g->r channel with
    Omega/2 and an r->g channel with conj(Omega)/2; per exchange pair
    (i, j, J, A) the I2 channels (i r, j g) -> conj(J), (i g, j r) -> J and
    the I3 channels (i g, j g) -> A, (i r, j r) -> conj(A).  The selector
    names the SOURCE bits; the target is source ^ mask."""
    n = int(n)
    om = np.asarray(omega, complex)
    out = []
    for i in range(n):
        if om[i] == 0:
            continue
        m = np.int64(1) << (n - 1 - i)
        out.append((((i, 0),), m, om[i] / 2.0))
        out.append((((i, 1),), m, np.conj(om[i]) / 2.0))
    for i, j, J, A in (exchange or ()):
        i, j, J, A = int(i), int(j), complex(J), complex(A)
        m = (np.int64(1) << (n - 1 - i)) ^ (np.int64(1) << (n - 1 - j))
        if J != 0:
            out.append((((i, 1), (j, 0)), m, np.conj(J)))
            out.append((((i, 0), (j, 1)), m, J))
        if A != 0:
            out.append((((i, 0), (j, 0)), m, A))
            out.append((((i, 1), (j, 1)), m, np.conj(A)))
    return out


def _channel_entries(n, codes, full, channels):
    """(target rows, source rows, amp) per channel; targets outside a
    restricted basis are dropped (channels.py:177-192)."""
    if not full:
        order = np.argsort(codes)
        sc = codes[order]
    for selector, mask, amp in channels:
        sel = np.ones(len(codes), bool)
        for site, bit in selector:
            sel &= ((codes >> (n - 1 - int(site))) & 1) == int(bit)
        src = np.flatnonzero(sel)
        targets = codes[src] ^ mask
        if full:
            yield targets, src, amp
            continue
        pos = np.searchsorted(sc, targets)
        ok = pos < len(sc)
        ok[ok] &= sc[pos[ok]] == targets[ok]
        yield order[pos[ok]], src[ok], amp


def _is_complex(omega, exchange, gamma=None):
    return bool(np.any(np.asarray(omega).imag != 0)) or any(
        complex(e[2]).imag != 0 or complex(e[3]).imag != 0 for e in (exchange or ())) or (
        gamma is not None and bool(np.any(np.asarray(gamma) != 0)))


def hv(n, codes, omega, delta, pairs, x, exchange=None, gamma=None):
    """y = H x on the full (codes=None) or restricted basis.

    Follows ChannelKernel.matvec (channels.py:210-221): the diagonal, then
    every channel of channel_list scatters amp * x[source] into its target."""
    n = int(n)
    full = codes is None
    codes = np.arange(1 << n, dtype=np.int64) if full else np.asarray(codes, np.int64)
    x = np.asarray(x)
    vec = x.ndim == 1
    X = x.reshape(len(codes), -1)
    d = diagonal(n, codes, delta, pairs)
    cplx = np.iscomplexobj(X) or _is_complex(omega, exchange, gamma)
    if gamma is not None:
        d = d + loss_diagonal(n, codes, gamma)
    Y = (d[:, None] * X).astype(complex if cplx else X.dtype)
    for loc, src, amp in _channel_entries(n, codes, full, channel_list(n, omega, exchange)):
        np.add.at(Y, loc, (amp if cplx else amp.real) * X[src])
    return Y.reshape(x.shape) if vec else Y


def sparse_h(n, codes, omega, delta, pairs, exchange=None, gamma=None):
    """CSR H from the same channel list as hv (the reference assembles its CSR
    in assemble.py:277-393 build_H_sparse; used here for the larger CPU
    baseline samples, where a dense matrix does not fit)."""
    import scipy.sparse as sp
    n = int(n)
    full = codes is None
    codes = np.arange(1 << n, dtype=np.int64) if full else np.asarray(codes, np.int64)
    dim = len(codes)
    d = diagonal(n, codes, delta, pairs)
    cplx = _is_complex(omega, exchange, gamma)
    if gamma is not None:
        d = d + loss_diagonal(n, codes, gamma)
    rows, cols, vals = [np.arange(dim)], [np.arange(dim)], [d.astype(complex if cplx else float)]
    for loc, src, amp in _channel_entries(n, codes, full, channel_list(n, omega, exchange)):
        rows.append(loc)
        cols.append(src)
        vals.append(np.full(len(src), amp if cplx else amp.real))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(dim, dim))


def dense_h(n, codes, omega, delta, pairs, exchange=None, gamma=None):
    """Dense H by applying hv to unit vectors (small systems only)."""
    dim = (1 << n) if codes is None else len(codes)
    E = np.eye(dim, dtype=complex if _is_complex(omega, exchange, gamma) else float)
    return hv(n, codes, omega, delta, pairs, E, exchange=exchange, gamma=gamma)


# ------------------------------------------------------------------- KPM

def kpm_bounds(H):
    """emin, emax, c, r (kpm.py:82-97; dense eigvalsh replaces eigsh here)."""
    w = np.linalg.eigvalsh(H)
    emin, emax = float(w[0]), float(w[-1])
    c = 0.5 * (emin + emax)
    r = 0.5 * (emax - emin) * (1.0 + 1e-3) + 1e-12
    return emin, emax, c, r


def kpm_moments(apply_h, dim, num, probes, c, r):
    """Hutchinson moments (kpm.py:133-151): T0 z = z, T1 z = Htil z,
    T_n z = 2 Htil T_{n-1} z - T_{n-2} z, acc[n] += Re <T_n z, z>,
    mu = acc / (nvec * D)."""
    probes = np.asarray(probes, dtype=np.float64)
    acc = np.zeros(num + 1)
    def htil(v):
        return (apply_h(v) - c * v) / r
    for z in probes:
        tp = z.copy()
        tc = htil(z)
        acc[0] += tp @ z
        if num >= 1:
            acc[1] += tc @ z
        for k in range(2, num + 1):
            tn = 2 * htil(tc) - tp
            acc[k] += tn @ z
            tp, tc = tc, tn
    return acc / (len(probes) * dim)


def kpm_moments_exact(H, num, c, r):
    """Exact moments mu_n = mean T_n(lambda) (kpm.py:122-132)."""
    lam = (np.linalg.eigvalsh(H) - c) / r
    mu = np.zeros(num + 1)
    t0 = np.ones_like(lam)
    t1 = lam.copy()
    mu[0] = t0.mean()
    if num >= 1:
        mu[1] = t1.mean()
    for k in range(2, num + 1):
        t2 = 2 * lam * t1 - t0
        mu[k] = t2.mean()
        t0, t1 = t1, t2
    return mu


def jackson_kernel(num):
    """Jackson damping factors (kpm.py:109-112)."""
    k = np.arange(num + 1)
    return ((num - k + 1) * np.cos(np.pi * k / (num + 1))
            + np.sin(np.pi * k / (num + 1)) / np.tan(np.pi / (num + 1))) / (num + 1)


def dos_from_moments(mu, c, r, energies, num, use_jackson=True):
    """Jackson-damped Chebyshev DOS (kpm.py:182-189)."""
    x = (np.asarray(energies, float) - c) / r
    xn = np.clip(x, -1 + 1e-9, 1 - 1e-9)
    G = jackson_kernel(num) if use_jackson else np.ones(num + 1)
    series = mu[0] * np.ones_like(xn)
    if num >= 1:
        t0 = np.ones_like(xn)
        t1 = xn.copy()
        series += 2 * G[1] * mu[1] * t1
        for k in range(2, num + 1):
            t2 = 2 * xn * t1 - t0
            series += 2 * G[k] * mu[k] * t2
            t0, t1 = t1, t2
    return np.maximum(series / (np.pi * np.sqrt(1 - xn ** 2)) / r, 0.0)


# ------------------------------------------------------------ evolution

def segment_intervals(a, b, segments):
    """Split [a, b] at drive boundaries (runtime.py:56-60)."""
    bounds = [float(a)] + sorted({float(s['t0']) for s in segments or []
                                  if a < float(s['t0']) < b}) + [float(b)]
    return list(zip(bounds[:-1], bounds[1:]))


def segment_drive(t, segments, n):
    """Latest segment with t0 <= t, 'left' rule (runtime.py:90-114)."""
    ordered = sorted(segments, key=lambda s: float(s['t0']))
    idx = 0
    for k, s in enumerate(ordered):
        if float(s['t0']) <= t:
            idx = k
    s = ordered[idx]
    om = np.asarray(s.get('Om', np.zeros(n)), float).reshape(-1)
    ph = np.asarray(s.get('phase', np.zeros(n)), float).reshape(-1)
    de = np.asarray(s.get('delta', np.zeros(n)), float).reshape(-1)
    return om * np.exp(1j * ph), de


def evolve_segments(n, codes, pairs, segments, psi0, t_grid, exchange=None, gamma=None):
    """Piecewise-constant exact propagation (engine_ed.py:130-147): for each
    output interval and each drive piece, psi <- expm_multiply(-i CONV dt H)."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import expm_multiply
    psi = np.asarray(psi0, complex).copy()
    t = np.asarray(t_grid, float)
    out = [psi.copy()]
    cache = {}
    for k in range(1, len(t)):
        for a, b in segment_intervals(t[k - 1], t[k], segments):
            om, de = segment_drive(0.5 * (a + b), segments, n)
            key = (tuple(om), tuple(de))
            if key not in cache:
                cache[key] = (sp.csr_matrix(dense_h(n, codes, om, de, pairs, exchange=exchange, gamma=gamma))
                              if len(psi) <= 4096
                              else sparse_h(n, codes, om, de, pairs, exchange=exchange, gamma=gamma))
            psi = expm_multiply((-1j * CONV * (b - a)) * cache[key], psi)
        out.append(psi.copy())
    return out


def site_occupations(n, codes, psi):
    """<n_i> = bits @ |psi|^2 (engine_ed.py:259-263)."""
    codes = np.arange(1 << n) if codes is None else codes
    p = np.abs(np.asarray(psi)) ** 2
    return basis_bits(n, codes).astype(float) @ p


def corr_matrix(bits, p):
    """C_ij = <n_i n_j> - <n_i><n_j> with weights p (observables.py:40-47)."""
    bits = np.asarray(bits, float)
    ni = bits @ p
    return (bits * p) @ bits.T - np.outer(ni, ni)


def spin_observables(n, codes, psi):
    """sx, sy, sz, sp, sm, phase per site and xy[i, j] = <sigma+_i sigma-_j>
    on the full (codes=None) or a restricted basis (observables.py:117-205;
    flip targets outside a restricted basis drop out)."""
    n = int(n)
    v = np.asarray(psi, complex).reshape(-1)
    codes = np.arange(1 << n, dtype=np.int64) if codes is None else np.asarray(codes, np.int64)
    pos = {int(c): k for k, c in enumerate(codes)}
    p = np.abs(v) ** 2
    bits = basis_bits(n, codes).astype(bool)
    sz = np.zeros(n)
    sm = np.zeros(n, complex)
    for i in range(n):
        m = 1 << (n - 1 - i)
        sz[i] = p[~bits[i]].sum() - p[bits[i]].sum()
        for k in np.flatnonzero(~bits[i]):
            t = pos.get(int(codes[k]) | m)
            if t is not None:
                sm[i] += np.conj(v[k]) * v[t]
    xy = np.zeros((n, n), complex)
    for i in range(n):
        mi = 1 << (n - 1 - i)
        xy[i, i] = p[bits[i]].sum()
        for j in range(n):
            if j == i:
                continue
            mj = 1 << (n - 1 - j)
            for k in np.flatnonzero(~bits[i] & bits[j]):
                t = pos.get((int(codes[k]) | mi) ^ mj)
                if t is not None:
                    xy[i, j] += np.conj(v[t]) * v[k]
    phase = np.angle(sm)
    phase[np.abs(sm) < 1e-14] = np.nan
    return dict(sx=2 * sm.real, sy=2 * sm.imag, sz=sz, sp=np.conj(sm), sm=sm, phase=phase, xy_corr=xy)


def pauli_expect(n, codes, psi, terms):
    """<psi|P|psi> for P = prod sigma^{axis} on distinct sites, standard
    Pauli matrices in the (|g>, |r>) basis; on a restricted basis targets
    outside it drop out (observables.py:546-622 PauliPlan, basis form)."""
    n = int(n)
    v = np.asarray(psi, complex).reshape(-1)
    codes = np.arange(1 << n, dtype=np.int64) if codes is None else np.asarray(codes, np.int64)
    pos = {int(c): k for k, c in enumerate(codes)}
    t = codes.copy()
    ph = np.ones(len(codes), complex)
    for site, axis in terms:
        m = np.int64(1) << (n - 1 - int(site))
        bit = (codes & m) != 0
        if axis == 'z':
            ph *= np.where(bit, -1.0, 1.0)
        elif axis == 'y':
            ph *= np.where(bit, -1j, 1j)
        if axis != 'z':
            t = t ^ m
    total = 0j
    for k in range(len(codes)):
        q = pos.get(int(t[k]))
        if q is not None:
            total += np.conj(v[q]) * ph[k] * v[k]
    return total


def entropy_cut(n, codes, psi, cut, max_entries=1 << 20):
    """Bipartite von Neumann entropy (nat) between the first `cut` sites and
    the rest: full basis as observables.py:50-80 entropy_at_cut, restricted
    basis on the occupied Schmidt rows/columns as observables.py:89-114
    entropy_in_basis (None beyond max_entries)."""
    n, cut = int(n), int(cut)
    v = np.asarray(psi, complex).reshape(-1)
    if codes is None:
        sv = np.linalg.svd(v.reshape(1 << cut, 1 << (n - cut)), compute_uv=False)
        w = sv ** 2
        w = w[w > 1e-15]
        return float(-np.sum(w * np.log(w))) if w.size else 0.0
    codes = np.asarray(codes, np.int64)
    _, li = np.unique(codes >> (n - cut), return_inverse=True)
    _, ri = np.unique(codes & ((1 << (n - cut)) - 1), return_inverse=True)
    shape = (int(li.max()) + 1, int(ri.max()) + 1)
    if shape[0] * shape[1] > max_entries:
        return None
    M = np.zeros(shape, complex)
    M[li, ri] = v
    w = np.linalg.svd(M, compute_uv=False) ** 2
    w = w / w.sum()
    w = w[w > 0]
    return float(-np.sum(w * np.log(w)))


# ------------------------------------------------------------ sector scan

def sector_scan(n, delta, pairs, exchange, sectors=None):
    """Per fixed-excitation sector the lowest two eigenvalues of H restricted
    to it, Omega = 0 (sector_scan.py:61-132; dense eigh per sector replaces
    its per-sector Krylov solve).  Returns (E0, best sector, rows) with rows
    (k, dim, E0, gap)."""
    n = int(n)
    ks = list(range(n + 1)) if sectors is None else [int(k) for k in sectors]
    rows = []
    for k in ks:
        codes = number_sector_basis(n, k)
        H = dense_h(n, codes, np.zeros(n), delta, pairs, exchange=exchange)
        w = np.linalg.eigvalsh(H)
        rows.append((k, len(codes), float(w[0]), float(w[1] - w[0]) if len(w) > 1 else 0.0))
    best = min(rows, key=lambda r: r[2])
    return best[2], best[0], rows


# ---------------------------------------------------------------- spectrum

def lanczos_tridiag(apply_h, phi, k, reorth=True):
    """alphas, betas, n of the Lanczos run from phi (spectrum.py:34-103):
    q_0 = phi/|phi|, alpha_j = Re<q_j, H q_j>, three-term recurrence, full
    Gram-Schmidt twice per step against the stored q's, stop at beta <= 1e-12
    or when the Krylov space is the whole space; beta_j kept while another
    step follows."""
    v = np.asarray(phi, complex).reshape(-1)
    dim = v.size
    k = min(int(k), dim)
    q = v / np.linalg.norm(v)
    q_prev = np.zeros_like(q)
    al, be, basis = [], [], []
    beta = 0.0
    for j in range(k):
        basis.append(q)
        w = np.asarray(apply_h(q), complex)
        alpha = float(np.vdot(q, w).real)
        w = w - alpha * q - (beta * q_prev if j else 0.0)
        if reorth:
            for _ in range(2):
                for b in basis:
                    w = w - np.vdot(b, w) * b
        beta = float(np.linalg.norm(w))
        al.append(alpha)
        if beta <= 1e-12 or len(al) >= dim:
            break
        if j + 1 < k:
            be.append(beta)
        q_prev, q = q, w / beta
    return np.asarray(al), np.asarray(be), len(al)

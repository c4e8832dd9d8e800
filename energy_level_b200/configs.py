"""Seeded synthetic Rydberg lattices for the five benchmark workloads.

Units follow the reference engine: energies in cyclic MHz, times in ns
(evolve_util.py:12, CONV = 2 pi 1e-3).  A quoted angular value "2 pi x f MHz"
is the reference input f; the detuning enters the reference diagonal as
+delta n (channels.py:68-73), so H = ... - Delta n means delta = -Delta.
Pair couplings are C6 / r^6 for every pair (the role of
calib_build.py:121-166 from_positions with a van der Waals kernel).

Workloads:
  chain12   open chain N=12, a=5.5 um, Omega=2, Delta=1, full basis (FP64 GS)
  square25  5x5 square, a=6 um, Omega=1.5, Delta_i ~ U(-3,3) seed 1, full 2^25
            (KPM DOS, 1024 moments, 32 probes)
  chain31   chain N=31 NN blockade (dim F(33)=3,524,578), Omega=2, Delta
            linear -6..+6 over 3000 ns in 300 piecewise-constant steps
  batch512  512 chains, N ~ U{16..22}, positions i*5.5 + U(-0.3, 0.3) um,
            Omega=2, Delta/Omega ~ U(0, 3), NN blockade sectors (seed 4)
  ring20    ring N=20, NN spacing 5.5 um, NN blockade incl. (19, 0),
            200 steps of (Omega_k, Delta_k) from a smooth random ramp (seed 5),
            objective |<Z2|psi(T)>|^2
  xy_chain  dipolar XY chain (Omega = 0): exchange J_ij = j0 (a / r_ij)^3 for
            every pair (I2) plus a van der Waals V_ij (I1), random fields
            delta_i ~ U(-1, 1); number-conserving, so it splits into the
            fixed-excitation sectors that the sector scan solves one by one
"""
from __future__ import annotations

import numpy as np

C6_70S = 862690.0      # MHz um^6  (2 pi x 862690 MHz um^6 quoted angular)


def pairs_from_positions(pos, c6=C6_70S):
    pos = np.asarray(pos, float)
    n = len(pos)
    out = []
    for i in range(n):
        for j in range(i + 1, n):
            r = float(np.linalg.norm(pos[j] - pos[i]))
            out.append((i, j, c6 / r ** 6))
    return out


def calib_from_positions(pos, c6=C6_70S):
    """calib dict in the reference's shape (atoms + pairs with V/J/A)."""
    pos = np.asarray(pos, float)
    if pos.shape[1] == 2:
        pos = np.column_stack([pos, np.zeros(len(pos))])
    pairs = [{'i': i, 'j': j, 'V': V, 'J': 0.0, 'A': 0.0}
             for i, j, V in pairs_from_positions(pos, c6)]
    return {'atoms': [{'id': i, 'pos': [float(x) for x in p]} for i, p in enumerate(pos)],
            'pairs': pairs, 'terms': ['I1']}


def chain_positions(n, a=5.5, jitter=None):
    x = np.arange(n, dtype=float) * a
    if jitter is not None:
        x = x + jitter
    return np.column_stack([x, np.zeros(n), np.zeros(n)])


def chain_edges(n):
    return [[i, i + 1] for i in range(n - 1)]


def ring_edges(n):
    return chain_edges(n) + [[n - 1, 0]]


def chain12():
    n = 12
    calib = calib_from_positions(chain_positions(n))
    return dict(name='chain12', n=n, calib=calib, Om=np.full(n, 2.0), delta=np.full(n, -1.0),
                edges=None, tol=1e-12, seed=0)


def square25(seed=1):
    n = 25
    pos = [[6.0 * m, 6.0 * k, 0.0] for m in range(5) for k in range(5)]
    calib = calib_from_positions(pos)
    Delta = np.random.default_rng(seed).uniform(-3.0, 3.0, n)
    return dict(name='square25', n=n, calib=calib, Om=np.full(n, 1.5), delta=-Delta,
                edges=None, num=1024, nvec=32, probe_seed=2)


def chain31(steps=300, total_ns=3000.0):
    n = 31
    calib = calib_from_positions(chain_positions(n))
    dt = total_ns / steps
    segments = []
    for k in range(steps):
        Delta = -6.0 + 12.0 * (k * dt) / total_ns
        segments.append({'t0': k * dt, 'Om': np.full(n, 2.0), 'delta': np.full(n, -Delta)})
    return dict(name='chain31', n=n, calib=calib, edges=chain_edges(n), segments=segments,
                t_grid=np.array([0.0, total_ns]), psi0='g' * n)


def batch512(count=512, seed=4):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(16, 23))
        jit = rng.uniform(-0.3, 0.3, n)
        calib = calib_from_positions(chain_positions(n, jitter=jit))
        Delta = 2.0 * rng.uniform(0.0, 3.0)
        out.append(dict(n=n, calib=calib, Om=np.full(n, 2.0), delta=np.full(n, -Delta),
                        edges=chain_edges(n)))
    return out


def ring_positions(n, spacing=5.5):
    R = spacing / (2.0 * np.sin(np.pi / n))
    ang = 2.0 * np.pi * np.arange(n) / n
    return np.column_stack([R * np.cos(ang), R * np.sin(ang), np.zeros(n)])


def smooth_ramp(steps, seed, total_ns):
    """Per-step (Omega_k, Delta_k): 4 low-frequency sines around Omega = 2 and
    around a linear Delta sweep -6 -> +6."""
    rng = np.random.default_rng(seed)
    s = (np.arange(steps) + 0.5) / steps
    om = np.full(steps, 2.0)
    de = -6.0 + 12.0 * s
    for q in range(1, 5):
        om += rng.uniform(-0.3, 0.3) * np.sin(np.pi * q * s + rng.uniform(0, 2 * np.pi))
        de += rng.uniform(-0.5, 0.5) * np.sin(np.pi * q * s + rng.uniform(0, 2 * np.pi))
    return om, de


def ring20(n=20, steps=200, seed=5, total_ns=2000.0):
    calib = calib_from_positions(ring_positions(n))
    om, Delta = smooth_ramp(steps, seed, total_ns)
    return dict(name='ring%d' % n, n=n, calib=calib, edges=ring_edges(n), omega_k=om,
                delta_k=-Delta, tau=np.full(steps, total_ns / steps),
                target='rg' * (n // 2) + ('r' if n % 2 else ''), psi0='g' * n)


def xy_chain(n, a=5.5, j0=-0.7, seed=7, c6=C6_70S, v_scale=1e-3):
    """Dipolar XY chain: calib with J (I2) and a weak V (I1) on every pair,
    per-site delta ~ U(-1, 1) (seed), Om = 0."""
    rng = np.random.default_rng(seed)
    pos = chain_positions(n, a=a)
    pairs = []
    for i in range(n):
        for j in range(i + 1, n):
            r = float(np.linalg.norm(pos[j] - pos[i]))
            pairs.append({'i': i, 'j': j, 'V': v_scale * c6 / r ** 6, 'J': j0 * (a / r) ** 3, 'A': 0.0})
    calib = {'atoms': [{'id': i, 'pos': [float(x) for x in p]} for i, p in enumerate(pos)],
             'pairs': pairs, 'terms': ['I1', 'I2']}
    return dict(calib=calib, n=n, Om=np.zeros(n), delta=rng.uniform(-1.0, 1.0, n))

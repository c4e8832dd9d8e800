"""Sector-by-sector ground-state scan on the B200 path.

``scan_ground_sectors`` has the signature and result of the reference's
sector_scan.py:61-132: for a number-conserving model (Omega = 0, no I3 pair
creation) it solves the ground state of every fixed-excitation sector
k = 0..N (or the given ``sectors``) and returns the lowest.  Each sector is a
native fixed-popcount basis (ranked through prefix/suffix tables, no code
list on the host) with its own Hamiltonian, solved by the device Lanczos with
Ritz-residual certification; the exchange channels J (I2) move excitations
inside the sector.  Small sectors are solved by the same device Lanczos,
whose Krylov space then spans the sector, instead of a host dense eigh
(sector_scan.py:38-46).

The sectors are independent (sector_scan.py:18 notes the scan is
parallelisable): ``workers`` host threads, each with its own library
context on its own CUDA stream, solve their share of the sectors (largest
first, round-robin), so the latency-bound Lanczos iterations of small
sectors overlap the large ones.  Results are assembled in sector order and
do not depend on the schedule.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import model, solvers

__all__ = ['scan_ground_sectors', 'SectorScan']


def _device_index(device):
    if isinstance(device, str):
        if device.startswith('cpu'):
            raise RuntimeError('CUDA 不可用')
        return int(device.split(':')[1]) if ':' in device else 0
    return int(device or 0)


class SectorScan:
    """The fixed-excitation sectors of one model, set up once on ``workers``
    contexts (one CUDA stream each) and solved by ``run()``.

    Set-up builds every sector's basis and Hamiltonian on the device (the
    part of the scan that does not depend on the solve); ``run()`` solves all
    sectors.  Sectors go round-robin, largest first, to the workers; a
    context (its workspace and result scalars) serves one thread only, so
    each worker solves the sectors set up on its own context."""

    def __init__(self, calib, delta=None, Om=None, gamma=None, terms=None, *, sectors=None,
                 device='cuda', workers=8, memory_budget_mb=None, dtype='float64', m=48):
        import threading
        import torch
        atoms = calib.get('atoms') or []
        n = len(atoms)
        if n <= 0:
            raise ValueError('calib 需要 atoms')
        delta = np.zeros(n) if delta is None else np.asarray(delta, float)
        Om = np.zeros(n, complex) if Om is None else np.asarray(Om, complex)
        gamma = np.zeros(n) if gamma is None else np.asarray(gamma, float)
        if np.any(gamma):
            raise ValueError('扫描基态要求厄米 Hamiltonian（gamma=0）')
        model.check_number_conserving(calib, Om, terms)
        ks = list(range(n + 1)) if sectors is None else [int(k) for k in sectors]
        for k in ks:
            if not 0 <= k <= n:
                raise ValueError('sector 必须在 [0, N]')
        self.n, self.ks = n, ks
        # the calib is parsed once; every sector gets its basis and H from it
        exchange = []
        _, om_arr, de_arr, vpairs = model.model_arrays(calib, Om, delta, gamma, terms, exchange=exchange)
        self.dev = _device_index(device)
        self.nw = max(1, min(int(workers), len(ks)))
        t_w = time.perf_counter()
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(self.nw)]
        self.ctxs = []
        with torch.cuda.device(self.dev):
            for st in self.streams:
                with torch.cuda.stream(st):
                    self.ctxs.append(model.Context(self.dev))
        torch.cuda.synchronize(self.dev)
        self.warmup_seconds = time.perf_counter() - t_w
        # sectors largest first, spread round-robin over the workers' contexts
        from math import comb
        self.order = sorted(ks, key=lambda k: -comb(n, k))
        self.owner = {k: i % self.nw for i, k in enumerate(self.order)}
        self.setup_seconds = {}
        self.sec = {}
        lock = threading.Lock()
        itemsize = {'float32': 4, 'float64': 8, 'complex64': 8, 'complex128': 16}.get(dtype, 16)

        def build(w):
            with torch.cuda.device(self.dev), torch.cuda.stream(self.streams[w]):
                for k in self.order:
                    if self.owner[k] != w:
                        continue
                    t0 = time.perf_counter()
                    basis = model.Basis(self.ctxs[w], n, kind='charge', k=k)
                    ham = model.Hamiltonian(self.ctxs[w], basis, om_arr, de_arr, vpairs, exchange=exchange)
                    if memory_budget_mb is not None and basis.dim * itemsize * (min(m, basis.dim) + 5) > \
                            float(memory_budget_mb) * 1024 ** 2:
                        raise MemoryError('GPU Krylov/transition 保守内存估算超过 memory_budget_mb')
                    with lock:
                        self.sec[k] = (basis, ham)
                        self.setup_seconds[k] = time.perf_counter() - t0
                torch.cuda.current_stream().synchronize()
        self._parallel(build)

    def _parallel(self, fn):
        if self.nw == 1:
            fn(0)
            return
        with ThreadPoolExecutor(max_workers=self.nw) as ex:
            for f in [ex.submit(fn, w) for w in range(self.nw)]:
                f.result()

    def run(self, dtype='float64', m=48, tol=None, seed=0):
        """Solve every sector; rows in sector order (keys of sector_scan.py:84-132)."""
        import torch
        if dtype not in ('float64', 'complex128', 'float32', 'complex64'):
            raise ValueError('dtype 必须为 float32/float64/complex64/complex128')
        double = dtype in ('float64', 'complex128')
        tolerance = float(tol if tol is not None else (1e-9 if double else 2e-5))
        m = max(2, int(m))
        rows = {}

        def worker(w):
            with torch.cuda.device(self.dev), torch.cuda.stream(self.streams[w]):
                # a context (workspace, scalars) serves one thread: each worker
                # solves the sectors set up on its own context, largest first
                for k in self.order:
                    if self.owner[k] != w:
                        continue
                    basis, ham = self.sec[k]
                    t0 = time.perf_counter()
                    r = solvers.lanczos_ground(ham, dtype=dtype, seed=seed, max_iter=m, max_restarts=8,
                                               tol=tolerance, nev=min(2, basis.dim))
                    ev = np.asarray(r['evals'], float)
                    res = np.asarray(r['residuals'], float).reshape(-1)
                    rows[k] = dict(sector=k, dim=int(basis.dim), E0=float(ev[0]),
                                   gap=float(ev[1] - ev[0]) if ev.size > 1 else 0.0,
                                   residual=float(res[0]) if res.size else 0.0,
                                   converged=bool(r['converged']), backend='b200-lanczos',
                                   seconds=time.perf_counter() - t0 + self.setup_seconds.get(k, 0.0))
                torch.cuda.current_stream().synchronize()
        self._parallel(worker)
        return [rows[k] for k in self.ks]

    def copied_bytes(self):
        """(host->device, device->host) bytes the scan's contexts have copied."""
        a = b = 0
        for c in self.ctxs:
            x, y = c.copied_bytes
            a += x
            b += y
        return a, b

    def close(self):
        self.sec.clear()
        for c in self.ctxs:
            c.close()
        self.ctxs = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def scan_ground_sectors(calib, delta=None, Om=None, gamma=None, terms=None, *,
                        sectors=None, backend='auto', m=48, tol=None,
                        dtype='float64', device='cuda', memory_budget_mb=None,
                        dense_max=2048, seed=0, progress=None, workers=8):
    """Ground state of each fixed-excitation sector; the lowest wins.

    Returns dict(E0, sector, per_sector=[{sector, dim, E0, gap, residual,
    converged, backend, seconds}], total_seconds, warmup_seconds,
    sectors_run, converged, dimension_sum, full_dimension) as
    sector_scan.py:84-132."""
    if backend not in ('auto', 'b200-lanczos', 'gpu-lanczos'):
        raise ValueError('scan backend must be auto, b200-lanczos or gpu-lanczos')
    if dtype not in ('float64', 'complex128', 'float32', 'complex64'):
        raise ValueError('dtype 必须为 float32/float64/complex64/complex128')
    t_start = time.perf_counter()
    scan = SectorScan(calib, delta, Om, gamma, terms, sectors=sectors, device=device, workers=workers,
                      memory_budget_mb=memory_budget_mb, dtype=dtype, m=m)
    try:
        t_start += scan.warmup_seconds
        rows = scan.run(dtype=dtype, m=m, tol=tol, seed=seed)
        moved = scan.copied_bytes()
    finally:
        scan.close()
    best = None
    for row in rows:
        if best is None or row['E0'] < best['E0']:
            best = dict(row)
        if progress is not None:
            progress(row)
    total = time.perf_counter() - t_start
    return dict(E0=best['E0'], sector=best['sector'], per_sector=rows,
                total_seconds=total, warmup_seconds=scan.warmup_seconds, sectors_run=scan.ks,
                converged=all(r['converged'] for r in rows),
                dimension_sum=int(sum(r['dim'] for r in rows)),
                full_dimension=int(1 << scan.n), transfer_bytes=moved)

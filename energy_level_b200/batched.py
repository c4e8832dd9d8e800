"""Batched ground states: hundreds of independent instances, one launch.

``BatchedGroundStates`` describes the batch once on the device
(el_batch_create), runs it as ONE persistent kernel (el_batch_run: CTAs pull
instances from an atomic queue, largest sector first) and reads the results
(el_batch_results).  ``autotune`` picks threads per CTA and CTAs per SM by
timing the candidates on the batch itself (CUDA events), ``capture`` records
the run in a CUDA graph for repeated solves.  The per-instance result keys
follow the reference's ground-state dicts (E0, gap, residuals, converged;
matrix_free.py:273-276) as arrays over the batch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .core import _torch, default_context
from .model import model_columns

_TUNED = {}


def _layout(n, edges):
    """Basis layout of one instance: the full basis without edges, the
    arithmetic Zeckendorf layouts for a nearest-neighbour path or cycle, and
    a code table for any other blockade graph.  Returns (layout, edge list)."""
    if not edges:
        return _lib.EL_LAYOUT_FULL, []
    es = sorted({tuple(sorted((int(a), int(b)))) for a, b in edges})
    for a, b in es:
        if a == b or a < 0 or b >= n:
            raise ValueError('bad blockade edge (%d, %d) for %d sites' % (a, b, n))
    chain = [(i, i + 1) for i in range(n - 1)]
    if es == chain:
        return _lib.EL_LAYOUT_CHAIN, es
    if n >= 3 and es == sorted(chain + [(0, n - 1)]):
        return _lib.EL_LAYOUT_RING, es
    return _lib.EL_LAYOUT_TABLE, es


def pack_instances(instances):
    """Host arrays of el_batch_create_graph for a list of instances: [n
    int32, layout int32, Omega float64 (concatenated), delta float64, pair
    offsets int32 [count + 1], i int32, j int32, V float64, edge offsets
    int32 [count + 1], edge ends int32, int32] (one dummy entry where a list
    is empty).  Raises the model's errors for an invalid instance."""
    ns, lays, om, de, npair, pi, pj, V = [], [], [], [], [], [], [], []
    nedge, ea, eb = [], [], []
    for inst in instances:
        n, o, d, (i, j, v) = model_columns(inst['calib'], inst.get('Om'), inst.get('delta'),
                                           inst.get('gamma'), inst.get('terms'))
        if np.any(o.imag != 0):
            raise ValueError('batched solves need real Omega')
        ns.append(n)
        lay, es = _layout(n, inst.get('edges'))
        lays.append(lay)
        ea.append([a for a, _ in es]); eb.append([b for _, b in es])
        nedge.append(len(es))
        om.append(o.real)
        de.append(d)
        pi.append(i); pj.append(j); V.append(v)
        npair.append(len(v))
    arr = lambda x, t: np.ascontiguousarray(np.asarray(x, dtype=t))
    cat = lambda x, t, empty: arr(np.concatenate(x) if sum(map(len, x)) else [empty], t)
    poff = np.concatenate([[0], np.cumsum(npair, dtype=np.int64)])
    eoff = np.concatenate([[0], np.cumsum(nedge, dtype=np.int64)])
    return [arr(ns, np.int32), arr(lays, np.int32), cat(om, np.float64, 0.0), cat(de, np.float64, 0.0),
            arr(poff, np.int32), cat(pi, np.int32, 0), cat(pj, np.int32, 0), cat(V, np.float64, 0.0),
            arr(eoff, np.int32), cat(ea, np.int32, 0), cat(eb, np.int32, 0)]


class BatchedGroundStates:
    """A batch of instances on the device.  occupations=True also forms each
    ground state's site occupations <n_i> (the n_atom of the reference's
    batched_ground_state, equilibrium.py:251-311) from the Krylov basis in
    every run; results() then carries an 'n_atom' array [count, max n]."""

    def __init__(self, instances, dtype='float32', max_iter=200, tol=None, device=0, ctx=None,
                 occupations=False):
        if dtype not in ('float32', 'float64'):
            raise ValueError('dtype 必须为 float32/float64')
        self.ctx = ctx or default_context(device)
        self._keep = pack_instances(instances)
        self.count = len(self._keep[0])
        self.n_sites = self._keep[0].astype(np.int64)
        self.dtype = dtype
        self.tol = float(tol if tol is not None else (1e-5 if dtype == 'float32' else 1e-10))
        k = self._keep
        h = C.c_void_p()
        self.ctx.call('el_batch_create_graph', C.c_int(self.count), C.c_void_p(k[0].ctypes.data),
                      C.c_void_p(k[1].ctypes.data), _lib.dptr(k[2]), _lib.dptr(k[3]),
                      C.c_void_p(k[4].ctypes.data), C.c_void_p(k[5].ctypes.data),
                      C.c_void_p(k[6].ctypes.data), _lib.dptr(k[7]), C.c_void_p(k[8].ctypes.data),
                      C.c_void_p(k[9].ctypes.data), C.c_void_p(k[10].ctypes.data),
                      C.c_int(_lib.DTYPES[dtype]), C.c_int(int(max_iter)), C.c_double(self.tol), C.byref(h))
        self.handle = h
        self.occupations = bool(occupations)
        if self.occupations:
            self.ctx.call('el_batch_want_occupations', self.handle, C.c_int(1))
        self.config = (512, 1)
        self.signature = (self.count, tuple(np.bincount(self.n_sites).tolist()), dtype, int(max_iter))

    def run(self, threads=None, ctas_per_sm=None, seed=0):
        t, c = self.config
        self.ctx.call('el_batch_run', self.handle, C.c_int(int(threads or t)),
                      C.c_int(int(ctas_per_sm or c)), C.c_uint64(int(seed)))

    def run_coop(self, seed=0, check_every=8, reorth_passes=2):
        """Each instance with the whole GPU: one cooperative launch per
        instance, Krylov slices in shared memory, full reorthogonalisation
        every step (el_batch_run_coop); for a few instances of a few
        thousand rows.  reorth_passes: Gram-Schmidt passes per step; one
        pass forms beta from |w|^2 - |c|^2, which loses accuracy when beta
        is small against |H v| (near an invariant subspace), so two is the
        safe default."""
        self.ctx.call('el_batch_run_coop', self.handle, C.c_int(int(reorth_passes)), C.c_int(int(check_every)),
                      C.c_uint64(int(seed)))

    def set_wait_limit(self, polls=1 << 22):
        """Polls each grid-barrier wait of run_coop makes before the solve
        gives up with RuntimeError (EL_ECUDA); see el_batch_set_wait_limit."""
        self.ctx.call('el_batch_set_wait_limit', self.handle, C.c_int32(int(polls)))

    def results(self):
        e0 = np.zeros(self.count)
        gap = np.zeros(self.count)
        res = np.zeros(self.count)
        it = np.zeros(self.count, np.int32)
        cv = np.zeros(self.count, np.int32)
        self.ctx.call('el_batch_results', self.handle, _lib.dptr(e0), _lib.dptr(gap), _lib.dptr(res),
                      C.c_void_p(it.ctypes.data), C.c_void_p(cv.ctypes.data))
        out = dict(E0=e0, gap=gap, residuals=res, iters=it, converged=cv.astype(bool),
                   backend='b200-batch-lanczos', dtype=self.dtype, tolerance=self.tol)
        if self.occupations:
            nat = np.zeros((self.count, 40))
            self.ctx.call('el_batch_occupations', self.handle, _lib.dptr(nat))
            out['n_atom'] = nat[:, :int(self.n_sites.max())]
        return out

    def autotune(self, candidates=((256, 1), (256, 2), (512, 1), (512, 2), (1024, 1)), reps=1):
        """Time each (threads, ctas_per_sm) on this batch; keep the fastest."""
        torch = _torch()
        if self.signature in _TUNED:
            self.config = _TUNED[self.signature][0]
            return _TUNED[self.signature]
        timings = {}
        stream = torch.cuda.current_stream()
        for cand in candidates:
            self.run(*cand)            # sizes the workspace, warms the code path
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(reps):
                self.run(*cand)
            ev1.record(stream)
            torch.cuda.synchronize()
            timings[cand] = ev0.elapsed_time(ev1) / reps
        best = min(timings, key=timings.get)
        self.config = best
        _TUNED[self.signature] = (best, timings)
        return best, timings

    def capture(self, seed=0):
        """CUDA graph of one batched solve with the current configuration."""
        torch = _torch()
        self.run(seed=seed)            # workspace sized outside capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(seed=seed)
        return g

    def close(self):
        if getattr(self, 'handle', None):
            self.ctx.lib.el_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


COOP_MAX_INSTANCES = 8


def batched_ground_states(instances, dtype='float32', max_iter=200, tol=None, device=0, tune=False,
                          mode='auto', occupations=True):
    """Ground energies, gaps and (occupations=True) site occupations n_atom
    of many instances: the keys of the reference's batched_ground_state
    (E0, gap, n_atom, backend; equilibrium.py:251-311) plus residuals,
    iterations and convergence flags.  mode 'batch': one persistent launch,
    one CTA per instance; 'coop': one cooperative launch per instance over
    many CTAs; 'auto': 'coop' for a few instances (<= COOP_MAX_INSTANCES)
    that fit it, else 'batch'."""
    if mode not in ('auto', 'batch', 'coop'):
        raise ValueError("mode must be 'auto', 'batch' or 'coop'")
    b = BatchedGroundStates(instances, dtype=dtype, max_iter=max_iter, tol=tol, device=device,
                            occupations=occupations)
    used = 'batch'
    try:
        if mode == 'coop' or (mode == 'auto' and b.count <= COOP_MAX_INSTANCES):
            try:
                b.run_coop(check_every=16)
                used = 'coop'
            except ValueError:
                if mode == 'coop':
                    raise
        if used == 'batch':
            if tune:
                b.autotune()
            b.run()
        out = b.results()
        out['config'] = b.config if used == 'batch' else 'coop'
        out['mode'] = used
    finally:
        b.close()
    return out

"""Matrix-free ground states and operators on the B200 path.

``b200_lanczos_ground_state`` takes the arguments of the reference's
torch_lanczos_ground_state (matrix_free.py:118-121) plus ``plan`` and returns
the same keys (matrix_free.py:273-286): E0, gap, evals, residuals, converged,
backend, dim, krylov_dim, restarts, tolerance[, vec, warning].  Unlike the
reference GPU path it accepts projected blockade plans (eq_route.py:690-691
refuses them there).  Residuals are the true ||H x - theta x|| of the
returned Ritz vectors, certified against tol * max(1, |theta|) as in
matrix_free.py:262-264.

``hamiltonian_operator`` is the device counterpart of
hamiltonian_linear_operator (matrix_free.py:51-62): a scipy LinearOperator
whose matvec copies the host vector in, applies H on the GPU and copies the
result back.
"""
from __future__ import annotations

import numpy as np

from . import model, solvers


def b200_lanczos_ground_state(calib, Om=None, delta=None, gamma=None, terms=None,
                              basis_indices=None, m=300, seed=0, dtype='float64', device='cuda',
                              tol=None, max_restarts=8, return_state=False, memory_budget_mb=None,
                              plan=None, reorth='partial', nev=2):
    if dtype not in ('float64', 'complex128', 'float32', 'complex64'):
        raise ValueError('dtype 必须为 float32/float64/complex64/complex128')
    if int(m) < 2 or int(max_restarts) < 0:
        raise ValueError('m 必须 >=2，max_restarts 必须 >=0')
    ctx, basis, ham, perm = model.build(calib, Om, delta, gamma, terms, plan=plan,
                                        basis_indices=basis_indices, device=device)
    double = dtype in ('float64', 'complex128')
    cplx = dtype.startswith('complex') or ham.complex_drive
    vdt = ('complex128' if double else 'complex64') if cplx else ('float64' if double else 'float32')
    itemsize = {'float32': 4, 'float64': 8, 'complex64': 8, 'complex128': 16}[vdt]
    kry = int(min(int(m), basis.dim))
    required = basis.dim * itemsize * (kry + 5)
    if memory_budget_mb is not None and required > float(memory_budget_mb) * 1024 ** 2:
        raise MemoryError('GPU Krylov/transition 保守内存估算超过 memory_budget_mb')
    tolerance = float(tol if tol is not None else (1e-9 if double else 2e-5))
    if tolerance <= 0 or not np.isfinite(tolerance):
        raise ValueError('tol 必须为正有限数')
    r = solvers.lanczos_ground(ham, dtype=vdt, seed=seed, max_iter=kry, max_restarts=max_restarts,
                               tol=tolerance, nev=min(int(nev), basis.dim), reorth=reorth,
                               return_vec=return_state)
    ev = np.asarray(r['evals'], float)
    conv = bool(r['converged'])
    out = dict(E0=float(ev[0]),
               gap=float(ev[1] - ev[0]) if conv and len(ev) > 1 else float('nan'),
               evals=ev, residuals=np.asarray(r['residuals'], float), converged=conv,
               backend='b200-lanczos', dim=basis.dim, krylov_dim=r['iters'],
               restarts=max(0, -(-r['iters'] // max(kry, 1)) - 1), tolerance=tolerance,
               dtype=vdt)
    if not conv:
        out['warning'] = '最低本征对未全部达到残差容限；gap 未报告'
    if plan is not None and plan.get('projected'):
        out['basis_states'] = basis.codes().cpu().numpy()
    if return_state:
        vec = r['vec'].detach().cpu().numpy()
        if perm is not None:
            back = np.empty_like(vec)
            back[perm] = vec
            vec = back
        out['vec'] = vec.astype(np.complex128)
    return out


def hamiltonian_operator(calib, Om=None, delta=None, gamma=None, terms=None, basis_indices=None,
                         plan=None, device='cuda', dtype='complex128'):
    """scipy LinearOperator applying H on the GPU (host vectors in and out)."""
    import ctypes as C
    import scipy.sparse.linalg as spla
    from . import _lib
    ctx, basis, ham, perm = model.build(calib, Om, delta, gamma, terms, plan=plan,
                                        basis_indices=basis_indices, device=device)
    code = _lib.DTYPES[dtype]
    npdt = np.dtype(dtype)

    def matvec(v):
        x = np.asarray(v, npdt).reshape(-1)
        if x.size != basis.dim:
            raise ValueError('通道内核：向量长度 %d ≠ 基维度 %d' % (x.size, basis.dim))
        if perm is not None:
            x = x[perm]
        x = np.ascontiguousarray(x)
        y = np.empty_like(x)
        ctx.call('el_hv_host', ham.handle, C.c_int(code), C.c_int(1),
                 C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data))
        if perm is not None:
            back = np.empty_like(y)
            back[perm] = y
            y = back
        return y

    op = spla.LinearOperator((basis.dim, basis.dim), matvec=matvec, dtype=npdt)
    op._b200 = (ctx, basis, ham)   # keep the handles alive with the operator
    return op

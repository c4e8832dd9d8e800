"""Pulse gradients of a fidelity or diagonal observable (adjoint method).

``pulse_gradient`` runs el_adjoint_pulse: forward evolution through K
piecewise-constant steps (Chebyshev propagator, one checkpoint per step),
then the reverse recurrence through each step's expansion, giving
dF/dOmega_k and dF/dDelta_k of the discretised map in one pass.
``PulseFidelity`` wraps it as a torch.autograd.Function so a pulse can be
optimised with torch optimisers; the native gradient is computed together
with F in forward() and scaled by the incoming gradient in backward().

Conventions: Omega_k multiplies every site's Rabi frequency (times an
optional site shape), Delta_k enters H as -Delta_k n_i (the reference's delta
is -Delta, channels.py:68-73), tau_k in ns, energies in cyclic MHz.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, model
from .core import _torch
from .state import state_vector


class PulseProblem:
    """Basis, couplings and end states of a pulse-optimisation problem."""

    def __init__(self, calib, psi0, target=None, observable=None, plan=None, dtype='complex64',
                 omega_shape=None, delta_shape=None, device='cuda', tol=None):
        n = len(calib['atoms'])
        # the reverse recurrence differentiates the Omega/delta/V model: a calib
        # with J or A channels in use is refused before anything is built
        model.model_columns(calib, np.zeros(n), np.zeros(n))
        torch = _torch()
        ctx, basis, ham, _ = model.build(calib, np.zeros(n), np.zeros(n), plan=plan, device=device)
        self.ctx, self.basis, self.ham, self.n = ctx, basis, ham, n
        self.dtype = dtype
        self.tol = float(tol if tol is not None else (1e-7 if dtype == 'complex64' else 1e-13))
        codes = basis.codes().cpu().numpy() if (plan is not None and plan.get('projected')) else None
        self.codes = codes
        td = getattr(torch, dtype)
        self.psi0 = torch.as_tensor(state_vector(psi0, n, codes), dtype=td, device=ctx.device)
        self.target = None
        self.obs = None
        if target is not None:
            self.target = torch.as_tensor(state_vector(target, n, codes), dtype=td, device=ctx.device)
        elif observable is not None:
            self.obs = torch.as_tensor(np.asarray(observable, float), dtype=torch.float64, device=ctx.device)
            if self.obs.numel() != basis.dim:
                raise ValueError('observable must have one value per basis state')
        else:
            raise ValueError('give a target state or a diagonal observable')
        self.oshape = None if omega_shape is None else np.ascontiguousarray(omega_shape, float)
        self.dshape = None if delta_shape is None else np.ascontiguousarray(delta_shape, float)

    def set_schedule(self, mode='auto'):
        """'coop' (and 'auto', the default): the whole gradient as one
        cooperative launch with grid barriers between its sweeps; 'stream':
        one launch per Chebyshev and reverse term (el_adjoint_set_mode)."""
        modes = {'auto': _lib.EL_ADJ_AUTO, 'stream': _lib.EL_ADJ_STREAM, 'coop': _lib.EL_ADJ_COOP}
        if mode not in modes:
            raise ValueError("schedule must be 'auto', 'stream' or 'coop'")
        self.ctx.call('el_adjoint_set_mode', C.c_int(modes[mode]))

    def evaluate(self, tau, omega_k, delta_k, want_state=False):
        """(F, dF/dOmega_k, dF/dDelta_k[, psi_K])."""
        torch = _torch()
        tau = np.ascontiguousarray(tau, float)
        om = np.ascontiguousarray(omega_k, float)
        de = np.ascontiguousarray(delta_k, float)
        K = len(tau)
        if om.shape != (K,) or de.shape != (K,):
            raise ValueError('tau, omega_k and delta_k must have the same length')
        F = C.c_double()
        go = np.zeros(K)
        gd = np.zeros(K)
        out = torch.empty_like(self.psi0) if want_state else None
        self.ctx.call('el_adjoint_pulse', self.ham.handle, C.c_int(_lib.DTYPES[self.dtype]), C.c_int(K),
                      _lib.dptr(tau), _lib.dptr(om), _lib.dptr(de), _lib.dptr(self.oshape),
                      _lib.dptr(self.dshape), C.c_void_p(self.psi0.data_ptr()),
                      C.c_void_p(self.target.data_ptr()) if self.target is not None else None,
                      C.c_void_p(self.obs.data_ptr()) if self.obs is not None else None,
                      C.c_double(self.tol), C.byref(F), _lib.dptr(go), _lib.dptr(gd),
                      C.c_void_p(out.data_ptr()) if out is not None else None)
        if want_state:
            return float(F.value), go, gd, out
        return float(F.value), go, gd


def pulse_gradient(problem: PulseProblem, tau, omega_k, delta_k):
    F, go, gd = problem.evaluate(tau, omega_k, delta_k)
    return dict(F=F, grad_omega=go, grad_delta=gd, backend='b200-adjoint', dtype=problem.dtype)


def _function():
    torch = _torch()

    class PulseFidelity(torch.autograd.Function):
        """F(Omega_k, Delta_k) with the native adjoint gradient."""

        @staticmethod
        def forward(ctx, omega_k, delta_k, problem, tau):
            F, go, gd = problem.evaluate(tau, omega_k.detach().cpu().numpy(),
                                         delta_k.detach().cpu().numpy())
            ctx.save_for_backward(torch.as_tensor(go, dtype=omega_k.dtype, device=omega_k.device),
                                  torch.as_tensor(gd, dtype=delta_k.dtype, device=delta_k.device))
            return torch.tensor(F, dtype=omega_k.dtype, device=omega_k.device)

        @staticmethod
        def backward(ctx, gF):
            go, gd = ctx.saved_tensors
            return gF * go, gF * gd, None, None

    return PulseFidelity


def pulse_fidelity(omega_k, delta_k, problem: PulseProblem, tau):
    """Differentiable F for torch tensors omega_k, delta_k (shape [K])."""
    return _function().apply(omega_k, delta_k, problem, np.asarray(tau, float))

"""KPM moments, density of states and thermodynamics on the B200 path.

Mirrors the reference's kpm.py: ``kpm_moments_b200`` returns ``(mu, c, r)``
like kpm_moments_gpu (kpm.py:26-75) with the same normalisation
mu_n = sum_probes <z, T_n(Htil) z> / (nvec D) and the same spectral
scaling c = (emin+emax)/2, r = (emax-emin)/2 (1+1e-3) + 1e-12 (kpm.py:95-96).
Differences, all stated in the result: the spectral bounds come from an FP64
Lanczos on the device instead of ARPACK; probes come from the library's
counter-based generator unless ``probes`` is given (e.g. the reference's own
numpy draws); the default recurrence uses the doubling identities (half the
H applications, same moments to rounding).  Post-processing (Jackson kernel,
DOS series, thermal Chebyshev coefficients) restates kpm.py:100-189 on the host.
"""
from __future__ import annotations

import numpy as np

from . import model, solvers


def kpm_scale(emin, emax):
    return solvers.kpm_scale(emin, emax)


def kpm_moments_b200(system, num=300, nvec=48, seed=0, device='cuda', chunk=32,
                     memory_budget_mb=None, dtype='float32', mode='doubling', probes=None,
                     bounds=None, return_info=False):
    """(mu[num+1], c, r) for the Hamiltonian described by ``system``.

    system: dict with 'calib' and optional 'Om', 'delta', 'gamma', 'terms',
    'plan' (the dict eq_route passes around)."""
    if dtype not in ('float32', 'float64'):
        raise ValueError('dtype 必须为 float32/float64')
    if int(num) < 1 or int(nvec) < 1:
        raise ValueError('num 和 nvec 必须为正整数')
    ctx, basis, ham, perm = model.build(system['calib'], system.get('Om'), system.get('delta'),
                                        system.get('gamma'), system.get('terms'),
                                        plan=system.get('plan'), device=device)
    if ham.complex_drive:
        raise model.ConfigConflict('KPM on the b200 path needs real Omega', keys=('manybody.drive_segments',))
    es = 4 if dtype == 'float32' else 8
    need = basis.dim * min(int(chunk), int(nvec)) * es * 3 + basis.dim * 16
    if memory_budget_mb is not None and need > float(memory_budget_mb) * 1024 ** 2:
        raise MemoryError('GPU KPM 算子和 probe 块超过 memory_budget_mb')
    if bounds is None:
        emin, emax = solvers.bounds(ham, max_iter=300, tol=1e-12, seed=0)
    else:
        emin, emax = bounds
    c, r = kpm_scale(emin, emax)
    if probes is not None and perm is not None:
        probes = np.asarray(probes)[:, perm]
    mu = solvers.kpm_moments(ham, int(num), int(nvec), c, r, dtype=dtype, chunk=int(chunk),
                             seed=int(seed), probes=probes, mode=mode)
    if return_info:
        return mu, c, r, dict(emin=emin, emax=emax, dim=basis.dim, launches=ctx.launches)
    return mu, c, r


def jackson_kernel(num):
    """g_n of the Jackson kernel (kpm.py:109-112)."""
    n = np.arange(num + 1)
    return ((num - n + 1) * np.cos(np.pi * n / (num + 1))
            + np.sin(np.pi * n / (num + 1)) / np.tan(np.pi / (num + 1))) / (num + 1)


def dos_from_moments(mu, c, r, energies, num, use_jackson=True):
    """Jackson-damped DOS normalised to 1 (kpm.py:182-189)."""
    x = (np.asarray(energies, float) - c) / r
    xn = np.clip(x, -1 + 1e-9, 1 - 1e-9)
    G = jackson_kernel(num) if use_jackson else np.ones(num + 1)
    coef = np.asarray(mu[:num + 1], float) * G
    coef[1:] *= 2.0
    series = np.polynomial.chebyshev.chebval(xn, coef)
    return np.maximum(series / (np.pi * np.sqrt(1 - xn ** 2)) / r, 0.0)


def _cheb_coeffs(func, num):
    p = np.polynomial.chebyshev.chebinterpolate(func, num)
    a = np.asarray(p.coef if hasattr(p, 'coef') else p, float)
    if a.size < num + 1:
        a = np.concatenate([a, np.zeros(num + 1 - a.size)])
    return a[:num + 1]


def thermal_from_moments(dim, betas, moments, num):
    """E, C, F, Z from moments (kpm.py:159-179: shifted partition function)."""
    mu, c, r = moments
    betas = np.atleast_1d(np.asarray(betas, float))
    E = np.zeros_like(betas); Cv = np.zeros_like(betas); F = np.zeros_like(betas)
    Z = np.zeros_like(betas); lnZ = np.zeros_like(betas)
    for i, b in enumerate(betas):
        shift = c - r
        fZ = lambda x, b=b: np.exp(-b * (r * x + c - shift))
        fE = lambda x, b=b: (r * x + c) * np.exp(-b * (r * x + c - shift))
        fE2 = lambda x, b=b: (r * x + c) ** 2 * np.exp(-b * (r * x + c - shift))
        z = float(np.dot(_cheb_coeffs(fZ, num), mu)) * dim
        e1 = float(np.dot(_cheb_coeffs(fE, num), mu)) * dim
        e2 = float(np.dot(_cheb_coeffs(fE2, num), mu)) * dim
        if not np.isfinite(z) or z <= 0:
            raise ValueError('KPM 配分函数非正；请增加 moments/probes 或降低 beta')
        E[i] = e1 / z
        Cv[i] = b * b * max(e2 / z - E[i] ** 2, 0.0)
        F[i] = shift - np.log(z) / b if b > 0 else np.nan
        lnZ[i] = np.log(z) - b * shift
        with np.errstate(over='ignore', under='ignore'):
            Z[i] = np.exp(lnZ[i])
    return dict(betas=betas, E=E, C=Cv, F=F, Z=Z, lnZ=lnZ)


def kpm_dos_b200(system, num=400, nvec=200, seed=0, dtype='float32', n_energies=400, chunk=32,
                 device='cuda', memory_budget_mb=None, mode='doubling'):
    """Density of states like eq_route._solve_dos (eq_route.py:772-788):
    400 energies spanning the bounds shrunk by 1e-6 of the span."""
    mu, c, r, info = kpm_moments_b200(system, num=num, nvec=nvec, seed=seed, dtype=dtype, chunk=chunk,
                                      device=device, memory_budget_mb=memory_budget_mb, mode=mode,
                                      return_info=True)
    lo, hi = info['emin'], info['emax']
    span = max(hi - lo, 1e-9)
    energies = np.linspace(lo + span * 1e-6, hi - span * 1e-6, int(n_energies))
    rho = dos_from_moments(mu, c, r, energies, int(num))
    return dict(energies=energies, rho=rho, mu=mu, c=c, r=r, emin=lo, emax=hi, dim=info['dim'])


def kpm_thermal_b200(system, betas, num=400, nvec=200, seed=0, dtype='float32', chunk=32,
                     device='cuda', memory_budget_mb=None, mode='doubling'):
    """Finite-temperature E/C/F/Z like eq_route._solve_thermal (eq_route.py:732-768)."""
    mu, c, r, info = kpm_moments_b200(system, num=num, nvec=nvec, seed=seed, dtype=dtype, chunk=chunk,
                                      device=device, memory_budget_mb=memory_budget_mb, mode=mode,
                                      return_info=True)
    th = thermal_from_moments(info['dim'], betas if betas is not None else [1.0], (mu, c, r), int(num))
    return dict(th, num=num, nvec=nvec, backend='b200-kpm')

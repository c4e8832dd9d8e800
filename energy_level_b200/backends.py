"""Backend names, capabilities and routing for the drop-in boundary.

The reference dispatches equilibrium work by name through EQ_BACKENDS
(backends.py:112-118) and eq_route.solve_equilibrium (eq_route.py:340-490),
and time evolution through TIME_BACKENDS -> runspec._ENGINE_TABLE
(backends.py:48-110, 177-179; runspec.py:660-697).  This module declares the
B200 backends in the same shapes:

    EQ_BACKENDS   'b200-lanczos': ('gs', 'spectrum', 'ramp')   'b200-kpm': ('thermal', 'dos')
    TIME_BACKENDS 'b200-cheb': TimeBackend(segments, projected, gamma, return_state,
                                           pauli='full')

``solve_equilibrium`` accepts the reference's ``system`` dict and keyword
arguments for these names and returns the same result keys as
eq_route._solve_ground / _solve_thermal / _solve_dos (and the spectrum and
ramp routes).  ``install_into`` adds the names to a module shaped like the
reference's backends.py (EQ_BACKENDS, TIME_BACKENDS, TimeBackend).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .model import ConfigConflict


@dataclass(frozen=True)
class TimeBackend:
    module: str
    function: str
    aliases: tuple = ()
    options: tuple = ()
    segments: bool = False
    projected: bool = False
    gamma: bool = False
    return_state: bool = False
    charge: bool = False
    order: bool = False
    pauli: str = ''
    native_state: str = ''
    algorithm: str = ''


EQ_BACKENDS = {
    'b200-lanczos': ('gs', 'spectrum', 'ramp'),
    'b200-kpm': ('thermal', 'dos'),
}

TIME_BACKENDS = {
    'b200-cheb': TimeBackend('energy_level_b200.engine', 'evolve_manybody',
                             aliases=('b200', 'b200-ed', 'chebyshev-gpu'),
                             options=(('memory_budget_mb', 'memory_budget_mb'), ('dtype', 'dtype'),
                                      ('device', 'device')),
                             segments=True, projected=True, gamma=True, return_state=True,
                             pauli='full', algorithm='chebyshev'),
}


def normalize_equilibrium_backend(name, want):
    name = str(name or '').lower()
    name = {'kpm-b200': 'b200-kpm', 'lanczos-b200': 'b200-lanczos'}.get(name, name)
    if name not in EQ_BACKENDS:
        raise ValueError('未知 b200 平衡态后端 %r' % name)
    if want not in EQ_BACKENDS[name]:
        raise ValueError('平衡态后端 %r 不支持 want=%r' % (name, want))
    return name


def normalize_time_backend(name):
    name = str(name or '').lower()
    if name in TIME_BACKENDS:
        return name
    for canon, b in TIME_BACKENDS.items():
        if name in b.aliases:
            return canon
    raise ValueError('未知多体 solver=%r；合法：%s' % (name, list(TIME_BACKENDS)))


def validate_time_capabilities(name, *, segments=None, plan=None, gamma=None, return_state=False,
                               charge_sector=None, psi0=None, pauli_strings=None, **_):
    """Refuse what b200-cheb does not implement, with ConfigConflict keys
    (backends.py:182-230 semantics)."""
    b = TIME_BACKENDS[normalize_time_backend(name)]
    if pauli_strings and not b.pauli:
        raise ConfigConflict('%s 不提供 Pauli 串观测' % name, keys=('manybody.pauli_strings',))
    if segments and not b.segments:
        raise ConfigConflict('%s 尚不支持 drive_segments' % name, keys=('manybody.drive_segments',))
    if plan and plan.get('projected') and not b.projected:
        raise ConfigConflict('%s 尚不支持 projected HamiltonianPlan' % name, keys=('manybody.constraint',))
    if gamma is not None and np.any(np.asarray(gamma) != 0) and not b.gamma:
        raise ConfigConflict('%s 仅支持 gamma=0' % name, keys=('manybody.gamma_mhz',))
    if charge_sector is not None:
        raise ConfigConflict('%s 尚不支持实时 charge_sector' % name, keys=('manybody.charge_sector',))
    if isinstance(psi0, str) and psi0 == 'ground':
        raise ValueError('%s 尚不支持 ground 初态；请先准备兼容初态' % name)


def engine_entries():
    """{(name, 'many'): (module, function)} like backends.py:177-179."""
    return {(name, 'many'): (b.module, b.function) for name, b in TIME_BACKENDS.items()}


def solve_equilibrium(system, want='gs', *, backend='b200-lanczos', betas=None, k=2, v0=None,
                      seed=0, num=400, nvec=200, dtype=None, memory_budget_mb=None,
                      return_state=False, sector=None, progress_arr=None, ramp=None, log=None,
                      exact=False, **unused):
    """eq_route.solve_equilibrium for the b200 names (same result keys).

    ``exact=True`` (the dense spectral trace of the CPU kpm / ed routes) is
    refused for b200-kpm with ValueError, as eq_route.py:446-447 refuses it
    for gpu-kpm: the moments here are always stochastic (Hutchinson)."""
    from . import kpm as bkpm
    from .matrix_free import b200_lanczos_ground_state
    if progress_arr is not None and float(progress_arr[1]) != 0:
        raise RuntimeError('用户取消')
    backend = normalize_equilibrium_backend(backend, want)
    if exact and backend == 'b200-kpm':
        raise ValueError('b200-kpm 不提供 exact 谱迹；请选择 CPU kpm 或 ed')
    system = dict(system)
    plan = system.get('plan') or {}
    for key in ('Om', 'delta', 'gamma', 'terms'):
        if system.get(key) is None and key in plan:
            system[key] = plan[key]
    if system.get('H') is not None or system.get('H_builder') is not None:
        raise ValueError('%s 需要物理 calib；不能忽略显式 H/H_builder' % backend)
    if 'calib' not in system:
        raise ValueError("%s 后端需要 system['calib']" % backend)
    n_sites = len(system['calib']['atoms'])
    base = dict(want=want, backend=backend, n_sites=n_sites)
    if want == 'gs':
        constraint = None
        if sector is not None or system.get('charge_sector') is not None:
            kq = int(sector if sector is not None else system['charge_sector'])
            from .model import check_number_conserving
            check_number_conserving(system['calib'], system.get('Om'), system.get('terms'))
            constraint = {'kind': 'charge', 'k': kq}
        from . import model, solvers
        if constraint is not None:
            ctx, basis, ham, _ = model.build(system['calib'], system.get('Om'), system.get('delta'),
                                             system.get('gamma'), system.get('terms'),
                                             constraint=constraint, device=system.get('device', 'cuda'))
            r = solvers.lanczos_ground(ham, dtype=dtype or 'float64', seed=seed,
                                       max_iter=min(300, basis.dim), tol=1e-9, nev=min(k, basis.dim),
                                       return_vec=True)
            vec = r['vec'].cpu().numpy()
            codes = basis.codes().cpu().numpy()
            bits = np.asarray([((codes >> (n_sites - 1 - i)) & 1) for i in range(n_sites)], float)
            out = dict(base, sector=int(constraint['k']), charge_sector=int(constraint['k']),
                       dim_sub=basis.dim, sector_idx=codes, E0=float(r['evals'][0]),
                       gap=float(r['evals'][1] - r['evals'][0]) if len(r['evals']) > 1 else 0.0,
                       evals=np.asarray(r['evals']), n_atom=bits @ (np.abs(vec) ** 2))
            if return_state:
                out['vec'] = vec.astype(np.complex128)
            return out
        r = b200_lanczos_ground_state(system['calib'], system.get('Om'), system.get('delta'),
                                      system.get('gamma'), system.get('terms'),
                                      m=system.get('krylov_dim', 300), seed=seed,
                                      dtype=dtype or 'float64', device=system.get('device', 'cuda'),
                                      return_state=True, memory_budget_mb=memory_budget_mb,
                                      plan=plan if plan.get('projected') else None, nev=k)
        vec = r.pop('vec')
        if plan.get('projected'):
            codes = np.asarray(r.pop('basis_states'), np.int64)
        else:
            codes = np.arange(1 << n_sites, dtype=np.int64)
        bits = np.asarray([((codes >> (n_sites - 1 - i)) & 1) for i in range(n_sites)], float)
        p = np.abs(vec) ** 2
        obs = dict(n_atom=bits @ p)
        if len(codes) <= (1 << 18):
            ni = obs['n_atom']
            obs['corr'] = (bits * p) @ bits.T - np.outer(ni, ni)
        out = dict(base, **r, **obs)
        out['backend'] = backend
        if return_state:
            out['vec'] = vec
        return out
    if want == 'ramp':
        return _solve_ramp(system, base, ramp, v0, seed, log, dtype, progress_arr)
    if want == 'spectrum':
        return _solve_spectrum(system, base, sector=sector, memory_budget_mb=memory_budget_mb,
                               progress_arr=progress_arr, dtype=dtype, seed=seed)
    if want == 'thermal':
        betas = np.atleast_1d(np.asarray([1.0] if betas is None else betas, float))
        if betas.ndim != 1 or not len(betas) or not np.isfinite(betas).all() or np.any(betas <= 0):
            raise ValueError('betas 须为非空、有限的正数数组')
        th = bkpm.kpm_thermal_b200(system, betas, num=num, nvec=nvec, seed=seed,
                                   dtype=dtype or 'float32', memory_budget_mb=memory_budget_mb,
                                   device=system.get('device', 'cuda'), chunk=system.get('kpm_chunk', 32))
        return dict(base, betas=th['betas'], E=th['E'], C=th['C'], F=th['F'])
    if want == 'dos':
        r = bkpm.kpm_dos_b200(system, num=num, nvec=nvec, seed=seed, dtype=dtype or 'float32',
                              memory_budget_mb=memory_budget_mb, device=system.get('device', 'cuda'),
                              chunk=system.get('kpm_chunk', 32))
        return dict(base, energies=r['energies'], rho=r['rho'])
    raise ValueError('want 需为 gs/thermal/dos，实=%r' % want)


def _solve_ramp(system, base, ramp, v0, seed, log, dtype, progress_arr):
    """Adiabatic sequence of ground states (eq_route.py:493-536 _solve_ramp)
    on the GPU: at every point tau_i, H(Omega_t[i], delta_t[i]) with the drive
    uniform over the sites (times system['Om_shape'] / ['delta_shape'] when
    given), ground state and gap by the device Lanczos, warm-started from the
    previous point's ground state when ramp['v0_warm'] (default).  The
    reference takes a host H_builder(Om, delta); this backend builds H from
    system['calib'] (and a projected plan, if any) instead."""
    from . import model, solvers
    if ramp is None:
        raise ValueError("want='ramp' 需要 ramp=dict(Om_t, de_t, L, ...)")
    if 'calib' not in system:
        raise ValueError("b200 ramp 需要 system['calib']（H_builder 是主机算子）")
    Om_t = np.asarray(ramp['Om_t'], float)
    de_t = np.asarray(ramp['de_t'], float)
    taus = np.asarray(ramp.get('taus', np.linspace(0.0, 1.0, len(Om_t))), float)
    if len(de_t) != len(Om_t) or len(taus) != len(Om_t):
        raise ValueError('ramp 的 Om_t/de_t/taus 长度须一致')
    L = ramp.get('L')
    if L is None:
        raise ValueError('ramp 需要 L（密度归一格点数）')
    n = len(system['calib']['atoms'])
    om_shape = np.asarray(system.get('Om_shape', np.ones(n)), float)
    de_shape = np.asarray(system.get('delta_shape', np.ones(n)), float)
    n_tot = np.asarray(ramp['n_tot'], float) if ramp.get('n_tot') is not None else None
    v0_warm = bool(ramp.get('v0_warm', True))
    plan = system.get('plan') or {}
    ctx, basis, ham, perm = model.build(system['calib'], Om_t[0] * om_shape, de_t[0] * de_shape,
                                        system.get('gamma'), system.get('terms'),
                                        plan=plan if plan.get('projected') else None,
                                        device=system.get('device', 'cuda'))
    if n_tot is not None and n_tot.size != basis.dim:
        raise ValueError('ramp n_tot 长度 %d ≠ 基维度 %d' % (n_tot.size, basis.dim))
    vdt = dtype or 'float64'
    v_i = v0
    gaps, ns, e0s, conv = [], [], [], []
    for it in range(len(taus)):
        if progress_arr is not None and float(progress_arr[1]) != 0:
            raise RuntimeError('用户取消')
        ham.set_drive(Om_t[it] * om_shape, de_t[it] * de_shape)
        r = solvers.lanczos_ground(ham, dtype=vdt, v0=v_i, seed=seed, max_iter=min(300, basis.dim),
                                   tol=1e-10 if vdt in ('float64', 'complex128') else 2e-5,
                                   nev=min(2, basis.dim), return_vec=True)
        if not r['converged'] and v_i is not None:
            r = solvers.lanczos_ground(ham, dtype=vdt, v0=None, seed=seed + 1, max_iter=min(300, basis.dim),
                                       tol=1e-10 if vdt in ('float64', 'complex128') else 2e-5,
                                       nev=min(2, basis.dim), return_vec=True)
        if v0_warm:
            # previous ground state plus a small seeded random part: a start
            # vector with the ground state's symmetry alone would never reach
            # an excited state of another symmetry sector, and the gap would
            # be that of the wrong state
            import torch
            gen = torch.Generator(device=r['vec'].device).manual_seed(int(seed) + 7919 * (it + 1))
            noise = torch.randn(r['vec'].shape, dtype=r['vec'].dtype, device=r['vec'].device, generator=gen)
            v_i = r['vec'] + 1e-2 * noise / noise.norm()
        else:
            v_i = None
        ev = np.asarray(r['evals'], float)
        e0s.append(float(ev[0]))
        gaps.append(float(ev[1] - ev[0]) if len(ev) > 1 else 0.0)
        conv.append(bool(r['converged']))
        if n_tot is not None:
            p = (r['vec'].abs() ** 2).double().cpu().numpy()
            ns.append(float(n_tot @ p) / float(L))
        else:
            ns.append(float('nan'))
        if progress_arr is not None:
            progress_arr[0] = (it + 1) / len(taus)
        if log is not None and (it % max(1, len(taus) // 10) == 0 or it == len(taus) - 1):
            log('ramp %d/%d Ω=%.3f δ=%.3f gap=%.4f n=%.4f' % (it + 1, len(taus), Om_t[it], de_t[it],
                                                             gaps[-1], ns[-1]))
    return dict(base, taus=taus, gaps=np.asarray(gaps, float), ns=np.asarray(ns, float),
                Om_t=Om_t, de_t=de_t, E0s=np.asarray(e0s), converged=np.asarray(conv))


def _solve_spectrum(system, base, *, sector, memory_budget_mb, progress_arr, dtype, seed):
    """Source-state spectrum (eq_route.py:260-337 _solve_spectrum) on the GPU:
    |0> is system['psi0'] (state grammar or vector) or the b200 Lanczos ground
    state; phi from system['source'] (eq_route.py:160-257); spectrum.py's
    source_spectrum with the device Lanczos."""
    from . import model, solvers
    from . import spectrum as spec
    from .state import state_vector
    n_sites = int(base['n_sites'])
    opts = dict(system.get('spectrum') or {})
    source = system.get('source')
    if source is None and system.get('psi0') is not None:
        source = {'kind': 'psi0'}
    if source is None:
        raise ValueError('want=spectrum 需要 system["source"] 或 system["psi0"]'
                         '（vector/psi0/diagonal/sparse/full_sparse）')
    plan = system.get('plan') or {}
    constraint = None
    if sector is not None:
        constraint = {'kind': 'charge', 'k': int(sector)}
        model.check_number_conserving(system['calib'], system.get('Om'), system.get('terms'))
    ctx, basis, ham, perm = model.build(system['calib'], system.get('Om'), system.get('delta'),
                                        system.get('gamma'), system.get('terms'),
                                        plan=plan if (plan.get('projected') and constraint is None) else None,
                                        constraint=constraint, device=system.get('device', 'cuda'))
    restricted = constraint is not None or plan.get('projected')
    codes = basis.codes().cpu().numpy() if restricted else None
    dim = basis.dim
    psi0 = system.get('psi0')
    E0 = float('nan')
    if psi0 is not None and not (isinstance(psi0, str) and psi0 == 'ground') and not isinstance(psi0, dict):
        if isinstance(psi0, np.ndarray) and psi0.ndim == 1 and psi0.size == dim and psi0.size != (1 << n_sites):
            vec = np.asarray(psi0, complex)
        else:
            vec = state_vector(psi0, n_sites, codes)
    else:
        r = solvers.lanczos_ground(ham, dtype='complex128' if ham.complex_drive else 'float64', seed=seed,
                                   max_iter=min(300, dim), tol=1e-12, nev=1, return_vec=True)
        vec = r['vec'].cpu().numpy().astype(complex)
        E0 = float(r['evals'][0])
    if progress_arr is not None and float(progress_arr[1]) != 0:
        raise RuntimeError('用户取消')
    phi, info = spec.resolve_source(source, vec, n_sites, codes)
    if progress_arr is not None:
        progress_arr[0] = 0.35
    out = spec.source_spectrum(
        ham, phi, shift=E0 if np.isfinite(E0) else 0.0,
        eta=float(opts.get('eta') or 0.05), n_krylov=int(opts.get('n_krylov') or 0) or None,
        omega_min=opts.get('omega_min'), omega_max=opts.get('omega_max'),
        n_omega=int(opts.get('n_omega') or 800), reortho=bool(opts.get('reortho', True)),
        memory_budget_mb=memory_budget_mb if memory_budget_mb is not None else 512.0,
        dtype=dtype if dtype in ('complex64', 'complex128') else None)
    if progress_arr is not None:
        progress_arr[0] = 1.0
    errors = dict(out.pop('error_report') or {})
    errors.update({'source_kind': info.get('kind'), 'sector': None if sector is None else int(sector),
                   'dim_basis': dim})
    for key, value in info.items():
        if key not in ('kind', 'dim'):
            errors.setdefault(key, value)
    res = dict(base, E0=E0 if np.isfinite(E0) else None, gap=None,
               evals=out['evals'], spectrum_weights=out['spectrum_weights'],
               energies=out['omega'], spectral=out['spectral'],
               source_norm=out['source_norm'], eta=out['eta'],
               krylov=out['krylov'], error_report=errors)
    if constraint is not None:
        res.update(sector_idx=codes, dim_sub=dim)
    return res


def install_into(reference_backends, shim_module='b200_shim'):
    """Register the b200 names into a reference backends module in place:
    EQ_BACKENDS gains 'b200-lanczos'/'b200-kpm', TIME_BACKENDS gains
    'b200-cheb' (constructed with the module's own TimeBackend class).  The
    reference resolves time engines as '.manybody.<module>' (backends.py:177),
    so the entry names a shim module in that package that re-exports
    energy_level_b200.engine.evolve_manybody."""
    import dataclasses
    eq = reference_backends.EQ_BACKENDS
    for name, wants in EQ_BACKENDS.items():
        eq[name] = tuple(wants)
    tb = reference_backends.TIME_BACKENDS
    cls = getattr(reference_backends, 'TimeBackend', TimeBackend)
    # every capability field the target class declares (pauli, charge, order,
    # native_state, algorithm, ... in backends.py:22-37), so that its own
    # validate_time_capabilities sees what this backend implements
    if dataclasses.is_dataclass(cls):
        names = [f.name for f in dataclasses.fields(cls)]
    else:
        names = [f.name for f in dataclasses.fields(TimeBackend)]
    ours = {f.name for f in dataclasses.fields(TimeBackend)}
    for name, b in TIME_BACKENDS.items():
        kw = {k: getattr(b, k) for k in names if k in ours and k not in ('module', 'function')}
        tb[name] = cls(shim_module, b.function, **kw)
    return reference_backends

"""Generate golden fixtures by running the reference lcodePy (CPU/numba path).

Run in a container that has the reference checkout and numba:

    python tests/golden/make_golden.py /path/to/lcodePy

The reference needs single-rank ``mpi4py`` and empty ``matplotlib`` stand-ins
to import (``tests/golden/refstubs``).  Outputs are small ``.npz`` files in
this directory; the tests read only those files, never the reference.

Fixtures:
  gen_beams.npz        -- lcode.alt_beam_generator.generate_beam outputs
  kat_kernels.npz      -- reference numba kernels on seeded random states
  kat_fields.npz       -- reference compute_fields on seeded random currents
  run_rigid_bg.npz     -- full xi loop, rigid driver, background ions
  run_rigid_mobile.npz -- full xi loop, rigid driver, mobile ions
  run_beam.npz         -- full xi loop, generated (non-rigid) beam, 1 time step
  run_profile_*.npz    -- rigid driver with a channel (9 per cell) and a
                          gaussian (1 per cell, mobile ions) transverse
                          plasma profile (with --profiles)
  run_test1.npz        -- the reference's own 3D golden configuration
                          (tests/integration/test_3D_part.py:9-56): strided
                          final state and on-axis Ez per xi step
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def rigid_driver(xp, xi, x, y):
    """rho_b = 0.1 exp(-r^2/2) (1 + cos(sqrt(pi/2) xi))/2 on -sqrt(2 pi) <= xi <= 0."""
    if -np.sqrt(2 * np.pi) <= xi <= 0:
        return 0.1 * xp.exp(-(x ** 2 + y ** 2) / 2) * (1 + np.cos(np.sqrt(np.pi / 2) * xi)) / 2
    return xp.zeros_like(x)


class OnAxis:
    """Diagnostic with the reference's hook signature: records on-axis Ez and
    the summed rho at the centre after every xi step."""

    def __init__(self):
        self.ez, self.ro = [], []

    def pull_config(self, config):
        self.N = config.getint('window-width-steps')

    def after_step_dxi(self, t, xi, particles, fields, currents, rho_beam):
        c = self.N // 2
        self.ez.append(fields.Ez[c, c])
        self.ro.append(currents.ro[:, c, c].sum())

    def dump(self, *a, **k):
        pass


def base_config(**kw):
    cfg = {'geometry': '3d', 'processing-unit-type': 'cpu',
           'window-width': 1.6, 'transverse-step': 0.05,
           'window-length': 2.0, 'xi-step': 0.05,
           'time-limit': 1, 'time-step': 1,
           'ion-model': 'background', 'plasma-particles-per-cell': 4}
    cfg.update(kw)
    return cfg


def run_sim(lcode, cfg, beam_parameters):
    diag = OnAxis()
    sim = lcode.Simulation(config=cfg, beam_parameters=beam_parameters,
                           diagnostics=[diag], runas_filename='')
    sim.step()
    particles, fields, currents = sim._Simulation__push_solver._plasmastate
    out = {'ez_axis': np.array(diag.ez), 'ro_axis': np.array(diag.ro)}
    for k in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi'):
        out['f_' + k] = np.asarray(getattr(fields, k))
    for k in ('ro', 'jx', 'jy', 'jz'):
        out['c_' + k] = np.asarray(getattr(currents, k))
    for sort, arr in particles.items():
        for k in ('x_offt', 'y_offt', 'px', 'py', 'pz', 'q'):
            out[f'p_{sort}_{k}'] = np.asarray(getattr(arr, k))
    return out


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, 'refstubs'))
    sys.path.insert(0, ref_root)
    import lcode
    from lcode.alt_beam_generator.beam_generator import generate_beam
    from lcode.config.config import Config
    from lcode.plasma3d import weights as pw, move as pm, fields as pf
    from lcode.plasma3d import initialization as pi
    from lcode.beam3d import weights as bw, beam_calculator as bc
    from lcode.plasma3d.data import Arrays

    # ---- generator ----
    gb = {}
    c1 = Config({'geometry': '3d', 'window-width': 8, 'transverse-step': 0.05,
                 'xi-step': 0.05})
    c1._adjust_config_values_3d()
    b = generate_beam(c1, {'current': 0.05, 'particles_in_layer': 150,
                           'default': {'length': 5.013256548}})
    gb['test1like'] = b
    c2 = Config({'geometry': '3d', 'window-width': 3.2, 'transverse-step': 0.05,
                 'xi-step': 0.1})
    c2._adjust_config_values_3d()
    b2 = generate_beam(c2, {'current': -0.3, 'particles_in_layer': 300, 'rng_seed': 7,
                            'seg1': {'length': 2.0, 'xishape': 'l', 'eshape': 'g',
                                     'espread': 10, 'radius': 0.5},
                            'seg2': {'length': 1.5, 'xishape': 'h', 'angspread': 1e-3,
                                     'mass_charge_ratio': 1836, 'eshape': 'u',
                                     'energy': 500, 'espread': 600}})
    gb['twoseg'] = b2
    np.savez_compressed(os.path.join(HERE, 'gen_beams.npz'),
                        **{k: v for k, v in gb.items()})

    # ---- per-kernel known answers ----
    rng = np.random.default_rng(20240601)
    N, h, dxi = 65, 0.05, 0.05
    bp = 10
    boundary = h * (N / 2 - bp)
    Ns = 68
    g = pi.make_plasma_grid(np, N - 30, h, 2)
    y_init = np.broadcast_to(g, (Ns, Ns)).copy()
    x_init = y_init.T.copy()
    kat = {'N': N, 'h': h, 'dxi': dxi, 'boundary': boundary,
           'x_init': x_init, 'y_init': y_init}
    shp = (Ns, Ns)
    xo_prev = rng.normal(0, 0.02, shp)
    yo_prev = rng.normal(0, 0.02, shp)
    px_prev = rng.normal(0, 0.05, shp)
    py_prev = rng.normal(0, 0.05, shp)
    pz_prev = rng.normal(0, 0.02, shp)
    m = np.full(shp, h ** 2 / 4)
    q = np.full(shp, -h ** 2 / 4)
    q[3, 5] = 0.0  # an absorbed particle
    # a few particles pushed across the reflection boundary
    xo_prev[0, :4] -= 0.3
    yo_prev[-1, -3:] += 0.3
    kat.update(xo_prev=xo_prev, yo_prev=yo_prev, px_prev=px_prev,
               py_prev=py_prev, pz_prev=pz_prev, m=m, q=q)
    # K1
    xo_full, yo_full = xo_prev.copy(), yo_prev.copy()
    pm.move_estimate_wo_fields_numba(dxi, m, xo_full, yo_full, px_prev.copy(),
                                     py_prev.copy(), pz_prev.copy(), m.size)
    kat.update(k1_xo=xo_full.copy(), k1_yo=yo_full.copy())
    # K2 with random smooth fields
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing='ij')
    F = {}
    for i, k in enumerate(('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz')):
        F[k] = 0.05 * np.sin(0.1 * (i + 1) * X + 0.07 * Y + i) * np.cos(0.05 * Y * (i + 1))
        kat['F_' + k] = F[k]
    q2 = q.copy()
    xf, yf = xo_full.copy(), yo_full.copy()
    pxf, pyf, pzf = px_prev.copy(), py_prev.copy(), pz_prev.copy()
    pm.move_smart_kernel_numba(dxi, boundary, h, N, F['Ex'], F['Ey'], F['Ez'],
                               F['Bx'], F['By'], F['Bz'], x_init, y_init,
                               xo_prev, yo_prev, px_prev, py_prev, pz_prev,
                               m, q2, xf, yf, pxf, pyf, pzf, m.size)
    kat.update(k2_xo=xf, k2_yo=yf, k2_px=pxf, k2_py=pyf, k2_pz=pzf, k2_q=q2)
    # K3
    out = [np.zeros((N, N)) for _ in range(4)]
    x_h = (x_init + xf) / h + 0.5
    y_h = (y_init + yf) / h + 0.5
    pw.deposit_plasma_numba(N, h, x_h, y_h, pxf, pyf, pzf, q2, m, *out, m.size)
    kat.update(k3_ro=out[0], k3_jx=out[1], k3_jy=out[2], k3_jz=out[3])
    # K4 beam deposit
    nb_ = 400
    bx = rng.normal(0, 0.4, nb_)
    by = rng.normal(0, 0.4, nb_)
    layer = 7
    bxi = rng.uniform(-(layer + 1) * dxi, -layer * dxi, nb_)
    bq = rng.uniform(-0.01, 0.01, nb_)
    r0, r1 = np.zeros((N, N)), np.zeros((N, N))
    bw.deposit_beam_numba(N, bx / h + 0.5, by / h + 0.5, (-dxi * layer - bxi) / dxi,
                          bq, r0, r1, nb_)
    kat.update(b_x=bx, b_y=by, b_xi=bxi, b_q=bq, b_layer=layer, k4_ro0=r0, k4_ro1=r1)
    # K6 substepping
    qm = rng.choice([-1.0, 1.0, 1 / 1836.0], 64)
    pzb = rng.uniform(0.5, 2000, 64)
    kat.update(k6_qm=qm, k6_pz=pzb, k6_dt=bc.beam_substepping_step_numba(qm, pzb, 2.0))
    np.savez_compressed(os.path.join(HERE, 'kat_kernels.npz'), **kat)

    # ---- field solver known answer ----
    cfg = Config({'geometry': '3d', 'processing-unit-type': 'cpu',
                  'window-width': 1.6, 'transverse-step': 0.05, 'xi-step': 0.05})
    cfg._adjust_config_values_3d()
    compute_fields = pf.get_field_computer(cfg)
    Nf = cfg.getint('window-width-steps')
    sub = cfg.getfloat('field-solver-subtraction-coefficient')
    const = Arrays(np, dirichlet_matrix=pi.dirichlet_matrix(np, Nf, h),
                   field_mixed_matrix=pi.mixed_matrix(np, Nf, h, sub),
                   neumann_matrix=pi.neumann_matrix(np, Nf, h))

    def smooth(seed):
        r = np.random.default_rng(seed)
        a = np.zeros((2, Nf, Nf))
        a[:, 3:-3, 3:-3] = r.normal(0, 1, (2, Nf - 6, Nf - 6))
        return a

    cp = Arrays(np, ro=smooth(1), jx=smooth(2), jy=smooth(3), jz=smooth(4))
    cfu = Arrays(np, ro=smooth(5), jx=smooth(6), jy=smooth(7), jz=smooth(8))
    fr = np.random.default_rng(9)
    fld = Arrays(np, **{k: fr.normal(0, 1, (Nf, Nf)) for k in
                        ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi')})
    fprev = Arrays(np, **{k: fr.normal(0, 1, (Nf, Nf)) for k in
                          ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi')})
    rbf = fr.normal(0, 1, (Nf, Nf))
    rbp = fr.normal(0, 1, (Nf, Nf))
    full, half = compute_fields(fld, fprev, const, rbf, rbp, cp, cfu)
    kf = {'N': Nf, 'h': h, 'dxi': 0.05, 'sub': sub, 'rb_full': rbf, 'rb_prev': rbp}
    for k in ('ro', 'jx', 'jy', 'jz'):
        kf['cp_' + k] = getattr(cp, k)
        kf['cf_' + k] = getattr(cfu, k)
    for k in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi'):
        kf['in_' + k] = getattr(fld, k)
        kf['prev_' + k] = getattr(fprev, k)
        kf['full_' + k] = getattr(full, k)
        kf['half_' + k] = getattr(half, k)
    np.savez_compressed(os.path.join(HERE, 'kat_fields.npz'), **kf)

    # ---- whole runs ----
    t = time.time()
    out = run_sim(lcode, base_config(**{'rigid-beam': True}), rigid_driver)
    np.savez_compressed(os.path.join(HERE, 'run_rigid_bg.npz'), **out)
    out = run_sim(lcode, base_config(**{'rigid-beam': True, 'ion-model': 'mobile',
                                        'window-length': 1.0, 'xi-step': 0.1}),
                  rigid_driver)
    np.savez_compressed(os.path.join(HERE, 'run_rigid_mobile.npz'), **out)
    out = run_sim(lcode, base_config(**{'window-length': 1.5}),
                  {'current': 0.05, 'particles_in_layer': 400,
                   'default': {'length': 2.0}})
    np.savez_compressed(os.path.join(HERE, 'run_beam.npz'), **out)
    print('whole runs', time.time() - t, 's')
    if '--test1' in sys.argv:
        make_test1(lcode)
    if '--profiles' in sys.argv:
        make_profiles(lcode)


def make_profiles(lcode):
    """Transverse plasma profiles and other lattice finenesses (rigid driver)."""
    out = run_sim(lcode, base_config(**{'rigid-beam': True, 'window-length': 1.0,
                                        'plasma-particles-per-cell': 9,
                                        'plasma-rshape': 'channel', 'plasma-width': 0.6,
                                        'plasma-width-2': 0.9, 'plasma-density-2': 0.5}),
                  rigid_driver)
    np.savez_compressed(os.path.join(HERE, 'run_profile_channel.npz'), **out)
    out = run_sim(lcode, base_config(**{'rigid-beam': True, 'window-length': 1.0,
                                        'plasma-particles-per-cell': 1, 'ion-model': 'mobile',
                                        'plasma-rshape': 'gaussian', 'plasma-width': 0.5}),
                  rigid_driver)
    np.savez_compressed(os.path.join(HERE, 'run_profile_gauss.npz'), **out)


def make_test1(lcode):
    cfg = {'geometry': '3d', 'processing-unit-type': 'cpu',
           'window-width': 8, 'transverse-step': 0.05,
           'window-length': 10, 'xi-step': 0.05,
           'time-limit': 1, 'time-step': 1, 'ion-model': 'background',
           'plasma-particles-per-cell': 4,
           'field-solver-subtraction-coefficient': 1.0}
    out = run_sim(lcode, cfg, {'current': 0.05, 'particles_in_layer': 5000,
                               'default': {'length': 5.013256548}})
    keep = {'ez_axis': out['ez_axis'], 'ro_axis': out['ro_axis']}
    for k, v in out.items():
        if k.startswith('f_'):
            keep[k] = v[::10, ::10]
        elif k.startswith('c_'):
            keep[k] = v[:, ::10, ::10].sum(axis=0)
        elif k.startswith('p_electrons_'):
            keep[k] = v[::10, ::10]
    np.savez_compressed(os.path.join(HERE, 'run_test1.npz'), **keep)


if __name__ == '__main__':
    args = [a for a in sys.argv[1:] if not a.startswith('--')]
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.ref_kernels import reference_root
    main(args[0] if args else reference_root())

"""Generate the diagnostics fixture by running the reference's FXiDiag and
SliceDiag (numpy path) on seeded synthetic xi steps.

    python tests/golden/make_diag_golden.py /path/to/lcodePy

The reference imports through the single-rank ``mpi4py`` and empty
``matplotlib`` stand-ins in ``tests/golden/refstubs``.  The synthetic steps
come from ``diag_steps`` below, which ``tests/test_diagnostics.py`` imports to
feed this package's diagnostics the same inputs; the fixture holds only the
reference's output files (``diag_golden.npz``: ``<case>|<file>|<key>``).
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CONFIG = {'geometry': '3d', 'processing-unit-type': 'cpu', 'window-width': 1.6,
          'transverse-step': 0.05, 'window-length': 0.5, 'xi-step': 0.05,
          'time-step': 1.0, 'time-limit': 2.0, 'ion-model': 'background',
          'plasma-particles-per-cell': 4, 'rigid-beam': False}

# (case name, class name, constructor keyword arguments)
CASES = [
    # every FXi quantity but the noise filter's chaotic displacements
    ('fxi_axis', 'FXiDiag', dict(output_period=1, f_xi=0x7ff, directory_name='fa')),
    # the noise filter's chaotic displacements (whole lattice and centre)
    ('fxi_chaotic', 'FXiDiag', dict(output_period=1, f_xi=0x4 | 0x7800, directory_name='fc')),
    ('fxi_lines', 'FXiDiag', dict(output_period=1, f_xi=0x4 | 0x80 | 0x200,
                                  probe_lines=[[0.0, 0.2, -0.35], [0.1, 0.0, 0.05]],
                                  directory_name='fl')),
    ('fxi_line1d', 'FXiDiag', dict(output_period=2, f_xi=0x1 | 0x20, probe_lines=[0.0, 0.3],
                                   directory_name='f1')),
    ('slice_xi_x', 'SliceDiag', dict(slice_type=0x2, slice_value=0x3ff, offset=0.12,
                                     output_period=1, directory_name='sx')),
    ('slice_xi_y', 'SliceDiag', dict(slice_type=0x4, slice_value=0x4 | 0x80, offset=-0.3,
                                     limits=[[-0.1, -0.4], [-0.5, 0.45]], output_period=1,
                                     directory_name='sy')),
    ('slice_x_y', 'SliceDiag', dict(slice_type=0x8, slice_value=0x4 | 0x200,
                                    limits=[[-0.4, 0.4], [-0.4, 0.4]], output_period=1,
                                    saving_xi_period=0.1, directory_name='sxy')),
    ('particles', 'ParticlesDiag', dict(save_beam=True, save_plasma=True, output_period=1,
                                        saving_xi_period=0.2, directory_name='pd')),
]


PARTICLE_KEYS = ('m', 'px', 'py', 'pz', 'dx_chaotic', 'dy_chaotic')


class StubDrain:
    """Stands in for the beam drain: ParticlesDiag only calls save()."""

    def save(self, filename):
        np.savez_compressed(filename, xi=np.linspace(0.0, -1.0, 5), id=np.arange(5))


def walk(root):
    """Relative paths of the files under root, sorted."""
    out = []
    for d, _, files in os.walk(root):
        out += [os.path.relpath(os.path.join(d, f), root) for f in files]
    return sorted(out)


def diag_steps(N, n_steps=11, times=(0.0, 1.0, 2.0), dxi=0.05, seed=77):
    """Seeded synthetic inputs: for each time and xi step, a dict of host
    arrays (fields Ex..Bz, Phi; currents ro (2, N, N); electrons m, px, py,
    pz, dx_chaotic, dy_chaotic (20 x 20); rho_beam).  The chaotic
    displacements come from a second stream, so the other inputs do not
    depend on them."""
    rng = np.random.default_rng(seed)
    rng_c = np.random.default_rng(seed + 1)
    out = []
    for t in times:
        for k in range(n_steps):
            f = {n: rng.standard_normal((N, N)) for n in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi')}
            f['ro'] = rng.standard_normal((2, N, N))
            f['rho_beam'] = rng.standard_normal((N, N))
            f['m'] = np.full((20, 20), 0.0025)
            for n in ('px', 'py', 'pz'):
                f[n] = rng.standard_normal((20, 20)) * 0.01
            for n in ('dx_chaotic', 'dy_chaotic'):
                f[n] = rng_c.standard_normal((20, 20)) * 1e-3
            out.append((t, -k * dxi, f))
    return out


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, 'refstubs'))
    sys.path.insert(0, ref_root)
    from lcode.config.config import Config
    from lcode.diagnostics.FXi.FXi import FXiDiag
    from lcode.diagnostics.slice import SliceDiag
    from lcode.diagnostics.particles import ParticlesDiag
    from lcode.plasma3d.data import Arrays

    cfg = Config(dict(CONFIG))
    cfg._adjust_config_values_3d()
    N = cfg.getint('window-width-steps')
    steps = diag_steps(N)
    classes = {'FXiDiag': FXiDiag, 'SliceDiag': SliceDiag, 'ParticlesDiag': ParticlesDiag}
    drain = StubDrain()
    result = {'N': np.array(N)}
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:
        os.chdir(td)
        try:
            for case, cls, kw in CASES:
                d = classes[cls](**kw)
                d.pull_config(cfg)
                last_t = None
                for t, xi, f in steps:
                    if last_t is not None and t != last_t:
                        d.dump(last_t, xi, particles, None, None, drain)
                    last_t = t
                    fields = Arrays(np, **{n: f[n] for n in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi')})
                    currents = Arrays(np, ro=f['ro'])
                    particles = {'electrons': Arrays(np, **{n: f[n] for n in PARTICLE_KEYS})}
                    d.after_step_dxi(t, xi, particles, fields, currents, f['rho_beam'])
                d.dump(last_t, 0.0, particles, None, None, drain)
                sub = os.path.join(td, 'diagnostics', kw['directory_name'])
                for fn in walk(sub):
                    with np.load(os.path.join(sub, fn)) as z:
                        for key in z.files:
                            result[f'{case}|{fn}|{key}'] = z[key]
        finally:
            os.chdir(cwd)
    np.savez_compressed(os.path.join(HERE, 'diag_golden.npz'), **result)
    print('wrote', len(result), 'arrays, N =', N)


if __name__ == '__main__':
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.ref_kernels import reference_root
    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())

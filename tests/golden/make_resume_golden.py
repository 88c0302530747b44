"""Golden resume: the reference's Simulation continuing from a plasma state
file that this package's writer produced.

    python tests/golden/make_resume_golden.py [/path/to/lcodePy]

1. The reference (CPU / numba path) runs the rigid-driver configuration
   below; a diagnostic with the reference's hook signature hands the state
   after xi layer K_STORE to ``lcodepy_b200.plasma_state.save_plasmastate``,
   which writes ``resume_state.npz`` (committed).
2. A second reference Simulation with ``external_plasmastate = True`` loads
   that file (lcode/simulation.py:71-72,154-165, load_plasma
   lcode/plasma3d/initialization.py:417-460) and runs the rest of the xi
   loop; its on-axis Ez per xi step and final fields, currents and particles
   go to ``run_resume.npz``.

tests/test_gpu_simulation.py resumes from the same file through this
package's Simulation and compares with ``run_resume.npz``.  The reference
imports through the single-rank ``mpi4py`` and empty ``matplotlib``
stand-ins in ``tests/golden/refstubs``.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from make_golden import OnAxis, base_config, rigid_driver  # noqa: E402

K_STORE = 56
CONFIG = dict(window_length=4.0)


def config():
    return base_config(**{'rigid-beam': True, 'window-length': CONFIG['window_length']})


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, 'refstubs'))
    sys.path.insert(0, ref_root)
    import lcode
    from lcodepy_b200.plasma_state import save_plasmastate

    state_path = os.path.join(HERE, 'resume_state.npz')

    class Store:
        def pull_config(self, config):
            self.k = 0

        def after_step_dxi(self, t, xi, particles, fields, currents, rho_beam):
            if self.k == K_STORE:
                save_plasmastate(state_path, particles, fields, currents, xi_plasma_layer=xi)
            self.k += 1

        def dump(self, *a, **k):
            pass

    sim = lcode.Simulation(config=config(), beam_parameters=rigid_driver,
                           diagnostics=[Store()], runas_filename='')
    sim.step()

    diag = OnAxis()
    sim2 = lcode.Simulation(config=config(), beam_parameters=rigid_driver,
                            diagnostics=[diag], runas_filename='')
    sim2.external_plasmastate = True
    sim2.path_to_plasmastate = state_path
    sim2.step()
    particles, fields, currents = sim2._Simulation__push_solver._plasmastate
    out = {'ez_axis': np.array(diag.ez), 'k_store': K_STORE}
    for k in ('Ex', 'Ey', 'Ez', 'Bx', 'By', 'Bz', 'Phi'):
        out['f_' + k] = np.asarray(getattr(fields, k))
    for k in ('ro', 'jx', 'jy', 'jz'):
        out['c_' + k] = np.asarray(getattr(currents, k))
    for k in ('x_offt', 'y_offt', 'px', 'py', 'pz', 'q'):
        out['p_electrons_' + k] = np.asarray(getattr(particles['electrons'], k))
    np.savez_compressed(os.path.join(HERE, 'run_resume.npz'), **out)
    print('resumed xi steps:', len(diag.ez))


if __name__ == '__main__':
    from oracle.ref_kernels import reference_root
    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())

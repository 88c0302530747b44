"""Golden data for the declustering noise filter, made by running the
reference (CPU / numba path, lcode/plasma3d/noise_filter.py:82-239):

    python tests/golden/make_noise_filter_golden.py [/path/to/lcodePy]

- kat_noise_filter.npz: the filter applied once to seeded electron arrays
  (offsets with exact zeros, momenta, previous chaotic displacements):
  inputs and the filtered px, py, dx_chaotic, dy_chaotic;
- run_declustering.npz: the whole xi loop (21 xi steps) of the rigid-driver
  configuration with 'declustering-enabled' (on-axis Ez per step, final
  fields, currents, electrons).

The reference reads the damping coefficient from 'damping-declustering'
(noise_filter.py:88), a key its defaults do not have, so both files set it.
The reference imports through the stand-ins in tests/golden/refstubs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import base_config, rigid_driver, run_sim  # noqa: E402

FILTER = {'declustering-averaging': 3, 'declustering-force': 0.3,
          'damping-declustering': 0.1, 'declustering-limit': 2e-3}


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, 'refstubs'))
    sys.path.insert(0, ref_root)
    import lcode
    from lcode.config.config import Config
    from lcode.plasma3d.data import Arrays
    from lcode.plasma3d.noise_filter import get_noise_filter

    # ---- one application on seeded arrays ----
    rng = np.random.default_rng(20250317)
    Ns, dxi = 40, 0.05
    cfg = Config({'geometry': '3d', 'processing-unit-type': 'cpu', 'xi-step': dxi, **FILTER})
    nf = get_noise_filter(cfg)
    shp = (Ns, Ns)

    def offsets():
        a = rng.normal(0.0, 1e-3, shp)
        a[rng.random(shp) < 0.05] = 0.0        # exact zeros switch stencil points off
        return a
    inp = {'x_offt': offsets(), 'y_offt': offsets(),
           'px': rng.normal(0, 0.05, shp), 'py': rng.normal(0, 0.05, shp),
           'pz': rng.normal(0, 0.05, shp),
           'dx_chaotic_prev': rng.normal(0, 5e-4, shp),
           'dy_chaotic_prev': rng.normal(0, 5e-4, shp)}
    z = np.zeros(shp)
    full = Arrays(np, q=z - 1, m=z + 1, x_init=z, y_init=z,
                  x_offt=inp['x_offt'].copy(), y_offt=inp['y_offt'].copy(),
                  px=inp['px'].copy(), py=inp['py'].copy(), pz=inp['pz'].copy(),
                  dx_chaotic=z, dy_chaotic=z, dx_chaotic_perp=z, dy_chaotic_perp=z)
    prev = Arrays(np, dx_chaotic=inp['dx_chaotic_prev'].copy(),
                  dy_chaotic=inp['dy_chaotic_prev'].copy(),
                  dx_chaotic_perp=z, dy_chaotic_perp=z)
    out = nf(full, prev)
    kat = {**inp, 'dxi': dxi, **{k.replace('-', '_'): v for k, v in FILTER.items()},
           'out_px': np.asarray(out.px), 'out_py': np.asarray(out.py),
           'out_dx_chaotic': np.asarray(out.dx_chaotic),
           'out_dy_chaotic': np.asarray(out.dy_chaotic)}
    np.savez_compressed(os.path.join(HERE, 'kat_noise_filter.npz'), **kat)

    # ---- a whole xi loop with the filter on ----
    # 21 xi steps: over longer windows this configuration amplifies rounding
    # differences by about 10x per 1.5 xi steps with the filter on, so that a
    # run on other hardware no longer tracks it within 1e-9
    run = run_sim(lcode, base_config(**{'rigid-beam': True, 'declustering-enabled': True,
                                        'window-length': 1.0, **FILTER}), rigid_driver)
    np.savez_compressed(os.path.join(HERE, 'run_declustering.npz'), **run)
    print('kat and run written;', 'max |dx_chaotic|', np.abs(kat['out_dx_chaotic']).max(),
          'steps', len(run['ez_axis']))


if __name__ == '__main__':
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.ref_kernels import reference_root
    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())

"""Known answers of the reference's own GPU beam kernels.

    python tests/golden/make_ref_kernel_golden.py

Builds the reference's CuPy kernel bodies for the host (oracle/ref_kernels.py
reads them from the reference checkout, ``LCODE_REFERENCE``) and runs them on
seeded beam layers.  The output, ``kat_ref_beam.npz``, holds the inputs and
the reference's outputs of:

- ``calculate_substepping_step`` (lcode/beam3d/beam_calculator.py:28-46) and
  ``move_beam_cupy`` (lcode/beam3d/move.py:139-276) on a 65 x 65 grid: a
  layer of 3000 particles (the last 300 fell from the previous layer and keep
  their dt / remaining steps), with particles that stay, fall and are lost,
  for time steps 1 and 5;
- ``deposit_beam_cupy`` (lcode/beam3d/weights.py:108-163) of one layer.

The GPU tests compare liblcb's beam kernels with this file; they never read
the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_kernels as R  # noqa: E402

KEYS6 = ("Ex", "Ey", "Ez", "Bx", "By", "Bz")


def fields(N, seed):
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    a = 0.2 + 0.05 * seed
    return [0.3 * np.sin(a * (i + 1) * X + 0.1 * Y + seed) for i in range(6)]


def push_case(out, tag, seed, time_step, N=65, h=0.05, dxi=0.05, n=3000, layer=9,
              fell_size=300):
    rng = np.random.default_rng(seed)
    b = dict(xi=rng.uniform(-layer * dxi, -(layer - 1) * dxi, n),
             x=rng.normal(0, 0.5, n), y=rng.normal(0, 0.5, n),
             px=rng.normal(0, 5, n), py=rng.normal(0, 5, n),
             pz=rng.choice([-50.0, 0.3, 20.0, 1000.0], n),
             q_m=rng.choice([-1.0, 1.0, 1 / 1836.0, -0.3], n),
             id=np.arange(1, n + 1, dtype=np.int64), dt=np.zeros(n),
             remaining_steps=np.zeros(n, np.int64))
    b["x"][:20] = 1.4   # at the loss radius
    rs0 = rng.integers(1, 4, fell_size)
    b["remaining_steps"][n - fell_size:] = rs0
    b["dt"][n - fell_size:] = time_step / rs0
    Fk, Fk1 = fields(N, seed), fields(N, seed + 7)
    for k, v in b.items():
        out[f"{tag}_in_{k}"] = v.copy()
    for k, f0, f1 in zip(KEYS6, Fk, Fk1):
        out[f"{tag}_fk_{k}"], out[f"{tag}_fk1_{k}"] = f0, f1
    size = n - fell_size
    dt1 = R.substepping(b["q_m"][:size].copy(), b["pz"][:size].copy(), 2.0)
    b["dt"][:size] = dt1 * time_step
    b["remaining_steps"][:size] = (1.0 / dt1).astype(np.int64)
    Rw = h * N / 2
    lost, moved, fell = R.move_beam(dxi, max(0.9 * Rw, Rw - 1), layer - 1, h, N, b["q_m"],
                                    b["dt"], Fk, Fk1, b["remaining_steps"], b["id"], b["x"],
                                    b["y"], b["xi"], b["px"], b["py"], b["pz"])
    for k, v in b.items():
        out[f"{tag}_out_{k}"] = v
    out[f"{tag}_lost"], out[f"{tag}_moved"], out[f"{tag}_fell"] = lost, moved, fell
    out[f"{tag}_params"] = np.array([N, h, dxi, layer, fell_size, time_step, 2.0])
    print(tag, "lost", lost.sum(), "moved", moved.sum(), "fell", fell.sum())


def deposit_case(out, N=65, h=0.05, dxi=0.05, layer=7, n=5000):
    rng = np.random.default_rng(5)
    x, y = rng.normal(0, 0.4, n), rng.normal(0, 0.4, n)
    xi = rng.uniform(-layer * dxi - dxi, -layer * dxi, n)
    q = rng.uniform(-1, 1, n)
    ro0, ro1 = rng.normal(0, 1, (N, N)), np.zeros((N, N))
    out.update(dep_x=x, dep_y=y, dep_xi=xi, dep_q=q, dep_ro0_in=ro0.copy(),
               dep_params=np.array([N, h, dxi, layer]))
    xi_loc = (-dxi * layer - xi) / dxi
    R.deposit_beam(N, x / h + 0.5, y / h + 0.5, xi_loc, q, ro0, ro1)
    out.update(dep_ro0=ro0, dep_ro1=ro1)


def main():
    R.build(force=True)
    out = {}
    push_case(out, "t1", 31, 1.0)
    push_case(out, "t5", 32, 5.0)
    deposit_case(out)
    np.savez_compressed(os.path.join(HERE, "kat_ref_beam.npz"), **out)


if __name__ == "__main__":
    main()

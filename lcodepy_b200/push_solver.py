"""The xi loop of one time step (lcode/push_solvers/push_solver.py:215-286).

Per xi step i = 0 .. round(window-length / xi-step) (inclusive, as in the
reference):
  1. beam layer i is laid out (rigid: fn(xi); otherwise deposit),
  2. the plasma advances one xi step (Plane2d3vPlasmaSolver.step_dxi),
  3. beam layer i-1 (plus particles that fell into it) is pushed between the
     previous and the new plasma fields; moved particles go to the drain,
  4. diagnostics see the new state.
On-axis Ez is recorded on the device every step and the reference's
"t=..., xi=..., Ez=..." lines are printed after the loop, so the loop never
waits for the host.
"""
from __future__ import annotations

import torch

from .beam3d import BeamCalculator, RigidBeamCalculator
from .config import Config
from .data import Arrays
from .solver import Plane2d3vPlasmaSolver


class PusherAndSolver3D:
    def __init__(self, config: Config, device=None):
        self.config = config
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.plasma_solver = Plane2d3vPlasmaSolver(config, self.device)
        self.rigid = config.getbool('rigid-beam')
        self.beam_calculator = (RigidBeamCalculator(config, self.device) if self.rigid
                                else BeamCalculator(config, self.device))
        self.xi_max = config.getfloat('window-length')
        self.xi_step_size = config.getfloat('xi-step')
        self.xi_steps = round(self.xi_max / self.xi_step_size)
        self.grid_steps = config.getint('window-width-steps')
        pe = config.getraw('print-every')
        self.print_every = 10 if pe is None else int(pe)
        self._plasmastate = None
        self.ez_axis = None
        self.lost = []

    def step_dt(self, xi_plasma_layer_start, beam_source, beam_drain,
                current_time, diagnostics_list=(), step_hook=None):
        """Run the xi loop of one time step.  The plasma state must have been
        initialised on the solver (Simulation does this).  ``step_hook(k)``,
        if given, is called before the k-th xi step and once after the last
        (k = number of steps); the benchmark uses it to place its events."""
        ps = self.plasma_solver
        bc = self.beam_calculator
        first = round(-xi_plasma_layer_start / self.xi_step_size) + 1
        last = self.xi_steps
        if self.rigid:
            bc.prepare(beam_source.get_beam_layer_to_layout(first), first, last)
        else:
            bc.start_time_step(beam_source)
            bc.layout_first(first)
        n_iter = max(last - first + 1, 0)
        hist, counter = ps.record_axis(self.xi_steps + 1)
        counter.zero_()
        self.lost = None
        for k, xi_i in enumerate(range(first, last + 1)):
            if step_hook is not None:
                step_hook(k)
            if self.rigid:
                rb_full, rb_prev = bc.layout_beam_layer(None, xi_i)
            else:
                rb_full, rb_prev = bc.rho(xi_i)
            ps.step_dxi(rb_full, rb_prev, bc.rho_divisor, stable_planes=True)
            if not self.rigid:
                # push layer i-1 between the previous and new fields, lay out i+1
                bc.after_plasma_step(xi_i, ps.last_fields, ps.prev_fields)
                stream_out = getattr(beam_drain, "after_xi_step", None)
                if stream_out is not None:    # a pipelined run streams its drain
                    stream_out(xi_i, bc)
            if diagnostics_list:
                xi_layer = -self.xi_step_size * xi_i
                rho = rb_full / bc.rho_divisor
                for d in diagnostics_list:
                    d.after_step_dxi(current_time, xi_layer,
                                     {k2: v.wrapped() for k2, v in ps.particles_dict().items()},
                                     ps.prev_fields.arrays().wrapped(),
                                     ps.prev_currents.arrays().wrapped(),
                                     Arrays(None, r=rho).wrapped().r)
        if step_hook is not None:
            step_hook(n_iter)
        ps.check_errors()
        if not self.rigid:
            e = int(bc.err.item())
            if e:
                bc.err.zero_()
                raise RuntimeError(f"beam device error word 0x{e:x}: a beam stencil "
                                   "left the grid, a substep limit was hit or a beam "
                                   "buffer would overflow")
            moved, self.lost = bc.finish()
            beam_drain.push_beam_layer(moved)
            if getattr(beam_source, "streaming", False):
                beam_source.finish()
        self.ez_axis = hist[:n_iter].clone()
        ez = self.ez_axis
        if self.print_every:
            vals = ez.cpu().numpy()
            for k, xi_i in enumerate(range(first, last + 1)):
                if xi_i % self.print_every == 0:
                    print(f't={current_time:+.4f}, xi={-xi_i * self.xi_step_size:+.4f} '
                          f'Ez={vals[k]:+.4e}', flush=True)
        xi_layer = -self.xi_step_size * self.xi_steps
        for d in diagnostics_list:
            d.dump(current_time, xi_layer,
                   {k2: v.wrapped() for k2, v in ps.particles_dict().items()},
                   ps.prev_fields.arrays().wrapped(), ps.prev_currents.arrays().wrapped(),
                   beam_drain)
        self._plasmastate = (ps.particles_dict(), ps.prev_fields.arrays(),
                             ps.prev_currents.arrays())

"""On-axis and slice diagnostics recorded on the device.

The reference's ``FXiDiag`` (lcode/diagnostics/FXi/FXi.py:48-160, 3D strategy
FXi/Strategy3D.py:28-95) and ``SliceDiag`` (lcode/diagnostics/slice.py:40-364)
read every recorded value back to the host as it is taken (``get(val)``, one
synchronisation per value and xi step).  Here the values stay on the device:
each xi step appends a device copy (a probe gather, a slice, or a reduction)
to a per-quantity list, and ``dump`` stacks the list, reads it back once and
writes the reference's npz files (same directory, file names, keys, shapes and
dtypes), so that post-processing written for the reference reads them
unchanged.

``ParticlesDiag`` (lcode/diagnostics/particles.py:11-110) writes plasma
particle snapshots and the moved beam in the reference's file names and npz
keys; its arrays are read back only when a snapshot is due.

The constructors, flag values and output cadence (``output_period`` in time,
``saving_xi_period`` in xi for x-y slices, the first time step always) are the
reference's.  Inputs are what the drop-in ``Simulation`` passes to
diagnostics (``DeviceArray`` views with the tensor in ``.t``); plain numpy
arrays are accepted too.  ``OutputType.PICTURES`` needs matplotlib, which
this package does not depend on.
"""
from __future__ import annotations

import math
from collections import defaultdict
from pathlib import Path

import numpy as np
import torch


class OutputType:
    """Output kinds (lcode/diagnostics/utils.py:3-8)."""
    __slots__ = ()
    NUMBERS = 0x1
    PICTURES = 0x2
    ALL = NUMBERS | PICTURES


class FXiType:
    """Quantities of FXiDiag (lcode/diagnostics/FXi/FXi.py:15-44)."""
    __slots__ = ()
    Ex = 0x1
    Ey = 0x2
    Ez = 0x4
    E = Ex | Ey | Ez
    Er = Ex
    Ef = Ey
    Bx = 0x8
    By = 0x10
    Bz = 0x20
    B = Bx | By | Bz
    Bf = Bx
    EB = E | B
    Phi = 0x40
    ne = 0x80
    ni = 0x100
    n = ne | ni
    rho_beam = 0x200
    Sf = 0x400
    dx_chaotic = 0x800
    dy_chaotic = 0x1000
    dx_chaotic_perp = 0x2000
    dy_chaotic_perp = 0x4000


class SliceType:
    """Slice planes of SliceDiag (lcode/diagnostics/slice.py:9-15)."""
    __slots__ = ()
    XI_R = 0x1
    XI_X = 0x2
    XI_Y = 0x4
    X_Y = 0x8


class SliceValue:
    """Quantities of SliceDiag (lcode/diagnostics/slice.py:17-38)."""
    __slots__ = ()
    Ex = 0x1
    Ey = 0x2
    Ez = 0x4
    E = Ex | Ey | Ez
    Er = Ex
    Ef = Ey
    Bx = 0x8
    By = 0x10
    Bz = 0x20
    B = Bx | By | Bz
    Bf = Bx
    EB = E | B
    Phi = 0x40
    ne = 0x80
    ni = 0x100
    n = ne | ni
    rho_beam = 0x200


def absremainder(x, y):
    """|IEEE remainder| (lcode/diagnostics/utils.py:41-53)."""
    return abs(math.remainder(x, y))


def _t(a) -> torch.Tensor:
    """The tensor behind a DeviceArray, a tensor, or a host array."""
    if hasattr(a, "t") and isinstance(a.t, torch.Tensor):
        return a.t
    if isinstance(a, torch.Tensor):
        return a
    return torch.as_tensor(np.asarray(a))


def _rank0() -> bool:
    # the reference records on MPI rank 0 only; this package runs one
    # process per simulation
    return True


class Diagnostic:
    """Base with the reference's cadence test (lcode/diagnostics/utils.py:16-24)."""

    @staticmethod
    def condition_check(current_time, output_period, time_step_size):
        return absremainder(current_time, output_period) <= time_step_size / 2

    @staticmethod
    def _stack(values: list) -> np.ndarray:
        """One read-back of a list of device tensors (or host scalars)."""
        if not values:
            return np.array([])
        if isinstance(values[0], torch.Tensor):
            return torch.stack(values).cpu().numpy()
        return np.array(values)


def _check_pictures(output_type):
    if output_type & OutputType.PICTURES:
        try:
            import matplotlib.pyplot  # noqa: F401
        except ImportError as e:
            raise ImportError("OutputType.PICTURES needs matplotlib, which is not "
                              "installed") from e


def _energy_flux(h, particles, fields) -> torch.Tensor:
    """Integral energy flux of the electromagnetic field and the electrons'
    motion (FXi/Strategy3D.py:6-25), reduced on the device."""
    Ex, Ey, Ez = _t(fields.Ex), _t(fields.Ey), _t(fields.Ez)
    Bx, By, Bz = _t(fields.Bx), _t(fields.By), _t(fields.Bz)
    se = (Ez ** 2 + Bz ** 2 + (Ex - By) ** 2 + (Ey + Bx) ** 2) * h ** 2 / 2
    el = particles['electrons']
    m, px, py, pz = _t(el.m), _t(el.px), _t(el.py), _t(el.pz)
    motion = torch.sqrt(m ** 2 + px ** 2 + py ** 2 + pz ** 2) - m
    return torch.sum(motion) + torch.sum(se)


class FXiDiag(Diagnostic):
    """Values at probe points per xi step (on-axis by default), written as
    diagnostics[/directory_name]/f_xi_<time>.npz with keys 'xi' and one per
    quantity (FXi/FXi.py:48-160)."""

    def __init__(self, output_period=100, saving_xi_period=100, f_xi=FXiType.Ez,
                 output_type=OutputType.NUMBERS, probe_lines=None, directory_name=None):
        self._f_xi = f_xi
        self._output_period = output_period
        self._saving_xi_period = saving_xi_period
        self._output_type = output_type
        self._probe_lines = probe_lines
        self._directory = Path('diagnostics') if directory_name is None else \
            Path('diagnostics') / directory_name
        self._data = defaultdict(list)
        self._data['xi'] = []
        self._first = _rank0()
        _check_pictures(output_type)

    def pull_config(self, config):
        self._h = config.getfloat('transverse-step')
        self._time_step = config.getfloat('time-step')
        self._xi_step = config.getfloat('xi-step')
        if self._output_period < self._time_step:
            self._output_period = self._time_step
        if self._saving_xi_period < self._xi_step:
            self._saving_xi_period = self._xi_step
        steps = config.getint('window-width-steps')
        pl = self._probe_lines
        if pl is None:
            ax, ay = 0, 0
        else:
            pl = np.array(pl)
            if pl.ndim < 1 or pl.ndim > 2:
                raise ValueError('probe_lines must be 1D or 2D')
            if pl.ndim == 1:
                ax, ay = pl, np.zeros_like(pl)
            else:
                ax, ay = pl[0], pl[1]
        # probe indices (FXi/Strategy3D.py:34-59)
        self._ix = (steps // 2 + np.round(ax / self._h)).astype(int)
        self._iy = (steps // 2 + np.round(ay / self._h)).astype(int)
        self._idx = None

    def _probe(self, plane: torch.Tensor) -> torch.Tensor:
        if self._idx is None or self._idx[0].device != plane.device:
            self._idx = (torch.as_tensor(self._ix, device=plane.device),
                         torch.as_tensor(self._iy, device=plane.device))
        return plane[self._idx].clone()

    def after_step_dxi(self, current_time, xi_plasma_layer, plasma_particles,
                       plasma_fields, plasma_currents, rho_beam):
        if not (self._first or self.condition_check(current_time, self._output_period,
                                                    self._time_step)):
            return
        d, f = self._data, self._f_xi
        for flag, name in ((FXiType.Ex, 'Ex'), (FXiType.Ey, 'Ey'), (FXiType.Ez, 'Ez'),
                           (FXiType.Bx, 'Bx'), (FXiType.By, 'By'), (FXiType.Bz, 'Bz')):
            if f & flag:
                d[name].append(self._probe(_t(getattr(plasma_fields, name))))
        if f & FXiType.ne:
            d['ne'].append(self._probe(_t(plasma_currents.ro)[0]))
        if f & FXiType.ni:
            d['ni'].append(self._probe(_t(plasma_currents.ro)[1]))
        if f & FXiType.rho_beam:
            d['rho_beam'].append(self._probe(_t(rho_beam)))
        if f & FXiType.Phi:
            d['Phi'].append(self._probe(_t(plasma_fields.Phi)))
        if f & FXiType.Sf:
            d['Sf'].append(_energy_flux(self._h, plasma_particles, plasma_fields))
        # the declustering filter's chaotic displacements of the electrons:
        # the largest |value| over the lattice, and over its central two
        # thirds for the "perp" quantities (Strategy3D.py:85-96, which reads
        # the same arrays for both)
        for flag, name, central in ((FXiType.dx_chaotic, 'dx', False),
                                    (FXiType.dy_chaotic, 'dy', False),
                                    (FXiType.dx_chaotic_perp, 'dx', True),
                                    (FXiType.dy_chaotic_perp, 'dy', True)):
            if f & flag:
                a = _t(getattr(plasma_particles['electrons'], f'{name}_chaotic'))
                if central:
                    a1 = int(a.shape[0] / 6)
                    a = a[a1:5 * a1, a1:5 * a1]
                d[f'{name}_chaotic' + ('_perp' if central else '')].append(a.abs().max())
        d['xi'].append(xi_plasma_layer)

    def dump(self, current_time, xi_plasma_layer, plasma_particles, plasma_fields,
             plasma_currents, beam_drain):
        if not self._first and not self.condition_check(current_time, self._output_period,
                                                        self._time_step):
            return
        self._directory.mkdir(parents=True, exist_ok=True)
        data = {k: self._stack(v) for k, v in self._data.items()}
        if self._output_type & OutputType.NUMBERS:
            np.savez(self._directory / f'f_xi_{current_time:08.2f}.npz', **data)
        if self._output_type & OutputType.PICTURES:
            import matplotlib.pyplot as plt
            for name, values in data.items():
                if name == 'xi':
                    continue
                plt.plot(data['xi'], values)
                plt.title(name)
                plt.savefig(self._directory / f'{name}_{current_time:08.2f}.jpg')
                plt.close()
        self._data = defaultdict(list)
        self._first = False


_SLICE_QUANTITIES = ((SliceValue.Ex, 'Ex'), (SliceValue.Ey, 'Ey'), (SliceValue.Ez, 'Ez'),
                     (SliceValue.Bx, 'Bx'), (SliceValue.By, 'By'), (SliceValue.Bz, 'Bz'),
                     (SliceValue.ne, 'ne'), (SliceValue.ni, 'ni'),
                     (SliceValue.rho_beam, 'rho_beam'), (SliceValue.Phi, 'Phi'))


def _limits(limits, default):
    if limits is None:
        return default
    lim = np.array(limits)
    if lim.ndim != 2:
        raise ValueError("limits must be 2D array")
    return lim[0, 0], lim[0, 1], lim[1, 0], lim[1, 1]


class _Slicer:
    """Common part of the 3D slicers: picks the diag's quantities from a
    window of the planes and appends device copies."""

    def __init__(self, diag):
        self.diag = diag
        c = diag._config
        self.window_length = c.getfloat('window-length')
        self.steps = c.getint('window-width-steps')
        self.width = c.getfloat('window-width')
        self.h = c.getfloat('transverse-step')

    def _index(self, i, j):
        """Clip an index pair to the grid like the reference."""
        raise NotImplementedError

    def _take(self, plane: torch.Tensor) -> torch.Tensor:
        raise NotImplementedError

    def record(self, xi, fields, currents, rho_beam):
        d, v = self.diag._data, self.diag._slice_value
        d['xi'].append(xi)
        for flag, name in _SLICE_QUANTITIES:
            if not v & flag:
                continue
            if name == 'ne':
                plane = _t(currents.ro)[0]
            elif name == 'ni':
                plane = _t(currents.ro)[1]
            elif name == 'rho_beam':
                plane = _t(rho_beam)
            else:
                plane = _t(getattr(fields, name))
            d[name].append(self._take(plane).clone())


class _XiX(_Slicer):
    """xi-x slices: the column at y = offset over [from_2, to_2) in x
    (slice.py:134-207)."""

    def __init__(self, diag):
        super().__init__(diag)
        n, h = self.steps, self.h
        f1, t1, f2, t2 = _limits(diag._limits, (0, -self.window_length, -self.width / 2,
                                                self.width / 2))
        self.from_1, self.to_1 = f1, t1
        self.from_2 = int(np.clip(np.round(f2 / h) + n // 2, 0, n))
        self.to_2 = int(np.clip(np.round(t2 / h) + n // 2, 0, n))
        self._grid = (np.arange(self.from_2, self.to_2) - n // 2) * h
        self.offset = int(np.clip(n // 2 + diag._offset // h, 0, n))

    def _take(self, plane):
        return plane[self.from_2:self.to_2, self.offset]

    def process(self, current_time, xi, particles, fields, currents, rho_beam):
        if xi < self.to_1 or xi > self.from_1:
            return
        self.record(xi, fields, currents, rho_beam)


class _XiY(_XiX):
    """xi-y slices: the row at x = offset over [from_2, to_2) in y
    (slice.py:209-276); the offset is clipped to the last row."""

    def __init__(self, diag):
        super().__init__(diag)
        self.offset = int(np.clip(self.steps // 2 + diag._offset // self.h, 0, self.steps - 1))

    def _take(self, plane):
        return plane[self.offset, self.from_2:self.to_2]


class _XY(_Slicer):
    """x-y slices every saving_xi_period of xi (slice.py:278-364)."""

    def __init__(self, diag):
        super().__init__(diag)
        n, h = self.steps, self.h
        f1, t1, f2, t2 = _limits(diag._limits, (-self.width / 2, self.width / 2,
                                                -self.width / 2, self.width / 2))
        self.from_1 = int(np.clip(np.round(f1 / h) + n // 2, 0, n - 1))
        self.to_1 = int(np.clip(np.round(t1 / h) + n // 2, 0, n - 1))
        self.from_2 = int(np.clip(np.round(f2 / h) + n // 2, 0, n - 1))
        self.to_2 = int(np.clip(np.round(t2 / h) + n // 2, 0, n - 1))
        gx = (np.arange(self.from_1, self.to_1) - n // 2) * h
        gy = (np.arange(self.from_2, self.to_2) - n // 2) * h
        self._grid = np.vstack((gx, gy))

    def _take(self, plane):
        return plane[self.from_1:self.to_1, self.from_2:self.to_2]

    def process(self, current_time, xi, particles, fields, currents, rho_beam):
        d = self.diag
        if not (absremainder(current_time, d._output_period) <= d._time_step / 2 and
                absremainder(xi, d._saving_xi_period) <= d._xi_step / 2):
            return
        self.record(xi, fields, currents, rho_beam)


class SliceDiag(Diagnostic):
    """Field / density slices per xi step, written as
    diagnostics[/directory_name]/slice_<time>.npz with keys 'xi', one per
    quantity and the slice's grid 'x' (slice.py:40-132).  3D geometry."""

    def __init__(self, slice_type, slice_value=SliceValue.rho_beam,
                 output_type=OutputType.NUMBERS, limits=None, offset=0, output_period=100,
                 saving_xi_period=100, directory_name=None):
        self._slice_type = slice_type
        self._slice_value = slice_value
        self._output_type = output_type
        self._limits = limits
        self._offset = offset
        self._output_period = output_period
        self._saving_xi_period = saving_xi_period
        self._first = _rank0()
        self._directory = Path('diagnostics') if directory_name is None else \
            Path('diagnostics') / directory_name
        self._data = defaultdict(list)

    def pull_config(self, config):
        self._config = config
        self._time_step = config.getfloat('time-step')
        self._xi_step = config.getfloat('xi-step')
        if self._output_period < self._time_step:
            self._output_period = self._time_step
        if config.get('geometry') != '3d':
            raise NotImplementedError("this package computes the 3D geometry only")
        st = self._slice_type
        if st == SliceType.XI_X or st == SliceType.XI_R:
            self._slicer = _XiX(self)
        elif st == SliceType.XI_Y:
            self._slicer = _XiY(self)
        elif st == SliceType.X_Y:
            self._slicer = _XY(self)
        else:
            raise NotImplementedError

    def after_step_dxi(self, current_time, *args, **kwargs):
        if self._first or absremainder(current_time, self._output_period) <= self._time_step / 2:
            self._slicer.process(current_time, *args, **kwargs)

    def dump(self, current_time, xi_plasma_layer, plasma_particles, plasma_fields,
             plasma_currents, beam_drain):
        if not self._first and not self.condition_check(current_time, self._output_period,
                                                        self._time_step):
            return
        self._directory.mkdir(parents=True, exist_ok=True)
        data = {k: self._stack(v) for k, v in self._data.items()}
        if self._output_type & OutputType.NUMBERS:
            np.savez(self._directory / f'slice_{current_time:08.2f}.npz', **data,
                     x=self._slicer._grid)
        self._data = defaultdict(list)
        self._first = False


class ParticlesDiag(Diagnostic):
    """Plasma particle snapshots every saving_xi_period of xi and at the end
    of a time step, and the moved beam at the end of a time step
    (lcode/diagnostics/particles.py:11-110): files
    diagnostics[/directory_name]/snapshots/plasma_<sort>_<time>_<xi>.npz,
    plasma_<sort>_<time>.npz and beam_<time>.npz."""

    def __init__(self, save_beam=False, save_plasma=False, output_period=1000.0,
                 saving_xi_period=math.inf, directory_name=None):
        self._save_beam = save_beam
        self._save_plasma = save_plasma
        self._output_period = output_period
        self._saving_xi_period = saving_xi_period
        self._directory = Path('diagnostics') if directory_name is None else \
            Path('diagnostics') / directory_name
        self._first = _rank0()

    def pull_config(self, config):
        self._time_step = config.getfloat('time-step')
        self._xi_step = config.getfloat('xi-step')
        if self._output_period < self._time_step:
            self._output_period = self._time_step
        if self._saving_xi_period < self._xi_step:
            self._saving_xi_period = self._xi_step
        if config.getbool('rigid-beam') and self._save_beam:
            raise Exception("We cannot save the beam in the case of a rigid beam."
                            "Please, change save_beam to False.")

    def conditions_check(self, current_time, xi_plasma_layer):
        return (absremainder(current_time, self._output_period) <= self._time_step / 2 and
                absremainder(xi_plasma_layer, self._saving_xi_period) <= self._xi_step / 2)

    @staticmethod
    def _save_sorts(particles, e_name, i_name):
        for sort, name in (('electrons', e_name), ('ions', i_name)):
            if sort in particles:
                particles[sort].save(name)

    def after_step_dxi(self, current_time, xi_plasma_layer, plasma_particles, plasma_fields,
                       plasma_currents, rho_beam):
        if self._saving_xi_period == math.inf or not self._save_plasma:
            return
        if not self.conditions_check(current_time, xi_plasma_layer):
            return
        snap = self._directory / "snapshots"
        snap.mkdir(parents=True, exist_ok=True)
        tag = f"{current_time:08.2f}_{xi_plasma_layer:+09.2f}"
        self._save_sorts(plasma_particles, snap / f"plasma_electrons_{tag}.npz",
                         snap / f"plasma_ions_{tag}.npz")

    def dump(self, current_time, xi_plasma_layer, plasma_particles, plasma_fields,
             plasma_currents, beam_drain):
        if not self._first and absremainder(current_time, self._output_period) > self._time_step / 2:
            return
        self._first = False
        self._directory.mkdir(parents=True, exist_ok=True)
        if self._save_beam:
            beam_drain.save(self._directory / f"beam_{current_time:08.2f}.npz")
        if self._save_plasma:
            self._save_sorts(plasma_particles,
                             self._directory / f"plasma_electrons_{current_time:08.2f}.npz",
                             self._directory / f"plasma_ions_{current_time:08.2f}.npz")

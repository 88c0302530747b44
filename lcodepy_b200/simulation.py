"""Top-level ``Simulation`` with the reference's constructor and ``step``
(lcode/simulation.py:27-269), 3D geometry only.

Everything runs on the current CUDA device: the config key
'processing-unit-type' is accepted for compatibility but this package has no
CPU path, and it raises if CUDA is unavailable or liblcb.so is missing.

When torch.distributed is initialised with more than one rank, ``step``
runs the reference's time-step pipeline (lcode/simulation.py:222-264 with
lcode/mpi/beam_io.py): rank r computes the time steps r, r + W, ... and
streams its moved beam to the next rank during its xi loop (pipeline.py).
"""
from __future__ import annotations

import copy

import numpy as np
import torch

from . import _lib
from .beam3d import (BeamDrain, BeamParticles, BeamSource, RigidBeamDrain,
                     RigidBeamSource)
from .beam_generator import generate_beam, particle_dtype3d
from .config import Config, default_config_values
from .push_solver import PusherAndSolver3D


class Simulation:
    def __init__(self, config=default_config_values, beam_parameters={},
                 diagnostics=[], runas_filename="runas.py"):
        self.config = copy.copy(config)
        self.beam_parameters = copy.copy(beam_parameters)
        self.diagnostics_list = copy.copy(diagnostics)
        self.runas_filename = runas_filename
        self.current_time = 0.
        self.beam_source = None
        self.beam_drain = None
        self.__beam_particles = None
        self.external_plasmastate = False
        self.path_to_plasmastate = 'plasmastate.npz'
        self.__geometry = None
        if not torch.cuda.is_available():
            raise RuntimeError("lcodepy_b200 needs a CUDA device (B200); there is no CPU path")
        _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.__push_solver = None
        self.__pull_config()

    def __pull_config(self):
        self.__config = Config(self.config)
        self.__time_limit = self.__config.getfloat('time-limit')
        self.__time_step_size = self.__config.getfloat('time-step')
        self.__rigid_beam = self.__config.getbool('rigid-beam')
        geometry = self.__config.get('geometry').lower()
        if self.__geometry is None:
            self.__geometry = geometry
        elif self.__geometry != geometry:
            raise Exception("Sorry, update geometry does not support now.")
        if self.__geometry != '3d':
            raise NotImplementedError("lcodepy_b200 implements the 3D geometry only "
                                      f"(got geometry={geometry!r})")
        self.particle_dtype = particle_dtype3d
        self.__config._adjust_config_values_3d()
        self.__push_solver = PusherAndSolver3D(self.__config, self.device)
        for diagnostic in self.diagnostics_list:
            diagnostic.pull_config(config=self.__config)

    @property
    def push_solver(self) -> PusherAndSolver3D:
        return self.__push_solver

    @property
    def effective_config(self) -> Config:
        return self.__config

    def load_beamfile(self, path_to_beamfile='beamfile.npz'):
        """simulation.py:136-146."""
        if self.__rigid_beam:
            raise Exception("We cannot load a beam in the case of a rigid beam.")
        self.__beam_particles = BeamParticles(self.device).load(path_to_beamfile)

    def step(self, N_steps=None):
        """Compute N time steps (simulation.py:173-269)."""
        self.__pull_config()
        if self.runas_filename:
            self.__config.dump(self.runas_filename)
        if self.__rigid_beam:
            N_steps = 1
            print("Since the beam is rigid, the code will simulate only one time step.")
        elif N_steps is None:
            N_steps = int(self.__time_limit / self.__time_step_size)
            print("Since the number of time steps hasn't been set explicitly,",
                  f"the code will simulate {N_steps} time steps with a time",
                  f"step size = {self.__time_step_size}.")
        else:
            self.__time_limit = N_steps * self.__time_step_size + self.current_time
            print("Since the number of time steps has been set explicitly,",
                  f"the code will simulate till time limit = {self.__time_limit},",
                  f"with a time step size = {self.__time_step_size}.")

        if self.__rigid_beam:
            self.beam_source = RigidBeamSource(self.__config, self.beam_parameters)
            self.beam_drain = RigidBeamDrain(self.__config)
        elif self.beam_source is None:
            if self.__beam_particles is None:
                beam = generate_beam(self.__config, self.beam_parameters)
            else:
                beam = self.__beam_particles
            self.beam_source = BeamSource(self.__config, beam, self.device)
            self.beam_drain = BeamDrain(self.__config, self.device)

        ps = self.__push_solver
        # an external plasma state replaces the initial plasma of every time
        # step, and the xi loop continues after its layer (simulation.py:154-165)
        state = None
        if self.external_plasmastate:
            from .plasma_state import load_plasmastate
            state = load_plasmastate(self.path_to_plasmastate, ps.plasma_solver.sort_names)

        def one_time_step(source, drain):
            ps.plasma_solver.init_state(self.current_time)
            xi_start = self.__config.getfloat('xi-step')
            if state is not None:
                xs = ps.plasma_solver.load_state(state)
                if xs is not None:
                    xi_start = xs
            ps.step_dt(xi_start, source, drain, self.current_time, self.diagnostics_list)

        world, rank = 1, 0
        # 'time-step-pipeline': False keeps every rank an independent replica
        # (a process group set up for something else, e.g. timing replicas)
        pipe = self.__config.getraw('time-step-pipeline')
        if (torch.distributed.is_available() and torch.distributed.is_initialized()
                and (pipe is None or bool(pipe))):
            world, rank = torch.distributed.get_world_size(), torch.distributed.get_rank()
        if world > 1:
            self.__step_pipelined(N_steps, world, rank, one_time_step)
            print('The work is done!')
            return
        self.current_time = self.__time_step_size
        for t_i in range(N_steps):
            one_time_step(self.beam_source, self.beam_drain)
            if t_i != N_steps - 1 and not self.__rigid_beam:
                self.beam_source = BeamSource(self.__config, self.beam_drain.beam_slice(),
                                              self.device)
                self.beam_drain = BeamDrain(self.__config, self.device)
            self.current_time = self.current_time + self.__time_step_size
        print('The work is done!')

    def __step_pipelined(self, N_steps, world, rank, one_time_step):
        """Time steps rank, rank + world, ... of N_steps (mpi/transport.py:
        50-52); the beam of time step t comes streamed from the rank that
        computed t - 1 and goes streamed to the rank that computes t + 1
        (pipeline.py).  The rank that computes the last time step keeps its
        moved beam in ``beam_drain``; a rigid driver is one time step, on
        rank 0."""
        from .pipeline import BeamTransport, StreamingDrain, StreamingSource, steps_of_rank
        mine = steps_of_rank(N_steps, rank, world)
        self.current_time = self.__time_step_size * (rank + 1)   # simulation.py:244
        if self.__rigid_beam:
            for _ in mine:
                one_time_step(self.beam_source, self.beam_drain)
                self.current_time += self.__time_step_size * world
            return
        if getattr(self.beam_source, "streaming", False):
            raise NotImplementedError("a pipelined run is one step() call; start a new "
                                      "Simulation for the next one")
        transport = BeamTransport(self.device)
        capacity = self.beam_source.beam.size
        chunk = int(self.__config.getraw('pipeline-chunk-steps') or 32)
        initial = self.beam_source
        for t in mine:
            source = (initial if t == 0 else
                      StreamingSource(self.__config, transport, (rank - 1) % world, capacity))
            drain = (BeamDrain(self.__config, self.device) if t == N_steps - 1 else
                     StreamingDrain(self.__config, transport, (rank + 1) % world, chunk,
                                    self.device))
            one_time_step(source, drain)
            self.beam_source, self.beam_drain = source, drain
            self.current_time += self.__time_step_size * world
        transport.wait()

"""RUMD's Python surface for the LJ/NVT path: ``import rumd_b200.rumd as rumd``.

The classes (Sample, Pot_LJ_12_6, Pot_IPL_12_6, Pot_LJ_12_6_smooth_2_4,
Pot_IPL_n, IntegratorNVT, IntegratorNVE)
are the C++ classes of ``_rumd`` (pybind11), named as RUMD's SWIG module names
them (Swig/rumd.i, Potentials.i, Integrators.i); ``NoShift``,
``ShiftedPotential`` and ``ShiftedForce`` are the cut-off methods
(Swig/Potentials.i:74-76).  ``Simulation`` follows Python/rumd/Simulation.py:
it owns the time-step loop, resets the total momentum every 100 steps, records
energies every 256 steps unless output is suppressed, writes the
"nsteps, time, MATS" timing line, and ends a run with one more CalcF.

The loop itself runs inside the engine as fused CUDA-graph launches
(``Sample.Run``); a per-step Python loop (``Simulation.RunStepwise``) drives
the same kernels one call at a time for callers that need Python hooks
between steps.
"""
import os
import time

import numpy as np

from . import build as _build

if not os.path.exists(_build.module_path()):
    raise ImportError(f"{_build.module_path()} is missing: run `python -m rumd_b200.build`")

from ._rumd import (  # noqa: E402,F401
    IntegratorNVE,
    IntegratorNVT,
    NoShift,
    PairPotential,
    Pot_IPL_12_6,
    Pot_IPL_n,
    Pot_LJ_12_6,
    Pot_LJ_12_6_smooth_2_4,
    RUMD_cudaResourceError,
    RUMD_Error,
    Sample,
    ShiftedForce,
    ShiftedPotential,
)

ENERGY_COLUMNS = ("pe", "ke", "p", "T", "Etot", "W", "Ps")


class Simulation:
    """Owns a Sample and the time-step loop (Python/rumd/Simulation.py:10-622)."""

    def __init__(self, filename=None, pb=0, tp=0, verbose=True, sample=None):
        if sample is None:
            sample = Sample(pb, tp)
            sample.SetVerbose(verbose)
            if filename is not None:
                sample.ReadConf(filename)
        self.sample = sample
        self.verbose = verbose
        self.itg = None
        self.potentialList = []
        self.momentum_reset_interval = 100      # Simulation.py:56-59
        self.energies_interval = 256            # Simulation.py:44
        self.energies = np.zeros((0, len(ENERGY_COLUMNS) + 1))
        self.timing = []
        self.elapsed = 0.0

    # -- set-up (Simulation.py:86-214) ---------------------------------------
    def SetVerbose(self, vb):
        self.verbose = vb
        self.sample.SetVerbose(vb)

    def SetPB_TP(self, pb, tp):
        self.sample.SetPB_TP(pb, tp)

    def SetPotential(self, potential):
        self.potentialList = [potential]
        self.sample.SetPotential(potential)

    def AddPotential(self, potential, clear=False):
        """Simulation.AddPotential (Simulation.py:178-196): appends to the list that
        CalcF evaluates (two pair potentials at most)."""
        if clear or not self.potentialList:
            self.SetPotential(potential)
        else:
            self.sample.AddPotential(potential)
            self.potentialList.append(potential)

    def SetIntegrator(self, itg):
        self.sample.SetIntegrator(itg)
        self.itg = itg

    def SetMomentumResetInterval(self, mom_reset_interval):
        self.momentum_reset_interval = int(mom_reset_interval)

    def SetOutputScheduling(self, manager, schedule, interval=None, **_):
        """Only the energies manager with a linear schedule is provided."""
        if manager != "energies":
            raise ValueError("only the 'energies' output is provided")
        if schedule == "none":
            self.energies_interval = 0
        elif schedule == "linear":
            self.energies_interval = int(interval)
        else:
            raise ValueError("energies output supports the 'linear' and 'none' schedules")

    def ResetMomentum(self):
        self.itg.SetMomentumToZero()

    def WriteConf(self, filename):
        self.sample.WriteConf(filename)

    def GetNumberOfParticles(self):
        return self.sample.GetNumberOfParticles()

    def GetVolume(self):
        return self.sample.GetVolume()

    # -- the time-step loop (Simulation.py:538-622) ---------------------------
    def _check(self):
        if self.itg is None:
            raise ValueError("Integrator has not been set")
        if len(self.potentialList) == 0:
            raise ValueError("Potential has not been set")

    def Run(self, num_iter, initializeOutput=True, restartBlock=None, suppressAllOutput=False, force_timing=False):
        """Runs num_iter time steps on the device and returns the elapsed time."""
        self._check()
        if restartBlock is not None:
            raise ValueError("restart files are not provided; use ReadConf on a written configuration")
        record = (not suppressAllOutput) and self.energies_interval > 0
        if record:
            cap = num_iter // self.energies_interval + 1
            self.sample.SetEnergyLog(self.energies_interval, cap)
        else:
            self.sample.SetEnergyLog(0, 0)
        t0 = time.time()
        self.sample.Run(int(num_iter), int(self.momentum_reset_interval))
        self.elapsed = time.time() - t0
        if record:
            self._collect_energies(initializeOutput)
        if (not suppressAllOutput) or force_timing:
            n = self.sample.GetNumberOfParticles()
            mats = n * num_iter / 1e6 / self.elapsed if self.elapsed > 0 else 0.0
            self.timing.append((num_iter, self.elapsed, mats))
        return self.elapsed

    def RunStepwise(self, num_iter, callback=None):
        """The reference's per-step loop, one CalcF + Integrate call per step
        (Simulation.py:579-598); callback(i, sample) runs after each CalcF."""
        self._check()
        for i in range(num_iter):
            if self.momentum_reset_interval > 0 and i % self.momentum_reset_interval == 0:
                self.itg.SetMomentumToZero()
            self.sample.CalcF(self.itg.RequiresStress())
            if callback is not None:
                callback(i, self.sample)
            self.itg.Integrate()
        self.sample.CalcF()

    def _collect_energies(self, reset):
        log = self.sample.GetEnergyLog()
        n = self.sample.GetNumberOfParticles()
        dof = self.sample.GetNumberOfDOFs()
        V = self.sample.GetVolume()
        step, pe, W, ke, xi = (log[:, k] for k in range(5))
        T = 2.0 * ke / dof
        p = (n * T + W) / V  # EnergiesOutputManager.cu:191
        rows = np.stack([step, pe / n, ke / n, p, T, (pe + ke) / n, W / n, xi], axis=1)
        self.energies = rows if reset else np.concatenate([self.energies, rows])

    def GetEnergies(self):
        """Energies rows: step, then pe, ke, p, T, Etot, W per particle / Ps."""
        return self.energies

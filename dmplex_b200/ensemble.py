"""Batched ensembles: many members on meshes of several levels, persistent launches per phase.

There is no ensemble in the reference (it runs one model per process); each member here
follows rk4_step! (src/TimeSteppers/RungeKutta.jl:18-29) on its group's model bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .model import TRiSKShallowWater, _state


class Ensemble:
    """groups: a list of (model, members, dt, nsteps). Members of a group share the model's
    tables; every group has its own time step and number of RK4 steps. state_bits = 32
    stores the members' states and work vectors as float (the arithmetic stays FP64)."""

    def __init__(self, groups, state_bits: int = 64):
        self.groups = list(groups)
        self.state_bits = int(state_bits)
        n = len(self.groups)
        models = (C.c_void_p * n)(*[g[0].handle.value for g in self.groups])
        members = np.array([g[1] for g in self.groups], dtype=np.int32)
        dts = np.array([g[2] for g in self.groups], dtype=np.float64)
        steps = np.array([g[3] for g in self.groups], dtype=np.int64)
        handle = C.c_void_p()
        check(lib.trisk_ensemble_create_precision(models, members.ctypes.data, dts.ctypes.data, steps.ctypes.data,
                                                  n, self.state_bits, C.byref(handle)))
        self._h = handle
        self._models = [g[0] for g in self.groups]  # the ensemble uses their device tables

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_ensemble_destroy(self._h)
            self._h = None

    def set_member(self, group: int, member: int, y) -> None:
        m: TRiSKShallowWater = self._models[group]
        check(lib.trisk_ensemble_set_member(self._h, group, member, _state(y, m)))

    def get_member(self, group: int, member: int, y=None):
        m: TRiSKShallowWater = self._models[group]
        if y is None:
            y = np.zeros(m.state_size)
        check(lib.trisk_ensemble_get_member(self._h, group, member, _state(y, m)))
        return y

    def autotune(self, steps: int = 10) -> float:
        """Picks the fastest phase block sizes and members per slice for these groups (states
        are left as they were); returns ms per RK4 step."""
        best = C.c_double()
        check(lib.trisk_ensemble_autotune(self._h, int(steps), C.byref(best)))
        return best.value

    def block(self) -> list:
        b = np.zeros(3, dtype=np.int32)
        check(lib.trisk_ensemble_get_block(self._h, b.ctypes.data))
        return b.tolist()

    def set_block(self, block) -> None:
        b = np.ascontiguousarray(block, dtype=np.int32)
        if b.shape != (3,):
            raise ValueError("three block sizes")
        check(lib.trisk_ensemble_set_block(self._h, b.ctypes.data))

    def slices(self) -> list:
        """Members per slice of every group: a slice's members are stored together and its
        three phases run back to back, so its work vectors stay in L2."""
        b = np.zeros(len(self.groups), dtype=np.int32)
        check(lib.trisk_ensemble_get_slices(self._h, b.ctypes.data))
        return b.tolist()

    def set_slices(self, members_per_slice) -> None:
        """Re-slices every group (the members' states are kept)."""
        b = np.ascontiguousarray(members_per_slice, dtype=np.int32)
        if b.shape != (len(self.groups),):
            raise ValueError("one slice size per group")
        check(lib.trisk_ensemble_set_slices(self._h, b.ctypes.data))

    @property
    def members_per_thread(self) -> int:
        """2 (two members per thread where a slice's member count is even) or 4."""
        v = C.c_int32()
        check(lib.trisk_ensemble_get_members_per_thread(self._h, C.byref(v)))
        return v.value

    def set_members_per_thread(self, members: int) -> None:
        check(lib.trisk_ensemble_set_members_per_thread(self._h, int(members)))

    def run_async(self, steps: int) -> None:
        check(lib.trisk_ensemble_run_async(self._h, int(steps)))

    def synchronize(self) -> None:
        check(lib.trisk_ensemble_synchronize(self._h))

    def run(self, steps: int) -> None:
        self.run_async(steps)
        self.synchronize()

    def steps_taken(self) -> list:
        out = np.zeros(len(self.groups), dtype=np.int64)
        check(lib.trisk_ensemble_steps(self._h, out.ctypes.data))
        return out.tolist()

    def reset(self) -> None:
        check(lib.trisk_ensemble_reset(self._h))

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib.trisk_ensemble_stream(self._h, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        return int(lib.trisk_ensemble_launch_count(self._h))

    def step_bytes(self) -> float:
        b = C.c_double()
        check(lib.trisk_ensemble_bytes(self._h, C.byref(b)))
        return b.value

    def energy(self, group: int) -> np.ndarray:
        """total_energy of every member of the group."""
        out = np.zeros(self.groups[group][1])
        check(lib.trisk_ensemble_energy(self._h, group, out.ctypes.data))
        return out

    def set_closure(self, group: int, net, geometry: np.ndarray, norm: np.ndarray, every_stage: bool = False,
                    work_free: bool = False, fused: bool = True, every: int = 1):
        """Learned closure for a group (net: closure.ClosureMLP, or None to remove it).
        every_stage: run the network at every RK4 stage; work_free: remove from each member's
        momentum correction its component along the energy gradient (no work on the flow);
        fused: features, network and corrections in one kernel (False: three launches with the
        features and outputs in HBM; the same numbers); every: run the network on every
        `every`-th step and keep its corrections on the steps between."""
        if not 1 <= int(every) <= 255:
            raise ValueError("every must be in 1..255")
        if net is None:
            check(lib.trisk_ensemble_set_closure(self._h, group, None, None, None, 0))
            self._net = None
            return
        geometry = np.ascontiguousarray(geometry, dtype=np.float32)
        norm = np.ascontiguousarray(norm, dtype=np.float64)
        check(lib.trisk_ensemble_set_closure(self._h, group, net.handle, geometry.ctypes.data, norm.ctypes.data,
                                             int(bool(every_stage)) | (2 if work_free else 0) |
                                             (0 if fused else 4) | (int(every) << 8)))
        self._net = net  # the ensemble launches it

    def closure_mask(self, group: int, member_on) -> None:
        on = np.ascontiguousarray(member_on, dtype=np.float32)
        check(lib.trisk_ensemble_closure_mask(self._h, group, on.ctypes.data))

    def features(self, group: int, X, norm: np.ndarray, geometry: np.ndarray):
        """Closure features of the group's member states into the CUDA bfloat16 tensor X
        (rows e * M + m in file edge order, 24 columns)."""
        norm = np.ascontiguousarray(norm, dtype=np.float64)
        geometry = np.ascontiguousarray(geometry, dtype=np.float32)
        check(lib.trisk_ensemble_features(self._h, group, X.data_ptr(), norm.ctypes.data, geometry.ctypes.data))
        return X

    def closure_check(self) -> None:
        check(lib.trisk_ensemble_closure_check(self._h))

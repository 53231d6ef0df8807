"""Kraus channels and the noise model: lqcs::KrausChannel / lqcs::NoiseModel
(include/lqcs/backend/noise.hpp:11-44, src/backend/noise.cpp:19-80)."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N


def _check_probability(p: float, name: str) -> None:
    if p < 0.0 or p > 1.0:
        raise ValueError(f"{name}: probability must be in [0, 1]")


class KrausChannel:
    """One-qubit channel rho -> sum_i K_i rho K_i^dagger; completeness is checked on
    construction within 1e-10 (src/backend/noise.cpp:19-39)."""

    def __init__(self, ops):
        ops = [tuple(complex(v) for v in np.asarray(k, dtype=np.complex128).reshape(-1)) for k in ops]
        if not ops:
            raise ValueError("KrausChannel: needs at least one operator")
        s = np.zeros((2, 2), dtype=np.complex128)
        for k in ops:
            m = np.array(k, dtype=np.complex128).reshape(2, 2)
            s += np.conj(m.T) @ m
        if np.max(np.abs(s - np.eye(2))) > 1e-10:
            raise ValueError("KrausChannel: completeness violated (sum K_i^dag K_i != I)")
        self.ops = ops

    @staticmethod
    def depolarizing(p: float) -> "KrausChannel":
        _check_probability(p, "depolarizing")
        k0 = math.sqrt(1.0 - 3.0 * p / 4.0)
        kp = math.sqrt(p / 4.0)
        return KrausChannel([(k0, 0, 0, k0), (0, kp, kp, 0), (0, -kp * 1j, kp * 1j, 0),
                             (kp, 0, 0, -kp)])

    @staticmethod
    def amplitude_damping(gamma: float) -> "KrausChannel":
        _check_probability(gamma, "amplitude_damping")
        return KrausChannel([(1, 0, 0, math.sqrt(1.0 - gamma)), (0, math.sqrt(gamma), 0, 0)])

    @staticmethod
    def phase_damping(gamma: float) -> "KrausChannel":
        _check_probability(gamma, "phase_damping")
        return KrausChannel([(1, 0, 0, math.sqrt(1.0 - gamma)), (0, 0, 0, math.sqrt(gamma))])

    @staticmethod
    def bit_flip(p: float) -> "KrausChannel":
        _check_probability(p, "bit_flip")
        a, b = math.sqrt(1.0 - p), math.sqrt(p)
        return KrausChannel([(a, 0, 0, a), (0, b, b, 0)])

    @staticmethod
    def phase_flip(p: float) -> "KrausChannel":
        _check_probability(p, "phase_flip")
        a, b = math.sqrt(1.0 - p), math.sqrt(p)
        return KrausChannel([(a, 0, 0, a), (b, 0, 0, -b)])

    def as_array(self) -> np.ndarray:
        return np.array(self.ops, dtype=np.complex128).reshape(-1, 2, 2)


class NoiseModel:
    """Every channel is applied after every unitary instruction to each qubit it touches
    (src/backend/statevector_simulator.cpp:146-153)."""

    def __init__(self):
        self._channels: list[KrausChannel] = []

    def add_all_qubit_channel(self, channel: KrausChannel) -> "NoiseModel":
        self._channels.append(channel)
        return self

    def channels(self) -> list:
        return list(self._channels)

    def empty(self) -> bool:
        return not self._channels

    def c_channels(self):
        """(pointer to lqcs_kraus_channel array, count, keepalive)."""
        if not self._channels:
            return None, 0, []
        arr = (N.KrausChannelC * len(self._channels))()
        keep = [arr]
        for i, ch in enumerate(self._channels):
            buf = np.ascontiguousarray(ch.as_array().reshape(-1)).view(np.float64)
            keep.append(buf)
            arr[i].n_ops = len(ch.ops)
            arr[i].ops = buf.ctypes.data_as(C.POINTER(C.c_double))
        return C.cast(arr, C.POINTER(N.KrausChannelC)), len(self._channels), keep

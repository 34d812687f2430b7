"""Acquisition geometry: Source, Receiver, Survey.

Same API as geobrain/physics/wave/survey/{source,receiver,survey}.py:
integer grid-index positions, one wavelet of length nt per source, optional
per-shot receiver masks (stored; the acoustic propagator, like the
reference's, records every receiver for every shot).
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np


class Source:
    def __init__(self, nt: int, dt: float, f0: float) -> None:
        self.nt, self.dt, self.f0 = nt, dt, f0
        self.t = np.arange(nt) * dt
        self.loc_x: List[int] = []
        self.loc_z: List[int] = []
        self.loc_y: List[int] = []
        self.type: List[str] = []
        self.wavelet: List[np.ndarray] = []
        self.moment_tensor: List[np.ndarray] = []
        self.num = 0

    def __repr__(self) -> str:
        if self.num == 0:
            return "Source: empty"
        x, z = np.array(self.loc_x), np.array(self.loc_z)
        return (f"Source:\n  Number: {self.num}\n  Time: {self.nt} samples @ {self.dt * 1000:.2f} ms\n"
                f"  X range: {x.min()} - {x.max()} (grid)\n  Z range: {z.min()} - {z.max()} (grid)\n"
                f"  Types: {sorted(set(self.type))}")

    def _check(self, wavelet, moment_tensor):
        wavelet = np.asarray(wavelet)
        if wavelet.shape[0] != self.nt:
            raise ValueError(f"Wavelet length {wavelet.shape[0]} != nt {self.nt}")
        mt = np.eye(3) if moment_tensor is None else np.asarray(moment_tensor)
        if mt.shape != (3, 3):
            raise ValueError(f"Moment tensor must be 3x3, got {mt.shape}")
        return wavelet, mt

    def add_source(self, x: int, z: int, wavelet: np.ndarray, y: Optional[int] = None, source_type: str = "mt",
                   moment_tensor: Optional[np.ndarray] = None) -> None:
        wavelet, mt = self._check(wavelet, moment_tensor)
        self.loc_x.append(int(x))
        self.loc_z.append(int(z))
        if y is not None:
            self.loc_y.append(int(y))
        self.type.append(source_type)
        self.wavelet.append(wavelet.copy())
        self.moment_tensor.append(mt.copy())
        self.num += 1

    def add_sources(self, x: np.ndarray, z: np.ndarray, wavelet: np.ndarray, y: Optional[np.ndarray] = None,
                    source_type: str = "mt", moment_tensor: Optional[np.ndarray] = None) -> None:
        x, z = np.asarray(x), np.asarray(z)
        if x.shape != z.shape:
            raise ValueError(f"x and z must have same shape: {x.shape} != {z.shape}")
        if y is not None and np.asarray(y).shape != x.shape:
            raise ValueError(f"y must have same shape as x: {np.asarray(y).shape} != {x.shape}")
        wavelet, mt = self._check(wavelet, moment_tensor)
        xs, zs = x.ravel().tolist(), z.ravel().tolist()
        self.loc_x.extend(int(v) for v in xs)
        self.loc_z.extend(int(v) for v in zs)
        if y is not None:
            self.loc_y.extend(int(v) for v in np.asarray(y).ravel().tolist())
        for _ in xs:
            self.type.append(source_type)
            self.wavelet.append(wavelet.copy())
            self.moment_tensor.append(mt.copy())
        self.num += len(xs)

    def get_loc(self) -> np.ndarray:
        cols = [np.array(self.loc_x).reshape(-1, 1)]
        if self.loc_y:
            cols.append(np.array(self.loc_y).reshape(-1, 1))
        cols.append(np.array(self.loc_z).reshape(-1, 1))
        return np.hstack(cols)

    def get_wavelet(self) -> np.ndarray:
        return np.array(self.wavelet)

    def get_moment_tensor(self) -> np.ndarray:
        return np.array(self.moment_tensor)

    def get_type(self, unique: bool = False) -> np.ndarray:
        types = np.array(self.type)
        return np.unique(types) if unique else types


class Receiver:
    VALID = ("pr", "vx", "vy", "vz")

    def __init__(self, nt: int, dt: float) -> None:
        self.nt, self.dt = nt, dt
        self.loc_x: List[int] = []
        self.loc_z: List[int] = []
        self.loc_y: List[int] = []
        self.type: List[str] = []
        self.num = 0

    def __repr__(self) -> str:
        if self.num == 0:
            return "Receiver: empty"
        x, z = np.array(self.loc_x), np.array(self.loc_z)
        return (f"Receiver:\n  Number: {self.num}\n  Recording: {self.nt} samples @ {self.dt * 1000:.2f} ms\n"
                f"  X range: {x.min()} - {x.max()} (grid)\n  Z range: {z.min()} - {z.max()} (grid)\n"
                f"  Types: {sorted(set(self.type))}")

    def _kind(self, rcv_type: str) -> str:
        if rcv_type.lower() not in self.VALID:
            raise ValueError(f"Receiver type must be one of {self.VALID}, got '{rcv_type}'")
        return rcv_type.lower()

    def add_receiver(self, x: int, z: int, rcv_type: str, y: Optional[int] = None) -> None:
        kind = self._kind(rcv_type)
        self.loc_x.append(int(x))
        self.loc_z.append(int(z))
        if y is not None:
            self.loc_y.append(int(y))
        self.type.append(kind)
        self.num += 1

    def add_receivers(self, x: np.ndarray, z: np.ndarray, rcv_type: str, y: Optional[np.ndarray] = None) -> None:
        x, z = np.asarray(x), np.asarray(z)
        if x.shape != z.shape:
            raise ValueError(f"x and z must have same shape: {x.shape} != {z.shape}")
        if y is not None and np.asarray(y).shape != x.shape:
            raise ValueError(f"y must have same shape as x: {np.asarray(y).shape} != {x.shape}")
        kind = self._kind(rcv_type)
        xs, zs = x.ravel().tolist(), z.ravel().tolist()
        self.loc_x.extend(int(v) for v in xs)
        self.loc_z.extend(int(v) for v in zs)
        if y is not None:
            self.loc_y.extend(int(v) for v in np.asarray(y).ravel().tolist())
        self.type.extend([kind] * len(xs))
        self.num += len(xs)

    def get_loc(self) -> np.ndarray:
        cols = [np.array(self.loc_x).reshape(-1, 1)]
        if self.loc_y:
            cols.append(np.array(self.loc_y).reshape(-1, 1))
        cols.append(np.array(self.loc_z).reshape(-1, 1))
        return np.hstack(cols)

    def get_type(self, unique: bool = False) -> np.ndarray:
        types = np.array(self.type)
        return np.unique(types) if unique else types


class Survey:
    def __init__(self, source: Source, receiver: Receiver, receiver_masks: Optional[np.ndarray] = None) -> None:
        self.source = source
        self.receiver = receiver
        self.receiver_masks = None
        if receiver_masks is not None:
            self.set_receiver_masks(receiver_masks)

    def __repr__(self) -> str:
        return (f"Survey:\n  Shots: {self.n_shots}\n  Receivers: {self.n_receivers}\n"
                f"  Time: {self.nt} samples @ {self.dt * 1000:.2f} ms\n"
                f"  Receiver masks: {'Yes' if self.receiver_masks is not None else 'No'}")

    def set_receiver_masks(self, receiver_masks: np.ndarray) -> None:
        receiver_masks = np.asarray(receiver_masks)
        expected = (self.n_shots, self.n_receivers)
        if receiver_masks.shape != expected:
            raise ValueError(f"Receiver mask shape {receiver_masks.shape} doesn't match survey geometry {expected}")
        self.receiver_masks = receiver_masks.astype(bool)

    @property
    def n_shots(self) -> int:
        return self.source.num

    @property
    def n_receivers(self) -> int:
        return self.receiver.num

    @property
    def nt(self) -> int:
        return self.source.nt

    @property
    def dt(self) -> float:
        return self.source.dt

    @property
    def f0(self) -> float:
        return self.source.f0

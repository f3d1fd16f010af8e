"""Delay-model file reader and beamset parser (the DelayManager's host logic).

File format (python/skyweaver/skyweaver.py:32-90, DelayManager.cuh:40-51):
repeated records of a packed header {uint32 nbeams, uint32 nantennas,
double start_epoch, double end_epoch} followed by float32
[nbeams][nantennas][3] = (antenna weight, delay offset s, delay rate s/s).

Behaviour follows cpp/skyweaver/src/DelayManager.cu:
  * delays(epoch) scans forward to the model whose [start, end] contains the
    epoch; an epoch before the current model raises InvalidDelayEpoch,
    running off the end raises "Reached end of delay model file"
    (:56-67,101-130);
  * models are zero padded to (nbeams, nantennas) of the pipeline (:75-97);
  * beamsets are runs of contiguous beams with identical antenna weights,
    parsed from the first model (:162-232).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

HEADER = struct.Struct("<IIdd")


class InvalidDelayEpoch(RuntimeError):
    def __init__(self, epoch):
        super().__init__(f"No valid delay model for epoch {epoch}")
        self.epoch = epoch


@dataclass
class DelayModel:
    start_epoch: float
    end_epoch: float
    delays: np.ndarray  # float32 [nbeams][nantennas][3]


@dataclass
class Beamsets:
    nbeamsets: int
    weights: np.ndarray  # float32 [nbeamsets][nantennas] (padded)
    mapping: np.ndarray  # int32 [nbeams] (padded)


def pack_model(m: DelayModel) -> bytes:
    nb, na, _ = m.delays.shape
    return HEADER.pack(nb, na, m.start_epoch, m.end_epoch) + \
        np.ascontiguousarray(m.delays, np.float32).tobytes()


def read_delay_file(path: str):
    models = []
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        if off + HEADER.size > len(data):
            raise RuntimeError("Reached end of delay model file")
        nb, na, start, end = HEADER.unpack_from(data, off)
        off += HEADER.size
        n = nb * na * 3 * 4
        if off + n > len(data):
            raise RuntimeError("Reached end of delay model file")
        d = np.frombuffer(data, np.float32, nb * na * 3, off).reshape(nb, na, 3).copy()
        off += n
        models.append(DelayModel(start, end, d))
    return models


def parse_beamsets(delays: np.ndarray, nbeams: int, nantennas: int) -> Beamsets:
    """DelayManager::parse_beamsets (DelayManager.cu:162-232)."""
    nb, na, _ = delays.shape
    mapping = np.zeros(nbeams, np.int32)
    sets = [np.zeros(nantennas, np.float32)]
    sets[0][:na] = delays[0, :, 0]
    cur = 0
    for b in range(1, nb):
        w = delays[b, :, 0]
        if np.any(w != sets[cur][:na]):
            sets.append(np.zeros(nantennas, np.float32))
            cur += 1
            sets[cur][:na] = w
        mapping[b] = cur
    return Beamsets(len(sets), np.stack(sets), mapping)


class DelayManager:
    """Reference-compatible delay manager over a delay-model file."""

    def __init__(self, path: str, nbeams: int, nantennas: int):
        self._models = read_delay_file(path)
        if not self._models:
            raise RuntimeError("Reached end of delay model file")
        self._idx = 0
        self.nbeams, self.nantennas = nbeams, nantennas
        first = self._models[0]
        if first.delays.shape[0] > nbeams:
            raise RuntimeError("Delay model contains too many beams for current skyweaver build")
        self._shape = first.delays.shape
        self._beamsets = parse_beamsets(first.delays, nbeams, nantennas)

    def epoch(self) -> float:
        return self._models[self._idx].start_epoch

    def delays(self, epoch: float) -> np.ndarray:
        m = self._models[self._idx]
        if epoch < m.start_epoch:
            raise InvalidDelayEpoch(epoch)
        while not (m.start_epoch <= epoch <= m.end_epoch):
            self._idx += 1
            if self._idx >= len(self._models):
                raise RuntimeError("Reached end of delay model file")
            m = self._models[self._idx]
            if m.delays.shape != self._shape:
                raise RuntimeError("Variable delay model parameters are unsupported")
        nb, na, _ = m.delays.shape
        if na > self.nantennas:
            raise RuntimeError("Delay model contains too many antennas")
        out = np.zeros((self.nbeams, self.nantennas, 3), np.float32)
        out[:nb, :na] = m.delays
        return out

    def beamset_weights(self) -> np.ndarray:
        return self._beamsets.weights

    def beamset_mapping(self) -> np.ndarray:
        return self._beamsets.mapping

    def nbeamsets(self) -> int:
        return self._beamsets.nbeamsets

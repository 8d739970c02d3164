"""HyperLogLog sketch for cardinality / union estimation (drop-in for the
reference's ``src/hll.py``).

``HLL`` keeps its 2^p uint8 registers in device memory.  ``add`` and
``add_array`` queue values on the host and hash them on the GPU in one launch
when the registers are next read (``estimate``, ``registers``,
``union_estimate``); the result is identical to adding them one by one because
register updates are max operations.  Hash, index/rank rule and estimator
follow src/hll.py:13-54,81-120 bit for bit (the sum of 2^-r is formed exactly,
then the FP64 corrections).
"""
from __future__ import annotations

from typing import List

import numpy as np
import torch

from . import _lib, core

_MASK64 = 0xFFFFFFFFFFFFFFFF


def _hash64(x: int) -> int:
    """64-bit splitmix64 finaliser of one integer (src/hll.py:13-19), computed
    on the device."""
    v = int(x) & _MASK64
    if v >= 1 << 63:
        v -= 1 << 64
    return int(core.hash64([v]).cpu().view(torch.int64).item()) & _MASK64


def hash64_array(values) -> np.ndarray:
    """_hash64 over an int64 array (device), returned as uint64."""
    return core.hash64(np.asarray(values, dtype=np.int64)).cpu().numpy()


def _alpha(m: int) -> float:
    """Bias-correction constant (src/hll.py:26-34)."""
    if m == 16:
        return 0.673
    if m == 32:
        return 0.697
    if m == 64:
        return 0.709
    return 0.7213 / (1.0 + 1.079 / m)


def _p_of(m: int) -> int:
    p = int(m).bit_length() - 1
    if m <= 0 or (1 << p) != m or not 4 <= p <= 16:
        raise ValueError(f"register count must be 2^p with p in [4, 16], got {m}")
    return p


def _estimate_from_registers(registers, alpha: float = None) -> float:
    """HLL estimate of a register array (src/hll.py:37-54), on the device.
    ``alpha`` is accepted for signature parity; the library derives the same
    constant from the register count."""
    regs = _lib.as_device_tensor(registers, torch.uint8, "registers")
    p = _p_of(int(regs.numel()))
    return float(core.estimate_pairs(regs, p, [0]).item())


class HLL:
    """HyperLogLog sketch with 2^p registers (src/hll.py:61-105)."""

    def __init__(self, p: int = 8, device=None) -> None:
        if not (4 <= p <= 16):
            raise ValueError(f"p must be in [4, 16], got {p}")
        _lib.require_cuda()
        self.p = p
        self.m: int = 1 << p
        self._alpha = _alpha(self.m)
        self._remaining_bits: int = 64 - p
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._regs = torch.zeros(self.m, dtype=torch.uint8, device=dev)
        self._pending: List[np.ndarray] = []
        self._pending_scalars: List[int] = []

    @classmethod
    def _from_row(cls, row: torch.Tensor, p: int) -> "HLL":
        """Wrap an existing device register row (a view; no copy)."""
        obj = cls.__new__(cls)
        obj.p = p
        obj.m = 1 << p
        obj._alpha = _alpha(obj.m)
        obj._remaining_bits = 64 - p
        obj._regs = row
        obj._pending = []
        obj._pending_scalars = []
        return obj

    # ------------------------------------------------------------------
    def add(self, x: int) -> None:
        """Add a single integer element."""
        v = int(x) & _MASK64
        self._pending_scalars.append(v - (1 << 64) if v >= 1 << 63 else v)
        if len(self._pending_scalars) >= 1 << 16:
            self._flush()

    def add_array(self, arr) -> None:
        """Add all integer elements of an array."""
        a = arr
        if isinstance(a, torch.Tensor):
            if a.numel():
                core.hll_add_tensor(self._regs, self.p, a.reshape(-1))
            return
        a = np.asarray(a)
        if a.size:
            self._pending.append(a.astype(np.int64, copy=False).reshape(-1))

    def _flush(self) -> None:
        parts = self._pending
        if self._pending_scalars:
            parts = parts + [np.asarray(self._pending_scalars, dtype=np.int64)]
        self._pending = []
        self._pending_scalars = []
        if parts:
            core.hll_add_tensor(self._regs, self.p, np.concatenate(parts))

    @property
    def registers(self) -> np.ndarray:
        """Host copy of the registers (uint8[2^p])."""
        self._flush()
        return self._regs.cpu().numpy()

    @registers.setter
    def registers(self, value) -> None:
        a = np.asarray(value, dtype=np.uint8).reshape(-1)
        if a.size != self.m:
            raise ValueError(f"expected {self.m} registers, got {a.size}")
        self._pending = []
        self._pending_scalars = []
        self._regs.copy_(torch.from_numpy(a.copy()))

    @property
    def registers_device(self) -> torch.Tensor:
        """The device register row (flushes pending adds)."""
        self._flush()
        return self._regs

    # ------------------------------------------------------------------
    def estimate(self) -> float:
        """Estimate the cardinality of the set."""
        self._flush()
        return float(core.estimate_pairs(self._regs, self.p, [0]).item())

    def memory_bytes(self) -> int:
        """Raw register storage: 1 byte per register."""
        return self.m


def union_estimate(hll1: HLL, hll2: HLL) -> float:
    """Estimate |A cup B| from the register-wise max of two sketches
    (src/hll.py:112-120)."""
    if hll1.p != hll2.p:
        raise ValueError("Both HLLs must have the same precision p")
    a = hll1.registers_device
    b = hll2.registers_device
    if b.device != a.device:
        b = b.to(a.device)
    rows = torch.stack([a, b]).reshape(-1)
    return float(core.estimate_pairs(rows, hll1.p, [0], [1]).item())

"""Energies and updates (mirror of src/energy.rs) over the packing of libgeq."""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Sequence

import numpy as np

from ._lib import GeqError, check, geq_energy_conf, lib

_u32 = C.POINTER(C.c_uint32)
_i32 = C.POINTER(C.c_int32)


def _p(a, t):
    return a.ctypes.data_as(t)


class EnergyConf:
    """EnergyConf (energy.rs:36-78)."""

    __slots__ = ("elements", "max")

    def __init__(self, elements: int, max: int):  # noqa: A002 - crate field name
        self.elements = int(elements)
        self.max = int(max)

    def _c(self):
        return geq_energy_conf(self.elements, self.max)

    def energy_size(self) -> int:
        return lib.geq_conf_energy_size(self._c())

    def energy_bits(self) -> int:
        return lib.geq_conf_energy_bits(self._c())

    def energy_mask(self) -> int:
        return lib.geq_conf_energy_mask(self._c())

    def update_size(self) -> int:
        return lib.geq_conf_update_size(self._c())

    def update_bits(self) -> int:
        return lib.geq_conf_update_bits(self._c())

    def update_mask(self) -> int:
        return lib.geq_conf_update_mask(self._c())

    def supported(self) -> bool:
        """A thermometer codec exists for this conf (the batched round
        kernels, device-resident games, the allocation-free entry point)."""
        return bool(lib.geq_conf_supported(self._c()))

    def solvable(self) -> bool:
        """EnergyGame.run, run_batch and the serving loop solve games of this
        conf (the multi-word solver takes the confs without a codec)."""
        return bool(lib.geq_conf_solvable(self._c()))

    def __eq__(self, o):
        return isinstance(o, EnergyConf) and (self.elements, self.max) == (o.elements, o.max)

    def __hash__(self):
        return hash((self.elements, self.max))

    def __repr__(self):
        return f"EnergyConf(elements={self.elements}, max={self.max})"


EnergyConf.STANDARD = EnergyConf(6, 3)
EnergyConf.SILENT_STEP = EnergyConf(8, 2)
EnergyConf.ONE_DIMENSION = EnergyConf(1, 0xFFFFFFFF)


def pack_energy(values: Sequence[int], conf: EnergyConf) -> np.ndarray | None:
    v = np.ascontiguousarray(values, dtype=np.uint32)
    out = np.zeros(conf.energy_size(), dtype=np.uint32)
    st = lib.geq_energy_pack(conf._c(), _p(v, _u32) if v.size else None, len(v), _p(out, _u32))
    return out if st == 0 else None


def unpack_energy(words, conf: EnergyConf) -> list[int]:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.zeros(conf.elements, dtype=np.uint32)
    lib.geq_energy_unpack(conf._c(), _p(w, _u32), _p(out, _u32))
    return [int(x) for x in out]


class Energy:
    """One energy tuple (energy.rs:81-141)."""

    __slots__ = ("data", "conf")

    def __init__(self, data, conf: EnergyConf):
        self.data = np.ascontiguousarray(data, dtype=np.uint32)
        self.conf = conf

    @classmethod
    def new(cls, values: Sequence[int], conf: EnergyConf) -> "Energy | None":
        w = pack_energy(values, conf)
        return None if w is None else cls(w, conf)

    @classmethod
    def zero(cls, conf: EnergyConf) -> "Energy":
        return cls(np.zeros(conf.energy_size(), dtype=np.uint32), conf)

    def raw_data(self) -> np.ndarray:
        return self.data

    def to_vec(self) -> list[int]:
        return unpack_energy(self.data, self.conf)

    def partial_cmp(self, other: "Energy"):
        """-1 / 0 / 1 or None for incomparable (PartialOrd, energy.rs:121-141)."""
        assert self.conf.elements == other.conf.elements, "Incompatible Energy configurations"
        less = greater = True
        for a, b in zip(self.to_vec(), other.to_vec()):
            if a < b:
                greater = False
            elif a > b:
                less = False
        if less and greater:
            return 0
        if less:
            return -1
        if greater:
            return 1
        return None

    def __le__(self, o):
        c = self.partial_cmp(o)
        return c is not None and c <= 0

    def __lt__(self, o):
        return self.partial_cmp(o) == -1

    def __eq__(self, o):
        return isinstance(o, Energy) and self.conf == o.conf and np.array_equal(self.data, o.data)

    def __hash__(self):
        return hash((self.conf, self.data.tobytes()))

    def __repr__(self):
        return "Energy(" + " ".join("∞" if v == self.conf.max else str(v) for v in self.to_vec()) + ")"


class EnergyArray:
    """A list of energies of one position (energy.rs:227-369).

    ``array`` is an (n, energy_size) uint32 array in the crate's packed layout.
    Equality follows the crate: same number of rows and every row of the
    right-hand side occurs among the rows of the left-hand side.
    """

    __slots__ = ("array", "conf")

    def __init__(self, array, conf: EnergyConf):
        a = np.ascontiguousarray(array, dtype=np.uint32)
        if a.ndim == 1:
            a = a.reshape(-1, conf.energy_size())
        assert a.shape[1] == conf.energy_size()
        self.array = a
        self.conf = conf

    @classmethod
    def empty(cls, conf: EnergyConf) -> "EnergyArray":
        return cls.zero(0, conf)

    @classmethod
    def zero(cls, n: int, conf: EnergyConf) -> "EnergyArray":
        return cls(np.zeros((n, conf.energy_size()), dtype=np.uint32), conf)

    @classmethod
    def from_conf(cls, rows: Iterable[Sequence[int]], conf: EnergyConf) -> "EnergyArray":
        """FromEnergyConf<&[Vec<u32>]> (energy.rs:431-441)."""
        rows = list(rows)
        a = np.zeros((len(rows), conf.energy_size()), dtype=np.uint32)
        for i, r in enumerate(rows):
            w = pack_energy(r, conf)
            if w is None:
                raise ValueError(f"energy {r} does not fit {conf}")
            a[i] = w
        return cls(a, conf)

    def n_energies(self) -> int:
        return self.array.shape[0]

    def is_empty(self) -> bool:
        return self.array.shape[0] == 0

    def get(self, i: int) -> Energy | None:
        return Energy(self.array[i], self.conf) if 0 <= i < self.n_energies() else None

    def iter(self):
        for r in self.array:
            yield Energy(r, self.conf)

    __iter__ = iter

    def __len__(self):
        return self.n_energies()

    def data(self) -> bytes:
        return self.array.tobytes()

    def to_lists(self) -> list[list[int]]:
        return [e.to_vec() for e in self.iter()]

    def test_equivalence(self, equivalence: Energy) -> bool:
        """EnergyArray::test_equivalence (energy.rs:307-318)."""
        assert self.conf == equivalence.conf, "Incompatible Energy configurations"
        a = self.array if self.array.size else np.zeros((1, self.conf.energy_size()), dtype=np.uint32)
        return bool(lib.geq_test_equivalence(self.conf._c(), _p(a, _u32), self.n_energies(),
                                             _p(equivalence.data, _u32)))

    def __eq__(self, other):
        if isinstance(other, EnergyArray):
            if self.conf != other.conf:
                return False
            other = other.array
        other = np.asarray(other)
        if other.ndim != 2 or other.shape != self.array.shape:
            return False
        rows = {r.tobytes() for r in self.array}
        return all(np.ascontiguousarray(r, dtype=np.uint32).tobytes() in rows for r in other)

    def canonical(self) -> list[tuple[int, ...]]:
        """Sorted rows: the canonical form used for set comparisons."""
        return sorted(tuple(int(x) for x in r) for r in self.array)

    def __repr__(self):
        return "[" + ", ".join(repr(e) for e in self.iter()) + "]"


# ---- updates ---------------------------------------------------------------
class Upd:
    """Upd (energy.rs:446-500) in its i32 form: 0 Zero, -1 Decrement, k Min(k)."""

    Zero = 0
    Decrement = -1

    @staticmethod
    def Min(k: int) -> int:  # noqa: N802 - crate name
        if k < 1:
            raise ValueError("Min is 1-indexed")
        return int(k)


def update(*values: int) -> list[int]:
    """The crate's ``update!`` macro (energy.rs:615-620)."""
    return [int(v) for v in values]


def pack_update(values: Sequence[int], conf: EnergyConf) -> np.ndarray | None:
    v = np.ascontiguousarray(values, dtype=np.int32)
    out = np.zeros(conf.update_size(), dtype=np.uint32)
    st = lib.geq_update_pack(conf._c(), _p(v, _i32) if v.size else None, len(v), _p(out, _u32))
    return out if st == 0 else None


class Update:
    """Update (energy.rs:503-541)."""

    __slots__ = ("data", "conf")

    def __init__(self, data, conf: EnergyConf):
        self.data = np.ascontiguousarray(data, dtype=np.uint32)
        self.conf = conf

    @classmethod
    def new(cls, values: Sequence[int], conf: EnergyConf) -> "Update | None":
        w = pack_update(values, conf)
        return None if w is None else cls(w, conf)

    @classmethod
    def zero(cls, conf: EnergyConf) -> "Update":
        return cls(np.zeros(conf.update_size(), dtype=np.uint32), conf)

    def raw_data(self):
        return self.data

    def to_vec(self) -> list[int]:
        out = np.zeros(self.conf.elements, dtype=np.int32)
        lib.geq_update_unpack(self.conf._c(), _p(self.data, _u32), _p(out, _i32))
        return [int(x) for x in out]

    def __eq__(self, o):
        return isinstance(o, Update) and self.conf == o.conf and np.array_equal(self.data, o.data)


class UpdateArray:
    """UpdateArray (energy.rs:623-802): (n, update_size) packed words."""

    __slots__ = ("array", "conf")

    def __init__(self, array, conf: EnergyConf):
        a = np.ascontiguousarray(array, dtype=np.uint32)
        if a.ndim == 1:
            a = a.reshape(-1, conf.update_size())
        self.array = a
        self.conf = conf

    @classmethod
    def from_conf(cls, rows, conf: EnergyConf) -> "UpdateArray":
        rows = list(rows)
        a = np.zeros((len(rows), conf.update_size()), dtype=np.uint32)
        for i, r in enumerate(rows):
            if isinstance(r, Update):
                a[i] = r.data
                continue
            w = pack_update(r, conf)
            if w is None:
                raise ValueError(f"update {r} does not fit {conf}")
            a[i] = w
        return cls(a, conf)

    def n_updates(self) -> int:
        return self.array.shape[0]

    def get(self, i):
        return Update(self.array[i], self.conf) if 0 <= i < self.n_updates() else None

    def set(self, i, upd: Update):
        if upd.conf != self.conf or not (0 <= i < self.n_updates()):
            return None
        self.array[i] = upd.data
        return True

    def __eq__(self, o):
        return isinstance(o, UpdateArray) and self.conf == o.conf and np.array_equal(self.array, o.array)


class std_equivalences:  # noqa: N801 - crate module name
    """Energy tuples of the standard equivalences (energy.rs:198-225)."""

    _T = {
        "enabledness": [1, 1],
        "traces": [3, 1],
        "failures": [3, 2, 0, 0, 1, 1],
        "failure_traces": [3, 3, 3, 0, 1, 1],
        "readiness": [3, 2, 1, 1, 1, 1],
        "readiness_traces": [3, 3, 3, 1, 1, 1],
        "revivals": [3, 2, 1, 0, 1, 1],
        "impossible_futures": [3, 2, 0, 0, 3, 1],
        "possible_futures": [3, 2, 3, 3, 3, 1],
        "simulation": [3, 3, 3, 3, 0, 0],
        "ready_simulation": [3, 3, 3, 3, 1, 1],
        "nested_2simulation": [3, 3, 3, 3, 3, 1],
        "bisimulation": [3, 3, 3, 3, 3, 3],
    }

    @classmethod
    def get(cls, name: str) -> Energy:
        return Energy.new(cls._T[name], EnergyConf.STANDARD)

    @classmethod
    def names(cls):
        return list(cls._T)


for _name in std_equivalences._T:
    setattr(std_equivalences, _name, classmethod(lambda cls, _n=_name: cls.get(_n)))

__all__ = ["EnergyConf", "Energy", "EnergyArray", "Upd", "Update", "UpdateArray", "update",
           "std_equivalences", "pack_energy", "unpack_energy", "pack_update", "GeqError", "check"]

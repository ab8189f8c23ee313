"""params.txt surface of the reference driver (testDensitySubGrid_omp.cpp:948-1013).

The reference reads a YAML subset (YAMLDictionary.hpp) with SI conversion of
``value unit`` strings (UnitConverter.hpp).  The keys the plain method reads
are parsed here; the task-runtime capacity keys are accepted and kept (the GPU
path has no use for them).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

# UnitConverter.hpp:97-110 (length units); dimensionless otherwise
_LENGTH_UNITS = {
    "m": 1.0, "cm": 0.01, "pc": 3.086e16, "kpc": 3.086e19, "angstrom": 1.0e-10, "km": 1000.0,
}

REQUIRED_KEYS = [
    "box:anchor", "box:sides", "reemission_probability", "ncell", "num_subgrid", "num_photon",
    "number_of_iterations", "number_of_sources", "random_density",
]
CAPACITY_KEYS = [
    "queue_size_per_thread", "memoryspace_size", "number_of_tasks", "MPI_buffer_size",
    "cost_copy_factor", "edge_copy_factor", "general_queue_size",
]


class ParameterError(ValueError):
    pass


def parse_yaml_subset(text: str) -> dict:
    """Flatten `key: value` lines with indentation nesting into 'a:b' keys."""
    out: dict[str, str] = {}
    stack: list[tuple[int, str]] = []
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].rstrip()
        if not line.strip():
            continue
        indent = len(line) - len(line.lstrip(" "))
        m = re.match(r"\s*([^:]+):\s*(.*)$", line)
        if not m:
            raise ParameterError(f"cannot parse line: {raw!r}")
        key, value = m.group(1).strip(), m.group(2).strip()
        while stack and stack[-1][0] >= indent:
            stack.pop()
        full = ":".join([k for _, k in stack] + [key])
        if value == "":
            stack.append((indent, key))
        else:
            out[full] = value
    return out


def _physical(value: str) -> float:
    parts = value.split()
    v = float(parts[0])
    if len(parts) > 1:
        unit = parts[1]
        if unit not in _LENGTH_UNITS:
            raise ParameterError(f"unknown unit {unit!r}")
        v *= _LENGTH_UNITS[unit]
    return v


def _vector(value: str, conv=_physical):
    m = re.match(r"\[(.*)\]$", value.strip())
    if not m:
        raise ParameterError(f"expected a vector, got {value!r}")
    items = [s.strip() for s in m.group(1).split(",")]
    if len(items) != 3:
        raise ParameterError(f"expected 3 components, got {value!r}")
    return tuple(conv(s) for s in items)


def _bool(value: str) -> bool:
    v = value.strip().lower()
    if v in ("true", "yes", "1"):
        return True
    if v in ("false", "no", "0"):
        return False
    raise ParameterError(f"not a boolean: {value!r}")


def _uint(value: str) -> int:
    v = float(value)
    if v < 0 or v != int(v):
        raise ParameterError(f"not an unsigned integer: {value!r}")
    return int(v)


@dataclass
class Parameters:
    box: tuple                      # anchor xyz, sides xyz (m)
    reemission_probability: float
    ncell: tuple
    num_subgrid: tuple
    num_photon: int
    number_of_iterations: int
    number_of_sources: int
    random_density: bool
    capacity: dict = field(default_factory=dict)

    @classmethod
    def from_text(cls, text: str) -> "Parameters":
        d = parse_yaml_subset(text)
        missing = [k for k in REQUIRED_KEYS if k not in d]
        if missing:
            raise ParameterError(f"missing parameter(s): {', '.join(missing)}")
        anchor = _vector(d["box:anchor"])
        sides = _vector(d["box:sides"])
        ncell = _vector(d["ncell"], lambda s: int(float(s)))
        nsub = _vector(d["num_subgrid"], lambda s: int(float(s)))
        for n, s in zip(ncell, nsub):
            if s <= 0 or n % s:
                raise ParameterError("ncell must be a multiple of num_subgrid")
        cap = {}
        for k in CAPACITY_KEYS:
            if k in d:
                cap[k] = float(d[k])
        return cls(box=tuple(anchor) + tuple(sides),
                   reemission_probability=float(d["reemission_probability"]),
                   ncell=ncell, num_subgrid=nsub, num_photon=_uint(d["num_photon"]),
                   number_of_iterations=_uint(d["number_of_iterations"]),
                   number_of_sources=_uint(d["number_of_sources"]),
                   random_density=_bool(d["random_density"]), capacity=cap)

    @classmethod
    def from_file(cls, path: str) -> "Parameters":
        with open(path) as f:
            return cls.from_text(f.read())

    def to_text(self) -> str:
        pc = _LENGTH_UNITS["pc"]
        a = ", ".join(f"{v / pc!r} pc" for v in self.box[:3])
        s = ", ".join(f"{v / pc!r} pc" for v in self.box[3:])
        lines = [
            "box:", f"  anchor: [{a}]", f"  sides: [{s}]",
            f"ncell: [{', '.join(str(int(v)) for v in self.ncell)}]",
            f"num_photon: {int(self.num_photon)}",
            f"number_of_iterations: {int(self.number_of_iterations)}",
            f"reemission_probability: {self.reemission_probability!r}",
            f"number_of_sources: {int(self.number_of_sources)}",
            f"random_density: {'true' if self.random_density else 'false'}",
            f"num_subgrid: [{', '.join(str(int(v)) for v in self.num_subgrid)}]",
        ]
        defaults = {"queue_size_per_thread": 100, "memoryspace_size": 50000,
                    "number_of_tasks": 500000, "MPI_buffer_size": 1000, "cost_copy_factor": 10,
                    "edge_copy_factor": 0.01, "general_queue_size": 100000}
        defaults.update(self.capacity)
        for k in CAPACITY_KEYS:
            lines.append(f"{k}: {defaults[k]:g}")
        return "\n".join(lines) + "\n"

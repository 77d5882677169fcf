"""Parameterisation tables (Kirkland / Peng / Lobato).

File format and validation follow Utils::readParams (src/simulation/utilities/stringutils.cpp:149-184)
and Parameterisation (src/simulation/structure/structureparameters.h:22-78): line 1 the name, line 2 the
form ("kirkland" | "peng" | "lobato"), line 3 the number of terms per atom, then whitespace-separated
values, one atom (Z = 1, 2, ...) after another.
"""
from dataclasses import dataclass
import json
import os

import numpy as np

from . import abi

_FORMS = {"kirkland": abi.KIRKLAND, "peng": abi.PENG, "lobato": abi.LOBATO}
_PER_I = {abi.KIRKLAND: 4, abi.PENG: 2, abi.LOBATO: 2}


@dataclass
class Parameterisation:
    name: str
    form: int
    i_per_atom: int
    values: np.ndarray  # float64, flat

    @property
    def max_atomic_number(self) -> int:
        return len(self.values) // (self.i_per_atom * _PER_I[self.form])


def _make(name, form_name, per, values, source):
    if form_name not in _FORMS:
        raise RuntimeError(f"Unknown parameterisation form {form_name} in file {source}")
    form = _FORMS[form_name]
    values = np.asarray(values, dtype=np.float64)
    per_atom = per * _PER_I[form]
    if values.size % per_atom != 0:
        raise RuntimeError(f"Parameterisation {name} does not contain correct parameters per atom")
    return Parameterisation(name, form, per, values)


def read_params(path: str) -> Parameterisation:
    """Read a clTEM params/*.dat file."""
    if not os.path.exists(path):
        raise RuntimeError("Error opening resource file: " + path)
    with open(path, "r") as f:
        name = f.readline().rstrip("\r\n")
        form = f.readline().rstrip("\r\n")
        per = int(f.readline().strip())
        vals = [float(t) for t in f.read().split()]
    return _make(name, form, per, vals, path)


def read_params_json(path: str) -> dict:
    """Read a JSON bundle {name: {"form": ..., "i_per_atom": ..., "values": [...]}}."""
    with open(path) as f:
        d = json.load(f)
    return {k: _make(k, v["form"], int(v["i_per_atom"]), v["values"], path) for k, v in d.items()}


def default_bundle_path() -> str:
    """The parameter tables shipped with the tests (tests/golden/params.json)."""
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(os.path.dirname(here), "tests", "golden", "params.json")


def load_default(name: str) -> Parameterisation:
    return read_params_json(default_bundle_path())[name]

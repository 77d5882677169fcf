"""Parameterisation tables (Kirkland / Peng / Lobato).

File format and validation follow Utils::readParams (src/simulation/utilities/stringutils.cpp:149-184)
and Parameterisation (src/simulation/structure/structureparameters.h:22-78): line 1 the name, line 2 the
form ("kirkland" | "peng" | "lobato"), line 3 the number of terms per atom, then whitespace-separated
values, one atom (Z = 1, 2, ...) after another.
"""
from dataclasses import dataclass
import json
import os
import re

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


# ---------------------------------------------------------------------------------------------------
# CCD tables (detective quantum efficiency and noise transfer function)
# ---------------------------------------------------------------------------------------------------
CCD_TABLE_SIZE = 725   # Utils::ccdToDqeNtf accepts exactly 725 values per table (stringutils.cpp:218,229)

_NUMBER = re.compile(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?")


def _stream_doubles(line: str):
    """The values `std::stringstream >> double` reads from a line, including runs such as "0.70.6" that it
    reads as two numbers (the reference's .dat files contain them)."""
    out = []
    for tok in line.split():
        pos = 0
        while pos < len(tok):
            m = _NUMBER.match(tok, pos)
            if not m:
                break
            out.append(float(m.group(0)))
            pos = m.end()
        else:
            continue
        break   # extraction stops at the first character that does not start a number
    return out


@dataclass
class CCD:
    name: str
    dqe: np.ndarray   # float64[725], radial, per binned pixel
    ntf: np.ndarray   # float64[725]


def read_ccd(path: str) -> CCD:
    """Read a clTEM ccds/*.dat file (Utils::ccdToDqeNtf, src/simulation/utilities/stringutils.cpp:186-236):
    line 1 the name, then a "DQE" line followed by one line of values and an "NTF" line followed by one line
    of values; each table must hold exactly 725 values."""
    if not os.path.exists(path):
        raise RuntimeError("Error opening resource file: " + path)
    with open(path) as f:
        lines = f.read().split("\n")
    name = lines[0].rstrip("\r")
    dqe = ntf = None
    i = 1
    while i < len(lines):
        head = "".join(lines[i].split())
        if head in ("DQE", "NTF") and i + 1 < len(lines):
            vals = _stream_doubles(lines[i + 1])
            if len(vals) == CCD_TABLE_SIZE:
                if head == "DQE":
                    dqe = np.asarray(vals)
                else:
                    ntf = np.asarray(vals)
            i += 2
            continue
        i += 1
    if dqe is None or ntf is None:
        raise RuntimeError("Could not find DQE and NTF in file: " + os.path.basename(path))
    return CCD(name, dqe, ntf)


def default_ccd_bundle_path() -> str:
    """The CCD tables shipped with the tests (tests/golden/ccds.json)."""
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(os.path.dirname(here), "tests", "golden", "ccds.json")


def load_ccds(path: str = None) -> dict:
    """{file stem: CCD} from a JSON bundle {stem: {"name", "dqe", "ntf"}} (default: the shipped one)."""
    with open(path or default_ccd_bundle_path()) as f:
        d = json.load(f)
    return {k: CCD(v["name"], np.asarray(v["dqe"], dtype=np.float64), np.asarray(v["ntf"], dtype=np.float64))
            for k, v in d.items()}
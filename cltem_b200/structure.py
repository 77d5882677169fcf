"""Structures: .xyz reading, structure limits, seeded synthetic supercells and frozen-phonon configs.

- read_xyz follows CrystalStructure::openXyz (src/simulation/structure/crystalstructure.cpp:44-188):
  line 1 atom count, line 2 column headers (A x y z [occ] [u] [u1 u2 u3], optional "nm" scale flag),
  coordinates parsed with std::stof (single precision) and widened to double.
- limits follow CrystalStructure::updateLimits/resetLimits (crystalstructure.cpp:238-267), including
  the reference's initial max of DBL_MIN (so an all-negative structure keeps max = DBL_MIN).
- Frozen-phonon displacements follow PhononScattering::generateTdsFactor
  (src/simulation/incoherence/inelastic/phonon.cpp:98-128): sqrt(u^2) * N(0,1) per axis along the
  u1/u2/u3 axes (identity for .xyz input, simulationgeneral.cpp:177-205). The reference seeds its RNG
  from the wall clock; here every configuration has an explicit seed.
"""
from dataclasses import dataclass, field
import math

import numpy as np

ELEMENTS = [
    "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca",
    "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",
    "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I", "Xe", "Cs", "Ba", "La", "Ce",
    "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W", "Re", "Os", "Ir",
    "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U", "Np", "Pu", "Am", "Cm",
    "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr",
]


def symbol_to_z(sym: str) -> int:
    s = sym.strip()
    if s.isdigit():
        return int(s)
    s = s[:1].upper() + s[1:].lower()
    if s not in ELEMENTS:
        raise RuntimeError("Unknown element symbol: " + sym)
    return ELEMENTS.index(s) + 1


@dataclass
class Structure:
    Z: np.ndarray          # int32[n]
    x: np.ndarray          # float64[n], Å
    y: np.ndarray
    z: np.ndarray
    u2: np.ndarray = None  # optional per-atom mean-square displacement (Å^2) per axis, float64[n,3]
    name: str = ""
    extra: dict = field(default_factory=dict)
    defined_u: np.ndarray = None  # bool[n]: u2 row given by the file (None: every row when u2 is set)
    axes: np.ndarray = None       # float64[3,3]: rows u1, u2, u3, the displacement axes (None: x, y, z)

    def __len__(self):
        return int(self.Z.shape[0])

    def limits(self):
        """[min_x, max_x, min_y, max_y, min_z, max_z] as CrystalStructure leaves them."""
        tiny = np.finfo(np.float64).tiny  # std::numeric_limits<double>::min()
        big = np.finfo(np.float64).max
        if len(self) == 0:
            return [big, tiny, big, tiny, big, tiny]
        return [min(big, float(self.x.min())), max(tiny, float(self.x.max())),
                min(big, float(self.y.min())), max(tiny, float(self.y.max())),
                min(big, float(self.z.min())), max(tiny, float(self.z.max()))]


def _stof(s: str) -> float:
    return float(np.float32(float(s)))


def read_xyz(path: str, seed: int = 0, occupancy_draw: str = "normal") -> Structure:
    """Read a clTEM .xyz file (CrystalStructure::openXyz, src/simulation/structure/crystalstructure.cpp:44-173):
    atom count, a header line of column names (A x y z [occ] [u] [u1 u2 u3], optional "nm" for nanometre units,
    or no names for the A x y z default), then one atom per line, coordinates parsed as std::stof does.
    With an occ column, consecutive atoms at the same position form one site resolved by one draw from a
    generator seeded by `seed` (process_occupancy; the reference's generator is clock-seeded)."""
    with open(path, "r") as f:
        lines = f.read().splitlines()
    try:
        n = int(lines[0].strip())
    except Exception as e:  # noqa: BLE001
        raise RuntimeError(f"Could not parse number of atoms (line 1, {e}).")
    headers = lines[1].split() if len(lines) > 1 else []
    scale = 1.0
    if "nm" in headers:
        scale = 10.0
        headers = [h for h in headers if h != "nm"]

    def idx(h):
        return headers.index(h) if h in headers else -1

    hA, hx, hy, hz = idx("A"), idx("x"), idx("y"), idx("z")
    hocc, hu, hu1, hu2, hu3 = idx("occ"), idx("u"), idx("u1"), idx("u2"), idx("u3")
    default = hA == -1 and hx == -1 and hy == -1 and hz == -1
    if default:
        hA, hx, hy, hz = 0, 1, 2, 3
    if -1 in (hA, hx, hy, hz):
        raise RuntimeError(".xyz file headers not complete (requires A, x, y, z)")
    if default:
        hocc, hu, hu1, hu2, hu3 = [h + 4 * (h != -1) for h in (hocc, hu, hu1, hu2, hu3)]
    max_header = max(hA, hx, hy, hz, hocc, hu, hu1, hu2, hu3)
    Z, X, Y, Zc, U, OCC = [], [], [], [], [], []
    defined_u = hu != -1 or hu1 != -1 or hu2 != -1 or hu3 != -1
    i = 0
    for line in lines[2:]:
        if not line:
            break
        if i > n:
            raise RuntimeError(f"Number of atoms does not match .xyz first line ({n})")
        v = line.split()
        if len(v) < max_header:
            raise RuntimeError(f".xyz file columns are fewer than header entries. line: {2 + i}")
        Z.append(symbol_to_z(v[hA]))
        X.append(_stof(v[hx]) * scale)
        Y.append(_stof(v[hy]) * scale)
        Zc.append(_stof(v[hz]) * scale)
        if hocc != -1:
            OCC.append(_stof(v[hocc]))
        if defined_u:
            u = [0.0, 0.0, 0.0]
            if hu != -1:
                u = [_stof(v[hu])] * 3
            if hu1 != -1:
                u[0] = _stof(v[hu1])
            if hu2 != -1:
                u[1] = _stof(v[hu2])
            if hu3 != -1:
                u[2] = _stof(v[hz])  # the reference reads the z column here (crystalstructure.cpp:176-177)
            U.append([q * scale * scale for q in u])
        i += 1
    if i != n:
        raise RuntimeError(f"Number of atoms does not match .xyz first line: {i} instead of {n}")
    keep = np.arange(len(Z))
    if hocc != -1:
        keep = process_occupancy(X, Y, Zc, OCC, np.random.default_rng(seed), occupancy_draw)
    U = np.asarray(U) if defined_u else None
    return Structure(np.asarray(Z, np.int32)[keep], np.asarray(X)[keep], np.asarray(Y)[keep], np.asarray(Zc)[keep],
                     U[keep] if U is not None else None, name=path)


def process_occupancy(X, Y, Zc, occ, rng, draw: str = "normal"):
    """Indices kept by CrystalStructure::processOccupancyList (crystalstructure.cpp:214-236) over runs of
    consecutive atoms at one position: a single fully occupied atom is kept; otherwise one draw r keeps the
    atom whose interval [sum of earlier occupancies, + its own) holds r (or the last, when r = 1 and the sum
    is exactly 1), and a site whose occupancies add up to more than 1 is an error.

    draw="normal" takes r from a standard normal, as the reference does (its `dist` is a
    std::normal_distribution<>(0, 1), crystalstructure.h:59), so a site keeps an atom with probability
    Phi(total occupancy) - 1/2 at most; draw="uniform" takes r uniform on [0, 1), which keeps each atom with
    the probability of its occupancy."""
    if draw not in ("normal", "uniform"):
        raise ValueError("occupancy draw must be 'normal' or 'uniform'")
    keep = []
    i, n = 0, len(X)
    while i < n:
        j = i + 1
        while j < n and X[j] == X[i] and Y[j] == Y[i] and Zc[j] == Zc[i]:
            j += 1
        if j - i == 1 and occ[i] == 1.0:
            keep.append(i)
        else:
            r = float(rng.standard_normal()) if draw == "normal" else float(rng.random())
            total = 0.0
            for k in range(i, j):
                if (total <= r < total + occ[k]) or (r == 1.0 and total + occ[k] == 1.0):
                    keep.append(k)
                total += occ[k]
            if total > 1.0000001:
                raise RuntimeError(".xyz has occupancies > 1.")
        i = j
    return np.asarray(keep, dtype=np.int64)


def write_xyz(s: Structure, path: str):
    with open(path, "w") as f:
        f.write(f"{len(s)}\nA x y z\n")
        for a, x, y, z in zip(s.Z, s.x, s.y, s.z):
            f.write(f"{ELEMENTS[int(a) - 1]} {x:.6f} {y:.6f} {z:.6f}\n")


def perovskite(nx: int, ny: int, nz: int, a: float = 3.905, A: int = 38, B: int = 22, X: int = 8) -> Structure:
    """Cubic ABX3 cell: A at (0,0,0), B at (1/2,1/2,1/2), X at face centres, tiled nx*ny*nz."""
    basis = [(A, 0.0, 0.0, 0.0), (B, 0.5, 0.5, 0.5), (X, 0.5, 0.5, 0.0), (X, 0.5, 0.0, 0.5), (X, 0.0, 0.5, 0.5)]
    return _tile(basis, a, nx, ny, nz, "perovskite")


def fcc(nx: int, ny: int, nz: int, a: float = 4.08, Zn: int = 79) -> Structure:
    basis = [(Zn, 0.0, 0.0, 0.0), (Zn, 0.5, 0.5, 0.0), (Zn, 0.5, 0.0, 0.5), (Zn, 0.0, 0.5, 0.5)]
    return _tile(basis, a, nx, ny, nz, "fcc")


def _tile(basis, a, nx, ny, nz, name):
    Z, X, Y, W = [], [], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for (zn, fx, fy, fz) in basis:
                    Z.append(zn)
                    X.append((i + fx) * a)
                    Y.append((j + fy) * a)
                    W.append((k + fz) * a)
    return Structure(np.asarray(Z, np.int32), np.asarray(X, np.float64), np.asarray(Y, np.float64),
                     np.asarray(W, np.float64), name=f"{name}_{nx}x{ny}x{nz}")


def _displaced(s: Structure, sd: np.ndarray, n_configs: int, seed: int, axes=None):
    out = []
    for c in range(n_configs):
        rng = np.random.Generator(np.random.PCG64([seed, c]))
        d = rng.standard_normal((len(s), 3)) * sd
        if axes is None:
            x, y, z = s.x + d[:, 0], s.y + d[:, 1], s.z + d[:, 2]
        else:   # x + d1 u1 + d2 u2 + d3 u3 (simulationgeneral.cpp:196-202)
            u1, u2, u3 = (np.asarray(a, dtype=np.float64) for a in axes)
            x = s.x + d[:, 0] * u1[0] + d[:, 1] * u2[0] + d[:, 2] * u3[0]
            y = s.y + d[:, 0] * u1[1] + d[:, 1] * u2[1] + d[:, 2] * u3[1]
            z = s.z + d[:, 0] * u1[2] + d[:, 1] * u2[2] + d[:, 2] * u3[2]
        out.append(Structure(s.Z.copy(), x, y, z, name=f"{s.name}#ph{c}"))
    return out


def phonon_configs(s: Structure, n_configs: int, u_rms: float, seed: int = 0):
    """n_configs frozen-phonon configurations: each atom displaced by N(0, u_rms^2) per axis (or by the
    structure's own u2 when it has one), FP64, configuration c drawn from numpy's PCG64 seeded with
    (seed, c)."""
    sd = np.sqrt(s.u2) if s.u2 is not None else np.full((len(s), 3), float(u_rms))
    return _displaced(s, sd, n_configs, seed)


@dataclass
class Vibrations:
    """Thermal-vibration settings of PhononScattering (src/simulation/incoherence/inelastic/phonon.cpp,
    read by JsonToThermalVibrations, src/simulation/utilities/jsonutils.cpp:368-418)."""
    default: float = 0.0          # Å^2, "default"/"value": every element not in `values`
    values: dict = field(default_factory=dict)   # atomic number -> Å^2 ("values")
    force_default: bool = False   # "force default"
    force_defined: bool = False   # "override file": the element table over the file's values
    force_xyz: bool = False       # "force xyz displacements": x, y, z axes over the structure's

    def vibration(self, Z: np.ndarray) -> np.ndarray:
        """PhononScattering::getVibrations for each atomic number."""
        table = np.full(max(int(np.max(Z, initial=0)), max(self.values, default=0)) + 1, float(self.default))
        for k, v in self.values.items():
            table[int(k)] = float(v)
        return table[np.asarray(Z, dtype=np.int64)]

    def mean_square(self, s: Structure) -> np.ndarray:
        """Per atom and axis the u^2 PhononScattering::generateTdsFactor (phonon.cpp:98-128) takes: the
        default when forced, else the element table when the file is overridden, else the file's value for
        atoms that define one, else the element table."""
        n = len(s)
        if self.force_default:
            return np.full((n, 3), float(self.default))
        table = np.repeat(self.vibration(s.Z)[:, None], 3, axis=1)
        if self.force_defined or s.u2 is None:
            return table
        defined = np.ones(n, dtype=bool) if s.defined_u is None else np.asarray(s.defined_u, dtype=bool)
        return np.where(defined[:, None], np.asarray(s.u2, dtype=np.float64), table)


def frozen_phonon_configs(s: Structure, n_configs: int, vib: Vibrations, seed: int = 0):
    """n_configs frozen-phonon configurations as SimulationGeneral::sortAtoms makes one
    (simulationgeneral.cpp:177-205): per atom three deviates sqrt(u^2) N(0, 1) along the structure's
    displacement axes (its rotated cell vectors for a CIF supercell; x, y, z for .xyz input or when
    forced), with u^2 from Vibrations.mean_square. Configuration c draws from numpy's PCG64 seeded with
    (seed, c); the reference's generator is clock-seeded."""
    with np.errstate(invalid="ignore"):
        sd = np.sqrt(vib.mean_square(s))
    axes = None if (vib.force_xyz or s.axes is None) else s.axes
    return _displaced(s, sd, n_configs, seed, axes)


def concat_configs(configs):
    """Concatenate configurations into the flat arrays mslice_stage_configs takes."""
    counts = np.asarray([len(c) for c in configs], dtype=np.uint64)
    Z = np.ascontiguousarray(np.concatenate([c.Z for c in configs]).astype(np.int32))
    x = np.ascontiguousarray(np.concatenate([c.x for c in configs]))
    y = np.ascontiguousarray(np.concatenate([c.y for c in configs]))
    z = np.ascontiguousarray(np.concatenate([c.z for c in configs]))
    return counts, Z, x, y, z


def wavelength(voltage_kv: float) -> float:
    """MicroscopeParameters::Wavelength (commonstructs.h:269-271), Å."""
    h, c, e, m = 6.6262e-034, 299792458.0, 1.6021773e-019, 9.10938291e-031
    V = voltage_kv * 1000
    return h * c / math.sqrt(e * V * (2 * m * c * c + e * V)) * 1e10

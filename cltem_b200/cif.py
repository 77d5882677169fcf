"""CIF input: cell geometry, symmetry operations, atom sites and the zone-axis supercell.

Restates clTEM's CIF path, which turns a crystallographic information file into the atom list a
simulation stages:

- CIFReader (src/simulation/cif/cifreader.cpp:9-486): comments and leading whitespace stripped
  (cifutilities.cpp:64-90), the _symmetry_equiv_pos_ loop, every _atom_site_ loop and the cell lengths and
  angles, with the same regular expressions (Python's `re` with the ASCII flag reads the reference's
  ECMAScript patterns the same way), the same error texts and the same optional fixes ("attempt_fixes":
  P1 when no symmetry loop exists, symbols taken from labels, symbol case corrected).
- SymmetryOperation (symmetryoperation.cpp:30-71): each of x', y', z' is xf x + yf y + zf z + c, terms
  split as [+-]?[^+-]+ and fractions read as "p/q".
- AtomSite (atomsite.cpp:9-77): positions wrapped into [0, 1) as wrapPosition does (so -1 wraps to 1),
  symmetry images appended when no existing position equals them exactly, several elements per site.
- CellGeometry (cellgeometry.cpp:21-44): a along x, b in the xy plane, c from the three angles.
- make_supercell (supercell.cpp:16-171): zone axis uvw rotated onto z, optional in-plane axis abc onto x,
  small tilts about x, y, z, the rotated basis tiled over the box [0, wx] x [0, wy] x [0, wz] (inclusive on
  both sides) with the tile range of calculateTiling (:174-227).
- read_cif_structure: CrystalStructure::openCif and processAtomList (crystalstructure.cpp:194-351):
  occupancy resolution over consecutive atoms at one position, per-atom thermal flags, and the normalised
  rotated basis vectors as the frozen-phonon displacement axes.

Arithmetic is IEEE double throughout, in the reference's operation order where the order is written in its
source; products and norms that the reference leaves to Eigen are formed here in plain left-to-right
order, so positions agree with the reference's to rounding (a few ulp) and atoms lying within rounding of
the supercell's boundary planes can differ.
"""
from dataclasses import dataclass, field
import math
import re

import numpy as np

from .structure import ELEMENTS, Structure, process_occupancy

# ---------------------------------------------------------------------------------------------------
# text helpers (cifutilities.cpp)
# ---------------------------------------------------------------------------------------------------
_NUM = re.compile(r"\s*[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)", re.ASCII | re.IGNORECASE)


def _std_stod(s: str) -> float:
    """std::stod: the longest leading decimal number after optional whitespace; ValueError when none."""
    m = _NUM.match(s)
    if not m:
        raise ValueError("stod: no conversion")
    v = float(m.group(0))
    if math.isinf(v) and "inf" not in m.group(0).lower():
        raise OverflowError("stod: out of range")
    return v


def _cif_stod(s: str) -> float:
    """Utilities::stod (cifutilities.cpp:36-41): "." (a CIF null) is 0."""
    return 0.0 if s == "." else _std_stod(s)


def _number_before_bracket(s: str) -> float:
    """The value of a CIF number with an uncertainty in brackets, "0.25(3)" -> 0.25 (the reference's
    stod(split(col, '(')[0]), cifreader.cpp:339-371)."""
    return _cif_stod(s.split("(")[0])


def _split_lines(s: str):
    """Utilities::split(s, '\\n') as getline yields the pieces: no trailing empty piece."""
    parts = s.split("\n")
    if parts and parts[-1] == "":
        parts.pop()
    return parts


def strip_comments_whitespace(text: str) -> str:
    """Utilities::stripCommentsWhitespace (cifutilities.cpp:64-90): per line, drop the leading
    whitespace, cut at the last '#', keep non-empty lines. Trailing whitespace stays on the line: the
    reference's substring length start - last + 1 wraps around (size_t) for any line longer than one
    character, so the substring runs to the end of the line."""
    out = []
    for line in text.split("\n"):
        start = None
        for i, ch in enumerate(line):
            if ch not in " \n\r\t":
                start = i
                break
        if start is None:
            continue
        last = max(i for i, ch in enumerate(line) if ch not in " \n\r\t")
        temp = line[start:] if last != start else line[start:start + 1]
        comm = temp.rfind("#")
        if comm >= 0:
            temp = temp[:comm]
        if temp:
            out.append(temp + "\n")
    return "".join(out)


ACCEPTED_ATOMS = ELEMENTS[:102]   # H .. No (cifutilities.cpp:93-194)


# ---------------------------------------------------------------------------------------------------
# symmetry (symmetryoperation.cpp)
# ---------------------------------------------------------------------------------------------------
def _fraction_to_decimal(s: str, null_return: float) -> float:
    """SymmetryOperation::fractionToDecimal (symmetryoperation.cpp:56-70). A term with no '/' other than
    a bare sign (e.g. "0.5" or "2x") indexes past the split in the reference; here it is an error."""
    if s == "":
        return null_return
    if s == "+":
        return 1.0
    if s == "-":
        return -1.0
    f = s.split("/")
    if len(f) < 2 or f[0] == "":
        raise RuntimeError(f"Problem parsing symmetry operation term: {s}")
    return _std_stod(f[0]) / _std_stod(f[1])


@dataclass
class SymmetryOperation:
    xf: float = 0.0
    yf: float = 0.0
    zf: float = 0.0
    c: float = 0.0

    @classmethod
    def from_terms(cls, terms):
        op = cls()
        for t in terms:
            if t.endswith("x"):
                op.xf += _fraction_to_decimal(t[:-1], 1.0)
            elif t.endswith("y"):
                op.yf += _fraction_to_decimal(t[:-1], 1.0)
            elif t.endswith("z"):
                op.zf += _fraction_to_decimal(t[:-1], 1.0)
            else:
                op.c += _fraction_to_decimal(t, 0.0)
        return op

    def apply(self, p):
        return self.xf * p[0] + self.yf * p[1] + self.zf * p[2] + self.c


@dataclass
class Symmetry:
    ops: tuple   # (x', y', z') SymmetryOperation

    @classmethod
    def identity(cls):
        return cls.from_strings(["x", "y", "z"])

    @classmethod
    def from_strings(cls, three):
        rx = re.compile(r"([+-]?[^+-]+)", re.ASCII)
        out = []
        for s in three:
            terms = rx.findall(s)
            if len(terms) < 1:
                raise RuntimeError("Problem parsing symmetry operation.")
            out.append(SymmetryOperation.from_terms(terms))
        return cls(tuple(out))


# ---------------------------------------------------------------------------------------------------
# atom sites (atomsite.cpp)
# ---------------------------------------------------------------------------------------------------
def wrap_position(p: float) -> float:
    """AtomSite::wrapPosition (atomsite.cpp:47-56): >= 1 keeps the fractional part, < 0 adds 1 to it."""
    if p >= 1.0:
        return math.modf(p)[0]
    if p < 0.0:
        return 1.0 + math.modf(p)[0]
    return p


@dataclass
class AtomSite:
    elements: list
    labels: list
    occupancies: list
    positions: list           # fractional [x, y, z] lists: the wrapped file position, then symmetry images
    thermal_u: list           # per element [u11, u22, u33] (Å^2)
    thermal_defined: bool = False

    @classmethod
    def create(cls, symmetries, symbol, label, x, y, z, occ):
        site = cls([symbol], [label], [occ], [[wrap_position(x), wrap_position(y), wrap_position(z)]],
                   [[0.0, 0.0, 0.0]])
        p0 = site.positions[0]
        for s in symmetries:
            img = [wrap_position(s.ops[0].apply(p0)), wrap_position(s.ops[1].apply(p0)),
                   wrap_position(s.ops[2].apply(p0))]
            if img not in site.positions:
                site.positions.append(img)
        return site

    def add_atom(self, symbol, label, occ):
        self.elements.append(symbol)
        self.labels.append(label)
        self.occupancies.append(occ)
        self.thermal_u.append([0.0, 0.0, 0.0])

    def set_iso_u(self, label, u):
        if label not in self.labels:
            return False
        self.thermal_u[self.labels.index(label)] = [u, u, u]
        self.thermal_defined = True
        return True

    def set_u(self, label, u, axis):
        if label not in self.labels:
            return False
        self.thermal_u[self.labels.index(label)][axis] = u
        self.thermal_defined = True
        return True


# ---------------------------------------------------------------------------------------------------
# cell geometry (cellgeometry.cpp)
# ---------------------------------------------------------------------------------------------------
@dataclass
class CellGeometry:
    a: float
    b: float
    c: float
    alpha: float
    beta: float
    gamma: float
    avec: list = field(default_factory=list)
    bvec: list = field(default_factory=list)
    cvec: list = field(default_factory=list)

    def __post_init__(self):
        f = np.float64
        ar = f(self.alpha) * (math.pi / 180)
        br = f(self.beta) * (math.pi / 180)
        gr = f(self.gamma) * (math.pi / 180)
        with np.errstate(all="ignore"):   # degenerate angles give inf / NaN as in the reference
            self.avec = [float(self.a), 0.0, 0.0]
            self.bvec = [float(f(self.b) * np.cos(gr)), float(f(self.b) * np.sin(gr)), 0.0]
            cv1 = f(self.c) * np.cos(br)
            cv2 = f(self.c) * (np.cos(ar) - np.cos(br) * np.cos(gr)) / np.sin(gr)
            cv3 = f(self.c) * np.sqrt((np.cos(br - gr) - np.cos(ar)) * (np.cos(ar) - np.cos(br + gr))) / np.sin(gr)
        self.cvec = [float(cv1), float(cv2), float(cv3)]


# ---------------------------------------------------------------------------------------------------
# reader (cifreader.cpp)
# ---------------------------------------------------------------------------------------------------
class CIFReader:
    """A parsed CIF (CIF::CIFReader). `fix` is the reference's attempt_fixes switch (the console's --fix):
    P1 symmetry when no _symmetry_equiv_pos_ loop exists, type symbols taken from labels when the
    _atom_site_type_symbol column is absent, and symbol case corrected (sr -> Sr)."""

    def __init__(self, path: str = None, fix: bool = False, text: str = None):
        if text is None:
            with open(path, "r", newline="") as f:
                text = f.read()
        self.file_path = path or ""
        self.fix = fix
        content = strip_comments_whitespace(text)
        errors = ""
        self.symmetries, self.sites, self.cell = [], [], None
        for step in (self._read_symmetry, self._read_atoms, self._read_cell):
            try:
                step(content)
            except RuntimeError as e:
                errors += str(e)
        if errors:
            raise RuntimeError(errors)

    # cifreader.cpp:52-173
    def _read_symmetry(self, content):
        self.symmetries = []
        m = re.search(r"(?:loop_\n)((?:_symmetry_equiv_pos_\w+?\n)+)", content, re.ASCII)
        if not m:
            if self.fix:
                self.symmetries = [Symmetry.identity()]
                return
            raise RuntimeError("Cannot find _symmetry_equiv_pos_ block\n")
        headers = _split_lines(m.group(1))
        if "_symmetry_equiv_pos_as_xyz" not in headers:
            raise RuntimeError("Could not find _symmetry_equiv_pos_as_xyz\n")
        xyzcol = headers.index("_symmetry_equiv_pos_as_xyz")
        cols = ["(?:['\"]?.+?,.+?,.+?['\"]?)" if i == xyzcol else r"\S+" for i in range(len(headers))]
        row_rx = re.compile("[ \\t]+".join(cols), re.ASCII)
        element_rx = re.compile(r"(['\"].+?['\"]|[\S]+)", re.ASCII)
        xyz_rx = re.compile(r"['\"]*\s*([^\s'\"]+)\s*,\s*([^\s'\"]+)\s*,\s*([^\s'\"]+)\s*['\"]*", re.ASCII)
        for line in content[m.end():].split("\n"):
            if not row_rx.fullmatch(line):
                break
            column = element_rx.findall(line)
            mx = xyz_rx.search(column[xyzcol])
            if not mx:
                raise RuntimeError("Problem parsing _symmetry_equiv_pos_ line\n")
            self.symmetries.append(Symmetry.from_strings([mx.group(1), mx.group(2), mx.group(3)]))
        if not self.symmetries:
            raise RuntimeError("Problem parsing _symmetry_equiv_pos_ block.")

    # cifreader.cpp:175-254
    def _read_atoms(self, content):
        self.sites = []
        header_rx = re.compile(r"(?:\nloop_\n)((?:_atom_site_\w+?\n)+)", re.ASCII)
        blocks = []
        for m in header_rx.finditer(content):
            headers = _split_lines(m.group(1))
            pat = r"((?:\s*" + r"\S+[ \t]+" * (len(headers) - 1) + r"\S+[ \t]*)+)"
            row_rx = re.compile(pat, re.ASCII)
            rows = []
            # the reference reads lines from the match's suffix to the end of the text
            for line in content[m.end():].split("\n"):
                if not row_rx.fullmatch(line) or line == "loop_":
                    break
                rows.append(line)
            blocks.append((headers, rows))
        if not blocks:
            raise RuntimeError("Could not find _atom_site_ block(s)\n")
        errors = []
        for headers, rows in blocks:
            try:
                self._read_positions(headers, rows)
                errors.append("")
            except RuntimeError as e:
                errors.append(str(e))
        if not any(e == "" for e in errors):
            raise RuntimeError("".join(errors))
        for headers, rows in blocks:
            self._read_thermals(headers, rows)
        if not self.sites:
            raise RuntimeError("Could not parse atom information")

    # cifreader.cpp:270-399
    def _read_positions(self, headers, rows):
        def col(name):
            return headers.index(name) if name in headers else len(headers)
        n = len(headers)
        labelcol, xcol, ycol, zcol = col("_atom_site_label"), col("_atom_site_fract_x"), \
            col("_atom_site_fract_y"), col("_atom_site_fract_z")
        symbolcol, occcol = col("_atom_site_type_symbol"), col("_atom_site_occupancy")
        found_label, found_symbol = labelcol != n, symbolcol != n
        if self.fix and not found_symbol and found_label:
            symbolcol, found_symbol = labelcol, True
        errors = ""
        if not found_label:
            errors += "Could not find _atom_site_label\n"
        if not found_symbol:
            errors += "Could not find _atom_site_type_symbol\n"
        if xcol == n:
            errors += "Could not find _atom_site_fract_x\n"
        if ycol == n:
            errors += "Could not find _atom_site_fract_y\n"
        if zcol == n:
            errors += "Could not find _atom_site_fract_z\n"
        if errors:
            raise RuntimeError(errors)
        name_rx = re.compile(r"([a-zA-Z]{1,2})", re.ASCII)
        for row in rows:
            columns = re.findall(r"\S+", row, re.ASCII)
            label = columns[labelcol]
            m = name_rx.search(columns[symbolcol])
            symbol = m.group(1) if m else ""
            if not m:
                errors += ("Could not find acceptable format _atom_site_type_symbol (need 1-2 letters) in: "
                           + columns[symbolcol] + "\n")
            if self.fix and symbol:
                symbol = symbol[0].upper() + symbol[1:].lower()
            if symbol not in ACCEPTED_ATOMS:
                errors += ("Could not detect valid atom from: " + columns[symbolcol] + " (sub string: " + symbol
                           + ")\n")
            pos = []
            for c in (xcol, ycol, zcol):
                try:
                    pos.append(_number_before_bracket(columns[c]))
                except ValueError:
                    errors += "Could not get number from position values (not a number): " + columns[c] + "\n"
                except OverflowError:
                    errors += "Could not get number from position values (value too large): " + columns[c] + "\n"
            occ = 1.0
            if occcol != n:
                try:
                    occ = _number_before_bracket(columns[occcol])
                except ValueError:
                    errors += "Could not get number from occupancy value (not a number): " + columns[occcol] + "\n"
                except OverflowError:
                    errors += "Could not get number from occupancy (value too large): " + columns[occcol] + "\n"
            if errors:
                continue   # once a row has failed the reference skips every later row of the block
            for site in self.sites:
                if pos in site.positions:
                    site.add_atom(symbol, label, occ)
                    break
            else:
                self.sites.append(AtomSite.create(self.symmetries, symbol, label, pos[0], pos[1], pos[2], occ))
        if errors:
            raise RuntimeError(errors)

    # cifreader.cpp:401-482
    def _read_thermals(self, headers, rows):
        def col(name):
            return headers.index(name) if name in headers else len(headers)
        n = len(headers)
        labelcol = col("_atom_site_label")
        if labelcol == n:
            labelcol = col("_atom_site_aniso_label")
        if labelcol == n:
            return
        isocol = col("_atom_site_B_iso_or_equiv")
        uxcol, uycol, uzcol = col("_atom_site_aniso_U_11"), col("_atom_site_aniso_U_22"), col("_atom_site_aniso_U_33")
        found_iso, found_ux, found_uy, found_uz = isocol != n, uxcol != n, uycol != n, uzcol != n
        if found_ux and not (found_uy and found_uz):
            # the reference reads the U_22 and U_33 columns whenever U_11 exists
            raise RuntimeError("_atom_site_aniso_U_11 given without _atom_site_aniso_U_22 and _U_33\n")
        for row in rows:
            columns = re.findall(r"\S+", row, re.ASCII)
            lbl = columns[labelcol]
            try:
                u_iso = _number_before_bracket(columns[isocol]) if found_iso else 0.0
                u = [_number_before_bracket(columns[c]) if found_ux else 0.0 for c in (uxcol, uycol, uzcol)]
            except (ValueError, OverflowError) as e:
                raise RuntimeError(f"Could not read thermal parameters of {lbl}: {e}\n")
            for site in self.sites:
                if found_iso:
                    site.set_iso_u(lbl, u_iso)
                if found_ux:
                    site.set_u(lbl, u[0], 0)
                if found_uy:
                    site.set_u(lbl, u[1], 1)
                if found_uz:
                    site.set_u(lbl, u[2], 2)

    # cifreader.cpp:256-266 (a missing tag reads as 0, Utilities::regexFindDoubleTag)
    def _read_cell(self, content):
        def tag(name):
            m = re.search(name + r"\s+([\d.]+)", content, re.ASCII)
            return _std_stod(m.group(1)) if m else 0.0
        self.cell = CellGeometry(tag("_cell_length_a"), tag("_cell_length_b"), tag("_cell_length_c"),
                                 tag("_cell_angle_alpha"), tag("_cell_angle_beta"), tag("_cell_angle_gamma"))


# ---------------------------------------------------------------------------------------------------
# rotations (cifutilities.h:44-95) and the supercell (supercell.cpp)
# ---------------------------------------------------------------------------------------------------
def _norm2(v):
    return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]


def _normalized(v):
    """Eigen's normalize(): unchanged when the norm is 0."""
    z = _norm2(v)
    if z > 0:
        r = math.sqrt(z)
        return [v[0] / r, v[1] / r, v[2] / r]
    return list(v)


def _is_approx(a, b, prec=1e-12):
    """Eigen's isApprox: |a - b|^2 <= prec^2 min(|a|^2, |b|^2)."""
    d = [a[0] - b[0], a[1] - b[1], a[2] - b[2]]
    return _norm2(d) <= prec * prec * min(_norm2(a), _norm2(b))


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _matmul(A, B):
    return [[A[i][0] * B[0][j] + A[i][1] * B[1][j] + A[i][2] * B[2][j] for j in range(3)] for i in range(3)]


def _matvec(A, v):
    return [A[i][0] * v[0] + A[i][1] * v[1] + A[i][2] * v[2] for i in range(3)]


_I3 = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]


def _skew(v):
    return [[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]]


def normalised_rotation(A, B):
    """Utilities::generateNormalisedRotationMatrix (cifutilities.h:44-74): the rotation taking the
    direction of A onto that of B, I + K + K^2 (1 - c) / s^2 with K = [A x B]_x, c = A.B, s = |A x B|.
    For antiparallel vectors the reference crosses A with x (or x + z) and keeps the same formula."""
    A, B = _normalized(A), _normalized(B)
    if _is_approx(A, B):
        return [row[:] for row in _I3]
    v = _cross(A, B)
    if _is_approx(A, [-B[0], -B[1], -B[2]]):
        temp = [1.0, 0.0, 0.0]
        if _is_approx(temp, A):
            temp[2] = 1.0
        v = _cross(A, temp)
    c = A[0] * B[0] + A[1] * B[1] + A[2] * B[2]
    s = math.sqrt(_norm2(v))
    K = _skew(v)
    KK = _matmul(K, K)
    with np.errstate(all="ignore"):   # s = 0 (a zero vector) gives NaN as in the reference
        X = [[float(np.float64(KK[i][j] * (1 - c)) / np.float64(s * s)) for j in range(3)] for i in range(3)]
    return [[_I3[i][j] + K[i][j] + X[i][j] for j in range(3)] for i in range(3)]


def axis_rotation(ax, theta):
    """Utilities::generateRotationMatrix (cifutilities.h:76-89): I + C sin(t) + C^2 (1 - cos(t)),
    C = [ax / |ax|]_x."""
    C = _skew(_normalized(ax))
    CC = _matmul(C, C)
    s, c1 = math.sin(theta), 1 - math.cos(theta)
    return [[_I3[i][j] + C[i][j] * s + CC[i][j] * c1 for j in range(3)] for i in range(3)]


def calculate_tiling(basis, wx, wy, wz):
    """calculateTiling (supercell.cpp:174-227): the box's 8 corners in the rotated basis, each
    coordinate rounded away from zero, min and max over the corners per axis. The reference's running
    extremes start from LONG_MIN / LONG_MAX narrowed into the int elements of an Eigen::Vector3i, i.e.
    0 and -1 under a 64-bit long, so the tile range always holds [-1, 0]."""
    M = np.eye(4)
    M[0, :] = 1.0
    M[0, 0] = 1.0
    for k in range(3):
        M[1:, k + 1] = basis[k]
    M[1:, 0] = 0.0
    T = np.linalg.inv(M)[1:, :]
    corners = [(0, 0, 0), (wx, 0, 0), (0, wy, 0), (0, 0, wz), (wx, wy, 0), (wx, 0, wz), (0, wy, wz), (wx, wy, wz)]
    mins, maxs = [-1, -1, -1], [0, 0, 0]
    for (cx, cy, cz) in corners:
        f = T @ np.array([1.0, cx, cy, cz])
        if not np.all(np.isfinite(f)):
            raise RuntimeError("Supercell basis is degenerate (non-finite tiling)")
        for a in range(3):
            r = int((1 if f[a] > 0 else (-1 if f[a] < 0 else 0)) * math.ceil(abs(f[a])))
            maxs[a] = max(maxs[a], r)
            mins[a] = min(mins[a], r)
    return mins, maxs


@dataclass
class SuperCellInfo:
    """CIF::SuperCellInfo (supercell.h:13-40) with its defaults."""
    uvw: tuple = (0.0, 0.0, 1.0)         # zone axis (lattice direction along z)
    abc: tuple = (0.0, 0.0, 0.0)         # lattice direction placed along x; all zero: no in-plane rotation
    widths: tuple = (100.0, 100.0, 100.0)  # Å
    tilts: tuple = (0.0, 0.0, 0.0)       # degrees about x, y, z


@dataclass
class SuperCell:
    symbols: list
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    occ: np.ndarray
    defined_u: np.ndarray
    u: np.ndarray              # float64[n, 3]
    basis: list                # the rotated a, b, c vectors (Å)


def make_supercell(cif: CIFReader, info: SuperCellInfo = None) -> SuperCell:
    """makeSuperCell (supercell.cpp:16-171): the atoms of the rotated, tiled crystal inside
    [0, wx] x [0, wy] x [0, wz], ordered by site, symmetry image, tile (z outermost, x innermost) and
    element of the site."""
    info = info or SuperCellInfo()
    geom = cif.cell
    a_v, b_v, c_v = geom.avec, geom.bvec, geom.cvec
    basis = [list(a_v), list(b_v), list(c_v)]
    u, v, w = (float(q) for q in info.uvw)
    uvw_vec = [u * a_v[i] + v * b_v[i] + w * c_v[i] for i in range(3)]
    zdir = [0.0, 0.0, 1.0]
    za = normalised_rotation(uvw_vec, zdir)
    if any(math.isnan(q) for row in za for q in row):
        raise RuntimeError("Zone axis rotation matrix contains NaNs")
    xy = [row[:] for row in _I3]
    if any(float(q) != 0 for q in info.abc):
        p, q, r = (float(t) for t in info.abc)
        abc_vec = [p * a_v[i] + q * b_v[i] + r * c_v[i] for i in range(3)]
        abc_vec = _matvec(za, abc_vec)
        abc_vec[2] = 0.0
        if abs(abc_vec[0]) < 1e-15:
            abc_vec[0] = 0.0
        if abs(abc_vec[1]) < 1e-15:
            abc_vec[1] = 0.0
        xdir = [1.0, 0.0, 0.0]
        n = _normalized(abc_vec)
        if _is_approx(xdir, [-n[0], -n[1], -n[2]]):
            xy = axis_rotation(zdir, math.pi)
        else:
            xy = normalised_rotation(xdir, abc_vec)
    if any(math.isnan(q) for row in xy for q in row):
        raise RuntimeError("Normal rotation matrix contains NaNs")
    tx, ty, tz = (float(t) * math.pi / 180 for t in info.tilts)
    rots = [za, xy, axis_rotation([1.0, 0.0, 0.0], tx), axis_rotation([0.0, 1.0, 0.0], ty),
            axis_rotation([0.0, 0.0, 1.0], tz)]
    for i in range(3):
        for R in rots:
            basis[i] = _matvec(R, basis[i])
    wx, wy, wz = (float(t) for t in info.widths)
    mins, maxs = calculate_tiling(basis, wx, wy, wz)
    # tile grid in loop order: k (c) outermost, then j (b), then i (a)
    K, J, I = np.meshgrid(np.arange(mins[2], maxs[2], dtype=np.float64),
                          np.arange(mins[1], maxs[1], dtype=np.float64),
                          np.arange(mins[0], maxs[0], dtype=np.float64), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    B = [np.asarray(b, dtype=np.float64) for b in basis]
    symbols, xs, ys, zs, occ, du, us = [], [], [], [], [], [], []
    for site in cif.sites:
        ne = len(site.elements)
        for pos in site.positions:
            p = [(pos[0] * B[0][c] + pos[1] * B[1][c]) + pos[2] * B[2][c] for c in range(3)]
            np_ = [((p[c] + B[0][c] * I) + B[1][c] * J) + B[2][c] * K for c in range(3)]
            keep = ((np_[0] >= 0.0) & (np_[0] <= wx) & (np_[1] >= 0.0) & (np_[1] <= wy) &
                    (np_[2] >= 0.0) & (np_[2] <= wz))
            idx = np.nonzero(keep)[0]
            if idx.size == 0:
                continue
            rep = np.repeat(idx, ne)
            el = np.tile(np.arange(ne), idx.size)
            xs.append(np_[0][rep])
            ys.append(np_[1][rep])
            zs.append(np_[2][rep])
            symbols.extend(site.elements[e] for e in el)
            occ.append(np.asarray(site.occupancies, dtype=np.float64)[el])
            us.append(np.asarray(site.thermal_u, dtype=np.float64).reshape(ne, 3)[el])
            du.append(np.full(rep.size, site.thermal_defined))
    if not xs:
        raise RuntimeError("Did not find any atoms inside limits")
    return SuperCell(symbols, np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), np.concatenate(occ),
                     np.concatenate(du), np.concatenate(us), basis)


def read_cif_structure(path: str, info: SuperCellInfo = None, fix: bool = False, seed: int = 0,
                       occupancy_draw: str = "normal", text: str = None) -> Structure:
    """A simulation structure from a CIF: CrystalStructure::openCif (crystalstructure.cpp:194-210) over
    make_supercell. Consecutive atoms at one position form a site resolved by one draw from a generator
    seeded by `seed` (processOccupancyList; see structure.process_occupancy for `occupancy_draw`). The
    structure carries the per-atom thermal flags and U values and, as displacement axes for frozen
    phonons, the rotated a, b, c directions normalised (u1_vector .. u3_vector)."""
    cif = CIFReader(path, fix=fix, text=text)
    sc = make_supercell(cif, info)
    Z = np.asarray([ELEMENTS.index(s) + 1 for s in sc.symbols], dtype=np.int32)
    keep = process_occupancy(sc.x, sc.y, sc.z, sc.occ, np.random.default_rng(seed), occupancy_draw)
    axes = np.asarray([_normalized(b) for b in sc.basis], dtype=np.float64)
    return Structure(Z[keep], sc.x[keep], sc.y[keep], sc.z[keep], u2=sc.u[keep], name=path or "cif",
                     defined_u=sc.defined_u[keep], axes=axes)

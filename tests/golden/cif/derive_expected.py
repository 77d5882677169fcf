"""Derives, step by step, the atom lists clTEM's CIF supercell code makes from the hand-made CIF files in this
folder, and writes them to expected.json. The test suite compares cltem_b200.cif against that file.

The derivation is independent of cltem_b200 (numpy only). Each step cites the clTEM source it restates
(paths relative to the clTEM project root; Eigen is not available here, so the reference itself cannot be
compiled and run on these files):
  1. symmetry images of each site: listed by hand below from the file's symmetry operations, each operation
     evaluated as xf*x + yf*y + zf*z + c (src/simulation/cif/symmetryoperation.cpp:53-55), wrapped into [0, 1)
     (atomsite.cpp:41-48), a new position kept only if not already in the site's list (atomsite.cpp:20-27);
     a later row at an existing position joins that site as another element (cifreader.cpp, the
     `_atom_site` loop);
  2. the cell's Cartesian a, b, c (cellgeometry.cpp:18-35);
  3. the zone-axis rotation taking u a + v b + w c onto z (supercell.cpp:37-45), the in-plane rotation taking
     x onto the projected a b c direction (supercell.cpp:48-69), the tilt rotations about x, y, z
     (supercell.cpp:72-79), applied to the basis in that order (supercell.cpp:81-87), each rotation built as
     in src/simulation/cif/cifutilities.h:47-89;
  4. the tile range: the box's 8 corners in the rotated basis, each coordinate rounded away from zero, min and
     max per axis (supercell.cpp:174-227), the running extremes starting at 0 and -1 (LONG_MIN / LONG_MAX
     narrowed into Eigen::Vector3i's int elements);
  5. the atoms: per site, per symmetry image, tiles with c outermost and a innermost, per element of the site,
     kept when inside [0, w] on all three axes, faces included (supercell.cpp:123-156, 235-237).

Run from the repository root: python tests/golden/cif/derive_expected.py
"""
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def wrap(p):
    """atomsite.cpp:41-48."""
    if p >= 1.0:
        return math.modf(p)[0]
    if p < 0.0:
        return 1.0 + math.modf(p)[0]
    return p


# Step 1 by hand: the symmetry images of every site, in the order the operations produce them.
CASES = {
    "simple_cubic_p1": {
        # one operation (x, y, z): the site's only position is its own
        "sites": [{"elements": ["Fe"], "occ": [1.0], "positions": [[0.25, 0.5, 0.75]]}],
        "cell": (4.0, 4.0, 4.0, 90.0, 90.0, 90.0),
        "uvw": (0.0, 0.0, 1.0), "abc": (0.0, 0.0, 0.0), "widths": (8.0, 8.0, 4.0), "tilts": (0.0, 0.0, 0.0),
    },
    "perovskite_m3m_001_tilted": {
        # the 48 signed permutations of (x, y, z): Sr (0, 0, 0) and Ti (1/2, 1/2, 1/2) map onto themselves (-0 and
        # -1/2 wrap to 0 and 1/2); O (1/2, 1/2, 0) gives (1/2, 1/2, 0) under the permutations fixing z, then
        # (1/2, 0, 1/2) first under (x, z, y) and (0, 1/2, 1/2) first under (z, x, y)... in the operations'
        # order: x,y,z first, then the first permutation moving z, which is +x,+z,+y
        "sites": [{"elements": ["Sr"], "occ": [1.0], "positions": [[0.0, 0.0, 0.0]]},
                  {"elements": ["Ti"], "occ": [1.0], "positions": [[0.5, 0.5, 0.5]]},
                  {"elements": ["O"], "occ": [1.0], "positions": [[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]}],
        "cell": (3.905, 3.905, 3.905, 90.0, 90.0, 90.0),
        "uvw": (0.0, 0.0, 1.0), "abc": (0.0, 0.0, 0.0), "widths": (7.0, 7.0, 7.0), "tilts": (0.4, 0.7, 0.0),
    },
    "perovskite_m3m_110_tilted": {
        "sites": [{"elements": ["Sr"], "occ": [1.0], "positions": [[0.0, 0.0, 0.0]]},
                  {"elements": ["Ti"], "occ": [1.0], "positions": [[0.5, 0.5, 0.5]]},
                  {"elements": ["O"], "occ": [1.0], "positions": [[0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]}],
        "cell": (3.905, 3.905, 3.905, 90.0, 90.0, 90.0),
        "uvw": (1.0, 1.0, 0.0), "abc": (0.0, 0.0, 1.0), "widths": (9.0, 8.0, 6.0), "tilts": (0.5, 0.3, 0.2),
    },
    "hexagonal_two_sites": {
        # operations x,y,z / -y,x-y,z / -x+y,-x,z. Zn (0, 0, 0): every image is (0, 0, 0) (-0 wraps to 0).
        # O at (0.1, 0.2, 0.375): (0.1, 0.2), then (-0.2, 0.1 - 0.2) -> (1 - 0.2, 1 - 0.1) = (0.8, 0.9), then
        # (-0.1 + 0.2, -0.1) -> (0.1, 0.9); N on the same position joins O's site as a second element.
        "sites": [{"elements": ["Zn"], "occ": [1.0], "positions": [[0.0, 0.0, 0.0]]},
                  {"elements": ["O", "N"], "occ": [0.5, 0.5],
                   "positions": [[0.1, 0.2, 0.375], [wrap(-0.2), wrap(0.1 - 0.2), 0.375], [wrap(-0.1 + 0.2), wrap(-0.1), 0.375]]}],
        "cell": (3.0, 3.0, 5.0, 90.0, 90.0, 120.0),
        "uvw": (0.0, 0.0, 1.0), "abc": (1.0, 1.0, 0.0), "widths": (6.5, 5.5, 5.0), "tilts": (0.6, -0.4, 1.5),
    },
}
FILES = {"simple_cubic_p1": "simple_cubic_p1.cif", "perovskite_m3m_001_tilted": "perovskite_m3m.cif",
         "perovskite_m3m_110_tilted": "perovskite_m3m.cif", "hexagonal_two_sites": "hexagonal_two_sites.cif"}


def cell_vectors(a, b, c, al, be, ga):
    """Step 2, cellgeometry.cpp:18-35."""
    ar, br, gr = al * (math.pi / 180), be * (math.pi / 180), ga * (math.pi / 180)
    av = np.array([a, 0.0, 0.0])
    bv = np.array([b * math.cos(gr), b * math.sin(gr), 0.0])
    cv = np.array([c * math.cos(br), c * (math.cos(ar) - math.cos(br) * math.cos(gr)) / math.sin(gr),
                   c * math.sqrt((math.cos(br - gr) - math.cos(ar)) * (math.cos(ar) - math.cos(br + gr))) / math.sin(gr)])
    return av, bv, cv


def rot_onto(A, B):
    """The rotation taking A's direction onto B's (cifutilities.h:47-75)."""
    A = A / np.linalg.norm(A)
    B = B / np.linalg.norm(B)
    if np.allclose(A, B, rtol=1e-12, atol=0):
        return np.eye(3)
    v = np.cross(A, B)
    if np.allclose(A, -B, rtol=1e-12, atol=0):
        t = np.array([1.0, 0.0, 0.0])
        if np.allclose(t, A, rtol=1e-12, atol=0):
            t[2] = 1.0
        v = np.cross(A, t)
    c = float(A @ B)
    s = float(np.linalg.norm(v))
    K = np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])
    return np.eye(3) + K + K @ K * (1 - c) / (s * s)


def rot_axis(ax, theta):
    """The rotation by theta about ax (cifutilities.h:80-89)."""
    ax = np.asarray(ax, dtype=np.float64) / np.linalg.norm(ax)
    C = np.array([[0.0, -ax[2], ax[1]], [ax[2], 0.0, -ax[0]], [-ax[1], ax[0], 0.0]])
    return np.eye(3) + C * math.sin(theta) + C @ C * (1 - math.cos(theta))


def rotated_basis(case):
    """Step 3, supercell.cpp:37-87."""
    av, bv, cv = cell_vectors(*case["cell"])
    u, v, w = case["uvw"]
    za = rot_onto(u * av + v * bv + w * cv, np.array([0.0, 0.0, 1.0]))
    xy = np.eye(3)
    if any(t != 0 for t in case["abc"]):
        p, q, r = case["abc"]
        d = za @ (p * av + q * bv + r * cv)
        d[2] = 0.0
        d[np.abs(d) < 1e-15] = 0.0
        if np.allclose(np.array([1.0, 0.0, 0.0]), -d / np.linalg.norm(d), rtol=1e-12, atol=0):
            xy = rot_axis([0.0, 0.0, 1.0], math.pi)
        else:
            xy = rot_onto(np.array([1.0, 0.0, 0.0]), d)
    tx, ty, tz = (t * math.pi / 180 for t in case["tilts"])
    rots = [za, xy, rot_axis([1.0, 0.0, 0.0], tx), rot_axis([0.0, 1.0, 0.0], ty), rot_axis([0.0, 0.0, 1.0], tz)]
    basis = []
    for vec in (av, bv, cv):
        for R in rots:
            vec = R @ vec
        basis.append(vec)
    return basis


def tiling(basis, widths):
    """Step 4, supercell.cpp:174-227."""
    M = np.zeros((4, 4))
    M[0, :] = 1.0
    for k in range(3):
        M[1:, k + 1] = basis[k]
    T = np.linalg.inv(M)[1:, :]
    wx, wy, wz = widths
    mins, maxs = [-1, -1, -1], [0, 0, 0]
    for cx, cy, cz in [(0, 0, 0), (wx, 0, 0), (0, wy, 0), (0, 0, wz), (wx, wy, 0), (wx, 0, wz), (0, wy, wz), (wx, wy, wz)]:
        f = T @ np.array([1.0, cx, cy, cz])
        for a in range(3):
            r = int(math.copysign(math.ceil(abs(f[a])), f[a])) if f[a] != 0 else 0
            maxs[a], mins[a] = max(maxs[a], r), min(mins[a], r)
    return mins, maxs


def atoms(case):
    """Step 5, supercell.cpp:123-156 and 235-237."""
    basis = rotated_basis(case)
    mins, maxs = tiling(basis, case["widths"])
    wx, wy, wz = case["widths"]
    out, near = [], 0
    for site in case["sites"]:
        for pos in site["positions"]:
            p = (pos[0] * basis[0] + pos[1] * basis[1]) + pos[2] * basis[2]
            for k in range(mins[2], maxs[2]):
                for j in range(mins[1], maxs[1]):
                    for i in range(mins[0], maxs[0]):
                        q = ((p + basis[0] * i) + basis[1] * j) + basis[2] * k
                        for e, el in enumerate(site["elements"]):
                            inside = 0 <= q[0] <= wx and 0 <= q[1] <= wy and 0 <= q[2] <= wz
                            # no atom may sit within rounding of a face of the box, where the order of the sums
                            # could decide whether it is kept (an exact 0, from the zero vector, is exact in every
                            # order)
                            loose = all(-1e-7 <= c <= w + 1e-7 for c, w in zip(q, (wx, wy, wz)))
                            strict = all(c == 0.0 or 1e-7 < c < w - 1e-7 for c, w in zip(q, (wx, wy, wz)))
                            if loose and not strict:
                                near += 1
                            if inside:
                                out.append([el, float(q[0]), float(q[1]), float(q[2]), float(site["occ"][e])])
    if near:
        raise AssertionError("an atom lies within rounding of a face of the box: choose other widths or tilts")
    return out, mins, maxs, [b.tolist() for b in basis]


def main():
    result = {}
    for name, case in CASES.items():
        lst, mins, maxs, basis = atoms(case)
        result[name] = {"cif": FILES[name], "uvw": case["uvw"], "abc": case["abc"], "widths": case["widths"],
                        "tilts": case["tilts"], "fractional_positions": [s["positions"] for s in case["sites"]],
                        "tile_min": mins, "tile_max": maxs, "basis": basis, "atoms": lst}
    with open(os.path.join(HERE, "expected.json"), "w") as f:
        json.dump(result, f, indent=1)
    for name, r in result.items():
        print(name, len(r["atoms"]), "atoms, tiles", r["tile_min"], r["tile_max"])


if __name__ == "__main__":
    main()

"""Make tests/golden/params.json from the reference's parameter tables.

Run where the clTEM sources are present (the path as the argument, else as oracle/build_ref.py finds it):
    python tests/golden/make_params_fixture.py [reference_root]
The tables (Kirkland, Peng, Lobato scattering-factor parameterisations) are the inputs the
multislice path reads at run time (src/simulation/utilities/stringutils.cpp:149-184); bundling them
lets the GPU tests and the benchmark run where the reference is not present.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cltem_b200.params import read_params  # noqa: E402

FORM_NAMES = {0: "kirkland", 1: "peng", 2: "lobato"}


def main():
    from oracle.build_ref import reference_root
    root = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    if root is None:
        raise SystemExit("reference tree not found: pass its path or set CLTEM_REFERENCE")
    out = {}
    for fn in ("kirkland.dat", "peng.dat", "lobato.dat"):
        p = read_params(os.path.join(root, "params", fn))
        out[p.name] = {"form": FORM_NAMES[p.form], "i_per_atom": p.i_per_atom,
                       "values": [float(v) for v in p.values], "source": "params/" + fn}
    with open(os.path.join(HERE, "params.json"), "w") as f:
        json.dump(out, f, indent=0)
    print({k: len(v["values"]) for k, v in out.items()})


if __name__ == "__main__":
    main()

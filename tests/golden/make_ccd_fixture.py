"""Make tests/golden/ccds.json from the reference's CCD tables.

Run where the clTEM sources are present (the path as the argument, else as oracle/build_ref.py finds it):
    python tests/golden/make_ccd_fixture.py [reference_root]
The tables (DQE and NTF of the K2 and Orius cameras, ccds/*.dat) are the inputs of clTEM's CTEM dose
simulation (src/simulation/microscope/simulationctem.cpp:88-108, 171-264); bundling them lets the tests
and the CLI run where the reference is not present.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cltem_b200.params import read_ccd  # noqa: E402


def main():
    from oracle.build_ref import reference_root
    root = reference_root(sys.argv[1] if len(sys.argv) > 1 else None)
    if root is None:
        raise SystemExit("reference tree not found: pass its path or set CLTEM_REFERENCE")
    out = {}
    for fn in sorted(os.listdir(os.path.join(root, "ccds"))):
        if fn.endswith(".dat"):
            c = read_ccd(os.path.join(root, "ccds", fn))
            out[fn[:-4]] = {"name": c.name, "dqe": [float(v) for v in c.dqe], "ntf": [float(v) for v in c.ntf],
                            "source": "ccds/" + fn}
    with open(os.path.join(HERE, "ccds.json"), "w") as f:
        json.dump(out, f, indent=0)
    print({k: (v["name"], len(v["dqe"]), len(v["ntf"])) for k, v in out.items()})


if __name__ == "__main__":
    main()

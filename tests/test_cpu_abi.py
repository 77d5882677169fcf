"""C ABI checks that need no GPU: the library loads, exports every entry point the header declares,
the ctypes mirror matches the C struct layouts, the host-only geometry matches the oracle bit for bit,
and compute calls fail loudly (no CPU fallback) when no device is present."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from cltem_b200 import abi, config, engine
from tests.cases import small_cbed, small_ctem, small_stem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mslice.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mslice_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mslice_ctx_create" in syms and "mslice_stem_run_staged" in syms
    assert len(syms) >= 25


def test_library_exports_every_declared_symbol():
    L = engine.load_library()
    for s in declared_symbols():
        assert hasattr(L, s), s
    assert L.mslice_version().startswith(b"mslice")


def test_struct_layouts_match_header():
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "mslice.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(mslice_config), sizeof(mslice_geometry),
         offsetof(mslice_config, detectors), offsetof(mslice_config, probe_batch),
         offsetof(mslice_geometry, crop), offsetof(mslice_geometry, n_outputs), sizeof(mslice_detector));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        exe = os.path.join(d, "p")
        open(c, "w").write(prog)
        subprocess.check_call([cc, "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    C = ctypes
    assert vals == [C.sizeof(abi.Config), C.sizeof(abi.Geometry), abi.Config.detectors.offset,
                    abi.Config.probe_batch.offset, abi.Geometry.crop.offset, abi.Geometry.n_outputs.offset,
                    C.sizeof(abi.Detector)]


@pytest.mark.parametrize("make", [lambda: small_stem()[0], lambda: small_ctem()[0], lambda: small_cbed()[0],
                                  lambda: config.perovskite_stem()[0], lambda: config.perovskite_ctem()[0],
                                  lambda: config.fcc_cbed()[0]])
def test_host_geometry_matches_oracle_exactly(oracle, make):
    s = make()
    g1 = engine.geometry(s.cfg)
    g2 = oracle.geometry(s.cfg)[0]
    assert abi.geometry_dict(g1) == abi.geometry_dict(g2)


def test_geometry_of_named_workloads():
    g = engine.geometry(config.perovskite_ctem()[0].cfg)
    assert g.n_slices == 20 and abs(g.real_scale - 19.525 / 256) < 1e-15
    g = engine.geometry(config.perovskite_stem()[0].cfg)
    assert g.n_slices == 40 and abs(g.real_scale - 0.05625) < 1e-15 and g.blocks_x == 4
    g = engine.geometry(config.fcc_cbed()[0].cfg)
    assert g.n_slices == 120 and g.blocks_x == 11


def test_geometry_rejects_bad_configs():
    s, _ = small_stem()
    s.cfg.resolution = 384     # not in clTEM's resolutionValid list ...
    with pytest.raises(engine.MsliceError) as e:
        engine.geometry(s.cfg)
    assert e.value.code == abi.ERR_ARG
    s.cfg.allow_any_resolution = 1   # ... unless the extension flag is set
    engine.geometry(s.cfg)
    s.cfg.slice_thickness = 0.0
    with pytest.raises(engine.MsliceError):
        engine.geometry(s.cfg)


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(engine.MsliceError) as e:
        engine.Context(0)
    assert e.value.code == abi.ERR_CUDA


def test_missing_library_fails_loudly(tmp_path):
    import importlib
    mod = importlib.import_module("cltem_b200.engine")
    saved = mod._lib
    try:
        mod._lib = None
        with pytest.raises(RuntimeError, match="no CPU fallback"):
            mod.load_library(str(tmp_path / "nope.so"))
    finally:
        mod._lib = saved

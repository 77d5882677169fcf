"""Command-line front end with clTEM_cmd's interface (src/console/main.cpp:43-73, 270-792).

    python -m cltem_b200 structure.xyz -c config.json -o outdir [-d device] [-p params_dir]

Reads the same JSON config and .xyz structure, runs the simulation on the GPU(s), and writes the same
outputs as clTEM_cmd's imageReturned (main.cpp:193-268): for CTEM EW_amplitude / EW_phase / Diff / Image,
for STEM one image per detector, for CBED Diff; float32 TIFFs (fileio.h:43-76) plus a settings JSON next to
each, and _NNN suffixes for intermediate-slice stacks (main.cpp:158-191).

Differences from clTEM_cmd, by design: OpenCL devices and math flags (-d platform:device, -f) do not apply
(-d takes CUDA device indices, "gpu"/"default" or "all"/"gpus"; -f is accepted and ignored); the
frozen-phonon, occupancy and incoherence draws take an explicit seed (--seed) instead of the wall clock.
A .cif structure takes the reference's supercell options: -s wx,wy,wz (Å) and -z u,v,w are required,
-n u,v,w (the lattice direction along x) and -t tx,ty,tz (degrees) are optional, --fix repairs common
file errors.
"""
import argparse
import copy
import json
import os
import sys
import threading
import time

import numpy as np

from . import abi
from .config import read_config
from .params import read_params, read_params_json, default_bundle_path
from .structure import frozen_phonon_configs, read_xyz
from .tiff import write_tiff

VERSION = "mslice-b200 CLI 1"


def _parse(argv):
    p = argparse.ArgumentParser(prog="cltem_b200", description="B200 multislice simulation (clTEM_cmd interface)")
    p.add_argument("structure", nargs="?")
    p.add_argument("-c", "--config")
    p.add_argument("-o", "--output")
    p.add_argument("-d", "--device", default="default")
    p.add_argument("-p", "--params", default=None, help="directory holding kirkland.dat / peng.dat / lobato.dat")
    p.add_argument("-f", "--flags", default="", help="accepted for compatibility; has no effect")
    p.add_argument("-l", "--list", action="store_true", help="list the CUDA devices and exit")
    p.add_argument("-v", "--version", action="store_true")
    p.add_argument("--seed", type=int, default=0, help="seed of the frozen-phonon and incoherence draws")
    p.add_argument("--ccds", default=None, help="directory holding the CCD tables <name>.dat named by ctem/ccd/name "
                                                "(default: the bundled K2 and Orius tables)")
    p.add_argument("--debug", action="store_true")
    p.add_argument("-s", "--size", default=None)
    p.add_argument("-z", "--zone", default=None)
    p.add_argument("-n", "--normal", default=None)
    p.add_argument("-t", "--tilts", default=None)
    p.add_argument("--fix", action="store_true")
    return p.parse_args(argv)


def _devices(spec):
    import torch
    n = torch.cuda.device_count()
    if n == 0:
        raise SystemExit("no CUDA device available")
    spec = spec.strip().lower()
    if spec in ("default", "gpu", ""):
        return [0]
    if spec in ("all", "gpus"):
        return list(range(n))
    if spec in ("cpu", "cpus"):
        raise SystemExit("this engine has no CPU device; use a GPU")
    out = []
    for tok in spec.split(","):
        tok = tok.split(":")[-1]
        d = int(tok)
        if d < 0 or d >= n:
            raise SystemExit(f"device {d} out of range (have {n})")
        out.append(d)
    return out


def _load_params(name, params_dir):
    if params_dir:
        for fn in sorted(os.listdir(params_dir)):
            if fn.endswith(".dat"):
                p = read_params(os.path.join(params_dir, fn))
                if p.name == name:
                    return p
        raise SystemExit(f"Could not find loaded parameters with name {name}")
    bundle = read_params_json(default_bundle_path())
    if name not in bundle:
        raise SystemExit(f"Could not find loaded parameters with name {name}")
    return bundle[name]


def _three(arg, what):
    """parseThreeCommaList (main.cpp:109-133): exactly three comma-separated numbers."""
    try:
        v = [float(t) for t in arg.split(",")]
    except ValueError:
        v = []
    if len(v) != 3:
        raise ValueError(f"Could not parse .cif {what} argument: {arg}")
    return tuple(v)


def _cif_info(a):
    """The supercell options of a .cif input (main.cpp:416-458): -s and -z required, -n and -t optional."""
    from .cif import SuperCellInfo
    errs = []
    if not a.size:
        errs.append(".cif files require a size arg (-s, --size)")
    if not a.zone:
        errs.append(".cif files require a zone axis arg (-z, --zone)")
    info = SuperCellInfo()
    for attr, arg, what in (("widths", a.size, "size"), ("uvw", a.zone, "zone"), ("abc", a.normal, "normal"),
                            ("tilts", a.tilts, "tilt")):
        if arg:
            try:
                setattr(info, attr, _three(arg, what))
            except ValueError as e:
                errs.append(str(e))
    return info, errs


def _load_ccd(name, ccds_dir):
    """The CCD named by ctem/ccd/name: <ccds_dir>/<name>.dat (CCDParams loaded from the executable's ccds
    folder, src/console/main.cpp:770-778), else the bundled tables (matched by file stem or by name)."""
    from .params import load_ccds, read_ccd
    if ccds_dir:
        return read_ccd(os.path.join(ccds_dir, name + ".dat"))
    for stem, c in load_ccds().items():
        if name in (stem, c.name):
            return c
    raise RuntimeError(f"unknown CCD {name!r}: give --ccds <dir> holding {name}.dat")


def _run_share(dev, settings, params, configs, out, idx, errors, cfg=None, passes=None, ccd=None):
    """Run a share on one device; store (sum of results, number of passes). Without `passes` the share is
    one pass per configuration; with it, `passes` incoherent passes over all the configurations (cfg
    carries the pass count and this device's seed)."""
    try:
        from .engine import Context, Simulation
        ctx = Context(dev)
        ctx.load_params(params)
        cfg = cfg if cfg is not None else settings.cfg
        sim = Simulation(ctx, cfg)
        mode = cfg.mode
        weight = passes if passes is not None else len(configs)
        if mode in (abi.MODE_STEM, abi.MODE_CBED):
            sim.stage(configs)
            sim.run_staged()
            r = sim.staged_result() * weight
            out[idx] = ({"main": r}, weight)
        else:
            if ccd is not None:
                sim.set_ccd(ccd, settings.ccd_binning, settings.ccd_dose)
            acc = None
            for c in configs:
                sim.set_atoms(c)
                ew, diff, img = sim.ctem()
                cur = {"EW": ew, "Diff": diff, "Image": img}
                acc = cur if acc is None else {k: acc[k] + cur[k] for k in acc}
            out[idx] = (acc, len(configs))
        sim.close()
        ctx.close()
    except Exception as e:  # noqa: BLE001
        errors.append(e)


def _save_stack(path_base, stack, settings_json, n_slices, interval):
    """saveTiffOutput (main.cpp:158-191): one file, or _NNN files for intermediate slices."""
    if path_base.endswith(".tif"):
        path_base = path_base[:-4]
    if stack.shape[0] > 1:
        if interval < 1:
            raise RuntimeError("Saving stack with < 0 slice step.")
        width = len(str(n_slices - 1))
        for i in range(stack.shape[0]):
            sid = min((i + 1) * interval - 1, n_slices - 1)
            write_tiff(f"{path_base}_{sid:0{width}d}.tif", stack[i])
    else:
        write_tiff(path_base + ".tif", stack[0])


def main(argv=None):
    a = _parse(argv)
    if a.version:
        print(VERSION)
        return 0
    if a.list:
        import torch
        for i in range(torch.cuda.device_count()):
            print(f"{i}: {torch.cuda.get_device_name(i)}")
        return 0
    if not a.structure or not a.config or not a.output:
        print("usage: python -m cltem_b200 structure_file -c config.json -o output_dir [-d device]", file=sys.stderr)
        return 1
    is_xyz, is_cif = a.structure.endswith(".xyz"), a.structure.endswith(".cif")
    if not is_xyz and not is_cif:
        print(f"Require a .xyz or .cif file non-option argument. Instead got: {a.structure}", file=sys.stderr)
        return 1
    if is_cif:
        info, errs = _cif_info(a)
        if errs:
            print("\n".join(errs), file=sys.stderr)
            return 1
    elif a.size or a.zone or a.normal or a.tilts:
        print("WARNING: .cif options have been set for .xyz file, these will be ignored", file=sys.stderr)
    with open(a.config) as f:
        raw = json.load(f)
    settings = read_config(raw)
    if is_cif:
        from .cif import read_cif_structure
        structure = read_cif_structure(a.structure, info, fix=a.fix, seed=a.seed)
    else:
        structure = read_xyz(a.structure, seed=a.seed)
    settings.attach_structure(structure)
    params = _load_params(settings.potentials, a.params)
    from .engine import geometry
    geo = geometry(settings.cfg)
    os.makedirs(a.output, exist_ok=True)

    # frozen phonon configurations (incoherence iterations; PhononScattering::generateTdsFactor). With
    # mixed static potentials the configurations are the sets and the iterations are passes drawing from
    # them; without phonons, chromatic / source-size iterations are passes over the one structure.
    iters = settings.effective_iterations()
    mixed = settings.cfg.mixed_static > 1
    settings.cfg.seed = a.seed
    by_pass = mixed or (not settings.phonon_enabled and iters > 1)
    n_conf = settings.cfg.mixed_static if mixed else (iters if settings.phonon_enabled else 1)
    settings.cfg.iterations = iters if by_pass else 0
    if settings.phonon_enabled:
        configs = frozen_phonon_configs(structure, n_conf, settings.vibrations, seed=a.seed)
    else:
        configs = [structure]

    ccd = None
    if settings.cfg.mode == abi.MODE_CTEM and settings.ccd_name not in ("", "Perfect"):
        ccd = _load_ccd(settings.ccd_name, a.ccds)
    devs = _devices(a.device)
    results, errors, threads = [None] * len(devs), [], []
    t0 = time.time()
    if by_pass and settings.cfg.mode in (abi.MODE_STEM, abi.MODE_CBED):
        # passes split over the devices; each device draws from its own seed
        for i, d in enumerate(devs):
            n_pass = iters // len(devs) + (1 if i < iters % len(devs) else 0)
            if n_pass == 0:
                continue
            cfg_i = copy.deepcopy(settings.cfg)
            cfg_i.iterations = n_pass
            cfg_i.seed = (a.seed + 0x9E3779B97F4A7C15 * i) % (1 << 64)
            th = threading.Thread(target=_run_share, args=(d, settings, params, configs, results, i, errors, cfg_i, n_pass))
            th.start()
            threads.append(th)
    else:
        shares = [configs[i::len(devs)] for i in range(len(devs))]
        for i, (d, sh) in enumerate(zip(devs, shares)):
            if not sh:
                continue
            cfg_i = copy.deepcopy(settings.cfg)   # own seed per device: dose noise draws differ between devices
            cfg_i.seed = (a.seed + 0x9E3779B97F4A7C15 * i) % (1 << 64)
            th = threading.Thread(target=_run_share, args=(d, settings, params, sh, results, i, errors, cfg_i, None, ccd))
            th.start()
            threads.append(th)
    for th in threads:
        th.join()
    if errors:
        raise errors[0]
    elapsed = time.time() - t0
    total = {}
    for r in results:
        if r is None:
            continue
        imgs, _ = r
        for k, v in imgs.items():
            total[k] = v if k not in total else total[k] + v
    weight = sum(r[1] for r in results if r is not None)
    total = {k: v / weight for k, v in total.items()}

    js = copy.deepcopy(raw)
    js["filename"] = os.path.abspath(a.structure)
    js["slice count"] = geo.n_slices
    js["simulation time"] = elapsed
    interval = settings.cfg.intermediate_slices
    sep = os.sep
    mode = settings.cfg.mode
    if mode == abi.MODE_STEM:
        r = total["main"]   # [n_out, n_det, py, px]
        for d, det in enumerate(settings.detectors):
            name = det[0]
            jd = copy.deepcopy(js)
            jd.get("microscope", {}).pop("alpha", None)
            jd.get("microscope", {}).pop("delta", None)
            with open(a.output + sep + name + ".json", "w") as f:
                json.dump(jd, f, indent=4)
            _save_stack(a.output + sep + name, r[:, d], jd, geo.n_slices, interval)
    elif mode == abi.MODE_CBED:
        jd = copy.deepcopy(js)
        for k in ("aberrations", "alpha", "delta", "objective aperture"):
            jd.get("microscope", {}).pop(k, None)
        with open(a.output + sep + "Diff.json", "w") as f:
            json.dump(jd, f, indent=4)
        _save_stack(a.output + sep + "Diff", total["main"], jd, geo.n_slices, interval)
    else:
        jd = copy.deepcopy(js)
        for k in ("aberrations", "alpha", "delta", "objective aperture"):
            jd.get("microscope", {}).pop(k, None)
        ew = total["EW"]
        for nm, arr in (("EW_amplitude", np.abs(ew)), ("EW_phase", np.angle(ew))):
            with open(a.output + sep + nm + ".json", "w") as f:
                json.dump(jd, f, indent=4)
            _save_stack(a.output + sep + nm, arr, jd, geo.n_slices, interval)
        with open(a.output + sep + "Diff.json", "w") as f:
            json.dump(jd, f, indent=4)
        _save_stack(a.output + sep + "Diff", total["Diff"], jd, geo.n_slices, interval)
        if settings.cfg.ctem_image:
            with open(a.output + sep + "Image.json", "w") as f:
                json.dump(js, f, indent=4)
            _save_stack(a.output + sep + "Image", total["Image"], js, geo.n_slices, interval)
    print(f"simulation finished in {elapsed:.2f} s -> {a.output}")
    return 0


if __name__ == "__main__":
    sys.exit(main())

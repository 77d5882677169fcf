"""torch autograd for the differentiable CTEM image loss.

ctem_image_loss(sim, Z, xyz, lens, target) returns L = sum (I - target)^2 as a 0-d tensor whose backward
runs the engine's hand-written adjoint (mslice_ctem_loss_grad). The autograd Function lives in libtorch C++
(cltem_b200/torch_ext/ctem_loss_op.cpp), compiled in-tree against libmslice.so by build_extension().
"""
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
EXT_DIR = os.path.join(HERE, "torch_ext")
_mod = None


def build_extension(verbose=False):
    """Compile (or load the already compiled) libtorch extension into cltem_b200/torch_ext/."""
    global _mod
    if _mod is not None:
        return _mod
    from torch.utils.cpp_extension import load
    os.makedirs(os.path.join(EXT_DIR, "build"), exist_ok=True)
    _mod = load(name="mslice_torch", sources=[os.path.join(EXT_DIR, "ctem_loss_op.cpp")],
                build_directory=os.path.join(EXT_DIR, "build"),
                extra_cflags=["-O2"], extra_ldflags=[os.path.join(HERE, "libmslice.so"), "-Wl,-rpath," + HERE],
                verbose=verbose)
    return _mod


def ctem_image_loss(sim, Z, xyz, lens, target, checkpoint_every=0):
    """sim: cltem_b200.engine.Simulation (CTEM); Z: int tensor [n]; xyz: float64 tensor [n, 3];
    lens: float64 tensor [2] = (C10, C30) in Å; target: float64 [res, res]."""
    m = build_extension()
    return m.ctem_image_loss(xyz, lens, int(sim.h.value), torch.as_tensor(Z), torch.as_tensor(target), int(checkpoint_every))

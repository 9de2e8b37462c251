"""The differentiable rollout as a torch autograd function.

`flock_loss` is implemented in C++ (csrc/torch_adjoint.cpp) as a
torch::autograd::Function over the C-ABI: its forward is brt_adjoint_forward
(taped rollout, FP64 per-flock loss) and its backward the CUDA adjoint
brt_adjoint_backward.  No reference counterpart.
"""
from __future__ import annotations

import importlib.util

from .build import torch_ext_path

_EXT = None


def _ext():
    global _EXT
    if _EXT is None:
        import torch  # noqa: F401  (loads libtorch before the extension)
        from . import _abi
        _abi.lib()  # the CUDA library must be built; there is no CPU fallback
        path = torch_ext_path()
        if not path.exists():
            raise RuntimeError("the torch extension is not built (run `python -m behavert_b200.build`)")
        spec = importlib.util.spec_from_file_location("_brt_torch", str(path))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _EXT = mod
    return _EXT


def flock_loss(engine, weights, pos0, vel0, target, dt: float, nsteps: int, checkpoint_every: int = 10):
    """Per-flock FP64 loss mean_i |minimum image(p_i(T) - target_i)|^2 of a
    rollout of `engine` from (pos0, vel0) with per-flock steering weights.

    weights: [nflocks, 3] float32 CUDA; pos0, vel0, target: [N, 3] float32
    CUDA in agent-id order.  Differentiable in weights, pos0 and vel0; the
    backward recomputes every checkpoint segment (hash, sort, neighbour
    lists) and runs the hand-written adjoint kernel.
    """
    return _ext().flock_loss(int(engine.handle.value), weights, pos0, vel0, target, float(dt), int(nsteps),
                             int(checkpoint_every))

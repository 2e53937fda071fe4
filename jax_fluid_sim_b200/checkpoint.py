"""Restart files in the reference driver's format (run_hybrid_sphere.py:36-45 writes them,
:123-131 reads them): one compressed npz with ``time``, ``step`` and ``U_<element type>`` arrays
of shape (E, Np, nvars), float64, in the reference's node order.

The states live on the GPU here.  ``save_restart`` copies every block to pinned host memory
with asynchronous copies on the current stream, waits once, and writes the file through a
temporary name that replaces the target at the end (a reader never sees a half-written file).
``load_restart`` reads the file and copies the blocks into the caller's existing device buffers
when given (``into=``), so pointers stay the same and a step replayed as a CUDA graph can go on
without a new capture; otherwise it allocates new device tensors.
"""

from pathlib import Path

import numpy as np
import torch


def _host_copies(states):
    out, on_device = {}, False
    for name, value in states.items():
        t = value if isinstance(value, torch.Tensor) else torch.as_tensor(np.asarray(value))
        if t.device.type == "cuda":
            h = torch.empty(t.shape, dtype=torch.float64, pin_memory=True)
            h.copy_(t, non_blocking=True)
            out[name] = h
            on_device = True
        else:
            out[name] = t.to(torch.float64)
    if on_device:
        torch.cuda.current_stream().synchronize()
    return {k: v.numpy() for k, v in out.items()}


def save_restart(path, states, current_time, step):
    """Write ``states`` ({element_type: (E, Np, nvars)}, device or host) with the time and step."""
    path = Path(path)
    host = _host_copies(states)
    temporary = path.with_name(path.stem + ".tmp.npz")
    np.savez_compressed(temporary, time=np.asarray(float(current_time)), step=np.asarray(int(step)),
                        **{f"U_{name}": value for name, value in host.items()})
    temporary.replace(path)


def load_restart(path, element_types=None, into=None, device="cuda"):
    """Read a restart file; returns (states, time, step).

    ``element_types``: the blocks to read (default: every ``U_*`` array in the file); a missing
    block raises ``KeyError`` as the reference's loader does.  ``into``: existing tensors
    {element_type: tensor} to fill in place (shapes must match); the copies are asynchronous on
    the current stream from pinned staging buffers, which are kept alive until one synchronisation
    of the stream after the last block.
    """
    with np.load(Path(path)) as restart:
        names = element_types if element_types is not None else [k[2:] for k in restart.files if k.startswith("U_")]
        arrays = {name: np.asarray(restart[f"U_{name}"], dtype=np.float64) for name in names}
        current_time = float(restart["time"])
        step = int(restart["step"]) if "step" in restart.files else 0
    for name, a in arrays.items():
        if into is not None and name in into and tuple(into[name].shape) != a.shape:
            raise ValueError(f"U_{name} has shape {a.shape}; the buffer has {tuple(into[name].shape)}")
    states = {}
    staging = []
    for name, a in arrays.items():
        if into is not None and name in into:
            dst = into[name]
            if dst.device.type == "cuda":
                pinned = torch.from_numpy(a).pin_memory()
                dst.copy_(pinned, non_blocking=True)
                staging.append(pinned)
            else:
                dst.copy_(torch.from_numpy(a))
            states[name] = dst
        else:
            states[name] = torch.as_tensor(a, device=device)
    if staging:
        # one wait for all blocks' copies; the pinned buffers live until then
        torch.cuda.current_stream().synchronize()
    return states, current_time, step

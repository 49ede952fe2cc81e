"""Raw binary state dumps of (u, uRec): the hand-off of a solver state between runs, and to the CPU oracle.

The reference writes its restart through the H5/JSON serialisers (EulerSolver_PrintData.hxx:886-1073
PrintRestart / ReadRestart, src/DNDS/Serializer/); the image has no HDF5 library, and the hot path only needs
the two state arrays.  A dump is two files: ``<path>`` holds u [nCell][nVars] and then uRec
[nCell][R][nVars], little-endian float64, C order, nothing between them; ``<path>.json`` holds the shapes,
the byte offsets and the caller's metadata (step, time, settings ...).  Loading gives back the same bits.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

FORMAT = "dndsb-state-1"


def save_state(path: str, u, uRec, **meta) -> None:
    """Writes u and uRec (torch tensors on any device, or numpy arrays) and a JSON header with ``meta``."""
    a = u.detach().cpu().numpy() if torch.is_tensor(u) else np.asarray(u)
    b = uRec.detach().cpu().numpy() if torch.is_tensor(uRec) else np.asarray(uRec)
    if a.dtype != np.float64 or b.dtype != np.float64:
        raise ValueError("save_state: u and uRec must be float64")
    if a.ndim != 2 or b.ndim != 3 or b.shape[0] != a.shape[0] or b.shape[2] != a.shape[1]:
        raise ValueError(f"save_state: shapes {a.shape} and {b.shape} are not [nCell][nVars] and [nCell][R][nVars]")
    header = {"format": FORMAT, "byteorder": "little", "dtype": "float64", "u": {"shape": list(a.shape), "offset": 0},
              "uRec": {"shape": list(b.shape), "offset": a.size * 8}, "meta": meta}
    tmp = path + ".part"
    with open(tmp, "wb") as fh:
        fh.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        fh.write(np.ascontiguousarray(b, dtype="<f8").tobytes())
    with open(path + ".json", "w") as fh:
        json.dump(header, fh, indent=1)
    os.replace(tmp, path)


def load_state(path: str, device=None):
    """(u, uRec, meta) from a dump: numpy arrays for ``device=None``, else torch tensors on ``device``."""
    with open(path + ".json") as fh:
        header = json.load(fh)
    if header.get("format") != FORMAT:
        raise ValueError(f"load_state: {path} is not a {FORMAT} dump")
    raw = np.fromfile(path, dtype="<f8")
    nu = int(np.prod(header["u"]["shape"]))
    nr = int(np.prod(header["uRec"]["shape"]))
    if raw.size != nu + nr:
        raise ValueError(f"load_state: {path} holds {raw.size} values, the header {nu + nr}")
    a = raw[:nu].reshape(header["u"]["shape"]).astype(np.float64)
    b = raw[nu:].reshape(header["uRec"]["shape"]).astype(np.float64)
    if device is None:
        return a, b, header["meta"]
    return torch.from_numpy(a).to(device), torch.from_numpy(b).to(device), header["meta"]

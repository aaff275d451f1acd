"""Helpers shared by the GPU parity tests."""
import numpy as np

import oracle as O
import pyg

I32, I64 = pyg.INT32, pyg.INT64


def struct(cols, types):
    dt = O.dtype_of(types)
    a = np.empty(len(cols[0]), dtype=dt)
    for i, c in enumerate(cols):
        a[f"c{i}"] = c
    return a


def to_device(torch, arr):
    """Copies a packed numpy array to a CUDA uint8 tensor (16-B aligned)."""
    raw = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    t = torch.empty(max(raw.shape[0], 16), dtype=torch.uint8, device="cuda")
    if raw.shape[0]:
        t[: raw.shape[0]].copy_(torch.from_numpy(raw))
    return t


def dev_rel(torch, arr, types):
    t = to_device(torch, arr)
    offs = [arr.dtype.fields[f"c{i}"][1] for i in range(len(types))]
    return pyg.Rel(t, arr.shape[0], types, tuple_bytes=arr.dtype.itemsize, offsets=offs)


def host_rel(arr, types):
    arr = np.ascontiguousarray(arr)
    offs = [arr.dtype.fields[f"c{i}"][1] for i in range(len(types))]
    return pyg.Rel(arr, arr.shape[0], types, tuple_bytes=arr.dtype.itemsize, offsets=offs, on_device=0)


def from_device(torch, t, n, dtype):
    nbytes = n * dtype.itemsize
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return t[:nbytes].cpu().numpy().view(dtype).copy()


def alloc(torch, nbytes):
    return torch.zeros(max(nbytes, 16), dtype=torch.uint8, device="cuda")


def rows(a):
    return [tuple(int(x) for x in r) for r in a.tolist()]


def canon_rows(a):
    return rows(O.canonical(a))

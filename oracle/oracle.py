"""ctypes binding of the C oracle (oracle/pyg_oracle.c -> oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product path never uses it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "pyg_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")

INT32, INT64 = 1, 2


class orc_rel(C.Structure):
    _fields_ = [("base", C.c_void_p), ("ntuples", C.c_int64), ("tuple_bytes", C.c_int32), ("ncols", C.c_int32),
                ("col_offset", C.c_int32 * 8), ("col_type", C.c_int32 * 8)]


class orc_proj(C.Structure):
    _fields_ = [("side", C.c_int32), ("col", C.c_int32)]


def build():
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB, SRC])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64
        R = C.POINTER(orc_rel)
        L.orc_hashjoin_agg.argtypes = [R, P, R, P, C.c_int, C.POINTER(orc_proj), C.c_int, C.c_uint, C.c_int, P, P]
        L.orc_hashjoin_materialize.argtypes = [R, P, R, P, C.c_int, C.POINTER(orc_proj), C.c_int, C.c_uint, C.c_int,
                                               P, I64, P]
        L.orc_hashjoin_materialize.restype = I64
        L.orc_groupby.argtypes = [R, P, C.c_int, C.c_int, C.c_int, C.c_uint, C.c_int, P, I64]
        L.orc_groupby.restype = I64
        L.orc_partition.argtypes = [R, C.c_int, C.c_int, C.c_uint, I64, I64, P, P, P]
        L.orc_sort.argtypes = [R, C.c_int, P]
        L.orc_mpsm_join.argtypes = [R, C.c_int, R, C.c_int, C.POINTER(orc_proj), C.c_int, P, I64, P, P]
        L.orc_mpsm_join.restype = I64
        L.orc_sortlimit.argtypes = [R, P, C.c_int, C.c_int, I64, P]
        L.orc_sortlimit.restype = I64
        L.orc_exactrange_bucket.argtypes = [I64, I64, I64, C.c_uint]
        L.orc_exactrange_min_for_bucket.argtypes = [C.c_uint, I64, I64, C.c_uint]
        L.orc_exactrange_min_for_bucket.restype = I64
        _lib = L
    return _lib


def dtype_of(types):
    return np.dtype([(f"c{i}", np.int32 if t == INT32 else np.int64) for i, t in enumerate(types)])


def as_struct(arr, types):
    """Views a 2-D int64 array or a structured array as packed tuples."""
    dt = dtype_of(types)
    if arr.dtype == dt:
        return np.ascontiguousarray(arr)
    out = np.empty(arr.shape[0], dtype=dt)
    for i in range(len(types)):
        out[f"c{i}"] = arr[:, i]
    return out


def _rel(a, types):
    r = orc_rel()
    r.base = a.ctypes.data
    r.ntuples = a.shape[0]
    r.tuple_bytes = a.dtype.itemsize
    r.ncols = len(types)
    for i, t in enumerate(types):
        r.col_offset[i] = a.dtype.fields[f"c{i}"][1]
        r.col_type[i] = t
    return r


def _projs(proj):
    return (orc_proj * max(1, len(proj)))(*[orc_proj(s, c) for s, c in proj])


def hashjoin_agg(R, rtypes, rk, S, stypes, sk, proj, buckets=1 << 16, bytes_hash=False):
    rk = (C.c_int * len(rk))(*rk)
    sk = (C.c_int * len(sk))(*sk)
    cnt = C.c_int64()
    sums = (C.c_int64 * 16)()
    rc = lib().orc_hashjoin_agg(C.byref(_rel(R, rtypes)), rk, C.byref(_rel(S, stypes)), sk, len(rk), _projs(proj),
                                len(proj), buckets, int(bytes_hash), C.byref(cnt), sums)
    assert rc == 0
    return cnt.value, [sums[i] for i in range(len(proj))]


def proj_dtype(rtypes, stypes, proj):
    return dtype_of([(stypes if s else rtypes)[c] for s, c in proj])


def hashjoin_materialize(R, rtypes, rk, S, stypes, sk, proj, buckets=1 << 16, bytes_hash=False):
    rk_ = (C.c_int * len(rk))(*rk)
    sk_ = (C.c_int * len(sk))(*sk)
    dt = proj_dtype(rtypes, stypes, proj)
    need = C.c_int64()
    lib().orc_hashjoin_materialize(C.byref(_rel(R, rtypes)), rk_, C.byref(_rel(S, stypes)), sk_, len(rk),
                                   _projs(proj), len(proj), buckets, int(bytes_hash), None, 0, C.byref(need))
    out = np.zeros(need.value, dtype=dt)
    n = lib().orc_hashjoin_materialize(C.byref(_rel(R, rtypes)), rk_, C.byref(_rel(S, stypes)), sk_, len(rk),
                                       _projs(proj), len(proj), buckets, int(bytes_hash), out.ctypes.data,
                                       need.value, C.byref(need))
    assert n == need.value
    return out


def groupby_dtype(types, key_cols, flags, sum_col):
    cols = [types[k] for k in key_cols]
    if flags & 1:
        cols.append(types[sum_col])
    if flags & 2:
        cols.append(INT64)
    return dtype_of(cols)


def groupby(A, types, key_cols, flags, sum_col=0, buckets=1 << 16, bytes_hash=False, sort=True):
    kc = (C.c_int * max(1, len(key_cols)))(*key_cols)
    dt = groupby_dtype(types, key_cols, flags, sum_col)
    out = np.zeros(max(1, A.shape[0]), dtype=dt)
    ng = lib().orc_groupby(C.byref(_rel(A, types)), kc, len(key_cols), flags, sum_col, buckets, int(bytes_hash),
                           out.ctypes.data, out.shape[0])
    assert ng >= 0
    out = out[:ng]
    if sort and len(key_cols):
        out = np.sort(out, order=[f"c{i}" for i in range(len(key_cols))], kind="stable")
    return out


def partition(A, types, key_col, kind, fanout, mn=0, mx=0, splitters=None):
    out = np.zeros_like(A)
    offs = np.zeros(fanout + 1, dtype=np.int64)
    sp = None if splitters is None else np.ascontiguousarray(splitters, dtype=np.int64)
    rc = lib().orc_partition(C.byref(_rel(A, types)), key_col, kind, fanout, mn, mx,
                             None if sp is None else sp.ctypes.data, out.ctypes.data, offs.ctypes.data)
    if rc != 0:
        raise ValueError("key outside exactrange")
    return out, offs


def sort(A, types, key_col):
    out = np.zeros_like(A)
    assert lib().orc_sort(C.byref(_rel(A, types)), key_col, out.ctypes.data) == 0
    return out


def mpsm_join(R, rtypes, rk, S, stypes, sk, proj, materialize=False):
    cnt = C.c_int64()
    sums = (C.c_int64 * 16)()
    n = lib().orc_mpsm_join(C.byref(_rel(R, rtypes)), rk, C.byref(_rel(S, stypes)), sk, _projs(proj), len(proj),
                            None, 0, C.byref(cnt), sums)
    if not materialize:
        return cnt.value, [sums[i] for i in range(len(proj))]
    dt = proj_dtype(rtypes, stypes, proj)
    out = np.zeros(cnt.value, dtype=dt)
    lib().orc_mpsm_join(C.byref(_rel(R, rtypes)), rk, C.byref(_rel(S, stypes)), sk, _projs(proj), len(proj),
                        out.ctypes.data, cnt.value, None, None)
    return out


def sortlimit(A, types, by, asc, limit):
    """The first `limit` tuples of A in SortLimit order (stable)."""
    b = (C.c_int * max(1, len(by)))(*by)
    out = np.zeros(max(0, min(limit, A.shape[0])), dtype=A.dtype)
    n = lib().orc_sortlimit(C.byref(_rel(A, types)), b, len(by), int(bool(asc)), limit,
                            out.ctypes.data if out.shape[0] else None)
    return out[:n]


def exactrange_bucket(v, mn, mx, k):
    return lib().orc_exactrange_bucket(v, mn, mx, k)


def exactrange_min_for_bucket(b, mn, mx, k):
    return lib().orc_exactrange_min_for_bucket(b, mn, mx, k)


def canonical(rows):
    """Rows sorted by every column (a multiset comparison key)."""
    names = list(rows.dtype.names)
    return np.sort(rows, order=names, kind="stable")

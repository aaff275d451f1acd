"""ctypes binding of libpyg.so (include/pyg.h) for tests, bench and tools.

The library is the product; this module only marshals arguments.  It loads
the in-tree libpyg.so and raises if it is missing or if no B200 is present:
there is no CPU fallback.

Relations are described by `Rel` (packed row-major tuples, as a reference
TupleBuffer page).  Device buffers may be torch CUDA tensors or `DevBuf`
objects from `Ctx.alloc`.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyg.so")

PYG_OK = 0
PYG_ERR_ARG = -1
PYG_ERR_OOM = -2
PYG_ERR_CUDA = -3
PYG_ERR_TABLE_FULL = -4
PYG_ERR_TIMEOUT = -5
PYG_ERR_CAPACITY = -6
PYG_ERR_NO_DEVICE = -7

INT32 = 1
INT64 = 2
MAX_COLS = 8

HT_AGGREGATE = 1
HT_MATERIALIZE = 2
AGG_SUM = 1
AGG_COUNT = 2

SPLIT_EXACTRANGE = 0
SPLIT_SPLITTERS = 1
SPLIT_RADIX = 2
SPLIT_HASH = 3

JOIN_AUTO = 0
JOIN_DIRECT = 1
JOIN_RADIX = 2

# Largest build side of pyg_hashjoin_agg_noalloc (PYG_NOALLOC_MAX_BUILD).
NOALLOC_MAX_BUILD = 1 << 18

MPSM_EXACTRANGE = 0
MPSM_SAMPLED = 1
MPSM_LEARNED = 2


class PygError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pyg error {code}: {msg}")
        self.code = code


class pyg_rel(C.Structure):
    _fields_ = [("base", C.c_void_p), ("ntuples", C.c_int64), ("tuple_bytes", C.c_int32), ("ncols", C.c_int32),
                ("col_offset", C.c_int32 * MAX_COLS), ("col_type", C.c_int32 * MAX_COLS),
                ("on_device", C.c_int32), ("reserved", C.c_int32)]


class pyg_proj(C.Structure):
    _fields_ = [("side", C.c_int32), ("col", C.c_int32)]


class pyg_join_result(C.Structure):
    _fields_ = [("count", C.c_int64), ("sums", C.c_int64 * MAX_COLS)]


class pyg_join_opts(C.Structure):
    _fields_ = [("algorithm", C.c_int32), ("radix_bits", C.c_int32), ("load_factor", C.c_float),
                ("reserved", C.c_int32)]


class pyg_join_stats(C.Structure):
    _fields_ = [("algorithm", C.c_int32), ("radix_bits", C.c_int32), ("build_partition_ms", C.c_double),
                ("build_ms", C.c_double), ("probe_partition_ms", C.c_double), ("probe_ms", C.c_double), ("overflow_tuples", C.c_int64),
                ("padded_tuples", C.c_int64), ("histogram_ms", C.c_double), ("histogram_tuples", C.c_int64),
                ("build_pass_ms", C.c_double * 2), ("probe_pass_ms", C.c_double * 2), ("build_packed", C.c_int32),
                ("probe_packed", C.c_int32), ("join_kernel_ms", C.c_double)]


class pyg_splitter(C.Structure):
    _fields_ = [("kind", C.c_int32), ("fanout", C.c_int32), ("range_min", C.c_int64), ("range_max", C.c_int64),
                ("splitters", C.POINTER(C.c_int64))]


class pyg_mpsm_opts(C.Structure):
    _fields_ = [("splitter_kind", C.c_int32), ("fanout", C.c_int32), ("sample_rate", C.c_double),
                ("cdf_leaves", C.c_int32), ("page_tuples", C.c_int32), ("seed", C.c_uint64)]


class pyg_mpsm_stats(C.Structure):
    _fields_ = [("max_partition_imbalance", C.c_double), ("max_partition", C.c_int64), ("splitter_ms", C.c_double),
                ("partition_ms", C.c_double), ("sort_ms", C.c_double), ("merge_ms", C.c_double)]


class pyg_cdf_train_opts(C.Structure):
    _fields_ = [("leaves", C.c_int32), ("epochs", C.c_int32), ("lr", C.c_float), ("seed", C.c_uint64)]


class pyg_fragment(C.Structure):
    _fields_ = [("build", C.c_void_p), ("nbuild", C.c_int64), ("probe", C.c_void_p), ("nprobe", C.c_int64)]


class pyg_tuning(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("blocks_per_sm", C.c_int32), ("load_factor", C.c_float),
                ("chunk_tuples", C.c_int32), ("large_build", C.c_int32)]


_lib = None

# (name, restype, argtypes) of every exported entry point in include/pyg.h.
_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)
SIGNATURES = [
    ("pyg_ctx_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("pyg_ctx_destroy", C.c_int, [_P]),
    ("pyg_ctx_set_stream", C.c_int, [_P, _P]),
    ("pyg_ctx_stream", _P, [_P]),
    ("pyg_ctx_sync", C.c_int, [_P]),
    ("pyg_ctx_kernel_launches", _I64, [_P]),
    ("pyg_last_error", C.c_char_p, []),
    ("pyg_version", C.c_char_p, []),
    ("pyg_alloc", C.c_int, [_P, C.c_size_t, C.POINTER(_P)]),
    ("pyg_free", C.c_int, [_P, _P]),
    ("pyg_host_alloc", C.c_int, [C.c_size_t, C.POINTER(_P)]),
    ("pyg_host_free", C.c_int, [_P]),
    ("pyg_memcpy_h2d", C.c_int, [_P, _P, _P, C.c_size_t]),
    ("pyg_memcpy_d2h", C.c_int, [_P, _P, _P, C.c_size_t]),
    ("pyg_memcpy_d2d", C.c_int, [_P, _P, _P, C.c_size_t]),
    ("pyg_upload_open", C.c_int, [_P, C.c_size_t, C.c_size_t, _I32, C.POINTER(_P)]),
    ("pyg_upload_slot", C.c_int, [_P, _P, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    ("pyg_upload_commit", C.c_int, [_P, _P, C.c_size_t]),
    ("pyg_upload_finish", C.c_int, [_P, _P, C.POINTER(_P), C.POINTER(C.c_size_t)]),
    ("pyg_upload_abort", C.c_int, [_P, _P]),
    ("pyg_hashjoin_build", C.c_int, [_P, C.POINTER(pyg_rel), _PI32, _I32, _PI32, _I32, _I32, C.c_float, C.POINTER(_P)]),
    ("pyg_hashtable_free", C.c_int, [_P, _P]),
    ("pyg_hashtable_stats", C.c_int, [_P, _P, _PI64, _PI64, _PI32]),
    ("pyg_hashjoin_probe_agg", C.c_int, [_P, _P, C.POINTER(pyg_rel), _PI32, C.POINTER(pyg_proj), _I32,
                                         C.POINTER(pyg_join_result)]),
    ("pyg_hashjoin_probe_materialize", C.c_int, [_P, _P, C.POINTER(pyg_rel), _PI32, C.POINTER(pyg_proj), _I32, _P,
                                                 _I64, _PI64]),
    ("pyg_hashjoin_agg", C.c_int, [_P, C.POINTER(pyg_rel), _PI32, C.POINTER(pyg_rel), _PI32, _I32, C.POINTER(pyg_proj),
                                   _I32, C.POINTER(pyg_join_opts), C.POINTER(pyg_join_result),
                                   C.POINTER(pyg_join_stats)]),
    ("pyg_hashjoin_agg_noalloc", C.c_int, [_P, _I64, _P, _I64, _P, _P]),
    ("pyg_groupby", C.c_int, [_P, C.POINTER(pyg_rel), _PI32, _I32, _I32, _I32, _I32, _I64, _P, _I64, _PI64]),
    ("pyg_partition", C.c_int, [_P, C.POINTER(pyg_rel), _I32, C.POINTER(pyg_splitter), _P, _PI64]),
    ("pyg_sort", C.c_int, [_P, C.POINTER(pyg_rel), _I32, _P]),
    ("pyg_lower_bound", C.c_int, [_P, C.POINTER(pyg_rel), _I32, _P, _I64, _P]),
    ("pyg_sortlimit", C.c_int, [_P, C.POINTER(pyg_rel), _PI32, _I32, _I32, _I64, _P, _I64, _PI64]),
    ("pyg_bitonic_sort", C.c_int, [_P, _P, _I64]),
    ("pyg_mpsm_join_agg", C.c_int, [_P, C.POINTER(pyg_rel), _I32, C.POINTER(pyg_rel), _I32, C.POINTER(pyg_proj), _I32,
                                    C.POINTER(pyg_mpsm_opts), C.POINTER(pyg_join_result), C.POINTER(pyg_mpsm_stats)]),
    ("pyg_mpsm_join_materialize", C.c_int, [_P, C.POINTER(pyg_rel), _I32, C.POINTER(pyg_rel), _I32,
                                            C.POINTER(pyg_proj), _I32, C.POINTER(pyg_mpsm_opts), _P, _I64, _PI64]),
    ("pyg_cdf_train", C.c_int, [_P, _P, _I64, C.POINTER(pyg_cdf_train_opts), C.POINTER(_P)]),
    ("pyg_cdf_free", C.c_int, [_P, _P]),
    ("pyg_cdf_splitters", C.c_int, [_P, _P, _I32, _PI64]),
    ("pyg_cdf_predict", C.c_int, [_P, _P, _P, _I64, _P]),
    ("pyg_cdf_bins", C.c_int, [_P, _P, _I32, _P, _I64, _P]),
    ("pyg_cdf_bin_splitters", C.c_int, [_P, _P, _I32, C.POINTER(C.c_int64)]),
    ("pyg_cdf_params", C.c_int, [_P, _P, C.POINTER(C.c_float), _I32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("pyg_cdf_loss_grad", C.c_int, [_P, _P, _I64, _I32, C.POINTER(C.c_float), C.c_double, C.c_double,
                                    C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    ("pyg_sampled_splitters", C.c_int, [_P, _P, _I64, _I32, _PI64]),
    ("pyg_cdf_estimate_distinct", C.c_int, [_P, _P, _I64, _PI64]),
    ("pyg_batch_create", C.c_int, [_P, C.POINTER(pyg_fragment), _I32, C.POINTER(pyg_tuning), C.POINTER(_P)]),
    ("pyg_batch_run", C.c_int, [_P, _P, _PI64, _PI64, C.POINTER(C.c_double)]),
    ("pyg_batch_free", C.c_int, [_P, _P]),
    ("pyg_batch_run_plain", C.c_int, [_P, C.POINTER(pyg_fragment), _I32, _PI64, _PI64, C.POINTER(C.c_double)]),
    ("pyg_batch_inject_stall", C.c_int, [_P, _P, _I32]),
    ("pyg_autotune", C.c_int, [_P, C.POINTER(pyg_fragment), _I32, C.c_char_p, C.POINTER(pyg_tuning)]),
    ("pyg_gen_pk", C.c_int, [_P, _P, _I64, _I64, C.c_uint64]),
    ("pyg_gen_fk", C.c_int, [_P, _P, _I64, _I64, C.c_double, C.c_uint64, _I64, C.c_uint64]),
]


def lib():
    """Loads libpyg.so (raises if it is missing; never falls back)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run pythia-core_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            if not hasattr(L, name):
                continue
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != PYG_OK:
        raise PygError(rc, lib().pyg_last_error().decode())
    return rc


def _ptr(x):
    """Device/host address of a torch tensor, numpy array, DevBuf or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ptr"):
        return x.ptr
    raise TypeError(type(x))


def _on_device(x):
    if isinstance(x, np.ndarray):
        return 0
    if hasattr(x, "is_cuda"):
        return 1 if x.is_cuda else 0
    if isinstance(x, DevBuf):
        return 1
    if isinstance(x, HostBuf):
        return 0
    raise TypeError(type(x))


class Rel:
    """A relation: buffer + column layout (types PYG_INT32 / PYG_INT64)."""

    def __init__(self, buf, ntuples, types, tuple_bytes=None, on_device=None, offsets=None):
        self.buf = buf  # keeps the buffer alive
        self.types = list(types)
        if offsets is None:
            offsets, o = [], 0
            for t in self.types:
                offsets.append(o)
                o += 4 if t == INT32 else 8
            tb = o
        else:
            tb = tuple_bytes
        self.offsets = list(offsets)
        self.tuple_bytes = tuple_bytes or tb
        self.ntuples = int(ntuples)
        self.on_device = _on_device(buf) if on_device is None else on_device

    def c(self):
        r = pyg_rel()
        r.base = _ptr(self.buf)
        r.ntuples = self.ntuples
        r.tuple_bytes = self.tuple_bytes
        r.ncols = len(self.types)
        for i, (o, t) in enumerate(zip(self.offsets, self.types)):
            r.col_offset[i] = o
            r.col_type[i] = t
        r.on_device = self.on_device
        return r


def structured_dtype(types):
    return np.dtype([(f"c{i}", np.int32 if t == INT32 else np.int64) for i, t in enumerate(types)])


def host_rel(arr, types):
    """Rel over a host numpy structured or 2-D int64 array."""
    arr = np.ascontiguousarray(arr)
    n = arr.shape[0]
    return Rel(arr, n, types)


class DevBuf:
    def __init__(self, ctx, nbytes, adopt=None):
        self.ctx = ctx
        self.nbytes = nbytes
        if adopt is not None:  # take ownership of a pyg_alloc'd pointer
            self.ptr = adopt
            return
        p = C.c_void_p()
        check(lib().pyg_alloc(ctx.h, nbytes, C.byref(p)))
        self.ptr = p.value

    def free(self):
        if self.ptr:
            lib().pyg_free(self.ctx.h, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class HostBuf:
    """Pinned host memory exposed as a numpy uint8 array (.np)."""

    def __init__(self, nbytes):
        p = C.c_void_p()
        check(lib().pyg_host_alloc(nbytes, C.byref(p)))
        self.ptr = p.value
        self.nbytes = nbytes
        self.np = np.ctypeslib.as_array((C.c_uint8 * max(nbytes, 1)).from_address(self.ptr))[:nbytes]

    def free(self):
        if self.ptr:
            lib().pyg_host_free(self.ptr)
            self.ptr = None


class Ctx:
    def __init__(self, device=0, use_torch_stream=True):
        L = lib()
        h = C.c_void_p()
        check(L.pyg_ctx_create(device, C.byref(h)))
        self.h = h.value
        if use_torch_stream:
            try:
                import torch
                if torch.cuda.is_available():
                    handle = torch.cuda.current_stream(device).cuda_stream
                    if handle:
                        check(L.pyg_ctx_set_stream(self.h, handle))
            except ImportError:
                pass

    def close(self):
        if self.h:
            lib().pyg_ctx_destroy(self.h)
            self.h = None

    def sync(self):
        check(lib().pyg_ctx_sync(self.h))

    def launches(self):
        return lib().pyg_ctx_kernel_launches(self.h)

    def alloc(self, nbytes):
        return DevBuf(self, nbytes)

    def h2d(self, dst, src_np):
        check(lib().pyg_memcpy_h2d(self.h, _ptr(dst), src_np.ctypes.data, src_np.nbytes))

    def d2h(self, dst_np, src):
        check(lib().pyg_memcpy_d2h(self.h, dst_np.ctypes.data, _ptr(src), dst_np.nbytes))

    def upload(self, chunks, capacity=0, slot_bytes=32 << 20, slots=3):
        """Streams an iterable of byte-like numpy arrays into one device
        buffer through the overlapped upload ring (pyg_upload_*); each
        chunk is split into slot-sized pieces.  Returns a DevBuf."""
        L = lib()
        up = C.c_void_p()
        check(L.pyg_upload_open(self.h, capacity, slot_bytes, slots, C.byref(up)))
        try:
            for chunk in chunks:
                b = np.ascontiguousarray(chunk).view(np.uint8).reshape(-1)
                off = 0
                while off < b.size:
                    buf, cap = C.c_void_p(), C.c_size_t()
                    check(L.pyg_upload_slot(self.h, up, C.byref(buf), C.byref(cap)))
                    k = min(cap.value, b.size - off)
                    C.memmove(buf.value, b.ctypes.data + off, k)
                    check(L.pyg_upload_commit(self.h, up, k))
                    off += k
        except BaseException:
            L.pyg_upload_abort(self.h, up)
            raise
        dev, total = C.c_void_p(), C.c_size_t()
        check(L.pyg_upload_finish(self.h, up, C.byref(dev), C.byref(total)))
        return DevBuf(self, total.value, adopt=dev.value)

    # -- hash join ----------------------------------------------------
    def hashjoin_build(self, rel, key_cols, payload_cols=(), mode=HT_AGGREGATE, load_factor=0.5):
        k = (C.c_int32 * len(key_cols))(*key_cols)
        p = (C.c_int32 * max(1, len(payload_cols)))(*payload_cols)
        ht = C.c_void_p()
        r = rel.c()
        check(lib().pyg_hashjoin_build(self.h, C.byref(r), k, len(key_cols), p, len(payload_cols), mode,
                                       load_factor, C.byref(ht)))
        return HashTable(self, ht.value)

    def hashjoin_probe_agg(self, ht, rel, key_cols, proj):
        k = (C.c_int32 * len(key_cols))(*key_cols)
        pj = (pyg_proj * max(1, len(proj)))(*[pyg_proj(s, c) for s, c in proj])
        out = pyg_join_result()
        r = rel.c()
        check(lib().pyg_hashjoin_probe_agg(self.h, ht.h, C.byref(r), k, pj, len(proj), C.byref(out)))
        return out.count, [out.sums[i] for i in range(len(proj))]

    def hashjoin_probe_materialize(self, ht, rel, key_cols, proj, out, capacity):
        k = (C.c_int32 * len(key_cols))(*key_cols)
        pj = (pyg_proj * max(1, len(proj)))(*[pyg_proj(s, c) for s, c in proj])
        cnt = C.c_int64()
        r = rel.c()
        rc = lib().pyg_hashjoin_probe_materialize(self.h, ht.h, C.byref(r), k, pj, len(proj), _ptr(out), capacity,
                                                  C.byref(cnt))
        if rc not in (PYG_OK, PYG_ERR_CAPACITY):
            check(rc)
        return rc, cnt.value

    def hashjoin_agg(self, R, rkeys, S, skeys, proj, algorithm=JOIN_AUTO, radix_bits=0, load_factor=0.5,
                     stats=False):
        rk = (C.c_int32 * len(rkeys))(*rkeys)
        sk = (C.c_int32 * len(skeys))(*skeys)
        pj = (pyg_proj * max(1, len(proj)))(*[pyg_proj(s, c) for s, c in proj])
        o = pyg_join_opts(algorithm, radix_bits, load_factor, 0)
        out = pyg_join_result()
        st = pyg_join_stats()
        r, s = R.c(), S.c()
        check(lib().pyg_hashjoin_agg(self.h, C.byref(r), rk, C.byref(s), sk, len(rkeys), pj, len(proj), C.byref(o),
                                     C.byref(out), C.byref(st) if stats else None))
        res = (out.count, [out.sums[i] for i in range(len(proj))])
        return (res, st) if stats else res

    def hashjoin_agg_prepared(self, R, rkeys, S, skeys, proj, algorithm=JOIN_AUTO, radix_bits=0, load_factor=0.5):
        """The same call with its ctypes arguments built once: returns a
        function that runs the join and returns (count, [sums]) (for timing
        loops where Python argument marshalling would dominate)."""
        rk = (C.c_int32 * len(rkeys))(*rkeys)
        sk = (C.c_int32 * len(skeys))(*skeys)
        pj = (pyg_proj * max(1, len(proj)))(*[pyg_proj(s, c) for s, c in proj])
        o = pyg_join_opts(algorithm, radix_bits, load_factor, 0)
        out = pyg_join_result()
        r, s = R.c(), S.c()
        f = lib().pyg_hashjoin_agg
        args = (self.h, C.byref(r), rk, C.byref(s), sk, len(rkeys), pj, len(proj), C.byref(o), C.byref(out), None)
        keep = (R, S)

        def call():
            check(f(*args))
            assert keep
            return out.count, [out.sums[i] for i in range(len(proj))]

        return call

    # -- group-by -----------------------------------------------------
    def groupby(self, rel, key_cols, flags, sum_col, sort_by_key, expected_groups, out, capacity):
        k = (C.c_int32 * max(1, len(key_cols)))(*key_cols)
        ng = C.c_int64()
        r = rel.c()
        rc = lib().pyg_groupby(self.h, C.byref(r), k, len(key_cols), flags, sum_col, int(sort_by_key),
                               int(expected_groups), _ptr(out), capacity, C.byref(ng))
        if rc not in (PYG_OK, PYG_ERR_CAPACITY):
            check(rc)
        return rc, ng.value

    # -- partition / sort ---------------------------------------------
    def partition(self, rel, key_col, kind, fanout, out, range_min=0, range_max=0, splitters=None):
        s = pyg_splitter()
        s.kind, s.fanout, s.range_min, s.range_max = kind, fanout, range_min, range_max
        keep = None
        if splitters is not None:
            keep = np.ascontiguousarray(splitters, dtype=np.int64)
            s.splitters = keep.ctypes.data_as(C.POINTER(C.c_int64))
        offs = np.zeros(fanout + 1, dtype=np.int64)
        r = rel.c()
        check(lib().pyg_partition(self.h, C.byref(r), key_col, C.byref(s), _ptr(out),
                                  offs.ctypes.data_as(C.POINTER(C.c_int64))))
        return offs

    def sort(self, rel, key_col, out):
        r = rel.c()
        check(lib().pyg_sort(self.h, C.byref(r), key_col, _ptr(out)))

    def sortlimit(self, rel, key_cols, asc, limit, out, capacity):
        k = (C.c_int32 * max(1, len(key_cols)))(*key_cols)
        n = C.c_int64()
        r = rel.c()
        rc = lib().pyg_sortlimit(self.h, C.byref(r), k, len(key_cols), int(bool(asc)), limit, _ptr(out), capacity,
                                 C.byref(n))
        if rc not in (PYG_OK, PYG_ERR_CAPACITY):
            check(rc)
        return rc, n.value

    def lower_bound(self, rel, key_col, queries, nq, out):
        r = rel.c()
        check(lib().pyg_lower_bound(self.h, C.byref(r), key_col, _ptr(queries), nq, _ptr(out)))

    # -- MPSM ---------------------------------------------------------
    @staticmethod
    def mpsm_opts(kind=MPSM_SAMPLED, fanout=1024, sample_rate=0.01, leaves=1024, page_tuples=256, seed=1):
        o = pyg_mpsm_opts()
        o.splitter_kind, o.fanout, o.sample_rate, o.cdf_leaves, o.page_tuples, o.seed = (
            kind, fanout, sample_rate, leaves, page_tuples, seed)
        return o

    def mpsm_join_agg(self, R, rk, S, sk, proj, opts):
        pj = (pyg_proj * max(1, len(proj)))(*[pyg_proj(s, c) for s, c in proj])
        out = pyg_join_result()
        st = pyg_mpsm_stats()
        r, s = R.c(), S.c()
        check(lib().pyg_mpsm_join_agg(self.h, C.byref(r), rk, C.byref(s), sk, pj, len(proj), C.byref(opts),
                                      C.byref(out), C.byref(st)))
        return out.count, [out.sums[i] for i in range(len(proj))], st

    def mpsm_join_materialize(self, R, rk, S, sk, proj, opts, out, capacity):
        pj = (pyg_proj * max(1, len(proj)))(*[pyg_proj(s, c) for s, c in proj])
        cnt = C.c_int64()
        r, s = R.c(), S.c()
        rc = lib().pyg_mpsm_join_materialize(self.h, C.byref(r), rk, C.byref(s), sk, pj, len(proj), C.byref(opts),
                                             _ptr(out), capacity, C.byref(cnt))
        if rc not in (PYG_OK, PYG_ERR_CAPACITY):
            check(rc)
        return rc, cnt.value

    # -- batched fragments ---------------------------------------------
    @staticmethod
    def fragments(pairs):
        """pairs: [(build_tensor, nbuild, probe_tensor, nprobe)] -> ctypes array."""
        arr = (pyg_fragment * len(pairs))()
        for i, (b, nb, p, np_) in enumerate(pairs):
            arr[i] = pyg_fragment(_ptr(b), nb, _ptr(p), np_)
        return arr

    def batch_create(self, frags, tuning=None):
        h = C.c_void_p()
        check(lib().pyg_batch_create(self.h, frags, len(frags), C.byref(tuning) if tuning else None, C.byref(h)))
        return h.value

    def batch_run(self, b, n):
        c = np.zeros(n, dtype=np.int64)
        s = np.zeros(n, dtype=np.int64)
        lat = np.zeros(n, dtype=np.float64)
        rc = lib().pyg_batch_run(self.h, b, c.ctypes.data_as(_PI64), s.ctypes.data_as(_PI64),
                                 lat.ctypes.data_as(C.POINTER(C.c_double)))
        return rc, c, s, lat

    def batch_free(self, b):
        check(lib().pyg_batch_free(self.h, b))

    def batch_run_plain(self, frags):
        n = len(frags)
        c = np.zeros(n, dtype=np.int64)
        s = np.zeros(n, dtype=np.int64)
        lat = np.zeros(n, dtype=np.float64)
        check(lib().pyg_batch_run_plain(self.h, frags, n, c.ctypes.data_as(_PI64), s.ctypes.data_as(_PI64),
                                        lat.ctypes.data_as(C.POINTER(C.c_double))))
        return c, s, lat

    def autotune(self, frags, cache_path=None):
        t = pyg_tuning()
        check(lib().pyg_autotune(self.h, frags, len(frags), cache_path.encode() if cache_path else None,
                                 C.byref(t)))
        return t

    # -- generators ---------------------------------------------------
    def gen_pk(self, out, n, mul, seed):
        check(lib().pyg_gen_pk(self.h, _ptr(out), n, mul, seed))

    def gen_fk(self, out, n, nkeys, theta, seed_keys, vmax, seed):
        check(lib().pyg_gen_fk(self.h, _ptr(out), n, nkeys, theta, seed_keys, vmax, seed))


class HashTable:
    def __init__(self, ctx, h):
        self.ctx = ctx
        self.h = h

    def stats(self):
        e, c, d = C.c_int64(), C.c_int64(), C.c_int32()
        check(lib().pyg_hashtable_stats(self.ctx.h, self.h, C.byref(e), C.byref(c), C.byref(d)))
        return e.value, c.value, d.value

    def free(self):
        if self.h:
            lib().pyg_hashtable_free(self.ctx.h, self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

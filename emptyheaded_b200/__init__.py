"""B200-native storage-engine hot path of EmptyHeaded: trie construction,
hybrid uint / bitset / block-bitset set layouts, set intersection and the
generic-join COUNT plans, as sm_100a CUDA kernels behind a C ABI
(include/eh_b200.h).

This module is a thin ctypes front end over that ABI, named after the
reference's storage-engine API:

    Trie            Trie<A,M> built from an encoded binary relation
                    (storage_engine/src/Trie.cpp:380-510)
    Trie.count()    a generated COUNT bag (EHGenerator.scala:728-838) run on
                    the device
    set_intersect   ops::set_intersect (trie/set/ops/intersection/set.hpp)

It never computes on the host: if the shared library or a GPU is missing,
calls raise.
"""
import atexit
import ctypes
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# EH_B200_LIB selects another build of the same library (a variant built
# with emptyheaded_b200.build.build(libdir=...)); default: the in-tree one
LIB_PATH = os.environ.get("EH_B200_LIB") or os.path.join(_HERE, "_lib", "libeh_b200.so")

# status codes and enums (include/eh_b200.h)
EH_OK = 0
STATUS_NAMES = {1: "INVALID", 2: "CUDA", 3: "OOM", 5: "UNSUPPORTED", 6: "IO", 7: "NO_DEVICE"}
RANGE_BITSET, UINTEGER, BLOCK_BITSET = 0, 1, 3
HEURISTIC, LEARNED, FORCED, EXPLICIT = 0, 1, 2, 3
QUERIES = {"triangle": 0, "clique4": 1, "lollipop": 2, "barbell": 3}
# equality-selection plans (Trie.count_select)
SELECT_QUERIES = {"clique4_sel": 4, "barbell_sel": 5}
QUERY_NAMES = {v: k for k, v in list(QUERIES.items()) + list(SELECT_QUERIES.items())}


class EHError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (%s)" % (msg, STATUS_NAMES.get(status, status)))
        self.status = status


class LayoutConfig(ctypes.Structure):
    _fields_ = [("policy", ctypes.c_int), ("forced_layout", ctypes.c_int), ("model", ctypes.c_void_p),
                ("max_bitset_bytes", ctypes.c_uint64), ("layouts", ctypes.c_void_p), ("min_gain", ctypes.c_float)]


class TrieInfo(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint64), ("n_head", ctypes.c_uint32), ("n_nodes", ctypes.c_uint32),
                ("head_layout", ctypes.c_uint32), ("n_uinteger", ctypes.c_uint32),
                ("n_range_bitset", ctypes.c_uint32), ("n_block_bitset", ctypes.c_uint32),
                ("bitset_words", ctypes.c_uint64), ("block_count", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64), ("max_set", ctypes.c_uint32), ("build_ms", ctypes.c_float)]


class ExecConfig(ctypes.Structure):
    _fields_ = [("warps_per_block", ctypes.c_int), ("chunk_pairs", ctypes.c_int), ("long_row", ctypes.c_int),
                ("smem_words", ctypes.c_int), ("record_timings", ctypes.c_int),
                ("shard_index", ctypes.c_int), ("shard_count", ctypes.c_int), ("no_block_items", ctypes.c_int)]


class Atom(ctypes.Structure):
    _fields_ = [("relation", ctypes.c_uint32), ("v0", ctypes.c_uint32), ("v1", ctypes.c_uint32)]


class Rule(ctypes.Structure):
    _fields_ = [("n_vars", ctypes.c_uint32), ("n_atoms", ctypes.c_uint32), ("atoms", ctypes.c_void_p),
                ("sel_var", ctypes.c_int32), ("sel_value", ctypes.c_uint32)]


class QueryStats(ctypes.Structure):
    _fields_ = [("query_ms", ctypes.c_float), ("kernel_ms", ctypes.c_float), ("launches", ctypes.c_uint32),
                ("work_items", ctypes.c_uint64), ("wedges", ctypes.c_uint64),
                ("algorithmic_bytes", ctypes.c_uint64)]


_lib = None

_P = ctypes.c_void_p
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def lib():
    """The loaded shared library (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EHError(5, "libeh_b200.so is not built; run python -m emptyheaded_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        L.eh_last_error.restype = ctypes.c_char_p
        L.eh_version.restype = ctypes.c_char_p
        sig = {
            "eh_context_create": [ctypes.c_int, ctypes.POINTER(_P)],
            "eh_context_destroy": [_P],
            "eh_context_sync": [_P],
            "eh_context_stream": [_P, ctypes.POINTER(_P)],
            "eh_context_memory": [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                  ctypes.POINTER(ctypes.c_uint64)],
            "eh_context_reserve": [_P, ctypes.c_uint64],
            "eh_device_alloc": [_P, ctypes.c_uint64, ctypes.POINTER(_P)],
            "eh_device_free": [_P, _P],
            "eh_memcpy": [_P, _P, _P, ctypes.c_uint64],
            "eh_graph_er": [_P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(_P),
                            ctypes.POINTER(_P)],
            "eh_graph_rmat": [_P, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, ctypes.POINTER(_P), ctypes.POINTER(_P)],
            "eh_graph_chunglu": [_P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double,
                                 ctypes.POINTER(_P), ctypes.POINTER(_P)],
            "eh_graph_preprocess": [_P, _P, _P, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_P),
                                    ctypes.POINTER(_P), _u64p, _u32p],
            "eh_trie_build": [_P, _P, _P, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(LayoutConfig),
                              ctypes.POINTER(_P)],
            "eh_trie_relayout": [_P, _P, ctypes.POINTER(LayoutConfig)],
            "eh_trie_free": [_P],
            "eh_trie_load_reference": [_P, ctypes.c_char_p, ctypes.POINTER(LayoutConfig), ctypes.POINTER(_P)],
            "eh_trie_save_reference": [_P, _P, ctypes.c_char_p, ctypes.c_uint32],
            "eh_trie_info_get": [_P, ctypes.POINTER(TrieInfo)],
            "eh_trie_export": [_P, _P, _P, _P, _P],
            "eh_trie_set_bytes": [_P, ctypes.c_uint32, _P, ctypes.c_uint64, _u64p, ctypes.POINTER(ctypes.c_uint8)],
            "eh_set_intersect_batch": [_P, _P, _P, ctypes.c_uint32, _P, _P, _P, ctypes.c_uint32, _P, _P, _P],
            "eh_encoding_build": [_P, _P, _P, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P)],
            "eh_encoding_encode": [_P, _P, _P, ctypes.c_uint64, ctypes.c_int, _P],
            "eh_encoding_decode": [_P, _P, _P, ctypes.c_uint64, ctypes.c_int, _P],
            "eh_encoding_size": [_P, _u64p],
            "eh_encoding_values": [_P, _P, _P, ctypes.c_uint64],
            "eh_encoding_free": [_P],
            "eh_query_count": [_P, _P, ctypes.c_int, ctypes.POINTER(ExecConfig), _u64p, ctypes.POINTER(QueryStats)],
            "eh_query_count_noalloc": [_P, _P, ctypes.c_int, ctypes.POINTER(ExecConfig), _u64p],
            "eh_rule_match": [ctypes.POINTER(Rule), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint32)],
            "eh_rule_count": [_P, _P, ctypes.c_uint32, ctypes.POINTER(Rule), ctypes.POINTER(ExecConfig), _u64p,
                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(QueryStats)],
            "eh_query_count_select": [_P, _P, ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(ExecConfig), _u64p,
                                      ctypes.POINTER(QueryStats)],
            "eh_query_materialize": [_P, _P, ctypes.c_int, ctypes.POINTER(ExecConfig), ctypes.c_int, _P, _P, _P,
                                     ctypes.c_uint64, _u64p],
            "eh_query_count_batched": [_P, _P, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ExecConfig), _P,
                                       ctypes.POINTER(QueryStats)],
            "eh_triangle_annotation": [_P, _P, ctypes.POINTER(ExecConfig), _P],
            "eh_query_weighted_root": [_P, _P, ctypes.c_int, _P, ctypes.c_uint32, _u64p],
            "eh_batch_create": [_P, _P, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ExecConfig),
                                ctypes.POINTER(_P)],
            "eh_batch_run": [_P, _P, _P, ctypes.POINTER(QueryStats)],
            "eh_batch_free": [_P],
            "eh_query_count_host_csr": [_P, _P, ctypes.c_uint32, _P, _P, ctypes.c_uint32,
                                        ctypes.POINTER(LayoutConfig), ctypes.c_int, ctypes.POINTER(ExecConfig), _u64p,
                                        ctypes.POINTER(QueryStats)],
            "eh_timing_records": [_P, _P, ctypes.c_uint64, _u64p],
            "eh_model_create": [_P, ctypes.c_int, _P, ctypes.c_uint64, ctypes.POINTER(_P)],
            "eh_model_free": [_P],
            "eh_model_params": [_P, _P, ctypes.c_uint64, _u64p, ctypes.c_int],
            "eh_model_train": [_P, _P, _P, _P, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32,
                               ctypes.POINTER(ctypes.c_float)],
            "eh_model_loss_grad": [_P, _P, _P, _P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float), _P],
            "eh_model_predict": [_P, _P, _P, ctypes.c_uint32, _P],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def _check(status):
    if status != EH_OK:
        raise EHError(status, lib().eh_last_error().decode())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


# ------------------------------------------------------------------ context
_live_contexts = weakref.WeakSet()


class Context:
    """Device, stream and events (the role of the reference's thread pool,
    utils/thread_pool.hpp:16-41).  Tries, models and device arrays made in a
    context must be freed before it; close() frees whatever is still alive,
    and every open context is closed at interpreter exit in that order."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _check(lib().eh_context_create(device, ctypes.byref(h)))
        self.h = h
        self._children = weakref.WeakSet()
        _live_contexts.add(self)

    def _adopt(self, obj):
        self._children.add(obj)

    def close(self):
        if getattr(self, "h", None):
            for c in list(self._children):
                c.free()
            lib().eh_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        _check(lib().eh_context_sync(self.h))

    def stream(self):
        s = ctypes.c_void_p()
        _check(lib().eh_context_stream(self.h, ctypes.byref(s)))
        return s.value

    def memory(self):
        """{reserved, used, peak} bytes of the engine's device memory pool
        (eh_context_memory); peak counts since the last reserve()."""
        r, u, p = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().eh_context_memory(self.h, ctypes.byref(r), ctypes.byref(u), ctypes.byref(p)))
        return {"reserved": r.value, "used": u.value, "peak": p.value}

    def reserve(self, nbytes):
        """Keep nbytes of device memory in the pool as one block
        (eh_context_reserve): calls whose peak fits then map no new memory."""
        _check(lib().eh_context_reserve(self.h, ctypes.c_uint64(int(nbytes))))


@atexit.register
def _close_all():
    for c in list(_live_contexts):
        try:
            c.close()
        except Exception:
            pass


_default = None


def default_context():
    global _default
    if _default is None:
        _default = Context(0)
    return _default


class DeviceArray:
    """A uint32 device array owned by the engine (eh_device_alloc)."""

    def __init__(self, ctx, ptr, n):
        self.ctx, self.ptr, self.n = ctx, ptr, n
        ctx._adopt(self)

    def free(self):
        if self.ptr:
            _check(lib().eh_device_free(self.ctx.h, ctypes.c_void_p(self.ptr)))
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def numpy(self):
        out = np.empty(self.n, np.uint32)
        if self.n:
            _check(lib().eh_memcpy(self.ctx.h, _ptr(out), ctypes.c_void_p(self.ptr), 4 * self.n))
        return out


def _pair(ctx, fn, m, *args):
    u, v = ctypes.c_void_p(), ctypes.c_void_p()
    _check(fn(ctx.h, *args, ctypes.byref(u), ctypes.byref(v)))
    return DeviceArray(ctx, u.value, m), DeviceArray(ctx, v.value, m)


def gen_er(seed, n, m, ctx=None):
    ctx = ctx or default_context()
    return _pair(ctx, lib().eh_graph_er, m, seed, n, m)


def gen_rmat(seed, scale, m, a=0.57, b=0.19, c=0.19, ctx=None):
    ctx = ctx or default_context()
    return _pair(ctx, lib().eh_graph_rmat, m, seed, scale, m, a, b, c)


def gen_chunglu(seed, n, m, gamma, ctx=None):
    ctx = ctx or default_context()
    return _pair(ctx, lib().eh_graph_chunglu, m, seed, n, m, gamma)


def preprocess(u, v, symmetric=False, ctx=None):
    """Device edge samples -> (src, dst, nodes): the encoded Edge relation."""
    ctx = ctx or default_context()
    s, d = ctypes.c_void_p(), ctypes.c_void_p()
    rows, nodes = ctypes.c_uint64(), ctypes.c_uint32()
    _check(lib().eh_graph_preprocess(ctx.h, ctypes.c_void_p(u.ptr), ctypes.c_void_p(v.ptr), u.n,
                                     1 if symmetric else 0, ctypes.byref(s), ctypes.byref(d), ctypes.byref(rows),
                                     ctypes.byref(nodes)))
    return DeviceArray(ctx, s.value, rows.value), DeviceArray(ctx, d.value, rows.value), nodes.value


def _layout_cfg(policy=HEURISTIC, forced=UINTEGER, model=None, max_bitset_bytes=0, layouts=None):
    c = LayoutConfig()
    c.policy = policy
    c.forced_layout = forced
    c.model = model.h.value if model is not None else None
    c.max_bitset_bytes = max_bitset_bytes
    c._keep = None
    if layouts is not None:
        c._keep = np.ascontiguousarray(layouts, np.uint8)
        c.layouts = c._keep.ctypes.data
    return c


def _exec_cfg(warps=0, chunk=0, smem_words=0, record=False, shard=(0, 1), long_row=0, block_items=True):
    e = ExecConfig()
    e.no_block_items = 0 if block_items else 1
    e.warps_per_block = warps
    e.chunk_pairs = chunk
    e.long_row = long_row
    e.smem_words = smem_words
    e.record_timings = 1 if record else 0
    e.shard_index, e.shard_count = shard
    return e


# --------------------------------------------------------------------- trie
class Trie:
    """Two-level trie over an encoded binary relation, resident on the GPU.

    Mirrors Trie<A,M>(path, max_set_sizes, attr_in, annotations)
    (storage_engine/src/Trie.cpp:380-510): rows in any order, duplicates
    allowed; the head is the distinct first-column values, each with the
    sorted set of its second-column values in a hybrid layout.
    """

    def __init__(self, col0, col1, policy=HEURISTIC, forced=UINTEGER, model=None, ctx=None, max_bitset_bytes=0):
        self.ctx = ctx or default_context()
        cfg = _layout_cfg(policy, forced, model, max_bitset_bytes)
        h = ctypes.c_void_p()
        if isinstance(col0, DeviceArray):
            _check(lib().eh_trie_build(self.ctx.h, ctypes.c_void_p(col0.ptr), ctypes.c_void_p(col1.ptr), col0.n, 1,
                                       ctypes.byref(cfg), ctypes.byref(h)))
        else:
            c0 = np.ascontiguousarray(col0, np.uint32)
            c1 = np.ascontiguousarray(col1, np.uint32)
            if c0.shape != c1.shape:
                raise ValueError("columns differ in length")
            _check(lib().eh_trie_build(self.ctx.h, _ptr(c0), _ptr(c1), len(c0), 0, ctypes.byref(cfg),
                                       ctypes.byref(h)))
        self.h = h
        self.ctx._adopt(self)

    @classmethod
    def load_reference(cls, path, policy=HEURISTIC, forced=UINTEGER, model=None, ctx=None, max_bitset_bytes=0):
        """Trie<void*,ParMemoryBuffer>::load (Trie.cpp:37-75) of a two-level
        trie the reference saved under path (path/ram/trieinfo.bin, ...)."""
        self = cls.__new__(cls)
        self.ctx = ctx or default_context()
        cfg = _layout_cfg(policy, forced, model, max_bitset_bytes)
        h = ctypes.c_void_p()
        _check(lib().eh_trie_load_reference(self.ctx.h, os.fsencode(path), ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.ctx._adopt(self)
        return self

    def save_reference(self, path, num_threads):
        """Trie::save (Trie.cpp:15-35) in the reference's format, loadable by
        an engine built with NUM_THREADS == num_threads."""
        _check(lib().eh_trie_save_reference(self.ctx.h, self.h, os.fsencode(path), int(num_threads)))

    def free(self):
        if getattr(self, "h", None):
            lib().eh_trie_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def info(self):
        i = TrieInfo()
        _check(lib().eh_trie_info_get(self.h, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in TrieInfo._fields_}

    def relayout(self, policy=HEURISTIC, forced=UINTEGER, model=None, max_bitset_bytes=0, layouts=None):
        """Re-pick the level-1 layouts: the density rule, the learned model,
        one forced layout, or (policy=EXPLICIT) one layout per set."""
        cfg = _layout_cfg(policy, forced, model, max_bitset_bytes, layouts)
        _check(lib().eh_trie_relayout(self.ctx.h, self.h, ctypes.byref(cfg)))

    def export(self):
        """(head, off, vals, layout) host copies (what Trie::foreach walks)."""
        inf = self.info()
        nh, rows = inf["n_head"], inf["rows"]
        head = np.empty(max(nh, 1), np.uint32)
        off = np.empty(nh + 1, np.uint64)
        vals = np.empty(max(rows, 1), np.uint32)
        lay = np.empty(max(nh, 1), np.uint8)
        _check(lib().eh_trie_export(self.h, _ptr(head), _ptr(off), _ptr(vals), _ptr(lay)))
        return head[:nh], off, vals[:rows], lay[:nh]

    def set_bytes(self, i):
        """Reference-format bytes of child set i (None: the head set) and its layout."""
        idx = 0xFFFFFFFF if i is None else i
        n = ctypes.c_uint64()
        lay = ctypes.c_uint8()
        _check(lib().eh_trie_set_bytes(self.h, idx, None, 0, ctypes.byref(n), ctypes.byref(lay)))
        out = np.empty(max(n.value, 1), np.uint8)
        _check(lib().eh_trie_set_bytes(self.h, idx, _ptr(out), n.value, ctypes.byref(n), ctypes.byref(lay)))
        return out[: n.value], lay.value

    def count(self, query="triangle", warps=0, chunk=0, smem_words=0, record=False, stats=False, shard=(0, 1),
              long_row=0, config=None, block_items=True):
        """Run a named COUNT plan; returns the count (and stats if asked).
        shard=(i, n) runs the i-th of n round-robin shares of the work items
        (the partial counts of the n shares sum to the count).  `config`
        (a dict from emptyheaded_b200.autotune) supplies the schedule knobs."""
        if config:
            warps = config.get("warps", warps)
            chunk = config.get("chunk", chunk)
            smem_words = config.get("smem_words", smem_words)
            long_row = config.get("long_row", long_row)
            block_items = config.get("block_items", block_items)
        e = _exec_cfg(warps, chunk, smem_words, record, shard, long_row, block_items)
        r = ctypes.c_uint64()
        st = QueryStats()
        _check(lib().eh_query_count(self.ctx.h, self.h, QUERIES[query], ctypes.byref(e), ctypes.byref(r),
                                    ctypes.byref(st)))
        if stats:
            return r.value, {k: getattr(st, k) for k, _ in QueryStats._fields_}
        return r.value

    def count_select(self, query, value, stats=False, config=None):
        """FliqueSelAgg (query="clique4_sel", Edge(a,x), x=value) or
        BarbellSelAgg (query="barbell_sel", Edge(a,p), Edge(p,x), p=value):
        the reference's equality-selection COUNT queries.  Raises when value
        is in neither column of the relation."""
        config = config or {}
        e = _exec_cfg(config.get("warps", 0), config.get("chunk", 0), config.get("smem_words", 0), False, (0, 1),
                      config.get("long_row", 0))
        r = ctypes.c_uint64()
        st = QueryStats()
        _check(lib().eh_query_count_select(self.ctx.h, self.h, SELECT_QUERIES[query], int(value), ctypes.byref(e),
                                           ctypes.byref(r), ctypes.byref(st)))
        if stats:
            return r.value, {k: getattr(st, k) for k, _ in QueryStats._fields_}
        return r.value

    def materialize(self, query="triangle", project=False):
        """Rows of Triangle(a,b,c) sorted by (a,b,c) as an (n, 3) uint32
        array; project=True gives TriangleProj(a,b), an (n, 2) array."""
        cols = 2 if project else 3
        e = _exec_cfg()
        n = ctypes.c_uint64()
        # the device builds the rows once to size them, then fills
        _check(lib().eh_query_materialize(self.ctx.h, self.h, QUERIES[query], ctypes.byref(e), cols, None, None,
                                          None, 0, ctypes.byref(n)))
        rows = n.value
        a = np.empty(max(rows, 1), np.uint32)
        b = np.empty(max(rows, 1), np.uint32)
        c = np.empty(max(rows, 1), np.uint32)
        _check(lib().eh_query_materialize(self.ctx.h, self.h, QUERIES[query], ctypes.byref(e), cols, _ptr(a),
                                          _ptr(b), _ptr(c), rows, ctypes.byref(n)))
        out = [a[:rows], b[:rows]] + ([] if project else [c[:rows]])
        return np.stack(out, 1)

    def weighted_root(self, query, z):
        """Root bag of lollipop / barbell over an annotation z given by node
        value (eh_query_weighted_root): lollipop sum_a z(a)|N(a)|, barbell
        sum over rows (a,x) of z(a)z(x), modulo 2^64."""
        z = np.ascontiguousarray(z, np.uint64)
        r = ctypes.c_uint64()
        _check(lib().eh_query_weighted_root(self.ctx.h, self.h, QUERIES[query], _ptr(z) if len(z) else None, len(z),
                                            ctypes.byref(r)))
        return r.value

    def triangle_annotation(self):
        nh = self.info()["n_head"]
        out = np.zeros(max(nh, 1), np.uint64)
        e = _exec_cfg()
        _check(lib().eh_triangle_annotation(self.ctx.h, self.h, ctypes.byref(e), _ptr(out)))
        return out[:nh]


def count_batched(tries, query="triangle", chunk=0, stats=False):
    ctx = tries[0].ctx
    arr = (ctypes.c_void_p * len(tries))(*[t.h.value for t in tries])
    res = np.zeros(len(tries), np.uint64)
    e = _exec_cfg(chunk=chunk)
    st = QueryStats()
    _check(lib().eh_query_count_batched(ctx.h, arr, len(tries), QUERIES[query], ctypes.byref(e), _ptr(res),
                                        ctypes.byref(st)))
    if stats:
        return res, {k: getattr(st, k) for k, _ in QueryStats._fields_}
    return res


class Batch:
    """Many tries, one plan, one CUDA-graph launch per run (eh_batch_*).
    The tries must stay alive and keep their layouts while the batch lives."""

    def __init__(self, tries, query="triangle", config=None):
        self.ctx = tries[0].ctx
        self.tries = list(tries)  # keep them alive
        c = config or {}
        e = _exec_cfg(c.get("warps", 0), c.get("chunk", 0), c.get("smem_words", 0), long_row=c.get("long_row", 0))
        arr = (ctypes.c_void_p * len(tries))(*[t.h.value for t in tries])
        h = ctypes.c_void_p()
        _check(lib().eh_batch_create(self.ctx.h, arr, len(tries), QUERIES[query], ctypes.byref(e), ctypes.byref(h)))
        self.h = h
        self.ctx._adopt(self)

    def run(self, stats=False):
        res = np.zeros(len(self.tries), np.uint64)
        st = QueryStats()
        _check(lib().eh_batch_run(self.ctx.h, self.h, _ptr(res), ctypes.byref(st)))
        if stats:
            return res, {k: getattr(st, k) for k, _ in QueryStats._fields_}
        return res

    def free(self):
        if getattr(self, "h", None):
            lib().eh_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def count_host_csr(head, off, vals, n_nodes, query="triangle", policy=HEURISTIC, model=None, ctx=None, stats=False,
                   config=None):
    """Host CSR in, count out: the reference-facing call with host buffers."""
    ctx = ctx or default_context()
    cfg = _layout_cfg(policy, UINTEGER, model)
    c = config or {}
    e = _exec_cfg(c.get("warps", 0), c.get("chunk", 0), c.get("smem_words", 0), long_row=c.get("long_row", 0))
    r = ctypes.c_uint64()
    st = QueryStats()
    _check(lib().eh_query_count_host_csr(ctx.h, _ptr(head), len(head), _ptr(off), _ptr(vals), n_nodes,
                                         ctypes.byref(cfg), QUERIES[query], ctypes.byref(e), ctypes.byref(r),
                                         ctypes.byref(st)))
    if stats:
        return r.value, {k: getattr(st, k) for k, _ in QueryStats._fields_}
    return r.value


def timing_records(ctx=None):
    ctx = ctx or default_context()
    n = ctypes.c_uint64()
    _check(lib().eh_timing_records(ctx.h, None, 0, ctypes.byref(n)))
    out = np.empty((max(n.value, 1), 8), np.float32)
    _check(lib().eh_timing_records(ctx.h, _ptr(out), n.value, ctypes.byref(n)))
    return out[: n.value]


# ------------------------------------------------------------------ set ops
def set_intersect(sets, layouts, pairs, materialize=False, ctx=None):
    """Pairwise ops::set_intersect on the device.

    sets: list of sorted uint32 arrays; layouts: per-set layout codes;
    pairs: (k, 2) array of set indices.  Returns counts (and the
    materialized intersections as a list when asked)."""
    ctx = ctx or default_context()
    sizes = np.array([len(s) for s in sets], np.uint64)
    off = np.zeros(len(sets) + 1, np.uint64)
    np.cumsum(sizes, out=off[1:])
    elems = np.ascontiguousarray(np.concatenate([np.asarray(s, np.uint32) for s in sets])
                                 if len(sets) else np.zeros(0, np.uint32), np.uint32)
    if elems.size == 0:
        elems = np.zeros(1, np.uint32)
    lay = np.ascontiguousarray(layouts, np.uint8)
    pairs = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
    pa = np.ascontiguousarray(pairs[:, 0])
    pb = np.ascontiguousarray(pairs[:, 1])
    counts = np.zeros(max(len(pa), 1), np.uint64)
    out_off = out = None
    if materialize:
        room = np.minimum(sizes[pa], sizes[pb])
        out_off = np.zeros(len(pa), np.uint64)
        if len(pa) > 1:
            np.cumsum(room[:-1], out=out_off[1:])
        out = np.zeros(max(int(room.sum()), 1), np.uint32)
    _check(lib().eh_set_intersect_batch(ctx.h, _ptr(elems), _ptr(off), len(sets), _ptr(lay), _ptr(pa), _ptr(pb),
                                        len(pa), _ptr(counts), _ptr(out_off), _ptr(out)))
    counts = counts[: len(pa)]
    if materialize:
        return counts, [out[int(o): int(o) + int(c)].copy() for o, c in zip(out_off, counts)]
    return counts


# -------------------------------------------------------------------- model
VALUE_TYPES = {"uint32": (0, np.uint32), "int32": (1, np.int32), "int64": (2, np.int64), "float32": (3, np.float32)}


class Encoding:
    """Dictionary encoding on the device, the reference's Encoding<T>
    (storage_engine/src/Encoding.cpp:21-48): keys in ascending value order
    over the distinct values of all the given columns.  value_type is one of
    "uint32", "int32", "int64", "float32" (uint32_t, int, long, float)."""

    def __init__(self, cols, value_type="uint32", ctx=None):
        self.ctx = ctx or default_context()
        self.value_type = value_type
        code, dt = VALUE_TYPES[value_type]
        self._dt = dt
        cols = [np.ascontiguousarray(c, dt) for c in cols]
        ptrs = (ctypes.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
        lens = np.array([len(c) for c in cols] or [0], np.uint64)
        h = ctypes.c_void_p()
        _check(lib().eh_encoding_build(self.ctx.h, ptrs, _ptr(lens), len(cols), code, 0, ctypes.byref(h)))
        self.h = h.value
        self.ctx._adopt(self)

    def __len__(self):
        n = ctypes.c_uint64()
        _check(lib().eh_encoding_size(self.h, ctypes.byref(n)))
        return n.value

    def encode(self, col):
        """encode_column: uint32 keys (raises for a value not in the encoding)"""
        col = np.ascontiguousarray(col, self._dt)
        keys = np.empty(max(1, len(col)), np.uint32)
        _check(lib().eh_encoding_encode(self.ctx.h, self.h, col.ctypes.data, len(col), 0, _ptr(keys)))
        return keys[: len(col)]

    def decode(self, keys):
        """key_to_value per key"""
        keys = np.ascontiguousarray(keys, np.uint32)
        out = np.empty(max(1, len(keys)), self._dt)
        _check(lib().eh_encoding_decode(self.ctx.h, self.h, _ptr(keys), len(keys), 0, out.ctypes.data))
        return out[: len(keys)]

    def values(self):
        """the key_to_value table"""
        n = len(self)
        out = np.empty(max(1, n), self._dt)
        _check(lib().eh_encoding_values(self.ctx.h, self.h, out.ctypes.data, n))
        return out[:n]

    def free(self):
        if getattr(self, "h", None):
            lib().eh_encoding_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Model:
    """Small fp32 MLP trained and evaluated by the engine's own kernels."""

    def __init__(self, dims, seed=0, ctx=None):
        self.ctx = ctx or default_context()
        self.dims = list(dims)
        d = (ctypes.c_int * len(dims))(*dims)
        h = ctypes.c_void_p()
        _check(lib().eh_model_create(self.ctx.h, len(dims) - 1, d, seed, ctypes.byref(h)))
        self.h = h
        self.ctx._adopt(self)

    def free(self):
        if getattr(self, "h", None):
            lib().eh_model_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def params(self):
        n = ctypes.c_uint64()
        _check(lib().eh_model_params(self.h, None, 0, ctypes.byref(n), 0))
        out = np.empty(n.value, np.float32)
        _check(lib().eh_model_params(self.h, _ptr(out), n.value, ctypes.byref(n), 0))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        n = ctypes.c_uint64()
        _check(lib().eh_model_params(self.h, _ptr(p), len(p), ctypes.byref(n), 1))

    def train(self, x, y, lr=1e-2, steps=1):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        _check(lib().eh_model_train(self.ctx.h, self.h, _ptr(x), _ptr(y), x.shape[0], lr, steps, ctypes.byref(loss)))
        return loss.value

    def loss_grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        loss = ctypes.c_float()
        g = np.empty(len(self.params()), np.float32)
        _check(lib().eh_model_loss_grad(self.ctx.h, self.h, _ptr(x), _ptr(y), x.shape[0], ctypes.byref(loss),
                                        _ptr(g)))
        return loss.value, g

    def predict(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((x.shape[0], self.dims[-1]), np.float32)
        _check(lib().eh_model_predict(self.ctx.h, self.h, _ptr(x), x.shape[0], _ptr(y)))
        return y

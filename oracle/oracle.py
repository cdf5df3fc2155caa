"""ctypes/numpy front end of the CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker, never by the product.

Two oracles live under this directory:
  * libeh_oracle.so (eh_oracle.c): a C restatement of the reference hot path;
  * _ref/eh_ref (ref_driver.cpp): the reference storage engine itself,
    compiled from its own sources, driven by hand-written generated-shape
    query code.
Both are built by oracle/Makefile.
"""
import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libeh_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "eh_ref")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_lib = None


def reference_dir():
    """The EmptyHeaded checkout the reference engine is compiled from:
    $EH_REFERENCE, else the directory `reference` beside this repository."""
    return os.environ.get("EH_REFERENCE") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def build(ref=True):
    """Compile the restatement (and, when the reference tree is present, the
    reference engine driver)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "restate"])
    if ref and os.path.isdir(reference_dir()):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", "REF=" + reference_dir()])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        L = ctypes.CDLL(LIB_PATH)
        L.eho_rand64.restype = ctypes.c_uint64
        L.eho_rand64.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.eho_gen_er.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, _u32p, _u32p]
        L.eho_rmat_thresholds.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, _u32p]
        L.eho_gen_rmat.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, _u32p, _u32p, _u32p]
        L.eho_chunglu_cdf.argtypes = [ctypes.c_uint32, ctypes.c_double, _u64p]
        L.eho_gen_chunglu.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, _u64p, _u32p, _u32p]
        L.eho_preprocess.restype = ctypes.c_uint64
        L.eho_preprocess.argtypes = [_u32p, _u32p, ctypes.c_uint64, ctypes.c_int, _u32p, _u32p,
                                     ctypes.POINTER(ctypes.c_uint32)]
        L.eho_trie_build.restype = ctypes.c_uint64
        L.eho_trie_build.argtypes = [_u32p, _u32p, ctypes.c_uint64, _u32p, _u64p, _u32p,
                                     ctypes.POINTER(ctypes.c_uint32)]
        L.eho_is_sparse.restype = ctypes.c_int
        L.eho_is_sparse.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.eho_hybrid_type.restype = ctypes.c_int
        L.eho_hybrid_type.argtypes = [_u32p, ctypes.c_uint64]
        L.eho_range_bitset_bytes.restype = ctypes.c_uint64
        L.eho_range_bitset_bytes.argtypes = [_u32p, ctypes.c_uint64]
        L.eho_range_bitset_build.restype = ctypes.c_uint64
        L.eho_range_bitset_build.argtypes = [_u32p, ctypes.c_uint64, _u8p]
        L.eho_intersect.restype = ctypes.c_uint64
        L.eho_intersect.argtypes = [_u32p, ctypes.c_uint64, _u32p, ctypes.c_uint64, ctypes.c_void_p]
        for q in ("eho_triangle", "eho_clique4", "eho_lollipop", "eho_barbell"):
            f = getattr(L, q)
            f.restype = ctypes.c_uint64
            f.argtypes = [_u32p, ctypes.c_uint32, _u64p, _u32p]
        L.eho_triangle_per_vertex.argtypes = [_u32p, ctypes.c_uint32, _u64p, _u32p, _u64p]
        for q in ("eho_clique4_sel", "eho_barbell_sel"):
            f = getattr(L, q)
            f.restype = ctypes.c_uint64
            f.argtypes = [_u32p, ctypes.c_uint32, _u64p, _u32p, ctypes.c_uint32]
        L.eho_triangle_list.restype = ctypes.c_uint64
        L.eho_triangle_list.argtypes = [_u32p, ctypes.c_uint32, _u64p, _u32p, _u32p, _u32p, _u32p, ctypes.c_uint64]
        L.eho_triangle_annot.argtypes = [_u32p, ctypes.c_uint32, _u64p, _u32p, _u64p]
        L.eho_mlp_loss_grad.restype = ctypes.c_double
        L.eho_mlp_loss_grad.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), _f64p, _f64p, _f64p,
                                        ctypes.c_int, ctypes.c_void_p]
        _lib = L
    return _lib


# ------------------------------------------------------------- generators
def rmat_thresholds(a=0.57, b=0.19, c=0.19):
    t = np.zeros(3, np.uint32)
    lib().eho_rmat_thresholds(a, b, c, t)
    return t


def gen_er(seed, n, m):
    u = np.empty(m, np.uint32)
    v = np.empty(m, np.uint32)
    lib().eho_gen_er(seed, n, m, u, v)
    return u, v


def gen_rmat(seed, scale, m, a=0.57, b=0.19, c=0.19):
    u = np.empty(m, np.uint32)
    v = np.empty(m, np.uint32)
    lib().eho_gen_rmat(seed, scale, m, rmat_thresholds(a, b, c), u, v)
    return u, v


def chunglu_cdf(n, gamma):
    cdf = np.empty(n, np.uint64)
    lib().eho_chunglu_cdf(n, gamma, cdf)
    return cdf


def gen_chunglu(seed, n, m, gamma):
    u = np.empty(m, np.uint32)
    v = np.empty(m, np.uint32)
    lib().eho_gen_chunglu(seed, n, m, chunglu_cdf(n, gamma), u, v)
    return u, v


def preprocess(u, v, symmetric=False):
    u = np.ascontiguousarray(u, np.uint32)
    v = np.ascontiguousarray(v, np.uint32)
    m = len(u)
    cap = max(1, 2 * m if symmetric else m)
    s = np.empty(cap, np.uint32)
    d = np.empty(cap, np.uint32)
    nodes = ctypes.c_uint32(0)
    r = lib().eho_preprocess(u, v, m, 1 if symmetric else 0, s, d, ctypes.byref(nodes))
    return s[:r].copy(), d[:r].copy(), nodes.value


# ------------------------------------------------------------------- trie
class Trie:
    """Two-level trie as sorted head + CSR of child sets."""

    def __init__(self, c0, c1):
        c0 = np.ascontiguousarray(c0, np.uint32)
        c1 = np.ascontiguousarray(c1, np.uint32)
        n = len(c0)
        head = np.empty(max(1, n), np.uint32)
        off = np.empty(max(1, n) + 1, np.uint64)
        vals = np.empty(max(1, n), np.uint32)
        nh = ctypes.c_uint32(0)
        r = lib().eho_trie_build(c0, c1, n, head, off, vals, ctypes.byref(nh))
        self.head = head[: nh.value].copy()
        self.off = off[: nh.value + 1].copy()
        self.vals = vals[:r].copy()

    @property
    def n_head(self):
        return len(self.head)

    def child(self, i):
        return self.vals[self.off[i]: self.off[i + 1]]

    def layouts(self):
        """hybrid layout code per child set (0 = RANGE_BITSET, 1 = UINTEGER)."""
        L = lib()
        return np.array([L.eho_hybrid_type(np.ascontiguousarray(self.child(i)), len(self.child(i)))
                         for i in range(self.n_head)], np.uint8)

    def _args(self):
        return (self.head, self.n_head, self.off, self.vals)

    def triangle(self):
        return int(lib().eho_triangle(*self._args()))

    def clique4(self):
        return int(lib().eho_clique4(*self._args()))

    def lollipop(self):
        return int(lib().eho_lollipop(*self._args()))

    def barbell(self):
        return int(lib().eho_barbell(*self._args()))

    def path2(self):
        """PathAgg(;z) :- Edge(a,b),Edge(b,c) COUNT in the plan order [a,b,c]
        (oracle/generated_bags.hpp): sum over rows (a,b) whose b heads a set
        of |N(b)|, modulo 2^64."""
        deg = np.zeros(int(max(self.head.max(initial=0), self.vals.max(initial=0))) + 1, np.uint64)
        deg[self.head] = np.diff(self.off).astype(np.uint64)
        return int(deg[self.vals].sum(dtype=np.uint64)) if len(self.vals) else 0

    def clique4_sel(self, v):
        """FliqueSelAgg: 4-cliques (a,b,c,d) with (a,v) in the relation."""
        return int(lib().eho_clique4_sel(*self._args(), v))

    def barbell_sel(self, v):
        """BarbellSelAgg: barbells joined through the selected vertex p = v."""
        return int(lib().eho_barbell_sel(*self._args(), v))

    def triangle_tuples(self):
        """Triangle(a,b,c) rows in (a,b,c) order, as an (n, 3) uint32 array."""
        L = lib()
        n = int(L.eho_triangle_list(*self._args(), np.zeros(1, np.uint32), np.zeros(1, np.uint32),
                                    np.zeros(1, np.uint32), 0))
        a = np.empty(max(n, 1), np.uint32)
        b = np.empty(max(n, 1), np.uint32)
        c = np.empty(max(n, 1), np.uint32)
        L.eho_triangle_list(*self._args(), a, b, c, n)
        return np.stack([a[:n], b[:n], c[:n]], 1)

    def triangle_projection(self):
        """TriangleProj(a,b) :- Edge(a,b),Edge(b,c),Edge(a,c) as the
        reference plans it: attributes that are neither materialized,
        selected nor aggregated are dropped from the loop nest
        (query_compiler/.../codegen/query/QueryPlan.scala:245), so c is never
        intersected and the rows are (a,b) with b in N(a) ∩ head, in trie
        order."""
        a = np.repeat(self.head, np.diff(self.off).astype(np.int64))
        keep = np.isin(self.vals, self.head)
        return np.stack([a[keep], self.vals[keep]], 1)

    def triangle_per_vertex(self):
        per = np.empty(max(1, self.n_head), np.uint64)
        lib().eho_triangle_per_vertex(*self._args(), per)
        return per[: self.n_head]


def hybrid_type(a):
    a = np.ascontiguousarray(a, np.uint32)
    return int(lib().eho_hybrid_type(a, len(a)))


def range_bitset(a):
    a = np.ascontiguousarray(a, np.uint32)
    nb = int(lib().eho_range_bitset_bytes(a, len(a)))
    out = np.zeros(max(nb, 1), np.uint8)
    lib().eho_range_bitset_build(a, len(a), out)
    return out[:nb]


def block_bitset(a):
    """block_bitset::build (layouts/block_bitset.hpp:112-131): per non-empty
    256-value block, [u32 block id][u32 index of its first element][4 x u64]."""
    a = np.ascontiguousarray(a, np.uint32)
    out = bytearray()
    i = 0
    while i < len(a):
        bid = int(a[i]) >> 8
        j = i
        words = [0, 0, 0, 0]
        while j < len(a) and (int(a[j]) >> 8) == bid:
            x = int(a[j]) & 255
            words[x >> 6] |= 1 << (x & 63)
            j += 1
        out += np.array([bid, i], np.uint32).tobytes() + np.array(words, np.uint64).tobytes()
        i = j
    return np.frombuffer(bytes(out), np.uint8)


def intersect(a, b):
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(b, np.uint32)
    out = np.empty(max(1, min(len(a), len(b))), np.uint32)
    c = lib().eho_intersect(a, len(a), b, len(b), out.ctypes.data)
    return out[:c].copy()


def mlp_loss_grad(dims, params, x, y):
    dims_c = (ctypes.c_int * len(dims))(*dims)
    params = np.ascontiguousarray(params, np.float64)
    grad = np.zeros_like(params)
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    loss = lib().eho_mlp_loss_grad(len(dims) - 1, dims_c, params, x, y, x.shape[0], grad.ctypes.data)
    return loss, grad


# ------------------------------------------------------- reference engine
def write_edge_file(path, src, dst):
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    with open(path, "wb") as f:
        f.write(b"EHEDGE01")
        f.write(np.uint64(len(src)).tobytes())
        f.write(src.tobytes())
        f.write(dst.tobytes())


def ref_available():
    return os.path.exists(REF_BIN)


def ref_query(mode, edges_path, repeats=1, threads=None, timeout=None, value=None):
    """Run the reference engine on an edge file; returns its JSON dict.
    `value` is the selection literal of the *_sel modes."""
    env = dict(os.environ)
    if threads:
        env["EH_REF_THREADS"] = str(threads)
    args = [REF_BIN, mode, edges_path, str(repeats)] + ([] if value is None else [str(int(value))])
    with tempfile.TemporaryDirectory() as td:
        env["TMPDIR"] = td
        out = subprocess.run(args, env=env, capture_output=True, text=True, timeout=timeout, check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def ref_query_edges(mode, src, dst, repeats=1, threads=None, timeout=None, value=None):
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "edges.bin")
        write_edge_file(p, src, dst)
        return ref_query(mode, p, repeats, threads, timeout, value)


# ---------------------------------------------------- dictionary encoding
VALUE_TYPES = {"uint32": (0, np.uint32), "int32": (1, np.int32), "int64": (2, np.int64), "float32": (3, np.float32)}


def encoding(cols, value_type):
    """Encoding<T>::build over every column, then encode_column per column
    (storage_engine/src/Encoding.cpp:21-48): keys in ascending value order
    over the distinct values (std::set order; -0.0 and +0.0 are one value).
    Returns (key_to_value, [keys per column])."""
    dt = VALUE_TYPES[value_type][1]
    cols = [np.ascontiguousarray(c, dt) for c in cols]
    allv = np.concatenate(cols) if cols else np.zeros(0, dt)
    if value_type == "float32":
        allv = np.where(allv == 0, np.float32(0), allv).astype(dt)
        assert not np.isnan(allv).any()
    values = np.unique(allv)
    keys = [np.searchsorted(values, np.where(c == 0, 0, c).astype(dt) if value_type == "float32" else c)
            .astype(np.uint32) for c in cols]
    return values, keys


def ref_encoding(cols, value_type):
    """The reference's own Encoding<T> (oracle/_ref/eh_ref encode)."""
    code, dt = VALUE_TYPES[value_type]
    cols = [np.ascontiguousarray(c, dt) for c in cols]
    with tempfile.TemporaryDirectory() as td:
        inp, outp = os.path.join(td, "cols.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.array([code, len(cols)], np.uint32).tobytes())
            for c in cols:
                f.write(np.uint64(len(c)).tobytes())
                f.write(c.tobytes())
        subprocess.run([REF_BIN, "encode", inp, outp], check=True, capture_output=True,
                       env=dict(os.environ, TMPDIR=td))
        buf = open(outp, "rb").read()
    nd = int(np.frombuffer(buf, np.uint32, 1, 0)[0])
    pos = 4
    values = np.frombuffer(buf, dt, nd, pos).copy()
    pos += nd * np.dtype(dt).itemsize
    keys = []
    for c in cols:
        keys.append(np.frombuffer(buf, np.uint32, len(c), pos).copy())
        pos += 4 * len(c)
    return values, keys


# ------------------------------------------- reference on-disk trie format
# Trie<A,M>::save / load (storage_engine/src/Trie.cpp:15-75),
# ParMemoryBuffer::save / load (src/utils/ParMemoryBuffer.cpp:64-100),
# MemoryBuffer::save / load (src/utils/MemoryBuffer.cpp:104-172):
#   <dir>/ram/trieinfo.bin   bool annotated, A annotation, size_t num_rows,
#                            size_t num_columns, size_t num_buffers,
#                            size_t head size, size_t size[num_buffers]
#   <dir>/ram/data_head.bin, data_<i>.bin   "<size> <offset> " + size bytes
# A block (TrieBlock<hybrid,M>, trie/TrieBlock.hpp): bool is_sparse, then a
# Set<hybrid> header (u32 cardinality, u32 range = last value, size_t
# number_of_bytes, u8 type; 24 bytes), the set's bytes, then (head) one
# NextLevel {int index; size_t offset} per element (sparse) or per value
# 0..range (dense), common::is_sparse(cardinality, range) deciding.

def _read_buffer(path):
    with open(path, "rb") as f:
        raw = f.read()
    sp1 = raw.index(b" ")
    sp2 = raw.index(b" ", sp1 + 1)
    size = int(raw[:sp1])
    return np.frombuffer(raw, np.uint8, size, sp2 + 1)


def _is_sparse(length, rng):
    return (rng / length) > 128.0 if length > 2 else True


def _set_values(buf, off):
    card, rng = np.frombuffer(buf, np.uint32, 2, off + 1)
    nb = int(np.frombuffer(buf, np.uint64, 1, off + 9)[0])
    ty = int(buf[off + 17])
    data = buf[off + 25: off + 25 + nb]
    if card == 0:
        vals = np.zeros(0, np.uint32)
    elif ty == 1:  # UINTEGER
        vals = data[: 4 * int(card)].copy().view(np.uint32)
    elif ty == 0:  # RANGE_BITSET [u64 start][u64 words x W][u32 rank x W]
        w = (nb - 8) // 12
        start = int(data[:8].copy().view(np.uint64)[0])
        words = data[8: 8 + 8 * w].copy().view(np.uint64)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little").reshape(w, 64)
        wi, bi = np.nonzero(bits)
        vals = ((start + wi) * 64 + bi).astype(np.uint32)
    elif ty == 3:  # BLOCK_BITSET [u32 id][u32 rank][4 x u64] per block
        nblk = nb // 40
        rec = data[: 40 * nblk].copy()
        ids = rec.reshape(nblk, 40)[:, :4].copy().view(np.uint32).ravel()
        words = rec.reshape(nblk, 40)[:, 8:].copy().view(np.uint64).reshape(nblk, 4)
        bits = np.unpackbits(words.view(np.uint8), bitorder="little").reshape(nblk, 256)
        bi, vi = np.nonzero(bits)
        vals = (ids[bi].astype(np.uint64) * 256 + vi).astype(np.uint32)
    else:
        raise ValueError("unknown set type %d" % ty)
    assert len(vals) == card
    return vals, int(card), int(rng), nb, ty


def read_reference_trie(dirpath):
    """A two-level trie the reference saved: (head, off, vals, types) with
    types[i] the stored layout of child set i and types[-1] the head's."""
    ram = os.path.join(dirpath, "ram")
    info = open(os.path.join(ram, "trieinfo.bin"), "rb").read()
    for sa in (8, 4):
        nbuf = int(np.frombuffer(info, np.uint64, 1, 1 + sa + 16)[0])
        if len(info) == 1 + sa + 32 + 8 * nbuf:
            break
    else:
        raise ValueError("unrecognised trieinfo.bin")
    ncols = int(np.frombuffer(info, np.uint64, 1, 1 + sa + 8)[0])
    assert ncols == 2, "two-level tries only"
    bufs = [_read_buffer(os.path.join(ram, "data_%d.bin" % i)) for i in range(nbuf)]
    bufs.append(_read_buffer(os.path.join(ram, "data_head.bin")))
    head, card, rng, nb, hty = _set_values(bufs[nbuf], 0)
    nxt = 25 + nb
    dense = not _is_sparse(card, rng)
    off = [0]
    vals, types = [], []
    for i, v in enumerate(head):
        e = int(v) if dense else i
        idx = int(np.frombuffer(bufs[nbuf], np.int32, 1, nxt + 16 * e)[0])
        boff = int(np.frombuffer(bufs[nbuf], np.uint64, 1, nxt + 16 * e + 8)[0])
        if idx < 0:
            child, ty = np.zeros(0, np.uint32), 1
        else:
            child, _, _, _, ty = _set_values(bufs[idx], boff)
        vals.append(child)
        types.append(ty)
        off.append(off[-1] + len(child))
    types.append(hty)
    return (head.astype(np.uint32), np.array(off, np.uint64),
            np.concatenate(vals).astype(np.uint32) if vals else np.zeros(0, np.uint32), np.array(types, np.uint8))


def _set_bytes_hybrid(a):
    """hybrid::build (layouts/hybrid.hpp:103-111): bytes and type"""
    if len(a) == 0:
        return b"", 1
    if hybrid_type(a) == 0:
        return range_bitset(a).tobytes(), 0
    return np.ascontiguousarray(a, np.uint32).tobytes(), 1


def _block(a, with_next=None):
    a = np.ascontiguousarray(a, np.uint32)
    data, ty = _set_bytes_hybrid(a)
    last = int(a[-1]) if len(a) else 0
    hdr = bytes([1 if _is_sparse(len(a), last) else 0])
    hdr += np.array([len(a), last], np.uint32).tobytes() + np.uint64(len(data)).tobytes() + bytes([ty]) + bytes(7)
    return hdr + data


def write_reference_trie(dirpath, head, off, vals, rows, num_threads):
    """The layout this project writes (and its device saver writes byte for
    byte): child blocks in num_threads buffers, head entries split into
    contiguous chunks per buffer; the head block and its NextLevel array in
    the head buffer; trieinfo of a Trie<void*,ParMemoryBuffer>."""
    ram = os.path.join(dirpath, "ram")
    os.makedirs(ram, exist_ok=True)
    nh = len(head)
    per = (nh + num_threads - 1) // num_threads if nh else 0
    bufs = [bytearray() for _ in range(num_threads)]
    loc = []
    for i in range(nh):
        b = min(i // per, num_threads - 1) if per else 0
        loc.append((b, len(bufs[b])))
        bufs[b] += _block(vals[off[i]: off[i + 1]])
    hb = bytearray(_block(head))
    last = int(head[-1]) if nh else 0
    dense = not _is_sparse(nh, last)
    n_next = (last + 1) if dense else nh
    nxt = np.zeros(n_next, dtype=[("index", "<i4"), ("pad", "<u4"), ("offset", "<u8")])
    nxt["index"] = -1
    for i in range(nh):
        e = int(head[i]) if dense else i
        nxt["index"][e] = loc[i][0]
        nxt["offset"][e] = loc[i][1]
    hb += nxt.tobytes()

    def put(name, b):
        with open(os.path.join(ram, name), "wb") as f:
            f.write(b"%d %d " % (len(b), len(b)))
            f.write(bytes(b))
    put("data_head.bin", hb)
    for i, b in enumerate(bufs):
        put("data_%d.bin" % i, b)
    info = bytes([0]) + np.uint64(0).tobytes() + np.array([rows, 2, num_threads, len(hb)], np.uint64).tobytes()
    info += np.array([len(b) for b in bufs], np.uint64).tobytes()
    with open(os.path.join(ram, "trieinfo.bin"), "wb") as f:
        f.write(info)


def ref_save(src, dst, dirpath, threads):
    """The reference engine's own Trie::save of the Edge trie into dirpath."""
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "edges.bin")
        write_edge_file(p, src, dst)
        subprocess.run([REF_BIN, "save", p, dirpath], check=True, capture_output=True,
                       env=dict(os.environ, EH_REF_THREADS=str(threads), TMPDIR=td))


def ref_load_triangle(dirpath, threads):
    """Trie::load of a saved trie by the reference engine, then TriangleAgg."""
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run([REF_BIN, "load_triangle", dirpath], check=True, capture_output=True, text=True,
                             env=dict(os.environ, EH_REF_THREADS=str(threads), TMPDIR=td)).stdout
    return json.loads(out.strip().splitlines()[-1])

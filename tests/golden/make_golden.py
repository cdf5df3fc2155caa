"""Regenerates the golden fixtures in this directory from the reference.

    python tests/golden/make_golden.py        (needs the reference checkout, $EH_REFERENCE or ../reference, and
                                               oracle/_ref/eh_ref, built by
                                               `make -C oracle`)

Writes:
  facebook.npz   the reference's own test graphs, test/graph/data/
                 facebook_pruned.tsv, facebook_duplicated.tsv, simple.tsv
                 (sorted rows, compressed)
  golden.json    known answers: the counts the reference's tests assert
                 (test/graph/travis.py) and counts the compiled reference
                 engine returns on seeded synthetic graphs
  setops.npz     per-pair ops::set_intersect results of the reference on
                 seeded random sets covering the layout pairs and edges
  triedump.npz   per-set layout, cardinality, range and bytes of reference
                 tries (Trie.cpp:380-510 + hybrid::build)
The GPU box has no reference tree; tests read only these files.
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

REF = O.reference_dir()
DATA = os.path.join(REF, "test", "graph", "data")


def load_tsv(name):
    a = np.loadtxt(os.path.join(DATA, name), dtype=np.uint32).reshape(-1, 2)
    order = np.lexsort((a[:, 1], a[:, 0]))
    return a[order]


def ref(mode, src, dst, repeats=1):
    return O.ref_query_edges(mode, src, dst, repeats=repeats)


def norm_bytes(layout, raw):
    """Reference range_bitset bytes leave the rank of an empty word
    unwritten (range_bitset.hpp:140-151); zero those entries."""
    raw = np.array(raw, np.uint8)
    if layout == 0 and len(raw) >= 8:
        w = (len(raw) - 8) // 12
        words = raw[8: 8 + 8 * w].view(np.uint64)
        rank = raw[8 + 8 * w: 8 + 12 * w].view(np.uint32).copy()
        rank[words == 0] = 0
        raw = np.concatenate([raw[: 8 + 8 * w], rank.view(np.uint8)])
    return raw


def trie_dump(src, dst):
    with tempfile.TemporaryDirectory() as td:
        e = os.path.join(td, "e.bin")
        o = os.path.join(td, "dump.bin")
        O.write_edge_file(e, src, dst)
        subprocess.check_call([O.REF_BIN, "trie_dump", e, o], stdout=subprocess.DEVNULL, env=dict(os.environ, TMPDIR=td))
        buf = open(o, "rb").read()
    pos = 0

    def read_set():
        nonlocal pos
        ty = buf[pos]
        card, rng = np.frombuffer(buf, np.uint32, 2, pos + 1)
        nb = int(np.frombuffer(buf, np.uint64, 1, pos + 9)[0])
        raw = np.frombuffer(buf, np.uint8, nb, pos + 17)
        pos += 17 + nb
        return int(ty), int(card), int(rng), norm_bytes(ty, raw)

    head = read_set()
    vals, types, cards, ranges, digests = [], [], [], [], []
    while pos < len(buf):
        v = int(np.frombuffer(buf, np.uint32, 1, pos)[0])
        present = buf[pos + 4]
        pos += 5
        if not present:
            continue
        ty, card, rng, raw = read_set()
        vals.append(v)
        types.append(ty)
        cards.append(card)
        ranges.append(rng)
        digests.append(np.frombuffer(hashlib.sha1(raw.tobytes()).digest(), np.uint8))
    return head, np.array(vals, np.uint32), np.array(types, np.uint8), np.array(cards, np.uint32), \
        np.array(ranges, np.uint32), np.array(digests, np.uint8).reshape(-1, 20)


def setops_cases(seed=7):
    rng = np.random.default_rng(seed)
    sets = []

    def add(a):
        sets.append(np.unique(np.asarray(a, np.uint32)))

    # edge cases: empty, singletons, len <= 2, word boundary straddles,
    # disjoint ranges, identical sets, dense runs, very uneven sizes
    add([])
    add([5])
    add([63, 64])
    add([0, 1, 2])
    add(np.arange(60, 70))
    add(np.arange(128, 192))
    add(np.arange(0, 4096, 2))
    add(np.arange(1, 4096, 2))
    add(np.arange(10000, 10300))
    add(np.arange(10000, 10300))
    add(np.arange(1 << 20, (1 << 20) + 500, 3))
    for _ in range(60):
        n = int(rng.choice([1, 2, 3, 7, 31, 32, 33, 100, 500, 2000]))
        span = int(rng.choice([n + 1, 2 * n, 64 * n, 200 * n, 5000 * n]))
        base = int(rng.integers(0, 1 << 24))
        add(base + rng.choice(span, size=min(n, span), replace=False))
    pairs = []
    k = len(sets)
    for i in range(k):
        for j in range(k):
            if (i * 31 + j * 17) % 5 == 0 or i < 11 and j < 11:
                pairs.append((i, j))
    return sets, np.array(pairs, np.uint32)


def run_setops(sets, pairs):
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "pairs.bin")
        out = os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.uint64(len(pairs)).tobytes())
            for a, b in pairs:
                for s in (sets[a], sets[b]):
                    f.write(np.uint32(len(s)).tobytes())
                    f.write(np.asarray(s, np.uint32).tobytes())
        subprocess.check_call([O.REF_BIN, "setops", inp, out], stdout=subprocess.DEVNULL)
        buf = open(out, "rb").read()
    pos = 0
    typeA, counts, rtypes, elems, elem_off, abytes, abytes_off = [], [], [], [], [0], [], [0]
    for _ in range(len(pairs)):
        ta, tb = buf[pos], buf[pos + 1]
        nba = int(np.frombuffer(buf, np.uint64, 1, pos + 2)[0])
        raw = norm_bytes(ta, np.frombuffer(buf, np.uint8, nba, pos + 10))
        pos += 10 + nba
        cnt = int(np.frombuffer(buf, np.uint64, 1, pos)[0])
        tc = buf[pos + 8]
        nout = int(np.frombuffer(buf, np.uint32, 1, pos + 9)[0])
        out_e = np.frombuffer(buf, np.uint32, nout, pos + 13)
        pos += 13 + 4 * nout
        typeA.append(ta)
        counts.append(cnt)
        rtypes.append(tc)
        elems.append(out_e)
        elem_off.append(elem_off[-1] + nout)
        abytes.append(raw)
        abytes_off.append(abytes_off[-1] + len(raw))
    return dict(typeA=np.array(typeA, np.uint8), counts=np.array(counts, np.uint64),
                rtypes=np.array(rtypes, np.uint8),
                elems=np.concatenate(elems) if elems else np.zeros(0, np.uint32),
                elem_off=np.array(elem_off, np.uint64),
                abytes=np.concatenate(abytes) if abytes else np.zeros(0, np.uint8),
                abytes_off=np.array(abytes_off, np.uint64))


def main():
    if not O.ref_available():
        O.build(ref=True)
    golden = {"_source": {
        "travis": "reference test/graph/travis.py (asserted counts)",
        "reference_engine": "oracle/_ref/eh_ref: the reference storage engine compiled from its sources, "
                            "driven by generated-shape query code"}}
    pruned = load_tsv("facebook_pruned.tsv")
    dup = load_tsv("facebook_duplicated.tsv")
    simple = load_tsv("simple.tsv")
    np.savez_compressed(os.path.join(HERE, "facebook.npz"), pruned=pruned, duplicated=dup, simple=simple)
    golden["travis"] = {
        "facebook_pruned": {"triangle": 1612010, "clique4": 30004668},       # travis.py:212, :253
        "facebook_duplicated": {"lollipop": 1426911480, "barbell": 20371831447136},  # travis.py:29, :70
    }
    eng = {}
    # path2 (Edge(a,b),Edge(b,c) COUNT) is a body no device plan runs: the
    # C++ layer's host loop is checked on it
    for name, a, modes in (("facebook_pruned", pruned, ("triangle", "clique4", "path2")),
                           ("facebook_duplicated", dup, ("triangle", "lollipop", "barbell", "clique4", "path2")),
                           ("simple", simple, ("triangle", "lollipop", "barbell", "clique4", "path2"))):
        eng[name] = {m: ref(m, a[:, 0], a[:, 1])["count_u64"] for m in modes}
    # seeded synthetic graphs, preprocessed by the oracle (bit-identical to
    # the device pipeline, checked by the GPU tests)
    synth = {}
    specs = [("er_16384_131072_s1", lambda: O.gen_er(1, 16384, 131072), ("triangle", "clique4"), False),
             ("rmat_s12_ef16_s3", lambda: O.gen_rmat(3, 12, 16 << 12), ("triangle", "clique4"), False),
             ("rmat_s16_ef16_s42", lambda: O.gen_rmat(42, 16, 16 << 16), ("triangle", "clique4"), False),
             ("rmat_s14_ef16_s5_sym", lambda: O.gen_rmat(5, 14, 16 << 14), ("triangle", "lollipop", "barbell", "clique4"),
              True),
             ("chunglu_n65536_d32_g2.1_s9_sym", lambda: O.gen_chunglu(9, 65536, 65536 * 16, 2.1),
              ("triangle", "lollipop", "barbell"), True)]
    for name, gen, modes, sym in specs:
        u, v = gen()
        s, d, nn = O.preprocess(u, v, symmetric=sym)
        synth[name] = {"rows": int(len(s)), "nodes": int(nn),
                       "sha1": hashlib.sha1(s.tobytes() + d.tobytes()).hexdigest()}
        for m in modes:
            synth[name][m] = ref(m, s, d)["count_u64"]
        print(name, synth[name], flush=True)
    if os.environ.get("EH_GOLDEN_FULL", "1") == "1":
        u, v = O.gen_rmat(42, 22, 16 << 22)
        s, d, nn = O.preprocess(u, v)
        del u, v
        r = ref("triangle", s, d)
        synth["rmat_s22_ef16_s42"] = {"rows": int(len(s)), "nodes": int(nn),
                                      "sha1": hashlib.sha1(s.tobytes() + d.tobytes()).hexdigest(),
                                      "triangle": r["count_u64"], "ref_query_s": r["query_s_median"],
                                      "ref_threads": r["threads"]}
        print("rmat22", synth["rmat_s22_ef16_s42"], flush=True)
    golden["reference_engine"] = eng
    golden["synthetic"] = synth
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)

    sets, pairs = setops_cases()
    res = run_setops(sets, pairs)
    lens = np.array([len(s) for s in sets], np.uint64)
    off = np.zeros(len(sets) + 1, np.uint64)
    np.cumsum(lens, out=off[1:])
    np.savez_compressed(os.path.join(HERE, "setops.npz"), set_elems=np.concatenate(sets), set_off=off,
                        pairs=pairs, **res)

    dumps = {}
    u, v = O.gen_er(1, 16384, 131072)
    es, ed, _ = O.preprocess(u, v)
    for name, s, d in (("facebook_pruned", pruned[:, 0], pruned[:, 1]), ("er", es, ed),
                       ("facebook_duplicated", dup[:, 0], dup[:, 1])):
        head, vals, types, cards, ranges, digests = trie_dump(s, d)
        dumps[name + "_head_type"] = np.array([head[0]], np.uint8)
        dumps[name + "_head_digest"] = np.frombuffer(hashlib.sha1(head[3].tobytes()).digest(), np.uint8)
        dumps[name + "_vals"] = vals
        dumps[name + "_types"] = types
        dumps[name + "_cards"] = cards
        dumps[name + "_ranges"] = ranges
        dumps[name + "_digests"] = digests
    np.savez_compressed(os.path.join(HERE, "triedump.npz"), **dumps)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()

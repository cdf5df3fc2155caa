"""A small, self-checking triangle COUNT case for profiler captures.

    python -m emptyheaded_b200.profile_case --scale 20 --repeat 2

Builds an R-MAT trie on the device (edge factor 16, a/b/c/d =
0.57/0.19/0.19/0.05, seed 42, degree-ordered src < dst) and runs the
triangle query `repeat` times, printing the count and device times.  At
scale 20 the trie (~0.4 GB with its reverse level) is larger than L2 and
the device holds well under the few-GB limit a full-metric capture allows.
"""
import argparse
import json
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--layout", default="heuristic", choices=["heuristic", "uint", "bitset", "block"])
    ap.add_argument("--warps", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--smem-words", type=int, default=0)
    a = ap.parse_args(argv)
    import emptyheaded_b200 as E

    u, v = E.gen_rmat(42, a.scale, 16 << a.scale)
    s, d, _ = E.preprocess(u, v)
    u.free()
    v.free()
    forced = {"uint": E.UINTEGER, "bitset": E.RANGE_BITSET, "block": E.BLOCK_BITSET}.get(a.layout)
    t = E.Trie(s, d, policy=E.FORCED if forced is not None else E.HEURISTIC,
               forced=forced if forced is not None else E.UINTEGER, max_bitset_bytes=1 << 50)
    out = []
    for _ in range(a.repeat):
        c, st = t.count("triangle", warps=a.warps, chunk=a.chunk, smem_words=a.smem_words, stats=True)
        out.append({"count": c, "query_ms": st["query_ms"], "kernel_ms": st["kernel_ms"]})
    print(json.dumps({"scale": a.scale, "layout": a.layout, "info": t.info(), "runs": out}))
    return 0


if __name__ == "__main__":
    sys.exit(main())

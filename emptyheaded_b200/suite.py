"""Device timings of every measured workload of the hot path, one JSON line each.

    python -m emptyheaded_b200.suite [--only NAME ...] [--repeat 5]

Workloads (seeded synthetic inputs built on the device; counts are checked
against the reference engine's, tests/golden/golden.json, where recorded):
  er            ER n=16,384, m=131,072 samples, seed 1, triangle COUNT
  rmat22        R-MAT scale 22 (edge factor 16, seed 42), triangle COUNT
  batch256      256 R-MAT graphs (scales 10..18), triangle COUNT, one
                CUDA-graph replay for the whole batch
  rmat20_c4     R-MAT scale 20 (seed 42), 4-clique COUNT
  chunglu23     Chung-Lu n=2^23, average degree 32, exponent 2.1,
                symmetrised: triangle, lollipop and barbell COUNT
Times are the engine's own CUDA-event query times (plan + kernels + result
to host) with the trie resident, median of `repeat` runs after one warm-up.
"""
import argparse
import json
import os
import statistics
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden", "golden.json")


def _golden():
    if os.path.exists(GOLDEN):
        with open(GOLDEN) as f:
            return json.load(f)
    return {}


def _time(fn, repeat):
    fn()  # warm-up
    ms, val = [], None
    for _ in range(repeat):
        val, st = fn()
        ms.append(st["query_ms"])
    return val, statistics.median(ms)


def _count(t, q, repeat):
    return _time(lambda: t.count(q, stats=True), repeat)


def run(names, repeat, E, W):
    g = _golden()
    syn = g.get("synthetic", {})
    out = []

    def emit(rec):
        out.append(rec)
        print(json.dumps(rec), flush=True)

    if "er" in names:
        u, v = E.gen_er(1, 16384, 131072)
        s, d, _ = E.preprocess(u, v)
        t = E.Trie(s, d)
        c, ms = _count(t, "triangle", repeat)
        want = syn.get("er_16384_131072_s1", {}).get("triangle")
        emit({"workload": "er", "query": "triangle", "count": c, "ok": want in (None, c), "ms": ms,
              "rows": t.info()["rows"]})
        t.free()
    if "rmat22" in names:
        t = W.build_rmat_trie(E, 22, 42)
        c, ms = _count(t, "triangle", repeat)
        want = syn.get("rmat_s22_ef16_s42", {}).get("triangle")
        emit({"workload": "rmat22", "query": "triangle", "count": c, "ok": want in (None, c), "ms": ms,
              "rows": t.info()["rows"], "build_ms": t.info()["build_ms"]})
        t.free()
    if "batch256" in names:
        tries = [W.build_rmat_trie(E, sc, sd) for sc, sd in W.batch256_spec()]
        b = E.Batch(tries)
        res, ms = _time(lambda: b.run(stats=True), repeat)
        want = [x["triangle"] for x in g.get("batch256", [])]
        emit({"workload": "batch256", "query": "triangle", "count": int(sum(int(x) for x in res)),
              "ok": (not want) or [int(x) for x in res] == want, "ms": ms,
              "rows": int(sum(x.info()["rows"] for x in tries)), "launches_per_run": 1})
        b.free()
        for x in tries:
            x.free()
    if "rmat20_c4" in names:
        t = W.build_rmat_trie(E, 20, 42)
        c, ms = _count(t, "clique4", repeat)
        want = syn.get("rmat_s20_ef16_s42", {}).get("clique4")
        emit({"workload": "rmat20_c4", "query": "clique4", "count": c, "ok": want in (None, c), "ms": ms,
              "rows": t.info()["rows"]})
        t.free()
    if "chunglu23" in names:
        t = W.build_chunglu_trie(E)
        for q in ("triangle", "lollipop", "barbell"):
            c, ms = _count(t, q, repeat)
            emit({"workload": "chunglu23", "query": q, "count": c, "ok": None, "ms": ms, "rows": t.info()["rows"],
                  "max_set": t.info()["max_set"]})
        t.free()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=["er", "rmat22", "batch256", "rmat20_c4", "chunglu23"])
    ap.add_argument("--repeat", type=int, default=5)
    a = ap.parse_args(argv)
    import emptyheaded_b200 as E
    from emptyheaded_b200 import workloads as W
    recs = run(a.only, a.repeat, E, W)
    return 0 if all(r["ok"] in (None, True) for r in recs) else 1


if __name__ == "__main__":
    sys.exit(main())

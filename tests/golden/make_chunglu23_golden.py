"""Adds the full-size barbell / lollipop configuration to golden.json:
Chung-Lu n = 2^23, average degree 32 (n * 16 samples), exponent 2.1,
seed 9, symmetrised (the oracle's generator and preprocessing), counted by
the reference engine itself (oracle/_ref/eh_ref).

    python tests/golden/make_chunglu23_golden.py   (needs the reference checkout, $EH_REFERENCE or ../reference, and
                                                    oracle/_ref/eh_ref; about
                                                    10 minutes on 8 cores)"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def main():
    n = 1 << 23
    u, v = O.gen_chunglu(9, n, n * 16, 2.1)
    s, d, nn = O.preprocess(u, v, symmetric=True)
    del u, v
    g = {"rows": int(len(s)), "nodes": int(nn), "sha1": hashlib.sha1(s.tobytes() + d.tobytes()).hexdigest()}
    for mode in ("triangle", "lollipop", "barbell"):
        r = O.ref_query_edges(mode, s, d, repeats=1, timeout=3600)
        g[mode] = r["count_u64"]
        g["ref_%s_query_s" % mode] = r["query_s"][0]
        g["ref_threads"] = r["threads"]
        print(mode, r["count_u64"], r["query_s"][0], flush=True)
    path = os.path.join(HERE, "golden.json")
    with open(path) as f:
        golden = json.load(f)
    golden["synthetic"]["chunglu_n8388608_d32_g2.1_s9_sym"] = g
    with open(path, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

"""Adds the 256-graph batch to golden.json: for every graph of
emptyheaded_b200.workloads.batch256_spec() the triangle count of the
reference engine (oracle/_ref/eh_ref) on the oracle-preprocessed rows, and
the rows' sha1.  Needs the reference checkout ($EH_REFERENCE or ../reference beside the repository; built oracle); run after
make_golden.py."""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from emptyheaded_b200.workloads import ABCD, EDGE_FACTOR, batch256_spec  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    path = os.path.join(HERE, "golden.json")
    with open(path) as f:
        golden = json.load(f)
    rows = []
    for scale, seed in batch256_spec():
        u, v = O.gen_rmat(seed, scale, EDGE_FACTOR << scale, *ABCD)
        s, d, nn = O.preprocess(u, v)
        r = O.ref_query_edges("triangle", s, d)
        rows.append({"scale": scale, "seed": seed, "rows": int(len(s)),
                     "sha1": hashlib.sha1(s.tobytes() + d.tobytes()).hexdigest(), "triangle": r["count_u64"]})
    golden["batch256"] = rows
    with open(path, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print("batch256:", len(rows), "graphs, total triangles", sum(x["triangle"] for x in rows))


if __name__ == "__main__":
    main()

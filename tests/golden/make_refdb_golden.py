"""Writes refdb.npz: tries saved by the reference engine itself
(Trie::save, storage_engine/src/Trie.cpp:15-35, through oracle/_ref/eh_ref
save), file by file, for the loader tests.

    python tests/golden/make_refdb_golden.py   (needs the reference checkout, $EH_REFERENCE or ../reference, and
                                                oracle/_ref/eh_ref)

Entries: facebook_pruned saved with 4 threads, the oriented R-MAT-12 graph
with 2 threads, the symmetric R-MAT-14 graph with 3 threads.  Keys are
"<name>/<file>" (files of <dir>/ram/), plus "<name>/threads"."""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
from oracle import oracle as O  # noqa: E402
from test_oracle import _gen  # noqa: E402


def main():
    fb = np.load(os.path.join(HERE, "facebook.npz"))
    graphs = [("facebook_pruned", fb["pruned"][:, 0], fb["pruned"][:, 1], 4)]
    for name, thr in (("rmat_s12_ef16_s3", 2), ("rmat_s14_ef16_s5_sym", 3)):
        (u, v), sym = _gen(O, name)
        s, d, _ = O.preprocess(u, v, symmetric=sym)
        graphs.append((name, s, d, thr))
    out = {}
    for name, s, d, thr in graphs:
        with tempfile.TemporaryDirectory() as td:
            dd = os.path.join(td, "Edge_0_1")
            O.ref_save(s, d, dd, thr)
            ram = os.path.join(dd, "ram")
            for fn in sorted(os.listdir(ram)):
                out["%s/%s" % (name, fn)] = np.frombuffer(open(os.path.join(ram, fn), "rb").read(), np.uint8)
        out[name + "/threads"] = np.array([thr])
        print(name, "saved with", thr, "threads")
    np.savez_compressed(os.path.join(HERE, "refdb.npz"), **out)


if __name__ == "__main__":
    main()

"""The reference's on-disk trie format on the device path:
eh_trie_load_reference reads tries the reference saved (fixture
tests/golden/refdb.npz, written by its own Trie::save), and
eh_trie_save_reference writes files byte-identical to the oracle's
restatement of the format, which the reference engine loads (checked here
when its compiled driver is present).  Integer data: exact."""
import os

import numpy as np
import pytest

from test_oracle import _gen, _refdb_dirs

pytestmark = pytest.mark.gpu


def _edges(oracle, facebook, name):
    if name == "facebook_pruned":
        p = facebook["pruned"]
        return p[:, 0], p[:, 1]
    (u, v), sym = _gen(oracle, name)
    s, d, _ = oracle.preprocess(u, v, symmetric=sym)
    return s, d


def _files(path):
    ram = os.path.join(path, "ram")
    return {fn: open(os.path.join(ram, fn), "rb").read() for fn in sorted(os.listdir(ram))}


@pytest.mark.parametrize("name", ["facebook_pruned", "rmat_s12_ef16_s3", "rmat_s14_ef16_s5_sym"])
def test_load_reference_saved_trie(eh, oracle, facebook, golden, tmp_path, name):
    path, _ = _refdb_dirs(tmp_path, [name])[name]
    s, d = _edges(oracle, facebook, name)
    ot = oracle.Trie(s, d)
    t = eh.Trie.load_reference(path)
    head, off, vals, lay = t.export()
    np.testing.assert_array_equal(head, ot.head)
    np.testing.assert_array_equal(off, ot.off)
    np.testing.assert_array_equal(vals, ot.vals)
    np.testing.assert_array_equal(lay, ot.layouts())
    assert t.count("triangle") == ot.triangle()
    if name == "facebook_pruned":
        assert t.count("triangle") == golden["travis"]["facebook_pruned"]["triangle"]


@pytest.mark.parametrize("name,threads", [("facebook_pruned", 4), ("rmat_s14_ef16_s5_sym", 3), ("rmat_s12_ef16_s3", 1)])
def test_save_matches_restatement_and_reference_loads(eh, oracle, facebook, tmp_path, name, threads):
    s, d = _edges(oracle, facebook, name)
    ot = oracle.Trie(s, d)
    # device layouts differ from the written ones on purpose: the file takes
    # hybrid::build's layouts whatever the device holds
    t = eh.Trie(s, d, policy=2, forced=3)
    mine = str(tmp_path / "device")
    t.save_reference(mine, threads)
    ref = str(tmp_path / "oracle")
    oracle.write_reference_trie(ref, ot.head, ot.off, ot.vals, len(ot.vals), threads)
    a, b = _files(mine), _files(ref)
    assert sorted(a) == sorted(b)
    for fn in a:
        assert a[fn] == b[fn], fn
    back = eh.Trie.load_reference(mine)
    np.testing.assert_array_equal(back.export()[2], ot.vals)
    assert back.count("triangle") == ot.triangle()
    if oracle.ref_available():
        assert oracle.ref_load_triangle(mine, threads)["count_u64"] == ot.triangle()


def test_round_trip_rmat18(eh, tmp_path):
    """Device save then load of an R-MAT-18 trie (4.2 M rows) keeps every
    row and the triangle count."""
    from emptyheaded_b200 import workloads
    t = workloads.build_rmat_trie(eh, 18, 42)
    want = t.count("triangle")
    head, off, vals, _ = t.export()
    t.save_reference(str(tmp_path / "r18"), 8)
    back = eh.Trie.load_reference(str(tmp_path / "r18"))
    h2, o2, v2, _ = back.export()
    np.testing.assert_array_equal(h2, head)
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(v2, vals)
    assert back.count("triangle") == want


def test_load_errors(eh, tmp_path):
    with pytest.raises(eh.EHError):
        eh.Trie.load_reference(str(tmp_path / "missing"))
    (tmp_path / "bad" / "ram").mkdir(parents=True)
    (tmp_path / "bad" / "ram" / "trieinfo.bin").write_bytes(b"\x00" * 7)
    with pytest.raises(eh.EHError):
        eh.Trie.load_reference(str(tmp_path / "bad"))

"""The C++ layer of include/eh/ (the reference's Trie / TrieBuilder /
TrieIterator / par::reducer API over the C ABI), on the CPU.

The generated bag code of oracle/generated_bags.hpp -- the same source the
reference engine runs in oracle/ref_driver.cpp -- is compiled against the
layer and linked against a CPU test double of the C ABI
(tests/cpp/fake_eh_abi.cpp), so the layer's symbolic pass, plan matching and
replay run here.  Each bag must give the reference's count, and the double's
call log shows which entry the bag went to: the device plans for the bags
they match, the host loop over device set intersections otherwise.  A second
build links the same program against libeh_b200.so (the product): it must
link, and fail cleanly without a GPU."""
import os
import shutil

import pytest

from conftest import compile_dropin, run_dropin, write_facebook_tsvs

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


@pytest.fixture(scope="module")
def build(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("dropin"))
    return {"fake": compile_dropin(d, fake=True), "tsv": write_facebook_tsvs(d), "dir": d}


def _run(build, query, graph, value=None, host_loop=False):
    log = os.path.join(build["dir"], "calls.log")
    if os.path.exists(log):
        os.remove(log)
    env = {"EH_FAKE_LOG": log}
    if host_loop:
        env["EH_DROPIN_HOST_LOOP"] = "1"
    out = run_dropin(build["fake"], query, build["tsv"][graph], value, env)
    calls = open(log).read().split() if os.path.exists(log) else []
    return out, calls


@pytest.mark.parametrize("query,graph,entry", [
    ("triangle", "pruned", "eh_rule_count"),
    ("clique4", "pruned", "eh_rule_count"),
    ("lollipop", "duplicated", "eh_query_weighted_root:lollipop"),
    ("barbell", "duplicated", "eh_query_weighted_root:barbell"),
])
def test_matching_bags_run_as_device_plans(build, golden, query, graph, entry):
    out, calls = _run(build, query, graph)
    assert out["count_u64"] == golden["travis"]["facebook_" + graph][query]
    assert entry in calls
    assert "eh_rule_count:unsupported" not in calls
    if query in ("lollipop", "barbell"):
        assert "eh_triangle_annotation" in calls  # the annotated bag bag_1(a;z)
    # one intersection per outer head build (head ∩ head), none inside the loops
    assert calls.count("eh_set_intersect_batch") <= 2


def test_other_bodies_take_the_host_loop(build, golden):
    """Edge(a,b),Edge(b,c) COUNT: no device plan; the generated loops run on
    the host with each intersection on the device."""
    out, calls = _run(build, "path2", "pruned")
    assert out["count_u64"] == golden["reference_engine"]["facebook_pruned"]["path2"]
    assert "eh_rule_count:unsupported" in calls
    assert calls.count("eh_set_intersect_batch") > 1000


def test_selection_bags(build, golden):
    out, _ = _run(build, "barbell_sel", "duplicated", 6)
    assert out["count_u64"] == golden["travis"]["facebook_duplicated"]["barbell_sel_p6"]


def test_host_loop_gives_the_same_counts(build, golden):
    out, calls = _run(build, "triangle", "pruned", host_loop=True)
    assert out["count_u64"] == golden["travis"]["facebook_pruned"]["triangle"]
    assert "eh_rule_count" not in calls
    out, _ = _run(build, "lollipop", "duplicated", host_loop=True)
    assert out["count_u64"] == golden["travis"]["facebook_duplicated"]["lollipop"]


def test_layer_links_against_the_product_library(tmp_path):
    """Linked against libeh_b200.so, the generated code builds; without a
    GPU every call fails with the library's error, never a CPU answer."""
    exe = compile_dropin(str(tmp_path), fake=False)
    tsv = write_facebook_tsvs(str(tmp_path))["simple"]
    out = run_dropin(exe, "triangle", tsv)
    if "error" in out:
        assert "device" in out["error"].lower() or "cuda" in out["error"].lower()


def test_c_translation_unit_against_the_abi(tmp_path):
    """A plain C99 translation unit includes include/eh_b200.h, calls the ABI
    and links against libeh_b200.so."""
    import subprocess
    from conftest import LIBDIR, ROOT
    src = tmp_path / "abi.c"
    src.write_text('#include "eh_b200.h"\n#include <stdio.h>\n'
                   'int main(void) { eh_context* c = 0; eh_status s = eh_context_create(0, &c);\n'
                   '  printf("%d %s\\n", s, s ? eh_last_error() : eh_version()); if (!s) eh_context_destroy(c);\n'
                   '  return 0; }\n')
    exe = str(tmp_path / "abi")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"), str(src),
                    "-L" + LIBDIR, "-leh_b200", "-Wl,-rpath," + LIBDIR, "-Wl,--allow-shlib-undefined", "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    status = int(r.stdout.split()[0])
    assert status in (0, 7)  # EH_OK on a GPU box, EH_ERR_NO_DEVICE here


def test_encoding_files_match_the_reference_format(tmp_path):
    """Encoding<T> writes the reference's encoding.bin (Encoding.cpp:52-130):
    the uint32 count, then the values in key order (a std::set gives
    ascending keys), strings as a size_t length and the characters; it reads
    them back, encodes columns through value_to_key, and keeps the
    reference's build() semantics for a vector with a repeated value."""
    import json
    import struct
    import subprocess

    from conftest import CPP, ROOT
    exe = str(tmp_path / "dropin_encoding")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "include", "eh"), os.path.join(CPP, "dropin_encoding.cpp"),
                    os.path.join(CPP, "fake_eh_abi.cpp"), "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])

    def file_bytes(sub):
        return (tmp_path / sub / "encoding.bin").read_bytes()

    assert file_bytes("u32") == struct.pack("<I4I", 4, 3, 5, 7, 900)
    assert file_bytes("long") == struct.pack("<I3q", 3, -2, 0, 1 << 40)
    want = struct.pack("<I", 3)
    for s in ("", "alpha", "b"):
        want += struct.pack("<Q", len(s)) + s.encode()
    assert file_bytes("str") == want
    assert out["u32"] == {"num_distinct": 4, "key_to_value": [3, 5, 7, 900], "encoded": [2, 0, 3, 0],
                          "lookups": [2, 0, 3, 0]}
    assert out["long"]["key_to_value"] == [-2, 0, 1 << 40] and out["long"]["encoded"] == [1, 2, 0]
    assert out["str"]["key_to_value"] == ["", "alpha", "b"] and out["str"]["encoded"] == [1, 0, 2]
    assert out["vector_num_distinct"] == 4 and out["vector_key_of_40"] == 0
    assert out["vector_key_to_value"] == [40, 10, 40, 20]
    assert out["unknown_throws"] is True


def test_encoding_files_equal_the_reference_engines(tmp_path):
    """The same dictionaries written by the reference's own Encoding<T>
    (oracle/ref_encoding.cpp, compiled from the reference's sources by
    `make -C oracle ref_encoding`) are byte-identical to the layer's."""
    import subprocess

    from conftest import CPP, ROOT
    from oracle import oracle as O
    if not os.path.isdir(os.path.join(O.reference_dir(), "storage_engine", "src")):
        pytest.skip("needs the reference checkout ($EH_REFERENCE)")
    mk = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref_encoding"], capture_output=True, text=True)
    assert mk.returncode == 0, mk.stderr[-2000:]
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref_dir.mkdir()
    our_dir.mkdir()
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "eh_ref_encoding"), str(ref_dir)], check=True, timeout=60)
    exe = str(tmp_path / "dropin_encoding")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "include", "eh"), os.path.join(CPP, "dropin_encoding.cpp"),
                    os.path.join(CPP, "fake_eh_abi.cpp"), "-o", exe], check=True, capture_output=True, text=True)
    subprocess.run([exe, str(our_dir)], check=True, capture_output=True, timeout=60)
    for sub in ("u32", "long", "str"):
        assert (our_dir / sub / "encoding.bin").read_bytes() == (ref_dir / sub / "encoding.bin").read_bytes(), sub


def test_set_intersect_forms(tmp_path):
    """ops::set_intersect in its four forms (trie/set/ops/intersection/
    set.hpp:9-167) over the layer's sets: the materialising forms give C the
    sorted intersection with its density-rule layout, the callback forms call
    f(x, index in A, index in B) per element in order, and an empty side
    gives an empty result."""
    import json
    import subprocess

    from conftest import CPP, ROOT
    exe = str(tmp_path / "dropin_setops")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(ROOT, "include", "eh"), os.path.join(CPP, "dropin_setops.cpp"),
                    os.path.join(CPP, "fake_eh_abi.cpp"), "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    out = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    a = [1, 5, 9, 64, 65, 300, 1000, 5000, 70000]
    b = list(range(256)) + list(range(990, 1010)) + [70000]
    want = sorted(set(a) & set(b))
    assert out["c1"] == want and out["c2"] == want
    assert out["triples"] == [[x, a.index(x), b.index(x)] for x in want]
    assert out["count_f"] == out["calls"] == out["count"] == len(want)
    assert out["count_empty"] == 0 and out["c3_cardinality"] == 0
    assert out["c1_range"] == want[-1]
    # the density rule (common::is_sparse): 6 elements over 70,000 values are a
    # uint list, B (277 elements over 70,001 values) too
    assert out["c1_type"] == 1 and out["b_type"] == 1

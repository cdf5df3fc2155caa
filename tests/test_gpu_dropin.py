"""The reference's generated bag code (oracle/generated_bags.hpp, the source
oracle/ref_driver.cpp runs on the reference engine) compiled against the
C++ layer of include/eh/ and linked against libeh_b200.so, on the B200: the
four travis.py goldens through the device plans, a body without a device
plan through the host loop, a selection query, and the host loop on the
device's set intersections for the triangle bag."""
import shutil

import pytest

from conftest import compile_dropin, run_dropin, write_facebook_tsvs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")]


@pytest.fixture(scope="module")
def build(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("dropin_gpu"))
    return {"exe": compile_dropin(d, fake=False), "tsv": write_facebook_tsvs(d)}


@pytest.mark.parametrize("query,graph", [("triangle", "pruned"), ("clique4", "pruned"), ("lollipop", "duplicated"),
                                         ("barbell", "duplicated")])
def test_generated_bags_give_the_travis_goldens(build, golden, query, graph):
    out = run_dropin(build["exe"], query, build["tsv"][graph])
    assert "error" not in out, out
    assert out["count_u64"] == golden["travis"]["facebook_" + graph][query]


def test_body_without_a_device_plan(build, golden):
    out = run_dropin(build["exe"], "path2", build["tsv"]["pruned"])
    assert out["count_u64"] == golden["reference_engine"]["facebook_pruned"]["path2"]


def test_selection_bag(build, golden):
    out = run_dropin(build["exe"], "barbell_sel", build["tsv"]["duplicated"], 6)
    assert out["count_u64"] == golden["travis"]["facebook_duplicated"]["barbell_sel_p6"]


def test_host_loop_on_device_set_ops(build, golden):
    out = run_dropin(build["exe"], "triangle", build["tsv"]["pruned"], env={"EH_DROPIN_HOST_LOOP": "1"})
    assert out["count_u64"] == golden["travis"]["facebook_pruned"]["triangle"]

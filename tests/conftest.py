import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def facebook():
    d = np.load(os.path.join(GOLDEN, "facebook.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def eh():
    import emptyheaded_b200 as E
    return E


@pytest.fixture(scope="session")
def ctx(eh):
    c = eh.default_context()
    yield c


# ------------------------------------------------------------ the C++ layer
CPP = os.path.join(ROOT, "tests", "cpp")
LIBDIR = os.path.join(ROOT, "emptyheaded_b200", "_lib")


def compile_dropin(out_dir, fake):
    """Compile tests/cpp/dropin_bags.cpp (generated bag code over the C++
    layer of include/eh/) and link it against libeh_b200.so, or, with fake,
    against the CPU test double of the C ABI.  Returns the binary's path."""
    import subprocess
    exe = os.path.join(out_dir, "dropin_fake" if fake else "dropin_bags")
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "include", "eh"),
           "-I" + os.path.join(ROOT, "oracle"), os.path.join(CPP, "dropin_bags.cpp")]
    if fake:
        cmd += [os.path.join(CPP, "fake_eh_abi.cpp")]
    else:
        cmd += ["-L" + LIBDIR, "-leh_b200", "-Wl,-rpath," + LIBDIR, "-Wl,--allow-shlib-undefined"]
    subprocess.run(cmd + ["-o", exe], check=True, capture_output=True, text=True)
    return exe


def write_facebook_tsvs(out_dir):
    """The reference's test graphs (tests/golden/facebook.npz) as .tsv files."""
    d = np.load(os.path.join(GOLDEN, "facebook.npz"))
    paths = {}
    for k in d.files:
        p = os.path.join(out_dir, k + ".tsv")
        np.savetxt(p, d[k], fmt="%d", delimiter="\t")
        paths[k] = p
    return paths


def run_dropin(exe, query, tsv, value=None, env=None, timeout=900):
    import subprocess
    e = dict(os.environ)
    e.update(env or {})
    args = [exe, query, tsv] + ([str(value)] if value is not None else [])
    r = subprocess.run(args, capture_output=True, text=True, env=e, timeout=timeout)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert line, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return json.loads(line[-1])

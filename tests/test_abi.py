"""C-ABI library checks that need no GPU: it builds, loads, exports every
symbol include/eh_b200.h declares, and fails loudly without a device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^(?:eh_status|const char\*)\s+(eh_\w+)\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol(eh):
    L = eh.lib()
    names = declared_symbols()
    assert len(names) >= 30
    for n in sorted(names):
        assert hasattr(L, n), n
    assert L.eh_version().decode().startswith("emptyheaded_b200")


def test_no_device_is_an_error_not_a_fallback(eh):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(eh.EHError) as e:
        eh.Context(0)
    assert e.value.status == 7  # EH_ERR_NO_DEVICE


def test_null_arguments_are_rejected(eh):
    L = eh.lib()
    assert L.eh_context_create(0, None) == 1
    assert L.eh_trie_info_get(None, None) == 1
    assert b"null" in L.eh_last_error()
    assert L.eh_context_memory(None, None, None, None) == 1
    assert L.eh_context_reserve(None, 1 << 20) == 1
    assert b"null" in L.eh_last_error()
    assert L.eh_trie_free(None) == 0
    assert L.eh_context_destroy(None) == 0

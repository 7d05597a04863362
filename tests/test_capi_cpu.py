"""The C ABI library without a GPU: it loads, exports every entry point that
include/nnm.h declares, and reports the absence of a device as an error
code instead of crashing."""
import ctypes
import os
import re

import pytest

import nnm
from nnm import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "nnm.h")).read()
    return sorted(set(re.findall(r"\b(nnm_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = nnm.load()
    decl = declared_functions()
    assert len(decl) >= 14
    for name in decl:
        assert hasattr(lib, name), name
    assert set(_lib.EXPORTED) <= set(decl)


def test_default_options_are_the_reference_constants():
    o = nnm.make_opts()
    assert o.sample_cap == 100            # kgraph.cpp:100
    assert abs(o.delta - 0.002) < 1e-9    # abstractgraph.cpp:4
    assert o.max_iter == 0 and o.metric == 0


def test_status_strings():
    lib = nnm.load()
    assert lib.nnm_status_string(0) == b"ok"
    assert lib.nnm_status_string(2) == b"unsupported metric"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_crash():
    with pytest.raises(nnm.NnmError) as e:
        nnm.Context(0)
    assert e.value.status == 5


def test_null_context_is_rejected():
    lib = nnm.load()
    o = nnm.make_opts()
    rc = lib.nnm_kgraph_build(None, None, 0, 0, 0, ctypes.byref(o), None, None, None, None)
    assert rc == 1

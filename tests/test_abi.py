"""The C ABI (CPU only): libtce.so loads, exports every symbol include/tce.h
declares, and fails loudly (status + message, no fallback) without a GPU."""
import os
import re

import pytest

from william_ci_b200 import engine as E
from william_ci_b200 import system as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "tce.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tce_[a-z0-9_]+)\s*\(", txt)))


def test_header_matches_binding_list():
    assert declared_symbols() == sorted(E.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = E.lib()
    for sym in declared_symbols():
        assert hasattr(lib, sym), sym
    assert b"sm_100a" in lib.tce_version()


def test_struct_layout_matches_oracle():
    import pyoracle
    assert [f for f, _ in E.TceSystem._fields_] == [f for f, _ in pyoracle.OrcSystem._fields_]


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_fails_loudly():
    s = S.build_system(*S.workload("h2_ring"))
    with pytest.raises(E.TCEError) as ei:
        E.Engine(s)
    assert ei.value.code == E.TCE_ERR_CUDA
    assert str(ei.value)


def test_bad_arguments_are_rejected_before_the_device():
    s = S.build_system(*S.workload("h2_ring"))
    with pytest.raises(E.TCEError) as ei:
        E.Engine(s, nquad=33)
    assert ei.value.code in (E.TCE_ERR_UNSUPPORTED, E.TCE_ERR_ARG)


def test_execution_options_reject_a_null_handle():
    """The pass's execution options (graph, tensor cores, list chains) check
    their handle before touching anything: a NULL handle is an argument error."""
    lib = E.lib()
    assert lib.tce_set_graph(None, 1) == E.TCE_ERR_ARG
    assert lib.tce_set_tensor_cores(None, 1) == E.TCE_ERR_ARG
    assert lib.tce_set_list_streams(None, 2) == E.TCE_ERR_ARG

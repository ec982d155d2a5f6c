"""The C-ABI library loads and exports every entry point include/tosca_gpu.h
declares (no GPU needed: nothing is called)."""
import ctypes
import os
import re

import pytest

import tosca_b200
from tosca_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "tosca_gpu.h")).read()
    # function declarations: "<return type> tg_name(" at the start of a line
    return sorted(set(re.findall(r"^(?:tg_status|const char \*)\s*(tg_[a-z_0-9]+)\(", src, re.M)))


# context-free device-pointer entry point: bound directly by its test, and not
# exported by the CPU restatement
NO_CONTEXT = {"tg_continuity_error_noalloc"}
# checkpointed adjoint drivers (device snapshots: the CPU restatement has the
# per-step adjoint only), the CUDA-graph replay switch and the mesh classification
GPU_ONLY = {"tg_adjoint_forward", "tg_adjoint_reverse", "tg_set_graphs", "tg_graph_info", "tg_mesh_info"}


def test_header_matches_bindings():
    decl = declared_symbols()
    assert decl, "no declarations found"
    bound = {"tg_" + n for n in api.ENTRY_POINTS}
    assert set(decl) == bound | NO_CONTEXT


def test_library_exports_all_symbols():
    if not os.path.exists(tosca_b200.LIB_PATH):
        pytest.skip("CUDA library not built")
    lib = ctypes.CDLL(tosca_b200.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_oracle_exports_same_entry_points():
    import oracle
    oracle.load()
    lib = oracle.lib()
    for name in declared_symbols():
        if name in NO_CONTEXT or name in GPU_ONLY:
            continue
        assert hasattr(lib, "tor_" + name[3:]), name


def test_config_struct_layout():
    # offsets of the C struct as laid out by the C compiler rules (x86-64)
    c = api.TgConfig
    assert c.bc.offset == 12 and c.nut_bc.offset == 36 and c.nut_bc_value.offset == 64
    assert ctypes.sizeof(api.TgStats) == 48


def test_bad_config_rejected_by_oracle():
    import oracle
    cfg = api.Config(mx=4, my=8, mz=8)
    with pytest.raises(api.TgError):
        oracle.solver(cfg)
    cfg = api.Config(mx=8, my=8, mz=8, bc=(api.BC_PERIODIC, api.BC_SLIP) + (api.BC_PERIODIC,) * 4)
    with pytest.raises(api.TgError):
        oracle.solver(cfg)

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
GPU_ONLY = {"tg_adjoint_forward", "tg_adjoint_reverse", "tg_adjoint_set_tapes", "tg_set_graphs", "tg_graph_info",
            "tg_mesh_info"}


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


STRUCTS = {"tg_config": api.TgConfig, "tg_stats": api.TgStats, "tg_turbine": api.TgTurbine,
           "tg_adjoint_stats": api.TgAdjointStats}


def test_struct_layouts_match_the_c_compiler(tmp_path):
    """Every field offset and the size of each struct in the ctypes mirror
    equal what gcc lays out from include/tosca_gpu.h."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "tosca_gpu.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in STRUCTS.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_bad_config_rejected_by_oracle():
    import oracle
    cfg = api.Config(mx=4, my=8, mz=8)
    with pytest.raises(api.TgError):
        oracle.solver(cfg)
    cfg = api.Config(mx=8, my=8, mz=8, bc=(api.BC_PERIODIC, api.BC_SLIP) + (api.BC_PERIODIC,) * 4)
    with pytest.raises(api.TgError):
        oracle.solver(cfg)
    # order of the extrapolated pressure guess: -1 (default), 0, 1 or 2
    for bad in (3, -2, -7):
        with pytest.raises(api.TgError):
            oracle.solver(api.Config(mx=8, my=8, mz=8, poisson_guess=bad))
    for good in (-1, 0, 1, 2):
        oracle.solver(api.Config(mx=8, my=8, mz=8, poisson_guess=good)).close()

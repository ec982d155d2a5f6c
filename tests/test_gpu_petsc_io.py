"""TOSCA field files between the CUDA library and the oracle: each reads what
the other wrote, bitwise."""
import numpy as np
import pytest

import oracle
import tosca_b200
from tosca_b200 import api, cases

pytestmark = pytest.mark.gpu


def test_field_files_cross_read(tmp_path):
    cfg, nodes, ucat, p, T = cases.hill_case(teqn=True, t_amp=0.5, nx=24, ny=12, nz=12)
    g, o = tosca_b200.gpu_solver(cfg), oracle.solver(cfg)
    for s in (g, o):
        cases.setup(s, nodes, ucat, p, T)
    g.step(2)
    g.write_fields(str(tmp_path / "gpu"))
    o.read_fields(str(tmp_path / "gpu"))
    for f in ("UCONT", "UCAT", "P", "NUT", "TMPRT"):
        assert np.array_equal(o.get(f), g.get(f)), f
    o.step(1)
    o.write_fields(str(tmp_path / "cpu"))
    g.read_fields(str(tmp_path / "cpu"))
    for f in ("UCONT", "UCAT", "P", "NUT", "TMPRT"):
        assert np.array_equal(o.get(f), g.get(f)), f
    g.close(); o.close()

"""Mesh classification that selects the kernel variants (tg_mesh_info):
axis-aligned meshes of planes (ABL, TGV) run the one-component metric
kernels, the curvilinear hill the general ones; both are held to the oracle
by the parity tests."""
import pytest

import tosca_b200
from tosca_b200 import cases
from tests.common import SMALL, build_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,expect", [("tgv", (True, True)), ("abl", (True, True)), ("hill", (False, False))])
def test_mesh_classification(name, expect):
    cfg, nodes, ucat, p, T = build_case(name, **SMALL[name])
    s = tosca_b200.gpu_solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    assert s.mesh_info() == expect
    s.close()

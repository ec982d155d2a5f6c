"""The allocation-free divergence check (tg_continuity_error_noalloc) against
the context-based one (tg_continuity_error), through the C-ABI, on two calls
in a row. It exists for callers that cannot allocate device memory (code
inside a CUDA graph capture, hosts whose device memory belongs to a fixed
pool, loops that cannot absorb cudaMalloc's synchronisation): its scratch is a
file-scope device array, so the call itself allocates nothing. The test
allocates its own inputs with torch."""
import ctypes

import numpy as np
import pytest

import tosca_b200
from tests.common import SMALL, build_case
from tosca_b200 import cases

pytestmark = pytest.mark.gpu


def _bind():
    lib = ctypes.CDLL(tosca_b200.LIB_PATH)
    fn = lib.tg_continuity_error_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                   ctypes.c_void_p, ctypes.c_void_p]
    return fn


CASES = {
    # axis-aligned ABL, square-ish planes
    "abl": lambda: build_case("abl", **SMALL["abl"]),
    # ragged, non-square planes (mx != my): exercises the i/j split of a plane
    "abl_ragged": lambda: build_case("abl", nx=14, ny=18, nz=10, Lx=140.0, Ly=180.0, H=100.0),
    # curvilinear metrics
    "hill": lambda: build_case("hill", **SMALL["hill"]),
    # shallow in k with large planes: each plane is split over several blocks
    "abl_shallow": lambda: build_case("abl", nx=8, ny=64, nz=48, Lx=80.0, Ly=640.0, H=300.0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_divergence_matches_context_entry_point(name):
    import torch
    fn = _bind()
    cfg, nodes, ucat, p, T = CASES[name]()
    s = tosca_b200.gpu_solver(cfg)
    cases.setup(s, nodes, ucat, p, T)
    dev = torch.device("cuda", cfg.device)
    torch.cuda.set_device(dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    for call in range(2):
        if call == 1:
            s.step(1)                       # different state on the second call
        ref = s.ContinuityErrorsOptimized()
        ucont = torch.from_numpy(np.ascontiguousarray(s.get("UCONT"))).to(dev)
        aj = torch.from_numpy(np.ascontiguousarray(s.get("AJ"))).to(dev)
        out.fill_(-1.0)
        stream = torch.cuda.current_stream(dev)
        st = fn(ucont.data_ptr(), aj.data_ptr(), cfg.mx, cfg.my, cfg.mz, out.data_ptr(),
                ctypes.c_void_p(stream.cuda_stream))
        assert st == 0
        stream.synchronize()
        got = float(out.item())
        # a maximum is independent of the reduction order: expect the same value
        assert got == pytest.approx(ref, rel=1e-15, abs=0.0), (call, got, ref)
        assert got > 0.0
    s.close()


def test_noalloc_rejects_too_many_planes():
    import torch
    fn = _bind()
    dev = torch.device("cuda", 0)
    dummy = torch.zeros(16, dtype=torch.float64, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    # 16384 interior planes is the limit of the scratch array: 16387 planes are refused
    st = fn(dummy.data_ptr(), dummy.data_ptr(), 4, 4, 16387, out.data_ptr(), None)
    assert st == 2

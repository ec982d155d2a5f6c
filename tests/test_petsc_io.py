"""TOSCA field files (PETSc binary VecView of a DMDA vector, io.c:247-420,
2261) through the oracle's reader and writer: byte layout, round trip, the
32-bit header variant, rejection of foreign files, and a field file that ships
with the reference against its committed summary (tests/golden)."""
import json
import os

import numpy as np
import pytest

import oracle
from tosca_b200 import api, cases

HERE = os.path.dirname(os.path.abspath(__file__))
# root of a reference checkout: TOSCA_REFERENCE_ROOT, else the checkout the
# reference harness compiles from (oracle/ref.py), if present on this machine
from oracle import ref as _ref  # noqa: E402
REF_ROOT = _ref.reference_src()


def _solver(n=8):
    cfg, nodes, ucat, p = cases.tgv_case(n)
    s = oracle.solver(cfg)
    cases.setup(s, nodes, ucat, p)
    return s


def test_layout_and_round_trip(tmp_path):
    s = _solver()
    rng = np.random.default_rng(1)
    u = rng.standard_normal(s.get("UCAT").shape)
    p = rng.standard_normal(s.get("P").shape)
    s.set("UCAT", u)
    s.set("P", p)
    s.write_fields(str(tmp_path))
    raw = open(tmp_path / "U", "rb").read()
    assert np.frombuffer(raw[:16], ">i8").tolist() == [1211214, u.size]
    assert np.array_equal(np.frombuffer(raw[16:], ">f8"), u.ravel())
    t = _solver()
    t.read_fields(str(tmp_path))
    assert np.array_equal(t.get("UCAT"), u) and np.array_equal(t.get("P"), p)
    assert np.array_equal(t.get("UCONT"), s.get("UCONT"))
    s.close(); t.close()


def test_32bit_header_and_rejections(tmp_path):
    s = _solver()
    p = np.random.default_rng(2).standard_normal(s.get("P").shape)
    with open(tmp_path / "p32", "wb") as f:
        f.write(np.array([1211214, p.size], ">i4").tobytes() + p.astype(">f8").tobytes())
    s.read_field_petsc("P", str(tmp_path / "p32"))
    assert np.array_equal(s.get("P"), p)
    with open(tmp_path / "bad", "wb") as f:
        f.write(np.array([1211216, p.size], ">i8").tobytes() + p.astype(">f8").tobytes())
    with pytest.raises(api.TgError) as e:
        s.read_field_petsc("P", str(tmp_path / "bad"))
    assert e.value.status == api.TG_ERR_BAD_ARG
    with pytest.raises(api.TgError):
        s.read_field_petsc("UCAT", str(tmp_path / "p32"))      # entry count of a scalar
    s.close()


def test_reference_field_file_matches_summary():
    summary = json.load(open(os.path.join(HERE, "golden", "channel_p_summary.json")))
    path = os.path.join(REF_ROOT or "", summary["file"])
    if not REF_ROOT or not os.path.exists(path):
        pytest.skip("no reference checkout on this machine")
    s = _solver(64)                                   # DMDA extent 66^3
    s.read_field_petsc("P", path)
    p = s.get("P")
    flat = p.ravel()
    assert flat.size == summary["n"]
    for q, v in summary["samples"].items():
        q = int(q)
        assert p[q // (66 * 66), (q // 66) % 66, q % 66] == v
    assert abs(flat.sum() - summary["sum"]) <= 1e-9 * abs(summary["sum"])
    assert flat.min() == summary["min"] and flat.max() == summary["max"]
    s.close()

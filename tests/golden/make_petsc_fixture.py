"""Summary of a field file that ships with the reference
(tests/ChannelFlowRe395Test/fields/5.00/p: PETSc binary VecView of a
66 x 66 x 66 DMDA scalar), read with plain numpy: header, entry count and the
values at a few natural indices. test_petsc_io.py reads the same file with
the oracle's and the CUDA library's readers and compares with this summary.

    python tests/golden/make_petsc_fixture.py <reference checkout>
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REL = "tests/ChannelFlowRe395Test/fields/5.00/p"


def main(ref_root):
    raw = open(os.path.join(ref_root, REL), "rb").read()
    cls, n = np.frombuffer(raw[:16], dtype=">i8")
    v = np.frombuffer(raw[16:], dtype=">f8")
    assert cls == 1211214 and n == v.size == 66 ** 3
    idx = [0, 1, 65, 66, 4356, 4357 + 66 + 1, 143748, 200000, 287495]
    out = {"file": REL, "class_id": int(cls), "n": int(n), "extent": [66, 66, 66],
           "sum": float(v.sum()), "min": float(v.min()), "max": float(v.max()),
           "samples": {str(i): float(v[i]) for i in idx}}
    with open(os.path.join(HERE, "channel_p_summary.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_petsc_fixture.py <reference checkout>")
    main(sys.argv[1])

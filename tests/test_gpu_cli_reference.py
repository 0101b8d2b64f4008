"""This library's bem_cuda CLI against the reference's own CLI.

oracle/Makefile compiles the reference's bin/bem_cuda from all of its
sources with its own compiler flags (architecture set to sm_100a) into
oracle/_ref/bem_cuda_ref; both programs run the dense solver with the same
command lines (main.cpp:94-181 flags; the dense branch main.cpp:660-854) and
their JSON files (output.cpp:5-64) are compared: the same keys and layout,
the same angles and parameters, and Mueller matrices that agree to the
accuracy of the reference's FP32 assembly kernel (assembly.cu:14-135, built
with --use_fast_math as its Makefile builds it), ~1e-6 relative.  Skipped
where the reference's build is absent (it is made from the reference
sources, which only the build machine holds)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(REPO, "bem-cpp_b200", "bin", "bem_cuda")
REF = os.path.join(REPO, "oracle", "_ref", "bem_cuda_ref")

CASES = {
    "c1_single": ["--ka", "1.0", "--ref", "2", "--ri", "1.3116", "0.0", "--single", "--ntheta", "181"],
    "hex_orient": ["--ka", "2.0", "--ref", "2", "--ri", "1.45", "0.01", "--shape", "hex", "--ar", "1.2",
                   "--orient", "4", "3", "1", "--ntheta", "37"],
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_matches_reference_cli(case, tmp_path):
    if not os.path.exists(REF):
        pytest.skip("the reference CLI was not built (oracle/Makefile needs the reference sources)")
    assert os.path.exists(OURS), "bem_cuda not built"
    out = {}
    for tag, exe in (("ours", OURS), ("ref", REF)):
        path = tmp_path / f"{tag}.json"
        r = subprocess.run([exe, "--solver", "dense", *CASES[case], "--out", str(path)], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, (tag, r.stdout[-1500:], r.stderr[-1500:])
        out[tag] = json.loads(path.read_text())
    a, b = out["ours"], out["ref"]
    assert set(a) == set(b), (set(a) ^ set(b))
    for k in a:
        if k not in ("mueller", "timing"):
            assert a[k] == b[k], (k, a[k], b[k])
    assert set(a["timing"]) == set(b["timing"])
    Ma, Mb = np.array(a["mueller"]), np.array(b["mueller"])
    assert Ma.shape == Mb.shape == (4, 4, a["ntheta"])
    err = rel(Ma, Mb)
    print(f"{case}: Mueller of this CLI vs the reference CLI: {err:.2e}")
    assert err < 1e-4

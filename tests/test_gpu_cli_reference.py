"""This library's bem_cuda CLI against the reference's own CLI.

oracle/Makefile compiles the reference's bin/bem_cuda from all of its
sources twice, architecture set to sm_100a: with its own compiler flags
(-O3 --use_fast_math, oracle/_ref/bem_cuda_ref) and without the fast-math
intrinsics (oracle/_ref/bem_cuda_ref_exact).  The programs run the dense
solver with the same command lines (main.cpp:94-181 flags; the dense branch
main.cpp:660-854) and their JSON files (output.cpp:5-64) are compared: the
same keys and layout, the same angles and parameters, and Mueller matrices
that agree with the exact-math build to the accuracy of the reference's
FP32 assembly kernel (assembly.cu:14-135), ~1e-6 relative, and with the
fast-math build to that build's own error (its approximate sincosf / expf
in the FP32 kernel move the Mueller matrices by ~1e-3).  Skipped where the
reference's build is absent (it is made from the reference sources, which
only the build machine holds)."""
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
REF_EXACT = os.path.join(REPO, "oracle", "_ref", "bem_cuda_ref_exact")
# Mueller agreement: with the exact-math reference build the FP32 assembly
# alone; with the reference's own fast-math build its intrinsics' error
BOUND = {"ref": 1e-2, "ref_exact": 2e-5}

CASES = {
    "c1_single": ["--ka", "1.0", "--ref", "2", "--ri", "1.3116", "0.0", "--single", "--ntheta", "181"],
    "hex_orient": ["--ka", "2.0", "--ref", "2", "--ri", "1.45", "0.01", "--shape", "hex", "--ar", "1.2",
                   "--orient", "4", "3", "1", "--ntheta", "37"],
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_cli_matches_reference_cli(case, tmp_path):
    progs = [(t, e) for t, e in (("ref", REF), ("ref_exact", REF_EXACT)) if os.path.exists(e)]
    if not progs:
        pytest.skip("the reference CLI was not built (oracle/Makefile needs the reference sources)")
    assert os.path.exists(OURS), "bem_cuda not built"
    out = {}
    for tag, exe in [("ours", OURS)] + progs:
        path = tmp_path / f"{tag}.json"
        r = subprocess.run([exe, "--solver", "dense", *CASES[case], "--out", str(path)], capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, (tag, r.stdout[-1500:], r.stderr[-1500:])
        out[tag] = json.loads(path.read_text())
    a = out["ours"]
    for tag, _ in progs:
        b = out[tag]
        assert set(a) == set(b), (set(a) ^ set(b))
        for k in a:
            if k not in ("mueller", "timing"):
                assert a[k] == b[k], (k, a[k], b[k])
        assert set(a["timing"]) == set(b["timing"])
        Ma, Mb = np.array(a["mueller"]), np.array(b["mueller"])
        assert Ma.shape == Mb.shape == (4, 4, a["ntheta"])
        err = rel(Ma, Mb)
        print(f"{case}: Mueller of this CLI vs the reference CLI ({tag}): {err:.2e}")
        assert err < BOUND[tag], (tag, err)

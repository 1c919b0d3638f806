"""The reference's own sampler and estimator run unmodified on the drop-in
``qed_fermion._C`` (this library's kernels), checked against the oracle.

The reference must be installed under baseline/_ref (a pip install of the
reference tree; it is not part of this repository).  Without it the test is
skipped with that reason.  The work runs in a fresh process
(tests/reference_dropin_check.py): the reference reads its configuration from
the environment when it is imported.
"""
import json
import os
import subprocess
import sys

import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")


def test_reference_sampler_on_dropin_kernels():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    if not os.path.exists(os.path.join(REF, "qed_fermion", "hmc_sampler_batch.py")):
        pytest.skip("the reference is not installed under baseline/_ref")
    res = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "reference_dropin_check.py"), REF, ROOT],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert res.returncode == 0, res.stderr[-3000:]
    out = json.loads(res.stdout.strip().splitlines()[-1])
    # complex64 solves to the reference's cg_rtol (set to 1e-6 here)
    assert out["xi_rel_err"] < 1e-4, out
    assert out["force_rel_err"] < 1e-4, out
    assert max(out["pcg_true_rel_residual"]) < 5e-6, out
    assert out["g_eta_rel_err"] < 1e-4, out
    assert out["bs_restored"] == 2

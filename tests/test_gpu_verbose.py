"""ONEDAL_VERBOSE: the reference gates its profiler/logger on this variable
(cpp/daal/src/services/service_profiler.h:141-151); here level >= 1 wraps the
hot-path phases in NVTX ranges named after the reference's profiler tasks and
logs one line per train / infer call to stderr. Run in a child process because
the level is read once per process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import numpy as np
from onedal_b200 import kmeans
rng = np.random.default_rng(0)
X = rng.standard_normal((5000, 16)).astype(np.float32)
d = kmeans.descriptor(np.float32).set_cluster_count(8).set_max_iteration_count(3)
r = kmeans.train(d, X, X[:8].copy())
kmeans.infer(d, r.get_model(), X)
print("done", r.get_iteration_count())
"""


@pytest.mark.parametrize("level,logged", [("1", True), ("0", False)])
def test_onedal_verbose_logs_calls(level, logged):
    env = dict(os.environ, ONEDAL_VERBOSE=level, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert "done 3" in r.stdout
    lines = [ln for ln in r.stderr.splitlines() if ln.startswith("onedal_b200: ")]
    if logged:
        assert any(ln.startswith("onedal_b200: train n=5000 d=16 k=8") and "iterations=3 status=0" in ln for ln in lines)
        assert any(ln.startswith("onedal_b200: infer n=5000 d=16 k=8") and "status=0" in ln for ln in lines)
    else:
        assert not lines

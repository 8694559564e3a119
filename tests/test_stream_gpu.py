"""Both kernel families on every precision: the streaming kernels (bulk
copies into shared memory, warp-specialised) and the register kernels are
forced in turn (AINV_STREAM=1 / 0, read once per process, hence the
subprocesses) and checked against the oracle by tests/stream_check.py."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("stream", ["1", "0"])
@pytest.mark.parametrize("idim", [48, 61])
def test_kernel_family_parity(stream, idim):
    env = dict(os.environ, AINV_STREAM=stream)
    p = subprocess.run([sys.executable, os.path.join(HERE, "stream_check.py"), str(idim)],
                       env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    out = json.loads(p.stdout.strip().splitlines()[-1])
    assert out["ok"], out

"""Every variant of the persistent guided kernel the autotuner may pick
(2 blocks per SM, 3 blocks per SM, tap windows staged in shared memory)
passes the batched-form parity test against the oracle. The variant is a
process-wide choice read once (LGCR_GUIDED_VARIANT), so each runs in a child
process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("variant", ["1", "2"])
def test_batched_parity_with_guided_variant(variant):
    env = dict(os.environ, LGCR_GUIDED_VARIANT=variant)
    target = os.path.join(HERE, "test_headline_gpu.py") + "::test_batched_and_graph_replay_vs_oracle"
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", target],
                       env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]

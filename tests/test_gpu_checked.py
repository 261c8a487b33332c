"""The checked build (chsga_b200/lib_checked, CHSGA_CHECKED): every kernel
checks each index it reads from a graph array against the size of what it
indexes, records the first one out of range and keeps the access in bounds;
the call then fails with CHSGA_ERR_INTERNAL. This stands in for a memory
checker: on a graph whose arrays are all consistent, every GPU path -- all
row kernels at 1 to 128 slots, 16- and 32-bit rows, the persistent kernel,
the no-alloc entry point, tracebacks (full matrix, checkpointed, batched)
and the serving loop -- must run with no check firing and give the oracle's
results. Runs in a child process, which loads the checked library."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "chsga_b200", "lib_checked", "libchsga.so")


@pytest.mark.skipif(not os.path.exists(CHECKED), reason="checked build absent (make -C chsga_b200 checked)")
def test_every_gpu_path_passes_the_index_checks(tmp_path):
    env = dict(os.environ, CHSGA_LIBRARY=CHECKED)
    res = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_run.py"), str(tmp_path)],
                         env=env, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0 and "checked ok" in res.stdout, res.stdout[-3000:] + res.stderr[-3000:]

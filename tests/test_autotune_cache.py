"""The autotuner's persistent cache ($JFDK_AUTOTUNE_CACHE): one line per shape,
"key slices-per-thread views-per-chunk tile-width", appended after a tuning
run and read back by later processes.  The file is read once per process,
so each step runs in a child process; what a child did shows in the file: a
shape found in it is not tuned again (nothing appended)."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

TESTS = os.path.join(ROOT, "tests")
CHILD = f"""
import sys
sys.path[:0] = [{ROOT!r}, {TESTS!r}]
from conftest import load_golden
from test_gpu_parity import engine_for
engine_for(load_golden("mini_c1")).autotune()
"""


def tune_in_child(cache):
    env = dict(os.environ, JFDK_AUTOTUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return cache.read_text().splitlines()


def test_cache_lines_are_written_and_read_back(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    cache = tmp_path / "tune.txt"
    lines = tune_in_child(cache)
    assert len(lines) == 1, lines
    key, z, ch, tx = lines[0].split()
    assert int(z) in (4, 8) and int(ch) in (16, 32, 64) and int(tx) in (4, 8, 32), lines
    # a valid line for the shape is used as it is: no tuning, nothing appended
    for line in (f"{key} 4 16 32", f"{key} 8 64"):      # the second without a width (width 4)
        cache.write_text(line + "\n")
        assert tune_in_child(cache) == [line]
    # an invalid width is ignored: the shape is tuned again and appended
    cache.write_text(f"{key} 8 32 16\n")
    lines = tune_in_child(cache)
    assert len(lines) == 2 and lines[1].split()[0] == key, lines

"""The host build of the inverse factor S runs its row recurrence over column blocks in parallel; every entry is
summed in the same order whatever the thread count, so S (and A^-1 b through it) must be bit-identical with 1
and with 4 OpenMP threads (CPU only; each count in its own process)."""
import os
import subprocess
import sys

import numpy as np

_SNIPPET = r"""
import sys, numpy as np
from diffphd_b200 import core, scenes
sc = scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=1)
d = core.from_scene(sc)
b = np.random.default_rng(5).standard_normal(sc.dofs)
np.save(sys.argv[1], d.debug_host_sts(b, sc.dt))
"""


def _run(threads, path):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run([sys.executable, "-c", _SNIPPET, path], check=True, env=env, cwd=root, timeout=600)
    return np.load(path)


def test_inverse_factor_is_bit_identical_across_thread_counts(tmp_path):
    x1 = _run(1, str(tmp_path / "t1.npy"))
    x4 = _run(4, str(tmp_path / "t4.npy"))
    assert np.all(np.isfinite(x1))
    assert np.array_equal(x1, x4)

"""The stats build (libeggsync_stats.so) computes the same labels as the
normal build and its interaction counters are consistent with the run."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO
from eggsync import _lib, data, egg_sync

pytestmark = pytest.mark.gpu

CHILD = r"""
import ctypes as C, json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from eggsync import data, egg_sync, _lib
c = data.c1(0)
lab, info = egg_sync(c["X"], c["eps"], full_update=True)
out = (C.c_int64 * 32)()
n = _lib.load().egg_update_counters(out, 32)
print(json.dumps({"n": n, "labels": lab.tolist(), "iterations": info["iterations"],
                  "counters": dict(zip(_lib.UPDATE_COUNTERS, [int(v) for v in out]))}))
"""


def test_stats_build_counters():
    lib = REPO / "egg-sync_b200" / "lib" / "libeggsync_stats.so"
    env = dict(os.environ, EGGSYNC_LIB=str(lib))
    r = subprocess.run([sys.executable, "-c", CHILD, str(REPO / "egg-sync_b200")], env=env, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    c = data.c1(0)
    lab, info = egg_sync(c["X"], c["eps"], full_update=True)
    assert res["n"] >= len(_lib.UPDATE_COUNTERS)
    assert np.array_equal(np.array(res["labels"], np.int32), lab)
    k = res["counters"]
    # every point is recomputed in every iteration with full_update
    assert k["points"] == len(c["X"]) * info["iterations"]
    assert k["small_pass"] <= k["cells"]
    assert k["full"] + k["tight_in"] + k["tight_out"] <= k["small_pass"]
    assert 0 < k["pairs"] and k["neighbors"] >= k["pairs_in"]

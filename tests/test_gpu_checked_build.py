"""GPU: the bounds-checked build (SUMMIT_B200_CHECKED=1 loads
liblds_checked.so) runs windowed and genome-wide estimates with no failed
index check and the same scores, bit for bit, as the ordinary build."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from summit_b200 import _lib
from summit_b200.session import GwSession, WinPlan
from summit_b200 import gwldcore
lib = _lib.load()
n, m = 1500, 2200
rows = gwldcore.synth_bed_rows(n, m, 99)
rng = np.random.default_rng(2)
annot = (rng.random((m, 4)) < 0.3).astype(float)
annot[:, 0] = 1.0
ws = np.array([0, 300, 301, 1000, 1800, m], dtype=np.int64)
out = {"checked": int(lib.lds_checked_build())}
for impute in ("mean", "hwe"):
    sess = GwSession(rows, n, impute_mode=impute, impute_seed=5)
    wp = WinPlan(sess, annot, ws, 24, 100, 3, "rademacher", vtile=16)
    wp.execute()
    out["win_" + impute] = wp.results()["ldscore"].tolist()
    gp = sess.plan(annot, 24, 100, 3, "rademacher")
    gp.execute()
    out["gw_" + impute] = gp.results()["ldscore"].tolist()
    wp.close(); gp.close(); sess.close()
import ctypes
code = ctypes.c_uint(0)
_lib.check(lib.lds_checked_errors(ctypes.byref(code)))
out["error_code"] = int(code.value)
print("RESULT " + json.dumps(out))
"""


def _run(checked: bool) -> dict:
    env = dict(os.environ)
    env["SUMMIT_B200_CHECKED"] = "1" if checked else "0"
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):])


def test_checked_build_runs_clean_and_matches():
    if not (ROOT / "summit_b200" / "liblds_checked.so").exists():
        pytest.skip("bounds-checked build not built (python -m summit_b200.build --checked)")
    plain, checked = _run(False), _run(True)
    assert plain["checked"] == 0 and checked["checked"] == 1
    assert checked["error_code"] == 0, hex(checked["error_code"])
    for key in ("win_mean", "win_hwe", "gw_mean", "gw_hwe"):
        np.testing.assert_array_equal(np.asarray(checked[key]), np.asarray(plain[key]), key)

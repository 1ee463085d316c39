"""The bounds-checked build (libmillefeuille_check.so, build.py --check).

1. The same calls through the normal and the checked library give the same
   results bit for bit, and no check fails: every index the kernels take from
   stored data stays inside its array on these inputs (slices spanning several
   tile-rows, a ragged last tile-row, every stored precision, several
   right-hand sides, batch queue and team items, graph replay, the SpMM
   kernels, the allocation-free SpMV).
2. The check path itself: with the test_check_limit hook the kernels check
   the gathered operand entries against a length shorter than the vector, so
   some gathers fail their check (every access stays inside the real vector).
   The solve returns MF_ERR_CHECK with the site on stderr, and the next solve
   on the same context converges.

Each build runs in its own process (MILLEFEUILLE_LIB selects the library)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "tests", "harness", "check_run.py")
LIBDIR = os.path.join(ROOT, "mille-feuille_b200", "millefeuille")


def _run(lib, out, *extra):
    env = dict(os.environ, MILLEFEUILLE_LIB=os.path.join(LIBDIR, lib))
    r = subprocess.run([sys.executable, HARNESS, str(out), *extra], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return np.load(out), r.stderr


@pytest.fixture(scope="module")
def check_lib(mf):
    if not os.path.exists(os.path.join(LIBDIR, "libmillefeuille_check.so")):
        import importlib
        importlib.import_module("build").build(check=True)
    return "libmillefeuille_check.so"


def test_checked_build_matches_normal_build_bit_for_bit(cuda, check_lib, tmp_path):
    ref, _ = _run("libmillefeuille.so", tmp_path / "normal.npz")
    chk, err = _run(check_lib, tmp_path / "checked.npz")
    assert str(ref["arch"]) == "sm_100a" and "bounds-checked" in str(chk["arch"])
    assert "bounds check failed" not in err, err[-2000:]
    keys = sorted(k for k in ref.files if k != "arch")
    assert keys == sorted(k for k in chk.files if k != "arch")
    assert len(keys) >= 30
    for k in keys:
        np.testing.assert_array_equal(chk[k], ref[k], err_msg=k)


def test_checked_build_reports_a_failed_check_and_stays_usable(cuda, check_lib, tmp_path):
    res, err = _run(check_lib, tmp_path / "narrowed.npz", "--narrowed")
    assert int(res["narrowed_status"]) == 9, int(res["narrowed_status"])      # MF_ERR_CHECK
    assert "millefeuille: bounds check failed" in err, err[-2000:]
    assert int(res["after_converged"]) == 1 and float(res["after_relres"]) <= 1e-8
    # the normal build ignores the hook
    res_n, err_n = _run("libmillefeuille.so", tmp_path / "narrowed_normal.npz", "--narrowed")
    assert int(res_n["narrowed_status"]) == 0 and "bounds check" not in err_n

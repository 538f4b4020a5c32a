"""The bounds-checked build on the GPU: parity with the oracle and no
skipped access (tests/checked_build_run.py, in a fresh process so that the
package binds libkls_checked.so instead of libkls.so)."""
import os
import subprocess
import sys

import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu


def test_checked_build_parity_and_no_out_of_bounds_access(lib_path):
    from kalnajs_log_spirals_b200 import build
    build.build(checked=True)                  # no-op when libkls_checked.so is current
    out = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_build_run.py")],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0 and "CHECKED_OK" in out.stdout, out.stdout + out.stderr[-3000:]

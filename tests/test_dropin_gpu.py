"""The integration notes' drop-ins, compiled: oracle/dropin_test.cc binds a
reference line_details_t to pg_line_t exactly as the notes show (the
reference's padded input layout included) and wraps pg_midsolve_batch as the
reference's midsolve(board, workspace); the program runs each beside the
reference's own schedule_compute_line / midsolve on the same buffers and
requires bit-identical outputs."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_test")


def test_dropins_match_reference_engine(cuda):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/dropin_test not built (it needs the reference sources)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin: ok" in r.stdout
    assert r.stdout.count("identical") == 9

"""The bounds-checked debug build (libipr_b200_dbg.so, -DIPR_BOUNDS_CHECK): it answers
bit-exactly with every check on and reports nothing; its launch-argument check flags a range
past a real allocation; and the fold's own index checks report a packing-output row beyond
the extent the launch gives, skipping those reads (the buffer itself is larger, so no
access leaves it).  Runs the case in a process of its own with IPR_B200_BOUNDS_CHECK=1."""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.gpu
def test_bounds_checked_build_is_exact_and_reports_failures():
    env = dict(os.environ, IPR_B200_BOUNDS_CHECK="1")
    r = subprocess.run([sys.executable, os.path.join(HERE, "bounds_debug_case.py")], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["build"] is True and d["library"] == "libipr_b200_dbg.so"
    assert d["exact"], "the debug build answers differently from the oracle"
    assert d["clean"] == [0, ""]
    assert d["inside"] == 0 and d["outside"] == -1  # IPR_OK, IPR_E_ARGS
    assert d["host_report"][0] == 1 and "ipr_debug_check_extent" in d["host_report"][1]
    assert d["cut_report"][0] >= 1 and "site 41" in d["cut_report"][1]
    assert d["cut_last_differs"] and d["cut_others_equal"]
    assert d["again_exact"] and d["final"] == [0, ""]

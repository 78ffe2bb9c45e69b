"""The drop-in executables driven as MGXBench's benchmark.py drives them, on the GPU.

tests/golden/make_dropin_records.py restates benchmark.py's command line and environment
(benchmark.py:113-130) and its acceptance checks (45-50, 147-156).  Here build/mm_1d (4 emulated
ranks, libraries MMM and SSS) and build/mm_2d (a 2 x 2 grid, MMM and NNN) run through
mgx-onegpu-launch exactly so, and every run must be accepted.  With MGXBENCH_RECORD_DROPIN set
to a path, the runs' outputs are written there: tests/golden/dropin_records.json holds such a
record, which tests/test_dropin_contract.py replays through the unmodified benchmark.py."""
import importlib.util
import json
import os
from pathlib import Path

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _records_module():
    spec = importlib.util.spec_from_file_location("make_dropin_records",
                                                  ROOT / "tests" / "golden" / "make_dropin_records.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_benchmark_py_command_lines_are_accepted():
    R = _records_module()
    assert (ROOT / "build" / "mm_1d").exists() and (ROOT / "build" / "mm_2d").exists()
    records = []
    for case in R.CASES:
        rec = R.run_case(*case)
        ok, why = R.accepts(rec["stdout"] + "\n" + rec["stderr"], rec["returncode"], rec["decomposition"],
                            rec["size"], rec["ranks"], rec["library"])
        assert ok, f"{case}: {why}\n{rec['stdout']}\n{rec['stderr']}"
        assert "NUMERICAL VALIDATION" in rec["stdout"] or rec["decomposition"] == "2d"
        records.append(rec)
    dest = os.environ.get("MGXBENCH_RECORD_DROPIN")
    if dest:
        Path(dest).write_text(json.dumps(records, indent=1) + "\n")

"""Drop-in for MGXBench's autotuning/predictive.py: `benchmark.py --libraries AUTO` imports
`auto` from here (benchmark.py:83-85) and gets this library's learned cost model instead of the
regression over communication libraries (autotuning/predictive.py:606-657).

Put this directory's `autotuning/` in MGXBench's tree in place of its own, or ahead of it on
sys.path.  The library is found as an installed `mgxbench_b200` package, else at
$MGXBENCH_B200_ROOT (the repository root), else relative to this file's place in the repository.
"""
import os
import sys
from pathlib import Path

try:
    import mgxbench_b200  # noqa: F401
except ImportError:
    _root = os.environ.get("MGXBENCH_B200_ROOT") or str(Path(__file__).resolve().parents[3])
    sys.path.insert(0, _root)

from mgxbench_b200.predictive import auto  # noqa: E402,F401

__all__ = ["auto"]

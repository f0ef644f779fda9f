"""The autotuner's decision table on the host (no GPU): SP2B_TUNE_FILE is read on first
use (comments skipped, the later line for a key wins), sp2b_tune_set records a decision
and appends it to the file, keys without spaces only; sp2b_tune_clear empties the table."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

SCRIPT = r"""
import sp2b
from sp2b import _lib
print(sp2b.tune_get("subgraph/f64/sm148/512x4,"))
print(sp2b.tune_get("f64-step/sm148/np1024"))
print(sp2b.tune_get("missing/key"))
sp2b.tune_set("subgraph/split/sm148/384x2,", 1)
print(sorted(sp2b.tune_keys()))
try:
    sp2b.tune_set("bad key", 1)
    print("accepted")
except _lib.SP2Error:
    print("rejected")
sp2b.tune_clear()
print(sp2b.tune_keys())
"""


def test_tune_table_file(tmp_path):
    f = tmp_path / "tune.txt"
    f.write_text("# launch choices\n"
                 "subgraph/f64/sm148/512x4, 32 1.5000 1.2500\n"
                 "f64-step/sm148/np1024 128 0.3 0.4\n"
                 "f64-step/sm148/np1024 64\n")
    env = dict(os.environ, SP2B_TUNE_FILE=str(f),
               PYTHONPATH=os.pathsep.join([os.path.join(REPO, "qmd-progress_b200"),
                                           os.environ.get("PYTHONPATH", "")]))
    out = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    assert lines[0] == "(32, [1.5, 1.25])"
    assert lines[1] == "(64, [])"
    assert lines[2] == "None"
    assert lines[3] == str(sorted(["subgraph/f64/sm148/512x4,", "f64-step/sm148/np1024",
                                   "subgraph/split/sm148/384x2,"]))
    assert lines[4] == "rejected"
    assert lines[5] == "[]"
    assert f.read_text().splitlines()[-1] == "subgraph/split/sm148/384x2, 1"

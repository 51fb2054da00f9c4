"""bench.py's command line on the CPU: a weight file named on the command line
that does not exist ends the run with an error before any device work (a
silent switch to the run without the learned start would time another
variant under the same metric)."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_missing_weight_file_is_an_error(tmp_path):
    missing = str(tmp_path / "no_such_weights.bin")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--unet-weights", missing],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode != 0
    assert "no weight file" in r.stderr
    assert r.stdout.strip() == ""

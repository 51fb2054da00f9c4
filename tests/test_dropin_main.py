"""The reference's own driver (main_3d.c, unchanged) linked against this
library runs a deck and writes the same output files as the reference
program.  Both executables come from oracle/Makefile (`make ref`)."""
import filecmp
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "oracle", "_ref", "hydro3d_b200")
REF = os.path.join(ROOT, "oracle", "_ref", "hydro3d_ref")

DECK_KH = """problem = KELVIN_HELMHOLTZ_3D
nx = 20
ny = 18
nz = 16
t_end = 0.02
output_dt = 0.01
cfl = 0.4
gamma = 1.4
G_const = 0.0
bc_xmin = PERIODIC
bc_xmax = PERIODIC
bc_ymin = REFLECTIVE
bc_ymax = REFLECTIVE
bc_zmin = PERIODIC
bc_zmax = PERIODIC
output_dir = output
"""

DECK_BLAST_GRAV = """problem = BLAST_WAVE_3D
nx = 16
ny = 16
nz = 16
xmin = -0.5
xmax = 0.5
ymin = -0.5
ymax = 0.5
zmin = -0.5
zmax = 0.5
t_end = 0.002
output_dt = 0.001
G_const = 1.0
bc_xmin = OUTFLOW
bc_xmax = OUTFLOW
bc_ymin = OUTFLOW
bc_ymax = OUTFLOW
bc_zmin = OUTFLOW
bc_zmax = OUTFLOW
output_dir = output
"""


def run(exe, d, deck):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "deck.txt"), "w") as f:
        f.write(deck)
    r = subprocess.run([exe, "deck.txt"], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return sorted(os.listdir(os.path.join(d, "output")))


@pytest.mark.skipif(not (os.path.exists(OURS) and os.path.exists(REF)), reason="drop-in binaries not built")
@pytest.mark.parametrize("deck", [DECK_KH, DECK_BLAST_GRAV], ids=["kh_periodic_reflective", "blast_gravity"])
def test_main_3d_dropin_outputs_identical(tmp_path, deck):
    a = run(OURS, str(tmp_path / "ours"), deck)
    b = run(REF, str(tmp_path / "ref"), deck)
    assert a == b and len(a) >= 4
    for fn in a:
        assert filecmp.cmp(tmp_path / "ours" / "output" / fn, tmp_path / "ref" / "output" / fn,
                           shallow=False), fn


@pytest.mark.skipif(not os.path.exists(OURS), reason="drop-in binary not built")
def test_main_3d_binary_checkpoint_restart(tmp_path):
    """The unchanged driver with `checkpoint_every` writes binary checkpoints in
    the background; restarting from one through the driver's own restart keys
    (load_from_csv_restart recognises the file) continues bit for bit: the
    final output equals the uninterrupted run's, byte for byte."""
    deck = DECK_BLAST_GRAV.replace("t_end = 0.002", "t_end = 0.004") + "checkpoint_every = 2\ncheckpoint_file = run.ckpt\n"
    full = tmp_path / "full"
    outs = run(OURS, str(full), deck)
    ck = full / "run.ckpt"
    assert ck.exists()
    rdir = tmp_path / "restart"
    os.makedirs(rdir / "output", exist_ok=True)
    restart = (deck.replace("checkpoint_every = 2\n", "") +
               f"restart = true\nrestart_file = {ck}\nrestart_time = 0.0\nrestart_step = 50\n")
    outs_r = run(OURS, str(rdir), restart)
    last = sorted(f for f in outs if f.endswith(".csv"))[-1]
    last_r = sorted(f for f in outs_r if f.endswith(".csv"))[-1]
    assert last_r >= "output_000050.csv"
    assert filecmp.cmp(full / "output" / last, rdir / "output" / last_r, shallow=False), (last, last_r)

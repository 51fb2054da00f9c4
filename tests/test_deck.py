"""Input-deck parser parity: this library's input_deck.c against the
reference's, field by field (oracle/deck_dump.c built against each)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "oracle", "deck_dump_b200")
REF = os.path.join(ROOT, "oracle", "_ref", "deck_dump_ref")

DECKS = {
    "octant": """# octant explosion layout
problem = STELLAR_OCTANT_EXPLOSION_3D
nx = 64
ny = 48
nz = 40      # trailing comment
xmin = 0.0
xmax = 1.5
  ymin=0.0
ymax =1.5
zmin= 0.0
zmax = 1.5
t_end = 5.0
output_dt = 0.01
cfl = 0.35
gamma = 1.666667
G_const = 1.0
bc_xmin = REFLECTIVE
bc_xmax = OUTFLOW
bc_ymin = REFLECTIVE
bc_ymax = OUTFLOW
bc_zmin = REFLECTIVE
bc_zmax = PERIODIC
stellar_profile = star n3.txt
explosion_energy = 0.1
explosion_radius = 0.2
explosion_type = kinetic
output_dir = out_dir # comment
restart = true
restart_file = out/output_000010.csv
restart_step = 10
restart_time = 1.0
enable_perturbations = 1
perturbation_seed = 7
perturb_velocity_modes = 5
perturb_density_amplitude = 0.05
enable_sph_harmonic_mode = true
sph_harmonic_l = 2
sph_harmonic_m = -1
enable_torus = true
torus_rotation_velocity = 0.3
""",
    "binary_and_junk": """
problem = BINARY_STAR_3D
star1_profile = s1.txt
star2_profile = s2.txt
binary_auto_orbit = false
binary_separation = 0.5
star1_vx = 1e-3
star2_vz = -2.5E+1
unknown_key = 5
= no key
novalue =
bc_xmin = SIDEWAYS
problem_extra = 1
G_const = -1
nx = 12abc
#commented = 3
   # indented comment
problem = NOT_A_PROBLEM
""",
    "defaults": "# nothing set\n",
}


@pytest.mark.skipif(not (os.path.exists(OURS) and os.path.exists(REF)),
                    reason="deck dump programs not built (make -C oracle; make -C oracle ref)")
@pytest.mark.parametrize("name", sorted(DECKS))
def test_deck_fields_match_reference(tmp_path, name):
    p = tmp_path / f"{name}.txt"
    p.write_text(DECKS[name])
    a = subprocess.run([OURS, str(p)], capture_output=True, text=True, check=True)
    b = subprocess.run([REF, str(p)], capture_output=True, text=True, check=True)
    assert a.stdout == b.stdout
    # same warnings, in the same order
    wa = [l for l in a.stderr.splitlines() if l.startswith("Warning")]
    wb = [l for l in b.stderr.splitlines() if l.startswith("Warning")]
    assert wa == wb


@pytest.mark.skipif(not os.path.exists(OURS), reason="deck dump not built")
def test_missing_deck_uses_defaults(tmp_path):
    a = subprocess.run([OURS, str(tmp_path / "absent.txt")], capture_output=True, text=True, check=True)
    assert "nx 128" in a.stdout and "Could not open input file" in a.stderr

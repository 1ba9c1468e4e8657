"""bin/elp_ne_list: the lines a tiled run needs in the reference analysis's
ne_list (analysis/mode_init.c:699-727 reads Ne and the time factor of the
run's Executable at its density), built from the efpol lines of a ne_list
with the time factor divided by the geometry's measured clock factor."""
import os
import subprocess

import elp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "mc-polymer-simulation_b200", "bin", "elp_ne_list")
SAMPLE = """# d // Ne-fac // Pre-fac // Time-factor // Moves/s (in millions)
efpol 1.2 124 1.08 0.85 30
efpol 0.9 132 0.91 0.85 30
gpupol3 1.2 121 1.05 1.1 4000
"""


def test_lines_for_every_measured_tile_shape(tmp_path):
    p = tmp_path / "ne_list.dat"
    p.write_text(SAMPLE)
    out = subprocess.run([BIN, str(p)], capture_output=True, text=True, check=True).stdout.splitlines()
    shapes = [s for s in [(32, 32, 32), (32, 32, 16), (32, 16, 16), (16, 16, 16), (48, 24, 24)]
              if elp.time_factor(0, *s) > 0]
    assert len(out) == 2 * len(shapes)                 # one per efpol line and shape
    for line in out:
        name, dens, ne, pre, tfac, _ = line.split()
        tx, ty, tz = (int(v) for v in name[len("elp_"):].split("x"))
        f = elp.time_factor(0, tx, ty, tz)
        assert dens in ("1.2", "0.9") and ne == ("124" if dens == "1.2" else "132")
        assert abs(float(tfac) - 0.85 / f) < 1e-3
    assert elp.time_factor(1, 32, 32, 32) == 1.0       # whole box: efpol's clock


def test_unreadable_list_is_an_error(tmp_path):
    r = subprocess.run([BIN, str(tmp_path / "missing.dat")], capture_output=True, text=True)
    assert r.returncode == 192

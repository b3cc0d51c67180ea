"""The literal drop-in: the reference's own Python module built with -DCUDA, its GPU seam
(include/OSCARSSR_Cuda.h) served by srs_b200 through srsoriginal_b200/adapter/ (oracle/Makefile,
target dropin).  calculate_*(gpu=1) of the reference's own code must equal its CPU path
(nthreads=1) on the same host-computed trajectory to the sum kernels' 1e-10, with the reference's
list shapes.  Runs in a subprocess: the module is named sr, like the CPU build of the reference."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")

SCRIPT = r"""
import io, json, sys
from contextlib import redirect_stdout
import numpy as np
sys.path.insert(0, sys.argv[1])
with redirect_stdout(io.StringIO()):
    import sr
o = sr.sr()
o.set_particle_beam(type="electron", name="b", energy_GeV=3.0, x0=[0, 0, -1], d0=[0, 0, 1], current=0.5)
o.set_ctstartstop(0, 2)
o.set_npoints_trajectory(20001)
o.add_bfield_undulator(bfield=[0, 1, 0], period=[0, 0, 0.049], nperiods=31)
out = {"ngpu": o.check_gpu()}
with redirect_stdout(io.StringIO()):
    sg = o.calculate_spectrum(obs=[0, 0, 30], npoints=200, energy_range_eV=[100, 1000], gpu=1)
    sc = o.calculate_spectrum(obs=[0, 0, 30], npoints=200, energy_range_eV=[100, 1000], nthreads=1)
    fg = o.calculate_flux_rectangle(plane="XY", energy_eV=152.25225225225225, width=[0.01, 0.01], npoints=[21, 21],
                                    translation=[0, 0, 30], gpu=1)
    fc = o.calculate_flux_rectangle(plane="XY", energy_eV=152.25225225225225, width=[0.01, 0.01], npoints=[21, 21],
                                    translation=[0, 0, 30], nthreads=1)
    pg = o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04], npoints=[21, 21], translation=[0, 0, 30],
                                             gpu=1)
    pc = o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04], npoints=[21, 21], translation=[0, 0, 30],
                                             nthreads=1)
def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
out["spectrum"] = rel([v for _, v in sg], [v for _, v in sc])
out["spectrum_e"] = rel([e for e, _ in sg], [e for e, _ in sc])
n = 21 * 21
out["flux_len"] = [len(fg), len(fc)]
out["flux"] = rel([v for _, v in fg][:n], [v for _, v in fc][:n])
out["pd_len"] = [len(pg), len(pc)]
out["pd"] = rel([v for _, v in pg][:n], [v for _, v in pc][:n])
print(json.dumps(out))
"""


def test_reference_module_runs_on_srs_b200():
    if not os.path.isdir(DROPIN) or not any(f.startswith("sr") for f in os.listdir(DROPIN)):
        pytest.skip("drop-in module not built (make -C oracle dropin, where the reference sources exist)")
    r = subprocess.run([sys.executable, "-c", SCRIPT, DROPIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["ngpu"] >= 1
    assert out["spectrum_e"] == 0.0
    assert out["spectrum"] <= 1e-10
    assert out["flux"] <= 1e-10 and out["pd"] <= 1e-10
    # the reference's list shapes: gpu=1 -> 2 * No entries (flux and power density, Q5), CPU 1 thread:
    # flux 2 * No, power density No
    assert out["flux_len"] == [2 * 21 * 21, 2 * 21 * 21]
    assert out["pd_len"] == [2 * 21 * 21, 21 * 21]

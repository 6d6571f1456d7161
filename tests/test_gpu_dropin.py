"""The unmodified reference driver (main.c, parameter reader, init, VTK
writer) linked against libhydro_b200.so in place of its hot path
(oracle/_ref/hydro_dropin) against the reference application itself
(oracle/_ref/hydro): same step lines and byte-identical VTK output files.
Skipped where the reference could not be compiled."""
import filecmp
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
NML = """&RUN
tend=200
nstepmax=60
noutput=20
/
&MESH
nx=250
ny=125
nxystep=125
dx=0.004
boundary_left=1
boundary_right=1
boundary_down=1
boundary_up=1
testcase=1
/
&HYDRO
courant_factor=0.8
niter_riemann=10
/
"""


@pytest.mark.skipif(not (os.path.exists(os.path.join(REF, "hydro_dropin"))
                         and os.path.exists(os.path.join(REF, "hydro"))),
                    reason="reference application not compiled here")
def test_reference_driver_runs_on_the_gpu_path(tmp_path, product_lib):
    outs = {}
    for name in ("hydro", "hydro_dropin"):
        d = tmp_path / name
        d.mkdir()
        (d / "in.nml").write_text(NML)
        env = dict(os.environ, HYDRO_B200_SYNC="1", OMP_NUM_THREADS="4")
        r = subprocess.run([os.path.join(REF, name), "-i", "in.nml"], cwd=d, env=env,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        steps = re.findall(r"--> step=\s*(\d+),\s*(\S+),\s*(\S+)", r.stdout)
        assert len(steps) == 60
        outs[name] = (d, steps)
    assert outs["hydro"][1] == outs["hydro_dropin"][1]
    a, b = outs["hydro"][0], outs["hydro_dropin"][0]
    files = sorted(os.path.relpath(os.path.join(dp, f), a)
                   for dp, _, fs in os.walk(a) for f in fs if f.endswith(".vtr"))
    assert len(files) >= 3
    for f in files:
        assert filecmp.cmp(os.path.join(a, f), os.path.join(b, f), shallow=False), f

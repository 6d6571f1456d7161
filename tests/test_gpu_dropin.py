"""The unmodified reference driver (main.c, parameter reader, init, VTK
writer) linked against libhydro_b200.so in place of its hot path
(oracle/_ref/hydro_dropin), and with the library's VTK writer too
(oracle/_ref/hydro_dropin_vtk), against the reference application itself
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
NML_TEMPLATE = """&RUN
tend=200
nstepmax=60
noutput=20
/
&MESH
nx={nx}
ny={ny}
nxystep={nxystep}
dx={dx}
boundary_left={b[0]}
boundary_right={b[1]}
boundary_down={b[2]}
boundary_up={b[3]}
testcase={tc}
/
&HYDRO
courant_factor={cf}
niter_riemann={niter}
scheme={scheme}
iorder={iorder}
slope_type={slope}
/
"""
# The 250x125 corner case of the bench configs, and two others that reach the
# absorbing / periodic walls, the other schemes, first order and slope_type != 1.
NMLS = {
    "corner_250x125": dict(nx=250, ny=125, nxystep=125, dx=0.004, b=(1, 1, 1, 1), tc=1, cf=0.8,
                           niter=10, scheme="muscl", iorder=2, slope=1.0),
    "sod_absorb_plmde": dict(nx=180, ny=96, nxystep=32, dx=0.01, b=(2, 2, 1, 2), tc=2, cf=0.7,
                             niter=10, scheme="plmde", iorder=2, slope=1.5),
    "centre_periodic_collela": dict(nx=128, ny=160, nxystep=64, dx=0.0078125, b=(3, 3, 3, 3),
                                    tc=0, cf=0.5, niter=5, scheme="collela", iorder=1, slope=1.0),
}
NML = NML_TEMPLATE.format(**NMLS["corner_250x125"])


def timer_line(stdout):
    """The driver's timer table (main.c:515-525): the label line (GATCON ...
    ALLRED) and the PE0_DP line of seconds under it, as {label: seconds}."""
    lines = stdout.splitlines()
    for k, line in enumerate(lines):
        if line.startswith("PE0_DP") and k > 0:
            return dict(zip(lines[k - 1].split(), (float(x) for x in line.split()[1:])))
    raise AssertionError("no PE0_DP timer line in the driver's output")


# hydro_dropin: the reference's own vtkfile.c reads the host array, which the
# library copies back after every step (HYDRO_B200_SYNC=1).
# hydro_dropin_vtk: the library's vtkfile writes from the device state; the
# host array is never updated during the run.
@pytest.mark.parametrize("nml", sorted(NMLS))
@pytest.mark.parametrize("name,sync", [("hydro_dropin", "1"), ("hydro_dropin_vtk", "0")])
def test_reference_driver_runs_on_the_gpu_path(tmp_path, product_lib, name, sync, nml):
    if not (os.path.exists(os.path.join(REF, name)) and os.path.exists(os.path.join(REF, "hydro"))):
        pytest.skip("reference application not compiled here")
    outs = {}
    for exe, env_sync in (("hydro", "0"), (name, sync)):
        d = tmp_path / exe
        d.mkdir()
        (d / "in.nml").write_text(NML_TEMPLATE.format(**NMLS[nml]))
        env = dict(os.environ, HYDRO_B200_SYNC=env_sync, OMP_NUM_THREADS="4")
        r = subprocess.run([os.path.join(REF, exe), "-i", "in.nml"], cwd=d, env=env,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        steps = re.findall(r"--> step=\s*(\d+),\s*(\S+),\s*(\S+)", r.stdout)
        assert len(steps) == 60
        outs[exe] = (d, steps, r.stdout)
    assert outs["hydro"][1] == outs[name][1]
    # The driver's per-stage timer line (main.c:515-530): the library adds the
    # device time of its fused sweeps to TIM_RIEMAN (the driver itself times
    # compute_deltat into TIM_COMPDT).
    tim = timer_line(outs[name][2])
    assert tim["RIEMAN"] > 0.0 and tim["COMPDT"] > 0.0, tim
    a, b = outs["hydro"][0], outs[name][0]
    files = sorted(os.path.relpath(os.path.join(dp, f), a)
                   for dp, _, fs in os.walk(a) for f in fs
                   if f.endswith((".vtr", ".pvtr", ".pvd")))
    assert sum(f.endswith(".vtr") for f in files) >= 3
    for f in files:
        assert filecmp.cmp(os.path.join(a, f), os.path.join(b, f), shallow=False), f


@pytest.mark.parametrize("nx,ny", [(37, 29), (33, 17), (34, 17), (250, 125)])
def test_vtk_base64_payload_matches_float_cast(product_lib, nx, ny):
    """The device encoder against numpy's float32 cast (round to nearest even,
    as C's (float) cast) and the standard base64 of the bytes."""
    import base64

    import numpy as np

    from hydro_b200 import Domain, make_params
    H = make_params(nx, ny)
    rng = np.random.default_rng(nx * ny)
    u = rng.standard_normal((4, ny + 4, nx + 4)) * np.exp(rng.uniform(-100, 100, (4, ny + 4, nx + 4)))
    u[0, 2, 2] = 1e-41  # a float subnormal after the cast
    u[1, 3, 3] = -0.0
    u[2, 2, 3] = 1.0000000596046448  # a tie between two floats
    d = Domain(H)
    d.upload(u)
    for v in range(4):
        with np.errstate(over="ignore"):  # values beyond float range become inf, as in C
            want = base64.b64encode(u[v, 2:-2, 2:-2].astype(np.float32).tobytes())
        assert d.vtk_base64(v) == want, v
    d.close()

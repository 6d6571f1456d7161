"""Domain split on one B200: every subdomain of the split held in this
process (the transport is a device copy), each advanced by the library's
single sweeps with halos packed and unpacked by its kernels.  The assembled
result must equal the single-grid run bit for bit (FP64: hence the
reference; mixed: the single-grid mixed run), with the same dt sequence."""
import numpy as np
import pytest
import torch

from hydro_b200 import Domain, init_state, make_params
from hydro_b200.params import init_noisy_blast
from hydro_b200.split import gather_global, split_gpu_local
from _helpers import describe_mismatch
from _split_oracle import strip_index

pytestmark = pytest.mark.gpu


def single(Hg, u0, nsteps, precision):
    d = Domain(Hg, precision=precision)
    d.upload(u0)
    d.set_clock()
    dts = []
    for _ in range(nsteps):
        d.launch_steps(1)
        dts.append(d.get_clock()[2])
    u = d.download()
    t, n, _ = d.get_clock()
    d.close()
    assert n == nsteps
    return u, dts, t


def outer_mask(Hg):
    m = np.zeros((Hg.ny + 4, Hg.nx + 4), dtype=bool)
    m[2:-2, :] = True
    m[:, 2:-2] = True
    return m


def test_halo_pack_unpack_layout(product_lib):
    H = make_params(29, 23, boundary=(0, 0, 0, 0))
    rng = np.random.default_rng(7)
    u = rng.random((4, 27, 33))
    d = Domain(H)
    d.upload(u)
    for idim in (1, 2):
        n = d.halo_count(idim)
        assert n == 8 * (23 if idim == 1 else 29)
        for side in (0, 1):
            buf = torch.empty(n, dtype=torch.float64, device="cuda")
            d.halo_pack(0, idim, side, buf.data_ptr())
            d.synchronize()
            r, c = strip_index(u.shape, idim, side, ghost=False)
            assert np.array_equal(buf.cpu().numpy(), u[:, r, c].reshape(-1))
            src = torch.from_numpy(rng.random(n)).cuda()
            torch.cuda.synchronize()
            d.halo_unpack(idim, side, src.data_ptr())
            got = d.download()
            r, c = strip_index(u.shape, idim, side, ghost=True)
            assert np.array_equal(got[:, r, c].reshape(-1), src.cpu().numpy())
            u = got
    d.close()


@pytest.mark.parametrize("gx,gy,tc,nparts,bnd", [
    (37, 29, 0, 4, (1, 1, 1, 1)),
    (256, 192, 1, 6, (1, 1, 1, 1)),
    (130, 70, 2, 2, (1, 1, 1, 1)),
    (96, 96, 0, 9, (2, 2, 2, 2)),
    (200, 120, 0, 3, (1, 2, 2, 1)),
    (1024, 1024, 0, 4, (1, 1, 1, 1)),
])
@pytest.mark.parametrize("overlap,kernels", [(False, None), (True, None),
                                             (True, ("march", "march")), (True, ("coop", "coop"))])
def test_split_equals_single_grid_fp64(product_lib, gx, gy, tc, nparts, bnd, overlap, kernels):
    """With overlap, every sweep runs as its ghost-free windows before the
    exchange and the other windows after the unpack, for each kind of sweep
    kernel."""
    Hg = make_params(gx, gy, testcase=tc, boundary=bnd)
    u0 = init_state(Hg, tc)
    nsteps = 40
    want, dts, t = single(Hg, u0, nsteps, "fp64")
    run = split_gpu_local(Hg, u0, nparts, overlap=overlap, kernels=kernels)
    assert run.run(nsteps) == nsteps
    got = gather_global(Hg, run.subs)
    m = outer_mask(Hg)
    assert np.array_equal(got[:, m], want[:, m]), describe_mismatch(got[:, m], want[:, m])
    assert run.dts == dts and run.t == t
    for s in run.subs:
        s.close()


def test_split_equals_single_grid_mixed(product_lib):
    Hg = make_params(300, 220, testcase=1)
    u0 = init_noisy_blast(Hg, 20261203, testcase=1)
    want, dts, t = single(Hg, u0, 30, "mixed")
    run = split_gpu_local(Hg, u0, 6, precision="mixed")
    run.run(30)
    got = gather_global(Hg, run.subs)
    m = outer_mask(Hg)
    assert np.array_equal(got[:, m], want[:, m]), describe_mismatch(got[:, m], want[:, m])
    assert run.dts == dts and run.t == t
    for s in run.subs:
        s.close()


@pytest.mark.parametrize("overlap", [0, 1])
def test_nccl_driver_single_rank(product_lib, tmp_path, overlap):
    """The torch.distributed driver on the GPU with NCCL, one rank: the dt
    all-reduce runs on the subdomain's stream and the run equals the
    single-grid run bit for bit.  (Halo exchanges between ranks need two GPUs;
    their host logic is covered by the gloo tests.)"""
    import json
    import os
    import subprocess
    import sys
    from test_multiproc import ROOT, free_port
    code = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, torch, torch.distributed as dist
from hydro_b200 import Domain, init_state, make_params
from hydro_b200.split import DistComm, GpuSubdomain, SplitRun, decompose, local_params, scatter_state
dist.init_process_group("nccl", init_method="env://", device_id=torch.device("cuda:0"))
Hg = make_params(200, 120, testcase=0)
u0 = init_state(Hg)
box = decompose(Hg.nx, Hg.ny, 1)[0]
sub = GpuSubdomain(local_params(Hg, box, 0, 1), box, 0, "cuda:0")
sub.upload(scatter_state(u0, box))
run = SplitRun(Hg, [sub], DistComm(), overlap=bool(int(sys.argv[2])))
run.run(24)
got = sub.download()
sub.close()
d = Domain(Hg); d.upload(u0); d.set_clock(); d.launch_steps(24); want = d.download(); t = d.get_clock()[0]; d.close()
print(json.dumps({"equal": bool(np.array_equal(got.view(np.uint64), want.view(np.uint64))),
                  "t_equal": run.t == t}))
dist.destroy_process_group()
"""
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(free_port()), NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", code, ROOT, str(overlap)], env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    assert rec == {"equal": True, "t_equal": True}, rec


@pytest.mark.parametrize("gx,gy,tc,nparts", [(256, 192, 1, 6), (200, 120, 0, 3)])
def test_split_against_the_oracle(product_lib, oracle, gx, gy, tc, nparts):
    """The split checked directly against the CPU oracle (itself bitwise the
    reference), not only through the single-grid GPU run: interior cells
    bitwise, the dt sequence equal."""
    from _helpers import orc_from_H
    Hg = make_params(gx, gy, testcase=tc)
    p = orc_from_H(oracle, Hg)
    want = oracle.init_state(p, tc)
    u0 = want.copy()
    nsteps = 30
    n, wdts, wt = oracle.run(p, want, nsteps)
    assert n == nsteps
    run = split_gpu_local(Hg, u0, nparts, overlap=True)
    assert run.run(nsteps) == nsteps
    got = gather_global(Hg, run.subs)
    assert np.array_equal(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2]), \
        describe_mismatch(got[:, 2:-2, 2:-2], want[:, 2:-2, 2:-2])
    assert list(run.dts) == list(wdts) and run.t == wt
    for s in run.subs:
        s.close()


def test_split_mixed_against_the_oracle(product_lib, oracle):
    """The mixed-precision split within the required bound of the CPU oracle."""
    from _helpers import orc_from_H
    from hydro_b200.metrics import field_errors
    Hg = make_params(300, 220, testcase=1)
    p = orc_from_H(oracle, Hg)
    want = oracle.init_state(p, 1)
    u0 = want.copy()
    n, _, wt = oracle.run(p, want, 30)
    run = split_gpu_local(Hg, u0, 6, precision="mixed")
    assert run.run(30) == 30
    got = gather_global(Hg, run.subs)
    err = field_errors(got[:, 2:-2, 2:-2].copy(), want[:, 2:-2, 2:-2].copy())
    assert err["rho"]["l1_rel"] <= 1e-5 and err["E"]["l1_rel"] <= 1e-5, err
    assert abs(run.t - wt) <= 1e-5 * wt
    for s in run.subs:
        s.close()

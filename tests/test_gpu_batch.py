"""Batches: many grids of different sizes advanced by one persistent launch
per sweep.  Each instance must produce exactly what it produces alone: FP64
instances bitwise equal to single-domain runs (hence to the reference), mixed
instances bitwise equal alone and in any mix, under any tiling, and when
admitted mid-run with a different step parity."""
import numpy as np
import pytest

from hydro_b200 import Batch, Domain, init_state, make_blast_mix, make_params
from hydro_b200.batch import blast_instance
from _helpers import bitwise_equal, describe_mismatch

pytestmark = pytest.mark.gpu
ARENA = 1 << 30


def alone(H, u0, nsteps, precision, tend=1e300):
    d = Domain(H, precision=precision)
    d.upload(u0)
    d.set_clock()
    d.launch_steps(nsteps, tend=tend)
    u = d.download()
    t, n, dt = d.get_clock()
    d.close()
    return u, t, n


def mix_of(n, seed, lo=24, hi=200):
    return make_blast_mix(n, seed, side_lo=lo, side_hi=hi)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("threads", [64, 128])
def test_batch_instances_equal_their_single_runs(product_lib, precision, threads):
    """Every instance equals its single-domain run bit for bit, for either CTA
    size of the item kernels (their register caps differ from the
    single-grid kernels')."""
    inst = mix_of(7, 11) + [(make_params(37, 29, testcase=1), init_state(make_params(37, 29), 1))]
    b = Batch(inst[0][0], capacity=16, arena_bytes=ARENA, precision=precision)
    b.set_tuning(64, 4, 0, threads)
    slots = [b.add(H, u) for H, u in inst]
    b.steps(30)
    for s, (H, u0) in zip(slots, inst):
        got = b.download(s)
        st = b.status(s)
        want, t, n = alone(H, u0, 30, precision)
        assert st["nstep"] == n == 30 and st["t"] == t
        assert bitwise_equal(got, want), (H.nx, H.ny, describe_mismatch(got, want))
    b.close()


def test_per_instance_tend(product_lib):
    inst = mix_of(4, 5)
    b = Batch(inst[0][0], capacity=8, arena_bytes=ARENA, precision="fp64")
    tends = []
    for k, (H, u) in enumerate(inst):
        _, t3, _ = alone(H, u, 3 + 2 * k, "fp64")
        tends.append(t3 * 0.999)  # stops after 3 + 2k steps
    slots = [b.add(H, u, tend=te) for (H, u), te in zip(inst, tends)]
    b.steps(20)
    for k, s in enumerate(slots):
        st = b.status(s)
        assert not st["active"] and st["nstep"] == 3 + 2 * k
        want, _, _ = alone(inst[k][0], inst[k][1], 3 + 2 * k, "fp64")
        assert bitwise_equal(b.download(s), want)
    b.close()


def test_alone_and_in_mix_and_any_tiling(product_lib):
    """Mixed precision: an instance's result does not depend on its company,
    the queue order, the tiling (threads per CTA included) or the autotuner."""
    H, u = blast_instance(160, 96, 0.3, 0.7, 2.0, 1.1)
    solo = Batch(H, capacity=2, arena_bytes=ARENA, precision="mixed")
    s0 = solo.add(H, u)
    solo.steps(24)
    ref = solo.download(s0)
    solo.close()
    for seg, claim, bps, threads in [(32, 1, 0, 64), (128, 16, 1, 128), (64, 4, 2, 64),
                                     (64, 4, 0, 128)]:
        b = Batch(H, capacity=32, arena_bytes=ARENA, precision="mixed")
        others = mix_of(12, seg + claim)
        for Ho, uo in others[:6]:
            b.add(Ho, uo)
        s = b.add(H, u)
        for Ho, uo in others[6:]:
            b.add(Ho, uo)
        b.set_tuning(seg, claim, bps, threads)
        b.steps(24)
        assert bitwise_equal(b.download(s), ref), (seg, claim, bps, threads)
        b.close()
    b = Batch(H, capacity=32, arena_bytes=ARENA, precision="mixed")
    for Ho, uo in mix_of(10, 99):
        b.add(Ho, uo)
    s = b.add(H, u, nstepmax=24)
    n = b.autotune(steps=1)
    b.steps(max(0, 24 - n) + 3)  # nstepmax stops it at 24
    assert b.status(s)["nstep"] == 24
    assert bitwise_equal(b.download(s), ref)
    b.close()


def test_admission_mid_run_with_other_parity(product_lib):
    inst = mix_of(5, 21)
    b = Batch(inst[0][0], capacity=8, arena_bytes=ARENA, precision="fp64")
    first = [b.add(H, u) for H, u in inst[:3]]
    b.steps(5)  # odd: the first three are now at odd steps
    late = [b.add(H, u) for H, u in inst[3:]]
    b.steps(8)
    for s, (H, u0) in zip(first, inst[:3]):
        want, _, _ = alone(H, u0, 13, "fp64")
        assert bitwise_equal(b.download(s), want)
    for s, (H, u0) in zip(late, inst[3:]):
        want, _, _ = alone(H, u0, 8, "fp64")
        assert bitwise_equal(b.download(s), want)
    # remove one and keep going: the others are unaffected
    b.remove(first[1])
    b.steps(2)
    want, _, _ = alone(inst[0][0], inst[0][1], 15, "fp64")
    assert bitwise_equal(b.download(first[0]), want)
    b.close()


def test_arena_budget_admission(product_lib):
    H = make_params(200, 200)
    need = Batch.bytes_needed(H)
    b = Batch(H, capacity=8, arena_bytes=3 * need + 1024, precision="mixed")
    u = init_state(H)
    got = [b.try_add(H, u) for _ in range(5)]
    assert [g >= 0 for g in got] == [True, True, True, False, False]
    b.remove(got[1])
    assert b.try_add(H, u) >= 0
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("at", [6, 7])
def test_checkpoint_resume_is_seamless(product_lib, precision, at):
    """Checkpoint an instance at an even or odd step, drop it, resume it in
    another batch: the result equals the uninterrupted run bit for bit."""
    H, u = blast_instance(96, 72, 0.4, 0.6, 1.5, 0.9)
    ref = Batch(H, capacity=2, arena_bytes=ARENA, precision=precision)
    s = ref.add(H, u)
    ref.steps(13)
    want = ref.download(s)
    ref.close()
    a = Batch(H, capacity=4, arena_bytes=ARENA, precision=precision)
    for Ho, uo in mix_of(3, 31):
        a.add(Ho, uo)
    s = a.add(H, u)
    a.steps(at)
    ck = a.checkpoint(s)
    a.remove(s)
    a.close()
    assert ck["nstep"] == at
    b = Batch(H, capacity=4, arena_bytes=ARENA, precision=precision)
    b.add(*mix_of(1, 32)[0])
    s2 = b.resume(ck)
    b.steps(13 - at)
    assert b.status(s2)["nstep"] == 13
    assert bitwise_equal(b.download(s2), want)
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_random_states_equal_single_runs(product_lib, precision):
    """Instances whose cells are all drawn at random (shocks everywhere,
    near-vacuum cells; see _helpers.random_state) in one batch: each equals
    its single-domain run bit for bit."""
    from _helpers import random_state
    inst = []
    for k, (nx, ny, kind) in enumerate([(37, 29, "rough"), (64, 48, "vacuum"), (130, 24, "smooth"),
                                         (24, 96, "vacuum"), (80, 80, "rough")]):
        inst.append((make_params(nx, ny), random_state(nx, ny, 100 + k, kind)))
    b = Batch(inst[0][0], capacity=8, arena_bytes=ARENA, precision=precision)
    slots = [b.add(H, u) for H, u in inst]
    b.steps(12)
    for s, (H, u0) in zip(slots, inst):
        want, t, n = alone(H, u0, 12, precision)
        st = b.status(s)
        assert st["nstep"] == n == 12 and st["t"] == t
        got = b.download(s)
        assert bitwise_equal(got, want), (H.nx, H.ny, describe_mismatch(got, want))
    b.close()


def test_full_batched_workload_fp64_sampled_bitwise(product_lib):
    """The batched workload at its full size (256 seeded instances, sides
    64..1024, 100 steps each) in FP64: every instance finishes its 100 steps,
    and every 16th equals its single-grid run bit for bit."""
    mix = make_blast_mix(256, 20261203)
    arena = sum(Batch.bytes_needed(H) for H, _ in mix) + (1 << 20)
    b = Batch(mix[0][0], capacity=256, arena_bytes=arena, precision="fp64")
    slots = [b.add(H, u, nstepmax=100) for H, u in mix]
    b.autotune(steps=1)
    while b.global_step < 110:
        b.steps(16)
    active, nstep, _ = b.table()
    assert all(nstep[s] == 100 and not active[s] for s in slots)
    for i in range(0, 256, 16):
        H, u0 = mix[i]
        want, _, _ = alone(H, u0, 100, "fp64")
        assert bitwise_equal(b.download(slots[i]), want), (i, H.nx, H.ny)
    b.close()


def test_many_instances_decode_their_items(product_lib):
    """1,100 small FP64 instances (over 1,024 item runs per list, so a warp's
    search for the run of a claimed item takes three rounds): every instance
    finishes its steps, and a sample equals its single-grid run bit for bit."""
    mix = make_blast_mix(1100, 7, side_lo=8, side_hi=48)
    arena = sum(Batch.bytes_needed(H) for H, _ in mix) + (1 << 20)
    b = Batch(mix[0][0], capacity=1100, arena_bytes=arena, precision="fp64")
    slots = [b.add(H, u, nstepmax=12) for H, u in mix]
    b.steps(14)
    active, nstep, _ = b.table()
    assert all(nstep[s] == 12 and not active[s] for s in slots)
    for i in list(range(0, 1100, 97)) + [1098, 1099]:
        H, u0 = mix[i]
        want, _, _ = alone(H, u0, 12, "fp64")
        assert bitwise_equal(b.download(slots[i]), want), (i, H.nx, H.ny)
    b.close()

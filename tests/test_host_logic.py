"""Host-side logic of the tracking loop (no GPU): the injection schedule, the
dump trigger, restart counters, the p/v conversions, the checkpoint file
format, the closed-orbit finder and the multi-rank particle split."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from pyffa_b200.bunch import divide_variables, injection_steps, restart_counters
from pyffa_b200.constants import FFAG_ConversionTools
from pyffa_b200.dump import StepDumpBunch
from pyffa_b200.track import StepDumpSchedule


def _reference_injection(inj_t, t0, dt, nsteps, head=0):
    """Step at which each particle gets injected by the oracle's restatement
    of InjectParticles, run step by step."""
    n = len(inj_t)
    mat = np.zeros((n, 16))
    mat[:, 6] = inj_t
    mat[:head, 7] = 1.0
    h = ctypes.c_int64(head)
    out = np.full(n, -1, np.int64)
    t = t0
    for s in range(nsteps):
        before = mat[:, 7].copy()
        O.lib().orc_inject(mat.ctypes.data, n, t, dt, ctypes.byref(h))
        out[(before == 0) & (mat[:, 7] == 1)] = s
        t = t + dt
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_injection_schedule_matches_step_by_step_rule(seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    dt = 0.37e-9
    t0 = -3.3e-9
    nsteps = 400
    t = t0 + dt * np.arange(nsteps + 1)
    t = np.add.accumulate(np.concatenate([[t0], np.full(nsteps, dt)]))
    # times on window edges, ties, before the first window, in the middle, past the end
    edges = t[rng.integers(0, nsteps, 40)] * 1e9
    inside = rng.uniform(t0 * 1e9 - 5, t[-1] * 1e9 + 5, 300)
    inj = np.sort(np.concatenate([edges, edges[:10], inside, [t0 * 1e9 - 50.0]]))
    ref = _reference_injection(inj, t0, dt, nsteps)
    lo, hi = (t[:nsteps] - dt) * 1e9, t[:nsteps] * 1e9
    got = injection_steps(inj, lo, hi, 0, 0)
    assert np.array_equal(got, ref)
    assert (ref == -1).any() and (ref >= 0).sum() > 100


def test_injection_schedule_with_restart_head():
    inj = np.sort(np.random.Generator(np.random.PCG64(4)).uniform(0, 50, 200))
    dt = 1e-9
    t = np.add.accumulate(np.concatenate([[5e-9], np.full(60, dt)]))
    ref = _reference_injection(inj, 5e-9, dt, 60, head=30)
    got = injection_steps(inj, (t[:60] - dt) * 1e9, t[:60] * 1e9, 0, 30)
    assert np.array_equal(got, ref)


class _FakeBunch:
    def __init__(self, mat):
        self.LocalBunch = mat


def test_dump_schedule_matches_check_and_dump():
    d = tempfile.mkdtemp()
    dump = StepDumpBunch(3.1e-9, 40e-9, 7.3e-9, save_folder=os.path.join(d, "x"))
    fired = []
    dump.dump_bunch = lambda b, t, data_type: fired.append(t)
    dt = 0.41e-9
    t = np.add.accumulate(np.concatenate([[0.0], np.full(200, dt)]))
    for s in range(200):
        dump.check_and_dump(t[s], t[s + 1], None, "Boris")
    steps = StepDumpSchedule(dump).steps_in(t[:200], t[1:201])
    assert np.allclose(t[steps + 1], fired) and len(fired) == len(steps) > 3


def test_checkpoint_file_format_and_append():
    d = tempfile.mkdtemp()
    dump = StepDumpBunch(0.0, 1.0, 1e-9, save_folder=os.path.join(d, "dumps"))
    rng = np.random.Generator(np.random.PCG64(3))
    p = np.zeros((10, 16))
    p[:, 0] = 8.2 + 1e-3 * rng.standard_normal(10)
    p[:, 1] = 1e-3 * rng.standard_normal(10)
    p[:, 5] = 300.0 + rng.standard_normal(10)
    p[:, 8] = 1.0
    p[3, 8] = 0.0
    v = FFAG_ConversionTools().ConvertPrzek2Vrzek_boris(p)
    dump.dump_bunch(_FakeBunch(v), 12.345e-9, "Boris")
    dump.dump_bunch(_FakeBunch(v), 12.345e-9, "Boris")
    fn = os.path.join(d, "dumps", "time_12.35_rank_0.npz")
    arr = np.load(fn)["particles"]
    assert arr.shape == (18, 17)                      # survivors only, appended twice, + time column
    assert np.all(arr[:, 16] == 12.345e-9)
    back = arr[:9, :16]
    np.testing.assert_allclose(back, p[p[:, 8] == 1], rtol=1e-12, atol=1e-15)


def test_conversion_round_trip():
    rng = np.random.Generator(np.random.PCG64(9))
    p = np.zeros((100, 16))
    p[:, 0] = 8 + rng.uniform(0, 1, 100)
    p[:, 1] = 0.05 * rng.standard_normal(100)
    p[:, 3] = 0.01 * rng.standard_normal(100)
    p[:, 5] = rng.uniform(100, 600, 100)
    c = FFAG_ConversionTools()
    np.testing.assert_allclose(c.ConvertVrzek2Przek_boris(c.ConvertPrzek2Vrzek_boris(p)), p, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(c.ConvertVrzek2Przek(c.ConvertPrzek2Vrzek(p)), p, rtol=1e-11, atol=1e-14)


def test_restart_counters():
    a = np.zeros((6, 16))
    a[:4, 7] = 1
    a[[0, 2, 3], 8] = 1
    c = restart_counters(a)
    assert c == {"head": 4, "injected": 4, "uninjected": 2, "survived": 3, "lost": 1}
    a[5, 7] = 1
    with pytest.raises(RuntimeError):
        restart_counters(a)


def test_closed_orbit_is_periodic_and_stable():
    from pyffa_b200 import orbit, synthetic
    cfg = synthetic.lattice_bmap()
    co = orbit.closed_orbits(cfg, np.array([300.0, 450.0]))
    fld = orbit.MidplaneField(cfg)
    p = synthetic.momentum(co["Ek"])
    y0 = np.stack([co["r0"], co["p_r"], np.zeros(2), np.zeros(2)])
    y1 = orbit.track_sector(y0, p, fld)
    np.testing.assert_allclose(y1[0], co["r0"], rtol=1e-10)
    assert np.all(np.isfinite(co["Qx"])) and np.all(np.isfinite(co["Qz"]))
    assert np.all(np.abs(co["trx"]) < 1) and np.all(np.abs(co["trz"]) < 1)


def test_divide_variables_matches_reference_rule():
    for total, size in ((10, 3), (7, 7), (5, 8), (100, 4)):
        parts = [divide_variables(total, r, size) for r in range(size)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(total))
        per = total // size
        for r, part in enumerate(parts):
            assert len(part) == per + (1 if r < total - per * size else 0)


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    total = 1001
    mine = divide_variables(total, rank, world)
    # counts of a bunch split over ranks, summed the way UpdateParticleNumGlobal does
    vals = torch.tensor([len(mine), len(mine) - (mine % 7 == 0).sum()], dtype=torch.int64)
    dist.all_reduce(vals)
    # timing: the max over ranks
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    q.put((rank, vals.tolist(), float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_split_and_reductions_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect_lost = (np.arange(1001) % 7 == 0).sum()
    for rank, vals, tmax in res:
        assert vals == [1001, 1001 - expect_lost]
        assert tmax == 2.0


@pytest.mark.parametrize("n,chunks", [(1, 2), (31, 2), (64, 2), (100000, 2), (3001, 2), (3001, 4), (5000, 1),
                                      (97, 8)])
def test_host_matrix_split_spans(n, chunks):
    from pyffa_b200.track import split_spans
    sp = split_spans(n, chunks)
    assert sp[0][0] == 0 and sp[-1][1] == n
    assert all(a < e for a, e in sp) and all(sp[i][1] == sp[i + 1][0] for i in range(len(sp) - 1))
    assert all(a % 32 == 0 for a, _ in sp)
    assert 1 <= len(sp) <= chunks
    if n >= 32 * chunks:
        assert len(sp) == chunks and max(e - a for a, e in sp) - min(e - a for a, e in sp) < 64

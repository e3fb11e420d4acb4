"""The push kernels' thread order (ffa_state_soa.order, Pusher order="morton"),
host side: morton_order returns a permutation of the range, sorted by the
interleaved-bit key of (r, vr, azimuth within the sector, f5), and tolerates
non-finite values; the bit spreading is exact."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyffa_b200.track import _part1by3, morton_order  # noqa: E402


def test_part1by3_spreads_fifteen_bits():
    x = torch.arange(0, 32768, dtype=torch.int64)
    want = torch.zeros_like(x)
    for b in range(15):
        want |= ((x >> b) & 1) << (4 * b)
    assert torch.equal(_part1by3(x), want)


def test_morton_order_is_a_sorted_permutation():
    rng = np.random.default_rng(3)
    n = 5000
    cols = {"r": torch.as_tensor(8.1 + 3e-3 * rng.standard_normal(n)),
            "vr": torch.as_tensor(2e5 * rng.standard_normal(n)),
            "fi": torch.as_tensor(rng.uniform(-20, 20, n)),
            "f5": torch.as_tensor(2.3e7 * (1 + 1e-3 * rng.standard_normal(n)))}
    cols["r"][7] = float("nan")
    cols["vr"][9] = float("inf")
    period = 2 * np.pi / 12
    for start, cnt in ((0, n), (1024, 2048)):
        p = morton_order(cols, start, cnt, period).numpy()
        assert p.dtype == np.int32 and np.array_equal(np.sort(p), np.arange(cnt))
        # consecutive particles of the order are close in the four coordinates
        # (each scaled to its span): far closer than in the given order
        x = np.stack([np.nan_to_num(cols[k].numpy()[start:start + cnt], nan=0.0, posinf=0.0, neginf=0.0)
                      for k in ("r", "vr", "fi", "f5")], 1)
        x[:, 2] = np.mod(x[:, 2], period)
        x = (x - x.min(0)) / (x.max(0) - x.min(0))
        d_ord = np.median(np.linalg.norm(np.diff(x[p], axis=0), axis=1))
        d_given = np.median(np.linalg.norm(np.diff(x, axis=0), axis=1))
        assert d_ord < 0.3 * d_given, (d_ord, d_given)


def test_particles_not_in_flight_come_last():
    """Lost or not yet injected particles (the push kernels' other branch)
    follow every particle in flight; each group keeps the Morton order."""
    rng = np.random.default_rng(5)
    n = 3000
    cols = {"r": torch.as_tensor(8.1 + 3e-3 * rng.standard_normal(n)),
            "vr": torch.as_tensor(2e5 * rng.standard_normal(n)),
            "fi": torch.as_tensor(rng.uniform(-20, 20, n)),
            "f5": torch.as_tensor(2.3e7 * (1 + 1e-3 * rng.standard_normal(n))),
            "inj": torch.as_tensor((rng.uniform(size=n) > 0.1).astype(np.uint8)),
            "surv": torch.as_tensor((rng.uniform(size=n) > 0.2).astype(np.uint8))}
    p = morton_order(cols, 0, n, 2 * np.pi / 12).numpy()
    assert np.array_equal(np.sort(p), np.arange(n))
    live = ((cols["inj"] == 1) & (cols["surv"] == 1)).numpy()
    k = int(live.sum())
    assert live[p[:k]].all() and not live[p[k:]].any()
    flat = {key: v for key, v in cols.items() if key not in ("inj", "surv")}
    q = morton_order(flat, 0, n, 2 * np.pi / 12).numpy()
    assert np.array_equal(p[:k], q[live[q]])        # the Morton order within the group

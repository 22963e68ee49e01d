"""The batch planner (host-only entry point sa_batch_plan): every problem on exactly one team,
teams contiguous inside the grid, large problems split over several CTAs, and the estimated
makespan close to the ideal. No GPU needed."""
import numpy as np
import pytest

from specann_b200 import batch, build


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build_all()


def c3_sizes(seed=7, count=64, seeds=4):
    """Sizes of the ragged C3 workload: log-uniform n in [2^10, 2^17], half ER (degree 20), half
    BA (m 10 or 20), each instance with `seeds` problems."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 17), count)).astype(np.int64)
    nnz = np.where(np.arange(count) % 2 == 0, 20 * n, 2 * np.where(rng.random(count) < 0.5, 10, 20) * n)
    return np.repeat(n, seeds), np.repeat(nnz, seeds)


def cost(n, z):
    return 8.0 * z + 100.0 * n


@pytest.mark.parametrize("blocks", [1, 7, 148, 296])
@pytest.mark.parametrize("split", [0.5, 1.0, 2.0, 4.0])
def test_plan_partitions_problems_and_grid(blocks, split):
    n, z = c3_sizes()
    team_of, b0, nb = batch.plan(n, z, blocks, split)
    assert len(team_of) == len(n)
    assert team_of.min() >= 0 and team_of.max() == len(b0) - 1
    # contiguous teams from CTA 0, inside the grid
    assert b0[0] == 0 and np.all(b0[1:] == b0[:-1] + nb[:-1]) and b0[-1] + nb[-1] <= blocks
    assert np.all(nb >= 1)
    # every team has work
    assert set(team_of.tolist()) == set(range(len(b0)))


def test_plan_splits_large_problems_and_balances():
    n, z = c3_sizes()
    blocks = 296
    team_of, b0, nb = batch.plan(n, z, blocks, 1.0, 0.05)
    c = cost(n, z)
    big = int(np.argmax(c))
    assert nb[team_of[big]] >= 2                      # the largest problem is split
    load = np.zeros(len(b0))
    for p, t in enumerate(team_of):
        load[t] += c[p] / nb[t] * (1.05 if nb[t] > 1 else 1.0)
    ideal = c.sum() / blocks
    assert load.max() <= 2.0 * ideal, (load.max(), ideal)


def test_plan_with_measured_costs():
    n, z = c3_sizes(count=16, seeds=1)
    cost = np.linspace(1.0, 100.0, len(n))[::-1]          # measured CTA-times, largest first
    team_of, b0, nb = batch.plan(n, z, 32, 1.0, 0.05, cost=cost)
    assert nb[team_of[0]] >= 2                             # the costliest problem is split
    assert set(team_of.tolist()) == set(range(len(b0)))
    with pytest.raises(Exception):
        batch.plan(n, z, 32, 1.0, 0.05, cost=np.zeros(len(n)))


def test_plan_rejects_bad_input():
    with pytest.raises(Exception):
        batch.plan([10, 20], [5, 5], 0)
    with pytest.raises(Exception):
        batch.plan([10, 0], [5, 5], 4)

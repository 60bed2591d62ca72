"""Scene partition of a batch across ranks (cpt.multi.assign_by_cost): every scene on
exactly one rank, the same answer on every rank, and the heaviest rank within one
scene's cost of an even split (the longest-processing-time bound)."""
import numpy as np
import pytest

from cpt.multi import assign_by_cost, scene_cost


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_every_scene_once_and_balanced(world):
    rng = np.random.default_rng(world)
    costs = rng.lognormal(0.0, 1.0, 64)
    parts = assign_by_cost(costs, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
    assert assign_by_cost(list(costs), world) == parts  # deterministic


def test_ties_and_edge_cases():
    assert assign_by_cost([1.0, 1.0, 1.0, 1.0], 2) == [[0, 2], [1, 3]]
    assert assign_by_cost([5.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        assign_by_cost([1.0], 0)


def test_cost_model_orders_scenes():
    small = scene_cost(256 * 256, 10_000, False)
    big = scene_cost(1024 * 1024, 10_000, False)
    hair = scene_cost(256 * 256, 10_000, True)
    assert big > small and hair > small

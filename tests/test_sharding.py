"""Spot sharding across ranks: the assignment on the host, and the sharded
field sum with world_size 2 over gloo (CPU processes, a stand-in march that
deposits a known pattern per spot)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from proton_dose_m1_b200 import Numerics, SolverConfig, phantoms
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.sharding import assign_spots, sharded_field_dose, spot_cost


def test_lpt_assignment_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 10, 101)
    for world in (1, 2, 3, 8):
        shares = assign_spots(costs, world)
        flat = sorted(sum(shares, []))
        assert flat == list(range(101))
        loads = [costs[s].sum() for s in shares]
        # LPT: the largest load exceeds the mean by at most the largest single cost
        assert max(loads) - np.mean(loads) <= costs.max() + 1e-9
    assert assign_spots([5.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        assign_spots(costs, 0)


def test_spot_cost_grows_with_energy_and_width():
    geo, _ = phantoms.ellipsoid_phantom(4)
    grid = Grid.from_geometry(geo)
    beams = phantoms.spot_grid(4, 4, 5e-3)
    cfg = SolverConfig(geometry=geo, beam=beams[0], numerics=Numerics(moving_active_domain=True))
    lo = min(beams, key=lambda b: (b.energy, b.sigma[0]))
    hi = max(beams, key=lambda b: (b.energy, b.sigma[0]))
    assert spot_cost(hi, cfg, grid) > spot_cost(lo, cfg, grid)


def _pattern(k, shape=(6, 5, 7)):
    out = torch.zeros(shape, dtype=torch.float64)
    out.view(-1)[k % out.numel()] = 1.0 + k
    out += 1e-3 * k
    return out


def _rank(rank, world, port, costs, result):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def march_share(idx):
            d = torch.zeros((6, 5, 7), dtype=torch.float64)
            for k in idx:
                d += _pattern(k)
            return d
        dose, share = sharded_field_dose(list(range(len(costs))), costs, rank, world, march_share, dist.all_reduce)
        result[rank] = (dose.numpy().copy(), share)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n_spots", [9, 1])
def test_sharded_field_sum_over_gloo(n_spots):
    costs = list(np.linspace(1, 3, n_spots))
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    result = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, costs, result)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    expect = sum(_pattern(k) for k in range(n_spots)).numpy()
    shares = []
    for r in range(world):
        dose, share = result[r]
        np.testing.assert_allclose(dose, expect, rtol=1e-15, atol=0)
        shares += share
    assert sorted(shares) == list(range(n_spots))

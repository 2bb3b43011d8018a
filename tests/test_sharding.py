"""Spot sharding across ranks: the assignment on the host, and the sharded
field sum over gloo (CPU processes): with a stand-in march that deposits a
known pattern per spot, and with the oracle's march of a small field."""

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


def _field():
    """Three spots on a small water phantom with a bone slab (moving box)."""
    from proton_dose_m1_b200 import Beam, Box, Geometry, Numerics, Physics, SolverConfig
    from proton_dose_m1_b200.enums import EnergyScheme, Material, Scattering
    geo = Geometry(size=(0.012, 0.010, 0.03), resolution=(12, 10, 30),
                   objects=[Box(-0.006, 0.006, -0.005, 0.005, 0.006, 0.009, Material.BONE_COMPACT)])
    beams = [Beam(n_protons=1e6, energy=e, energy_spread=1.0, sigma=(s, s), center=c)
             for e, s, c in ((34.0, 0.0015, (-0.002, 0.0)), (40.0, 0.002, (0.0, 0.001)),
                             (28.0, 0.0012, (0.002, -0.001)))]
    cfg = SolverConfig(geometry=geo, beam=beams[0], physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                                         moving_active_domain=True))
    return cfg, beams


def _oracle_spots(cfg, beams, idx):
    from dataclasses import replace
    from oracle.oracle import OracleProblem, set_threads
    set_threads(1)   # one core per rank: the ranks share the host
    out = np.zeros(tuple(cfg.geometry.resolution))
    for k in idx:
        out += OracleProblem(replace(cfg, beam=beams[k])).march(None)[1]
    return out


def _oracle_rank(rank, world, port, result):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg, beams = _field()
        grid = Grid.from_geometry(cfg.geometry)
        costs = [spot_cost(b, cfg, grid) for b in beams]
        dose, share = sharded_field_dose(beams, costs, rank, world,
                                         lambda idx: torch.from_numpy(_oracle_spots(cfg, beams, idx)),
                                         dist.all_reduce)
        result[rank] = (dose.numpy().copy(), share)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_field_of_oracle_marches_over_gloo(world):
    """Each rank marches its share of a three-spot field with the oracle (the
    CPU restatement of the march; the product marches it on the GPU); the
    all-reduced field dose equals the sum of the single-spot marches.  With
    four ranks one share is empty and its rank still takes the reduction."""
    ctx = mp.get_context("spawn")
    result = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_rank, args=(r, world, port, result)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    cfg, beams = _field()
    expect = _oracle_spots(cfg, beams, range(len(beams)))
    assert expect.max() > 0.0
    shares = []
    for r in range(world):
        dose, share = result[r]
        np.testing.assert_allclose(dose, expect, rtol=0, atol=1e-14 * expect.max())
        shares += share
    assert sorted(shares) == [0, 1, 2]
    assert world < 4 or any(len(result[r][1]) == 0 for r in range(world))

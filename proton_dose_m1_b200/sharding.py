"""Spot sharding of a field over the GPUs of one node.

Pencil beams do not interact (the M1 closure is nonlinear, so every beam is
its own march and the field dose is the sum of the beams' doses), so a field
shards across ranks with no exchange inside the march: each rank marches its
share of the spots as one batched field on its own GPU, and one reduction of
the FP64 field dose (a sum) ends the job.  The reference has no counterpart:
it solves one beam per ``Solver.solve`` call (proton_solver/solver.py:34-218).

``assign_spots`` balances the ranks by longest-processing-time first on a
cost model of the moving-box march: energy steps grow with the start energy
(the CFL step is bounded by the stopping power), box volume with the beam
width and range.
"""

from __future__ import annotations

import heapq

import numpy as np


def spot_cost(beam, config, grid) -> float:
    """Relative cost of one spot's moving-box march: estimated box cells times
    energy steps (both upper estimates)."""
    from .numerics.energy import estimate_box_cells
    num = config.numerics
    E0 = beam.energy + num.energy_window_sigma * beam.energy_spread
    steps = E0 / num.max_energy_step + 1.0
    return float(estimate_box_cells(config, grid, beam)) * steps


def assign_spots(costs, world: int):
    """Longest-processing-time assignment of spots (by cost) to ``world`` ranks.
    Returns one sorted list of spot indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for k in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(s) for s in shares]


def sharded_field_dose(beams, costs, rank: int, world: int, march_share, reduce_sum):
    """This rank's part of a field, then the sum over ranks.

    ``march_share(indices)`` marches the given spots and returns their summed
    dose (a tensor; zeros for an empty share); ``reduce_sum(tensor)`` sums it
    over the ranks in place (e.g. ``torch.distributed.all_reduce``).  Every
    rank takes the same collective step, including a rank whose share is
    empty.  Returns (field dose, this rank's spot indices)."""
    share = assign_spots(costs, world)[rank]
    dose = march_share(share)
    reduce_sum(dose)
    return dose, share


__all__ = ["spot_cost", "assign_spots", "sharded_field_dose"]

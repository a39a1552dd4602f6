"""Density scans sharded over ranks (one process per GPU).

The solves of a scan are independent, so the multi-GPU form shards them: every
rank runs its share with the batched CG driver (``solver.solve_batch``) on its
own GPU and the per-solve scalars are gathered once at the end.  There is no
collective on the data path.  The partition is a greedy longest-processing-time
schedule on a cost estimate (per-k work ~ nk nb^3, FFT ~ nk nb^2 log nk), so
ranks finish close together.  The reference has no multi-device scan; its
users loop over ``solve`` calls (e.g. continuation.py:78-147).
"""

from __future__ import annotations

from typing import Callable, Sequence


def solve_cost(nk1: int, nk2: int, nb: int) -> float:
    """Relative cost of one solve (the ordering key of the batched driver)."""
    return float(nk1) * nk2 * nb * nb * (nb + 8.0)


def partition_solves(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Greedy longest-first assignment of solve indices to ranks (deterministic)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world_size
    parts: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += float(costs[i])
    return parts


def solve_scan(shapes: Sequence[tuple[int, int, int]], run_local: Callable[[list[int]], list[dict]],
               group=None) -> list[dict]:
    """Runs a scan over the ranks of ``group`` (or the default group, or alone).

    shapes: (nk1, nk2, nb) per solve, for the partition.  run_local(indices) runs the
    given solves on this rank and returns one dict of scalars per index (e.g. energy,
    mu, n_iter, converged).  Returns the dicts of all solves in scan order on every rank.
    """
    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    ws = dist.get_world_size(group) if distributed else 1
    rank = dist.get_rank(group) if distributed else 0
    parts = partition_solves([solve_cost(*s) for s in shapes], ws)
    mine = parts[rank]
    local = run_local(list(mine)) if mine else []
    if len(local) != len(mine):
        raise RuntimeError(f"run_local returned {len(local)} results for {len(mine)} solves")
    if not distributed:
        gathered = [local]
    else:
        gathered = [None] * ws
        dist.all_gather_object(gathered, local, group=group)
    out: list[dict | None] = [None] * len(shapes)
    for r, idx in enumerate(parts):
        for i, res in zip(idx, gathered[r]):
            out[i] = res
    return out  # type: ignore[return-value]


def batched_runner(problems, config, lanes: int = 16, device=None):
    """run_local for ``solve_scan`` over synthetic problems with the batched CG driver."""
    def run(indices: list[int]) -> list[dict]:
        import torch
        import jax_hf_b200 as G
        from .solver import solve_batch
        dev = device or torch.device("cuda", torch.cuda.current_device())
        Ks = [G.HartreeFockKernel(**problems[i].kernel_kwargs(), device=dev) for i in indices]
        P0s = [torch.zeros((problems[i].nk, problems[i].nk, problems[i].nb, problems[i].nb),
                           dtype=torch.complex128, device=dev) for i in indices]
        res, times = solve_batch(Ks, P0s, [problems[i].n_electrons for i in indices], config=config,
                                 lanes=lanes, return_times=True)
        return [dict(energy=float(r.energy), mu=float(r.mu), n_iter=int(r.n_iter), converged=bool(r.converged),
                     ms=float(t)) for r, t in zip(res, times)]
    return run


def scan_shapes(problems) -> list[tuple[int, int, int]]:
    return [(p.nk, p.nk, p.nb) for p in problems]


__all__ = ["solve_cost", "partition_solves", "solve_scan", "batched_runner", "scan_shapes"]

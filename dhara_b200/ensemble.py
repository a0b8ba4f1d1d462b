"""Sharding a batch of independent domains over the ranks of a job.

The domains of an ensemble exchange nothing, so a job with one GPU per rank
gives each rank a share of the domains, advances that share in one handle of
its own, and gathers the per-domain diagnostics afterwards; no collective
runs while the domains are stepped.  The share is a greedy bin-pack on the
cell count, which is what a step's work is proportional to.
"""
import numpy as np


def partition(cells, nranks):
    """Domain indices per rank: domains in decreasing cell count (ties by
    index) each go to the rank with the fewest cells so far (ties by rank).
    Every domain lands on exactly one rank; each rank's list is sorted."""
    if nranks < 1:
        raise ValueError("nranks must be at least 1")
    load = [0] * nranks
    share = [[] for _ in range(nranks)]
    for i in sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i)):
        r = min(range(nranks), key=lambda r: (load[r], r))
        share[r].append(i)
        load[r] += int(cells[i])
    return [sorted(s) for s in share]


def gather_diagnostics(local, world):
    """Merges {domain index: diagnostics} from every rank into one dict, the
    same on every rank (torch.distributed all_gather_object when world > 1)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, dict(local))
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise ValueError(f"domain {k} was advanced by two ranks")
            merged[k] = v
    return merged


def run_sharded(domains, nsteps, rank, world, device=0, graph=True, autotune=0):
    """Advances this rank's share of `domains` (inputs.Domain objects) for
    nsteps in one handle on `device`; returns this rank's device time in ms
    (CUDA events on the handle's stream), the number of kernel launches it
    made, and the diagnostics of all domains (plus each domain's largest
    |psi| after the run, "psi_abs_max", and under "launch_config" the
    schedule used), gathered from every rank.  autotune > 0 first lets
    dhara_autotune choose the tile shapes and schedules with that many trial
    steps (the state is restored before the timed run)."""
    import torch
    import dhara_b200 as db
    cells = [d.ncells for d in domains]
    mine = partition(cells, world)[rank]
    local = {}
    ms, launches = 0.0, 0
    if mine:
        s = db.Solver([domains[i].params for i in mine], device=device)
        try:
            for j, i in enumerate(mine):
                s.load(domains[i], j)
            s.prepare()
            cfg = s.autotune(autotune) if autotune > 0 else s.launch_config()
            stream = torch.cuda.ExternalStream(s.stream, device=device)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            s.synchronize()
            lc0 = s.launch_count()
            e0.record(stream)
            s.step(nsteps, graph=graph)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            launches = s.launch_count() - lc0
            for j, i in enumerate(mine):
                local[i] = s.diagnostics(j)
                local[i]["psi_abs_max"] = float(np.abs(s.download("psi", j)).max())
                local[i]["launch_config"] = cfg
        finally:
            s.close()
    return ms, launches, gather_diagnostics(local, world)


def balance(cells, nranks):
    """Largest rank load over the mean load of a partition (1.0 = even)."""
    share = partition(cells, nranks)
    loads = np.array([sum(int(cells[i]) for i in s) for s in share], dtype=np.float64)
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0

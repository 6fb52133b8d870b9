"""Ensembles of independent velocity solves, spread over one process per GPU.

An ensemble member is a (name, grid, config, fields) tuple, e.g. from
``synth.ensemble``.  Members share nothing, so the multi-GPU layout is a
partition: each rank owns a subset of members (longest-processing-time greedy
on the expected cost, columns x expected viscosity iterations), solves them on
its own GPU with the batched entry point (one viscosity iteration of every
unfinished member of a group in flight), and no data crosses GPUs during the
solves.  The per-member reports are gathered on the host at the end
(``torch.distributed.all_gather_object``), the one collective.

The reference has no ensemble driver; each member's solve is its
``solve_DIVA`` (ice_velocity_module.f90:249-374), so a member's result equals
a lone solve of the same inputs.
"""
import heapq
import time

from . import diva

# device bytes of one context per grid column (nz = 15: the 127 fields, the solver's
# work space and the state snapshot taken before each solve), ~18 GB at 1501 x 1501
BYTES_PER_COLUMN = 8.5e3
# viscosity iterations to rel-res 1e-6 observed per member kind (the cost model's
# second factor; only the ratios matter)
EXPECTED_ITERATIONS = {"channel": 90, "icecap": 80, "sheet": 400}


def _grid(g):
    """A member's grid: a diva.Grid or the keyword dict the synth generators return."""
    return diva.Grid(**g) if isinstance(g, dict) else g


def member_cost(member):
    """Expected work of one member: columns x expected viscosity iterations."""
    name, grid = member[0], _grid(member[1])
    kind = name.split("-")[0]
    return grid.nx * grid.ny * EXPECTED_ITERATIONS.get(kind, 100)


def partition(costs, nranks):
    """Longest-processing-time greedy: members in decreasing cost, each to the rank
    with the least load so far (ties to the lowest rank).  Deterministic; returns one
    sorted index list per rank.  The largest load is at most 4/3 of the optimum."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0.0, r) for r in range(nranks)]
    out = [[] for _ in range(nranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + costs[k], r))
    return [sorted(ix) for ix in out]


def groups(members, indices, budget_bytes):
    """Split this rank's members into groups whose contexts fit in ``budget_bytes`` of
    device memory together (a member larger than the budget forms a group of its own)."""
    out, cur, used = [], [], 0.0
    for k in indices:
        g = _grid(members[k][1])
        b = BYTES_PER_COLUMN * g.nx * g.ny
        if cur and used + b > budget_bytes:
            out.append(cur)
            cur, used = [], 0.0
        cur.append(k)
        used += b
    if cur:
        out.append(cur)
    return out


def _prepare(ctx, fields):
    ctx.upload(fields)
    ctx.update_general_ice_model_data()
    ctx.calc_pressure_melting_point()
    ctx.calc_ice_rheology()
    ctx.update_general_ice_model_data()


def solve_members(members, indices, backend, budget_bytes=40e9, outputs=("u_vav_cx", "v_vav_cy"),
                  tile_cache=None):
    """Solve members ``indices`` on this process's device, group by group.  Returns
    {index: {"name", "report", "seconds", <outputs>}}; a member whose solve fails
    carries its status and message in the report instead of outputs.  With
    ``tile_cache`` (a JSON path) each member's smoother tile shapes come from the
    autotuner, which times each grid shape once and caches the choice there; the
    results are the same bit for bit, only the time per V-cycle changes."""
    res = {}
    batched = getattr(backend.lib, backend.prefix + "solve_diva_batch", None) is not None
    for grp in groups(members, indices, budget_bytes):
        ctxs = []
        try:
            for k in grp:
                name, grid, cfg, fields = members[k]
                c = diva.Context(_grid(grid), cfg, backend)
                ctxs.append(c)
                _prepare(c, fields)
                if tile_cache:
                    from . import autotune
                    autotune.tune_tile_edges(c, cache=tile_cache)
                c.state_save()
            t0 = time.perf_counter()
            if batched:
                try:
                    reps = diva.solve_DIVA_batch(ctxs)
                except diva.DivaError:
                    reps = None
            else:
                reps = None
            if reps is None:   # one member failed (or no batched entry point): solve one by one
                reps = []
                for c in ctxs:
                    c.state_restore()          # the prepared state, whatever a failed batch left
                    try:
                        reps.append(c.solve_DIVA())
                    except diva.DivaError as e:
                        reps.append({"status": e.status, "error": str(e)})
            dt = (time.perf_counter() - t0) / len(grp)
            for k, c, r in zip(grp, ctxs, reps):
                ent = {"name": members[k][0], "report": r, "seconds": dt}
                if r.get("status") in (0, 1):
                    ent.update(c.download(list(outputs)))
                res[k] = ent
        finally:
            for c in ctxs:
                c.close()
    return res


def solve_ensemble(members, backend, rank=0, world=1, group=None, budget_bytes=40e9,
                   outputs=("u_vav_cx", "v_vav_cy"), gather=True, tile_cache=None):
    """Solve an ensemble with ``world`` processes: this rank solves its share of the
    longest-processing-time partition.  With ``gather`` (and world > 1) every rank
    returns the results of all members (host all-gather through torch.distributed on
    ``group``); otherwise only its own."""
    parts = partition([member_cost(m) for m in members], world)
    mine = solve_members(members, parts[rank], backend, budget_bytes, outputs, tile_cache)
    if not gather or world == 1:
        return mine, parts
    import torch.distributed as dist
    everything = [None] * world
    dist.all_gather_object(everything, mine, group=group)
    out = {}
    for part in everything:
        out.update(part)
    return out, parts

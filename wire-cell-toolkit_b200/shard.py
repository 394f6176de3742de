"""Work distribution over ranks (one process per GPU).

Events are independent: DepoTransform::operator() (gen/src/DepoTransform.cxx:155-224)
reads nothing but the event's own depos, the face geometry and the plane
responses.  So are the planes of one event: each plane's BinnedDiffusion and
ImpactTransform use only that plane's Pimpos and PIR (:169-213).  Hence:

  * a batch of events is spread over ranks by a greedy balance of depo
    counts (largest event first, onto the least loaded rank);
  * one large event can be split by plane: each rank configures only its
    planes (``plane_config``) and the frame rows are gathered on one rank
    (``gather_rows``);
  * the forward pass needs no collective.  The drift-parameter fit sums its
    loss and three gradients over ranks once per step (``allreduce_sum``).

The collectives go through torch.distributed (NCCL between GPUs, gloo on
CPU); every rank calls them in the same order.
"""

import numpy as np


def greedy_partition(counts, nranks):
    """Event indices per rank, balancing the sum of ``counts``.

    Events are taken in decreasing count (ties by index) and each goes to the
    rank with the smallest load so far (ties to the rank with fewer events,
    then the lower rank), so every rank computes the same assignment.  The
    loads then differ by at most the largest count.  Each rank's list is returned in increasing event order."""
    counts = np.asarray(counts, dtype=np.int64)
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(counts)), key=lambda e: (-int(counts[e]), e))
    load = [0] * nranks
    parts = [[] for _ in range(nranks)]
    for e in order:
        r = min(range(nranks), key=lambda k: (load[k], len(parts[k]), k))
        parts[r].append(e)
        load[r] += int(counts[e])
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def local_events(offsets, rank, nranks):
    """This rank's events of a batch given by ``offsets`` (event e holds depos
    offsets[e] .. offsets[e+1]).  Returns (event indices, depo row indices of
    those events in order, local offsets)."""
    off = np.asarray(offsets, dtype=np.int64)
    if off.ndim != 1 or len(off) < 1 or np.any(np.diff(off) < 0):
        raise ValueError("offsets must be a non-decreasing 1-D array")
    ev = greedy_partition(np.diff(off), nranks)[rank]
    counts = off[1:][ev] - off[:-1][ev]
    loc = np.zeros(len(ev) + 1, dtype=np.int64)
    np.cumsum(counts, out=loc[1:])
    rows = np.concatenate([np.arange(off[e], off[e + 1], dtype=np.int64) for e in ev]) if len(ev) else \
        np.zeros(0, dtype=np.int64)
    return ev, rows, loc


def plane_partition(nplanes, nranks):
    """Planes of one event per rank, round robin (plane p on rank p % nranks)."""
    return [list(range(r, nplanes, nranks)) for r in range(nranks)]


def face_order(gathered, parts, nwires):
    """Rows gathered in rank order (``gather_rows`` of a ``plane_partition``)
    put back in the face's plane order.  nwires[p] = rows of plane p."""
    import torch
    start = {}
    at = 0
    for planes in parts:
        for p in planes:
            start[p] = at
            at += nwires[p]
    if at != gathered.shape[0]:
        raise ValueError("face_order: %d rows gathered, planes hold %d" % (gathered.shape[0], at))
    return torch.cat([gathered[start[p]:start[p] + nwires[p]] for p in range(len(nwires))])


def plane_config(cfg, planes):
    """A copy of a workload configuration (the dict that ``from_config`` takes)
    that keeps only the listed planes and their field responses.  Its frame
    rows equal the full configuration's rows of those planes for the
    unfluctuated forward (the random streams of a fluctuated forward are keyed
    by the plane's position in the face, which changes)."""
    c = dict(cfg)
    c["planes"] = [cfg["planes"][p] for p in planes]
    c["fr"] = [cfg["fr"][p] for p in planes]
    return c


def _dist():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist
    return None


def world():
    """(rank, world size) of the default process group, (0, 1) without one."""
    d = _dist()
    if d is None:
        return 0, 1
    return d.get_rank(), d.get_world_size()


def _coll_device(d, group):
    import torch
    backend = d.get_backend(group)
    return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def allreduce_sum(values, group=None):
    """Sum of a small float64 vector over all ranks (returned as numpy); the
    values themselves without a process group."""
    v = np.asarray(values, dtype=np.float64)
    d = _dist()
    if d is None or d.get_world_size(group) == 1:
        return v.copy()
    import torch
    t = torch.from_numpy(v.copy()).to(_coll_device(d, group))
    d.all_reduce(t, op=d.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def gather_rows(rows, dst=0, group=None):
    """Gather a [n_r][m] float32 tensor from every rank onto rank ``dst``,
    stacked in rank order (the plane-split frame).  Ranks may hold different
    row counts; the rows are padded to the largest for the collective and
    trimmed after.  Returns the stacked tensor on ``dst``, None elsewhere."""
    import torch
    d = _dist()
    if d is None or d.get_world_size(group) == 1:
        return rows
    dev = _coll_device(d, group)
    nr = torch.tensor([rows.shape[0], rows.shape[1]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(nr) for _ in range(d.get_world_size(group))]
    d.all_gather(sizes, nr, group=group)
    sizes = [tuple(int(x) for x in s.cpu()) for s in sizes]
    if len({s[1] for s in sizes}) != 1:
        raise ValueError("gather_rows: ranks hold rows of different lengths")
    nmax = max(s[0] for s in sizes)
    pad = torch.zeros((nmax, rows.shape[1]), dtype=rows.dtype, device=dev)
    pad[:rows.shape[0]].copy_(rows)
    me = d.get_rank(group)
    if me == dst:
        bufs = [torch.empty_like(pad) for _ in sizes]
        d.gather(pad, gather_list=bufs, dst=dst, group=group)
        return torch.cat([b[:s[0]] for b, s in zip(bufs, sizes)]).to(rows.device)
    d.gather(pad, dst=dst, group=group)
    return None

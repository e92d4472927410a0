"""The halo exchange of a partitioned step between processes, on CPU with two gloo ranks.

Each rank owns half of the glevel-4 grid (5 of its 10 rhombi; the poles with rank 1) and gets its
halo plan from thorx_halo_columns (host code, no GPU). The ranks swap the lists of what each needs
from the other, then exchange a field by send/recv of packed columns, as a multi-GPU driver would
around thorx_pack_columns / thorx_unpack_columns. Checks: after the exchange every rank holds the
owner's values on its halo; and the plan covers every neighbour of every owned column, with the
neighbours restated here from the reference's rhombus halo tiles
(src/headers/kernel_halo_helpers.h:47-128: the 6 tile offsets, and point_local for the poles).
"""
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def neighbours(grid):
    """{column: set of stencil neighbours} from the rhombus maps (halo tiles) and point_local."""
    import numpy as np
    N, nl, nr = grid["point_num"], grid["nl_region"], grid["nr"]
    nhl = nl + 2
    maps = np.asarray(grid["maps"]).reshape(nr, nhl, nhl)
    out = {}
    for r in range(nr):
        m = maps[r]
        for y in range(nl):
            for x in range(nl):
                ids = [m[y + 2, x + 1], m[y + 2, x + 2], m[y + 1, x + 2], m[y, x + 1], m[y, x],
                       m[y + 1, x]]
                out[int(m[y + 1, x + 1])] = {int(v) for v in ids if v >= 0}
    pl = np.asarray(grid["point_local"]).reshape(N, 6)
    for c in (N - 2, N - 1):
        out[c] = {int(v) for v in pl[c, :5]}
    return out


def _worker(rank, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import numpy as np
    import torch
    import torch.distributed as dist
    import thor_b200
    dist.init_process_group("gloo", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    try:
        grid = thor_b200.Icogrid(4, 8).as_dict()
        N, L = grid["point_num"], 8 * 3  # a field of 8 levels x 3 components per column
        ranges = [(0, 1280), (1280, N)]
        a, b = ranges[rank]
        other = 1 - rank
        halo = thor_b200.halo_columns(grid, 4, a, b)
        # what this rank needs from the other (every halo column belongs to the other here)
        need = torch.from_numpy(halo.astype(np.int64))
        n_mine = torch.tensor([need.numel()])
        n_theirs = torch.zeros(1, dtype=torch.int64)
        if rank == 0:
            dist.send(n_mine, other)
            dist.recv(n_theirs, other)
        else:
            dist.recv(n_theirs, other)
            dist.send(n_mine, other)
        theirs = torch.zeros(int(n_theirs), dtype=torch.int64)  # what the other needs from me
        if rank == 0:
            dist.send(need, other)
            dist.recv(theirs, other)
        else:
            dist.recv(theirs, other)
            dist.send(need, other)
        # the field: a value per (column, level, component) on the owned columns, NaN elsewhere
        field = np.full((N, L), np.nan)
        cidx = np.arange(a, b)
        field[a:b] = cidx[:, None] * 1000.0 + np.arange(L)[None, :]
        send = torch.from_numpy(field[theirs.numpy()].copy())   # packed [n][L]
        recv = torch.zeros((need.numel(), L), dtype=torch.float64)
        if rank == 0:
            dist.send(send, other)
            dist.recv(recv, other)
        else:
            dist.recv(recv, other)
            dist.send(send, other)
        field[need.numpy()] = recv.numpy()                        # unpacked
        want = halo[:, None] * 1000.0 + np.arange(L)[None, :]
        exchanged = bool(np.array_equal(field[halo], want))
        nb = neighbours(grid)
        covered = all(v in set(range(a, b)) or v in set(halo.tolist())
                      for c in range(a, b) for v in nb[c])
        outside = bool(np.all((halo < a) | (halo >= b)))
        no_nan = bool(np.all(np.isfinite(field[[v for c in range(a, b) for v in nb[c]]])))
        q.put((rank, int(need.numel()), int(theirs.numel()), exchanged, covered, outside, no_nan))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_exchange_their_halos():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in (0, 1)]
    for p in procs:
        p.start()
    got = {r[0]: r[1:] for r in (q.get(timeout=180) for _ in procs)}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        need, theirs, exchanged, covered, outside, no_nan = got[r]
        assert exchanged and covered and outside and no_nan, (r, got[r])
        assert need > 0 and theirs == got[1 - r][0]

"""Sessions sharded across GPUs by the router (firepro/router.py), on CPU: the deterministic
assignment alone, and two ranks of a `gloo` process group routing the same arrivals with a
stand-in front end per rank (no GPU). Every rank must agree on where each session lives, no
rank may hold more bytes than its budget or more sessions than its limit, and bytes freed by a
closed session must admit waiting ones."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from firepro.router import Account, SessionRouter, assign


def test_assign_most_free_rank_first():
    accounts = [Account(0, 0), Account(300, 1), Account(0, 4)]
    placed, waiting = assign(accounts, 1000, 4, [(0, 500), (1, 600), (2, 400), (3, 2000)])
    # rank 2 is full (4 sessions); rank 0 has the most free bytes, then rank 1 (700 free vs 500)
    assert [(p.key, p.rank) for p in placed] == [(0, 0), (1, 1), (2, 0)]
    assert waiting == [(3, 2000)]


def test_assign_respects_budget_and_limit():
    accounts = [Account(0, 0), Account(0, 0)]
    arrivals = [(k, 100 + 37 * (k % 7)) for k in range(40)]
    placed, waiting = assign(accounts, 1500, 6, arrivals)
    for r in range(2):
        mine = [p for p in placed if p.rank == r]
        assert sum(p.bytes for p in mine) <= 1500 and len(mine) <= 6
    assert len(placed) + len(waiting) == 40
    # the waiting keep their arrival order
    assert [k for k, _ in waiting] == sorted(k for k, _ in waiting)


class FakeServer:
    def __init__(self):
        self.open_sessions = {}
        self.next = 0

    def open(self, grid):
        s = self.next
        self.next += 1
        self.open_sessions[s] = grid
        return s

    def close(self, s):
        del self.open_sessions[s]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        srv = FakeServer()
        budget, limit = 1000, 5
        router = SessionRouter(srv, budget, limit)
        arrivals = [(k, 120 + 90 * (k % 5), f"grid{k}") for k in range(30)]
        seen = []
        for rnd in range(6):
            batch = arrivals[rnd * 5:(rnd + 1) * 5]
            router.round(batch)
            acc = router.gather()
            for a in acc:
                assert a.bytes <= budget and a.sessions <= limit
            seen.append((rnd, dict(router.where), [len(router.waiting)]))
            # every rank closes its two oldest sessions after round 2
            if rnd >= 2:
                for key in sorted(router.local)[:2]:
                    router.close(key)
        for _ in range(6):  # let the waiting drain as sessions close
            router.round([])
            for key in sorted(router.local)[:3]:
                router.close(key)
        assert len(srv.open_sessions) == len(router.local)
        gathered = [None] * world
        dist.all_gather_object(gathered, (router.where, seen, len(router.waiting)))
        q.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_agree_and_stay_within_budget():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = results[0]
    assert g[0] == g[1]  # every rank holds the same placements, round by round
    where = g[0][0]
    assert len(where) == 30 and g[0][2] == 0  # every arrival placed once the closes freed room
    assert {r for r in where.values()} == {0, 1}  # both GPUs serve sessions

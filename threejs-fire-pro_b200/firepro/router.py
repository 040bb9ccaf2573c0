"""Sessions sharded across GPUs: one serving front end per GPU, one process per GPU.

The step of a simulation never crosses GPUs (a simulation is one GPU's work); serving shards
by session. Every rank of a `torch.distributed` process group owns one server (fp_server_*)
on its own GPU. Each routing round:

  1. every rank reports its accounting (device bytes its admitted sessions hold, their count)
     with one all_gather of a few integers (the `gloo` backend: host-side control messages, no
     device data crosses ranks);
  2. every rank runs the same deterministic assignment over the same arrivals: an arrival goes
     to the rank with the most free bytes (its budget less what its sessions hold) among those
     with a free session slot and room for the session, ties to the lowest rank; an arrival no
     rank has room for waits, in order, for a later round;
  3. each rank opens the sessions assigned to it.

So ranks never disagree about where a session lives, and no rank exceeds its memory budget or
session limit. No reference counterpart: the reference runs one simulation on one device
(FireSimulation.ts:197).
"""
from __future__ import annotations

from dataclasses import dataclass, field


@dataclass
class Account:
    """One rank's admitted sessions: device bytes held, count."""

    bytes: int = 0
    sessions: int = 0


@dataclass
class Placement:
    key: int      # the arrival's key (its position in the arrival order)
    rank: int
    bytes: int


def assign(accounts: list, budget: int, max_sessions: int, arrivals: list) -> tuple:
    """The deterministic assignment of step 2. `accounts` per rank, `arrivals` a list of
    (key, bytes) in arrival order. Returns (placements, waiting): the arrivals placed, with
    their rank, and those left waiting (a session larger than any rank's budget never fits
    and stays waiting; the caller refuses it at open)."""
    free = [budget - a.bytes for a in accounts]
    slots = [max_sessions - a.sessions for a in accounts]
    placed, waiting = [], []
    for key, need in arrivals:
        best = -1
        for r in range(len(accounts)):
            if slots[r] > 0 and free[r] >= need and (best < 0 or free[r] > free[best]):
                best = r
        if best < 0:
            waiting.append((key, need))
            continue
        free[best] -= need
        slots[best] -= 1
        placed.append(Placement(key, best, need))
    return placed, waiting


class SessionRouter:
    """The routing rounds of one rank. `server` is this rank's front end: an object with
    open(grid) -> session, close(session) and memory(session) -> bytes it was admitted with
    (a FireServer through `ServerShard`, or a stand-in in tests). `group` is a process group
    (gloo), or None for a single process."""

    def __init__(self, server, budget: int, max_sessions: int, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group) if group is not None or dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if group is not None or dist.is_initialized() else 1
        self.server = server
        self.budget = budget
        self.max_sessions = max_sessions
        self.local = {}       # key -> (session, bytes) of the sessions this rank holds
        self.waiting = []     # (key, bytes, grid) in arrival order, the same on every rank
        self.where = {}       # key -> rank, the same on every rank

    def account(self) -> Account:
        return Account(sum(b for _, b in self.local.values()), len(self.local))

    def gather(self) -> list:
        mine = [self.account().bytes, self.account().sessions]
        if self.world == 1:
            return [Account(*mine)]
        import torch

        t = torch.tensor(mine, dtype=torch.int64)
        out = [torch.zeros(2, dtype=torch.int64) for _ in range(self.world)]
        self.dist.all_gather(out, t, group=self.group)
        return [Account(int(o[0]), int(o[1])) for o in out]

    def round(self, arrivals=()) -> list:
        """One routing round with this round's `arrivals`, a list of (key, bytes, grid) that
        every rank passes alike. Returns the keys this rank opened."""
        self.waiting += list(arrivals)
        accounts = self.gather()
        placed, left = assign(accounts, self.budget, self.max_sessions, [(k, b) for k, b, _ in self.waiting])
        grids = {k: g for k, _, g in self.waiting}
        keep = {k for k, _ in left}
        self.waiting = [w for w in self.waiting if w[0] in keep]
        opened = []
        for p in placed:
            self.where[p.key] = p.rank
            if p.rank == self.rank:
                self.local[p.key] = (self.server.open(grids[p.key]), p.bytes)
                opened.append(p.key)
        return opened

    def close(self, key: int):
        """Close a session this rank holds; its bytes count as free from the next round."""
        session, _ = self.local.pop(key)
        self.server.close(session)

    def session(self, key: int):
        """This rank's session of `key`, or None when another rank holds it."""
        got = self.local.get(key)
        return got[0] if got else None


class ServerShard:
    """This rank's FireServer as the router's front end: admission bytes from
    fp_grid_memory_bytes, the server's own budget the router's per-rank budget."""

    def __init__(self, server, cutoff: float = 0.05, ground: bool = True):
        self.srv = server
        self.cutoff, self.ground = cutoff, ground

    def open(self, grid):
        return self.srv.open(grid, self.cutoff, self.ground)

    def close(self, session):
        self.srv.close(session)

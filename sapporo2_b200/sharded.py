"""j-particles sharded over the ranks of a torch.distributed process group,
one process per GPU: the multi-GPU scheme of the reference, which spreads j
over its devices round-robin by address (lib/src/sapporohostclass.cpp:473-474:
device = address % nDev, slot = address / nDev), sends every i to every
device, sums the devices' partial forces and takes the nearest neighbour as
a min-loc on (ds2, id) (:749-799), and concatenates the neighbour lists in
device order (:804-880).

Here each rank drives its own GPU (or, in tests, a CPU stand-in) and the
exchange is one collective per force call: an all-reduce SUM of the ten
force fields and an all-reduce MIN of the 64-bit nearest-neighbour keys,
both on the device when the group is NCCL.  Neighbour lists, which only
the host reads, are all-gathered on request.
"""
from __future__ import annotations

import numpy as np

from . import NGB_PB, RES_STRIDE

NO_NGB_DS2 = 1.0e11  # ds2 reported when a rank found no neighbour


def local_count(nj: int, rank: int, world: int) -> int:
    """Number of addresses a < nj with a % world == rank."""
    return max(0, (nj - rank + world - 1) // world)


def nn_keys(res):
    """64-bit keys (float ds2 bits << 32 | id as unsigned 32 bits) of result
    records [ni, RES_STRIDE] (torch float64); the minimum key is the nearest
    neighbour with ties to the smallest id, the device kernels' rule."""
    import torch
    ds2 = res[:, 10].to(torch.float32)
    bits = ds2.view(torch.int32).to(torch.int64)
    ids = res[:, 11].to(torch.int64) & 0xFFFFFFFF
    return (bits << 32) | ids


def decode_keys(keys, res):
    """Writes ds2 and id of the keys back into res[:, 10:12]."""
    import torch
    hi = (keys >> 32).to(torch.int32)
    res[:, 10] = hi.view(torch.float32).to(torch.float64)
    lo = (keys & 0xFFFFFFFF).to(torch.int64)
    lo = torch.where(lo >= 2 ** 31, lo - 2 ** 32, lo)
    res[:, 11] = lo.to(torch.float64)


def combine_partials(res, group=None):
    """All-reduces partial result records [ni, RES_STRIDE] (torch float64,
    on the device for NCCL, on the host for gloo) in place: fields 0..9
    summed, nearest neighbour by minimum key.  Every rank ends with the
    same records."""
    import torch
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return res
    if dist.get_world_size(group) == 1:
        return res
    sums = res[:, :10].contiguous()
    keys = nn_keys(res)
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(keys, op=dist.ReduceOp.MIN, group=group)
    res[:, :10] = sums
    decode_keys(keys, res)
    return res


def merge_lists(counts, lists, ipipe: int, maxlength: int = NGB_PB):
    """The neighbours of i-particle `ipipe` from the per-rank counts [W, ni]
    and lists [W, ni, NGB_PB]: concatenated in rank order, each rank giving
    min(its count, NGB_PB, room left) ids; overflow when the running total
    reaches maxlength (sapporo::get_ngb_list, lib/src/sapporohostclass.cpp:
    837-880) or a rank's count reaches NGB_PB (its ids beyond NGB_PB were not
    stored), as the class does over its devices.  Returns (overflow, total
    count, sorted ids)."""
    out = []
    nblen = 0
    overflow = False
    for r in range(counts.shape[0]):
        n = int(counts[r, ipipe])
        take = max(0, min(n, NGB_PB, maxlength - nblen))
        out.append(lists[r, ipipe, :take])
        nblen += n
        if n >= NGB_PB:
            overflow = True
        if nblen >= maxlength:
            overflow = True
            break
    ids = np.sort(np.concatenate(out)) if out else np.zeros(0, dtype=np.int32)
    return overflow, nblen, ids


class ShardedSapporo:
    """The `Sapporo` interface over the ranks of a process group.  Every rank
    makes the same calls with the same (global) arguments; each keeps the j
    whose address % world == rank.  `backend` is the rank's own `Sapporo`
    (or an object with its methods: set_j_particles, set_time, start,
    raw_results, neighbour_counts, neighbour_lists, close)."""

    def __init__(self, backend, group=None, device=None):
        import torch.distributed as dist
        self.b = backend
        self.group = group
        init = dist.is_available() and dist.is_initialized()
        self.world = dist.get_world_size(group) if init else 1
        self.rank = dist.get_rank(group) if init else 0
        self.device = device  # torch device of the collectives (None: host)
        self._ni = 0
        self._nj_local = 0
        self._lists = None

    # --- j side ----------------------------------------------------------
    def set_j_particles(self, address, id, t, mass, x, v, a, jrk, snp=None, crk=None, eps=None):
        address = np.asarray(address)
        mine = np.nonzero(address % self.world == self.rank)[0]
        if len(mine) == 0:
            return

        def sel(q):
            return None if q is None else np.asarray(q)[mine]
        self.b.set_j_particles(address[mine] // self.world, sel(id), sel(t), sel(mass), sel(x),
                               sel(v), sel(a), sel(jrk), sel(snp), sel(crk), sel(eps))

    def set_time(self, t):
        self.b.set_time(t)

    # --- force -----------------------------------------------------------
    def start(self, nj, id, xi, vi, ai=None, eps2=0.0, h2=None):
        self._ni = len(id)
        self._lists = None
        self._nj_local = local_count(nj, self.rank, self.world)
        if self._nj_local > 0:
            self.b.start(self._nj_local, id, xi, vi, ai, eps2, h2)

    def _local_records(self, ni):
        if self._nj_local > 0:
            return self.b.raw_results(ni)
        r = np.zeros((ni, RES_STRIDE))  # this rank holds no j: neutral partials
        r[:, 10], r[:, 11] = NO_NGB_DS2, -1
        return r

    def raw_results(self, ni=None):
        import torch
        ni = self._ni if ni is None else ni
        res = torch.from_numpy(self._local_records(ni))
        if self.device is not None:
            res = res.to(self.device)
        combine_partials(res, self.group)
        return res.cpu().numpy()

    def results(self, nj, ni=None, ngb=True) -> dict:
        """Combined results in the form of `Sapporo.results` (nearest
        neighbour reported when ds2 < 1e10, lib/src/sapporohostclass.cpp:
        767-774)."""
        r = self.raw_results(ni)
        n = len(r)
        out = {"acc": r[:, 0:3].copy(), "pot": r[:, 3].copy(), "jrk": r[:, 4:7].copy(),
               "snp": r[:, 7:10].copy(), "nnb": np.zeros(n, dtype=np.int32),
               "ds2min": np.full(n, np.nan)}
        if ngb:
            hit = r[:, 10] < 1.0e10
            out["nnb"][hit] = r[hit, 11].astype(np.int32)
            out["ds2min"][hit] = r[hit, 10]
        return out

    # --- neighbour lists -----------------------------------------------------
    def _gather_lists(self):
        if self._lists is not None:
            return self._lists
        import torch
        import torch.distributed as dist
        if self._nj_local > 0:
            cnt, lst = self.b.neighbour_lists(self._ni)
        else:
            cnt = np.zeros(self._ni, dtype=np.int32)
            lst = np.zeros((self._ni, NGB_PB), dtype=np.int32)
        c = torch.from_numpy(np.ascontiguousarray(cnt, dtype=np.int32))
        l_ = torch.from_numpy(np.ascontiguousarray(lst, dtype=np.int32))
        if self.world > 1:
            if self.device is not None:
                c, l_ = c.to(self.device), l_.to(self.device)
            cs = [torch.empty_like(c) for _ in range(self.world)]
            ls = [torch.empty_like(l_) for _ in range(self.world)]
            dist.all_gather(cs, c, group=self.group)
            dist.all_gather(ls, l_, group=self.group)
            counts = torch.stack(cs).cpu().numpy()
            lists = torch.stack(ls).cpu().numpy()
        else:
            counts, lists = c.numpy()[None], l_.numpy()[None]
        self._lists = (counts, lists)
        return self._lists

    def read_ngb_list(self) -> int:
        """1 when any rank's count for any i reached NGB_PB (the reference
        checks each device's counts, lib/src/sapporohostclass.cpp:804-835)."""
        counts, _ = self._gather_lists()
        return int(np.any(counts >= NGB_PB))

    def get_ngb_list(self, ipipe: int, maxlength: int = NGB_PB):
        counts, lists = self._gather_lists()
        ovf, n, ids = merge_lists(counts, lists, ipipe, maxlength)
        return int(ovf), n, ids

    def neighbour_counts(self, ni=None) -> np.ndarray:
        """Exact counts summed over the ranks (one all-reduce of ni ints)."""
        import torch
        import torch.distributed as dist
        ni = self._ni if ni is None else ni
        local = self.b.neighbour_counts(ni) if self._nj_local > 0 else np.zeros(ni)
        c = torch.from_numpy(np.ascontiguousarray(local, dtype=np.int64))
        if self.world > 1:
            if self.device is not None:
                c = c.to(self.device)
            dist.all_reduce(c, op=dist.ReduceOp.SUM, group=self.group)
        return c.cpu().numpy()

    def close(self):
        self.b.close()

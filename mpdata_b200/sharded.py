"""One grid split into z-slabs over the ranks of a torch.distributed group.

Each rank steps its own planes plus a halo of P planes (2P-1 with the
limiter) on each side with an ordinary solver; before every step after the
first the halo planes are refreshed from the ranks that own them by
point-to-point messages (NCCL on CUDA tensors, or gloo through host
buffers).  With that depth the owned planes after each step equal those of
a single-domain run bit for bit (the depth the decomposed msmolar path uses;
tests/test_decomposition.py shows it is exact and one plane less is not).

The split of the z axis (shell planes included) follows the remainder
spreading of the reference's block sizing (multigrid/src/grid.c:68-144),
as msmolar does.  The x and y extents are not split.
"""
from __future__ import annotations

import numpy as np


def split(n: int, parts: int) -> list[int]:
    """Start indices of `parts` contiguous blocks of n (the first n % parts
    blocks one longer), plus n."""
    base, rem = divmod(n, parts)
    st = [0]
    for b in range(parts):
        st.append(st[-1] + base + (1 if b < rem else 0))
    return st


class SlabPlan:
    """Owned and extended (owned + halo) plane ranges of every rank, and the
    messages of one halo refresh."""

    def __init__(self, ns: int, world: int, halo: int):
        if world < 1 or world > ns:
            raise ValueError(f"cannot split {ns} planes over {world} ranks")
        st = split(ns, world)
        self.ns, self.world, self.halo = ns, world, halo
        self.own = [(st[r], st[r + 1]) for r in range(world)]
        self.ext = [(max(0, lo - halo), min(ns, hi + halo)) for lo, hi in self.own]
        for r, (a, b) in enumerate(self.ext):
            if b - a < 3:
                raise ValueError(f"rank {r}: slab of {b - a} planes (at least 3 needed)")

    def owner_pieces(self, a: int, b: int) -> list[tuple[int, int, int]]:
        """[a, b) cut at slab boundaries: (owner rank, start, stop) pieces."""
        out = []
        for r, (lo, hi) in enumerate(self.own):
            s, e = max(a, lo), min(b, hi)
            if s < e:
                out.append((r, s, e))
        return out

    def recvs(self, r: int) -> list[tuple[int, int, int]]:
        """(peer, start, stop) global plane ranges rank r receives, sorted."""
        (lo, hi), (elo, ehi) = self.own[r], self.ext[r]
        return sorted(self.owner_pieces(elo, lo) + self.owner_pieces(hi, ehi))

    def sends(self, r: int) -> list[tuple[int, int, int]]:
        """(peer, start, stop) ranges of rank r's own planes that other ranks
        receive, sorted; matches recvs() of every peer in order."""
        out = []
        for peer in range(self.world):
            if peer != r:
                out += [(peer, s, e) for (o, s, e) in self.recvs(peer) if o == r]
        return sorted(out)


class ShardedSolver:
    """A grid of nx x ny x ns cells over the ranks of `group` (default: the
    default process group), z-slab decomposed.  `make_solver(nx, ny, ns)`
    builds the per-rank solver (default: :class:`mpdata_b200.Solver` with the
    given order, dtype and options); it must offer set_faces, set_field,
    step, get_planes, set_planes and get_field on (ns, ny, nx) arrays.

    With the NCCL backend the halo planes travel as CUDA tensors on the
    current stream (the solver is attached to it); with any other backend
    through host arrays."""

    def __init__(self, nx: int, ny: int, ns: int, order: int = 2, limiter: bool = False,
                 dtype=np.float32, group=None, make_solver=None, **opts):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nx, self.ny, self.ns = nx, ny, ns
        self.dtype = np.dtype(dtype)
        self.halo = order + (order - 1 if limiter else 0)
        self.plan = SlabPlan(ns, self.world, self.halo)
        self.lo, self.hi = self.plan.own[self.rank]
        self.elo, self.ehi = self.plan.ext[self.rank]
        self.device = dist.get_backend(group) == "nccl"
        if make_solver is None:
            import mpdata_b200 as m
            self.local = m.Solver(nx, ny, self.ehi - self.elo, order=order, dtype=dtype,
                                  limiter=limiter, **opts)
            if self.device:
                import torch
                self.local.set_stream(torch.cuda.current_stream().cuda_stream)
        else:
            self.local = make_solver(nx, ny, self.ehi - self.elo)
        self._fresh = False  # halo planes hold the owners' current values

    # -- set-up (global arrays, every rank passes the same ones) --
    def set_faces(self, U, V, W):
        self.local.set_faces(*(np.ascontiguousarray(x[self.elo:self.ehi], self.dtype)
                               for x in (U, V, W)))

    def set_field(self, c):
        self.local.set_field(np.ascontiguousarray(c[self.elo:self.ehi], self.dtype))
        self._fresh = True

    # -- stepping --
    def _buffer(self, nk):
        shape = (nk, self.ny, self.nx)
        if self.device:
            import torch
            tdt = torch.float32 if self.dtype == np.float32 else torch.float64
            return torch.empty(shape, dtype=tdt, device="cuda")
        import torch
        return torch.from_numpy(np.empty(shape, self.dtype))

    def exchange(self):
        """Refresh the halo planes from their owners (one message per
        contiguous range and peer, in plane order)."""
        dist = self.dist
        recv = []
        reqs = []
        for peer, a, b in self.plan.recvs(self.rank):
            buf = self._buffer(b - a)
            reqs.append(dist.irecv(buf, src=peer, group=self.group))
            recv.append((a, buf))
        for peer, a, b in self.plan.sends(self.rank):
            buf = self._buffer(b - a)
            if self.device:
                self.local.get_planes(a - self.elo, b - a, out=buf)
            else:
                self.local.get_planes(a - self.elo, b - a, out=buf.numpy())
            reqs.append(dist.isend(buf, dst=peer, group=self.group))
        for rq in reqs:
            rq.wait()
        for a, buf in recv:
            self.local.set_planes(a - self.elo, buf if self.device else buf.numpy())
        self._fresh = True

    def step(self, nsteps: int = 1):
        for _ in range(nsteps):
            if not self._fresh:
                self.exchange()
            self.local.step(1)
            self._fresh = False

    # -- results --
    def owned(self) -> np.ndarray:
        """This rank's own planes [lo, hi) of the newest field (host array)."""
        return self.local.get_planes(self.lo - self.elo, self.hi - self.lo)

    def gather(self, root: int = 0):
        """The whole newest field on `root` (None elsewhere)."""
        import torch
        part = torch.from_numpy(np.ascontiguousarray(self.owned()))
        if self.device:
            part = part.cuda()
        sizes = [hi - lo for lo, hi in self.plan.own]
        full = None
        if self.rank == root:
            bufs = [torch.empty((n, self.ny, self.nx), dtype=part.dtype, device=part.device)
                    for n in sizes]
        reqs = []
        if self.rank == root:
            for r in range(self.world):
                if r == root:
                    bufs[r].copy_(part)
                else:
                    reqs.append(self.dist.irecv(bufs[r], src=r, group=self.group))
            for rq in reqs:
                rq.wait()
            full = torch.cat(bufs).cpu().numpy()
        else:
            self.dist.send(part, dst=root, group=self.group)
        return full

"""Sharding of a batch of independent systems over ranks.

The reference is single-process (README.md:327); its only parallelism is
shared-memory threading.  A batch of independent structures (the training set
of design_matrix, ACE/fitting.jl:18-67) shards without any data exchange:
every rank evaluates its own systems with one batched launch, and the
per-system results are gathered once at the end.

  system_costs   expected directed edges per system, n·(n/V)·(4/3)π c³
  shard          greedy longest-processing-time bin packing of the costs
  gather_rows    all_gather of per-system result rows (padded to the largest
                 shard) back into the original system order, on any
                 torch.distributed backend (NCCL on GPUs, gloo on CPUs)

One large periodic box decomposes into slabs instead (one exchange step):

  slab_domains      slabs along the axis with the largest face height; each
                    rank's subsystem is its owned atoms followed by ghost
                    copies (periodic images included) within `halo` of the
                    slab, with the slab axis open
  evaluate_domains  every rank evaluates its subsystem with pfw_set_owned, so
                    forces of owned atoms are exact (the halo covers their
                    neighbourhood: c for pairs, 2c for ACE, whose forces
                    gather site terms of neighbours) and energies and virials
                    count only owned shares; one all-reduce of E and W and
                    one all-gather of the owned forces assemble the result

With the positions resident on the devices, the per-step exchange runs
there too:

  SlabPlan          the decomposition's host plan (axis, band thickness,
                    owned atoms, image shifts)
  SlabRank          one rank's owned positions on its GPU; pfw_slab_bands
                    selects the atoms within the halo of its two faces, and
                    evaluate() assembles owned + ghosts on the device
  slab_step_dist    one step over torch.distributed: band sizes and bands
                    all-gathered, neighbours' bands taken as ghosts, energy
                    and virial all-reduced; forces stay with their owners
  slab_step_local   all ranks of a decomposition in turn on one GPU
"""
from __future__ import annotations

import heapq
import math

import numpy as np


def system_costs(systems, cutoff):
    """Expected directed neighbour count of each system (uniform density)."""
    ball = 4.0 / 3.0 * math.pi * cutoff ** 3
    out = np.zeros(len(systems))
    for k, s in enumerate(systems):
        n = len(s.species)
        V = abs(float(np.linalg.det(np.asarray(s.H, np.float64).reshape(3, 3))))
        out[k] = n * (n / V) * ball if V > 0 else n * n
    return out


def shard(costs, world):
    """Greedy LPT: systems in decreasing cost (ties by index) go to the least
    loaded rank (ties by rank).  Returns one sorted index list per rank."""
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(p) for p in parts]


def gather_rows(local_rows, parts, rank, group=None, device=None):
    """local_rows [len(parts[rank]), k] float64 → [nsys, k] on every rank."""
    import torch
    import torch.distributed as dist
    world = len(parts)
    k = local_rows.shape[1] if local_rows.ndim == 2 else 1
    width = max(len(p) for p in parts)
    buf = torch.zeros((width, k), dtype=torch.float64, device=device)
    if len(parts[rank]):
        buf[: len(parts[rank])] = torch.as_tensor(np.asarray(local_rows).reshape(len(parts[rank]), k), device=device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    nsys = sum(len(p) for p in parts)
    out = np.zeros((nsys, k))
    for r in range(world):
        rows = bufs[r].cpu().numpy()
        for i, s in enumerate(parts[r]):
            out[s] = rows[i]
    return out


class Domain:
    """One rank's subsystem: X, species (owned first), H, pbc, the owned
    atoms' original indices."""

    def __init__(self, X, species, H, pbc, owned):
        self.X, self.species, self.H, self.pbc, self.owned = X, species, H, pbc, owned

    @property
    def n_owned(self):
        return len(self.owned)


def slab_axis(H):
    """Cell axis with the largest distance between its opposite faces."""
    H = np.asarray(H, np.float64).reshape(3, 3)
    V = abs(np.linalg.det(H))
    heights = [V / np.linalg.norm(np.cross(H[:, (a + 1) % 3], H[:, (a + 2) % 3])) for a in range(3)]
    return int(np.argmax(heights)), heights


def slab_domains(system, world, halo):
    """Slab decomposition of a fully periodic system into `world` domains."""
    H = np.asarray(system.H, np.float64).reshape(3, 3)
    if not all(system.pbc):
        raise ValueError("slab decomposition needs a fully periodic box")
    a, heights = slab_axis(H)
    d = halo / heights[a]
    if d >= 1.0:
        raise ValueError("halo thicker than the box")
    f = np.linalg.solve(H, np.asarray(system.X, np.float64).T).T
    f -= np.floor(f)
    species = np.asarray(system.species, np.int32)
    pbc = [True, True, True]
    pbc[a] = False
    out = []
    for r in range(world):
        lo, hi = r / world, (r + 1) / world
        own = np.nonzero((f[:, a] >= lo) & (f[:, a] < hi))[0]
        ghosts_f, ghosts_z = [], []
        for k in (-1.0, 0.0, 1.0):
            g = f[:, a] + k
            sel = ((g >= lo - d) & (g < lo)) | ((g >= hi) & (g < hi + d))
            if np.any(sel):
                gf = f[sel].copy()
                gf[:, a] += k
                ghosts_f.append(gf)
                ghosts_z.append(species[sel])
        F = np.concatenate([f[own]] + ghosts_f) if ghosts_f else f[own]
        Z = np.concatenate([species[own]] + ghosts_z) if ghosts_z else species[own]
        out.append(Domain(np.ascontiguousarray(F @ H.T), np.ascontiguousarray(Z, np.int32), H, tuple(pbc), own))
    return out


def evaluate_domains(h, system, model, world, halo, request=7, rank=None, group=None, device=None):
    """Energy, forces (original order) and virial of `system` from its slab
    domains.  rank None: every domain in turn on this handle (one device);
    else this rank's domain, combined over `group` with one all-reduce of E
    and W and one all-gather of the owned forces."""
    doms = slab_domains(system, world, halo)
    n = len(system.species)
    mine = range(world) if rank is None else [rank]
    E, W = 0.0, np.zeros((3, 3))
    F = np.zeros((n, 3))
    rows = None
    for r in mine:
        dm = doms[r]
        h.set_geometry(dm.X, dm.H, dm.pbc, dm.species)
        h.set_owned(dm.n_owned)
        e, f, w = h.evaluate(model, request)
        E += e
        W += w
        if f is not None:
            F[dm.owned] = f[: dm.n_owned]
            rows = f[: dm.n_owned]
    if rank is None:
        return E, F, W
    import torch
    import torch.distributed as dist
    t = torch.tensor(np.concatenate([[E], W.ravel()]), dtype=torch.float64, device=device)
    dist.all_reduce(t, group=group)
    tot = t.cpu().numpy()
    parts = [list(map(int, dm.owned)) for dm in doms]
    full = gather_rows(rows if rows is not None else np.zeros((doms[rank].n_owned, 3)), parts, rank, group, device)
    return float(tot[0]), full, tot[1:].reshape(3, 3)


# ---------------------------------------------------------------------------
# slab decomposition with the per-step exchange on the devices
# ---------------------------------------------------------------------------
class SlabPlan:
    """Host plan of a slab decomposition of one fully periodic box over
    `world` ranks: the slab axis (largest face height), the row of H⁻¹ that
    gives the fractional coordinate along it, the band thickness d = halo /
    height (with a relative margin of 1e-9, so that rounding at a band edge
    can only add a ghost, never drop one), each rank's owned atoms (original
    indices, fractional coordinate in [r/world, (r+1)/world)) and the
    positions wrapped along the slab axis.  The halo must not exceed a
    slab's thickness: ghosts come from the two neighbouring slabs only."""

    def __init__(self, system, world, halo):
        H = np.asarray(system.H, np.float64).reshape(3, 3)
        if not all(system.pbc):
            raise ValueError("slab decomposition needs a fully periodic box")
        a, heights = slab_axis(H)
        self.axis, self.world, self.H = a, int(world), H
        self.d = halo / heights[a] * (1.0 + 1e-9)
        if self.d > 1.0 / world:
            raise ValueError("halo thicker than one slab: use fewer ranks or a larger box")
        self.frac_row = np.linalg.inv(H)[a].copy()
        X = np.asarray(system.X, np.float64)
        fa = np.linalg.solve(H, X.T).T[:, a]
        k = np.floor(fa)
        self.X = np.ascontiguousarray(X - np.outer(k, H[:, a]))
        fa = fa - k
        self.species = np.ascontiguousarray(system.species, np.int32)
        self.owned = [np.nonzero((fa >= r / world) & (fa < (r + 1) / world))[0] for r in range(world)]
        pbc = [True, True, True]
        pbc[a] = False
        self.pbc = tuple(pbc)
        self.n = len(self.species)

    def bounds(self, rank):
        return rank / self.world, (rank + 1) / self.world

    def shifts(self, rank):
        """Cartesian shifts of this rank's lower and upper bands: the lower
        band becomes rank-1's upper ghosts (+box vector when it wraps from
        rank 0), the upper band rank+1's lower ghosts (-box from the last)."""
        box = self.H[:, self.axis]
        lower = box if rank == 0 else np.zeros(3)
        upper = -box if rank == self.world - 1 else np.zeros(3)
        return lower, upper


class SlabRank:
    """One rank's slab, its owned positions resident on `device`.  bands()
    queues pfw_slab_bands (the atoms within d of the slab's faces, shifted
    for the receiving ranks); evaluate(ghosts_lower, ghosts_upper, ...)
    assembles [owned | lower ghosts | upper ghosts] on the device and runs
    pfw_set_owned + pfw_evaluate_device: owned forces in the first n_owned
    rows of F, energy and virial of the owned shares."""

    def __init__(self, h, plan, rank, device):
        import torch
        self.h, self.plan, self.rank, self.device = h, plan, rank, device
        own = plan.owned[rank]
        self.n_owned = len(own)
        self.X = torch.from_numpy(plan.X[own].copy()).to(device)
        self.Z = torch.from_numpy(plan.species[own].copy()).to(device)
        cap = max(self.n_owned, 1)
        self.lower = torch.zeros((cap, 4), dtype=torch.float64, device=device)
        self.upper = torch.zeros((cap, 4), dtype=torch.float64, device=device)
        self.counts = torch.zeros(2, dtype=torch.int32, device=device)

    def bands(self):
        import ctypes as C
        lo, hi = self.plan.bounds(self.rank)
        sl, su = self.plan.shifts(self.rank)
        self.h.slab_bands(self.n_owned, C.c_void_p(self.X.data_ptr()), C.c_void_p(self.Z.data_ptr()),
                          self.plan.frac_row, lo, hi, self.plan.d, sl, su, C.c_void_p(self.lower.data_ptr()),
                          C.c_void_p(self.upper.data_ptr()), C.c_void_p(self.counts.data_ptr()))
        return self.counts

    def evaluate(self, ghosts_lower, ghosts_upper, E, F, W, model, request=7):
        import ctypes as C

        import torch
        Xs = torch.cat([self.X, ghosts_lower[:, :3], ghosts_upper[:, :3]]).contiguous()
        Zs = torch.cat([self.Z, ghosts_lower[:, 3].to(torch.int32), ghosts_upper[:, 3].to(torch.int32)]).contiguous()
        n = Xs.shape[0]
        if F.shape[0] < n:
            raise ValueError("force buffer smaller than owned + ghost atoms")
        self._keep = (Xs, Zs)
        self.h.set_geometry_device(n, C.c_void_p(Xs.data_ptr()), self.plan.H, self.plan.pbc,
                                   C.c_void_p(Zs.data_ptr()))
        self.h.set_owned(self.n_owned)
        self.h.evaluate_device(model, request, C.c_void_p(E.data_ptr()), C.c_void_p(F.data_ptr()),
                               C.c_void_p(W.data_ptr()))


def slab_step_local(ranks, E, F, W, model, request=7):
    """Every rank of one slab decomposition evaluated in turn on one device
    (the exchange done by indexing): returns E, forces in the original order
    and W as numpy.  E, F, W are scratch device buffers (F sized for the
    largest subsystem)."""
    import torch
    plan = ranks[0].plan
    world = plan.world
    counts = [r.bands().cpu().numpy().copy() for r in ranks]
    Etot, Wtot = 0.0, np.zeros((3, 3))
    Fall = np.zeros((plan.n, 3))
    for r, rk in enumerate(ranks):
        below, above = ranks[(r - 1) % world], ranks[(r + 1) % world]
        gl = below.upper[: int(counts[(r - 1) % world][1])]
        gu = above.lower[: int(counts[(r + 1) % world][0])]
        rk.evaluate(gl, gu, E, F, W, model, request)
        torch.cuda.synchronize(rk.device)
        Etot += float(E.item())
        Wtot += W.cpu().numpy().reshape(3, 3, order="F")
        Fall[plan.owned[r]] = F[: rk.n_owned].cpu().numpy()
    return Etot, Fall, Wtot


def slab_step_dist(rank_obj, E, F, W, model, request=7, group=None):
    """One step of this rank's slab over torch.distributed (NCCL between
    GPUs, gloo on CPUs): the band sizes are all-gathered, then both bands
    (padded to the largest) are all-gathered, each rank takes its
    neighbours' bands as ghosts, evaluates, and the energy and virial are
    all-reduced (10 doubles).  Returns the reduced [E, W(9)] tensor; the
    owned forces stay in F[:n_owned] (the owner keeps them, as a molecular
    dynamics step would)."""
    import torch
    import torch.distributed as dist
    plan, r = rank_obj.plan, rank_obj.rank
    world = plan.world
    counts = rank_obj.bands()
    allc = [torch.zeros_like(counts) for _ in range(world)]
    dist.all_gather(allc, counts, group=group)
    allc = [c.cpu().numpy() for c in allc]
    width = max(1, max(int(max(c[0], c[1])) for c in allc))
    lower = rank_obj.lower[:width] if rank_obj.lower.shape[0] >= width else torch.nn.functional.pad(
        rank_obj.lower, (0, 0, 0, width - rank_obj.lower.shape[0]))
    upper = rank_obj.upper[:width] if rank_obj.upper.shape[0] >= width else torch.nn.functional.pad(
        rank_obj.upper, (0, 0, 0, width - rank_obj.upper.shape[0]))
    lowers = [torch.empty_like(lower) for _ in range(world)]
    uppers = [torch.empty_like(upper) for _ in range(world)]
    dist.all_gather(lowers, lower.contiguous(), group=group)
    dist.all_gather(uppers, upper.contiguous(), group=group)
    below, above = (r - 1) % world, (r + 1) % world
    gl = uppers[below][: int(allc[below][1])]
    gu = lowers[above][: int(allc[above][0])]
    rank_obj.evaluate(gl, gu, E, F, W, model, request)
    t = torch.cat([E.reshape(1), W.reshape(9)]).clone()
    dist.all_reduce(t, group=group)
    return t

"""Multi-rank paths on CPU (world sizes 2 and 3, gloo).  Batches: the LPT shards
cover every system once and balance the expected edge counts; each rank
evaluates its shard with the CPU oracle (standing in for the rank's GPU batch
launch) and the gathered per-system energies, virials and forces equal a
serial evaluation of the whole batch.  One box: each rank evaluates its slab
domain (owned atoms + 2c ghost halo) with the ACE oracle standing in for
pfw_set_owned + pfw_evaluate; the all-reduced energy and all-gathered forces
equal the serial evaluation.  The per-step exchange of the device-resident
slabs (parallel.slab_step_dist: band sizes and bands all-gathered,
neighbours' bands as ghosts, energy all-reduced) gives the same with the
bands selected by a numpy restatement of pfw_slab_bands."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pfw_b200 import parallel as PAR
from pfw_b200 import workloads as WL


def test_shard_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(3.0, 1.0, 500)
    parts = PAR.shard(costs, 4)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(500))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) - min(loads) <= costs.max()
    assert PAR.shard(costs, 4) == parts  # deterministic


def test_system_costs_scale():
    systems = WL.batched(seed=3, nsys=6, nmin=8, nmax=64)
    c = PAR.system_costs(systems, 5.5)
    for s, v in zip(systems, c):
        n = len(s.species)
        assert v == pytest.approx(n * n / abs(np.linalg.det(s.H)) * 4.0 / 3.0 * np.pi * 5.5 ** 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = WL.batched(seed=17, nsys=9, nmin=8, nmax=40, workers=1)
        parts = PAR.shard(PAR.system_costs(systems, 2.0), world)
        rows = []
        for k in parts[rank]:
            s = systems[k]
            e, f, w, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "smooth", WL.SMOOTH_A, 2.0)
            rows.append(np.concatenate([[e], w.ravel(order="F"), [np.abs(f).sum()]]))
        rows = np.array(rows).reshape(len(parts[rank]), 11)
        full = PAR.gather_rows(rows, parts, rank)
        if rank == 0:
            np.save(out_path, full)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_batch_matches_serial(tmp_path):
    from oracle import oracle as O
    out = str(tmp_path / "gathered.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    full = np.load(out)
    systems = WL.batched(seed=17, nsys=9, nmin=8, nmax=40, workers=1)
    for k, s in enumerate(systems):
        e, f, w, _ = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "smooth", WL.SMOOTH_A, 2.0)
        assert full[k, 0] == e
        assert np.array_equal(full[k, 1:10], w.ravel(order="F"))
        assert full[k, 10] == np.abs(f).sum()


class OracleDomainHandle:
    """The three handle calls evaluate_domains makes, answered by the ACE
    oracle: energy of the owned sites, forces of every atom, no virial."""

    def __init__(self, model):
        from oracle import oracle as O
        self.ace = O.AceOracle(model)
        self.n_owned = -1

    def set_geometry(self, X, H, pbc, species):
        self.geom = (X, H, pbc, species)
        self.n_owned = -1

    def set_owned(self, n):
        self.n_owned = n

    def evaluate(self, model, request):
        X, H, pbc, species = self.geom
        r = self.ace.evaluate(X, H, pbc, species, site_energies=True)
        k = len(species) if self.n_owned < 0 else self.n_owned
        return float(r["site_energies"][:k].sum()), r["forces"], np.zeros((3, 3))


def _tial():
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tial_ace.npz"))
    from pfw_b200.ace_model import PackedACE
    return PackedACE.from_npz_dict(d, "model_")


def _domain_main(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = _tial()
        s = WL.b2(seed=9, nc=6, a=2.95)
        E, F, W = PAR.evaluate_domains(OracleDomainHandle(m), s, 1, world, 2.0 * m.cutoff, rank=rank)
        if rank == 0:
            np.save(out_path, np.concatenate([[E], F.ravel()]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_slab_domains_match_serial(tmp_path):
    from oracle import oracle as O
    out = str(tmp_path / "dom.npy")
    mp.start_processes(_domain_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    m = _tial()
    s = WL.b2(seed=9, nc=6, a=2.95)
    r = O.AceOracle(m).evaluate(s.X, s.H, s.pbc, s.species)
    assert abs(got[0] - r["energy"]) <= 1e-9 * abs(r["energy"])
    assert np.allclose(got[1:].reshape(-1, 3), r["forces"], rtol=0, atol=1e-9 * np.abs(r["forces"]).max())


class CpuSlabRank:
    """Stands in for parallel.SlabRank on CPU tensors: bands() restates
    pfw_slab_bands in numpy, evaluate() answers with the ACE oracle (energy of
    the owned sites, forces of every atom, no virial)."""

    def __init__(self, plan, rank, model):
        import torch
        from oracle import oracle as O
        self.plan, self.rank, self.ace = plan, rank, O.AceOracle(model)
        own = plan.owned[rank]
        self.n_owned = len(own)
        self.X, self.Z = plan.X[own], plan.species[own]
        self.lower = torch.zeros((max(self.n_owned, 1), 4), dtype=torch.float64)
        self.upper = torch.zeros_like(self.lower)
        self.counts = torch.zeros(2, dtype=torch.int32)

    def bands(self):
        import torch
        f = self.X @ self.plan.frac_row
        lo, hi = self.plan.bounds(self.rank)
        sl, su = self.plan.shifts(self.rank)
        for k, (buf, sel, sh) in enumerate(((self.lower, f < lo + self.plan.d, sl),
                                            (self.upper, f >= hi - self.plan.d, su))):
            rows = np.concatenate([self.X[sel] + sh, self.Z[sel, None].astype(np.float64)], axis=1)
            buf[: len(rows)] = torch.from_numpy(rows)
            self.counts[k] = len(rows)
        return self.counts

    def evaluate(self, gl, gu, E, F, W, model, request=7):
        X = np.concatenate([self.X, gl[:, :3].numpy(), gu[:, :3].numpy()])
        Z = np.concatenate([self.Z, gl[:, 3].numpy().astype(np.int32), gu[:, 3].numpy().astype(np.int32)])
        r = self.ace.evaluate(X, self.plan.H, self.plan.pbc, Z, site_energies=True)
        E[0] = float(r["site_energies"][: self.n_owned].sum())
        F[: len(Z)] = __import__("torch").from_numpy(r["forces"])
        W.zero_()


def _exchange_main(rank, world, port, out_path, nc=10):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = _tial()
        s = WL.b2(seed=9, nc=nc, a=2.95)
        plan = PAR.SlabPlan(s, world, 2.0 * m.cutoff)
        rk = CpuSlabRank(plan, rank, m)
        E = torch.zeros(1, dtype=torch.float64)
        W = torch.zeros(9, dtype=torch.float64)
        F = torch.zeros((3 * len(s.species), 3), dtype=torch.float64)
        t = PAR.slab_step_dist(rk, E, F, W, 1)
        rows = F[: rk.n_owned].numpy()
        parts = [list(map(int, o)) for o in plan.owned]
        full = PAR.gather_rows(rows, parts, rank)
        if rank == 0:
            np.save(out_path, np.concatenate([t.numpy()[:1], full.ravel()]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nc", [(2, 10), (3, 14)])
def test_slab_exchange_matches_serial(tmp_path, world, nc):
    """With 2 ranks a rank's lower and upper neighbour are the same rank; with
    3 they are different ranks, and every band crosses to its own receiver."""
    from oracle import oracle as O
    out = str(tmp_path / "exch.npy")
    mp.start_processes(_exchange_main, args=(world, _free_port(), out, nc), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    m = _tial()
    s = WL.b2(seed=9, nc=nc, a=2.95)
    r = O.AceOracle(m).evaluate(s.X, s.H, s.pbc, s.species)
    assert abs(got[0] - r["energy"]) <= 1e-9 * abs(r["energy"])
    assert np.allclose(got[1:].reshape(-1, 3), r["forces"], rtol=0, atol=1e-9 * np.abs(r["forces"]).max())


def test_slab_plan_partition_and_shifts():
    s = WL.lj_fcc(seed=3, nc=6)
    s.X[:5] += 3.0 * s.H[:, 2]  # atoms outside the box along the slab axis wrap into it
    plan = PAR.SlabPlan(s, 3, WL.LJ_CUTOFF * 0.5)
    assert sorted(np.concatenate(plan.owned).tolist()) == list(range(len(s.species)))
    f = plan.X @ plan.frac_row
    assert np.all((f >= -1e-12) & (f < 1.0 + 1e-12))
    box = s.H[:, plan.axis]
    assert np.array_equal(plan.shifts(0)[0], box) and not plan.shifts(0)[1].any()
    assert np.array_equal(plan.shifts(2)[1], -box) and not plan.shifts(1)[0].any()
    with pytest.raises(ValueError):
        PAR.SlabPlan(s, 8, WL.LJ_CUTOFF)  # halo thicker than a slab

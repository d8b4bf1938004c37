"""Multi-rank paths on CPU (world size 2, gloo).  Batches: the LPT shards
cover every system once and balance the expected edge counts; each rank
evaluates its shard with the CPU oracle (standing in for the rank's GPU batch
launch) and the gathered per-system energies, virials and forces equal a
serial evaluation of the whole batch.  One box: each rank evaluates its slab
domain (owned atoms + 2c ghost halo) with the ACE oracle standing in for
pfw_set_owned + pfw_evaluate; the all-reduced energy and all-gathered forces
equal the serial evaluation."""
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

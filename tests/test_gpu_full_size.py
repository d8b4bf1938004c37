"""GPU parity against the oracle on the evaluation configurations at their
stated sizes (the small-case tests elsewhere cover the edge cases):

  * Lennard-Jones FCC 40³ (256,000 atoms), cubic and shear 0.2: FP64
    energy/forces/virial within 1e-10 relative, pair count equal, and the
    directed neighbour snapshot equal as a set of (i, j, S) with R bit for
    bit (NeighbourList/interface.jl:85-143; test/neighbour_interface.jl:21-49);
  * Lennard-Jones 4·64³ (1,048,576 atoms): energy/forces/virial, pair count;
  * ACE on B2 20³ (16,000 atoms) with the synthetic model (8 radials, lmax 4,
    order 3, degree 12): energy/forces/virial and site energies;
  * the 4096-system batch (log-uniform 8..256 atoms, random triclinic cells):
    every system's energy/forces/virial and fitting features, checked against
    the oracle on a seeded sample of 256 systems that includes the smallest
    and the largest;
  * the mixed-precision forms of the pair and ACE configurations against the
    FP64 oracle: force RMSE within 1e-3 eV/Å.

The oracle runs on all host threads; the sets are compared as sorted arrays.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import read_resolved

pytestmark = pytest.mark.gpu
RTOL = 1e-10
THREADS = max(1, min(os.cpu_count() or 1, 64))
LJ = (WL.LJ_EPS, WL.LJ_SIGMA)


def assert_close(E, F, W, Eo, Fo, Wo, rtol=RTOL, atol=1e-12):
    assert abs(E - Eo) <= rtol * max(1.0, abs(Eo)), (E, Eo)
    fs = max(1e-300, float(np.abs(Fo).max()))
    err = float(np.abs(F - Fo).max())
    assert err <= rtol * fs + atol, (err, fs)
    assert float(np.abs(W - Wo).max()) <= rtol * max(1.0, float(np.abs(Wo).max()))


def sorted_snapshot(offs, j, S, R):
    """Entries ordered by (i, j, S): the snapshot as a comparable set."""
    i = np.repeat(np.arange(len(offs) - 1, dtype=np.int64), np.diff(offs))
    order = np.lexsort((S[:, 2], S[:, 1], S[:, 0], j, i))
    return i[order], j[order], S[order], R[order]


@pytest.fixture(scope="module")
def h64():
    return lib.Handle(lib.FP64)


@pytest.fixture(scope="module")
def h32():
    return lib.Handle(lib.MIXED)


@pytest.mark.parametrize("shear", [0.0, 0.2])
def test_lj_256000_energy_forces_virial_and_snapshot(h64, shear):
    s = WL.lj_fcc(nc=40, shear=shear)
    h64.set_geometry(s.X, s.H, s.pbc, s.species)
    h64.lj(*LJ, WL.LJ_CUTOFF)
    E, F, W = h64.evaluate(lib.MODEL_PAIR, 7)
    Eo, Fo, Wo, npairs = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", LJ, WL.LJ_CUTOFF, nthreads=THREADS)
    assert_close(E, F, W, Eo, Fo, Wo)
    assert h64.pair_count() == npairs
    g = sorted_snapshot(*h64.neighbour_list(WL.LJ_CUTOFF))
    o = sorted_snapshot(*O.neighbour_list(s.X, s.H, s.pbc, WL.LJ_CUTOFF))
    assert len(g[0]) == len(o[0]) == 2 * npairs
    for a, b in zip(g, o):
        assert np.array_equal(a, b)


def test_lj_1048576_energy_forces_virial(h64):
    s = WL.lj_1m()
    h64.set_geometry(s.X, s.H, s.pbc, s.species)
    h64.lj(*LJ, WL.LJ_CUTOFF)
    E, F, W = h64.evaluate(lib.MODEL_PAIR, 7)
    Eo, Fo, Wo, npairs = O.pair_evaluate(s.X, s.H, s.pbc, s.species, "lj", LJ, WL.LJ_CUTOFF, nthreads=THREADS)
    assert_close(E, F, W, Eo, Fo, Wo)
    assert h64.pair_count() == npairs


@pytest.mark.parametrize("config", ["lj_256000", "lj_256000_shear", "smooth_2048"])
def test_mixed_pairs_against_fp64_oracle(h32, config):
    if config == "smooth_2048":
        s, kind, params, c = WL.smooth_fcc(), "smooth", WL.SMOOTH_A, WL.SMOOTH_CUTOFF
    else:
        s, kind, params, c = WL.lj_fcc(nc=40, shear=0.2 if "shear" in config else 0.0), "lj", LJ, WL.LJ_CUTOFF
    h32.set_geometry(s.X, s.H, s.pbc, s.species)
    if kind == "smooth":
        h32.smooth(params, c)
    else:
        h32.lj(*params, c)
    E, F, W = h32.evaluate(lib.MODEL_PAIR, 7)
    Eo, Fo, Wo, npairs = O.pair_evaluate(s.X, s.H, s.pbc, s.species, kind, params, c, nthreads=THREADS)
    rmse = float(np.sqrt(np.mean((F - Fo) ** 2)))
    assert rmse <= 1e-3, rmse
    assert h32.pair_count() == npairs  # the mixed form keeps the exact neighbour set
    assert abs(E - Eo) <= 1e-6 * max(1.0, abs(Eo))


@pytest.fixture(scope="module")
def b2model():
    return read_resolved(G.generate_b2_model())


@pytest.fixture(scope="module")
def b2_16000():
    return WL.b2()


def test_ace_b2_16000(h64, b2model, b2_16000):
    s = b2_16000
    h64.ace(b2model)
    h64.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h64.evaluate(lib.MODEL_ACE, 7)
    r = O.AceOracle(b2model).evaluate(s.X, s.H, s.pbc, s.species, site_energies=True, nthreads=THREADS)
    assert_close(E, F, W, r["energy"], r["forces"], r["virial"])
    es = h64.site_energies()
    assert float(np.abs(es - r["site_energies"]).max()) <= RTOL * max(1.0, float(np.abs(r["site_energies"]).max()))


def test_ace_b2_16000_mixed_against_fp64_oracle(h32, b2model, b2_16000):
    s = b2_16000
    h32.ace(b2model)
    h32.set_geometry(s.X, s.H, s.pbc, s.species)
    E, F, W = h32.evaluate(lib.MODEL_ACE, 7)
    r = O.AceOracle(b2model).evaluate(s.X, s.H, s.pbc, s.species, nthreads=THREADS)
    rmse = float(np.sqrt(np.mean((F - r["forces"]) ** 2)))
    assert rmse <= 1e-3, rmse
    assert abs(E - r["energy"]) <= 1e-5 * len(s)


def test_ace_batch_4096_against_oracle_sample(b2model):
    systems = WL.batched()
    assert len(systems) == 4096
    h = lib.Handle(lib.FP64)
    h.ace(b2model)
    h.set_batch(systems)
    E, F, W, X = h.evaluate_batch(lib.MODEL_ACE, 7, features=True)
    offs = h.batch_offsets
    sizes = np.array([len(sy) for sy in systems])
    rng = np.random.default_rng(4096)
    sample = set(rng.choice(len(systems), 254, replace=False).tolist())
    sample |= {int(np.argmin(sizes)), int(np.argmax(sizes))}
    ace = O.AceOracle(b2model)
    for s in sorted(sample):
        sy = systems[s]
        r = ace.evaluate(sy.X, sy.H, sy.pbc, sy.species, features=True)
        assert_close(E[s], F[offs[s]:offs[s + 1]], W[s], r["energy"], r["forces"], r["virial"])
        feat = r["features"].sum(axis=0)
        assert float(np.abs(X[s] - feat).max()) <= RTOL * max(1.0, float(np.abs(feat).max()))
    assert len(sample) >= 256

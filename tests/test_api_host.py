"""Host-side behaviour of the pfw_b200 API mirror that needs no GPU: the pair
models' parameter interface (PairPotentials/parameters.jl:34-54,
lennard_jones.jl:20-27) with the reference's error messages, the request
normalisation (NeighbourList/execution.jl:155-163), `neighbours` and the
in-place destinations' shape check."""
import re

import numpy as np
import pytest

from pfw_b200 import api
from pfw_b200.errors import ArgumentError, DimensionMismatch


def test_smooth_parameters_are_the_upper_triangle_in_column_order():
    A = np.array([[1.0, 0.7, 0.2], [0.7, 1.3, 0.4], [0.2, 0.4, 0.9]])
    p = api.SmoothPair(["H", "He", "Li"], A, 2.0)
    ps = api.get_parameters(p)
    assert set(ps) == {"amplitudes"}
    # j = 1..n, i = 1..j: A11, A12, A22, A13, A23, A33
    assert ps["amplitudes"].tolist() == [1.0, 0.7, 1.3, 0.2, 0.4, 0.9]
    q = api.set_parameters(p, {"amplitudes": ps["amplitudes"] * 2})
    assert q is not p and np.array_equal(q.amplitudes, 2 * A) and q.radius == 2.0 and q.labels == p.labels
    assert np.array_equal(p.amplitudes, A)  # the model is immutable
    assert np.array_equal(api.with_parameters(p, ps).amplitudes, A)


@pytest.mark.parametrize("ps,msg", [
    ({"amplitudes": [1.0, 2.0], "radius": 2.0}, "must contain only amplitudes"),
    ({"amplitudes": [1.0, 2.0]}, "length n*(n+1)/2"),
    ({"amplitudes": [1.0, np.inf, 2.0]}, "amplitudes must be finite"),
])
def test_smooth_parameter_errors_follow_the_reference(ps, msg):
    p = api.SmoothPair(["H", "He"], [[1.0, 0.7], [0.7, 1.3]], 2.0)
    with pytest.raises(ArgumentError, match=re.escape(msg)):
        api.with_parameters(p, ps)


def test_lennard_jones_parameters():
    p = api.lennard_jones(epsilon=0.0104, sigma=3.4, radius=8.5)
    assert api.get_parameters(p) == {"epsilon": 0.0104, "sigma": 3.4}
    q = api.set_parameters(p, {"epsilon": 0.02, "sigma": 3.0})
    assert (q.epsilon, q.sigma, q.radius) == (0.02, 3.0, 8.5) and p.epsilon == 0.0104
    with pytest.raises(ArgumentError, match="require epsilon and sigma; cutoff is fixed"):
        api.with_parameters(p, {"epsilon": 0.02})
    with pytest.raises(ArgumentError, match="positive and finite"):
        api.with_parameters(p, {"epsilon": -1.0, "sigma": 3.0})


def test_cutoff():
    assert api.cutoff(api.lennard_jones(radius=8.5)) == 8.5
    assert api.cutoff(api.SmoothPair(["H"], [[1.0]], 2.0)) == 2.0
    with pytest.raises(ArgumentError):
        api.cutoff(object())


def test_models_without_parameters_are_rejected():
    with pytest.raises(ArgumentError):
        api.get_parameters(object())
    with pytest.raises(ArgumentError):
        api.set_parameters(object(), {})


def test_smooth_constructor_checks():
    with pytest.raises(ArgumentError, match="size must match"):
        api.SmoothPair(["H"], [[1.0, 0.0], [0.0, 1.0]], 2.0)
    with pytest.raises(ArgumentError, match="unique"):
        api.SmoothPair(["H", "H"], [[1.0, 0.0], [0.0, 1.0]], 2.0)
    with pytest.raises(ArgumentError, match="finite and symmetric"):
        api.SmoothPair(["H", "He"], [[1.0, 0.5], [0.7, 1.0]], 2.0)
    with pytest.raises(ArgumentError, match="cutoff"):
        api.SmoothPair(["H"], [[1.0]], 0.0)


def test_request_normalisation():
    from pfw_b200 import lib
    assert api._request_bits(api.EnergyOnly()) == lib.REQ_E
    assert api._request_bits(api.EnergyForcesVirial) == 7
    assert api._request_bits((api.Forces(),)) == lib.REQ_F
    assert api._request_bits((api.Energy, api.Virial)) == lib.REQ_E | lib.REQ_V
    assert api._request_bits(("energy", "forces", "virial")) == 7
    with pytest.raises(ArgumentError):
        api._request_bits(("stress",))


def test_neighbours_returns_independent_arrays():
    offs = np.array([0, 2, 2, 3])
    snap = api.NeighbourSnapshot(offs, np.array([1, 2, 0], np.int32), np.zeros((3, 3), np.int32),
                                 np.arange(9.0).reshape(3, 3))
    assert len(snap) == 3 and snap.npairs() == 3
    js, Rs, Ss = api.neighbours(snap, 0)
    assert js.tolist() == [1, 2] and Rs.shape == (2, 3) and Ss.shape == (2, 3)
    js[0] = 99
    assert snap.j[0] == 1
    assert len(api.neighbours(snap, 1)[0]) == 0
    with pytest.raises(IndexError):
        api.neighbours(snap, 3)


def test_in_place_destinations_check_their_shape():
    F = np.zeros((4, 3))
    api._add_into(F, np.ones((4, 3)))
    assert F.sum() == 12
    with pytest.raises(DimensionMismatch):
        api._add_into(F, np.ones((3, 3)))


def test_device_tables_reject_products_above_order_4():
    import dataclasses

    from pfw_b200 import ace_generate as G
    from pfw_b200.ace_model import MAX_ORDER, read_resolved
    m = read_resolved(G.generate_b2_model())
    assert max(len(p) for p in m.products) <= MAX_ORDER
    m.tables()  # the shipped order-3 model packs
    long = dataclasses.replace(m, products=[list(p) for p in m.products])
    long.products[0] = [0, 1, 2, 3, 4]
    with pytest.raises(ArgumentError, match="correlation order above 4"):
        long.tables()
    empty = dataclasses.replace(m, products=[list(p) for p in m.products])
    empty.products[-1] = []
    with pytest.raises(ArgumentError, match="empty ACE product"):
        empty.tables()


def test_species_channels():
    # integer arrays are channel indices
    assert api.species_channels(np.array([1, 0, 1]), ["H", "He"]).tolist() == [1, 0, 1]
    # labels by equality (SmoothPair)
    assert api.species_channels(np.array(["He", "H"]), ["H", "He"]).tolist() == [1, 0]
    # ACE models are labelled by atomic number: element symbols map through it
    assert api.species_channels(["Ti", "Al", "Ti"], [22, 13]).tolist() == [0, 1, 0]
    assert api.species_channels(["V", "Al", "Ti"], [22, 13, 23]).tolist() == [2, 1, 0]
    with pytest.raises(ArgumentError, match="no parameters for species Fe"):
        api.species_channels(["Ti", "Fe"], [22, 13])
    with pytest.raises(ArgumentError, match="no parameters for species Li"):
        api.species_channels(["Li"], ["H", "He"])

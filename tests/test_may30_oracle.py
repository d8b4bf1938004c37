"""The May30 Ti–Al–V model (real solid harmonics through l = 6, 114 radial
channels on 1000 spline nodes, PolyEnvelope1sR pair channels, 5652 products)
on CPU: the oracle against the reference's cached ACEpotentials predictions
for bcc-128, hcp-150 and omega-240 at the reference's own tolerances
(test/ace_may30.jl:3-7: energy atol 2e-8 eV, forces atol 2e-9 eV/Å + rtol
2e-11, virial atol 2e-8 eV + rtol 2e-11); solid harmonics are r^l times the
spherical ones with the Cartesian product derivative (ace_may30.jl:21-29);
the PolyEnvelope1sR pair envelope (ace_may30.jl:38-51).  The packed model
tables are generated from the reference data by tests/golden/make_may30.py
(run by build()); without them the model tests skip."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200.ace_model import PackedACE

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL = os.path.join(HERE, "golden", "may30_model.npz")
needs_model = pytest.mark.skipif(not os.path.exists(MODEL), reason="May30 model tables not generated")


def agrees(r, fr, k):
    assert abs(r["energy"] - float(fr[f"f{k}_energy"])) <= 2e-8
    F = fr[f"f{k}_forces"]
    assert np.all(np.abs(r["forces"] - F) <= 2e-9 + 2e-11 * np.abs(F))
    W = fr[f"f{k}_virial"]
    assert np.all(np.abs(r["virial"] - W) <= 2e-8 + 2e-11 * np.abs(W))


@pytest.fixture(scope="module")
def may30():
    return PackedACE.from_npz_dict(np.load(MODEL), "model_"), np.load(os.path.join(HERE, "golden", "may30_frames.npz"))


@needs_model
def test_model_shape(may30):
    m, _ = may30
    assert m.atomic_numbers == [22, 13, 23] and m.angular_kind == 1 and m.lmax == 6
    assert (m.nbasis, m.pair.nchannels, m.nproducts, m.ndensity) == (2155, 10, 5652, 156)
    assert m.radial.nchannels == 114 and m.radial.nknots == 1000
    assert set(m.pair.envelope_kind.tolist()) == {3}


@needs_model
@pytest.mark.parametrize("k", [0, 1, 2])
def test_oracle_matches_reference_predictions(may30, k):
    m, fr = may30
    r = O.AceOracle(m).evaluate(fr[f"f{k}_X"], fr[f"f{k}_H"], (1, 1, 1), fr[f"f{k}_species"], nthreads=4)
    agrees(r, fr, k)


def test_solid_harmonics_are_scaled_spherical():
    for r in (0.3, 1.0, 2.7):
        d = r * np.array([0.3, -0.7, 0.9])
        Y, dY = O.angular_ed(6, d)
        Ys, dYs = O.angular_ed(6, d, solid=True)
        rr = np.linalg.norm(d)
        for l in range(7):
            for k in range(l * l, (l + 1) ** 2):
                g = l * rr ** (l - 2) * d if l > 0 else np.zeros(3)
                assert abs(Ys[k] - rr ** l * Y[k]) <= 2e-11 + 2e-12 * abs(rr ** l * Y[k])
                ref = rr ** l * dY[k] + g * Y[k]
                assert np.all(np.abs(dYs[k] - ref) <= 2e-11 + 2e-12 * np.abs(ref))


@needs_model
def test_poly_envelope_1sr_pair_channels(may30):
    m, _ = may30
    ace = O.AceOracle(m)
    nz = m.nz
    for iz in range(nz):
        for jz in range(nz):
            k = iz * nz + jz
            rc, p = m.pair.envelope[k, 0], int(m.pair.envelope[k, 1])
            for r in (1.2, 2.8, 5.99, rc - 1e-7, rc, rc + 1e-7):
                v, dv = ace.radial_ed(1, iz, jz, r)
                h = 1e-6
                vp, _ = ace.radial_ed(1, iz, jz, r + h)
                vm, _ = ace.radial_ed(1, iz, jz, r - h)
                if r < rc - 2 * h:
                    assert np.allclose(dv, (vp - vm) / (2 * h), rtol=1e-6, atol=1e-6)
                if r >= rc:
                    assert not v.any() and not dv.any()

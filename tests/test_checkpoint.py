"""ACECalculator checkpoints on CPU, restating the reference's
test/ace_persistence.jl: nested parameters and state keep their values,
element types and shapes; explicit parameters are saved without being
installed; failed saves leave an existing file intact; the file's content,
not its extension, identifies a checkpoint; version-1 checkpoints without a
basis policy load; schema and shape errors raise ArgumentError /
DimensionMismatch.  Energies of restored calculators are checked with the CPU
oracle, which applies the trainable radial scales at run time as the
reference does, against the device tables, which fold them into the splines
(FP64 bar: 1e-10 relative)."""
import os
import tomllib

import numpy as np
import pytest

from oracle import oracle as O
from pfw_b200 import ace_generate as G
from pfw_b200 import api
from pfw_b200 import checkpoint as CK
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import PackedACE, read_resolved
from pfw_b200.errors import ArgumentError, DimensionMismatch

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def tial():
    d = np.load(os.path.join(HERE, "golden", "tial_ace.npz"))
    return PackedACE.from_npz_dict(d, "model_"), d


@pytest.fixture(scope="module")
def b2():
    return read_resolved(G.generate_b2_model())


def tables_equal(a, b):
    x, y = a.to_npz_dict(), b.to_npz_dict()
    return x.keys() == y.keys() and all(np.array_equal(x[k], y[k]) for k in x)


def tree_equal(a, b):
    if isinstance(a, dict):
        return isinstance(b, dict) and list(a) == list(b) and all(tree_equal(a[k], b[k]) for k in a)
    if isinstance(a, tuple):
        return isinstance(b, tuple) and len(a) == len(b) and all(tree_equal(x, y) for x, y in zip(a, b))
    if isinstance(a, np.ndarray):
        return isinstance(b, np.ndarray) and a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b)
    if isinstance(a, np.generic):
        return type(a) is type(b) and a == b
    return a == b


def tuned(model, seed=0):
    """The reference test's tuning: WB·0.83, Wpair·1.12, radial scale[:,1,2]·0.91,
    pair scale[1,2,1] = 0 and [2,1,2] = 1.17 (Julia 1-based)."""
    tp = CK.trainable_parameters(model, model.default_parameters())
    tp["WB"] *= 0.83
    tp["Wpair"] *= 1.12
    tp["radial"]["scale"][:, 0, 1] *= 0.91
    tp["pair"]["scale"][0, 1, 0] = 0.0
    tp["pair"]["scale"][1, 0, 1] = 1.17
    return tp


STATE = {"epoch": np.int32(7), "rate": np.float32(0.002), "tag": "tuned",
         "extra": (None, True, np.zeros((0, 2), np.float32))}


def test_encode_decode_keeps_types_and_shapes():
    tree = {"a": np.arange(24, dtype=np.int16).reshape(2, 3, 4), "b": np.float32(1.5), "c": 3, "d": 2.5,
            "e": (None, "x", np.array([True, False])), "f": {}, "g": np.zeros((0, 3), np.uint8),
            "h": np.array([[1.0, 2.0], [3.0, 4.0]], np.float32)}
    back = CK.decode(CK.encode(tree))
    ref = dict(tree, b=np.float32(1.5), c=np.int64(3), d=np.float64(2.5), e=(None, "x", np.array([True, False])))
    assert tree_equal(back, ref)
    # arrays are stored column-major, as Julia's vec
    enc = CK.encode(np.array([[1, 2], [3, 4]], np.int32))
    assert enc["shape"] == [2, 2] and enc["values"] == [1, 3, 2, 4] and enc["eltype"] == "Int32"
    assert CK.encode(np.float32(0.25)) == {"kind": "scalar", "eltype": "Float32", "value": 0.25}


@pytest.mark.parametrize("bad", [np.array([1.0, np.nan]), float("inf"), {1: 2.0}, object(), np.array([1j]),
                                 {1.0, 2.0}])
def test_encode_rejects_unsupported_and_nonfinite(bad):
    with pytest.raises(ArgumentError):
        CK.encode({"x": bad})


def test_decode_errors():
    with pytest.raises(DimensionMismatch):
        CK.decode({"kind": "array", "eltype": "Float64", "shape": [2, 2], "values": [1.0, 2.0]})
    with pytest.raises(DimensionMismatch):
        CK.decode({"kind": "array", "eltype": "Float64", "shape": [-1], "values": []})
    with pytest.raises(ArgumentError):
        CK.decode({"kind": "array", "eltype": "Complex64", "shape": [1], "values": [1.0]})
    with pytest.raises(ArgumentError):
        CK.decode({"kind": "namedtuple", "names": ["a", "a"], "items": [{"kind": "nothing"}] * 2})
    with pytest.raises(ArgumentError):
        CK.decode({"kind": "pointer"})


def test_toml_writer_round_trips():
    tree = {"schema": "x", "n": 3, "flag": False, "neg0": -0.0, "tiny": 1e-300, "big": 5e20, "third": 1 / 3,
            "quoted key": 'a "b" \\ c\nd\teé\u0001', "empty": [], "nested": [[1, 2], [3]],
            "t": {"u": {"v": [1.5, 2.5]}, "w": {}},
            "items": [{"kind": "array", "shape": [2], "items": [{"k": 1}, {"k": 2, "sub": {"z": "q"}}]},
                      {"kind": "nothing"}]}
    back = tomllib.loads(CK.dumps(tree))
    assert back == tree
    assert str(back["neg0"]) == "-0.0"


def test_resolved_tables_regenerate_exactly(tial, b2):
    for m in (tial[0], b2):
        bare = PackedACE(**{k: getattr(m, k) for k in m.__dataclass_fields__ if k not in ("resolved", "_keep")})
        d = bare.resolved_dict()
        d["parameters"] = {"WB_shape": [m.nbasis, m.nz], "Wpair_shape": [m.pair.nchannels, m.nz],
                           "ordering": "vec(WB), vec(Wpair); Julia column-major",
                           "flat": list(np.concatenate([m.WB.T.ravel(order="F"), m.Wpair.T.ravel(order="F")]))}
        again = read_resolved(tomllib.loads(CK.dumps(d)))
        assert tables_equal(m, again)


@pytest.mark.parametrize("which", ["tial", "b2"])
def test_save_and_restore(tmp_path, tial, b2, which):
    model = tial[0] if which == "tial" else b2
    original = api.ACECalculator(model)
    before = original.get_parameters()
    trained = tuned(model)
    path = str(tmp_path / "trained.toml")
    assert api.save_calculator(path, original, trained, STATE) == path
    assert tree_equal(original.parameters, before)  # an explicit override does not install parameters
    assert original.state == {}
    saved = tomllib.loads(open(path).read())
    assert set(saved) == {"schema", "schema_version", "writer", "model", "parameters", "state"}
    assert "parameters" not in saved["model"]
    relocated = tmp_path / "moved" / "checkpoint.ace"
    relocated.parent.mkdir()
    os.replace(path, relocated)
    restored = api.ACECalculator(str(relocated), width=8, slots=1)
    assert tree_equal(restored.parameters, trained)
    assert tree_equal(restored.state, STATE)
    assert restored.parameters["WB"] is not trained["WB"]
    assert restored.model.source_sha256 == model.source_sha256
    assert np.array_equal(restored.model.coupling_vals, model.coupling_vals)
    assert restored.model.products == model.products


def test_scales_folded_match_runtime_scales(tmp_path, tial):
    model, d = tial
    trained = tuned(model)
    path = str(tmp_path / "c.toml")
    api.save_calculator(path, api.ACECalculator(model), trained)
    dev = api.ACECalculator(path).device_model()
    runtime = O.AceOracle(model.with_parameters({"WB": trained["WB"], "Wpair": trained["Wpair"]}),
                          trained["radial"]["scale"], trained["pair"]["scale"])
    folded = O.AceOracle(dev)
    plain = O.AceOracle(model)
    for k in (0, 7):
        X, H, z = d[f"f{k}_X"], d[f"f{k}_H"], d[f"f{k}_species"]
        a = runtime.evaluate(X, H, (1, 1, 1), z)
        b = folded.evaluate(X, H, (1, 1, 1), z)
        c = plain.evaluate(X, H, (1, 1, 1), z)
        assert abs(a["energy"] - c["energy"]) > 1e-3  # the tuning changes the energy
        assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(a["energy"])
        assert np.allclose(a["forces"], b["forces"], rtol=0, atol=1e-10 * np.abs(a["forces"]).max())
        assert np.allclose(a["virial"], b["virial"], rtol=0, atol=1e-10 * np.abs(a["virial"]).max())


def test_set_parameters_and_resave(tmp_path, b2):
    c = api.ACECalculator(b2)
    trained = tuned(b2)
    c.set_parameters(dict(trained, WB=trained["WB"] * 0.7))
    path = str(tmp_path / "c.toml")
    api.save_calculator(path, c)
    twice = api.ACECalculator(path)
    assert tree_equal(twice.parameters, c.get_parameters())
    assert tables_equal(twice.device_model(), c.device_model())
    with pytest.raises(DimensionMismatch):
        c.set_parameters({"WB": np.zeros((1, 1)), "Wpair": trained["Wpair"]})


def test_float32_parameters_keep_type(tmp_path, b2):
    t = tuned(b2)
    ps32 = {"WB": t["WB"].astype(np.float32), "Wpair": t["Wpair"].astype(np.float32),
            "radial": {"scale": t["radial"]["scale"].astype(np.float32)},
            "pair": {"scale": t["pair"]["scale"].astype(np.float32)}}
    path = str(tmp_path / "c32.toml")
    api.save_calculator(path, api.ACECalculator(b2), ps32)
    assert tree_equal(api.ACECalculator(path).parameters, ps32)


def test_failed_saves_preserve_existing_file(tmp_path, b2):
    original = api.ACECalculator(b2)
    trained = tuned(b2)
    path = str(tmp_path / "c.toml")
    api.save_calculator(path, original, trained)
    intact = open(path, "rb").read()

    class Ref:
        pass

    for ps, st, err in ((dict(trained, WB=np.full_like(trained["WB"], np.nan)), {}, ArgumentError),
                        (trained, {"bad": Ref()}, ArgumentError),
                        (dict(trained, radial={"scale": np.ones((2, 2))}), {}, DimensionMismatch),
                        ({"WB": np.zeros((1, 1)), "Wpair": trained["Wpair"]}, {}, DimensionMismatch)):
        with pytest.raises(err):
            api.save_calculator(path, original, ps, st)
        assert open(path, "rb").read() == intact
    assert sorted(os.listdir(tmp_path)) == ["c.toml"]  # no temporary file left behind


def test_content_decides_and_legacy_and_errors(tmp_path, b2):
    original = api.ACECalculator(b2)
    jsonpath = str(tmp_path / "checkpoint.json")
    api.save_calculator(jsonpath, original)
    assert tree_equal(api.ACECalculator(jsonpath).parameters, original.parameters)
    saved = tomllib.loads(open(jsonpath).read())
    legacy = dict(saved, schema_version=1)
    legacy["model"] = {k: v for k, v in saved["model"].items() if k != "interface_policy"}
    lp = tmp_path / "legacy.toml"
    lp.write_text(CK.dumps(legacy))
    assert tree_equal(api.ACECalculator(str(lp)).parameters, original.parameters)
    bad = tmp_path / "bad.toml"
    bad.write_text(CK.dumps(dict(saved, schema_version=999)))
    with pytest.raises(ArgumentError):
        api.ACECalculator(str(bad))
    saved["parameters"]["items"][0]["shape"] = [1, 1]
    bad.write_text(CK.dumps(dict(saved, schema_version=1)))
    with pytest.raises(DimensionMismatch):
        api.ACECalculator(str(bad))
    (tmp_path / "recipe.json").write_text('{"model": 1}')
    with pytest.raises(ArgumentError):
        api.ACECalculator(str(tmp_path / "recipe.json"))


def default_policy(m, **kw):
    """checkpoint_policy of default_policy (interface.jl:14-18,
    interface_persistence.jl:1-7) with optional overrides."""
    p = {"version": 1, "origin": "ab" * 32, "rows": list(range(1, m.nbasis + 1)),
         "products": list(range(1, m.nproducts + 1)), "density": list(range(1, m.ndensity + 1)),
         "radial": list(range(1, m.radial.nchannels + 1)), "mask": [True] * m.nbasis, "species": [],
         "orders": [], "pair": True, "reference": True}
    p.update(kw)
    return p


def test_reference_written_checkpoint_with_policy_loads(tmp_path, tial):
    """A checkpoint as the reference writes it: the model tree carries the
    default interface_policy and the writer_julia key."""
    m, d = tial
    tree = m.resolved_dict()
    tree["interface_policy"] = default_policy(m)
    ck = {"schema": CK.CHECKPOINT_SCHEMA, "schema_version": 2, "writer_julia": "1.13.2", "model": tree,
          "parameters": CK.encode(m.default_parameters()), "state": CK.encode({})}
    path = tmp_path / "julia.toml"
    path.write_text(CK.dumps(ck))
    c = api.ACECalculator(str(path))
    assert tables_equal(c.device_model(), m)


def test_policy_mask_pair_and_reference(tial):
    m, d = tial
    rng = np.random.default_rng(5)
    mask = rng.random(m.nbasis) < 0.6
    tree = m.resolved_dict()
    tree["interface_policy"] = default_policy(m, mask=[bool(v) for v in mask], pair=False, reference=False)
    tree["parameters"] = {"WB_shape": [m.nbasis, m.nz], "Wpair_shape": [m.pair.nchannels, m.nz],
                          "ordering": "vec(WB), vec(Wpair); Julia column-major",
                          "flat": list(np.concatenate([m.WB.T.ravel(order="F"), m.Wpair.T.ravel(order="F")]))}
    pm = read_resolved(tree)
    assert np.all(mask[pm.coupling_rows]) and not np.any(pm.pair_allowed) and not np.any(pm.reference)
    # the same numbers by hand: masked readout rows, no pair term, no reference energies
    hand = PackedACE(**{k: getattr(m, k) for k in m.__dataclass_fields__ if k != "_keep"})
    hand.WB = np.ascontiguousarray(m.WB * mask[None, :])
    hand.Wpair = np.zeros_like(m.Wpair)
    hand.reference = np.zeros_like(m.reference)
    X, H, z = d["f3_X"], d["f3_H"], d["f3_species"]
    a = O.AceOracle(pm).evaluate(X, H, (1, 1, 1), z)
    b = O.AceOracle(hand).evaluate(X, H, (1, 1, 1), z)
    assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(b["energy"])
    assert np.allclose(a["forces"], b["forces"], rtol=0, atol=1e-10 * np.abs(b["forces"]).max())
    for bad in (dict(species=[1], orders=[0, 2]), dict(origin="short"), dict(version=2), dict(mask=[1] * m.nbasis)):
        tree["interface_policy"] = default_policy(m, **bad)
        with pytest.raises(ArgumentError):
            read_resolved(tree)


def test_calculate_parameters_route_through_with_parameters(b2):
    c = api.ACECalculator(b2, state={"k": 1})
    t = tuned(b2)
    c2 = api.with_parameters(c, t)
    assert isinstance(c2, api.ACECalculator) and c2.state == {"k": 1}
    assert tree_equal(c.parameters, b2.default_parameters())
    s = WL.b2(seed=1, nc=2)
    r = api.calculate((), s, c)
    assert r == {"state": {"k": 1}}

"""The library's own launch counter (pfw_launch_count, the figure the
benchmark reports as its kernel launches) equals the number of library
kernels the CUDA profiler sees execute: eager pair evaluations, replays of
the captured pair graph, skin-list reuse, ACE evaluations and a replayed
batch graph."""
import numpy as np
import pytest

from pfw_b200 import ace_generate as G
from pfw_b200 import lib
from pfw_b200 import workloads as WL
from pfw_b200.ace_model import read_resolved

pytestmark = pytest.mark.gpu


def counted(h, body):
    """(library kernels the profiler saw execute, counter delta) over body()."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        l0 = h.launches
        body()
        torch.cuda.synchronize()
        delta = h.launches - l0
    seen = sum(1 for e in prof.events() if e.device_type.name == "CUDA" and "pfw::" in e.name)
    return seen, delta


def test_pair_eager_graph_and_skin_counts():
    s = WL.lj_fcc(seed=1, nc=8)
    h = lib.Handle(lib.FP64)
    h.lj(0.0104, 3.4, 8.5)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    seen, delta = counted(h, lambda: h.evaluate(lib.MODEL_PAIR, 7))  # eager, then capture
    assert seen == delta > 0
    seen, delta = counted(h, lambda: [h.evaluate(lib.MODEL_PAIR, 7) for _ in range(3)])  # graph replays
    assert seen == delta > 0
    h.pair_skin(1.0)
    seen, delta = counted(h, lambda: [h.evaluate(lib.MODEL_PAIR, 7) for _ in range(3)])  # build + reuse
    assert seen == delta > 0


def test_ace_and_batch_graph_counts():
    import torch
    m = read_resolved(G.generate_b2_model())
    s = WL.b2(seed=2, nc=4)
    h = lib.Handle(lib.FP64)
    h.ace(m)
    h.set_geometry(s.X, s.H, s.pbc, s.species)
    seen, delta = counted(h, lambda: h.evaluate(lib.MODEL_ACE, 7))
    assert seen == delta > 0
    systems = WL.batched(seed=5, nsys=6, nmin=8, nmax=40, workers=1)
    h.set_batch(systems)
    dev = torch.device("cuda", 0)
    E = torch.zeros(h.nsys, dtype=torch.float64, device=dev)
    F = torch.zeros(h.n * 3, dtype=torch.float64, device=dev)
    W = torch.zeros(h.nsys * 9, dtype=torch.float64, device=dev)

    def replay():
        for _ in range(2):
            h.batch_graph_launch(7, E.data_ptr(), F.data_ptr(), W.data_ptr(), None)
            h.batch_graph_sync()
    seen, delta = counted(h, replay)
    assert seen == delta > 0

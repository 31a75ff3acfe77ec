"""sgs_batch.graph_capture (CPU, with torch.cuda.graph replaced by a recording stand-in): the cyclic
garbage collector runs before the capture, is off inside it, and is restored afterwards, also when
the capture raises; a collector that was off stays off."""
import contextlib
import gc

import pytest
import torch

import sgs_batch


class _Cycle:
    def __init__(self, log):
        self.me = self
        self.log = log

    def __del__(self):
        self.log.append("finalised")


@pytest.fixture
def fake_graph(monkeypatch):
    log = []

    @contextlib.contextmanager
    def fake(graph, **kwargs):
        log.append(("begin", gc.isenabled(), kwargs))
        yield
        log.append(("end", gc.isenabled()))

    monkeypatch.setattr(torch.cuda, "graph", fake)
    return log


def test_collects_before_and_disables_during(fake_graph):
    was = gc.isenabled()
    gc.enable()
    try:
        _Cycle(fake_graph)  # garbage only the cyclic collector can free
        with sgs_batch.graph_capture(object(), pool=None):
            fake_graph.append(("inside", gc.isenabled()))
        assert fake_graph[0] == "finalised"
        assert fake_graph[1] == ("begin", False, {"pool": None})
        assert fake_graph[2] == ("inside", False)
        assert fake_graph[3] == ("end", False)
        assert gc.isenabled()
    finally:
        if not was:
            gc.disable()


def test_restores_the_collector_when_the_capture_raises(fake_graph):
    was = gc.isenabled()
    gc.enable()
    try:
        with pytest.raises(RuntimeError, match="capture failed"):
            with sgs_batch.graph_capture(object()):
                raise RuntimeError("capture failed")
        assert gc.isenabled()
    finally:
        if not was:
            gc.disable()


def test_a_disabled_collector_stays_disabled(fake_graph):
    was = gc.isenabled()
    gc.disable()
    try:
        with sgs_batch.graph_capture(object()):
            pass
        assert not gc.isenabled()
    finally:
        if was:
            gc.enable()

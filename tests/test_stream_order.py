"""Host logic of the Python layer's stream ordering (no GPU): device-pointer calls run on the library's
non-blocking streams, so the wrapper makes the library stream wait for torch's current stream before the
call and torch's stream wait for the library stream after it.  A stand-in torch module records the waits."""
import sys
import types

import pytest

import giem2g_b200 as g2


class _Stream:
    def __init__(self, name, log):
        self.name, self.log = name, log

    def wait_stream(self, other):
        self.log.append((self.name, "waits for", other.name))


def _fake_torch(log, initialized=True, current_ptr=1):
    cur = _Stream("torch", log)
    cur.cuda_stream = current_ptr
    cuda = types.SimpleNamespace(is_initialized=lambda: initialized, current_stream=lambda: cur,
                                 ExternalStream=lambda ptr: _Stream(f"lib:{ptr}", log))
    return types.SimpleNamespace(cuda=cuda)


def test_waits_both_ways(monkeypatch):
    log = []
    monkeypatch.setitem(sys.modules, "torch", _fake_torch(log))
    with g2._torch_ordered(0x1234):
        log.append("call")
    assert log == [("lib:4660", "waits for", "torch"), "call", ("torch", "waits for", "lib:4660")]


def test_exit_wait_after_a_failed_call(monkeypatch):
    log = []
    monkeypatch.setitem(sys.modules, "torch", _fake_torch(log))
    with pytest.raises(g2.Giem2gError):
        with g2._torch_ordered(7):
            raise g2.Giem2gError("status -1")
    assert log == [("lib:7", "waits for", "torch"), ("torch", "waits for", "lib:7")]


def test_nothing_without_cuda_set_up(monkeypatch):
    log = []
    monkeypatch.setitem(sys.modules, "torch", _fake_torch(log, initialized=False))
    with g2._torch_ordered(7):
        log.append("call")
    assert log == ["call"]


def test_nothing_when_torch_runs_on_the_library_stream(monkeypatch):
    log = []
    monkeypatch.setitem(sys.modules, "torch", _fake_torch(log, current_ptr=7))
    with g2._torch_ordered(7):
        log.append("call")
    assert log == ["call"]


def test_nothing_without_torch(monkeypatch):
    monkeypatch.delitem(sys.modules, "torch", raising=False)
    with g2._torch_ordered(7):
        pass

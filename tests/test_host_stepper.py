"""HostStepper (solver/stream.py) on CPU with a fake step plan and stand-ins
for the CUDA stream and event calls (no GPU): every input reaches its own
output through the step, for any pipeline depth and count, and each step
reads and writes one buffer pair that the stream waits protect (the copy into
an input buffer waits for the step that last read it; the step waits for
its input's copy and for the copy-out of the output buffer it overwrites)."""
import contextlib
from types import SimpleNamespace

import pytest
import torch

from famrdp_jax_b200.solver import stream as S


class _Log:
    def __init__(self):
        self.ops = []
        self.cur = None


LOG = _Log()


class _Stream:
    def __init__(self, *a, **k):
        self.name = f"s{len([o for o in LOG.ops if o[0] == 'new'])}"
        LOG.ops.append(("new", self.name))

    def wait_stream(self, other):
        pass

    def wait_event(self, ev):
        LOG.ops.append(("wait", self.name, ev.id))


class _Event:
    count = 0

    def __init__(self, *a, **k):
        _Event.count += 1
        self.id = _Event.count

    def record(self, stream=None):
        LOG.ops.append(("record", stream.name, self.id))


@contextlib.contextmanager
def _use(s):
    prev, LOG.cur = LOG.cur, s
    try:
        yield
    finally:
        LOG.cur = prev


class _Plan:
    shapes = [(5, 2, 3, 2), (5, 3, 2, 2)]
    device = torch.device("cpu")

    def __init__(self):
        self.calls = []

    def run(self, qs, outs, dt, graph=True):
        self.calls.append((tuple(id(q) for q in qs), tuple(id(o) for o in outs)))
        for q, o in zip(qs, outs):
            o.copy_(2 * q + dt)


@pytest.fixture
def fake_streams(monkeypatch):
    LOG.ops.clear()
    monkeypatch.setattr(torch.cuda, "Stream", _Stream)
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda device=None: SimpleNamespace(
        wait_stream=lambda s: None, name="caller"))
    monkeypatch.setattr(torch.cuda, "stream", _use)


@pytest.mark.parametrize("depth", [1, 2, 3])
@pytest.mark.parametrize("count", [1, 2, 5])
def test_every_input_reaches_its_output(fake_streams, depth, count):
    plan = _Plan()
    hs = S.HostStepper(plan, depth=depth)
    rng = torch.Generator().manual_seed(count)
    ins = [[torch.rand(s, generator=rng, dtype=torch.float64) for s in plan.shapes] for _ in range(count)]
    outs = [[torch.empty(s, dtype=torch.float64) for s in plan.shapes] for _ in range(count)]
    hs.run(ins, outs, 0.25)
    for i, o in zip(ins, outs):
        for a, b in zip(i, o):
            assert torch.equal(b, 2 * a + 0.25)
    # step i runs on buffer pair i mod depth
    for i, (qi, qo) in enumerate(plan.calls):
        k = i % depth
        assert qi == tuple(id(t) for t in hs.din[k]) and qo == tuple(id(t) for t in hs.dout[k])


def test_waits_guard_buffer_reuse(fake_streams):
    plan = _Plan()
    hs = S.HostStepper(plan, depth=2)
    ins = [[torch.zeros(s, dtype=torch.float64) for s in plan.shapes] for _ in range(4)]
    outs = [[torch.empty(s, dtype=torch.float64) for s in plan.shapes] for _ in range(4)]
    hs.run(ins, outs, 0.0)
    h2d, comp, d2h = hs.h2d.name, hs.comp.name, hs.d2h.name
    waits = [(o[1], o[2]) for o in LOG.ops if o[0] == "wait"]
    records = [(o[1], o[2]) for o in LOG.ops if o[0] == "record"]
    for k in range(2):
        assert (h2d, hs.in_free[k].id) in waits       # the copy in waits for the step that read din[k]
        assert (comp, hs.in_ready[k].id) in waits     # the step waits for its input
        assert (comp, hs.out_free[k].id) in waits     # and for dout[k]'s previous copy out
        assert (d2h, hs.out_ready[k].id) in waits     # the copy out waits for the step
        assert (comp, hs.in_free[k].id) in records and (comp, hs.out_ready[k].id) in records
        assert (h2d, hs.in_ready[k].id) in records and (d2h, hs.out_free[k].id) in records


def test_depth_must_be_positive(fake_streams):
    with pytest.raises(ValueError):
        S.HostStepper(_Plan(), depth=0)
    hs = S.HostStepper(_Plan(), depth=1)
    with pytest.raises(ValueError):
        hs.run([[torch.zeros(1)]], [], 0.0)

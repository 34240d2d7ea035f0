"""The checkpointed adjoint's schedule (solver/adjoint.py) on CPU, with a
fake step plan, a fake step VJP and stand-ins for the CUDA stream calls (no
GPU): every step's VJP runs exactly once, in reverse step order, on the
states kept for that step; the reverse sweep recomputes only the segments
before the last two (second saved-state pool) or before the last one
(without it: overlap=False, or no room for the pool)."""
import contextlib

import pytest
import torch

from famrdp_jax_b200.solver import adjoint as A


class _Plan:
    """States are constant tensors holding the step count: a step adds 1, and
    run_save keeps (q, q + 1/4, q + 1/2) as (start state, stage 1, stage 2)."""
    mu0s = None
    dts = None

    def __init__(self):
        self.saves = []  # the step index of every run_save, in call order

    def run(self, qs, outs, dt, graph=False):
        for q, o in zip(qs, outs):
            o.copy_(q + 1)

    def run_save(self, qs, outs, q0s, q1s, q2s, dt):
        self.saves.append(int(qs[0].flatten()[0]))
        for q, o, a, b, c in zip(qs, outs, q0s, q1s, q2s):
            a.copy_(q)
            b.copy_(q + 0.25)
            c.copy_(q + 0.5)
            o.copy_(q + 1)


class _Stream:
    def __init__(self, *a, **k):
        pass

    def wait_stream(self, other):
        pass

    def wait_event(self, ev):
        pass


class _Event:
    def record(self, stream=None):
        pass


@pytest.fixture
def fake_cuda(monkeypatch):
    monkeypatch.setattr(torch.cuda, "Stream", _Stream)
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda device=None: _Stream())
    monkeypatch.setattr(torch.cuda, "stream", lambda s: contextlib.nullcontext())
    visits = []

    def step_vjp_saved(saved, metrics, cfg, dt, lams, *, tables=None, dmu=None, mu0s=None, dts=None, out=None):
        q0s, q1s, q2s = saved
        n = int(q0s[0].flatten()[0])
        for a, b, c in zip(q0s, q1s, q2s):
            assert torch.all(a == n) and torch.all(b == n + 0.25) and torch.all(c == n + 0.5)
        visits.append(n)
        for o, l in zip(out, lams):
            o.copy_(l + 1)
        return out

    monkeypatch.setattr(A, "step_vjp_saved", step_vjp_saved)
    return visits


def _run(nsteps, every, overlap):
    return A._Run(cfg=None, metrics=None, dt=0.1, nsteps=nsteps, every=every, plan=_Plan(), tables=None,
                  overlap=overlap)


@pytest.mark.parametrize("nsteps,every", [(23, 5), (20, 5), (4, 10), (10, 10), (11, 10), (7, 1)])
@pytest.mark.parametrize("overlap", [True, False])
def test_every_step_adjoint_once_in_reverse_order(fake_cuda, nsteps, every, overlap):
    run = _run(nsteps, every, overlap)
    q0 = [torch.zeros(2, 3, dtype=torch.float64), torch.zeros(4, dtype=torch.float64)]
    final, checkpoints = A._forward_with_checkpoints(run, q0)
    nseg = -(-nsteps // every)
    assert len(checkpoints) == nseg
    assert all(torch.all(c[0] == s * every) for s, c in enumerate(checkpoints))
    assert all(torch.all(f == nsteps) for f in final)
    seg_of = lambda n: n // every  # noqa: E731
    kept = {seg_of(n) for n in run.plan.saves}
    assert kept == ({nseg - 1, nseg - 2} if overlap and nseg >= 2 else {nseg - 1})
    run.plan.saves.clear()
    lams = A._reverse_sweep(run, checkpoints, [torch.zeros_like(q) for q in q0])
    assert fake_cuda == list(range(nsteps - 1, -1, -1))
    assert all(torch.all(l == nsteps) for l in lams)
    recomputed = {seg_of(n) for n in run.plan.saves}
    assert recomputed == set(range(nseg - 2 if overlap else nseg - 1))
    assert len(run.plan.saves) == sum(min(every, nsteps - s * every) for s in recomputed)


def test_no_room_for_the_second_pool_falls_back_to_one(fake_cuda, monkeypatch):
    def no_room(*a, **k):
        raise torch.cuda.OutOfMemoryError("no room")

    monkeypatch.setattr(torch.cuda, "Stream", no_room)
    run = _run(23, 5, True)
    q0 = [torch.zeros(3, dtype=torch.float64)]
    final, checkpoints = A._forward_with_checkpoints(run, q0)
    assert run.overlap is False and run._saved2 is None
    run.plan.saves.clear()
    lams = A._reverse_sweep(run, checkpoints, [torch.zeros(3, dtype=torch.float64)])
    assert fake_cuda == list(range(22, -1, -1))
    assert {n // 5 for n in run.plan.saves} == {0, 1, 2, 3}
    assert torch.all(lams[0] == 23)

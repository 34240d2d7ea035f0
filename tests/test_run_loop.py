"""The monitored time loop (solver/run.py) on CPU, with a fake step plan and
fake state checks (no GPU): the residual log's rows and file format, and the
NaN guard's step number, message and dumped states."""
from types import SimpleNamespace

import pytest
import torch

from famrdp_jax_b200.core.types import Block, State
from famrdp_jax_b200.solver import run as R


class _Plan:
    """A step adds 1 to every value; step `bad` (1-based) writes a NaN."""

    def __init__(self, bad=None):
        self.bad, self.n = bad, 0

    def run(self, a, b, dt, graph=True):
        self.n += 1
        for x, y in zip(a, b):
            y.copy_(x + 1)
            if self.n == self.bad:
                y.view(-1)[0] = float("nan")


@pytest.fixture
def fakes(monkeypatch):
    def residual(cur, prev, dt, ghost):
        return [float(cur.blocks[0].q.view(-1)[-1])] * 5

    def check_state(cur, gamma, raise_on_error=True):
        nonfinite = sum(int((~torch.isfinite(b.q)).sum()) for b in cur.blocks)
        return nonfinite, 1.0, 1.0

    monkeypatch.setattr(R.diagnostics, "residual", residual)
    monkeypatch.setattr(R.diagnostics, "check_state", check_state)


def _state(step=10, t=1.0):
    q = torch.zeros(5, 2, 2, 2, dtype=torch.float64)
    return State(blocks=(Block(q=q, xyz=torch.zeros(3, 2, 2, 2, dtype=torch.float64)),), metrics=(None,),
                 t=t, step=step)


def _cfg(nan_check=True):
    return SimpleNamespace(ghost=2, nan_check=nan_check, gas=SimpleNamespace(gamma=1.4))


def test_residual_rows_and_final_state(fakes, tmp_path):
    st = _state()
    final, log = R.run(st, _cfg(), 0.5, 5, plan=_Plan(), residual_every=2)
    assert [r[0] for r in log.rows] == [12, 14]
    assert [r[1] for r in log.rows] == [2.0, 3.0]
    assert [r[2][0] for r in log.rows] == [2.0, 4.0]
    assert final.step == 15 and final.t == 3.5
    assert torch.all(final.blocks[0].q == 5)
    assert torch.all(st.blocks[0].q == 0)  # the input state is not modified
    path = tmp_path / "res.txt"
    R.write_residual_log(path, log)
    lines = path.read_text().splitlines()
    assert lines[0].startswith("# step t res_rho") and len(lines) == 3
    assert lines[1].split()[0] == "12" and len(lines[1].split()) == 7


def test_nan_guard_names_the_step_and_dumps_both_states(fakes, tmp_path):
    with pytest.raises(FloatingPointError, match=r"step 13: 1 non-finite"):
        R.run(_state(), _cfg(), 0.5, 5, plan=_Plan(bad=3), dump_dir=tmp_path)
    good = torch.load(tmp_path / "step0000012_good.pt")
    bad = torch.load(tmp_path / "step0000013_bad.pt")
    assert torch.all(good[0] == 2)
    assert torch.isnan(bad[0].view(-1)[0]) and torch.all(bad[0].view(-1)[1:] == 3)


def test_no_check_without_nan_check(fakes):
    final, log = R.run(_state(), _cfg(nan_check=False), 0.5, 4, plan=_Plan(bad=2), residual_every=0)
    assert log.rows == [] and final.step == 14
    assert torch.isnan(final.blocks[0].q.view(-1)[0])


def test_check_every_skips_steps_between_checks(fakes):
    # the NaN of step 1 is first seen by the check after step 2 (the NaN propagates)
    with pytest.raises(FloatingPointError, match=r"step 12:"):
        R.run(_state(), _cfg(), 0.5, 5, plan=_Plan(bad=1), check_every=2)

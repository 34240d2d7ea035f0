"""The adjoint configuration at full size: 96^3 Taylor-Green block (M0 0.3,
Re 800, 1 % noise), J = interior kinetic energy after 50 TVD-RK3 steps, a
checkpoint every 10 steps, 16 seeded unit directions, eps = 1e-6 (the
configuration's own values), FP64.

Bounds (see famrdp_jax_b200/solver/gradcheck.py for the two error measures):
  * every direction: |fd - ad| <= 1e-6 |grad J|;
  * the gradient direction: |fd - |g|| <= 1e-6 |g| (a per-direction relative
    bound where the directional derivative is large enough to resolve);
  * dJ/dmu0: relative error <= 1e-6 (central difference in mu0 with step
    1e-3 mu0; see gradcheck.py for why not 1e-6).
The per-direction relative errors of the random directions are printed, not
bounded: their derivatives are about |grad J| / sqrt(5e6) and FP64 rounding
of J divided by eps is of that order.
"""
import pytest

from famrdp_jax_b200 import cases
from famrdp_jax_b200.solver import diagnostics
from famrdp_jax_b200.solver.gradcheck import fd_check_kinetic_energy

pytestmark = pytest.mark.gpu


def test_adjoint_full_size_matches_central_differences(cuda_device):
    c = cases.tgv(n=96, M0=0.3, Re=800.0, noise=0.01, seed=0)
    st = cases.to_state(c, cuda_device)
    dt = diagnostics.cfl_dt(st, c.cfg, c.cfl)
    r = fd_check_kinetic_energy(st, c.cfg, dt, 50, checkpoint_every=10, eps=1e-6, ndirs=16, seed=0)
    print({k: v for k, v in r.items() if k != "per_direction"})
    for row in r["per_direction"]:
        print("  fd %.12e ad %.12e rel %.2e rel|g| %.2e" % (row["fd"], row["ad"], row["rel_direction"],
                                                         row["rel_gradnorm"]))
    assert r["max_rel_gradnorm"] <= 1e-6, r["max_rel_gradnorm"]
    assert r["gradient_direction_rel"] <= 1e-6, r["gradient_direction_rel"]
    assert r["dJ_dmu0_rel"] <= 1e-6, r["dJ_dmu0_rel"]

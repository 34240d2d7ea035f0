"""Helpers shared by the GPU parity tests (no test functions here)."""
import numpy as np
import torch

from famrdp_jax_b200.core.types import Block, Metrics, State


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def dev(x, device="cuda"):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device=device)


def host(t):
    return t.detach().cpu().numpy()


def state_from_case(case, device="cuda"):
    blocks, metrics = [], []
    for q, (jac, kxyz, vol) in zip(case.qs, case.metrics):
        xyz = torch.zeros((3,) + q.shape[1:], dtype=torch.float64, device=device)
        blocks.append(Block(q=dev(q, device), xyz=xyz))
        metrics.append(Metrics(jac=dev(jac, device), kxyz=dev(kxyz, device), vol=dev(vol, device)))
    return State(blocks=tuple(blocks), metrics=tuple(metrics), t=0.0, step=0)


def random_block(shape, seed, M=0.3, noise=0.05, metric_noise=0.1, gamma=1.4):
    """A non-uniform state and a perturbed, non-diagonal metric field."""
    rng = np.random.default_rng(seed)
    ni, nj, nk = shape
    rho = 1.0 + noise * rng.standard_normal(shape)
    u = M + noise * rng.standard_normal(shape)
    v = -0.5 * M + noise * rng.standard_normal(shape)
    w = 0.25 * M + noise * rng.standard_normal(shape)
    p = 1.0 / gamma * (1.0 + noise * rng.standard_normal(shape))
    ke = 0.5 * (u * u + v * v + w * w)
    q = np.stack([rho, rho * u, rho * v, rho * w, p / (gamma - 1) + rho * ke])
    kxyz = np.eye(3)[:, :, None, None, None] * 4.0 + metric_noise * 4.0 * rng.standard_normal((3, 3) + shape)
    vol = (1.0 / 64.0) * (1.0 + 0.1 * rng.random(shape))
    return q, kxyz, vol

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


# ---- the oracle's block right-hand sides on a pool of host processes ----------
_POOL_STATE = {}


def _pool_init(metrics, cfg):
    _POOL_STATE["metrics"] = metrics
    _POOL_STATE["cfg"] = cfg


def _pool_rhs(args):
    from oracle.ref import NP
    b, q = args
    kxyz, vol = _POOL_STATE["metrics"][b]
    return NP.rhs_block(q, kxyz, vol, _POOL_STATE["cfg"])


class OraclePool:
    """Evaluates the NumPy oracle's per-block RHS (the blocks are independent
    within a stage) on spawned worker processes, one block per task, so that
    multi-block trajectories of a few hundred steps finish in seconds.  Use as
    ``NP.step(qs, metrics, cfg, dt, rhs_map=pool.rhs_map)``.  Workers are
    started with ``spawn`` (never forked from a process that holds a CUDA
    context)."""

    def __init__(self, metrics, cfg, workers=None):
        import concurrent.futures
        import multiprocessing
        import os
        n = workers or max(1, min(len(metrics), len(os.sched_getaffinity(0))))
        self.ex = concurrent.futures.ProcessPoolExecutor(
            max_workers=n, mp_context=multiprocessing.get_context("spawn"), initializer=_pool_init,
            initargs=(list(metrics), cfg))

    def rhs_map(self, qs):
        return list(self.ex.map(_pool_rhs, list(enumerate(qs))))

    def close(self):
        self.ex.shutdown(wait=True, cancel_futures=True)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

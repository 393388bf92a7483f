"""Batch composition helpers: seeded synthetic states and their assignment to GPUs.

States are independent, so a batch shards across ranks with no data-path collective (weak
scaling); each rank evaluates its own states. The cost model used for balancing is the
trajectory work, D^3 times the step count, with the step count unknown in advance: states are
dealt by decreasing D^3 to the rank with the least assigned work.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["random_state", "z2_state", "config_states", "uneven_states", "shard"]


def _draw(rng, n):
    return (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2.0)


def random_state(d, seed, scale=0.2):
    """R and A with i.i.d. standard complex Gaussian entries times `scale` (NumPy PCG64,
    R drawn first), K = (A + A^dag)/2."""
    rng = np.random.default_rng(seed)
    r = scale * _draw(rng, d)
    a = scale * _draw(rng, d)
    return r, (a + a.conj().T) / 2


def z2_state(d, seed, scale=0.2):
    """R odd and K even under the split into two halves of d/2 (blocks drawn k1, k2, R12, R21)."""
    if d % 2:
        raise ValueError("Z2 states need an even D")
    n = d // 2
    rng = np.random.default_rng(seed)
    z = np.zeros((n, n), complex)
    k1, k2 = _draw(rng, n), _draw(rng, n)
    r = scale * np.block([[z, _draw(rng, n)], [_draw(rng, n), z]])
    k = scale * np.block([[(k1 + k1.conj().T) / 2, z], [z, (k2 + k2.conj().T) / 2]])
    return r, k


def config_states(name):
    """(R list, K list, couplings, description) of a named workload.
    d64_mixed: 16 random (seeds 0..15) + 16 Z2 (seeds 100..115) states at D = 64, g = 2;
    d32_batch: 64 random D = 32 states (seeds 0..63), g ~ U[0.5, 3] (seed 12345);
    d64_pair: the first random and the first Z2 state of d64_mixed (a small profiling case);
    d64_single: the first random state of d64_mixed alone (the latency of one evaluation, the call
    an L-BFGS trial makes);
    uneven200: 200 random states with D drawn from {16, 32, 48, 64, 96, 128}, g ~ U[0.5, 3] and
    atol, rtol each drawn from {1e-10, 1e-12} (use uneven_states for the tolerances)."""
    if name == "uneven200":
        R, K, g, _ = uneven_states(200)
        return R, K, g, "200 random states D in {16,32,48,64,96,128} (scaling 0.2), g~U[0.5,3], mixed atol/rtol"
    if name == "d64_mixed":
        R, K = [], []
        for s in range(16):
            r, k = random_state(64, s)
            R.append(r)
            K.append(k)
        for s in range(16):
            r, k = z2_state(64, 100 + s)
            R.append(r)
            K.append(k)
        return R, K, [2.0] * 32, "32 states D=64: 16 random + 16 Z2 (scaling 0.2), g=2"
    if name == "d64_pair":
        (r0, k0), (r1, k1) = random_state(64, 0), z2_state(64, 100)
        return [r0, r1], [k0, k1], [2.0, 2.0], "2 states D=64: 1 random + 1 Z2 (scaling 0.2), g=2"
    if name == "d64_single":
        r0, k0 = random_state(64, 0)
        return [r0], [k0], [2.0], "1 random state D=64 (seed 0, scaling 0.2), g=2"
    if name == "d32_batch":
        R, K = zip(*(random_state(32, s) for s in range(64)))
        g = np.random.default_rng(12345).uniform(0.5, 3.0, 64)
        return list(R), list(K), [float(x) for x in g], "64 random states D=32 (scaling 0.2), g~U[0.5,3]"
    raise ValueError(f"unknown workload {name!r}")


UNEVEN_DIMS = (16, 32, 48, 64, 96, 128)
UNEVEN_TOLERANCES = (1e-10, 1e-12)


def uneven_states(count=200, seed=2024):
    """The uneven workload: state i has D drawn from UNEVEN_DIMS, R, K from random_state(D,
    4000 + i), a coupling g ~ U[0.5, 3] and a tolerance pair (atol, rtol) with both drawn from
    UNEVEN_TOLERANCES; all draws come from one default_rng(seed) stream, state by state.
    Returns (R list, K list, couplings, tolerances)."""
    rng = np.random.default_rng(seed)
    R, K, g, tol = [], [], [], []
    for i in range(count):
        d = int(rng.choice(UNEVEN_DIMS))
        r, k = random_state(d, 4000 + i)
        R.append(r)
        K.append(k)
        g.append(float(rng.uniform(0.5, 3.0)))
        tol.append((float(rng.choice(UNEVEN_TOLERANCES)), float(rng.choice(UNEVEN_TOLERANCES))))
    return R, K, g, tol


def shard(dims, rank, world):
    """Indices of the states of `rank` out of `world`: greedy by decreasing D^3."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    load = [0.0] * world
    owner = [0] * len(dims)
    for i in sorted(range(len(dims)), key=lambda i: (-dims[i] ** 3, i)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[i] = r
        load[r] += dims[i] ** 3
    return [i for i in range(len(dims)) if owner[i] == rank]

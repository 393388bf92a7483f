"""Generate the golden vectors of tests/golden/ by running RcmpsCore.jl's own NumPy path.

This script imports the reference package rcmps_gpu read-only from a local checkout of the
reference (its gpu/src directory, given as --reference PATH or in the environment variable
RCMPS_REFERENCE_SRC; there is no default) and writes .npz files:
  small.npz     D = 4, 6, 8 random and D = 8 Z2 states at W = 30, n_quad = 64, 128 kinetic nodes
  d16.npz       one D = 16 random state at the optimizer defaults (W = 30, n_quad = 512, 512 nodes)
  d64.npz       the seed-42 D = 64 random state at the optimizer defaults
  samples_d5.npz  trajectory samples of the reduced quartic system, D = 5, W = 2, n_quad = 16
  phi.npz       <phi> in closed form (ode_backend.phi_expectation) and by the ODE of the first
                monomial (validate_sweep.phi_by_ode, host NumPy integrator): D = 4 random (W = 6,
                n_quad = 24), D = 8 Z2 (W = 20, n_quad = 64) and D = 16 random at the refined
                validation settings (W = 40, n_quad = 1024, 1e-14/1e-13)
  optim.npz     eight L-BFGS iterations of the reference's controller (runtime/optimizer.py) from a
                D = 4 random state, objective = quartic (W = 6, n_quad = 24) + kinetic (32 nodes)
                + finished gradient, stationary densities by numerics.stationary_state: per
                accepted iteration the energy, step alpha, trials and gradient norm
  config0.npz   the same controller for 100 iterations from the seed-42 D = 8 random state with
                g = 2 at the optimizer defaults (W = 30, n_quad = 512, 512 kinetic nodes)
  finish.npz    the reference's preconditioned boundary solve and finished gradient
                (numerics.finish_gradient) with its GMRES matvec count, on random states D = 8, 16
                and a Z2 state D = 16 with seeded covectors and environments
  packed.npz    the packed Z2 route (evaluate_quartic(..., packed_z2=True), the default of the
                persistent trajectory) on Z2 states D = 4, 8 (W = 30, n_quad = 64), 16 and 32
                (W = 30, n_quad = 512, 512 kinetic nodes: the optimizer defaults, with the
                kinetic term and the finished gradient), and the packed trajectory samples of a
                D = 4 Z2 state at W = 2, n_quad = 16
  d32batch.npz  the first 8 states of the 64-state D = 32 batch workload (random seeds 0..7,
                couplings g ~ U[0.5, 3] from default_rng(12345)) at the optimizer defaults
  bench.npz     four states of the 32-state D = 64 benchmark workload at the optimizer defaults:
                random seeds 0 and 1 (unpacked reduced route) and Z2 seeds 100 and 101 (the
                packed route, with the reference's own stationary density), each with the kinetic
                term and the finished gradient
  uneven.npz    states 0, 1, 2, 4, 5, 6 (D = 16, 32, 48) of the uneven 200-state workload, each at
                its own drawn (atol, rtol) pair, W = 30, n_quad = 512, 512 kinetic nodes
  ode.npz       the all-ODE route (evaluate_phi4: kinetic1 + kinetic2 + g phi^4 as 26 channels):
                D = 3 (W = 6, n_quad = 24), D = 8 random and Z2 (W = 20, n_quad = 64) and
                D = 16 (W = 20, n_quad = 192, the Julia defaults of the fixture)
Each state record holds R, K, rho (the reference's stationary_state at tolerance 1e-13), the
coupling, the settings, and the reference outputs: quartic value/covector/environment and its
DOP853 step counts, kinetic value/covector/environment, the summed energy and the finished
gradient (finish_gradient, metric_reg 1e-3). The copied Julia fixture phi4_g2_D16_z2_portable/
is the reference's test/fixtures/phi4_g2_D16_z2_portable (exported by RcmpsCore 0.2.0).

States: NumPy PCG64 default_rng(seed); R and A with i.i.d. standard complex Gaussian entries
times 0.2 (R drawn first), K = (A + A^dag)/2; Z2 states draw blocks in the order k1, k2, R12, R21.
Run: python tests/golden/make_golden.py --reference PATH/gpu/src [name ...]  (all files by
default; names: small d16 d64 samples ode packed phi optim config0 finish d32batch bench uneven; the D = 64
records dominate, about a minute each on one core)
"""
from __future__ import annotations

import math
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
kb = nm = ob = None     # the reference's runtime modules, imported by _import_reference


def _import_reference(path):
    """Import rcmps_gpu's runtime modules from the reference checkout at `path` (gpu/src)."""
    global kb, nm, ob
    if not path:
        raise SystemExit("give the reference's gpu/src directory: --reference PATH or RCMPS_REFERENCE_SRC")
    if not (Path(path) / "rcmps_gpu").is_dir():
        raise SystemExit(f"{path} holds no rcmps_gpu package")
    sys.path.insert(0, str(path))
    from rcmps_gpu.optimizer.runtime import kinetic_backend, numerics, ode_backend
    kb, nm, ob = kinetic_backend, numerics, ode_backend


def draw(rng, n):
    return (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2.0)


def random_state(d, seed, scale=0.2):
    rng = np.random.default_rng(seed)
    r = scale * draw(rng, d)
    a = scale * draw(rng, d)
    return r, (a + a.conj().T) / 2


def z2_state(d, seed, scale=0.2):
    n = d // 2
    rng = np.random.default_rng(seed)
    z = np.zeros((n, n), complex)
    k1, k2 = draw(rng, n), draw(rng, n)
    r = scale * np.block([[z, draw(rng, n)], [draw(rng, n), z]])
    k = scale * np.block([[(k1 + k1.conj().T) / 2, z], [z, (k2 + k2.conj().T) / 2]])
    return r, k


def evaluate(r, k, g, window, nq, nodes, atol=1e-13, rtol=1e-12):
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    quartic = ob.evaluate_quartic(r, q, rho, g, xp=np, half_window=window, n_quad=nq, atol=atol, rtol=rtol,
                                  reduced=True)
    kinetic = kb.kinetic_raw(q, r, rho, nodes, xp=np, tolerance=1e-12, maxdim=1024)
    cov = quartic["covector"] + kinetic["covector"]
    env = quartic["environment"] + kinetic["environment"]
    grad, _ = nm.finish_gradient(q, r, rho, cov, env, metric_reg=1e-3)
    return dict(R=r, K=k, rho=rho, g=g, window=window, n_quad=nq, nodes=nodes, atol=atol, rtol=rtol,
                quartic_value=quartic["value"], quartic_covector=quartic["covector"],
                quartic_environment=quartic["environment"],
                accepted=quartic["stats"]["accepted_steps"], rejected=quartic["stats"]["rejected_steps"],
                kinetic_value=kinetic["value"], kinetic_covector=kinetic["covector"],
                kinetic_environment=kinetic["environment"],
                energy=quartic["value"] + kinetic["value"], gradient=grad)


def evaluate_packed(r, k, g, window, nq, nodes=None):
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    quartic = ob.evaluate_quartic(r, q, rho, g, xp=np, half_window=window, n_quad=nq, atol=1e-13, rtol=1e-12,
                                  packed_z2=True)
    rec = dict(R=r, K=k, rho=rho, g=g, window=window, n_quad=nq, quartic_value=quartic["value"],
               quartic_covector=quartic["covector"], quartic_environment=quartic["environment"],
               accepted=quartic["stats"]["accepted_steps"], rejected=quartic["stats"]["rejected_steps"])
    if nodes:
        kinetic = kb.kinetic_raw(q, r, rho, nodes, xp=np, tolerance=1e-12, maxdim=1024)
        cov = quartic["covector"] + kinetic["covector"]
        env = quartic["environment"] + kinetic["environment"]
        grad, _ = nm.finish_gradient(q, r, rho, cov, env, metric_reg=1e-3)
        rec.update(nodes=nodes, energy=quartic["value"] + kinetic["value"], gradient=grad)
    return rec


def packed_samples():
    r, k = z2_state(4, 404)
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    rhs = ob._PackedZ2QuarticRHS(q, r, rho, np)
    points, _ = ob.quadrature(2.0, 16)
    samples, stats = ob._integrate(rhs, np.r_[points, math.sqrt(2.0)], atol=1e-13, rtol=1e-12, initial_step=None,
                                   max_steps=100000)
    return dict(R=r, K=k, rho=rho, window=2.0, n_quad=16, samples=samples,
                accepted=stats["accepted_steps"], rejected=stats["rejected_steps"])


def evaluate_phi(r, k, window, nq, atol=1e-13, rtol=1e-12):
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    spec = ob._Spec(2, ((0, 1, True, 1.), (0, 1, False, 1.)))
    out = ob._evaluate(r, q, rho, [spec], [1.], xp=np, half_window=window, n_quad=nq, atol=atol, rtol=rtol,
                       initial_step=None, max_steps=1_000_000, use_graph=False, progress=None)
    return dict(R=r, K=k, rho=rho, window=window, n_quad=nq, atol=atol, rtol=rtol,
                phi_ode=float(out["value"]), phi=ob.phi_expectation(r, rho, window),
                accepted=out["stats"]["accepted_steps"], rejected=out["stats"]["rejected_steps"])


OPTIM = dict(seed=414, d=4, g=1.0, window=6.0, n_quad=24, nodes=32, iterations=8)
# the config-0 run: D = 8, seed 42, g = 2 at the optimizer defaults, 100 L-BFGS iterations
CONFIG0 = dict(seed=42, d=8, g=2.0, window=30.0, n_quad=512, nodes=512, iterations=100)


def optim_run(c=OPTIM):
    from rcmps_gpu.optimizer.runtime import optimizer as opt
    r, k = random_state(c["d"], c["seed"])

    def objective(rr, kk, rho):
        q = -1j * kk - rr.conj().T @ rr / 2
        quartic = ob.evaluate_quartic(rr, q, rho, c["g"], xp=np, half_window=c["window"], n_quad=c["n_quad"],
                                      atol=1e-13, rtol=1e-12, reduced=True)
        kinetic = kb.kinetic_raw(q, rr, rho, c["nodes"], xp=np, tolerance=1e-12, maxdim=1024)
        grad, _ = nm.finish_gradient(q, rr, rho, quartic["covector"] + kinetic["covector"],
                                     quartic["environment"] + kinetic["environment"], metric_reg=1e-3)
        return quartic["value"] + kinetic["value"], grad, {}

    q0 = -1j * k - r.conj().T @ r / 2
    rho0, _ = nm.stationary_state(q0, r, tolerance=1e-13)
    e0, g0, _ = objective(r, k, rho0)
    events = list(opt.optimize(r, k, rho0, e0, g0, objective, dict(max_iterations=c["iterations"], gradient_tol=1e-9)))
    accepted = [ev for ev in events if ev["type"] == "accepted"]
    last = accepted[-1]["state"]
    return dict(R=r, K=k, rho=rho0, energy0=e0, gradient0=g0, **{key: value for key, value in c.items()},
                energies=[ev["energy"] for ev in accepted], alphas=[ev["alpha"] for ev in accepted],
                trials=[ev["trials"] for ev in accepted], gradient_norms=[ev["gradient_norm"] for ev in accepted],
                R_final=last["R"], K_final=last["K"], stop_reason=events[-1].get("reason", ""),
                trial_iteration=[ev["iteration"] for ev in events if ev["type"] == "trial"],
                trial_energy=[ev.get("energy", np.nan) for ev in events if ev["type"] == "trial"],
                trial_bound=[ev.get("armijo_bound", np.nan) for ev in events if ev["type"] == "trial"])


def finish_record(r, k, seed):
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    rng = np.random.default_rng(seed)
    d = len(r)
    env = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    env = (env + env.conj().T) / 2
    cov = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    grad, st = nm.finish_gradient(q, r, rho, cov, env, metric_reg=1e-3)
    return dict(R=r, K=k, rho=rho, covector=cov, environment=env, gradient=grad, matvecs=st["matvecs"])


def evaluate_ode(r, k, g, window, nq):
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    out = ob.evaluate_phi4(r, q, rho, g, xp=np, half_window=window, n_quad=nq, atol=1e-13, rtol=1e-12)
    grad, _ = nm.finish_gradient(q, r, rho, out["covector"], out["environment"], metric_reg=1e-3)
    return dict(R=r, K=k, rho=rho, g=g, window=window, n_quad=nq, value=out["value"],
                covector=out["covector"], environment=out["environment"],
                accepted=out["stats"]["accepted_steps"], rejected=out["stats"]["rejected_steps"],
                gradient=grad)


def save(name, records):
    flat = {}
    for i, rec in enumerate(records):
        for key, value in rec.items():
            flat[f"s{i}_{key}"] = np.asarray(value)
    flat["count"] = np.asarray(len(records))
    np.savez_compressed(HERE / name, **flat)


def main(names):
    t0 = time.time()
    if "small" in names:
        small = [evaluate(*random_state(d, 500 + d), 0.5 + 0.5 * i, 30.0, 64, 128) for i, d in enumerate((4, 6, 8))]
        small.append(evaluate(*z2_state(8, 508), 2.0, 30.0, 64, 128))
        save("small.npz", small)
    if "d16" in names:
        save("d16.npz", [evaluate(*random_state(16, 16), 2.0, 30.0, 512, 512)])
    if "d64" in names:
        save("d64.npz", [evaluate(*random_state(64, 42), 2.0, 30.0, 512, 512)])
    if "ode" in names:
        save("ode.npz", [evaluate_ode(*random_state(3, 703), 1.5, 6.0, 24),
                         evaluate_ode(*random_state(8, 708), 2.0, 20.0, 64),
                         evaluate_ode(*z2_state(8, 718), 2.5, 20.0, 64),
                         evaluate_ode(*random_state(16, 716), 2.0, 20.0, 192)])
    if "samples" in names:
        samples_d5()
    if "phi" in names:
        save("phi.npz", [evaluate_phi(*random_state(4, 904), 6.0, 24),
                         evaluate_phi(*z2_state(8, 908), 20.0, 64),
                         evaluate_phi(*random_state(16, 916), 40.0, 1024, 1e-14, 1e-13)])
    if "finish" in names:
        save("finish.npz", [finish_record(*random_state(8, 808), 1), finish_record(*random_state(16, 816), 2),
                            finish_record(*z2_state(16, 826), 3)])
    if "optim" in names:
        save("optim.npz", [optim_run()])
    if "config0" in names:
        save("config0.npz", [optim_run(CONFIG0)])
    if "d32batch" in names:
        gs = np.random.default_rng(12345).uniform(0.5, 3.0, 64)
        save("d32batch.npz", [evaluate(*random_state(32, seed), float(gs[seed]), 30.0, 512, 512) for seed in range(8)])
    if "uneven" in names:
        draws = uneven_draws(20)
        save("uneven.npz", [dict(evaluate(*random_state(d, seed), g, 30.0, 512, 512, atol, rtol), index=i)
                            for i, (d, seed, g, atol, rtol) in enumerate(draws) if i in UNEVEN_PINNED])
    if "bench" in names:
        save("bench.npz", [evaluate(*random_state(64, 0), 2.0, 30.0, 512, 512),
                           evaluate(*random_state(64, 1), 2.0, 30.0, 512, 512),
                           evaluate_packed(*z2_state(64, 100), 2.0, 30.0, 512, 512),
                           evaluate_packed(*z2_state(64, 101), 2.0, 30.0, 512, 512)])
    if "packed" in names:
        save("packed.npz", [evaluate_packed(*z2_state(4, 604), 1.5, 30.0, 64),
                            evaluate_packed(*z2_state(8, 508), 2.0, 30.0, 64),
                            evaluate_packed(*z2_state(16, 616), 2.0, 30.0, 512, 512),
                            evaluate_packed(*z2_state(32, 632), 2.0, 30.0, 512, 512),
                            packed_samples()])
    print(f"golden vectors written in {time.time() - t0:.1f} s")


def samples_d5():
    # trajectory samples of the reduced system (the persistent kernel's channels)
    r, k = random_state(5, 5)
    q = -1j * k - r.conj().T @ r / 2
    rho, _ = nm.stationary_state(q, r, tolerance=1e-13)
    rhs = ob._UnpackedQuarticRHS(q, r, rho, np)
    points, _ = ob.quadrature(2.0, 16)
    samples, stats = ob._integrate(rhs, np.r_[points, math.sqrt(2.0)], atol=1e-13, rtol=1e-12, initial_step=None,
                                   max_steps=100000)
    np.savez_compressed(HERE / "samples_d5.npz", R=r, K=k, rho=rho, window=2.0, n_quad=16, samples=samples,
                        accepted=stats["accepted_steps"], rejected=stats["rejected_steps"])


UNEVEN_PINNED = (0, 1, 2, 4, 5, 6)


def uneven_draws(count, seed=2024):
    """(D, state seed, g, atol, rtol) of the uneven workload's first `count` states: one
    default_rng(seed) stream draws, state by state, D from {16, 32, 48, 64, 96, 128}, g ~ U[0.5, 3]
    and atol, rtol from {1e-10, 1e-12}; state i is random_state(D, 4000 + i)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        d = int(rng.choice((16, 32, 48, 64, 96, 128)))
        g = float(rng.uniform(0.5, 3.0))
        atol, rtol = float(rng.choice((1e-10, 1e-12))), float(rng.choice((1e-10, 1e-12)))
        out.append((d, 4000 + i, g, atol, rtol))
    return out


ALL = ["small", "d16", "d64", "ode", "samples", "packed", "phi", "optim", "config0", "finish", "d32batch", "bench",
       "uneven"]

if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reference", default=os.environ.get("RCMPS_REFERENCE_SRC"),
                    help="the reference's gpu/src directory (default: $RCMPS_REFERENCE_SRC)")
    ap.add_argument("names", nargs="*", choices=ALL + [[]], default=[])
    a = ap.parse_args()
    _import_reference(a.reference)
    main(a.names or ALL)

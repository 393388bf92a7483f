"""CPU oracle of the phi^4 energy-and-gradient evaluation fg_phi4 (test infrastructure only).

This module is the checker, not the product. Only tests, the smoke check of
__graft_entry__ and the CPU-baseline leg of bench.py may import it. The CUDA path never
calls it, and nothing in the product falls back to it.

It restates in NumPy/SciPy the algorithm of the reference's GPU objective
(gpu/src/rcmps_gpu/optimizer/runtime/ of RcmpsCore.jl): the seven-channel reduced
quartic system integrated by adaptive DOP853 with order-7 dense output at the Gauss
nodes, the quadrature pullback, the kinetic infinite-line resolvents by shifted Arnoldi,
the stationary density and the boundary Poisson correction with the metric solve.
Each function names the reference lines it follows.

Pinning (tests/test_oracle.py):
  * the Julia fixture test/fixtures/phi4_g2_D16_z2_portable (energy -0.15648780475169466
    and its gradient, exported by RcmpsCore 0.2.0), copied into tests/golden/;
  * golden vectors produced by the reference's own NumPy path imported read-only
    (tests/golden/make_golden.py writes them; the committed .npz files are its output).

Third-party arithmetic: the DOP853 tables come from SciPy
(scipy.integrate._ivp.dop853_coefficients), which is what the reference uses too
(ode_backend.py:23); the Bessel function K_{1/4} from scipy.special.kv.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.integrate._ivp import dop853_coefficients as DOP
from scipy.special import gamma, kv

__all__ = [
    "OracleFailure", "source", "quadrature", "angular_grid", "lindblad", "lindblad_adjoint",
    "QuarticSystem", "integrate", "quartic_pullback", "evaluate_quartic", "kinetic_raw",
    "stationary_state", "boundary_environment", "finish_gradient", "metric", "fg_phi4",
    "phi4_state", "z2_state", "left_canonical_q", "PackedZ2System", "z2_structure_ok",
    "source_integral", "phi_expectation", "phi_by_ode", "NoJumpInverse",
    "boundary_environment_preconditioned",
]


class OracleFailure(RuntimeError):
    """A numerical requirement of the oracle failed."""


# --------------------------------------------------------------------------- basics

_J_NORM = 2.0 ** 2.25 * math.sqrt(math.pi) * gamma(1.25)


def source(t):
    """2|t| J(t^2), the transformed smearing source (ode_backend.py:27-34,
    src/observables.jl:79-82); its finite limit at t = 0 is 1/sqrt(pi)."""
    a = abs(float(t))
    if a == 0.0:
        return 1.0 / math.sqrt(math.pi)
    return 2.0 * a * kv(0.25, a * a) / (_J_NORM * math.sqrt(a))


def quadrature(half_window, n_quad):
    """Gauss-Legendre nodes on [0, sqrt(W)], mirrored to [-sqrt(W), 0] (ode_backend.py:37-44,
    src/observables.jl:142-152). Returns (points, weights), both of length 2 n_quad."""
    if half_window <= 0 or n_quad < 8:
        raise ValueError("positive half_window and n_quad >= 8 required")
    x, w = np.polynomial.legendre.leggauss(int(n_quad))
    half = math.sqrt(half_window) / 2.0
    p, q = (x + 1.0) * half, w * half
    return np.concatenate([-p[::-1], p]), np.concatenate([q[::-1], q])


def angular_grid(nodes):
    """cos(theta) and weights (including 2/pi) of the kinetic angular integral
    (kinetic_backend.py:51-57, src/kinetic.jl kinetic_grid)."""
    x, w = np.polynomial.legendre.leggauss(int(nodes))
    return np.cos(0.25 * math.pi * (x + 1.0)), 0.5 * w


def adj(x):
    return np.swapaxes(x, -1, -2).conj()


def lindblad(q, r, x):
    """L(X) = QX + XQ^dag + RXR^dag (src/transfer.jl:2)."""
    return q @ x + x @ adj(q) + r @ x @ adj(r)


def lindblad_adjoint(q, r, x):
    """L*(X) = Q^dag X + XQ + R^dag X R (src/transfer.jl:4)."""
    return adj(q) @ x + x @ q + adj(r) @ x @ r


def left_canonical_q(r, k):
    """Q = -iK - R^dag R / 2 (src/state.jl:47)."""
    return -1j * k - adj(r) @ r / 2.0


def phi4_state(d, seed, scale=0.2):
    """Seeded synthetic state: R and A with i.i.d. standard complex Gaussian entries (NumPy
    PCG64, R drawn first) times `scale`, K = (A + A^dag)/2."""
    rng = np.random.default_rng(seed)

    def draw():
        return (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / math.sqrt(2.0)
    r = scale * draw()
    a = scale * draw()
    return r, (a + adj(a)) / 2.0


def z2_state(d, seed, scale=0.2):
    """Seeded Z2-symmetric state: R odd and K even under the parity split into two halves of
    D/2 (src/state.jl:61-70); i.i.d. standard complex Gaussian blocks times `scale`."""
    if d % 2:
        raise ValueError("Z2 states need an even D")
    n = d // 2
    rng = np.random.default_rng(seed)

    def draw():
        return (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2.0)
    z = np.zeros((n, n), complex)
    k1, k2 = draw(), draw()
    r = scale * np.block([[z, draw()], [draw(), z]])
    k = scale * np.block([[(k1 + adj(k1)) / 2.0, z], [z, (k2 + adj(k2)) / 2.0]])
    return r, k


# --------------------------------------------------------------------------- quartic system

# Insertion edges of the reduced quartic system (ode_backend.py:193): channel -> (source, coefficient).
# Channels 0-2 are the forward F1..F3, 3-6 the adjoint A0..A3 (A4 = I and F0 = rho are fixed).
INSERTIONS = {1: (0, 2.0), 2: (1, 3.0), 3: (4, 1.0), 4: (5, 2.0), 5: (6, 3.0)}
FORWARD = (0, 1, 2)


class QuarticSystem:
    """The seven live D x D channels plus one scalar of the g*phi^4 term
    (ode_backend.py:170-233, 718-747; src/observables.jl:114-140 with monomial_spec(4)).

    For channel c with operators (Qc, Rc) = (Q, R) forward or (Q^dag, R^dag) adjoint:
        dX_c/dt = jac (Qc X_c + X_c Qc^dag + Rc X_c Rc^dag)
                  + src (coef_c (Rc X_s + X_s Rc^dag) + fixed_c),
    where (s, coef_c) = INSERTIONS[c], fixed_0 = R rho + rho R^dag, fixed_6 = 4 (R + R^dag),
    jac = 2|t| and src = source(t). The scalar accumulates 4 src Re tr(R F3 + F3 R^dag);
    its endpoint value is the quartic energy density."""

    def __init__(self, q, r, rho):
        self.q, self.r, self.rho = (np.asarray(x, dtype=np.complex128) for x in (q, r, rho))
        self.d = len(self.q)
        d = self.d
        self.size = 7 * d * d + 1
        self.ops = [(self.q, self.r) if c in FORWARD else (adj(self.q), adj(self.r)) for c in range(7)]
        self.fixed = np.zeros((7, d, d), complex)
        self.fixed[0] = self.r @ self.rho + self.rho @ adj(self.r)
        self.fixed[6] = 4.0 * (self.r + adj(self.r))
        self.calls = 0

    def initial(self):
        return np.zeros(self.size, complex)

    def __call__(self, t, y, src=None):
        self.calls += 1
        d = self.d
        jac = 2.0 * abs(t)
        src = source(t) if src is None else src
        x = y[:-1].reshape(7, d, d)
        out = np.empty_like(y)
        o = out[:-1].reshape(7, d, d)
        for c in range(7):
            qc, rc = self.ops[c]
            value = jac * (qc @ x[c] + x[c] @ adj(qc) + rc @ x[c] @ adj(rc)) + src * self.fixed[c]
            if c in INSERTIONS:
                s, coef = INSERTIONS[c]
                value = value + (src * coef) * (rc @ x[s] + x[s] @ adj(rc))
            o[c] = value
        f3 = x[2]
        out[-1] = 4.0 * src * np.trace(self.r @ f3 + f3 @ adj(self.r)).real
        return out


# --------------------------------------------------------------------------- packed Z2 route

# Parity of the seven channels of a Z2-symmetric state (R odd, Q and rho even): odd channels
# have only the off-diagonal blocks, even channels only the diagonal ones.
PARITY = (1, 0, 1, 0, 1, 0, 1)
# Packed vector: per channel its upper off-diagonal block (odd) or its two diagonal blocks
# (even), in channel order, then the scalar; 10 (D/2)^2 + 1 entries (ode_backend.py:236-275).
PACKED_BLOCKS = tuple((c, (0, 1)) if PARITY[c] else (c, blk) for c in range(7)
                      for blk in (((0, 1),) if PARITY[c] else ((0, 0), (1, 1))))


def z2_structure_ok(r, q, rho):
    """The exact block structure the packed route requires (ode_backend.py:246-256): even D,
    R's diagonal blocks and the off-diagonal blocks of Q and rho exactly zero, rho Hermitian to
    1e-13 relative. Nothing is projected."""
    d2 = len(q)
    if d2 % 2 or d2 == 0:
        return False
    n = d2 // 2
    zero = (r[:n, :n], r[n:, n:], q[:n, n:], q[n:, :n], rho[:n, n:], rho[n:, :n])
    if any(np.any(b != 0) for b in zero):
        return False
    return np.linalg.norm(rho - adj(rho)) <= 1e-13 * max(1.0, np.linalg.norm(rho))


def _bmul(a, b):
    """Product of 2x2 block matrices whose blocks are arrays or None (structural zero)."""
    out = [[None, None], [None, None]]
    for i in range(2):
        for j in range(2):
            acc = None
            for k in range(2):
                if a[i][k] is not None and b[k][j] is not None:
                    term = a[i][k] @ b[k][j]
                    acc = term if acc is None else acc + term
            out[i][j] = acc
    return out


def _badj(a):
    return [[None if a[j][i] is None else adj(a[j][i]) for j in range(2)] for i in range(2)]


def _blk(x, i, j):
    return 0.0 if x[i][j] is None else x[i][j]


class PackedZ2System:
    """The quartic system of a Z2-symmetric state on its structurally nonzero blocks: the
    seven-channel equations of QuarticSystem evaluated block by block (the reference writes the
    same blocks as ten (D/2)^2 channels with gathered adjoints, ode_backend.py:236-473). An odd
    channel [[0, U], [U^dag, 0]] is carried by U, an even one by its two diagonal blocks, so the
    state vector and the DOP853 error norm have 10 (D/2)^2 + 1 entries. The scalar is
    4 src Re tr(R F3 + F3 R^dag) = 8 src Re(tr(a U^dag) + tr(b U)) for F3 = [[0, U], [U^dag, 0]]
    and R = [[0, a], [b, 0]]."""

    def __init__(self, q, r, rho):
        q, r, rho = (np.asarray(x, dtype=np.complex128) for x in (q, r, rho))
        if not z2_structure_ok(r, q, rho):
            raise ValueError("the packed Z2 route requires exact balanced block structure; nothing is projected")
        self.q, self.r, self.rho = q, r, rho
        self.full_d = len(q)
        n = self.full_d // 2
        self.n = n
        self.d = self.full_d
        self.size = 10 * n * n + 1
        qb = [[q[:n, :n], None], [None, q[n:, n:]]]
        rb = [[None, r[:n, n:]], [r[n:, :n], None]]
        self.a, self.b = r[:n, n:], r[n:, :n]
        self.ops = [(qb, rb) if c in FORWARD else (_badj(qb), _badj(rb)) for c in range(7)]
        # fixed_0 = R rho + rho R^dag and fixed_6 = 4 (R + R^dag), both odd: their upper blocks
        self.fixed = {0: [[None, self.a @ rho[n:, n:] + rho[:n, :n] @ adj(self.b)], [None, None]],
                      6: [[None, 4.0 * (self.a + adj(self.b))], [None, None]]}
        self.calls = 0

    def initial(self):
        return np.zeros(self.size, complex)

    def unpack_channels(self, y):
        """The seven channels as 2x2 block matrices (None = structural zero)."""
        n = self.n
        blocks = y[:-1].reshape(10, n, n)
        chans = []
        i = 0
        for c in range(7):
            if PARITY[c]:
                u = blocks[i]
                chans.append([[None, u], [adj(u), None]])
                i += 1
            else:
                chans.append([[blocks[i], None], [None, blocks[i + 1]]])
                i += 2
        return chans

    def unpack(self, y):
        """Packed vector -> the dense seven-channel vector of QuarticSystem (7 D^2 + 1)."""
        n, d = self.n, self.full_d
        out = np.zeros(7 * d * d + 1, complex)
        mats = out[:-1].reshape(7, d, d)
        for c, x in enumerate(self.unpack_channels(y)):
            for i in range(2):
                for j in range(2):
                    if x[i][j] is not None:
                        mats[c, i * n:(i + 1) * n, j * n:(j + 1) * n] = x[i][j]
        out[-1] = y[-1]
        return out

    def __call__(self, t, y, src=None):
        self.calls += 1
        n = self.n
        jac = 2.0 * abs(t)
        src = source(t) if src is None else src
        x = self.unpack_channels(y)
        out = np.empty_like(y)
        blocks = out[:-1].reshape(10, n, n)
        i = 0
        for c in range(7):
            qc, rc = self.ops[c]
            qch, rch = _badj(qc), _badj(rc)
            lin = [_bmul(qc, x[c]), _bmul(x[c], qch), _bmul(_bmul(rc, x[c]), rch)]
            ins = None
            if c in INSERTIONS:
                s, coef = INSERTIONS[c]
                ins = (coef, [_bmul(rc, x[s]), _bmul(x[s], rch)])
            for (bi, bj) in (((0, 1),) if PARITY[c] else ((0, 0), (1, 1))):
                v = jac * sum(_blk(m, bi, bj) for m in lin)
                if ins is not None:
                    v = v + (src * ins[0]) * sum(_blk(m, bi, bj) for m in ins[1])
                if c in self.fixed:
                    v = v + src * _blk(self.fixed[c], bi, bj)
                blocks[i] = v
                i += 1
        u = x[2][0][1]
        out[-1] = 8.0 * src * (np.trace(self.a @ adj(u)) + np.trace(self.b @ u)).real
        return out


# --------------------------------------------------------------------------- DOP853

def integrate(system, points, *, atol=1e-13, rtol=1e-12, initial_step=None, max_steps=1_000_000,
              trace=None):
    """Adaptive DOP853 from -a to a = points[-1] with order-7 dense output at `points`
    (ode_backend.py:500-586; controller persistent_trajectory_backend.py:92-131;
    interpolation :135-153). No accepted step crosses t = 0. The step controller:
      err = h e5 / sqrt((e5 + 0.01 e3) N), e5/e3 the squared scaled error norms,
      factor = min(10, 0.9 err^(-1/8)); reject if err > 1 (h *= max(0.2, factor));
      after a rejection the next accepted step may not grow (factor <= 1).
    Returns (samples [len(points), N], stats)."""
    a_mat, b, c, e3, e5, dmat = DOP.A, DOP.B, DOP.C, DOP.E3, DOP.E5, DOP.D
    ns = DOP.N_STAGES            # 12
    nx = DOP.N_STAGES_EXTENDED   # 16
    points = np.asarray(points, dtype=np.float64)
    end = float(points[-1])
    y = system.initial()
    n = y.size
    t = -end
    h = min(0.01 if initial_step is None else float(initial_step), 2.0 * end)
    f = system(t, y)
    k = np.empty((nx, n), complex)
    samples = np.empty((len(points), n), complex)
    nxt = accepted = rejected = attempts = dense_steps = 0
    after_reject = False
    while t < end:
        boundary = 0.0 if t < 0.0 else end
        h = min(h, boundary - t)
        if h <= 10.0 * abs(np.nextafter(t, math.inf) - t):
            raise OracleFailure(f"step underflow at t={t}, h={h}")
        if attempts >= max_steps:
            raise OracleFailure("max_steps exceeded")
        attempts += 1
        k[0] = f
        for s in range(1, ns + 1):
            w = b if s == ns else a_mat[s, :s]
            z = y + h * (w @ k[:len(w)])
            if s == ns:
                proposed = z
            k[s] = system(t + c[s] * h if s < ns else t + h, z)
        scale = atol + rtol * np.maximum(np.abs(y), np.abs(proposed))
        s5 = float(np.sum(np.abs((e5 @ k[:ns + 1]) / scale) ** 2))
        s3 = float(np.sum(np.abs((e3 @ k[:ns + 1]) / scale) ** 2))
        den = s5 + 0.01 * s3
        err = h * s5 / math.sqrt(den * n) if den > 0 else 0.0
        if not math.isfinite(err):
            raise OracleFailure("nonfinite error estimate")
        factor = min(10.0, 0.9 * err ** (-1.0 / 8.0)) if err > 0 else 10.0
        if trace is not None:
            trace.append((t, h, err))
        if err > 1.0:
            rejected += 1
            after_reject = True
            h *= max(0.2, factor)
            continue
        accepted += 1
        t_new = boundary if h == boundary - t else t + h
        first = nxt
        while nxt < len(points) and points[nxt] <= t_new:
            nxt += 1
        if nxt > first:
            dense_steps += 1
            for s in range(ns + 1, nx):
                z = y + h * (a_mat[s, :s] @ k[:s])
                k[s] = system(t + c[s] * h, z)
            delta = proposed - y
            coeff = [delta, h * f - delta, 2.0 * delta - h * (k[ns] + f)]
            coeff += [h * (dmat[row] @ k) for row in range(4)]
            for node in range(first, nxt):
                if points[node] == t_new:
                    samples[node] = proposed
                    continue
                x = (points[node] - t) / h
                acc = np.zeros(n, complex)
                for i, cf in enumerate(reversed(coeff)):
                    acc = (acc + cf) * (x if i % 2 == 0 else 1.0 - x)
                samples[node] = acc + y
        y, f, t = proposed, k[ns].copy(), t_new
        h *= min(1.0, factor) if after_reject else factor
        after_reject = False
    if nxt != len(points):
        raise OracleFailure("not every node was sampled")
    return samples, dict(attempts=attempts, accepted=accepted, rejected=rejected,
                         dense_steps=dense_steps, rhs_calls=system.calls)


def quartic_pullback(system, samples, points, weights):
    """Covector, environment and value of the quartic term from the samples
    (ode_backend.py:589-637 with the reduced interfaces; src/observables.jl:238-276).

    The monomial spec has forward channels f0 = rho, f1..f3, f4 = 0 and adjoint channels
    b0..b3, b4 = I; at node i the forward sample is paired with the adjoint sample of node
    n-1-i. With w_i = weights_i 2|t_i| and j_i = weights_i source(t_i):
        m  = sum_i w_i sum_k f_k (R^dag b_k - b_k R^dag) + sum_i j_i sum_k (k+1) f_k b_{k+1}
        nn = sum_i w_i sum_k (b_k R - R b_k) f_k + sum_i j_i sum_k (k+1) b_{k+1} f_k
    covector = (m + nn^dag)/2, environment = Herm(b0 at the endpoint), value = Re scalar(a)."""
    d, n = system.d, len(points)
    r, rho = system.r, system.rho
    rh = adj(r)
    mats = samples[:, :-1].reshape(len(samples), 7, d, d)
    eye = np.eye(d, dtype=complex)
    m = np.zeros((d, d), complex)
    nn = np.zeros((d, d), complex)
    for i in range(n):
        fw = [rho, mats[i, 0], mats[i, 1], mats[i, 2]]
        bw = [mats[n - 1 - i, 3], mats[n - 1 - i, 4], mats[n - 1 - i, 5], mats[n - 1 - i, 6], eye]
        wi = weights[i] * 2.0 * abs(points[i])
        ji = weights[i] * source(points[i])
        for kk in range(4):
            f, bk = fw[kk], bw[kk]
            m += wi * (f @ rh @ bk - f @ bk @ rh)
            nn += wi * (bk @ r @ f - r @ bk @ f)
            m += (ji * (kk + 1)) * (f @ bw[kk + 1])
            nn += (ji * (kk + 1)) * (bw[kk + 1] @ f)
    covector = (m + adj(nn)) / 2.0
    env = mats[-1, 3]
    return float(samples[-1, -1].real), covector, (env + adj(env)) / 2.0


def evaluate_quartic(r, q, rho, g=1.0, *, half_window=30.0, n_quad=512, atol=1e-13, rtol=1e-12,
                     max_steps=1_000_000, return_samples=False, packed_z2=False):
    """g times (value, covector, environment) of the quartic term
    (persistent_trajectory_backend.py:439-461, ode_backend.py:861-870). packed_z2: integrate
    the packed Z2 system (ValueError unless the state has the exact Z2 block structure) and
    pull back from its unpacked samples (ode_backend.py:700-716); the samples returned are
    then the packed ones."""
    system = PackedZ2System(q, r, rho) if packed_z2 else QuarticSystem(q, r, rho)
    points, weights = quadrature(half_window, n_quad)
    nodes = np.r_[points, math.sqrt(half_window)]
    samples, stats = integrate(system, nodes, atol=atol, rtol=rtol, max_steps=max_steps)
    if packed_z2:
        dense = np.stack([system.unpack(x) for x in samples])
        value, cov, env = quartic_pullback(system, dense, points, weights)
    else:
        value, cov, env = quartic_pullback(system, samples, points, weights)
    out = dict(value=g * value, covector=g * cov, environment=g * env, stats=stats)
    if return_samples:
        out["samples"] = samples
    return out


# --------------------------------------------------------------------------- full ODE route

# Channel specs of the all-ODE evaluation (ode_backend.py:60-73, 851-858; Julia's default
# kinetic_backend=:ode, src/observables.jl:131-159): (channels, edges, commutator) with edges
# (source, destination, side, coefficient), side "L" a left insertion O X, "R" a right one X O^dag.
_SQRT2 = math.sqrt(2.0)
KINETIC_EDGES = ((0, 1, "L", _SQRT2), (0, 2, "R", _SQRT2), (2, 3, "L", _SQRT2), (1, 3, "R", _SQRT2))
QUARTIC_EDGES = tuple((k, k + 1, side, float(k + 1)) for k in range(4) for side in ("L", "R"))
FULL_SPECS = ((4, KINETIC_EDGES, False), (4, KINETIC_EDGES, True), (5, QUARTIC_EDGES, False))


class FullSystem:
    """The 26 D x D channels of kinetic1 + kinetic2 + phi^4 as ODEs (ode_backend.py:76-167).

    Forward channels 0..12 (specs at offsets 0, 4, 8), adjoint channels 13..25. Channel k has
    (ql, rl, ol) = (Q, R, O) forward or (Q^dag, R^dag, O^dag) adjoint, O = R or the commutator
    [Q, R] of its spec, and
        dX_k/dt = jac (ql X_k + X_k ql^dag + rl X_k rl^dag)
                  + src (sum_{left (a, c)} c ol_a X_a + sum_{right (b, c)} c X_b ol_b^dag).
    A forward edge a -> b (side, c) inserts into forward b; its trace dual inserts adjoint b
    into adjoint a on the other side (ode_backend.py:108-113). Initial values: rho in each
    spec's first forward channel, I in its last adjoint channel, zero elsewhere."""

    def __init__(self, q, r, rho, specs=FULL_SPECS):
        self.q, self.r, self.rho = (np.asarray(x, dtype=np.complex128) for x in (q, r, rho))
        self.d = d = len(self.q)
        self.specs = specs
        self.offsets = list(np.cumsum([0] + [sp[0] for sp in specs])[:-1])
        self.half = half = sum(sp[0] for sp in specs)
        self.channels = 2 * half
        self.size = self.channels * d * d
        comm = self.q @ self.r - self.r @ self.q
        self.ops = [None] * self.channels
        self.left = [[] for _ in range(self.channels)]
        self.right = [[] for _ in range(self.channels)]
        for off, (nch, edges, commutator) in zip(self.offsets, specs):
            op = comm if commutator else self.r
            for i in range(nch):
                self.ops[off + i] = (self.q, self.r, op)
                self.ops[half + off + i] = (adj(self.q), adj(self.r), adj(op))
            for src, dst, side, coef in edges:
                (self.left if side == "L" else self.right)[off + dst].append((off + src, coef))
                (self.right if side == "L" else self.left)[half + off + src].append((half + off + dst, coef))
        self.calls = 0

    def initial(self):
        d = self.d
        y = np.zeros((self.channels, d, d), complex)
        for off, (nch, _, _) in zip(self.offsets, self.specs):
            y[off] = self.rho
            y[self.half + off + nch - 1] = np.eye(d)
        return y.reshape(-1)

    def __call__(self, t, y, src=None):
        self.calls += 1
        d = self.d
        jac = 2.0 * abs(t)
        src = source(t) if src is None else src
        x = y.reshape(self.channels, d, d)
        out = np.empty_like(x)
        for k in range(self.channels):
            ql, rl, _ = self.ops[k]
            value = jac * (ql @ x[k] + x[k] @ adj(ql) + rl @ x[k] @ adj(rl))
            for a, coef in self.left[k]:
                value = value + (src * coef) * (self.ops[a][2] @ x[a])
            for b, coef in self.right[k]:
                value = value + (src * coef) * (x[b] @ adj(self.ops[b][2]))
            out[k] = value
        return out.reshape(-1)


def full_pullback(system, samples, points, weights, coefficients):
    """Value, covector and environment of every spec, summed with `coefficients`
    (ode_backend.py:589-619, 834-838; src/observables.jl:161-199). Per spec, with forward
    samples f_k at node i, adjoint samples b_k at node n-1-i, w_i = weights_i 2|t_i| and
    j_i = weights_i source(t_i):
        m  = sum_i w_i sum_k f_k (R^dag b_k - b_k R^dag),  nn = sum_i w_i sum_k (b_k R - R b_k) f_k,
        u  = sum_{left edges} c sum_i j_i f_src b_dst,     v  = sum_{right edges} c sum_i j_i b_dst f_src;
    a commutator spec adds u Q - Q u - R u R^dag + u R R^dag to m and
    Q^dag v - v Q^dag - R v R^dag + R R^dag v to nn, the others u and v;
    covector = (m + nn^dag)/2, environment = Herm(first adjoint channel at the endpoint),
    value = Re tr(last forward channel at the endpoint)."""
    d, n = system.d, len(points)
    q, r = system.q, system.r
    rh = adj(r)
    mats = samples.reshape(len(samples), system.channels, d, d)
    wi = np.asarray(weights) * 2.0 * np.abs(points)
    ji = np.asarray(weights) * np.array([source(t) for t in points])
    total_value, total_cov, total_env = 0.0, np.zeros((d, d), complex), np.zeros((d, d), complex)
    for coefficient, off, (nch, edges, commutator) in zip(coefficients, system.offsets, system.specs):
        f = mats[:n, off:off + nch]
        b = mats[n - 1::-1, system.half + off:system.half + off + nch]
        m = np.einsum("i,ikab,ikbc->ac", wi, f, rh @ b - b @ rh)
        nn = np.einsum("i,ikab,ikbc->ac", wi, b @ r - r @ b, f)
        u = np.zeros((d, d), complex)
        v = np.zeros((d, d), complex)
        for src, dst, side, coef in edges:
            if side == "L":
                u += coef * np.einsum("i,iab,ibc->ac", ji, f[:, src], b[:, dst])
            else:
                v += coef * np.einsum("i,iab,ibc->ac", ji, b[:, dst], f[:, src])
        if commutator:
            m += u @ q - q @ u - r @ u @ rh + u @ r @ rh
            nn += adj(q) @ v - v @ adj(q) - r @ v @ rh + r @ rh @ v
        else:
            m += u
            nn += v
        env = mats[-1, system.half + off]
        total_value += coefficient * float(np.trace(mats[-1, off + nch - 1]).real)
        total_cov += coefficient * (m + adj(nn)) / 2.0
        total_env += coefficient * (env + adj(env)) / 2.0
    return total_value, total_cov, total_env


# The first monomial's spec, phi_monomial(s, 1) of RcmpsCore (validate_sweep.py:23-32): forward
# F0 = rho, dF1 = 2|t| L(F1) dt + j(t) (R F0 + F0 R^dag) dt, with its adjoint channels.
PHI1_SPECS = ((2, ((0, 1, "L", 1.0), (0, 1, "R", 1.0)), False),)


def source_integral(half_window):
    """Integral of the source over x in [-W, W] (ode_backend.py:782-790): 2^-1/2, its integral
    over the line, minus twice the tail integral of K_{1/4}(x) x^{-1/4} beyond W, normalised by
    2^{9/4} sqrt(pi) Gamma(5/4)."""
    from scipy.integrate import quad
    if not half_window > 0:
        raise ValueError("positive half_window required")
    tail = quad(lambda x: kv(0.25, x) / x ** 0.25, half_window, np.inf, epsabs=0, epsrel=1e-12, limit=200)[0]
    return 2 ** -0.5 - 2.0 * tail / (2 ** 2.25 * math.sqrt(math.pi) * gamma(1.25))


def phi_expectation(r, rho, half_window):
    """<phi> on the window W in closed form (ode_backend.py:793-797): the first monomial's
    tr F1(a) = source_integral(W) tr(R rho + rho R^dag), since the Lindbladian preserves the
    trace."""
    r, rho = np.asarray(r), np.asarray(rho)
    return 2.0 * source_integral(half_window) * float(np.real(np.trace(rho @ r)))


def phi_by_ode(r, k, rho, *, half_window, n_quad, atol=1e-13, rtol=1e-12, max_steps=1_000_000):
    """<phi> as phi_monomial(s, 1) integrates it (validate_sweep.py:23-32): the four channels of
    PHI1_SPECS by DOP853 with dense output at the Gauss nodes; the value is Re tr F1 at the
    endpoint. Returns (value, stats)."""
    r, k, rho = (np.asarray(x, complex) for x in (r, k, rho))
    q = left_canonical_q(r, k)
    system = FullSystem(q, r, rho, specs=PHI1_SPECS)
    points, _ = quadrature(half_window, n_quad)
    samples, stats = integrate(system, np.r_[points, math.sqrt(half_window)], atol=atol, rtol=rtol,
                               max_steps=max_steps)
    d = len(r)
    end = samples[-1].reshape(system.channels, d, d)
    return float(np.trace(end[1]).real), stats


def evaluate_phi4(r, q, rho, g, *, half_window=20.0, n_quad=192, atol=1e-13, rtol=1e-12,
                  max_steps=1_000_000):
    """kinetic1 + kinetic2 + g phi^4 entirely by ODEs: value, raw covector, environment
    (ode_backend.py:851-858, the objective's --mode ode, sweep_driver.py:90-92)."""
    system = FullSystem(q, r, rho)
    points, weights = quadrature(half_window, n_quad)
    nodes = np.r_[points, math.sqrt(half_window)]
    samples, stats = integrate(system, nodes, atol=atol, rtol=rtol, max_steps=max_steps)
    value, cov, env = full_pullback(system, samples, points, weights, (1.0, 1.0, float(g)))
    return dict(value=value, covector=cov, environment=env, stats=stats)


# --------------------------------------------------------------------------- kinetic

def _vec(x):
    return x.reshape(-1)


def _mat(v, d):
    return v.reshape(d, d)


def _shifted_arnoldi(apply, rhs, shifts, d, *, tolerance, initialdim, maxdim):
    """Solve (I - c A) x = rhs for every shift c on one Arnoldi basis of A and rhs
    (kinetic_backend.py:302-336, 389-412, 438-496; src/kinetic_krylov.jl:113-156).

    Two-pass classical Gram-Schmidt; breakdown when the new norm is below 10 eps times the
    norm before projection. Projected solutions y_c = beta (I - c H_k)^-1 e1; their estimate
    max_c |c H[k, k-1] y_c[k-1]| / beta. Once it is below the tolerance (or the basis is
    terminal) the solutions are reconstructed and every true residual
    ||x - c A x - rhs|| / beta is checked; otherwise the basis doubles, up to maxdim."""
    n = d * d
    b = _vec(rhs)
    beta = float(np.linalg.norm(b))
    if beta == 0.0:
        return np.zeros((len(shifts), d, d), complex), dict(basis_size=0, residual=0.0)
    initialdim, maxdim = min(initialdim, n), min(maxdim, n)
    v = np.zeros((n, maxdim + 1), complex)
    hm = np.zeros((maxdim + 1, maxdim), complex)
    v[:, 0] = b / beta
    k, exhausted = 0, False
    eps = np.finfo(float).eps

    def extend(target):
        nonlocal k, exhausted
        for j in range(k, target):
            w = _vec(apply(_mat(v[:, j], d)))
            old = float(np.linalg.norm(w))
            basis = v[:, :j + 1]
            for _ in range(2):
                hcol = basis.conj().T @ w
                hm[:j + 1, j] += hcol
                w = w - basis @ hcol
            nrm = float(np.linalg.norm(w))
            hm[j + 1, j] = nrm
            k = j + 1
            if nrm <= 10.0 * eps * max(old, eps) or k == n:
                exhausted = True
                return
            v[:, j + 1] = w / nrm

    extend(initialdim)
    while True:
        e1 = np.zeros(k, complex)
        e1[0] = beta
        eye = np.eye(k)
        ys = np.stack([np.linalg.solve(eye - c * hm[:k, :k], e1) for c in shifts], axis=1)
        estimate = float(np.max(np.abs(shifts * hm[k, k - 1] * ys[k - 1]))) / beta
        terminal = exhausted or k == maxdim
        if estimate <= tolerance or terminal:
            xs = (v[:, :k] @ ys).T.reshape(len(shifts), d, d)
            worst = 0.0
            for i, c in enumerate(shifts):
                res = np.linalg.norm(xs[i] - c * apply(xs[i]) - rhs) / beta
                worst = max(worst, float(res))
            if worst <= tolerance:
                return xs, dict(basis_size=k, residual=worst)
            if exhausted:
                raise OracleFailure(f"Arnoldi exhausted at {k} with residual {worst}")
        if terminal:
            raise OracleFailure("shifted Arnoldi did not converge")
        extend(min(2 * k, maxdim))


def kinetic_raw(q, r, rho, nodes=512, *, tolerance=1e-12, initialdim=16, maxdim=1024):
    """Both infinite-line kinetic terms (unit coefficients) and their raw covector and
    environment (kinetic_backend.py:499-592; src/kinetic_krylov.jl:157-189).

    For op in (R, [Q,R]): X_c = (I - c L)^-1 (rho op^dag), A_c = (I - c L*)^-1 (op^dag),
    value = sum_c w_c Re tr(op X_c); with a_c = A_c^dag,
      m  = sum w c [X R^dag a - X a R^dag] (+ u or the [Q,R] pullback of u = sum w X)
      nn = sum w c [a R X - R a X]        (+ v or the [Q,R] pullback of v = sum w a rho)
      env = sum w op^dag a, covector += (m + nn^dag)/2, environment += Herm(env)."""
    q, r, rho = (np.asarray(x, dtype=np.complex128) for x in (q, r, rho))
    d = len(q)
    shifts, weights = angular_grid(nodes)
    rh = adj(r)
    value = 0.0
    covector = np.zeros((d, d), complex)
    environment = np.zeros((d, d), complex)
    info = {}
    for commutator in (False, True):
        op = q @ r - r @ q if commutator else r
        xs, sx = _shifted_arnoldi(lambda x: lindblad(q, r, x), rho @ adj(op), shifts, d,
                                  tolerance=tolerance, initialdim=initialdim, maxdim=maxdim)
        value += float(np.sum(weights * np.einsum("ij,nji->n", op, xs).real))
        aas, sa = _shifted_arnoldi(lambda x: lindblad_adjoint(q, r, x), adj(op), shifts, d,
                                   tolerance=tolerance, initialdim=initialdim, maxdim=maxdim)
        info[("commutator" if commutator else "R") + "_forward"] = sx
        info[("commutator" if commutator else "R") + "_adjoint"] = sa
        a = adj(aas)
        wz = (weights * shifts)[:, None, None]
        w = weights[:, None, None]
        m = np.sum(wz * (xs @ rh @ a - xs @ a @ rh), axis=0)
        nn = np.sum(wz * (a @ r @ xs - r @ a @ xs), axis=0)
        u = np.sum(w * xs, axis=0)
        v = np.sum(w * (a @ rho), axis=0)
        env = np.sum(w * (adj(op) @ a), axis=0)
        if commutator:
            m += u @ q - q @ u - r @ u @ rh + u @ r @ rh
            nn += adj(q) @ v - v @ adj(q) - r @ v @ rh + r @ rh @ v
        else:
            m += u
            nn += v
        covector += (m + adj(nn)) / 2.0
        environment += (env + adj(env)) / 2.0
    return dict(value=value, covector=covector, environment=environment, solves=info)


# --------------------------------------------------------------------------- rho0, boundary, metric

def _superop(f, d):
    """Dense D^2 x D^2 matrix of a linear map on D x D matrices (row-major vec)."""
    n = d * d
    out = np.empty((n, n), complex)
    for i in range(n):
        e = np.zeros(n, complex)
        e[i] = 1.0
        out[:, i] = _vec(f(_mat(e, d)))
    return out


def _solve(op, b, d, method, tolerance):
    """x with op(x) = b for a linear map op on D x D matrices: a dense LU of the D^2 x D^2
    matrix ("dense"), or restarted GMRES on its action ("krylov") for sizes where the dense
    matrix is too costly. The reference's GMRES (numerics.py:55-71) is right-preconditioned by
    the no-jump inverse; the oracle's is not: only the solution is compared, not the iterates."""
    if method == "dense":
        return _mat(np.linalg.solve(_superop(op, d), _vec(b)), d)
    if method != "krylov":
        raise ValueError(f"unknown method {method!r}")
    from scipy.sparse.linalg import LinearOperator, gmres
    n = d * d
    lin = LinearOperator((n, n), matvec=lambda v: _vec(op(_mat(np.asarray(v).ravel(), d))), dtype=np.complex128)
    x, info = gmres(lin, _vec(b), rtol=tolerance, atol=0.0, restart=min(64, n), maxiter=400)
    if info != 0:
        raise OracleFailure(f"GMRES did not converge (info={info})")
    return _mat(x, d)


def stationary_state(q, r, *, tolerance=1e-11, method="dense"):
    """Stationary density: L(rho) = 0, tr rho = 1, Hermitian, positive (numerics.py:74-100,
    src/transfer.jl:33-115). The oracle solves the same bordered equation
    -L(x) + tr(x) I / D = I / D (directly, or by GMRES with method="krylov"); the checks of
    checked_density follow."""
    q, r = np.asarray(q, complex), np.asarray(r, complex)
    d = len(q)
    eye = np.eye(d, dtype=complex)
    rho = _solve(lambda x: -lindblad(q, r, x) + np.trace(x) / d * eye, eye / d, d, method, tolerance)
    rho = rho / np.trace(rho)
    if np.linalg.norm(rho - adj(rho)) > 100 * tolerance:
        raise OracleFailure("stationary state is not Hermitian")
    rho = (rho + adj(rho)) / 2.0
    residual = float(np.linalg.norm(lindblad(q, r, rho)))
    scale = max(1.0, 2 * np.linalg.norm(q, 2) + np.linalg.norm(r, 2) ** 2)
    if residual > tolerance * scale or np.linalg.eigvalsh(rho).min() < -10 * tolerance:
        raise OracleFailure("invalid stationary density")
    return rho


def boundary_environment(q, r, rho, environment, *, method="dense"):
    """H with -L*(H) + tr(rho H) I = A - tr(rho A) I (numerics.py:103-117,
    src/transfer.jl:119-153), solved directly (or by GMRES with method="krylov")."""
    d = len(q)
    eye = np.eye(d, dtype=complex)
    b = environment - np.trace(rho @ environment) * eye
    return _solve(lambda x: -lindblad_adjoint(q, r, x) + np.trace(rho @ x) * eye, b, d, method, 1e-13)


class NoJumpInverse:
    """The no-jump inverse of the reference's preconditioner (numerics.py:40-53): with the complex
    Schur form Q = U T U^dag and T_s = T - (shift/2) I, y -> -U X U^dag where X solves the
    triangular Sylvester equation T_s X + X T_s^dag = U^dag y U (T_s^dag X + X T_s for the adjoint
    map). The shift is max(1, |Q|_2, |R|_2^2) when T has an eigenvalue with real part above
    -100 eps times that scale, else 0."""

    def __init__(self, q, r):
        from scipy.linalg import get_lapack_funcs, schur
        t, self.u = schur(np.asarray(q, complex), output="complex")
        scale = max(1.0, np.linalg.norm(q, 2), np.linalg.norm(r, 2) ** 2)
        self.shift = scale if np.real(np.diag(t)).max() >= -100 * np.finfo(float).eps * scale else 0.0
        self.t = np.asfortranarray(t - self.shift / 2 * np.eye(len(q)))
        self.trsyl = get_lapack_funcs("trsyl", (self.t,))

    def __call__(self, y, adjoint=False):
        c = np.asfortranarray(adj(self.u) @ y @ self.u)
        x, scale, info = self.trsyl(self.t, self.t, c, trana="C" if adjoint else "N",
                                    tranb="N" if adjoint else "C")
        if info < 0 or not np.isfinite(scale) or scale <= 0:
            raise OracleFailure(f"Sylvester inverse failed: info={info}, scale={scale}")
        return self.u @ (-x / scale) @ adj(self.u)


def boundary_environment_preconditioned(q, r, rho, environment, *, tolerance=1e-13):
    """The reference's boundary solve itself (numerics.py:55-71, 103-117): GMRES(min(40, D^2))
    with rtol = atol = tolerance on the column-major vectorization, right-preconditioned by the
    adjoint no-jump inverse with the Sherman-Morrison correction for the tr(rho x) I term.
    Returns (H, matvecs)."""
    from scipy.sparse.linalg import LinearOperator, gmres
    q, r, rho = (np.asarray(x, complex) for x in (q, r, rho))
    d = len(q)
    eye = np.eye(d, dtype=complex)
    b = environment - np.trace(rho @ environment) * eye
    inverse = NoJumpInverse(q, r)
    z = inverse(eye, adjoint=True)
    den = 1.0 + np.trace(rho @ z)

    def pre(y):
        x = inverse(y, adjoint=True)
        return x - np.trace(rho @ x) / den * z

    def op(x):
        return -lindblad_adjoint(q, r, x) + np.trace(rho @ x) * eye

    count = [0]

    def matvec(v):
        count[0] += 1
        return op(pre(np.asarray(v).reshape((d, d), order="F"))).reshape(-1, order="F")

    lin = LinearOperator((d * d, d * d), matvec=matvec, dtype=np.complex128)
    y, info = gmres(lin, b.reshape(-1, order="F"), rtol=tolerance, atol=tolerance, restart=min(40, d * d),
                    maxiter=200)
    h = pre(y.reshape((d, d), order="F"))
    residual = np.linalg.norm(op(h) - b)
    if info != 0 or not np.isfinite(residual) or residual > 20 * tolerance * max(1.0, np.linalg.norm(b)):
        raise OracleFailure(f"preconditioned boundary GMRES failed: info={info}, residual={residual:.3e}")
    return h, count[0]


def finish_gradient(q, r, rho, covector, environment, *, metric_reg=1e-3, method="dense"):
    """gradient = ((rho + reg I)^-1 (covector + rho R^dag H - rho H R^dag))^dag
    (numerics.py:120-126, src/observables.jl:278-289). method "preconditioned" solves for H as
    the reference does (boundary_environment_preconditioned)."""
    if method == "preconditioned":
        h, _ = boundary_environment_preconditioned(q, r, rho, environment)
    else:
        h = boundary_environment(q, r, rho, environment, method=method)
    c = covector + rho @ adj(r) @ h - rho @ h @ adj(r)
    return adj(np.linalg.solve(rho + metric_reg * np.eye(len(r)), c))


def metric(rho, x, y, metric_reg=1e-3):
    """<x, y> = 2 Re tr(x^dag y (rho + reg I)) (numerics.py:129-130)."""
    return float(2.0 * np.vdot(x, y @ (rho + metric_reg * np.eye(len(rho)))).real)


def fg_phi4(r, k, rho, g, *, half_window=30.0, n_quad=512, atol=1e-13, rtol=1e-12, nodes=512,
            krylov_tolerance=1e-12, maxdim=1024, metric_reg=1e-3, method="dense", packed_z2=False):
    """(energy, gradient, parts) of the phi^4 density: kinetic1 + kinetic2 + g phi^4, the
    sum computed by the reference's GPU objective (overlap_sweep_driver.py:132-212,
    sweep_driver.py:78-119; src/observables.jl:332-334). packed_z2 selects the packed Z2
    quartic route (sweep_driver.py:48-50, 100-101)."""
    r, k, rho = (np.asarray(x, complex) for x in (r, k, rho))
    q = left_canonical_q(r, k)
    quartic = evaluate_quartic(r, q, rho, g, half_window=half_window, n_quad=n_quad, atol=atol, rtol=rtol,
                               packed_z2=packed_z2)
    kinetic = kinetic_raw(q, r, rho, nodes, tolerance=krylov_tolerance, maxdim=maxdim)
    covector = quartic["covector"] + kinetic["covector"]
    environment = quartic["environment"] + kinetic["environment"]
    energy = quartic["value"] + kinetic["value"]
    gradient = finish_gradient(q, r, rho, covector, environment, metric_reg=metric_reg, method=method)
    return energy, gradient, dict(quartic=quartic, kinetic=kinetic, covector=covector,
                                  environment=environment)

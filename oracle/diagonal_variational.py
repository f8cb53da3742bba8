"""Diagonal variational boundary MPS for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/contraction/diagonal_variational.jl``
(``BoundaryMPSDiagonalVariational``): a diagonal layer is absorbed by a
two-site variational fit of the candidate frontier MPS C to the target chain
of raw site blocks (normalised so that the target has unit norm), starting
from the previous boundary (frontier edges matched by their transverse
coordinate, vanished end edges capped with the identity, new ones added as
identity products, physical legs mapped onto the new spaces).  Sweeps run
both ways; the fit keeps the candidate of least residual |C - T|^2, stops at
``max_sweep`` or when C's squared norm changes by at most
``threshold_sweep``, and falls back to the SVD absorption of
``BoundaryMPSDiagonal`` on a numerical failure when that fits better.

The reference factors cross-block two-site projections through the target
bond for a cheaper SVD (``_variational_small_svd``) and checks that the
factored SVD keeps the same space, else it takes the full SVD; the oracle
takes the full two-site SVD everywhere (the same kept space and singular
values).  The target-block cache (``target_cache_bytes``) only saves work and
is not restated, and of the Schmidt entropies only the maximum is kept (the
reference also lists them per cut, ``northwest_cuts`` / ``southeast_cuts``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import z2
from . import diagonal as dg
from .diagonal import LT, join, reorder, unit_lt
from .variational import VariationalNumericalError, summary, space_map
from .z2 import T, norm

EPS = np.finfo(np.float64).eps
FLOATMIN = np.finfo(np.float64).tiny


@dataclass
class BoundaryMPSDiagonalVariational:
    """``BoundaryMPSDiagonalVariational(chi; sector_space, max_sweep,
    threshold_sweep, target_cache_bytes)`` (diagonal_variational.jl:12-30)."""
    chi: int
    space: tuple | None = None
    max_sweep: int = 4
    threshold_sweep: float = 1e-8
    target_cache_bytes: int = 256 * 1024 ** 2
    variational = True

    def __post_init__(self):
        if self.chi < 1:
            raise ValueError("chi must be positive")
        if self.max_sweep < 1:
            raise ValueError("max_sweep must be positive")
        if not (math.isfinite(self.threshold_sweep) and self.threshold_sweep >= 0):
            raise ValueError("threshold_sweep must be finite and nonnegative")
        if self.target_cache_bytes < 0:
            raise ValueError("target_cache_bytes must be nonnegative")


def coordinate(edge):
    """``_diagonal_coordinate`` (diagonal_variational.jl:52-60): twice the
    transverse coordinate x - y of the edge's midpoint."""
    kind, x, y = edge
    return 2 * x - 1 - 2 * y if kind == "h" else 2 * x - 2 * y + 1


def identity_leg(p) -> T:
    """``_variational_identity`` of a single-layer leg with parities p, on its
    fused (ket, bra) leg."""
    d = len(p)
    v = np.zeros(d * d)
    v[np.arange(d) * d + np.arange(d)] = 1.0 / math.sqrt(d)
    return T(v, [z2.fused_parity([p, p])])


def _msg(t, log_scale=0.0):
    """``_variational_message`` of a labelled tensor."""
    if not isinstance(t.t, T):
        s = abs(t.t)
    else:
        s = norm(t.t)
    if not math.isfinite(s):
        raise VariationalNumericalError("nonfinite_overlap")
    if s == 0:
        return t, -math.inf
    return LT(t.t / s, t.labels), log_scale + math.log(s)


class _Target:
    """``_DiagonalLayerTarget`` (diagonal_variational.jl:96-217): the layer's
    raw blocks in frontier order, each divided by its norm and by the chain's
    norm shared equally, so that the target has unit norm."""

    def __init__(self, inp: dg.DiagonalBoundary, site_tensor, Lx, Ly, t, reverse):
        L = dg.layer_layout(inp, Lx, Ly, t, reverse)
        self.input, self.Lx, self.Ly, self.t, self.reverse = inp, Lx, Ly, t, reverse
        self.sites, self.inputs, self.outputs, self.ranges, self.edges = (
            L["sites"], L["inputs"], L["outputs"], L["ranges"], L["edges"])
        self.site_tensor = site_tensor
        self.tensors = [site_tensor(s) for s in self.sites]
        self.owner, self.physical, self.identities = [], [], []
        for j, site in enumerate(self.sites):
            ports = dg.ports_of(site)
            A = self.tensors[j]
            for port in self.outputs[j]:
                axis = dg.VIRTUAL_AXES[ports.index(port)]
                self.owner.append(j)
                self.physical.append(z2.fused_parity([A.p[axis], A.p[axis]]))
                self.identities.append(identity_leg(A.p[axis]))
        raw = [dg.raw_block(inp, A, Lx, Ly, s, self.inputs[j], self.outputs[j], reverse)
               for j, (s, A) in enumerate(zip(self.sites, self.tensors))]
        self.norms = [norm(B) for B in raw]
        if not all(math.isfinite(n) for n in self.norms):
            raise RuntimeError("nonfinite variational target block")
        self.blocks = [B if n == 0 else B / n for B, n in zip(raw, self.norms)]
        self.log_scale = inp.log_scale
        self.weight = 1.0
        if any(n == 0 for n in self.norms):
            self.log_scale = -math.inf
        elif self.edges:
            ln = _chain_lognorm(self.blocks)
            self.log_scale += sum(math.log(n) for n in self.norms) + ln
            self.weight = math.exp(-ln / len(self.blocks)) if math.isfinite(ln) else 1.0
            self.blocks = [B * self.weight for B in self.blocks]
        else:
            self.log_scale += sum(math.log(n) for n in self.norms)

    def labelled_block(self, j):
        return LT(self.blocks[j], [("tb", j)] + list(self.outputs[j]) + [("tb", j + 1)])

    def edge(self, C, left):
        """``_variational_edge``: unit target and candidate bonds at one end."""
        j = 0 if left else len(self.sites)
        i = 0 if left else len(C.tensors)
        return _msg(join(unit_lt(("tb", j)), unit_lt(("cb", i))))

    def step(self, m, i, A, left):
        """``_variational_step``: a block joins at its first (last) output, then
        the candidate tensor i."""
        E, ls = m
        j = self.owner[i]
        rng = self.ranges[j]
        if i == (rng[0] if left else rng[-1]):
            E = join(E, self.labelled_block(j))
        E = join(E, LT(A, [("cb", i), self.edges[i], ("cb", i + 1)]))
        return _msg(E, ls)

    def messages(self, C, left):
        n = len(C.tensors)
        out = [None] * (n + 1)
        if left:
            out[0] = self.edge(C, True)
            for i in range(n):
                out[i + 1] = self.step(out[i], i, C.tensors[i], True)
        else:
            out[n] = self.edge(C, False)
            for i in range(n - 1, -1, -1):
                out[i] = self.step(out[i + 1], i, C.tensors[i], False)
        return out

    def pair(self, i, L, R) -> T:
        """``_variational_pair``: the two-site projection (cb_i, e_i, e_i+1, cb_i+2)."""
        E = L[0]
        for j in sorted(set(self.owner[i:i + 2])):
            rng = self.ranges[j]
            if rng[0] >= i and rng[-1] <= i + 1:
                E = join(E, self.labelled_block(j))
        E = join(E, R[0])
        out = reorder(E, [("cb", i), self.edges[i], self.edges[i + 1], ("cb", i + 2)]).t
        return out * math.exp(L[1] + R[1])


def _chain_lognorm(blocks):
    """``_variational_chain_lognorm``: log of the norm of the chain of blocks,
    through QR with the factor carried on normalised."""
    carry = None
    total = 0.0
    for A in blocks:
        if carry is not None:
            A = z2.matmul_view(carry, [0], [1], A, [0], list(range(1, A.ndim)))
        _, R = z2.qr(A, list(range(A.ndim - 1)), [A.ndim - 1])
        s = norm(R)
        if not math.isfinite(s):
            raise VariationalNumericalError("nonfinite_norm")
        if s == 0:
            return -math.inf
        total += math.log(s)
        carry = R / s
    return total


def _product(t: _Target):
    """``_variational_product``: identity vectors on every output edge."""
    tensors = [T(v.a.reshape(1, -1, 1), [z2.leg(1, 0), v.p[0], z2.leg(1, 0)]) for v in t.identities]
    return dg.DiagonalBoundary(tensors, list(t.edges), 0, 0.0, 0.0, 1.0)


def _move_center(C, target):
    """``_diagonal_center!``."""
    B = C.tensors
    while C.center < target:
        i = C.center
        Q, R = z2.qr(B[i], [0, 1], [2])
        B[i] = Q
        B[i + 1] = z2.einsum("lk,kpr->lpr", R, B[i + 1])
        C.center += 1
    while C.center > target:
        i = C.center
        L, Q = z2.lq(B[i], [0], [1, 2])
        B[i] = Q
        B[i - 1] = z2.einsum("lpk,kr->lpr", B[i - 1], L)
        C.center -= 1


def _input_identity(t: _Target, edge):
    """``_variational_input_identity``: the identity on the input edge's leg."""
    for j, site in enumerate(t.sites):
        ports = dg.ports_of(site)
        if edge in ports:
            return identity_leg(t.tensors[j].p[dg.VIRTUAL_AXES[ports.index(edge)]])
    raise RuntimeError("input edge missing from variational layer")


def _warm_start(t: _Target):
    """``_variational_warm_start`` (diagonal_variational.jl:238-301)."""
    old = t.input
    if not old.tensors:
        return _product(t)
    C = dg.DiagonalBoundary(list(old.tensors), list(old.edges), max(old.center, 0), 0.0, 0.0, old.scalar)
    coords = [coordinate(e) for e in t.edges]
    oldc = [coordinate(e) for e in C.edges]
    # an end edge that leaves the frontier is capped with the identity
    while C.tensors and oldc[0] not in coords:
        _move_center(C, 0)
        A = C.tensors[0]
        h = z2.einsum("lpr,p->r", A, _input_identity(t, C.edges[0]))
        C.tensors.pop(0)
        C.edges.pop(0)
        oldc.pop(0)
        if not C.tensors:
            break
        nxt = C.tensors[0]
        C.tensors[0] = T(np.einsum("r,rps->ps", h.a, nxt.a)[None], [z2.leg(1, 0), nxt.p[1], nxt.p[2]])
        C.center = 0
    while C.tensors and oldc[-1] not in coords:
        _move_center(C, len(C.tensors) - 1)
        A = C.tensors[-1]
        h = z2.einsum("lpr,p->l", A, _input_identity(t, C.edges[-1]))
        C.tensors.pop()
        C.edges.pop()
        oldc.pop()
        if not C.tensors:
            break
        prv = C.tensors[-1]
        C.tensors[-1] = T(np.einsum("lpr,r->lp", prv.a, h.a)[:, :, None], [prv.p[0], prv.p[1], z2.leg(1, 0)])
        C.center = len(C.tensors) - 1
    if not C.tensors:
        return _product(t)
    # physical maps at their centres: embeddings keep the canonical form,
    # projections first move the centre there
    for i in range(len(C.tensors)):
        j = coords.index(oldc[i])
        P, Q = C.tensors[i].p[1], t.physical[j]
        if np.array_equal(P, Q):
            continue
        if any(np.sum(P == c) > np.sum(Q == c) for c in (0, 1)):
            _move_center(C, i)
        A = C.tensors[i]
        C.tensors[i] = T(np.einsum("qp,lpr->lqr", space_map(P, Q), A.a), [A.p[0], Q, A.p[2]])
    product = _product(t)
    while oldc[0] > coords[0]:
        j = coords.index(oldc[0]) - 1
        C.tensors.insert(0, product.tensors[j])
        oldc.insert(0, coords[j])
        C.center += 1
    while oldc[-1] < coords[-1]:
        j = coords.index(oldc[-1]) + 1
        C.tensors.append(product.tensors[j])
        oldc.append(coords[j])
    C.edges = list(t.edges)
    s = norm(C.tensors[C.center])
    if s == 0:
        return product
    if not math.isfinite(s):
        raise RuntimeError("nonfinite variational warm start")
    C.tensors[C.center] = C.tensors[C.center] / s
    return C


def _nonnegative_residual(value, scale=1.0):
    if not math.isfinite(value):
        raise VariationalNumericalError("nonfinite_residual")
    if not value >= -512 * EPS * max(1.0, scale):
        raise VariationalNumericalError("negative_residual")
    return max(0.0, value)


def _projected_residual(norm2):
    if not (math.isfinite(norm2) and norm2 >= 0):
        raise VariationalNumericalError("nonfinite_norm")
    return _nonnegative_residual(1 - norm2, norm2)


def _overlap_residual(t: _Target, C, left=True, terminal=None):
    """``_variational_overlap_residual``: |C - T|^2 with |T| = 1."""
    if terminal is None:
        terminal = t.edge(C, left)
        order = range(len(C.tensors)) if left else range(len(C.tensors) - 1, -1, -1)
        for i in order:
            terminal = t.step(terminal, i, C.tensors[i], left)
    edge = t.edge(C, not left)
    overlap = dg.scalar(join(terminal[0], edge[0])) * math.exp(terminal[1] + edge[1])
    norm2 = norm(C.tensors[C.center]) ** 2
    if not (math.isfinite(overlap) and math.isfinite(norm2)):
        raise VariationalNumericalError("nonfinite_overlap")
    return _nonnegative_residual(1 + norm2 - 2 * overlap, max(norm2, 2 * abs(overlap)))


def _half_sweep(C, t: _Target, method, right, entropy, profile, fixed):
    """``_variational_half_sweep!`` (diagonal_variational.jl:470-499)."""
    n = len(C.tensors)
    rolling = t.edge(C, right)
    nextfixed = [None] * (n + 1)
    nextfixed[0 if right else n] = rolling
    maxdiscard = 0.0
    last = None
    for i in (range(n - 1) if right else range(n - 2, -1, -1)):
        L = rolling if right else fixed[i]
        R = fixed[i + 2] if right else rolling
        M = t.pair(i, L, R)
        U, S, V, err, ent = z2.svd_trunc(M, [0, 1], [2, 3], chi=method.chi, space=method.space,
                                         entropy=entropy is not None)
        if entropy is not None:
            entropy.maximum = max(entropy.maximum, ent)
            profile[i] = ent
        magnitude = norm(M)
        if magnitude == 0:
            raise VariationalNumericalError("zero_local_projection")
        last = np.concatenate(S)
        maxdiscard = max(maxdiscard, (err / magnitude) ** 2)
        if right:
            C.tensors[i] = U
            C.tensors[i + 1] = T(V.a * last[:, None, None], V.p)
        else:
            C.tensors[i] = T(U.a * last[None, None, :], U.p)
            C.tensors[i + 1] = V
        C.center = i + 1 if right else i
        k = i if right else i + 1
        rolling = t.step(rolling, k, C.tensors[k], right)
        nextfixed[k + 1 if right else k] = rolling
    norm2 = float(np.sum(last * last))
    if norm2 == 0:
        raise VariationalNumericalError("zero_local_projection")
    return maxdiscard, nextfixed, norm2


def _copy(C):
    return dg.DiagonalBoundary(list(C.tensors), list(C.edges), C.center, C.log_scale, C.max_truncation, C.scalar)


def _fit(t: _Target, method, entropy):
    """``_variational_fit`` (diagonal_variational.jl:501-539)."""
    C = _warm_start(t)
    n = len(C.tensors)
    right = C.center < n - 1 - C.center or (C.center == n - 1 - C.center and not t.reverse)
    _move_center(C, 0 if right else n - 1)
    fixed = t.messages(C, not right)
    initial = _overlap_residual(t, C, left=not right, terminal=fixed[0 if right else n])
    best, cost = _copy(C), initial
    bestprofile = [math.nan] * max(0, n - 1)
    relative_change, discard, sweeps, reason, fallback = math.inf, 0.0, 0, "sweep_limit", None
    previous = math.nan
    for sweep in range(1, method.max_sweep + 1):
        profile = [math.nan] * (n - 1)
        sweeps = sweep
        current = math.inf
        try:
            d1, fixed, _ = _half_sweep(C, t, method, right, entropy, profile, fixed)
            d2, fixed, norm2 = _half_sweep(C, t, method, not right, entropy, profile, fixed)
            discard = max(discard, d1, d2)
            current = _projected_residual(norm2)
            if not current <= cost + 512 * EPS * max(1.0, cost):
                raise VariationalNumericalError("residual_increase")
            relative_change = math.inf if sweep == 1 else abs(norm2 - previous) / max(norm2, previous, FLOATMIN)
            previous = norm2
        except (VariationalNumericalError, np.linalg.LinAlgError) as ex:
            fallback = dict(reason=ex.reason if isinstance(ex, VariationalNumericalError)
                            else "factorization_failure", used_svd=False)
            reason = "numerical_fallback"
            break
        if current <= cost:
            best, cost, bestprofile = _copy(C), current, list(profile)
        if sweep > 1 and method.threshold_sweep > 0 and relative_change <= method.threshold_sweep:
            reason = "threshold_sweep"
            break
    return best, dict(sweeps=sweeps, relative_change=relative_change, stop_reason=reason, initial_residual=initial,
                      residual=cost, max_local_discarded_weight=discard, fallback=fallback), bestprofile


def _recover(t: _Target, method, C, report, profile):
    """``_variational_recover``: the SVD absorption of the same layer when it
    fits better."""
    alternate = t.input.copy()
    alternate.max_truncation = 0.0
    dg.absorb_layer(alternate, t.site_tensor, t.Lx, t.Ly, t.t, dg.BoundaryMPSDiagonal(method.chi, method.space),
                    reverse=t.reverse)
    alternate.tensors[alternate.center] = alternate.tensors[alternate.center] * \
        math.exp(alternate.log_scale - t.log_scale)
    cost = _overlap_residual(t, alternate)
    if not math.isfinite(cost):
        raise VariationalNumericalError("failed_svd_fallback")
    use_svd = C is None or cost < report["residual"]
    if use_svd:
        C = alternate
        profile = [math.nan] * (len(C.tensors) - 1)
    report = dict(report, residual=cost if use_svd else report["residual"],
                  max_local_discarded_weight=max(report["max_local_discarded_weight"], alternate.max_truncation),
                  fallback=dict(report["fallback"], used_svd=use_svd))
    return C, report, profile


def absorb_layer_variational(env: dg.DiagonalBoundary, site_tensor, Lx, Ly, t, method, reverse=False,
                             entropy=None):
    """``_diagonal_absorb_layer!`` for the variational method
    (diagonal_variational.jl:561-614).  Modifies and returns ``env``."""
    tg = _Target(env, site_tensor, Lx, Ly, t, reverse)
    n = len(tg.edges)
    profile = [math.nan] * max(0, n - 1)
    report = dict(sweeps=0, relative_change=0.0, stop_reason="direct", initial_residual=0.0, residual=0.0,
                  max_local_discarded_weight=0.0, fallback=None)
    if tg.log_scale == -math.inf:
        if n == 0:
            C = dg.DiagonalBoundary(scalar=0.0)
        else:
            C = _product(tg)
            C.tensors[C.center] = C.tensors[C.center] * 0.0
        report.update(stop_reason="zero_target", residual=math.nan, initial_residual=math.nan)
    elif n <= 1:
        H = tg.blocks[0]
        if n == 0:
            C = dg.DiagonalBoundary(scalar=float(H.a.reshape(-1)[0]))
        else:
            C = dg.DiagonalBoundary([H], list(tg.edges), 0, 0.0, 0.0, 1.0)
    elif len(tg.sites) == 1:
        H = tg.blocks[0]
        U, S, V, err, ent = z2.svd_trunc(H, [0, 1], [2, 3], chi=method.chi, space=method.space,
                                         entropy=entropy is not None)
        if entropy is not None:
            entropy.maximum = max(entropy.maximum, ent)
            profile[0] = ent
        s = np.concatenate(S)
        C = dg.DiagonalBoundary([U, T(V.a * s[:, None, None], V.p)], list(tg.edges), 1, 0.0, 0.0, 1.0)
        report.update(residual=err * err, max_local_discarded_weight=err * err)
    else:
        try:
            C, report, profile = _fit(tg, method, entropy)
        except (VariationalNumericalError, np.linalg.LinAlgError) as ex:
            C = None
            report.update(stop_reason="numerical_fallback", initial_residual=math.nan, residual=math.inf,
                          fallback=dict(reason=ex.reason if isinstance(ex, VariationalNumericalError)
                                        else "factorization_failure", used_svd=False))
        if report["fallback"] is not None:
            C, report, profile = _recover(tg, method, C, report, profile)
    scale = 1.0 if n == 0 else norm(C.tensors[C.center])
    if not math.isfinite(scale):
        raise RuntimeError("nonfinite variational boundary norm")
    if n > 0 and scale != 0:
        C.tensors[C.center] = C.tensors[C.center] / scale
    env.tensors, env.edges, env.center, env.scalar = C.tensors, C.edges, C.center, C.scalar
    env.log_scale = -math.inf if scale == 0 else tg.log_scale + math.log(scale)
    if not math.isnan(report["residual"]):
        env.max_truncation = max(env.max_truncation, report["residual"])
    env.variational = list(env.variational) + [dict(report, layer=t, reverse=reverse)]
    return env

"""Row variational boundary MPS for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/contraction/row_variational.jl`` (``BoundaryMPSRowVariational``)
with the helpers it takes from ``src/contraction/diagonal_variational.jl``
(``_VariationalNumericalError``, ``_variational_message``,
``_variational_identity``, ``_variational_space_map``,
``_variational_summary``).  A row is absorbed by a two-site variational fit
of the truncated candidate MPS C to the target T = (input boundary) x (row):
the candidate starts from the input boundary with its physical legs mapped
onto the row's output legs, each two-site update is the normalised
projection of T onto C's environment split by a truncated SVD, and sweeps
(left to right, then back) stop at ``max_sweep`` or when the squared norm
changes by at most ``threshold_sweep``.  The amplitude of C stays in a log
scale; the best admissible candidate is kept.

The reference keeps each row site as separate ket and bra factors
(``FactorizedRowSite``, ``src/contraction/row_factorized.jl``); here a row
site is its fused double layer (w, n, e, s), the same tensor, so the row
steps, environments, sampling and full update of ``boundary.py`` serve the
variational method unchanged and only the absorption differs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import z2
from .z2 import T, einsum, norm

EPS = np.finfo(np.float64).eps
FLOATMIN = np.finfo(np.float64).tiny


@dataclass
class BoundaryMPSRowVariational:
    """``BoundaryMPSRowVariational(chi; sector_space, max_sweep, threshold_sweep)``
    (row_variational.jl:10-25)."""
    chi: int
    space: tuple | None = None
    max_sweep: int = 4
    threshold_sweep: float = 1e-8
    zipup = False
    variational = True

    def __post_init__(self):
        if self.chi < 1:
            raise ValueError("chi must be positive")
        if self.max_sweep < 1:
            raise ValueError("max_sweep must be positive")
        if not (math.isfinite(self.threshold_sweep) and self.threshold_sweep >= 0):
            raise ValueError("threshold_sweep must be finite and nonnegative")


class VariationalNumericalError(RuntimeError):
    """``_VariationalNumericalError`` (diagonal_variational.jl:32-37)."""

    def __init__(self, reason):
        super().__init__("variational boundary: " + reason)
        self.reason = reason


def summary(records):
    """``_variational_summary`` (diagonal_variational.jl:40-46)."""
    return dict(layers=list(records), max_sweeps=max([r["sweeps"] for r in records], default=0),
                sweep_limit_hits=sum(r["stop_reason"] == "sweep_limit" for r in records),
                fallback_count=sum(r["fallback"] is not None for r in records),
                max_relative_change=max([r["relative_change"] for r in records
                                         if math.isfinite(r["relative_change"])], default=0.0))


def message(t: T, log_scale=0.0):
    """``_variational_message``: (t / |t|, log_scale + log |t|)."""
    s = norm(t)
    if not math.isfinite(s):
        raise VariationalNumericalError("nonfinite_overlap")
    if s == 0:
        return t, -math.inf
    return t / s, log_scale + math.log(s)


def identity_vector(p) -> T:
    """``_variational_identity``: the normalised identity of a single-layer leg
    as a vector on its fused (ket, bra) leg of parities ``p``."""
    d = int(round(math.sqrt(len(p))))
    v = np.zeros(d * d)
    v[np.arange(d) * d + np.arange(d)] = 1.0 / math.sqrt(d)
    return T(v, [p])


def space_map(P, Q) -> np.ndarray:
    """``_variational_space_map`` (diagonal_variational.jl:232-237): Q <- P, the
    identity on the first min(P_c, Q_c) states of each parity c."""
    M = np.zeros((len(Q), len(P)))
    for c in (0, 1):
        qi, pi = np.nonzero(Q == c)[0], np.nonzero(P == c)[0]
        r = min(len(qi), len(pi))
        M[qi[:r], pi[:r]] = 1.0
    return M


def _side_legs(side):
    # (input leg, output leg) of a double layer (w, n, e, s)
    return (1, 3) if side == "north" else (3, 1)


class _Target:
    """``_RowLayerTarget`` (row_variational.jl:53-77): the input boundary and
    the row's double layers, each divided by |ket| |bra|, with the log scale."""

    def __init__(self, env, row, side):
        if len(env.tensors) != len(row):
            raise ValueError("row boundary length")
        self.input = env
        self.side = side
        self.log_scale = env.log_scale
        self.zero = env.log_scale == -math.inf
        self.reference = math.nan
        self.row = []
        for E in row:
            # |ket| |bra| of a ket = bra layer: its trace over every (ket, bra) pair
            d = [int(round(math.sqrt(n))) for n in E.shape]
            ab = float(np.einsum("aabbccdd->", E.a.reshape([d[0], d[0], d[1], d[1], d[2], d[2], d[3], d[3]])))
            if not math.isfinite(ab):
                raise VariationalNumericalError("nonfinite_target")
            if ab <= 0:
                self.zero = True
                self.row.append(E)
            else:
                self.row.append(E / ab)
                self.log_scale += math.log(ab)
        self.inp, self.out = _side_legs(side)

    def half(self, msg, i, left):
        """``_row_half_projection``: (cand, out, input bond, horizontal) after
        the input tensor and the row site i, entering from the left or right."""
        t, ls = msg
        B, E = self.input.tensors[i], self.row[i]
        if left:   # msg (c, a, w) -> (c, o, b, e)
            spec = "caw,apb,wpeo->cobe" if self.side == "north" else "caw,apb,woep->cobe"
        else:      # msg (c, b, e) -> (c, o, a, w)
            spec = "cbe,apb,wpeo->coaw" if self.side == "north" else "cbe,apb,woep->coaw"
        return message(einsum(spec, t, B, E), ls)

    def mixed_step(self, msg, i, A, left):
        """``_row_mixed_step``: the half projection closed with the candidate."""
        t, ls = self.half(msg, i, left)
        spec = "cobe,coC->Cbe" if left else "coaw,Coc->Caw"
        return message(einsum(spec, t, A), ls)

    def edge(self, C, left):
        """``_row_mixed_edge``: unit legs at the chain's end."""
        i = 0 if left else len(self.row) - 1
        a = 0 if left else 2
        legs = [C.tensors[i].p[a], self.input.tensors[i].p[a], self.row[i].p[0 if left else 2]]
        return message(z2.unit(legs))

    def messages(self, C, left):
        n = len(C.tensors)
        out = [None] * (n + 1)
        if left:
            out[0] = self.edge(C, True)
            for i in range(n):
                out[i + 1] = self.mixed_step(out[i], i, C.tensors[i], True)
        else:
            out[n] = self.edge(C, False)
            for i in range(n - 1, -1, -1):
                out[i] = self.mixed_step(out[i + 1], i, C.tensors[i], False)
        return out

    def project_pair(self, i, L, R):
        """``_row_project_pair``: the normalised two-site projection (c, o, O, C)."""
        lt, lls = self.half(L, i, True)
        rt, rls = self.half(R, i + 1, False)
        theta = einsum("cobe,CObe->coOC", lt, rt)
        s = norm(theta)
        if not math.isfinite(s):
            raise VariationalNumericalError("nonfinite_projection")
        if s == 0:
            raise VariationalNumericalError("zero_local_projection")
        ln = lls + rls + math.log(s)
        if not math.isfinite(ln):
            raise VariationalNumericalError("zero_local_projection")
        return theta / s, ln


class _Candidate:
    __slots__ = ("tensors", "center", "log_scale", "max_truncation")

    def __init__(self, tensors, center=0, log_scale=0.0, max_truncation=0.0):
        self.tensors, self.center, self.log_scale, self.max_truncation = list(tensors), center, log_scale, \
            max_truncation

    def copy(self):
        return _Candidate(self.tensors, self.center, self.log_scale, self.max_truncation)


def _move_center(C, target):
    """``_diagonal_center!``: exact QR / LQ moves of the canonical centre."""
    B = C.tensors
    while C.center < target:
        i = C.center
        Q, R = z2.qr(B[i], [0, 1], [2])
        B[i] = Q
        B[i + 1] = einsum("lk,kpr->lpr", R, B[i + 1])
        C.center += 1
    while C.center > target:
        i = C.center
        L, Q = z2.lq(B[i], [0], [1, 2])
        B[i] = Q
        B[i - 1] = einsum("lpk,kr->lpr", B[i - 1], L)
        C.center -= 1


def _product(t: _Target):
    """``_row_product``: identity vectors on the output legs, unit bonds."""
    tensors = []
    for E in t.row:
        v = identity_vector(E.p[t.out])
        tensors.append(T(v.a.reshape(1, -1, 1), [z2.leg(1, 0), v.p[0], z2.leg(1, 0)]))
    return _Candidate(tensors, 0)


def _warm_start(t: _Target):
    """``_row_warm_start`` (row_variational.jl:100-117)."""
    C = _Candidate(t.input.tensors, t.input.center)
    for i in range(len(C.tensors)):
        P, Q = C.tensors[i].p[1], t.row[i].p[t.out]
        if np.array_equal(P, Q):
            continue
        projects = any(np.sum(P == c) > np.sum(Q == c) for c in (0, 1))
        if projects:
            _move_center(C, i)
        M = space_map(P, Q)
        A = C.tensors[i]
        C.tensors[i] = T(np.einsum("qp,lpr->lqr", M, A.a), [A.p[0], Q, A.p[2]])
    _move_center(C, 0)
    s = norm(C.tensors[0])
    if not math.isfinite(s):
        raise VariationalNumericalError("nonfinite_initialization")
    if s == 0:
        return _product(t)
    C.tensors[0] = C.tensors[0] / s
    return C


def _allowed(C, method):
    """``_row_candidate_allowed``: every bond within chi and the sector budget."""
    for A in C.tensors[:-1]:
        p = A.p[2]
        if len(p) > method.chi:
            return False
        if method.space is not None and (np.sum(p == 0) > method.space[0] or np.sum(p == 1) > method.space[1]):
            return False
    return True


def _initialize_amplitude(t: _Target, C, fixed):
    """``_row_initialize_amplitude!`` (row_variational.jl:172-186)."""
    terminal = fixed[0]
    edge = t.edge(C, True)
    z = float(np.sum(terminal[0].a * edge[0].a))
    if not math.isfinite(z):
        raise VariationalNumericalError("nonfinite_overlap")
    if z == 0 or terminal[1] == -math.inf:
        C.log_scale = -math.inf
        return False
    t.reference = math.log(abs(z)) + terminal[1] + edge[1]
    C.tensors[0] = C.tensors[0] * (1.0 if z > 0 else -1.0)
    C.log_scale = 0.0
    return True


def _half_sweep(C, t: _Target, method, right, entropy, profile, fixed):
    """``_row_half_sweep!`` (row_variational.jl:197-233)."""
    n = len(C.tensors)
    rolling = t.edge(C, right)
    bounded = _allowed(C, method)
    nextfixed = [None] * (n + 1)
    nextfixed[0 if right else n] = rolling
    for i in (range(n - 1) if right else range(n - 2, -1, -1)):
        L = rolling if right else fixed[i]
        R = fixed[i + 2] if right else rolling
        theta, logtheta = t.project_pair(i, L, R)
        if math.isnan(t.reference):
            t.reference = logtheta
        U, S, V, err, ent = z2.svd_trunc(theta, [0, 1], [2, 3], chi=method.chi, space=method.space,
                                         entropy=entropy is not None)
        if entropy is not None:
            entropy.maximum = max(entropy.maximum, ent)
        s = math.sqrt(sum(float(np.sum(x * x)) for x in S))
        if not (math.isfinite(s) and s > 0):
            raise VariationalNumericalError("zero_local_projection")
        newscale = logtheta - t.reference + math.log(s)
        if bounded and not newscale >= C.log_scale - 512 * EPS * max(1.0, abs(C.log_scale)):
            raise VariationalNumericalError("objective_increase")
        kept = np.concatenate(S) / s
        if right:
            C.tensors[i] = U
            C.tensors[i + 1] = T(V.a * kept[:, None, None], V.p)
        else:
            C.tensors[i] = T(U.a * kept[None, None, :], U.p)
            C.tensors[i + 1] = V
        C.center = i + 1 if right else i
        C.log_scale = newscale
        profile[i] = ent if entropy is not None else math.nan
        C.max_truncation = max(C.max_truncation, err * err)
        k = i if right else i + 1
        rolling = t.mixed_step(rolling, k, C.tensors[k], right)
        nextfixed[k + 1 if right else k] = rolling
    return nextfixed


def _relative_change(a, b):
    """``_row_relative_change``: |1 - exp(-|a - b|)| relative to the larger of two logs."""
    largest = max(a, b)
    return -math.expm1(-abs(a - b)) * math.exp(largest - max(largest, math.log(FLOATMIN)))


def _fit(t: _Target, method, entropy):
    """``_row_variational_fit`` (row_variational.jl:240-286)."""
    C = _warm_start(t)
    n = len(C.tensors)
    fixed = t.messages(C, False)
    valid = _initialize_amplitude(t, C, fixed)
    best = C.copy() if valid and _allowed(C, method) else None
    profile = [math.nan] * (n - 1)
    bestprofile = list(profile)
    previous = math.nan
    relative_change = math.inf
    sweeps = 0
    reason = "sweep_limit"
    fallback = None
    maxdiscard = 0.0
    for sweep in range(1, method.max_sweep + 1):
        sweeps = sweep
        try:
            for right in (True, False):
                fixed = _half_sweep(C, t, method, right, entropy, profile, fixed)
                if _allowed(C, method) and (best is None or C.log_scale >= best.log_scale):
                    best, bestprofile = C.copy(), list(profile)
        except (VariationalNumericalError, np.linalg.LinAlgError) as ex:
            failure = ex.reason if isinstance(ex, VariationalNumericalError) else "factorization_failure"
            if math.isfinite(C.log_scale) and _allowed(C, method) and (best is None or C.log_scale > best.log_scale):
                best, bestprofile = C.copy(), list(profile)
            if best is None:
                raise
            fallback = dict(reason=failure, used_svd=False)
            reason = "numerical_fallback"
            maxdiscard = max(maxdiscard, C.max_truncation)
            break
        maxdiscard = max(maxdiscard, C.max_truncation)
        w = 2 * C.log_scale
        relative_change = math.inf if sweep == 1 else _relative_change(w, previous)
        previous = w
        if sweep > 1 and method.threshold_sweep > 0 and relative_change <= method.threshold_sweep:
            reason = "threshold_sweep"
            break
    if best is None:
        raise VariationalNumericalError("no_valid_candidate")
    return best, dict(sweeps=sweeps, relative_change=relative_change, stop_reason=reason,
                      max_local_discarded_weight=maxdiscard, fallback=fallback), bestprofile


def _direct(t: _Target):
    """``_row_direct`` (row_variational.jl:288-304): one site, no fit."""
    C = _product(t)
    edge = t.edge(C, True)
    h, ls = t.half(edge, 0, True)             # (c, o, b, e), b and e trivial
    A = T(h.a.sum(axis=(2, 3))[:, :, None], [h.p[0], h.p[1], z2.leg(1, 0)])
    s = norm(A)
    if not math.isfinite(s):
        raise VariationalNumericalError("nonfinite_projection")
    C.tensors[0] = A if s == 0 else A / s
    C.log_scale = -math.inf if s == 0 else ls + math.log(s)
    t.reference = 0.0
    return C


def absorb_variational(env, row, method: BoundaryMPSRowVariational, side="north", entropy=None, row_cut=0):
    """``_absorb`` for the row variational method (row_variational.jl:306-329)."""
    from .boundary import Env
    if side not in ("north", "south"):
        raise ValueError("invalid row absorption side")
    t = _Target(env, row, side)
    n = len(row)
    profile = [math.nan] * max(0, n - 1)
    report = dict(sweeps=0, relative_change=0.0, stop_reason="direct", max_local_discarded_weight=0.0,
                  fallback=None)
    if t.zero:
        C = _product(t)
        C.tensors[0] = C.tensors[0] * 0.0
        C.log_scale = -math.inf
        t.reference = 0.0
        report["stop_reason"] = "zero_target"
    elif n == 1:
        C = _direct(t)
        if C.log_scale == -math.inf:
            report["stop_reason"] = "zero_target"
    else:
        C, report, profile = _fit(t, method, entropy)
    out = Env(C.tensors, C.log_scale + t.log_scale + t.reference,
              max(env.max_truncation, report["max_local_discarded_weight"]), C.center,
              list(env.variational) + [dict(report, layer=row_cut if side == "north" else row_cut + 1,
                                            reverse=side == "south")])
    if entropy is not None and entropy.Se is not None and 1 <= row_cut <= entropy.Se["north"].shape[0]:
        entropy.Se[side][row_cut - 1, :] = profile
    return out

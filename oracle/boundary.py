"""Row boundary-MPS contraction for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/contraction/boundary_mps.jl`` (the whole file) for Z2 dense
tensors.  Function names follow the reference; line citations are given per
function.  All indices are 0-based here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import z2
from .z2 import T, einsum, fuse, norm, unit


@dataclass
class BoundaryMPS:
    """``BoundaryMPS(chi, sector_space)`` (``boundary_mps.jl:11-18``).

    ``zipup`` selects the zip-up row absorption of ``absorb_zipup`` (the
    GPU engine's batched variant, which has no counterpart in the reference)
    in place of the reference's exact-LQ-plus-SVD compression.
    """
    chi: int
    space: tuple | None = None
    zipup: bool = False


@dataclass
class Env:
    """``BoundaryEnvironment`` (``boundary_mps.jl:79-83``); ``center`` and
    ``variational`` (the fit records) are kept by the variational method
    (``RowVariationalBoundary``, ``row_variational.jl:37-43``)."""
    tensors: list
    log_scale: float = 0.0
    max_truncation: float = 0.0
    center: int = 0
    variational: list = field(default_factory=list)


class Entropy:
    """``BoundaryEntropy`` (``boundary_mps.jl:44-57``)."""

    def __init__(self, Lx=None, Ly=None):
        self.maximum = 0.0
        self.Se = None
        if Lx is not None:
            self.Se = {"north": np.full((Ly - 1, Lx - 1), np.nan),
                       "south": np.full((Ly - 1, Lx - 1), np.nan)}

    def record(self, side, row, bond, value):
        self.maximum = max(self.maximum, value)
        if self.Se is not None and 1 <= row <= self.Se["north"].shape[0]:
            self.Se[side][row - 1, bond - 1] = value


class Slab:
    """``SlabColumn`` (``boundary_mps.jl:212-215``)."""
    __slots__ = ("upper", "lower")

    def __init__(self, upper, lower):
        self.upper, self.lower = upper, lower


def act(A: T, O: np.ndarray | T, axis: int, out_par=None) -> T:
    """``_act`` (``boundary_mps.jl:59-62``): A[..i'..] = sum_k O[i',k] A[..k..]."""
    if not isinstance(O, T):
        assert out_par is not None
        O = T(O, [out_par, A.p[axis]])
    a = np.tensordot(O.a, A.a, axes=([1], [axis]))
    a = np.moveaxis(a, 0, axis)
    p = list(A.p)
    p[axis] = O.p[0]
    return T(a, p)


def double_layer(ket: T, bra: T | None = None, physical=None) -> T:
    """``double_layer`` (``boundary_mps.jl:65-73``): fused (W,N,E,S), each (ket,bra)."""
    if bra is None:
        bra = ket
    A = ket if physical is None else act(ket, physical, 2, out_par=ket.p[2])
    raw = einsum("wnpaes,WNpaES->wWnNeEsS", A, bra)
    for axis in (6, 4, 2, 0):
        raw = fuse(raw, axis, 2)
    return raw


def row_layers(s):
    return [[double_layer(s.sites[x][y]) for y in range(s.Ly)] for x in range(s.Lx)]


def col(layers, y):
    return [layers[x][y] for x in range(len(layers))]


def trivial_boundary(row, side) -> Env:
    """``_trivial_boundary`` (``boundary_mps.jl:86-91``)."""
    axis = 1 if side == "north" else 3
    return Env([unit([z2.leg(1, 0), A.p[axis], z2.leg(1, 0)]) for A in row], 0.0, 0.0)


def compress_boundary(B, chi, reverse=False, space=None, observer=None):
    """``compress_boundary!`` (``boundary_mps.jl:94-134``)."""
    if chi < 1:
        raise ValueError("chi must be positive")
    N = len(B)
    max_error = 0.0
    want_ent = observer is not None
    if not reverse:
        for x in range(N - 1, 0, -1):
            L, Q = z2.lq(B[x], [0], [1, 2])
            B[x] = Q
            B[x - 1] = einsum("lpk,kr->lpr", B[x - 1], L)
        for x in range(N - 1):
            nM = norm(B[x])
            U, S, V, err, ent = z2.svd_trunc(B[x], [0, 1], [2], chi=chi, space=space, entropy=want_ent)
            if want_ent:
                observer(x + 1, ent)
            max_error = max(max_error, 0.0 if nM == 0 else (err / nM) ** 2)
            B[x] = U
            R = einsum("k,kr->kr", T(np.concatenate(S), [V.p[0]]), V)
            B[x + 1] = einsum("lk,kpr->lpr", R, B[x + 1])
    else:
        for x in range(N - 1):
            Q, R = z2.qr(B[x], [0, 1], [2])
            B[x] = Q
            B[x + 1] = einsum("lk,kpr->lpr", R, B[x + 1])
        for x in range(N - 1, 0, -1):
            nM = norm(B[x])
            U, S, V, err, ent = z2.svd_trunc(B[x], [0], [1, 2], chi=chi, space=space, entropy=want_ent)
            if want_ent:
                observer(x, ent)
            max_error = max(max_error, 0.0 if nM == 0 else (err / nM) ** 2)
            B[x] = V
            L = einsum("lk,k->lk", U, T(np.concatenate(S), [U.p[1]]))
            B[x - 1] = einsum("lpk,kr->lpr", B[x - 1], L)
    center = 0 if reverse else N - 1
    scale = norm(B[center])
    if not math.isfinite(scale):
        raise RuntimeError("nonfinite boundary norm")
    if scale != 0.0:
        B[center] = B[center] / scale
    return max_error, (-math.inf if scale == 0.0 else math.log(scale))


def absorb_zipup(env: Env, row, method: BoundaryMPS, side="north") -> Env:
    """Zip-up row absorption, the GPU engine's variant (no counterpart in the reference).

    The boundary is first brought into the canonical form opposite to the
    sweep (an LQ sweep north, a QR sweep south, on the small chi-bond tensors).
    Then one sweep over the row: the carried factor times the boundary tensor times
    the row tensor is split by a truncated SVD (``truncrank(chi) &
    truncspace(space)``, as in ``_boundary_svd``, ``boundary_mps.jl:33-42``);
    the isometry becomes the new boundary tensor and the rest (S V^T north,
    U S south) is carried to the next site.  No canonical form is built, so
    each truncation is local; the centre (last site north, first site south)
    is normalised as in ``compress_boundary!`` (``boundary_mps.jl:129-133``).
    """
    N = len(row)
    maxe = 0.0
    out = [None] * N
    E = list(env.tensors)
    if side == "north":
        # right-canonical boundary (LQ sweep), so that everything right of the
        # zip front except the row is an isometry
        for x in range(N - 1, 0, -1):
            L, Q = z2.lq(E[x], [0], [1, 2])
            E[x] = Q
            E[x - 1] = einsum("lnk,kr->lnr", E[x - 1], L)
        C = unit([z2.leg(1, 0), E[0].p[0], row[0].p[0]])      # (a, l, w)
        for x in range(N):
            T1 = einsum("alw,lnr->awnr", C, E[x])
            Tt = einsum("awnr,wnes->asre", T1, row[x])
            if x == N - 1:
                out[x] = fuse(Tt, 2, 2)
                continue
            nM = norm(Tt)
            U, S, V, err, _ = z2.svd_trunc(Tt, [0, 1], [2, 3], chi=method.chi, space=method.space)
            maxe = max(maxe, 0.0 if nM == 0 else (err / nM) ** 2)
            out[x] = U
            C = einsum("k,kre->kre", T(np.concatenate(S), [V.p[0]]), V)
        center = N - 1
    else:
        # left-canonical boundary (QR sweep)
        for x in range(N - 1):
            Q, R = z2.qr(E[x], [0, 1], [2])
            E[x] = Q
            E[x + 1] = einsum("lk,knr->lnr", R, E[x + 1])
        C = unit([E[N - 1].p[2], row[N - 1].p[2], z2.leg(1, 0)])   # (r, e, a)
        for x in range(N - 1, -1, -1):
            T1 = einsum("lsr,rea->lsea", E[x], C)
            Tt = einsum("lsea,wnes->lwna", T1, row[x])
            if x == 0:
                out[x] = fuse(Tt, 0, 2)
                continue
            nM = norm(Tt)
            U, S, V, err, _ = z2.svd_trunc(Tt, [0, 1], [2, 3], chi=method.chi, space=method.space)
            maxe = max(maxe, 0.0 if nM == 0 else (err / nM) ** 2)
            out[x] = V
            C = einsum("lwk,k->lwk", U, T(np.concatenate(S), [U.p[2]]))
        center = 0
    scale = norm(out[center])
    if not math.isfinite(scale):
        raise RuntimeError("nonfinite boundary norm")
    if scale != 0.0:
        out[center] = out[center] / scale
    ls = -math.inf if scale == 0.0 else math.log(scale)
    return Env(out, env.log_scale + ls, max(env.max_truncation, maxe))


def absorb(env: Env, row, method: BoundaryMPS, side="north", entropy=None, row_cut=0) -> Env:
    """``_absorb`` for the row method (``boundary_mps.jl:136-151``); the row
    variational method absorbs by its fit (``variational.absorb_variational``)."""
    from .variational import BoundaryMPSRowVariational, absorb_variational
    if isinstance(method, BoundaryMPSRowVariational):
        return absorb_variational(env, row, method, side, entropy, row_cut)
    if method.zipup:
        return absorb_zipup(env, row, method, side)
    B = []
    for A, E in zip(env.tensors, row):
        if side == "north":
            C = einsum("lnr,wnep->lwpre", A, E)
        else:
            C = einsum("lsr,wpes->lwpre", A, E)
        B.append(fuse(fuse(C, 3, 2), 0, 2))
    observer = None
    if entropy is not None:
        observer = lambda b, se: entropy.record(side, row_cut, b, se)
    mt, ls = compress_boundary(B, method.chi, reverse=(side == "south"), space=method.space,
                               observer=observer)
    return Env(B, env.log_scale + ls, max(env.max_truncation, mt))


def close_boundary(B) -> float:
    """``_close_boundary`` (``boundary_mps.jl:153-163``)."""
    V = np.ones(B[0].shape[0])
    for A in B:
        assert A.shape[1] == 1
        V = np.einsum("l,lr->r", V, A.a[:, 0, :])
    return float(V.sum())


def contract_layers(layers, method):
    """``contract_layers`` (``boundary_mps.jl:165-172``)."""
    env = trivial_boundary(col(layers, 0), "north")
    for y in range(len(layers[0])):
        env = absorb(env, col(layers, y), method)
    return close_boundary(env.tensors), env.log_scale, env.max_truncation


def positive_real(z, name):
    """``_positive_real`` (``boundary_mps.jl:187-191``)."""
    if not (math.isfinite(z) and z > 0):
        raise RuntimeError(f"{name} requires a finite positive real value; received {z}")
    return float(z)


def lognorm(s, method):
    """``lognorm`` (``boundary_mps.jl:180-186``; the variational method adds its
    fit summary, ``row_variational.jl:331-339``)."""
    layers = row_layers(s)
    env = trivial_boundary(col(layers, 0), "north")
    for y in range(len(layers[0])):
        env = absorb(env, col(layers, y), method, row_cut=y + 1)
    v = positive_real(close_boundary(env.tensors), "norm")
    out = dict(log_norm=math.log(v) + env.log_scale + 2 * s.log_amplitude,
               tensor_log_norm=math.log(v) + env.log_scale, max_environment_truncation=env.max_truncation)
    if env.variational:
        from .variational import summary
        out["boundary_variational"] = summary(env.variational)
    return out


def boundary_environments(layers, method, side="both", entropy=None):
    """``boundary_environments`` (``boundary_mps.jl:193-209``)."""
    Ly = len(layers[0])
    north = [None] * (Ly + 1)
    south = [None] * (Ly + 1)
    north[0] = trivial_boundary(col(layers, 0), "north")
    south[Ly] = trivial_boundary(col(layers, Ly - 1), "south")
    if side != "south":
        for y in range(Ly):
            north[y + 1] = absorb(north[y], col(layers, y), method, entropy=entropy, row_cut=y + 1)
    if side != "north":
        for y in range(Ly - 1, -1, -1):
            south[y] = absorb(south[y + 1], col(layers, y), method, side="south",
                              entropy=entropy, row_cut=y)
    mx = max(0.0 if side == "south" else north[Ly].max_truncation,
             0.0 if side == "north" else south[0].max_truncation)
    return north, south, mx


# --- row environments (boundary_mps.jl:216-284) -----------------------------

def left_step(L, Tt, E, B):
    if isinstance(E, Slab):
        X = einsum("awvb,anc->wvbnc", L, Tt)
        Y = einsum("wvbnc,wnek->vbcek", X, E.upper)
        Z = einsum("vbcek,vkfs->bcefs", Y, E.lower)
        return einsum("bcefs,bsd->cefd", Z, B)
    X = einsum("awb,anc->wbnc", L, Tt)
    Y = einsum("wbnc,wnes->bces", X, E)
    return einsum("bces,bsd->ced", Y, B)


def right_step(Tt, E, B, R):
    if isinstance(E, Slab):
        X = einsum("anc,cefd->anefd", Tt, R)
        Y = einsum("anefd,wnek->awkfd", X, E.upper)
        Z = einsum("awkfd,vkfs->awvsd", Y, E.lower)
        return einsum("awvsd,bsd->awvb", Z, B)
    X = einsum("anc,ced->aned", Tt, R)
    Y = einsum("aned,wnes->awsd", X, E)
    return einsum("awsd,bsd->awb", Y, B)


def row_edge(top, row, bottom, side):
    i = 0 if side == "left" else len(row) - 1
    a = 0 if side == "left" else 2
    E = row[i]
    if isinstance(E, Slab):
        return unit([top[i].p[a], E.upper.p[a], E.lower.p[a], bottom[i].p[a]])
    return unit([top[i].p[a], E.p[a], bottom[i].p[a]])


def safe_scale(t):
    s = norm(t)
    if not math.isfinite(s):
        raise RuntimeError("nonfinite row environment")
    return t if s == 0.0 else t / s


def row_environments(top, row, bottom, side="both"):
    N = len(row)
    left = [None] * (N + 1)
    right = [None] * (N + 1)
    left[0] = row_edge(top, row, bottom, "left")
    right[N] = row_edge(top, row, bottom, "right")
    if side != "right":
        for x in range(N):
            left[x + 1] = safe_scale(left_step(left[x], top[x], row[x], bottom[x]))
    if side != "left":
        for x in range(N - 1, -1, -1):
            right[x] = safe_scale(right_step(top[x], row[x], bottom[x], right[x + 1]))
    return left, right


def join_scalars(L, R) -> float:
    return float(np.sum(L.a * R.a))


def row_scalar(L, Tt, E, B, R) -> float:
    return join_scalars(left_step(L, Tt, E, B), R)


@dataclass
class BondEnvironment:
    """``BondEnvironment`` (``boundary_mps.jl:291-298``)."""
    left: T
    right: T
    top: tuple
    bottom: tuple
    outer: tuple
    direction: str


def bond_environment(state, layers, north, south, i, j, direction, left=None, right=None):
    """``bond_environment`` (``boundary_mps.jl:300-327``) for the row method."""
    x, y = i
    top = north[y].tensors
    bottom = south[y + (1 if direction == "horizontal" else 2)].tensors
    lastx = x + 1 if direction == "horizontal" else x
    if left is None or right is None:
        if direction == "horizontal":
            row = col(layers, y)
        else:
            row = [Slab(layers[k][y], layers[k][y + 1]) for k in range(len(layers))]
        le, ri = row_environments(top, row, bottom)
        left, right = le[x], ri[lastx + 1]
    if direction == "horizontal":
        Tt = (top[x], top[x + 1])
        Bt = (bottom[x], bottom[x + 1])
        outer = ((i, 0), (i, 1), (i, 5), (j, 1), (j, 4), (j, 5))
    else:
        Tt = (top[x],)
        Bt = (bottom[x],)
        outer = ((i, 0), (i, 1), (i, 4), (j, 0), (j, 4), (j, 5))
    spaces = tuple(state[s].p[ax] for (s, ax) in outer)
    return BondEnvironment(left, right, Tt, Bt, spaces, direction)


def bond_hole(env: BondEnvironment) -> T:
    """``bond_hole`` (``boundary_mps.jl:331-350``): six double legs, each split (ket,bra)."""
    left, right = env.left, env.right
    if env.direction == "horizontal":
        T1, T2 = env.top
        B1, B2 = env.bottom
        X = einsum("awb,anc->wbnc", left, T1)
        L = einsum("wbnc,bsf->cwnfs", X, B1)
        Y = einsum("deg,cvd->cveg", right, T2)
        R = einsum("cveg,ftg->cveft", Y, B2)
        H = einsum("cwnfs,cveft->wnsvet", L, R)
    else:
        Tt = env.top[0]
        Bt = env.bottom[0]
        L = einsum("awvb,anc->wvbnc", left, Tt)
        R = einsum("bsd,cefd->bscef", Bt, right)
        H = einsum("wvbnc,bscef->wnevfs", L, R)
    for k in range(5, -1, -1):
        V = env.outer[k]
        H = z2.split(H, k, (V, V))
    return H

"""Diagonal boundary-MPS contraction for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/contraction/diagonal_mps.jl`` (``BoundaryMPSDiagonal``: the
lattice is swept by anti-diagonal layers x + y = t; each layer is absorbed
as one raw block per site, the blocks are brought into an exact canonical
form and only the bonds that a site opens inside its block are truncated),
the Born sampling of ``src/sampling/diagonal_born.jl`` and the energy of
``src/measurement/diagonal_energy.jl``.

Conventions.  Sites are 0-based (x, y); layer t = x + y runs over
0 .. Lx+Ly-2 (the reference's t - 2 with 1-based sites, so parities of t
agree).  A lattice edge is named ``('h', x, y)`` (between (x-1, y) and
(x, y); x = 0 and x = Lx are the open boundary) or ``('v', x, y)``
(between (x, y-1) and (x, y)); these replace the reference's integer edge
labels (``_diagonal_ports``, diagonal_mps.jl:91-97).  A double-layer leg is
the (ket, bra) pair fused ket-major, as in ``boundary.double_layer``.
Networks are built from labelled tensors that contract every label they
share (``_DiagonalTensor`` / ``_diagonal_join``, diagonal_mps.jl:14-32).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import z2
from .z2 import T

VIRTUAL_AXES = (0, 1, 4, 5)   # w, n, e, s of a site tensor (w, n, p, a, e, s)
TRIV = z2.leg(1, 0)


@dataclass
class BoundaryMPSDiagonal:
    """``BoundaryMPSDiagonal(chi, sector_space)`` (diagonal_mps.jl:3-9)."""
    chi: int
    space: tuple | None = None


# ---------------------------------------------------------------------------
# labelled tensors (diagonal_mps.jl:14-50)
# ---------------------------------------------------------------------------

class LT:
    """A Z2 tensor (or a plain number) with one label per leg."""
    __slots__ = ("t", "labels")

    def __init__(self, t, labels):
        self.t = t
        self.labels = list(labels)
        if isinstance(t, T):
            assert t.ndim == len(self.labels), (t.shape, self.labels)
        else:
            assert not self.labels


def _letters(labels):
    table = {}
    for k in labels:
        if k not in table:
            table[k] = chr(ord("a") + len(table)) if len(table) < 26 else chr(ord("A") + len(table) - 26)
    return table


def join(a: LT, b: LT) -> LT:
    """``_diagonal_join``: contract the shared labels; a's free labels, then b's."""
    if not isinstance(a.t, T):
        return LT(a.t * b.t, b.labels)
    if not isinstance(b.t, T):
        return LT(a.t * b.t, a.labels)
    common = [k for k in a.labels if k in b.labels]
    free = [k for k in a.labels if k not in common] + [k for k in b.labels if k not in common]
    tab = _letters(a.labels + b.labels)
    spec = "".join(tab[k] for k in a.labels) + "," + "".join(tab[k] for k in b.labels) + "->" + \
        "".join(tab[k] for k in free)
    if not free:
        return LT(float(np.einsum(spec, a.t.a, b.t.a)), [])
    return LT(z2.einsum(spec, a.t, b.t), free)


def reorder(a: LT, labels) -> LT:
    """``_diagonal_reorder``."""
    labels = list(labels)
    if len(labels) != len(a.labels) or set(labels) != set(a.labels):
        raise ValueError("diagonal tensor labels")
    if not labels:
        return a
    return LT(z2.perm(a.t, [a.labels.index(k) for k in labels]), labels)


def unit_lt(label) -> LT:
    """``_diagonal_unit`` on a trivial (open-boundary) leg."""
    return LT(z2.unit([TRIV]), [label])


def scalar(a: LT) -> float:
    """``_diagonal_scalar``."""
    if a.labels:
        raise RuntimeError("unclosed diagonal network")
    return float(a.t)


def scale(a: LT) -> LT:
    """``_diagonal_scale``: divide by the Frobenius norm unless it is zero."""
    v = z2.norm(a.t) if isinstance(a.t, T) else abs(a.t)
    if not math.isfinite(v):
        raise RuntimeError("nonfinite diagonal environment")
    if v == 0:
        return a
    return LT(a.t / v, a.labels)


def apply(message: LT, A: T, B: T, ports, inputs, physical=None) -> LT:
    """``_diagonal_apply`` (diagonal_mps.jl:58-88): contract the two input
    ports of ``message`` with the ket A, then the bra B; the other two
    virtual legs leave as fused (ket, bra) ports appended in w, n, e, s order.
    ``physical`` = (ket label, bra label) keeps the physical legs open."""
    if len(inputs) != 2:
        raise ValueError("a diagonal vertex has two input ports")
    rk = [("k", 0), ("k", 1), ("p",), ("aux",), ("k", 4), ("k", 5)]
    rb = [("b", 0), ("b", 1), ("p",), ("aux",), ("b", 4), ("b", 5)]
    if physical is not None:
        rk[2], rb[2] = physical
    for port in inputs:
        axis = VIRTUAL_AXES[list(ports).index(port)]
        pos = message.labels.index(port)
        t = z2.split(message.t, pos, [A.p[axis], B.p[axis]])
        labels = message.labels[:pos] + [rk[axis], rb[axis]] + message.labels[pos + 1:]
        message = LT(t, labels)
    message = join(message, LT(A, rk))
    message = join(message, LT(B, rb))
    for axis, port in zip(VIRTUAL_AXES, ports):
        if port in inputs:
            continue
        pair = [rk[axis], rb[axis]]
        others = [k for k in message.labels if k not in pair]
        message = reorder(message, others + pair)
        message = LT(z2.fuse(message.t, len(others), 2), others + [port])
    return message


# ---------------------------------------------------------------------------
# lattice bookkeeping (diagonal_mps.jl:91-104, 158-176)
# ---------------------------------------------------------------------------

def ports_of(site):
    """(west, north, east, south) edge names of a 0-based site."""
    x, y = site
    return (("h", x, y), ("v", x, y), ("h", x + 1, y), ("v", x, y + 1))


def inside_of(Lx, Ly, site):
    x, y = site
    return (x > 0, y > 0, x < Lx - 1, y < Ly - 1)


def layer_count(Lx, Ly):
    return Lx + Ly - 1


def layer_sites(Lx, Ly, t):
    """Sites of layer t by increasing x - y (that is, increasing x)."""
    return [(x, t - x) for x in range(max(0, t - Ly + 1), min(Lx - 1, t) + 1)]


def draw_sites(Lx, Ly, t, reverse=False):
    """``_diagonal_sites``: x ascending on even layers, descending on odd ones."""
    s = layer_sites(Lx, Ly, t)
    if t % 2 == 1:
        s.reverse()
    if reverse:
        s.reverse()
    return s


def draw_order(Lx, Ly):
    """``_diagonal_order``: the order in which a draw visits the sites."""
    return [s for t in range(layer_count(Lx, Ly)) for s in draw_sites(Lx, Ly, t)]


@dataclass
class DiagonalBoundary:
    """``DiagonalBoundary`` (diagonal_mps.jl:106-118): one tensor (l, edge, r)
    per frontier edge, in frontier order."""
    tensors: list = field(default_factory=list)
    edges: list = field(default_factory=list)
    center: int = -1
    log_scale: float = 0.0
    max_truncation: float = 0.0
    scalar: float = 1.0
    variational: list = field(default_factory=list)   # fit records of the variational method

    def copy(self):
        return DiagonalBoundary(list(self.tensors), list(self.edges), self.center, self.log_scale,
                                self.max_truncation, self.scalar, list(self.variational))


class DiagonalEntropy:
    """``_diagonal_entropy`` (diagonal_mps.jl:143-146): the largest Schmidt
    entropy and, per site, the value of the bond its block split opened."""

    def __init__(self, Lx, Ly, profile=False):
        self.maximum = 0.0
        self.Se = {"northwest": np.full((Lx, Ly), np.nan), "southeast": np.full((Lx, Ly), np.nan)} \
            if profile else None

    def record(self, reverse, site, value):
        self.maximum = max(self.maximum, value)
        if self.Se is not None:
            self.Se["southeast" if reverse else "northwest"][site] = value


def layer_layout(inp: DiagonalBoundary, Lx, Ly, t, reverse=False):
    """``_diagonal_layer_layout`` (diagonal_mps.jl:158-176)."""
    sites = layer_sites(Lx, Ly, t)
    ia = (3, 2) if reverse else (0, 1)
    oa = (0, 1) if reverse else (3, 2)
    inputs, outputs, ranges, edges = [], [], [], []
    for site in sites:
        ports = ports_of(site)
        inside = inside_of(Lx, Ly, site)
        incoming = [ports[k] for k in ia if inside[k]]
        p = inp.edges.index(incoming[0]) if incoming else 0
        if inp.edges[p:p + len(incoming)] != incoming:
            raise RuntimeError("nonadjacent diagonal frontier inputs")
        out = [ports[k] for k in oa if inside[k]]
        inputs.append(list(range(p, p + len(incoming))))
        outputs.append(out)
        ranges.append(list(range(len(edges), len(edges) + len(out))))
        edges.extend(out)
    return dict(sites=sites, inputs=inputs, outputs=outputs, ranges=ranges, edges=edges)


def raw_block(inp: DiagonalBoundary, A: T, Lx, Ly, site, indices, outputs, reverse=False) -> T:
    """``_diagonal_raw_block`` (diagonal_mps.jl:179-209): the input frontier
    tensors of one site contracted with its ket and bra; legs
    (left, outputs..., right)."""
    ports = ports_of(site)
    inside = inside_of(Lx, Ly, site)
    ia = (3, 2) if reverse else (0, 1)
    oa = (0, 1) if reverse else (3, 2)
    inputs = [ports[k] for k in ia if inside[k]]
    L, R, R2 = ("L",), ("R",), ("R2",)
    if not inputs:
        if inp.tensors:
            raise RuntimeError("disconnected diagonal initialization")
        phi = LT(z2.unit([TRIV, TRIV]), [L, R])
    else:
        phi = LT(inp.tensors[indices[0]], [L, inputs[0], R])
        if len(inputs) == 2:
            phi = LT(phi.t, [L, inputs[0], R2])
            phi = join(phi, LT(inp.tensors[indices[-1]], [R2, inputs[1], R]))
    for k in ia:
        if not inside[k]:
            phi = join(phi, unit_lt(ports[k]))
    theta = apply(phi, A, A, ports, [ports[k] for k in ia])
    for k in oa:
        if not inside[k]:
            theta = join(theta, unit_lt(ports[k]))
    return reorder(theta, [L] + list(outputs) + [R]).t


def normalized(A: T):
    """``_diagonal_normalized``: (A / |A|, log |A|)."""
    s = z2.norm(A)
    if not math.isfinite(s):
        raise RuntimeError("nonfinite diagonal boundary norm")
    if s == 0:
        return A, -math.inf
    return A / s, math.log(s)


# ---------------------------------------------------------------------------
# absorbing a layer (diagonal_mps.jl:219-297)
# ---------------------------------------------------------------------------

def _block_center_step(blocks, j, right):
    """``_diagonal_block_center_step!``: move the centre one block right (QR
    over the last leg) or left (LQ over the first leg); the factor carried on
    is normalised and its log norm returned."""
    A = blocks[j]
    rank = A.ndim
    if right:
        Q, R = z2.qr(A, list(range(rank - 1)), [rank - 1])
        blocks[j] = Q
        R, s = normalized(R)
        nxt = blocks[j + 1]
        blocks[j + 1] = z2.matmul_view(R, [0], [1], nxt, [0], list(range(1, nxt.ndim)))
    else:
        L, Q = z2.lq(A, [0], list(range(1, rank)))
        blocks[j] = Q
        L, s = normalized(L)
        prev = blocks[j - 1]
        last = prev.ndim - 1
        blocks[j - 1] = z2.matmul_view(prev, list(range(last)), [last], L, [0], [1])
    return s


def compress_blocks(blocks, layout, method: BoundaryMPSDiagonal, right, reverse=False, entropy=None):
    """``_diagonal_compress_blocks!`` (diagonal_mps.jl:240-271): an exact
    canonical sweep over the blocks, then a sweep that splits every
    two-output block by a truncated SVD and moves the centre exactly across
    the bonds between blocks (which already meet the budget)."""
    n = len(blocks)
    total = 0.0
    max_error = 0.0
    for j in (range(n - 1, 0, -1) if right else range(n - 1)):
        total += _block_center_step(blocks, j, not right)
    tensors = [None] * len(layout["edges"])
    for j in (range(n) if right else range(n - 1, -1, -1)):
        cut = layout["ranges"][j]
        if len(cut) == 2:
            M = blocks[j]
            U, S, V, err, ent = z2.svd_trunc(M, [0, 1], [2, 3], chi=method.chi, space=method.space,
                                             entropy=entropy is not None)
            if entropy is not None:
                entropy.record(reverse, layout["sites"][j], ent)
            mag = z2.norm(M)
            max_error = max(max_error, 0.0 if mag == 0 else (err / mag) ** 2)
            s = np.concatenate(S)
            if right:
                tensors[cut[0]] = U
                blocks[j] = T(V.a * s[:, None, None], V.p)
            else:
                tensors[cut[-1]] = V
                blocks[j] = T(U.a * s[None, None, :], U.p)
        if j == (n - 1 if right else 0):
            blocks[j], inc = normalized(blocks[j])
            total += inc
        else:
            total += _block_center_step(blocks, j, right)
        tensors[cut[-1] if right else cut[0]] = blocks[j]
    return dict(tensors=tensors, center=len(tensors) - 1 if right else 0, log_scale=total,
                max_truncation=max_error)


def absorb_layer(env: DiagonalBoundary, site_tensor, Lx, Ly, t, method: BoundaryMPSDiagonal, reverse=False,
                 entropy=None) -> DiagonalBoundary:
    """``_diagonal_absorb_layer!`` (diagonal_mps.jl:272-297); ``site_tensor``
    maps a site to its tensor.  Modifies and returns ``env``.  The diagonal
    variational method absorbs by its fit (``diagonal_variational``)."""
    from . import diagonal_variational as dv
    if isinstance(method, dv.BoundaryMPSDiagonalVariational):
        return dv.absorb_layer_variational(env, site_tensor, Lx, Ly, t, method, reverse, entropy)
    if method.chi < 1:
        raise ValueError("chi must be positive")
    layout = layer_layout(env, Lx, Ly, t, reverse)
    blocks = []
    total = env.log_scale
    for j, site in enumerate(layout["sites"]):
        A = raw_block(env, site_tensor(site), Lx, Ly, site, layout["inputs"][j], layout["outputs"][j], reverse)
        A, inc = normalized(A)
        blocks.append(A)
        total += inc
    if not layout["edges"]:
        # the last corner: two unit boundary bonds
        (A,) = blocks
        env.tensors, env.center, env.scalar = [], -1, float(A.a.reshape(-1)[0])
    else:
        right = (not reverse) if len(blocks) < 2 else ((t % 2 == 0) != reverse)
        res = compress_blocks(blocks, layout, method, right, reverse, entropy)
        env.tensors, env.center = res["tensors"], res["center"]
        env.max_truncation = max(env.max_truncation, res["max_truncation"])
        total += res["log_scale"]
    env.edges = layout["edges"]
    env.log_scale = total
    return env


def boundaries(state, method: BoundaryMPSDiagonal, side="both", entropy=None):
    """``_diagonal_boundaries`` (diagonal_mps.jl:298-314): ``nw[t]`` holds the
    layers before t, ``se[t]`` the layers from t on (0-based t)."""
    if side not in ("both", "northwest", "southeast"):
        raise ValueError("invalid diagonal boundary side")
    Lx, Ly = state.Lx, state.Ly
    nl = layer_count(Lx, Ly)
    nw = [None] * (nl + 1)
    se = [None] * (nl + 1)
    nw[0] = DiagonalBoundary()
    se[nl] = DiagonalBoundary()
    at = lambda s: state[s[0], s[1]]
    if side != "southeast":
        for t in range(nl):
            nw[t + 1] = absorb_layer(nw[t].copy(), at, Lx, Ly, t, method, entropy=entropy)
    if side != "northwest":
        for t in range(nl - 1, -1, -1):
            se[t] = absorb_layer(se[t + 1].copy(), at, Lx, Ly, t, method, reverse=True, entropy=entropy)
    return nw, se


def lognorm(state, method: BoundaryMPSDiagonal):
    """``lognorm`` for the diagonal method (diagonal_mps.jl:315-323)."""
    from .boundary import positive_real
    env = DiagonalBoundary()
    at = lambda s: state[s[0], s[1]]
    for t in range(layer_count(state.Lx, state.Ly)):
        absorb_layer(env, at, state.Lx, state.Ly, t, method)
    value = math.log(positive_real(env.scalar, "norm")) + env.log_scale
    out = dict(log_norm=value + 2 * state.log_amplitude, tensor_log_norm=value,
               max_environment_truncation=env.max_truncation)
    if env.variational:
        from .variational import summary
        out["boundary_variational"] = summary(env.variational)
    return out


# ---------------------------------------------------------------------------
# strips between cached boundaries (diagonal_mps.jl:325-443)
# ---------------------------------------------------------------------------

class Strip:
    """``DiagonalStrip`` / ``_diagonal_strip`` (diagonal_mps.jl:325-363): the
    sites of layers first..last by increasing x - y, the frontier tensors of
    the two boundaries attached to the site that owns their edge, unit
    vectors on open-boundary ports, and the unit ends of the boundary chains."""

    def __init__(self, state, first, last, nw: DiagonalBoundary, se: DiagonalBoundary):
        Lx, Ly = state.Lx, state.Ly
        self.sites = sorted([s for t in range(first, last + 1) for s in layer_sites(Lx, Ly, t)],
                            key=lambda s: s[0] - s[1])
        self.ports = [ports_of(s) for s in self.sites]
        self.attachments = [[] for _ in self.sites]
        left, right = LT(1.0, []), LT(1.0, [])
        base = 0
        for b in (nw, se):
            if not b.tensors:
                continue
            assert b.tensors[0].shape[0] == 1 and b.tensors[-1].shape[2] == 1
            left = join(left, unit_lt(("bond", base)))
            right = join(right, unit_lt(("bond", base + len(b.tensors))))
            for k, (A, edge) in enumerate(zip(b.tensors, b.edges)):
                owner = [i for i, p in enumerate(self.ports) if edge in p]
                if not owner:
                    raise RuntimeError("boundary edge and diagonal strip are disconnected")
                self.attachments[owner[0]].append(LT(A, [("bond", base + k), edge, ("bond", base + k + 1)]))
            base += len(b.tensors) + 1
        for k, site in enumerate(self.sites):
            inside = inside_of(Lx, Ly, site)
            for j in range(4):
                if not inside[j]:
                    self.attachments[k].append(unit_lt(self.ports[k][j]))
        self.left, self.right = left, right
        self.max_truncation = max(nw.max_truncation, se.max_truncation)


def _attach(message: LT, pending):
    """``_diagonal_attach``: the pending tensor sharing most labels (the first
    on ties); with none shared, the first open-boundary unit vector."""
    scores = [len(set(message.labels) & set(A.labels)) for A in pending]
    index = int(np.argmax(scores))
    if scores[index] == 0:
        units = [i for i, A in enumerate(pending) if len(A.labels) == 1]
        if not units:
            raise RuntimeError("disconnected diagonal strip attachment")
        index = units[0]
    return join(message, pending.pop(index))


def step(message: LT, strip: Strip, k, A: T, B: T | None = None, physical=None) -> LT:
    """``_diagonal_step`` (diagonal_mps.jl:380-394)."""
    B = A if B is None else B
    pending = list(strip.attachments[k])
    ports = strip.ports[k]
    while sum(p in message.labels for p in ports) < 2:
        if not pending:
            raise RuntimeError("missing diagonal strip inputs")
        message = _attach(message, pending)
    inputs = [p for p in ports if p in message.labels]
    if len(inputs) != 2:
        raise RuntimeError("diagonal strip step has more than two inputs")
    message = apply(message, A, B, ports, inputs, physical)
    while pending:
        message = _attach(message, pending)
    return message


def messages(state, strip: Strip, side="both"):
    """``_diagonal_messages`` (diagonal_mps.jl:395-412): ``left[k]`` has
    absorbed sites before k, ``right[k]`` sites from k on."""
    if side not in ("both", "left", "right"):
        raise ValueError("invalid strip message side")
    n = len(strip.sites)
    left = [None] * (n + 1)
    right = [None] * (n + 1)
    left[0], right[n] = strip.left, strip.right
    if side != "right":
        for k in range(n):
            s = strip.sites[k]
            left[k + 1] = scale(step(left[k], strip, k, state[s[0], s[1]]))
    if side != "left":
        for k in range(n - 1, -1, -1):
            s = strip.sites[k]
            right[k] = scale(step(right[k + 1], strip, k, state[s[0], s[1]]))
    return left, right


def value(left: LT, right: LT) -> float:
    return scalar(join(left, right))


def site_value(left, right, strip, k, A, B=None) -> float:
    """``_diagonal_site_value``."""
    return value(step(left, strip, k, A, B), right)


def hole(left: LT, right: LT, strip: Strip, positions, output) -> T:
    """``_diagonal_hole`` (diagonal_mps.jl:415-433): the attachments of the
    given sites joined to whichever half shares more labels, then the halves."""
    pending = [A for k in positions for A in strip.attachments[k]]
    while pending:
        ls = [len(set(left.labels) & set(A.labels)) for A in pending]
        rs = [len(set(right.labels) & set(A.labels)) for A in pending]
        li, ri = int(np.argmax(ls)), int(np.argmax(rs))
        useleft = ls[li] > rs[ri] or (ls[li] == rs[ri] and len(left.labels) <= len(right.labels))
        A = pending.pop(li if useleft else ri)
        if useleft:
            left = join(left, A)
        else:
            right = join(right, A)
    return reorder(join(left, right), output).t


def site_hole(left, right, strip, k, A: T) -> T:
    """``_diagonal_site_hole`` (diagonal_mps.jl:435-443) in the layout of
    ``sampling.site_hole``: legs (wk, wb, nk, nb, ek, eb, sk, sb)."""
    H = hole(left, right, strip, [k], list(strip.ports[k]))
    for i, axis in reversed(list(enumerate(VIRTUAL_AXES))):
        H = z2.split(H, i, [A.p[axis], A.p[axis]])
    return H


# ---------------------------------------------------------------------------
# Born sampling (src/sampling/diagonal_born.jl)
# ---------------------------------------------------------------------------

class DiagonalSamplingCache:
    """``SamplingCache(state, ::BoundaryMPSDiagonal; kind)`` (diagonal_born.jl:11-21):
    the southeast boundaries of every layer and the draw order."""

    def __init__(self, state, method: BoundaryMPSDiagonal, kind="auxiliary"):
        if kind not in ("auxiliary", "physical"):
            raise ValueError("unknown sampling kind")
        self.state, self.method, self.kind = state, method, kind
        self.target = None
        if kind == "physical":
            self.target = 0
            for y in range(state.Ly):
                for x in range(state.Lx):
                    if state[x, y].shape[3] != 1:
                        raise ValueError("proposal requires PEPS")
                    self.target ^= int(state[x, y].p[3][0])
        _, self.southeast = boundaries(state, method, side="southeast")
        self.order = draw_order(state.Lx, state.Ly)


def sample_configuration(cache: DiagonalSamplingCache, uniforms=None, configuration=None):
    """``sample_configuration`` for the diagonal method (diagonal_born.jl:24-97).

    Sites are drawn layer by layer in ``draw_order``; ``uniforms[i]`` is the
    uniform of the i-th site drawn.  Each layer is sampled inside a strip
    between the projected northwest boundary and the cached southeast one,
    then absorbed into the northwest boundary (the physical kind skips the
    last layer).  Configuration labels are 1/2 indexed [x][y]."""
    from .sampling import project, project_physical, born_probabilities, categorical, positive_metric_root
    st = cache.state
    Lx, Ly = st.Lx, st.Ly
    N = Lx * Ly
    nl = layer_count(Lx, Ly)
    physical = cache.kind == "physical"
    if uniforms is None and configuration is None:
        raise ValueError("an explicit RNG is required")
    selected = [[0] * Ly for _ in range(Lx)] if configuration is None else [list(c) for c in configuration]
    if configuration is not None:
        for x in range(Lx):
            for y in range(Ly):
                if selected[x][y] not in (1, 2):
                    raise ValueError("configuration contains an unknown basis label")
    nw = DiagonalBoundary()
    projected = {}
    logp = 0.0
    conditionals, repairs = [], []
    maxtr = cache.southeast[0].max_truncation

    def result(lp):
        return dict(configuration=selected, log_probability=lp, conditionals=conditionals,
                    max_environment_truncation=maxtr, repairs=repairs)

    if configuration is not None and physical:
        charge = 0
        for x in range(Lx):
            for y in range(Ly):
                charge ^= int(st[x, y].p[2][selected[x][y] - 1])
        if charge != cache.target:
            return result(-math.inf)
    prefix = 0
    position = 0
    proj = project_physical if physical else project
    for t in range(nl):
        strip = Strip(st, t, t, nw, cache.southeast[t + 1])
        rightward = t % 2 == 0
        le, ri = messages(st, strip, side="right" if rightward else "left")
        message = strip.left if rightward else strip.right
        n = len(strip.sites)
        for k in (range(n) if rightward else range(n - 1, -1, -1)):
            x, y = strip.sites[k]
            A = st[x, y]
            left = message if rightward else le[k]
            right = ri[k + 1] if rightward else message
            if physical:
                allowed = [position < N - 1 or (prefix ^ int(A.p[2][j])) == cache.target for j in (0, 1)]
            else:
                allowed = [True, True]
            if not any(allowed):
                raise RuntimeError("sampling prefix violates the total symmetry sector")
            cands = [proj(A, j) for j in (0, 1)]
            if physical:
                roots, diag = positive_metric_root(site_hole(left, right, strip, k, A))
                repairs.append(dict(diag, site=(x + 1, y + 1)))
                values = []
                for j in (0, 1):
                    if not allowed[j]:
                        values.append(0.0)
                        continue
                    vb = z2.MatView(cands[j], [0, 1, 4, 5], [2, 3]).blocks
                    values.append(sum(float(np.sum((r.T @ b) ** 2)) for r, b in zip(roots, vb) if r.size and b.size))
                total = sum(values)
                if total == 0:
                    m = sum(allowed)
                    probs = [1.0 / m if a else 0.0 for a in allowed]
                    repairs.append(dict(site=(x + 1, y + 1), reason="zero_proposal_weights", allowed_outcomes=m))
                else:
                    probs = [v / total for v in values]
            else:
                raw = [site_value(left, right, strip, k, C) for C in cands]
                probs = born_probabilities(raw, x, y)
            if configuration is None:
                lm = [math.log(p) if p > 0 else -math.inf for p in probs]
                j = categorical(lm, uniforms[position])
            else:
                j = selected[x][y] - 1
            selected[x][y] = j + 1
            p = probs[j]
            conditionals.append(p)
            position += 1
            if p == 0.0:
                return result(-math.inf)
            logp += math.log(p)
            projected[(x, y)] = cands[j]
            prefix ^= int(A.p[2][j])
            message = scale(step(message, strip, k, cands[j]))
        if not physical or t < nl - 1:
            absorb_layer(nw, lambda s: projected[s], Lx, Ly, t, cache.method)
            maxtr = max(maxtr, nw.max_truncation)
    return result(logp)


# ---------------------------------------------------------------------------
# energy (src/measurement/diagonal_energy.jl, diagonal_update.jl:54-59)
# ---------------------------------------------------------------------------

def layer_bonds(Lx, Ly, t, direction, reverse=False):
    """``_diagonal_layer_bonds``: bonds from layer t to layer t+1."""
    dx, dy = (1, 0) if direction == "horizontal" else (0, 1)
    return [((x, y), (x + dx, y + dy)) for (x, y) in draw_sites(Lx, Ly, t, reverse)
            if x + dx < Lx and y + dy < Ly]


def pair_value(state, strip, le, ri, i, j, A, B) -> float:
    """``_diagonal_pair_value`` (diagonal_energy.jl:1-10): kets A at i and B at j."""
    a, b = strip.sites.index(i), strip.sites.index(j)
    if abs(a - b) != 1:
        raise RuntimeError("nonadjacent diagonal observable")
    message = le[min(a, b)]
    for k in range(min(a, b), max(a, b) + 1):
        s = strip.sites[k]
        message = step(message, strip, k, A if s == i else B, state[s[0], s[1]])
    return value(message, ri[max(a, b) + 1])


def measure_energy(state, model, method: BoundaryMPSDiagonal, record_entropy=False):
    """``measure_energy`` for the diagonal method (diagonal_energy.jl:12-45),
    with the per-site <X_i> and sums of ``sampling.measure_energy``."""
    from . import boundary as bm
    from .model import spin_operators
    from .sampling import operator_factors, operator_pair, real_ratio
    Lx, Ly = state.Lx, state.Ly
    nl = layer_count(Lx, Ly)
    entropy = DiagonalEntropy(Lx, Ly, profile=True) if record_entropy else None
    nw, se = boundaries(state, method, entropy=entropy)
    X, _, _ = spin_operators()
    F, G = operator_factors()
    site_x = np.zeros((Lx, Ly))
    xsum = zzsum = 0.0
    for t in range(nl):
        strip = Strip(state, t, t, nw[t], se[t + 1])
        le, ri = messages(state, strip)
        for k, (x, y) in enumerate(strip.sites):
            A = state[x, y]
            den = site_value(le[k], ri[k + 1], strip, k, A)
            num = site_value(le[k], ri[k + 1], strip, k, bm.act(A, X, 2, out_par=A.p[2]), A)
            r = real_ratio(num, den)
            site_x[x, y] = r
            xsum += r
        if t == nl - 1:
            continue
        strip = Strip(state, t, t + 1, nw[t], se[t + 2])
        le, ri = messages(state, strip)
        for direction in ("horizontal", "vertical"):
            for i, j in layer_bonds(Lx, Ly, t, direction):
                C, D = operator_pair(state[i[0], i[1]], state[j[0], j[1]], F, G, direction)
                num = pair_value(state, strip, le, ri, i, j, C, D)
                den = pair_value(state, strip, le, ri, i, j, state[i[0], i[1]], state[j[0], j[1]])
                zzsum += real_ratio(num, den)
    final = nw[nl]
    log_norm = math.log(bm.positive_real(final.scalar, "norm")) + final.log_scale
    hx = xsum * model.h if getattr(model, "fields", None) is None else float(
        sum(model.field(x, y, Lx) * site_x[x, y] for x in range(Lx) for y in range(Ly)))
    et = -model.J * zzsum - hx
    return dict(energy_total=et, energy_per_site=et / (Lx * Ly), log_norm=log_norm + 2 * state.log_amplitude,
                tensor_log_norm=log_norm, max_environment_truncation=max(final.max_truncation,
                                                                          se[0].max_truncation),
                Se=(entropy.Se if entropy is not None else None),
                max_boundary_entropy=(entropy.maximum if entropy is not None else math.nan),
                x_sum=xsum, magnetization=xsum / (Lx * Ly), site_x=site_x, zz_sum=zzsum)


# ---------------------------------------------------------------------------
# full-update bond environments (src/evolution/diagonal_update.jl)
# ---------------------------------------------------------------------------

def external_axes(direction):
    """``_diagonal_external_axes``: the exterior virtual legs of the bond's two
    sites, in the order of the reduced pair's Q factors."""
    return ((0, 1, 5), (1, 4, 5)) if direction == "horizontal" else ((0, 1, 4), (0, 4, 5))


@dataclass
class DiagonalBondEnvironment:
    """``DiagonalBondEnvironment`` (diagonal_update.jl:1-20)."""
    strip: Strip
    left: LT
    right: LT
    positions: tuple
    first: tuple
    second: tuple
    direction: str
    outer: tuple   # parities of the six exterior legs


def bond_environment(state, strip, left, right, i, j, direction):
    """``_diagonal_bond_environment`` (diagonal_update.jl:13-20)."""
    a, b = strip.sites.index(i), strip.sites.index(j)
    if abs(a - b) != 1:
        raise RuntimeError("bond sites must be adjacent in a diagonal strip")
    ax = external_axes(direction)
    outer = tuple(state[i[0], i[1]].p[k] for k in ax[0]) + tuple(state[j[0], j[1]].p[k] for k in ax[1])
    return DiagonalBondEnvironment(strip, left, right, (min(a, b), max(a, b)), i, j, direction, outer)


def bond_hole(env: DiagonalBondEnvironment) -> T:
    """``bond_hole`` (diagonal_update.jl:21-29): the six exterior double legs of
    the bond, each split (ket, bra), in the layout of ``boundary.bond_hole``."""
    ax = external_axes(env.direction)
    ports = [ports_of(env.first), ports_of(env.second)]
    output = [ports[k][VIRTUAL_AXES.index(a)] for k in (0, 1) for a in ax[k]]
    H = hole(env.left, env.right, env.strip, list(range(env.positions[0], env.positions[1] + 1)), output)
    for k in range(5, -1, -1):
        H = z2.split(H, k, [env.outer[k], env.outer[k]])
    return H


def core_site(Q: T, direction, first) -> T:
    """``_diagonal_core_site`` (diagonal_update.jl:32-38): a reduced factor Q
    (three exterior legs, auxiliary, core) as a site tensor whose physical leg
    is the core leg and whose bond leg is trivial."""
    ax = external_axes(direction)[0 if first else 1]
    missing = [a for a in VIRTUAL_AXES if a not in ax][0]
    site = join(LT(Q, list(ax) + [3, 2]), unit_lt(missing))
    return reorder(site, [0, 1, 2, 3, 4, 5]).t


def reduced_metric(env: DiagonalBondEnvironment, Qa: T, Qb: T) -> T:
    """``_reduced_metric(::DiagonalBondEnvironment)`` (diagonal_update.jl:39-52):
    each core site closed against its own half of the strip, the open core
    pairs joined; legs (rb, sb, rk, sk) as ``full_update.reduced_metric``."""
    A = core_site(Qa, env.direction, True)
    B = core_site(Qb, env.direction, False)

    def absorb(message, k):
        isfirst = env.strip.sites[k] == env.first
        return step(message, env.strip, k, A if isfirst else B,
                    physical=(("core", "ka"), ("core", "ba")) if isfirst else (("core", "kb"), ("core", "bb")))

    left = absorb(env.left, env.positions[0])
    right = absorb(env.right, env.positions[1])
    return reorder(join(left, right), [("core", "ba"), ("core", "bb"), ("core", "ka"), ("core", "kb")]).t


def sweep(state, model, delta, D, method, contraction: BoundaryMPSDiagonal, direction, reverse, space=None,
          entropy=None, force_repair_bonds=()):
    """``_sweep!`` for the diagonal method (diagonal_update.jl:61-102): the
    bonds from layer t to t+1 are updated in a strip of the two layers
    between the rolling boundary of the updated layers and the cached one of
    the others; the rolling boundary then absorbs the finished layer."""
    from . import full_update as fu
    from .model import trotter_gate
    Lx, Ly = state.Lx, state.Ly
    nl = layer_count(Lx, Ly)
    nw, se = boundaries(state, contraction, side="northwest" if reverse else "southeast", entropy=entropy)
    fixed = nw[1:nl + 1] if reverse else se[0:nl - 1]
    env_err = max([e.max_truncation for e in fixed], default=0.0)
    rolling = DiagonalBoundary()
    records = []
    at = lambda s: state[s[0], s[1]]
    for t in (range(nl - 2, -1, -1) if reverse else range(nl - 1)):
        strip = Strip(state, t, t + 1, nw[t] if reverse else rolling, rolling if reverse else se[t + 2])
        order = draw_sites(Lx, Ly, t, reverse)
        rightward = (not reverse) if len(order) < 2 else order[0][0] < order[-1][0]
        le, ri = messages(state, strip, side="right" if rightward else "left")
        message = strip.left if rightward else strip.right
        n = len(strip.sites)
        cursor = 0 if rightward else n - 1
        for i, j in layer_bonds(Lx, Ly, t, direction, reverse):
            a, b = sorted([strip.sites.index(i), strip.sites.index(j)])
            while (cursor < a) if rightward else (cursor > b):
                message = scale(step(message, strip, cursor, at(strip.sites[cursor])))
                cursor += 1 if rightward else -1
            left = message if rightward else le[a]
            right = ri[b + 1] if rightward else message
            env = bond_environment(state, strip, left, right, i, j, direction)
            gate = trotter_gate(model, Lx, Ly, i, j, delta)
            records.append(fu.update_bond(state, i, j, gate, D, method, env, direction,
                                          boundary_error=strip.max_truncation, space=space,
                                          force_repair=(i, j) in force_repair_bonds))
            for k in (range(a, b + 1) if rightward else range(b, a - 1, -1)):
                message = scale(step(message, strip, k, at(strip.sites[k])))
            cursor = b + 1 if rightward else a - 1
        absorb_layer(rolling, at, Lx, Ly, t + 1 if reverse else t, contraction, reverse=reverse, entropy=entropy)
        env_err = max(env_err, rolling.max_truncation)
    return records, env_err

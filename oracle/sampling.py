"""Born sampling and energy measurement for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/sampling/born.jl:27-163`` (``kind=:auxiliary``),
``src/sampling/basis.jl:36-87`` for ``SymmetryBasis``,
``src/resample/selection.jl:1-7,68-80,122-140`` and
``src/measurement/energy.jl``.  Configuration labels are the reference's
``SymmetryBasis`` labels: 1 for the even auxiliary charge, 2 for the odd one.
The random stream is replaced by explicit uniforms (one per site, row-major).
"""
from __future__ import annotations

import math

import numpy as np

from . import z2
from .z2 import T, einsum, fuse, EPS, FLOATMIN
from . import boundary as bm
from .model import State, normalize_state, spin_operators, TFIM


def project(A: T, k: int) -> T:
    """``_project(A,B,k,:auxiliary)``: keep auxiliary state k (0 even, 1 odd)."""
    return T(A.a[:, :, :, k:k + 1, :, :], [A.p[0], A.p[1], A.p[2], z2.leg(1, 0) if k == 0 else z2.leg(0, 1),
                                          A.p[4], A.p[5]])


def project_physical(A: T, k: int) -> T:
    """``_project(A,B,k,:physical)`` for ``SymmetryBasis`` (``basis.jl:64-68,87``):
    the physical leg restricted to its basis state k, a one-dimensional leg of
    that state's parity."""
    c = int(A.p[2][k])
    return T(A.a[:, :, k:k + 1, :, :, :], [A.p[0], A.p[1], z2.leg(1, 0) if c == 0 else z2.leg(0, 1),
                                          A.p[3], A.p[4], A.p[5]])


class SamplingCache:
    """``SamplingCache(state, method; kind)`` (``born.jl:56-73``).

    ``kind="auxiliary"`` labels the auxiliary leg of a PEPO; ``kind="physical"``
    the physical leg of a PEPS (the resampling proposal), whose configurations
    must fuse to the PEPS's total charge: the fusion of its one-dimensional
    auxiliary legs (``_state_charge``, ``basis.jl:89-92``)."""

    def __init__(self, state: State, method: bm.BoundaryMPS, kind="auxiliary"):
        if kind not in ("auxiliary", "physical"):
            raise ValueError("unknown sampling kind")
        self.state = state
        self.method = method
        self.kind = kind
        self.target = None
        if kind == "physical":
            self.target = 0
            for y in range(state.Ly):
                for x in range(state.Lx):
                    A = state[x, y]
                    if A.shape[3] != 1:
                        raise ValueError("proposal requires PEPS")
                    self.target ^= int(A.p[3][0])
        proj = project_physical if kind == "physical" else project
        self.layers = bm.row_layers(state)
        self.candidates = [[[bm.double_layer(proj(state[x, y], k)) for k in (0, 1)]
                            for y in range(state.Ly)] for x in range(state.Lx)]
        Ly = state.Ly
        self.south = [None] * (Ly + 1)
        self.south[Ly] = bm.trivial_boundary(bm.col(self.layers, Ly - 1), "south")
        for y in range(Ly - 1, -1, -1):
            self.south[y] = bm.absorb(self.south[y + 1], bm.col(self.layers, y), method, side="south",
                                      row_cut=y)


def logsumexp(x):
    """``_rs_logsumexp`` (``selection.jl:1-7``)."""
    if len(x) == 0:
        return -math.inf
    pivot = max(x)
    if pivot == -math.inf:
        return -math.inf
    if not math.isfinite(pivot):
        raise ValueError("nonfinite positive log mass")
    return pivot + math.log(sum(math.exp(v - pivot) for v in x))


def categorical(log_mass, u):
    """``_categorical`` (``selection.jl:68-80``) with the uniform ``u`` supplied (0-based result)."""
    z = logsumexp(log_mass)
    if not math.isfinite(z):
        raise ValueError("proposal requires positive total probability")
    cumulative = 0.0
    last = -1
    for j, lm in enumerate(log_mass):
        if lm == -math.inf:
            continue
        last = j
        cumulative += math.exp(lm - z)
        if u < cumulative:
            return j
    return last


def born_probabilities(raw, x, y):
    """Validity check and normalisation of one conditional (``born.jl:136-143``)."""
    scale = max((abs(z) for z in raw), default=0.0)
    for z in raw:
        if not (math.isfinite(z) and z >= -64 * EPS * scale):
            raise RuntimeError(f"invalid Born conditional at ({x + 1},{y + 1}); increase chi_sampling")
    values = [max(z, 0.0) for z in raw]
    total = sum(values)
    if not total > 0:
        raise RuntimeError(f"Born conditional has zero total mass at ({x + 1},{y + 1})")
    return [v / total for v in values]


def sample_configuration(cache: SamplingCache, uniforms=None, configuration=None):
    """``sample_configuration`` (``born.jl:86-163``), auxiliary kind.

    ``uniforms`` (length Lx*Ly, row-major) replaces ``rand(rng)``;
    ``configuration`` (labels 1/2, indexed [x][y]) evaluates a given draw.
    """
    if cache.kind == "physical":
        return sample_physical(cache, uniforms, configuration)
    rows = sample_rows(cache, uniforms, configuration)
    while True:
        try:
            next(rows)
        except StopIteration as done:
            return done.value


def sample_rows(cache: SamplingCache, uniforms=None, configuration=None):
    """``sample_configuration`` as a generator that yields after every row (its
    Lx conditionals and the absorption of the chosen row into the north
    boundary); the draw's result is the generator's return value.  Lets a
    caller time a draw row by row."""
    Lx, Ly = cache.state.Lx, cache.state.Ly
    if uniforms is None and configuration is None:
        raise ValueError("an explicit RNG is required")
    selected = [[0] * Ly for _ in range(Lx)] if configuration is None else [list(c) for c in configuration]
    north = bm.trivial_boundary(bm.col(cache.layers, 0), "north")
    logp = 0.0
    conditionals = []
    raws = []
    maxtr = max(e.max_truncation for e in cache.south)
    for y in range(Ly):
        row = bm.col(cache.layers, y)
        top = north.tensors
        bottom = cache.south[y + 1].tensors
        _, ri = bm.row_environments(top, row, bottom, side="right")
        left = bm.row_edge(top, row, bottom, "left")
        for x in range(Lx):
            cands = cache.candidates[x][y]
            raw = [bm.row_scalar(left, top[x], E, bottom[x], ri[x + 1]) for E in cands]
            raws.append(raw)
            probs = born_probabilities(raw, x, y)
            if configuration is None:
                lm = [math.log(p) if p > 0 else -math.inf for p in probs]
                k = categorical(lm, uniforms[x + y * Lx])
            else:
                k = selected[x][y] - 1
            selected[x][y] = k + 1
            p = probs[k]
            conditionals.append(p)
            if p == 0.0:
                return dict(configuration=selected, log_probability=-math.inf, conditionals=conditionals,
                            max_environment_truncation=maxtr, raw=raws)
            logp += math.log(p)
            row[x] = cands[k]
            if x < Lx - 1:
                left = bm.safe_scale(bm.left_step(left, top[x], row[x], bottom[x]))
        north = bm.absorb(north, row, cache.method, row_cut=y + 1)
        maxtr = max(maxtr, north.max_truncation)
        yield y
    return dict(configuration=selected, log_probability=logp, conditionals=conditionals,
                max_environment_truncation=maxtr, raw=raws)


def site_hole(L: T, Tt: T, B: T, R: T, A: T) -> T:
    """``_site_hole`` (``born.jl:75-84``): the row environments around one site,
    each fused double-layer leg split into (ket, bra); legs (wk,wb,nk,nb,ek,eb,sk,sb)."""
    X = einsum("awb,anc->wbnc", L, Tt)
    Y = einsum("bsd,ced->bsce", B, R)
    H = einsum("wbnc,bsce->wnes", X, Y)
    for k, axis in reversed(list(enumerate((0, 1, 4, 5)))):
        H = z2.split(H, k, [A.p[axis], A.p[axis]])
    return H


def positive_metric_root(H: T):
    """``_positive_metric(N; square_root=true)`` (``tensors.jl:65-94``) of a site
    hole: scaled by its Frobenius norm, symmetrised, eigendecomposed per parity
    block, negative eigenvalues clipped.  Returns per block the eigenvectors
    times the square roots of the clipped eigenvalues (rows in the bra-leg
    order of the (bras | kets) view, which is also the ket-leg order), and the
    diagnostic record."""
    if not np.all(np.isfinite(H.a)):
        raise RuntimeError("nonfinite norm metric")
    scale = z2.norm(H)
    v = z2.MatView(H, [1, 3, 5, 7], [0, 2, 4, 6])
    roots, vals = [], []
    defect_num = defect_den = 0.0
    for b in v.blocks:
        M = b / scale if scale != 0 else b.copy()
        defect_num += float(np.sum((M - M.T) ** 2))
        defect_den += float(np.sum(M * M))
        M = 0.5 * (M + M.T)
        if M.size == 0:
            roots.append(np.zeros((M.shape[0], 0)))
            continue
        w, V = np.linalg.eigh(M)
        vals.extend(w.tolist())
        roots.append(V * np.sqrt(np.maximum(w, 0.0)))
    vals = np.asarray(vals)
    lo = min(float(vals.min()) if vals.size else 0.0, 0.0)
    hi = max(float(np.abs(vals).max()) if vals.size else 0.0, FLOATMIN)
    neg = vals[vals < 0]
    report = dict(minimum_relative_eigenvalue=lo / hi, negative_eigenvalues=int(neg.size),
                  negative_multiplets=int(neg.size),
                  negative_spectral_fraction=float(np.sqrt(np.sum(neg * neg)) / max(np.sqrt(np.sum(vals * vals)),
                                                                                    FLOATMIN)),
                  hermiticity_defect=math.sqrt(defect_num) / max(math.sqrt(defect_den), FLOATMIN))
    return roots, report


def sample_physical(cache: SamplingCache, uniforms=None, configuration=None):
    """``sample_configuration`` for ``kind=:physical`` (``born.jl:86-163``).

    Each conditional weighs the site's two physically projected kets with the
    PSD-projected site hole (``born.jl:117-126``); outcomes that cannot reach
    the total charge get no weight (``born.jl:110-116``: with both parities
    available at every site only the last site is bound); all-zero weights
    fall back to the uniform choice among the allowed outcomes
    (``born.jl:127-131``); the last row is not absorbed (``born.jl:155-158``).
    ``repairs`` holds one diagnostic record per site plus the zero-weight ones.
    """
    st = cache.state
    Lx, Ly = st.Lx, st.Ly
    N = Lx * Ly
    if uniforms is None and configuration is None:
        raise ValueError("an explicit RNG is required")
    selected = [[0] * Ly for _ in range(Lx)] if configuration is None else [list(c) for c in configuration]
    north = bm.trivial_boundary(bm.col(cache.layers, 0), "north")
    maxtr = max(e.max_truncation for e in cache.south)
    logp = 0.0
    conditionals, repairs = [], []

    def result(lp):
        return dict(configuration=selected, log_probability=lp, conditionals=conditionals,
                    max_environment_truncation=maxtr, repairs=repairs)

    if configuration is not None:
        charge = 0
        for x in range(Lx):
            for y in range(Ly):
                lab = selected[x][y]
                if lab not in (1, 2):
                    raise ValueError("configuration contains an unknown basis label")
                charge ^= int(st[x, y].p[2][lab - 1])
        if charge != cache.target:
            return result(-math.inf)
    prefix = 0
    for y in range(Ly):
        row = bm.col(cache.layers, y)
        top = north.tensors
        bottom = cache.south[y + 1].tensors
        _, ri = bm.row_environments(top, row, bottom, side="right")
        left = bm.row_edge(top, row, bottom, "left")
        for x in range(Lx):
            position = x + y * Lx
            A = st[x, y]
            allowed = [position < N - 1 or (prefix ^ int(A.p[2][k])) == cache.target for k in (0, 1)]
            if not any(allowed):
                raise RuntimeError("sampling prefix violates the total symmetry sector")
            roots, diag = positive_metric_root(site_hole(left, top[x], bottom[x], ri[x + 1], A))
            repairs.append(dict(diag, site=(x + 1, y + 1)))
            values = []
            for k in (0, 1):
                if not allowed[k]:
                    values.append(0.0)
                    continue
                vb = z2.MatView(project_physical(A, k), [0, 1, 4, 5], [2, 3]).blocks
                values.append(sum(float(np.sum((r.T @ b) ** 2)) for r, b in zip(roots, vb) if r.size and b.size))
            total = sum(values)
            if total == 0:
                n = sum(allowed)
                probs = [1.0 / n if a else 0.0 for a in allowed]
                repairs.append(dict(site=(x + 1, y + 1), reason="zero_proposal_weights", allowed_outcomes=n))
            else:
                probs = [v / total for v in values]
            if configuration is None:
                lm = [math.log(p) if p > 0 else -math.inf for p in probs]
                k = categorical(lm, uniforms[position])
            else:
                k = selected[x][y] - 1
            selected[x][y] = k + 1
            p = probs[k]
            conditionals.append(p)
            if p == 0.0:
                return result(-math.inf)
            logp += math.log(p)
            row[x] = cache.candidates[x][y][k]
            prefix ^= int(A.p[2][k])
            if x < Lx - 1:
                left = bm.safe_scale(bm.left_step(left, top[x], row[x], bottom[x]))
        if y < Ly - 1:
            north = bm.absorb(north, row, cache.method, row_cut=y + 1)
            maxtr = max(maxtr, north.max_truncation)
    return result(logp)


def project_configuration(checkpoint: State, configuration):
    """``project_configuration`` (``born.jl:27-36``)."""
    sites = [[project(checkpoint[x, y], configuration[x][y] - 1) for y in range(checkpoint.Ly)]
             for x in range(checkpoint.Lx)]
    st = State(checkpoint.Lx, checkpoint.Ly, sites, checkpoint.beta, checkpoint.log_amplitude, "peps")
    records = normalize_state(st)
    return st, records


def group_configurations(configurations):
    """``_group_configurations`` (``selection.jl:122-140``), 0-based draws."""
    first, mult, d2g = [], [], []
    lookup = {}
    for d, x in enumerate(configurations):
        key = tuple(v for colv in x for v in colv)
        j = lookup.get(key)
        if j is None:
            first.append(d)
            mult.append(0)
            j = len(first) - 1
            lookup[key] = j
        mult[j] += 1
        d2g.append(j)
    return dict(first_draw=first, multiplicity=mult, draw_to_group=d2g)


# ---------------------------------------------------------------------------
# energy (src/measurement/energy.jl)
# ---------------------------------------------------------------------------

def real_ratio(a, b):
    """``_real_ratio`` (``energy.jl:1-6``)."""
    if b == 0:
        raise RuntimeError("zero local norm environment")
    z = a / b
    if not math.isfinite(z):
        raise RuntimeError(f"nonreal observable: {z}")
    return float(z)


def operator_factors():
    """``_operator_factors(ZZ)`` (``energy.jl:8-12``): F[p,u,r], G[r,q,v]."""
    _, _, ZZ = spin_operators()
    P2 = z2.leg(1, 1)
    M = T(ZZ, [P2] * 4)
    nrm = z2.norm(M)
    U, S, V, _, _ = z2.svd_trunc(z2.perm(M, (0, 2, 1, 3)), [0, 1], [2, 3], atol=64 * EPS * nrm)
    s = np.concatenate(S)
    F = T(U.a * s[None, None, :], U.p)
    return F, V


def operator_pair(A, B, F, G, direction):
    """``_operator_pair`` (``energy.jl:13-23``)."""
    if direction == "horizontal":
        C = einsum("wnuaes,pur->wnpaers", A, F)
        D = einsum("wnvaes,rqv->wrnqaes", B, G)
        return fuse(C, 4, 2), fuse(D, 0, 2)
    C = einsum("wnuaes,pur->wnpaesr", A, F)
    D = einsum("wnvaes,rqv->wnrqaes", B, G)
    return fuse(C, 5, 2), fuse(D, 1, 2)


def measure_energy(state: State, model: TFIM, method: bm.BoundaryMPS, record_entropy=False):
    """``measure_energy`` (``energy.jl:31-78``).

    Also returns ``x_sum`` = sum_i <X_i> (the on-site ratio sum the
    reference forms at ``energy.jl:43-46``), exposed as a magnetisation.
    """
    Lx, Ly = state.Lx, state.Ly
    layers = bm.row_layers(state)
    entropy = bm.Entropy(Lx, Ly) if record_entropy else None
    north, south, mx = bm.boundary_environments(layers, method, entropy=entropy)
    X, _, _ = spin_operators()
    Xl = [[bm.double_layer(state[x, y], physical=X) for y in range(Ly)] for x in range(Lx)]
    F, G = operator_factors()
    xsum = 0.0
    zzsum = 0.0
    site_x = np.zeros((Lx, Ly))
    for y in range(Ly):
        row = bm.col(layers, y)
        top = north[y].tensors
        bottom = south[y + 1].tensors
        le, ri = bm.row_environments(top, row, bottom)
        for x in range(Lx):
            den = bm.row_scalar(le[x], top[x], row[x], bottom[x], ri[x + 1])
            num = bm.row_scalar(le[x], top[x], Xl[x][y], bottom[x], ri[x + 1])
            r = real_ratio(num, den)
            site_x[x, y] = r
            xsum += r
        for x in range(Lx - 1):
            A, B = state[x, y], state[x + 1, y]
            C, D = operator_pair(A, B, F, G, "horizontal")
            left = bm.left_step(le[x], top[x], bm.double_layer(C, A), bottom[x])
            num = bm.row_scalar(left, top[x + 1], bm.double_layer(D, B), bottom[x + 1], ri[x + 2])
            left = bm.left_step(le[x], top[x], row[x], bottom[x])
            den = bm.row_scalar(left, top[x + 1], row[x + 1], bottom[x + 1], ri[x + 2])
            zzsum += real_ratio(num, den)
    for y in range(Ly - 1):
        row = [bm.Slab(layers[x][y], layers[x][y + 1]) for x in range(Lx)]
        top = north[y].tensors
        bottom = south[y + 2].tensors
        le, ri = bm.row_environments(top, row, bottom)
        for x in range(Lx):
            A, B = state[x, y], state[x, y + 1]
            C, D = operator_pair(A, B, F, G, "vertical")
            imp = bm.Slab(bm.double_layer(C, A), bm.double_layer(D, B))
            den = bm.row_scalar(le[x], top[x], row[x], bottom[x], ri[x + 1])
            num = bm.row_scalar(le[x], top[x], imp, bottom[x], ri[x + 1])
            zzsum += real_ratio(num, den)
    final = north[Ly]
    log_norm = math.log(bm.positive_real(bm.close_boundary(final.tensors), "norm")) + final.log_scale
    hx = xsum * model.h if model.fields is None else float(
        sum(model.field(x, y, Lx) * site_x[x, y] for x in range(Lx) for y in range(Ly)))
    et = -model.J * zzsum - hx
    return dict(energy_total=et, energy_per_site=et / (Lx * Ly), log_norm=log_norm + 2 * state.log_amplitude,
                tensor_log_norm=log_norm, max_environment_truncation=mx,
                Se=(entropy.Se if entropy is not None else None), x_sum=xsum,
                magnetization=xsum / (Lx * Ly), site_x=site_x, zz_sum=zzsum)

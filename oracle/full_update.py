"""Full update (environment-gauged ALS) for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/evolution/full_update.jl`` (whole file, including the PSD
repair path) for Z2 dense tensors.  0-based indices throughout.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import z2
from .z2 import T, einsum, perm, norm, dot, EPS, FLOATMIN
from . import boundary as bm
from .model import trotter_gate, onsite_gate, normalize_state, TFIM

RESIDUAL_ROUNDOFF_TOLERANCE = 1e-8


@dataclass
class FullUpdate:
    """``FullUpdate`` options (``full_update.jl:11-17``)."""
    max_iterations: int = 4
    error_tolerance: float = 1e-8
    diagonal_shift: float = 1e-10
    linear_max_iterations: int = 24
    linear_tolerance: float = 1e-9


class RepairNeeded(Exception):
    pass


PA = {"horizontal": (0, 1, 5, 3, 2, 4), "vertical": (0, 1, 4, 3, 2, 5)}
PB = {"horizontal": (1, 4, 5, 3, 2, 0), "vertical": (0, 4, 5, 3, 2, 1)}


def invperm(p):
    out = [0] * len(p)
    for i, k in enumerate(p):
        out[k] = i
    return tuple(out)


def reduced_pair(A, B, gate, direction):
    """``_reduced_pair`` (``full_update.jl:21-29``)."""
    pa, pb = PA[direction], PB[direction]
    Qa, Ca = z2.qr(perm(A, pa), [0, 1, 2, 3], [4, 5])
    Qb, Cb = z2.qr(perm(B, pb), [0, 1, 2, 3], [4, 5])
    b = perm(Cb, (2, 1, 0))
    target = einsum("ruk,kvs,pquv->rpqs", Ca, b, gate)
    return dict(Qa=Qa, Qb=Qb, target=target, pa=pa, pb=pb)


def fu_svd_initial(target, D, space):
    """``_fu_svd_initial`` (``full_update.jl:31-42``)."""
    cutoff = EPS * max(target.shape) * norm(target)
    U, S, V, _, _ = z2.svd_trunc(target, [0, 1], [2, 3], chi=D, space=space, atol=cutoff)
    if len(S[0]) + len(S[1]) == 0:
        raise RuntimeError("gate produced a zero target")
    root = np.sqrt(np.concatenate(S))
    left = T(U.a * root[None, None, :], U.p)
    right = T(V.a * root[:, None, None], V.p)
    return left, right


def svd_compact_2leg(C):
    v, bl = z2.svd_blocks(C, [0], [1])
    us = [b[0] for b in bl]
    ss = [b[1] for b in bl]
    vs = [b[2] for b in bl]
    nl = z2.leg(len(ss[0]), len(ss[1]))
    U = z2.from_blocks(us, v.rp, [nl])
    V = z2.from_blocks(vs, [nl], v.cp)
    return U, np.concatenate(ss), V


def fu_balance_bond(QA, C, QB):
    """``_fu_balance_bond`` (``full_update.jl:45-52``)."""
    U, s, V = svd_compact_2leg(C)
    root = np.sqrt(s)
    Ur = T(U.a * root[None, :], U.p)
    Vr = T(V.a * root[:, None], V.p)
    A = einsum("fpb,bk->fpk", QA, Ur)
    B = einsum("kb,bqs->kqs", Vr, QB)
    return A, B


def fu_transform_metric(N, Li, Ri):
    """``_fu_transform_metric`` (``full_update.jl:55-62``)."""
    first = einsum("ijkl,ix->jklx", N, Li)
    second = einsum("jklx,jy->klxy", first, Ri)
    third = einsum("klxy,kz->lxyz", second, Li)
    return einsum("lxyz,lw->xyzw", third, Ri)


def block_inverse(R):
    """inv of a square 2-leg block matrix (out,in) -> (in,out)."""
    v = z2.MatView(R, [0], [1])
    inv = [np.linalg.inv(b) if b.size else np.zeros((b.shape[1], b.shape[0])) for b in v.blocks]
    return z2.from_blocks(inv, v.cp, v.rp)


def eigh_blocks(H4):
    """Per-block eigendecomposition of a (rb,sb;rk,sk) metric; returns (values, vectors tensor)."""
    v = z2.MatView(H4, [0, 1], [2, 3])
    vals, vecs = [], []
    for b in v.blocks:
        if b.size == 0:
            vals.append(np.zeros(0))
            vecs.append(np.zeros((b.shape[0], 0)))
            continue
        w, V = np.linalg.eigh(b)
        vals.append(w)
        vecs.append(V)
    nl = z2.leg(len(vals[0]), len(vals[1]))
    Vt = z2.from_blocks(vecs, v.rp, [nl])
    return vals, Vt


def fu_environment_gauge(N):
    """``_fu_environment_gauge`` (``full_update.jl:72-106``)."""
    if not np.all(np.isfinite(N.a)):
        raise RuntimeError("nonfinite FU norm metric")
    scale = norm(N)
    if not scale > 0:
        raise RuntimeError("zero FU norm metric")
    nrm = N / scale
    H = T(0.5 * (nrm.a + np.transpose(nrm.a, (2, 3, 0, 1))), nrm.p)
    vals, Vt = eigh_blocks(H)
    allv = np.concatenate(vals)
    spectral = float(np.max(np.abs(allv))) if allv.size else 0.0
    relative_floor = max(math.sqrt(EPS), N.shape[2] * N.shape[3] * EPS)
    spectral = 1.0 if spectral == 0.0 else spectral
    floor = relative_floor * spectral
    floored = int(np.sum(allv < floor))
    root = np.sqrt(np.maximum(allv, floor))
    Z = T(np.transpose(Vt.a, (2, 0, 1)) * root[:, None, None], [Vt.p[2], Vt.p[0], Vt.p[1]])
    _, left = z2.qr(Z, [0, 2], [1])
    _, right = z2.qr(Z, [0, 1], [2])
    Li = block_inverse(left)
    Ri = block_inverse(right)
    metric = fu_transform_metric(N, Li, Ri)
    diag = dict(relative_floor=relative_floor, floored_multiplets=floored,
                floored_eigenvalues=floored,
                minimum_relative_eigenvalue=float(allv.min() / spectral) if allv.size else math.inf,
                hermiticity_defect=float(np.sqrt(np.sum((nrm.a - np.transpose(nrm.a, (2, 3, 0, 1))) ** 2))))
    return dict(left=left, right=right, left_inverse=Li, right_inverse=Ri, metric=metric, diagnostic=diag)


def act(A, O, axis):
    """``_act`` with a 2-leg tensor O[out,in] acting on leg ``axis``."""
    a = np.tensordot(O.a, A.a, axes=([1], [axis]))
    a = np.moveaxis(a, 0, axis)
    p = list(A.p)
    p[axis] = O.p[0]
    return T(a, p)


def initialize_pair(pair, N, D, space):
    """``_initialize_pair`` (``full_update.jl:108-115``)."""
    g = fu_environment_gauge(N)
    wt = act(act(pair["target"], g["left"], 0), g["right"], 3)
    left, right = fu_svd_initial(wt, D, space)
    out = dict(pair)
    out.update(left=left, right=right, working_target=wt, working_metric=g["metric"],
               left_inverse=g["left_inverse"], right_inverse=g["right_inverse"],
               gauge_diagnostic=g["diagnostic"])
    return out


def fu_original_cores(pair, A, B):
    return act(A, pair["left_inverse"], 0), act(B, pair["right_inverse"], 2)


def restore_pair(pair, A, B):
    """``_restore_pair`` (``full_update.jl:128-133``)."""
    first = einsum("uvwar,rpb->uvwapb", pair["Qa"], A)
    second = einsum("uvwar,bpr->uvwapb", pair["Qb"], B)
    return perm(first, invperm(pair["pa"])), perm(second, invperm(pair["pb"]))


def reduced_layer(Q):
    """``_reduced_layer`` (``full_update.jl:143-149``): legs (w,n,e,rb,rk)."""
    A = einsum("wneuk,WNEub->wWnNeEbk", Q, Q)
    for k in (4, 2, 0):
        A = z2.fuse(A, k, 2)
    return A


def reduced_metric(env, Qa, Qb):
    """``_reduced_metric(::BondEnvironment,...)`` (``full_update.jl:151-172``);
    a diagonal bond environment takes ``diagonal.reduced_metric``."""
    from . import diagonal as dg
    if isinstance(env, dg.DiagonalBondEnvironment):
        return dg.reduced_metric(env, Qa, Qb)
    A = reduced_layer(Qa)
    B = reduced_layer(Qb)
    left, right = env.left, env.right
    if env.direction == "horizontal":
        T1, T2 = env.top
        B1, B2 = env.bottom
        X = einsum("awb,anc->bncw", left, T1)
        Y = einsum("bncw,wnsBK->bcsBK", X, A)
        L = einsum("bcsBK,bsf->cfBK", Y, B1)
        U = einsum("deg,cvd->cveg", right, T2)
        V = einsum("cveg,vetSP->cgtSP", U, B)
        R = einsum("cgtSP,ftg->cfSP", V, B2)
        return einsum("cfBK,cfSP->BSKP", L, R)
    Tt = env.top[0]
    bot = env.bottom[0]
    X = einsum("awvb,anc->wvbnc", left, Tt)
    Y = einsum("wvbnc,wneBK->vbceBK", X, A)
    L = einsum("vbceBK,cefd->vbfdBK", Y, right)
    R = einsum("vfsSP,bsd->vfSPbd", B, bot)
    return einsum("vbfdBK,vfSPbd->BSKP", L, R)


def positive_reduced_metric(env, Qa, Qb):
    """``_positive_reduced_metric`` (``full_update.jl:278-340``).

    Projects the complete bond hole (an operator on the exterior ket legs)
    onto its positive spectrum, scaled by its Frobenius norm, and reduces it
    with Qa, Qb.  The reference forms the same operator in a grouped
    two-leg basis to save memory; the positive projection is basis
    independent, so the result agrees to roundoff.
    """
    from . import diagonal as dg
    H = dg.bond_hole(env) if isinstance(env, dg.DiagonalBondEnvironment) else bm.bond_hole(env)
    # legs (k1,b1,k2,b2,...,k6,b6)
    kets = [0, 2, 4, 6, 8, 10]
    bras = [1, 3, 5, 7, 9, 11]
    if not np.all(np.isfinite(H.a)):
        raise RuntimeError("nonfinite norm metric")
    scale = norm(H)
    v = z2.MatView(H, bras, kets)
    blocks = []
    negative = 0
    minimum = 0.0
    spectral = 0.0
    for b in v.blocks:
        if b.size == 0:
            blocks.append(b.copy())
            continue
        M = b / scale if scale != 0 else b.copy()
        M = 0.5 * (M + M.T)
        w, V = np.linalg.eigh(M)
        minimum = min(minimum, float(w.min()))
        spectral = max(spectral, float(np.abs(w).max()))
        negative += int(np.sum(w < 0))
        pos = w > 0
        blocks.append((V[:, pos] * w[pos]) @ V[:, pos].T)
    Hp = z2.from_blocks(blocks, v.rp, v.cp)   # legs (b1..b6, k1..k6)
    H12 = perm(Hp, (6, 0, 7, 1, 8, 2, 9, 3, 10, 4, 11, 5))
    N = einsum("aAbBcCdDeEfF,abcuK,ABCuk,defvS,DEFvs->ksKS", H12, Qa, Qa, Qb, Qb)
    report = dict(minimum_relative_eigenvalue=minimum / max(spectral, FLOATMIN),
                  negative_multiplets=negative)
    return N, report


def apply_pair_metric(N, theta):
    return einsum("rstu,tpqu->rpqs", N, theta)


def pair_tensor(A, B):
    return einsum("rpb,bqs->rpqs", A, B)


def residual_cost(N, A, B, target):
    res = pair_tensor(A, B) - target
    return dot(res, apply_pair_metric(N, res))


def repair_trigger(raw, target):
    """``_repair_trigger`` (``full_update.jl:355-363``) for real scalars."""
    scale = max(abs(target), FLOATMIN)
    if not (math.isfinite(raw) and math.isfinite(target)):
        raise RuntimeError("nonfinite FU residual/target")
    if raw / scale < -RESIDUAL_ROUNDOFF_TOLERANCE:
        return "negative_residual"
    if target < 0:
        return "negative_target_norm"
    return None


def cost_evaluation(raw, target):
    """``_cost_evaluation`` (``full_update.jl:364-369``)."""
    rel = raw / max(abs(target), FLOATMIN)
    if not math.isfinite(rel):
        raise RuntimeError("nonfinite relative FU residual")
    if rel < -RESIDUAL_ROUNDOFF_TOLERANCE:
        raise RuntimeError("negative FU residual needs PSD repair")
    return abs(rel), rel < 0, rel


def solve_core(metric, rhs, initial, opt: FullUpdate):
    """``_solve_core`` (``full_update.jl:371-400``): Jacobi-preconditioned CG.

    ``metric`` is a 4-leg (a,b;c,d) tensor, ``rhs``/``initial`` are 3-leg
    (a,b,physical); the operator acts on the fused (a,b) index.
    """
    n = metric.shape[0] * metric.shape[1]
    M = metric.a.reshape(n, n)
    shp = rhs.shape
    b = rhs.a.reshape(n, -1)
    d = np.maximum(np.diag(M), 0.0)
    scale = float(d.max()) if d.size else 0.0
    shift = opt.diagonal_shift * max(scale, FLOATMIN)
    floor = max(shift, EPS * scale, FLOATMIN)
    den = np.maximum(d + shift, floor)[:, None]

    def action(v):
        return M @ v + shift * v

    x = initial.a.reshape(n, -1).copy()
    r = b - action(x)
    rhsnorm = max(float(np.sqrt(np.sum(b * b))), FLOATMIN)
    residual = float(np.sqrt(np.sum(r * r))) / rhsnorm
    if residual <= opt.linear_tolerance:
        return T(x.reshape(shp), rhs.p), residual
    z = r / den
    p = z.copy()
    rz = float(np.sum(r * z))
    for _ in range(opt.linear_max_iterations):
        Ap = action(p)
        curvature = float(np.sum(p * Ap))
        pn = float(np.sqrt(np.sum(p * p)))
        apn = float(np.sqrt(np.sum(Ap * Ap)))
        if not curvature > EPS * max(pn * apn, FLOATMIN):
            break
        alpha = rz / curvature
        x = x + alpha * p
        r = r - alpha * Ap
        residual = float(np.sqrt(np.sum(r * r))) / rhsnorm
        if residual <= opt.linear_tolerance:
            break
        z = r / den
        nxt = float(np.sum(r * z))
        if not nxt >= 0:
            break
        p = z + (nxt / max(rz, FLOATMIN)) * p
        rz = nxt
    return T(x.reshape(shp), rhs.p), float(residual)


def left_normal_equation(metric, right, wt):
    """``_left_normal_equation`` (``full_update.jl:402-408``)."""
    normal = einsum("fsgn,bps,opn->fbgo", metric, right, right)
    rhs = einsum("fpqs,bqs->fpb", wt, right)
    return normal, perm(rhs, (0, 2, 1))


def right_normal_equation(metric, left, wt):
    """``_right_normal_equation`` (``full_update.jl:410-416``)."""
    normal = einsum("wsen,wpb,epo->bson", metric, left, left)
    rhs = einsum("wqps,wqb->bps", wt, left)
    return normal, perm(rhs, (0, 2, 1))


def optimize_pair(pair, N, opt: FullUpdate):
    """``_optimize_pair`` (``full_update.jl:418-482``)."""
    A = pair["left"].copy()
    B = pair["right"].copy()
    target = pair["working_target"]
    metric = pair["working_metric"]
    target_norm = dot(pair["target"], apply_pair_metric(N, pair["target"]))
    oA, oB = fu_original_cores(pair, A, B)
    raw = residual_cost(N, oA, oB, pair["target"])
    trig = repair_trigger(raw, target_norm)
    if trig is not None:
        return dict(trigger=trig, stage="initial_local_svd", iteration=0, raw=raw, target_norm=target_norm)
    init_cost, init_fb, init_rel = cost_evaluation(raw, target_norm)
    bestA, bestB = oA, oB
    best = init_cost
    residual = 0.0
    best_factors = None
    fallbacks = []
    iterations = 0
    limit_reached = False
    stop = "disabled" if opt.max_iterations == 0 else "iteration_limit"
    if init_fb:
        stop = "residual_fallback"
        fallbacks.append(dict(iteration=0, relative_cost=init_rel, used_initial_local_svd=True))
    elif opt.max_iterations > 0 and best <= opt.error_tolerance:
        stop = "error_tolerance"
    elif opt.max_iterations > 0:
        wt = apply_pair_metric(metric, target)
        for it in range(1, opt.max_iterations + 1):
            MA, ya = left_normal_equation(metric, B, wt)
            sol, ra = solve_core(MA, ya, perm(A, (0, 2, 1)), opt)
            QA, R = z2.qr(sol, [0, 2], [1])           # rows (first, physical), col bond
            right_initial = einsum("nb,bqs->nqs", R, B)
            A = QA
            MB, yb = right_normal_equation(metric, A, wt)
            sol, rb = solve_core(MB, yb, perm(right_initial, (0, 2, 1)), opt)
            C, QB = z2.lq(sol, [0], [2, 1])           # rows bond, cols (physical, south)
            A = einsum("fpn,nm->fpm", QA, C)
            B = QB
            oA, oB = fu_original_cores(pair, A, B)
            raw = residual_cost(N, oA, oB, pair["target"])
            trig = repair_trigger(raw, target_norm)
            if trig is not None:
                return dict(trigger=trig, stage="als_iteration", iteration=it, raw=raw, target_norm=target_norm)
            cost, fb, rel = cost_evaluation(raw, target_norm)
            residual = max(ra, rb)
            iterations = it
            if fb:
                stop = "residual_fallback"
                fallbacks.append(dict(iteration=it, relative_cost=rel, used_initial_local_svd=False))
                break
            if cost <= best:
                best = cost
                bestA, bestB = oA, oB
                best_factors = (QA, C, QB)
            if best <= opt.error_tolerance:
                stop = "error_tolerance"
                break
            limit_reached = it == opt.max_iterations
    if best_factors is not None:
        A, B = fu_balance_bond(*best_factors)
        bestA, bestB = fu_original_cores(pair, A, B)
    return dict(trigger=None, left=bestA, right=bestB, initial_cost=init_cost, final_cost=best,
                residual=residual, iterations=iterations, iteration_limit_reached=limit_reached,
                fallbacks=fallbacks, stop_reason=stop)


def update_bond(state, i, j, gate, D, method: FullUpdate, hole, direction, boundary_error=0.0,
                space=None, force_repair=False):
    """``update_bond!`` (``full_update.jl:484-508``).

    ``force_repair`` is a test hook: it treats the first fit as triggered so
    the PSD-repair path can be exercised on well-conditioned inputs.
    """
    pair = reduced_pair(state[i], state[j], gate, direction)
    N = reduced_metric(hole, pair["Qa"], pair["Qb"])
    initial = initialize_pair(pair, N, D, space)
    fit = optimize_pair(initial, N, method)
    repairs = []
    if fit["trigger"] is not None or force_repair:
        repaired, diag = positive_reduced_metric(hole, pair["Qa"], pair["Qb"])
        repairs.append(dict(diag, reason=fit.get("trigger") or "forced"))
        initial = initialize_pair(pair, repaired, D, space)
        fit = optimize_pair(initial, repaired, method)
        if fit["trigger"] is not None:
            raise RuntimeError("PSD repair did not remove the FU residual failure")
    state[i], state[j] = restore_pair(pair, fit["left"], fit["right"])
    return dict(bond=(i, j), direction=direction, initial_cost=fit["initial_cost"],
                final_cost=fit["final_cost"], residual=fit["residual"], iterations=fit["iterations"],
                iteration_limit_reached=fit["iteration_limit_reached"], stop_reason=fit["stop_reason"],
                max_environment_truncation=boundary_error, fallbacks=fit["fallbacks"], repairs=repairs)


def sweep(state, model, delta, D, method, contraction, direction, reverse, space=None,
          entropy=None, force_repair_bonds=()):
    """``_sweep!`` for the row method (``full_update.jl:510-557``)."""
    Lx, Ly = state.Lx, state.Ly
    layers = bm.row_layers(state)
    north, south, env_err = bm.boundary_environments(layers, contraction,
                                                     side="north" if reverse else "south",
                                                     entropy=entropy)
    ymax = Ly if direction == "horizontal" else Ly - 1
    xmax = Lx - 1 if direction == "horizontal" else Lx
    records = []
    ys = range(ymax - 1, -1, -1) if reverse else range(ymax)
    for y in ys:
        top = north[y].tensors
        lastrow = y + (0 if direction == "horizontal" else 1)
        bottom = south[lastrow + 1].tensors
        if direction == "horizontal":
            row = bm.col(layers, y)
        else:
            row = [bm.Slab(layers[x][y], layers[x][y + 1]) for x in range(Lx)]
        le, ri = bm.row_environments(top, row, bottom, side="left" if reverse else "right")
        rolling = ri[Lx] if reverse else le[0]
        xs = range(xmax - 1, -1, -1) if reverse else range(xmax)
        for x in xs:
            i = (x, y)
            j = (x + 1, y) if direction == "horizontal" else (x, y + 1)
            finalx = x + 1 if direction == "horizontal" else x
            left = le[x] if reverse else rolling
            right = rolling if reverse else ri[finalx + 1]
            H = bm.bond_environment(state, layers, north, south, i, j, direction, left=left, right=right)
            gate = trotter_gate(model, Lx, Ly, i, j, delta)
            err = max(north[y].max_truncation, south[lastrow + 1].max_truncation)
            rec = update_bond(state, i, j, gate, D, method, H, direction, boundary_error=err, space=space,
                              force_repair=(i, j) in force_repair_bonds)
            records.append(rec)
            layers[i[0]][i[1]] = bm.double_layer(state[i])
            layers[j[0]][j[1]] = bm.double_layer(state[j])
            column = finalx if reverse else x
            if x != (0 if reverse else xmax - 1):
                if direction == "horizontal":
                    E = layers[column][y]
                else:
                    E = bm.Slab(layers[column][y], layers[column][y + 1])
                if reverse:
                    rolling = bm.safe_scale(bm.right_step(top[column], E, bottom[column], rolling))
                else:
                    rolling = bm.safe_scale(bm.left_step(rolling, top[column], E, bottom[column]))
        if reverse:
            south[lastrow] = bm.absorb(south[lastrow + 1], bm.col(layers, lastrow), contraction,
                                       side="south", entropy=entropy, row_cut=lastrow)
            env_err = max(env_err, south[lastrow].max_truncation)
        else:
            north[y + 1] = bm.absorb(north[y], bm.col(layers, y), contraction, entropy=entropy,
                                     row_cut=y + 1)
            env_err = max(env_err, north[y + 1].max_truncation)
    return records, env_err


def evolution_step(state, model: TFIM, delta, D, method: FullUpdate, contraction, order=2,
                   space=None, record_entropy=False, force_repair_bonds=()):
    """``evolution_step!`` (``full_update.jl:559-597``)."""
    from . import diagonal as dg, diagonal_variational as dv
    diagonal = isinstance(contraction, (dg.BoundaryMPSDiagonal, dv.BoundaryMPSDiagonalVariational))
    records = []
    env_err = 0.0
    entropy = None
    if record_entropy:
        entropy = dg.DiagonalEntropy(state.Lx, state.Ly) if diagonal else bm.Entropy()
    gate_delta = delta / 2 if order == 2 else delta
    sweeps = ([("horizontal", False), ("vertical", False), ("vertical", True), ("horizontal", True)]
              if order == 2 else [("horizontal", False), ("vertical", False)])
    if state.Lx * state.Ly == 1:
        state[0, 0] = act(state[0, 0], T(onsite_gate(model, delta), [state[0, 0].p[2]] * 2), 2)
    else:
        for direction, rev in sweeps:
            if direction == "horizontal" and state.Lx < 2:
                continue
            if direction == "vertical" and state.Ly < 2:
                continue
            r, e = (dg.sweep if diagonal else sweep)(state, model, gate_delta, D, method, contraction, direction,
                                                      rev, space=space, entropy=entropy,
                                                      force_repair_bonds=force_repair_bonds)
            records.extend(r)
            env_err = max(env_err, e)
    state.beta += 2 * delta
    norms = normalize_state(state)
    return dict(beta=state.beta, delta_tau=delta, normalizations=norms, bond_updates=len(records),
                iteration_limit_hits=sum(r["iteration_limit_reached"] for r in records),
                max_state_truncation=max([r["final_cost"] for r in records], default=0.0),
                max_environment_truncation=env_err,
                max_boundary_entropy=(entropy.maximum if entropy is not None else math.nan),
                max_solver_residual=max([r["residual"] for r in records], default=0.0),
                stop_reasons={k: sum(r["stop_reason"] == k for r in records)
                              for k in ("error_tolerance", "iteration_limit", "residual_fallback", "disabled")},
                repairs=sum(len(r["repairs"]) for r in records),
                records=records)

"""Reverse-mode derivative of the row boundary-MPS lognorm for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

The reference has no derivatives; this is the adjoint of its ``lognorm``
(``src/contraction/boundary_mps.jl:180-186``) through ``double_layer``
(:65-73), ``_absorb`` (:136-151), ``compress_boundary!`` (:94-134: the exact
LQ sweep, the truncated SVD sweep and the centre normalisation) and
``_close_boundary`` (:153-163), with respect to every site tensor: the first
piece of per-site-field gradients, which chain through it.

Each factorization is differentiated per parity block of its matrix view:
the canonical sweep by a full SVD (default) or by QR / LQ (the standard
reverse rule with the wide-matrix split), the truncated SVD through the thin
full SVD with the discarded columns' cotangents zero.  The SVD couplings
1 / (s_j^2 - s_i^2) are split into 1 / (s_j - s_i) and 1 / (s_j + s_i) terms,
each Lorentzian-broadened, d / (d^2 + eps), and 1 / s is s / (s^2 + eps).
The forward pass repeats ``boundary.lognorm`` (exact compression) and keeps
what the backward pass needs.
"""
from __future__ import annotations

import math

import numpy as np

from . import z2
from .z2 import T, einsum

BROADENING = 1e-24


def _blocks(t: T, rows, cols):
    v = z2.MatView(t, rows, cols)
    return v


def _scatter(v: z2.MatView, grads, shape_legs, order):
    """The tensor gradient of a matrix view from per-block gradients."""
    full = np.zeros((v.M, v.N))
    for c in (0, 1):
        if grads[c] is not None and grads[c].size:
            full[np.ix_(v.ridx[c], v.cidx[c])] = grads[c]
    sh = [len(p) for p in shape_legs]
    perm_shape = [sh[k] for k in order]
    arr = full.reshape(perm_shape)
    inv = np.argsort(order)
    return np.transpose(arr, inv)


def _copyltu(M):
    return np.tril(M) + np.tril(M, -1).T


def _qr_backward(A, Q, R, Qb, Rb):
    """Reverse rule of the reduced QR A = Q R (A m x n)."""
    m, n = A.shape
    if m >= n:
        M = R @ Rb.T - Qb.T @ Q
        rhs = Qb + Q @ _copyltu(M)
        # rhs R^{-T}: solve R X^T = rhs^T
        return np.linalg.lstsq(R, rhs.T, rcond=None)[0].T
    # wide: A = Q [R1 R2] with R1 m x m
    X, Y = A[:, :m], A[:, m:]
    R1, R2 = R[:, :m], R[:, m:]
    Rb1, Rb2 = Rb[:, :m], Rb[:, m:]
    Yb = Q @ Rb2
    Xb = _qr_backward(X, Q, R1, Qb + Y @ Rb2.T, Rb1)
    return np.concatenate([Xb, Yb], axis=1)


def _svd_backward(A, U, s, Vt, Ub, sb, Vtb):
    """Reverse rule of the thin SVD A = U diag(s) Vt, all min(m, n) values."""
    m, n = A.shape
    V, Vb = Vt.T, Vtb.T
    # the couplings (A_ij s_j + s_i B_ij) / (s_j^2 - s_i^2), A = U^T Ub - Ub^T U,
    # B = V^T Vb - Vb^T V, split as (A + B)_ij / 2 (s_j - s_i) + (A - B)_ij / 2
    # (s_j + s_i): for a gauge-invariant function A + B vanishes with s_j - s_i,
    # so the broadening of 1 / (s_j - s_i) only removes rounding noise
    dm = s[None, :] - s[:, None]
    dp = s[None, :] + s[:, None]
    Fm = dm / (dm * dm + BROADENING)
    Fp = dp / (dp * dp + BROADENING)
    np.fill_diagonal(Fm, 0.0)
    np.fill_diagonal(Fp, 0.0)
    X = U.T @ Ub
    Y = V.T @ Vb
    Aa = X - X.T
    Bb = Y - Y.T
    core = 0.5 * Fm * (Aa + Bb) + 0.5 * Fp * (Aa - Bb) + np.diag(sb)
    sinv = s / (s * s + BROADENING)
    Ab = U @ core @ Vt
    if m > len(s):
        Ab += (np.eye(m) - U @ U.T) @ Ub * sinv[None, :] @ Vt
    if n > len(s):
        Ab += U @ (sinv[:, None] * Vb.T) @ (np.eye(n) - V @ V.T)
    return Ab


def _lq_forward(t: T):
    """LQ over (leg 0 | legs 1, 2) per block, recorded."""
    v = _blocks(t, [0], [1, 2])
    ls, qs, rec = [], [], []
    for c in (0, 1):
        b = v.blocks[c]
        m, n = b.shape
        if min(m, n) == 0:
            ls.append(np.zeros((m, 0)))
            qs.append(np.zeros((0, n)))
            rec.append(None)
            continue
        q, r = np.linalg.qr(b.T, mode="reduced")
        ls.append(r.T)
        qs.append(q.T)
        rec.append((b.T, q, r))
    nl = z2.newleg(ls[0].shape[1], ls[1].shape[1])
    L = z2.from_blocks(ls, v.rp, [nl])
    Q = z2.from_blocks(qs, [nl], v.cp)
    return L, Q, (v, rec, t.p)


def _lq_backward(info, Lbar: T, Qbar: T):
    v, rec, legs = info
    lb = z2.MatView(Lbar, [0], [1]).blocks
    qb = z2.MatView(Qbar, [0], [1, 2]).blocks
    grads = []
    for c in (0, 1):
        if rec[c] is None:
            grads.append(None)
            continue
        At, q, r = rec[c]
        # A = L Q with A^T = q r: Q = q^T, L = r^T
        gt = _qr_backward(At, q, r, qb[c].T, lb[c].T)
        grads.append(gt.T)
    return _scatter(v, grads, legs, [0, 1, 2])


def _svdc_forward(t: T):
    """Canonical step by a full thin SVD over (leg 0 | legs 1, 2) per block:
    L = U S, Q = V^T (the gauge the device's canonical sweep takes)."""
    v = _blocks(t, [0], [1, 2])
    full = []
    for c in (0, 1):
        b = v.blocks[c]
        if min(b.shape) == 0:
            full.append((np.zeros((b.shape[0], 0)), np.zeros(0), np.zeros((0, b.shape[1]))))
        else:
            full.append(np.linalg.svd(b, full_matrices=False))
    nl = z2.newleg(len(full[0][1]), len(full[1][1]))
    L = z2.from_blocks([u * s[None, :] for u, s, _ in full], v.rp, [nl])
    Q = z2.from_blocks([vt for _, _, vt in full], [nl], v.cp)
    return L, Q, (v, full, t.p)


def _svdc_backward(info, Lbar: T, Qbar: T):
    """L = U S: Ubar = Lbar S, sbar = diag(U^T Lbar); Q = V^T: (V^T)bar = Qbar."""
    v, full, legs = info
    lb = z2.MatView(Lbar, [0], [1]).blocks
    qb = z2.MatView(Qbar, [0], [1, 2]).blocks
    grads = []
    for c in (0, 1):
        u, s, vt = full[c]
        if s.size == 0:
            grads.append(None)
            continue
        grads.append(_svd_backward(v.blocks[c], u, s, vt, lb[c] * s[None, :], np.sum(u * lb[c], axis=0), qb[c]))
    return _scatter(v, grads, legs, [0, 1, 2])


def _svd_forward(t: T, chi, space):
    """Truncated SVD over (legs 0, 1 | leg 2) per block, recorded."""
    v = _blocks(t, [0, 1], [2])
    full = []
    for c in (0, 1):
        b = v.blocks[c]
        if min(b.shape) == 0:
            full.append((np.zeros((b.shape[0], 0)), np.zeros(0), np.zeros((0, b.shape[1]))))
        else:
            full.append(np.linalg.svd(b, full_matrices=False))
    keep = z2.select_truncation([f[1] for f in full], chi, space)
    us = [f[0][:, k] for f, k in zip(full, keep)]
    ss = [f[1][k] for f, k in zip(full, keep)]
    vs = [f[2][k, :] for f, k in zip(full, keep)]
    nl = z2.newleg(len(ss[0]), len(ss[1]))
    U = z2.from_blocks(us, v.rp, [nl])
    V = z2.from_blocks(vs, [nl], v.cp)
    return U, ss, V, (v, full, keep, t.p)


def _svd_backward_blocks(info, Ubar: T, sbar, Vbar: T):
    v, full, keep, legs = info
    ub = z2.MatView(Ubar, [0, 1], [2]).blocks
    vb = z2.MatView(Vbar, [0], [1]).blocks
    grads = []
    for c in (0, 1):
        u, s, vt = full[c]
        if s.size == 0:
            grads.append(None)
            continue
        k = keep[c]
        Ub = np.zeros_like(u)
        Ub[:, k] = ub[c]
        Vtb = np.zeros_like(vt)
        Vtb[k, :] = vb[c]
        sb = np.zeros_like(s)
        sb[k] = sbar[c]
        grads.append(_svd_backward(v.blocks[c], u, s, vt, Ub, sb, Vtb))
    return _scatter(v, grads, legs, [0, 1, 2])


def lognorm_with_gradient(state, chi, space=None, canonical="svd"):
    """``lognorm`` of a state with the row method's exact compression and
    its derivative with respect to every site tensor: (value, grads) with
    grads[x][y] shaped like the site tensor.  ``canonical`` is the gauge of
    the exact canonical sweep: "svd" (L = U S, Q = V^T, the device's) or
    "lq" as the reference's forward pass; the truncated boundary and the value
    do not depend on it.  The LQ reverse rule solves with L, so on boundaries
    whose blocks are numerically rank deficient (synthetic 4x4 D=4 states)
    it loses accuracy (1e-4 against central differences) where the SVD rule,
    regularised by the broadening, keeps 1e-9."""
    if canonical not in ("lq", "svd"):
        raise ValueError("canonical is 'lq' or 'svd'")
    canon_forward, canon_backward = (_lq_forward, _lq_backward) if canonical == "lq" else \
        (_svdc_forward, _svdc_backward)
    from . import boundary as bm
    Lx, Ly = state.Lx, state.Ly
    sites = [[state[x, y] for y in range(Ly)] for x in range(Lx)]
    layers = [[bm.double_layer(sites[x][y]) for y in range(Ly)] for x in range(Lx)]
    env = bm.trivial_boundary([layers[x][0] for x in range(Lx)], "north").tensors
    log_scale = 0.0
    tape = []
    for y in range(Ly):
        row = [layers[x][y] for x in range(Lx)]
        B0 = []
        for A, E in zip(env, row):
            C = einsum("lnr,wnep->lwpre", A, E)
            B0.append(z2.fuse(z2.fuse(C, 3, 2), 0, 2))
        rec = dict(env=env, row=row, lq=[None] * Lx, svd=[None] * Lx)
        B = list(B0)
        for x in range(Lx - 1, 0, -1):
            L, Q, info = canon_forward(B[x])
            rec["lq"][x] = (info, B[x - 1], L)
            B[x] = Q
            B[x - 1] = einsum("lpk,kr->lpr", B[x - 1], L)
        for x in range(Lx - 1):
            U, S, V, info = _svd_forward(B[x], chi, space)
            s = np.concatenate(S)
            R = T(V.a * s[:, None], V.p)
            rec["svd"][x] = (info, S, V, R, B[x + 1])
            B[x] = U
            B[x + 1] = einsum("lk,kpr->lpr", R, B[x + 1])
        scale = z2.norm(B[Lx - 1])
        if not (math.isfinite(scale) and scale > 0):
            raise RuntimeError("nonfinite or zero boundary norm")
        rec["center"] = (B[Lx - 1], scale)
        B[Lx - 1] = B[Lx - 1] / scale
        log_scale += math.log(scale)
        tape.append(rec)
        env = B
    # close: V_0 = 1, V_{x+1} = V_x A_x[:, 0, :], value = sum V_N
    vecs = [np.ones(env[0].shape[0])]
    for A in env:
        vecs.append(vecs[-1] @ A.a[:, 0, :])
    closed = float(vecs[-1].sum())
    if not closed > 0:
        raise RuntimeError("norm requires a finite positive real value")
    value = math.log(closed) + log_scale + 2 * state.log_amplitude

    # backward: d value / d closed = 1 / closed, d value / d log_scale = 1
    vb = np.ones(env[-1].shape[2]) / closed
    envbar = [None] * Lx
    for x in range(Lx - 1, -1, -1):
        A = env[x]
        g = np.zeros_like(A.a)
        g[:, 0, :] = np.outer(vecs[x], vb)
        envbar[x] = T(g, A.p)
        vb = A.a[:, 0, :] @ vb
    layerbar = [[None] * Ly for _ in range(Lx)]
    for y in range(Ly - 1, -1, -1):
        rec = tape[y]
        Bbar = list(envbar)
        # centre normalisation: out = B / s, log s enters value with weight 1
        Bc, s = rec["center"]
        out = Bc.a / s
        gbar = Bbar[Lx - 1].a
        Bbar[Lx - 1] = T((gbar - np.sum(gbar * out) * out + out) / s, Bc.p)
        # SVD sweep, last step first
        for x in range(Lx - 2, -1, -1):
            info, S, V, R, Bnext = rec["svd"][x]
            G = Bbar[x + 1]                            # cotangent of R . B_old[x+1]
            Rbar = einsum("lpr,kpr->lk", G, Bnext)
            Bbar[x + 1] = einsum("lk,lpr->kpr", R, G)
            s = np.concatenate(S)
            sbar_all = np.sum(Rbar.a * V.a, axis=1)
            Vbar = T(Rbar.a * s[:, None], V.p)
            n0 = len(S[0])
            Bbar[x] = T(_svd_backward_blocks(info, Bbar[x], [sbar_all[:n0], sbar_all[n0:]], Vbar), info[3])
        # LQ sweep, in the forward order reversed
        for x in range(1, Lx):
            info, Bprev, L = rec["lq"][x]
            G = Bbar[x - 1]                            # cotangent of B_old[x-1] . L
            Lbar = einsum("lpr,lpk->kr", G, Bprev)
            Bbar[x - 1] = einsum("lpr,kr->lpk", G, L)
            Qbar = Bbar[x]
            Bbar[x] = T(canon_backward(info, Lbar, Qbar), info[2])
        # absorption: B0 = fuse(fuse(einsum(env, row)))
        newenv = [None] * Lx
        for x in range(Lx):
            A, E = rec["env"][x], rec["row"][x]
            C = einsum("lnr,wnep->lwpre", A, E)
            Cbar = T(Bbar[x].a.reshape(C.shape), C.p)
            newenv[x] = einsum("lwpre,wnep->lnr", Cbar, E)
            layerbar[x][y] = einsum("lwpre,lnr->wnep", Cbar, A)
        envbar = newenv
    grads = [[None] * Ly for _ in range(Lx)]
    for x in range(Lx):
        for y in range(Ly):
            A = sites[x][y]
            Db = layerbar[x][y]
            d = [len(p) for p in A.p]
            raw = Db.a.reshape(d[0], d[0], d[1], d[1], d[4], d[4], d[5], d[5])
            g = np.einsum("wWnNeEsS,WNpaES->wnpaes", raw, A.a) + np.einsum("wWnNeEsS,wnpaes->WNpaES", raw, A.a)
            grads[x][y] = g
    return value, grads


def field_gradient(state, chi, space=None):
    """Per-site <X_i> from one reverse pass (half the derivative of lnZ along
    A_i -> A_i + e X A_i, X on the physical leg) and d lnZ/dh_i = beta <X_i>
    of the thermal state the PEPO represents: (value, site_x[x, y],
    d_fields in x + y*Lx order).  The reference's direct route to <X_i> is one
    ratio per site (``src/measurement/energy.jl:43-46``)."""
    from . import model as md
    X = md.spin_operators()[0]
    value, g = lognorm_with_gradient(state, chi, space)
    site_x = np.zeros((state.Lx, state.Ly))
    for x in range(state.Lx):
        for y in range(state.Ly):
            XA = np.einsum("pu,wnuaes->wnpaes", X, state[x, y].a)
            site_x[x, y] = 0.5 * float(np.sum(g[x][y] * XA))
    return value, site_x, state.beta * site_x.T.reshape(-1)

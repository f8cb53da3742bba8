"""Z2-graded dense tensors for the CPU oracle.

TEST INFRASTRUCTURE ONLY. This package is the checker for the CUDA path:
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it.  Nothing in the product library calls it.

The reference stores every tensor as a TensorKit ``TensorMap`` over Z2
graded spaces (``src/states/tensors.jl``).  Z2 is abelian with bosonic
braiding, so permutations carry no signs and every block structure is
determined by one parity bit per basis state.  The oracle therefore keeps a
tensor as a dense float64 array plus, for every leg, the parity of each
basis state.  Entries whose leg parities sum to an odd number are structural
zeros.  Contractions are plain dense contractions (structural zeros stay
zero); every factorization (QR, LQ, SVD, eigh) is done per parity block of a
matrix view, as TensorKit does per coupled sector.

Matrix-view convention (shared with the CUDA engine): for a bipartition
(row legs | column legs) the rows of block c are the row-major fused indices
of the row legs whose parity is c, in increasing order; columns likewise.
New legs created by a factorization list the block-0 states first.
Fusing two legs is a reshape (row-major, first leg slowest) and the fused
parity is the XOR of the parts.  These basis choices are gauge choices: every
scalar the pipeline reports is invariant under them.
"""
from __future__ import annotations

import numpy as np

EPS = np.finfo(np.float64).eps
FLOATMIN = np.finfo(np.float64).tiny


def leg(n0: int, n1: int) -> np.ndarray:
    """Parity vector of a leg with n0 even states followed by n1 odd states."""
    return np.concatenate([np.zeros(n0, np.int8), np.ones(n1, np.int8)])


def fused_parity(pars) -> np.ndarray:
    out = np.zeros(1, np.int8)
    for p in pars:
        out = (out[:, None] ^ np.asarray(p, np.int8)[None, :]).reshape(-1)
    return out


class T:
    """Dense Z2 tensor: ``a`` (float64 ndarray) and one parity vector per leg."""

    __slots__ = ("a", "p")

    def __init__(self, a, p):
        self.a = np.ascontiguousarray(a, dtype=np.float64)
        self.p = tuple(np.asarray(x, np.int8) for x in p)
        assert self.a.ndim == len(self.p), (self.a.shape, len(self.p))
        for n, x in zip(self.a.shape, self.p):
            assert n == len(x), (self.a.shape, [len(q) for q in self.p])

    @property
    def shape(self):
        return self.a.shape

    @property
    def ndim(self):
        return self.a.ndim

    def copy(self) -> "T":
        return T(self.a.copy(), self.p)

    def __mul__(self, s: float) -> "T":
        return T(self.a * s, self.p)

    __rmul__ = __mul__

    def __truediv__(self, s: float) -> "T":
        return T(self.a / s, self.p)

    def __add__(self, o: "T") -> "T":
        return T(self.a + o.a, self.p)

    def __sub__(self, o: "T") -> "T":
        return T(self.a - o.a, self.p)

    def sector_dims(self, k: int):
        x = self.p[k]
        return int((x == 0).sum()), int((x == 1).sum())


def parity_mask(p) -> np.ndarray:
    """Boolean mask of even-total-parity entries for legs with parities ``p``."""
    return fused_parity(p).reshape([len(x) for x in p]) == 0 if len(p) else np.ones((), bool)


def odd_weight(t: T) -> float:
    """Largest magnitude found on a structurally-zero (odd parity) entry."""
    m = ~parity_mask(t.p)
    return float(np.abs(t.a[m]).max()) if m.any() else 0.0


def einsum(spec: str, *ts: T) -> T:
    """``numpy.einsum`` that carries leg parities by label."""
    ins, out = spec.replace(" ", "").split("->")
    ins = ins.split(",")
    assert len(ins) == len(ts)
    lab = {}
    for s, t in zip(ins, ts):
        assert len(s) == t.ndim, (spec, s, t.shape)
        for ch, p in zip(s, t.p):
            if ch in lab:
                assert len(lab[ch]) == len(p) and np.array_equal(lab[ch], p), (spec, ch)
            else:
                lab[ch] = p
    a = np.einsum(spec, *[t.a for t in ts], optimize=True)
    return T(a, [lab[ch] for ch in out])


def perm(t: T, order) -> T:
    return T(np.transpose(t.a, order), [t.p[k] for k in order])


def fuse(t: T, first: int, count: int) -> T:
    """Fuse legs first..first+count-1 (0-based) into one leg (row-major)."""
    if count == 1:
        return t.copy()
    sh = list(t.shape)
    n = int(np.prod(sh[first:first + count]))
    p = list(t.p)
    fp = fused_parity(p[first:first + count])
    newsh = sh[:first] + [n] + sh[first + count:]
    newp = p[:first] + [fp] + p[first + count:]
    return T(t.a.reshape(newsh), newp)


def split(t: T, axis: int, pars) -> T:
    """Inverse of ``fuse``: split leg ``axis`` into legs with parities ``pars``."""
    assert np.array_equal(fused_parity(pars), t.p[axis])
    sh = list(t.shape)
    newsh = sh[:axis] + [len(x) for x in pars] + sh[axis + 1:]
    newp = list(t.p[:axis]) + list(pars) + list(t.p[axis + 1:])
    return T(t.a.reshape(newsh), newp)


def norm(t: T) -> float:
    return float(np.sqrt(np.sum(t.a * t.a)))


def dot(a: T, b: T) -> float:
    return float(np.sum(a.a * b.a))


def unit(pars) -> T:
    """All-ones tensor on one-dimensional even legs (``_unit_tensor``)."""
    for p in pars:
        assert len(p) == 1 and p[0] == 0, "nontrivial OBC leg"
    return T(np.ones([1] * len(pars)), pars)


# ---------------------------------------------------------------------------
# matrix views
# ---------------------------------------------------------------------------

class MatView:
    """The two parity blocks of a tensor seen as (rows | cols)."""

    def __init__(self, t: T, rows, cols):
        rows, cols = list(rows), list(cols)
        self.rows, self.cols = rows, cols
        self.rp = [t.p[k] for k in rows]
        self.cp = [t.p[k] for k in cols]
        self.rsh = [t.shape[k] for k in rows]
        self.csh = [t.shape[k] for k in cols]
        M = int(np.prod(self.rsh)) if rows else 1
        N = int(np.prod(self.csh)) if cols else 1
        full = np.transpose(t.a, rows + cols).reshape(M, N)
        rfp, cfp = fused_parity(self.rp), fused_parity(self.cp)
        self.ridx = [np.nonzero(rfp == c)[0] for c in (0, 1)]
        self.cidx = [np.nonzero(cfp == c)[0] for c in (0, 1)]
        self.blocks = [full[np.ix_(self.ridx[c], self.cidx[c])] for c in (0, 1)]
        self.M, self.N = M, N


def from_blocks(blocks, rp, cp) -> T:
    """Assemble a tensor with row legs ``rp`` and column legs ``cp``."""
    rsh = [len(x) for x in rp]
    csh = [len(x) for x in cp]
    M = int(np.prod(rsh)) if rp else 1
    N = int(np.prod(csh)) if cp else 1
    rfp, cfp = fused_parity(rp), fused_parity(cp)
    full = np.zeros((M, N))
    for c in (0, 1):
        ri = np.nonzero(rfp == c)[0]
        ci = np.nonzero(cfp == c)[0]
        b = blocks[c]
        assert b.shape == (len(ri), len(ci)), (b.shape, len(ri), len(ci))
        if b.size:
            full[np.ix_(ri, ci)] = b
    return T(full.reshape(rsh + csh), list(rp) + list(cp))


def newleg(k0: int, k1: int) -> np.ndarray:
    return leg(k0, k1)


def qr(t: T, rows, cols):
    """Compact QR per parity block (``left_orth``): t = Q R."""
    v = MatView(t, rows, cols)
    qs, rs = [], []
    for c in (0, 1):
        b = v.blocks[c]
        m, n = b.shape
        k = min(m, n)
        if k == 0:
            qs.append(np.zeros((m, 0)))
            rs.append(np.zeros((0, n)))
            continue
        q, r = np.linalg.qr(b, mode="reduced")
        qs.append(q)
        rs.append(r)
    nl = newleg(qs[0].shape[1], qs[1].shape[1])
    Q = from_blocks(qs, v.rp, [nl])
    R = from_blocks(rs, [nl], v.cp)
    return Q, R


def lq(t: T, rows, cols):
    """Compact LQ per parity block (``right_orth``): t = L Q."""
    v = MatView(t, rows, cols)
    ls, qs = [], []
    for c in (0, 1):
        b = v.blocks[c]
        m, n = b.shape
        k = min(m, n)
        if k == 0:
            ls.append(np.zeros((m, 0)))
            qs.append(np.zeros((0, n)))
            continue
        q, r = np.linalg.qr(b.T, mode="reduced")
        ls.append(r.T)
        qs.append(q.T)
    nl = newleg(ls[0].shape[1], ls[1].shape[1])
    L = from_blocks(ls, v.rp, [nl])
    Q = from_blocks(qs, [nl], v.cp)
    return L, Q


def svd_blocks(t: T, rows, cols):
    """Compact SVD per parity block; returns the view and (U, S, Vt) per block."""
    v = MatView(t, rows, cols)
    out = []
    for c in (0, 1):
        b = v.blocks[c]
        m, n = b.shape
        if min(m, n) == 0:
            out.append((np.zeros((m, 0)), np.zeros(0), np.zeros((0, n))))
            continue
        u, s, vt = np.linalg.svd(b, full_matrices=False)
        out.append((u, s, vt))
    return v, out


def select_truncation(svals, chi=None, space=None, atol=None):
    """Kept indices per block for ``truncrank(chi) & truncspace(space) & trunctol(atol)``.

    MatrixAlgebraKit combines strategies with ``&`` as an intersection of the
    index sets each strategy keeps (``src/contraction/boundary_mps.jl:18``,
    ``src/evolution/full_update.jl:34``).  ``truncrank`` keeps the ``chi``
    largest values over both sectors (ties broken sector 0 first, then by
    position); ``truncspace`` keeps the leading ``space[c]`` values of sector
    c; ``trunctol`` keeps values strictly above ``atol``.
    """
    keep = [np.ones(len(s), bool) for s in svals]
    if chi is not None:
        allv = [(-float(svals[c][i]), c, i) for c in (0, 1) for i in range(len(svals[c]))]
        allv.sort()
        sel = [np.zeros(len(v), bool) for v in svals]
        for _, c, i in allv[:chi]:
            sel[c][i] = True
        keep = [k & q for k, q in zip(keep, sel)]
    if space is not None:
        for c in (0, 1):
            k = np.zeros(len(svals[c]), bool)
            k[: space[c]] = True
            keep[c] &= k
    if atol is not None:
        for c in (0, 1):
            keep[c] &= svals[c] > atol
    return keep


def svd_trunc(t: T, rows, cols, chi=None, space=None, atol=None, entropy=False):
    """Truncated SVD: (U, S, V, err, entropy) with U (rows, new), S diag blocks, V (new, cols).

    ``err`` is the 2-norm of the discarded singular values (MatrixAlgebraKit
    ``truncation_error!``); ``entropy`` is the pretruncation Schmidt entropy
    (``src/contraction/boundary_mps.jl:21-30``) when requested.
    """
    v, bl = svd_blocks(t, rows, cols)
    svals = [b[1] for b in bl]
    ent = None
    if entropy:
        ent = schmidt_entropy(svals)
    keep = select_truncation(svals, chi, space, atol)
    disc = np.concatenate([svals[c][~keep[c]] for c in (0, 1)])
    err = float(np.sqrt(np.sum(disc * disc)))
    us, ss, vs = [], [], []
    for c in (0, 1):
        u, s, vt = bl[c]
        k = keep[c]
        us.append(u[:, k])
        ss.append(s[k])
        vs.append(vt[k, :])
    nl = newleg(len(ss[0]), len(ss[1]))
    U = from_blocks(us, v.rp, [nl])
    V = from_blocks(vs, [nl], v.cp)
    return U, ss, V, err, ent


def schmidt_entropy(svals) -> float:
    allv = np.concatenate(svals)
    scale = float(np.sqrt(np.sum(allv * allv)))
    if scale == 0.0:
        return float("nan")
    ent = 0.0
    for s in allv:
        p = (s / scale) ** 2
        if p != 0.0:
            ent -= p * np.log(p)
    return max(0.0, float(ent))


def diag_tensor(svals, transform=None) -> T:
    """Diagonal (new, new) tensor from per-block values."""
    nl = newleg(len(svals[0]), len(svals[1]))
    vals = np.concatenate(svals)
    if transform is not None:
        vals = transform(vals)
    return T(np.diag(vals), [nl, nl])


def matmul_view(a: T, arows, acols, b: T, brows, bcols) -> T:
    """(a as rows|cols) @ (b as rows|cols), keeping a's row legs and b's column legs."""
    ra = list(arows) + list(acols)
    rb = list(brows) + list(bcols)
    A = perm(a, ra)
    B = perm(b, rb)
    na = len(arows)
    nb = len(bcols)
    ka = A.ndim - na
    res = np.tensordot(A.a, B.a, axes=(list(range(na, na + ka)), list(range(ka))))
    return T(res, list(A.p[:na]) + list(B.p[ka:]))

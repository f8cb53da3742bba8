"""Device-resident states and the hot-path calls, through the C ABI.

Each function here keeps the name, argument meaning and error behaviour of
the reference function it stands for (``lognorm``, ``measure_energy``,
``evolution_step!``, ``SamplingCache``, ``sample_configuration``,
``project_configuration``, ``normalize_state!``, ``identity_pepo``).  The
work runs in ``libstopeps_gpu.so``; there is no host fallback.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np

from . import _lib
from .config import BoundaryMPS, BoundaryMPSDiagonal, BoundaryMPSDiagonalVariational, BoundaryMPSRowVariational, BoundaryMPSZipUp, RunConfig, TFIM, FullUpdate, Z2Space


def _arr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def _boundary(m: BoundaryMPS, e=None):
    """The C ABI's sps_boundary of a method; a variational method also sets the
    engine's sweep options (``max_sweep``, ``threshold_sweep``)."""
    b = _lib.sps_boundary()
    b.chi = int(m.chi)
    if m.sector_space is None:
        b.space0 = b.space1 = -1
    else:
        b.space0, b.space1 = int(m.sector_space.n0), int(m.sector_space.n1)
    b.absorption = 2 if isinstance(m, BoundaryMPSDiagonal) else 1 if isinstance(m, BoundaryMPSZipUp) else 0
    if isinstance(m, (BoundaryMPSRowVariational, BoundaryMPSDiagonalVariational)):
        b.absorption = 4 if isinstance(m, BoundaryMPSDiagonalVariational) else 3
        if e is not None:
            e.check(e.lib.sps_set_variational(e.h, int(m.max_sweep), float(m.threshold_sweep)))
    return b


class Engine:
    """One device handle for a lattice, model, full-update options and Trotter order."""

    def __init__(self, Lx, Ly, model: TFIM = TFIM(), update: FullUpdate = FullUpdate(), trotter_order=2,
                 record_boundary_entropy=True, device=0):
        self.lib = _lib.load()
        cfg = _lib.sps_config()
        cfg.Lx, cfg.Ly = int(Lx), int(Ly)
        cfg.J, cfg.h = float(model.J), float(model.h)
        cfg.trotter_order = int(trotter_order)
        cfg.fu_max_iterations = int(update.max_iterations)
        cfg.fu_error_tolerance = float(update.error_tolerance)
        cfg.fu_diagonal_shift = float(update.diagonal_shift)
        cfg.fu_linear_max_iterations = int(update.linear_max_iterations)
        cfg.fu_linear_tolerance = float(update.linear_tolerance)
        cfg.record_boundary_entropy = 1 if record_boundary_entropy else 0
        cfg.device = int(device)
        h = C.c_void_p()
        code = self.lib.sps_create(C.byref(cfg), C.byref(h))
        if code != 0:
            raise _lib.EngineError(code, "sps_create failed (is a CUDA device visible?)")
        self.h = h
        self.Lx, self.Ly = int(Lx), int(Ly)
        self.model = model
        if getattr(model, "fields", None) is not None:
            f = np.ascontiguousarray(model.fields, np.float64)
            if f.size != self.Lx * self.Ly:
                raise ValueError("per-site fields need one value per lattice site")
            self.check(self.lib.sps_set_site_fields(self.h, int(f.size), f.ctypes.data_as(C.POINTER(C.c_double))))
        self.update = update

    @classmethod
    def from_config(cls, c: RunConfig, device=0):
        return cls(c.lattice.Lx, c.lattice.Ly, c.model, c.update, c.trotter_order, c.record_boundary_entropy,
                   device)

    def check(self, code):
        if code != 0:
            buf = C.create_string_buffer(4096)
            self.lib.sps_last_error(self.h, buf, 4096)
            raise _lib.EngineError(code, buf.value.decode(errors="replace"))

    def counters(self):
        n = C.c_longlong()
        f = C.c_double()
        self.check(self.lib.sps_counters(self.h, C.byref(n), C.byref(f)))
        return n.value, f.value

    def set_concurrency(self, samples: int):
        """How many samples ``sample_batch`` draws at the same time (own stream and workspace each)."""
        self.check(self.lib.sps_set_concurrency(self.h, int(samples)))

    def set_sm_share(self, ctas: int):
        """Cap this handle's own cooperative launches at ``ctas`` CTAs each (0: the whole GPU)."""
        self.check(self.lib.sps_set_sm_share(self.h, int(ctas)))

    PRECISIONS = {"fp64": 0, "tf32": 1, "3xtf32": 2, "3xbf16": 3}

    def set_precision(self, mode="fp64"):
        """Arithmetic of the large contraction GEMMs: "fp64" (default), or on the
        tcgen05 tensor cores with FP32 accumulation "tf32", "3xtf32" (split
        operands) or "3xbf16" (split operands); factorizations, normalisations
        and log-weights stay FP64."""
        if mode not in self.PRECISIONS:
            raise ValueError(f"unknown precision {mode!r}; one of {sorted(self.PRECISIONS)}")
        self.check(self.lib.sps_set_precision(self.h, self.PRECISIONS[mode]))

    def set_truncated_svd(self, method="subspace"):
        """``"subspace"`` (default): truncated SVDs keeping a few vectors of a large
        block take the subspace iteration when no entropy is recorded;
        ``"full"``: every truncated SVD from the full spectrum."""
        if method not in ("subspace", "full"):
            raise ValueError("method is 'subspace' or 'full'")
        self.check(self.lib.sps_set_truncated_svd(self.h, 1 if method == "full" else 0))

    def set_autotune(self, enable=True):
        """Pick launch shapes (split-K slices, tcgen05 tile width) by timing the
        candidates on first use; the choices are shared process-wide."""
        self.check(self.lib.sps_set_autotune(self.h, 1 if enable else 0))

    def autotune_report(self) -> dict:
        buf = C.create_string_buffer(1 << 20)
        self.check(self.lib.sps_autotune_report(self.h, buf, 1 << 20))
        return json.loads(buf.value.decode())

    def set_injection(self, force_repair=False, svd_sweep_cap=0, multi_cta_eigh_min=0):
        """Host-side failure injection for tests: force the PSD-repair branch of
        every bond update; cap the small-block Jacobi sweeps (0 = default);
        route repair eigendecompositions of blocks with at least
        ``multi_cta_eigh_min`` rows to the multi-CTA solver (0 = default 1024)."""
        self.check(self.lib.sps_set_injection(self.h, 1 if force_repair else 0, int(svd_sweep_cap),
                                              int(multi_cta_eigh_min)))

    def set_profile(self, enable):
        """0/False off, 1/True per-kernel stats, 2 also per-shape contraction stats (resets the stats)."""
        self.check(self.lib.sps_set_profile(self.h, int(enable)))

    def kernel_stats(self) -> dict:
        import json
        buf = C.create_string_buffer(1 << 16)
        self.check(self.lib.sps_kernel_stats_json(self.h, buf, 1 << 16))
        return json.loads(buf.value.decode())

    def timer_start(self):
        self.check(self.lib.sps_timer_start(self.h))

    def timer_stop(self) -> float:
        ms = C.c_double()
        self.check(self.lib.sps_timer_stop(self.h, C.byref(ms)))
        return ms.value

    def la_svd(self, a):
        """Engine SVD of one host matrix: (u, s, vt, sweeps, device_ms)."""
        a = np.asfortranarray(np.asarray(a, np.float64))
        m, n = a.shape
        k = min(m, n)
        u = np.zeros((m, k), order="F")
        s = np.zeros(k)
        vt = np.zeros((k, n), order="F")
        sw = C.c_int32()
        ms = C.c_double()
        self.check(self.lib.sps_la_svd(self.h, m, n, _arr(a, C.c_double), _arr(u, C.c_double), _arr(s, C.c_double),
                                       _arr(vt, C.c_double), C.byref(sw), C.byref(ms)))
        return u, s, vt, sw.value, ms.value

    def la_svd_left(self, a):
        """Left singular vectors and values (m >= n) by the U-only Jacobi: (u, s, sweeps, device_ms)."""
        a = np.asfortranarray(np.asarray(a, np.float64))
        m, n = a.shape
        u = np.zeros((m, n), order="F")
        s = np.zeros(n)
        sw = C.c_int32()
        ms = C.c_double()
        self.check(self.lib.sps_la_svd_left(self.h, m, n, _arr(a, C.c_double), _arr(u, C.c_double),
                                            _arr(s, C.c_double), C.byref(sw), C.byref(ms)))
        return u, s, sw.value, ms.value

    def la_gemm(self, a, b, c=None, alpha=1.0, beta=0.0, transpose_a=False):
        """Engine FP64 GEMM alpha op(a) b + beta c: (c, device_ms)."""
        a = np.asfortranarray(np.asarray(a, np.float64))
        b = np.asfortranarray(np.asarray(b, np.float64))
        m = a.shape[1] if transpose_a else a.shape[0]
        k, n = b.shape
        if (a.shape[0] if transpose_a else a.shape[1]) != k:
            raise ValueError("inner dimensions differ")
        c = np.zeros((m, n), order="F") if c is None else np.asfortranarray(np.array(c, np.float64))
        ms = C.c_double()
        self.check(self.lib.sps_la_gemm(self.h, int(transpose_a), m, n, k, float(alpha), _arr(a, C.c_double),
                                        _arr(b, C.c_double), float(beta), _arr(c, C.c_double), C.byref(ms)))
        return c, ms.value

    def la_gemm_mixed(self, a, b, mode="3xtf32"):
        """tcgen05 GEMM a @ b in a low-precision mode ("tf32", "3xtf32", "3xbf16"): (c, device_ms)."""
        a = np.ascontiguousarray(np.asarray(a, np.float64))
        b = np.ascontiguousarray(np.asarray(b, np.float64))
        m, k = a.shape
        k2, n = b.shape
        if k != k2:
            raise ValueError("inner dimensions differ")
        c = np.zeros((m, n))
        ms = C.c_double()
        self.check(self.lib.sps_la_gemm_mixed(self.h, self.PRECISIONS[mode], m, n, k, _arr(a, C.c_double),
                                              _arr(b, C.c_double), _arr(c, C.c_double), C.byref(ms)))
        return c, ms.value

    def la_svd_topk(self, a, k, gram=False, rtol=0.0):
        """Leading k singular triplets by subspace iteration: (u, s, v, iterations, device_ms).

        ``gram`` iterates on a a^T; ``rtol`` is the residual bound relative to
        the largest singular value (0: rounding level, 5e-14)."""
        a = np.asfortranarray(np.asarray(a, np.float64))
        m, n = a.shape
        u = np.zeros((m, k), order="F")
        v = np.zeros((n, k), order="F")
        s = np.zeros(k)
        it = C.c_int32()
        ms = C.c_double()
        self.check(self.lib.sps_la_svd_topk(self.h, m, n, k, _arr(a, C.c_double), int(bool(gram)), float(rtol),
                                            _arr(u, C.c_double), _arr(s, C.c_double), _arr(v, C.c_double),
                                            C.byref(it), C.byref(ms)))
        return u, s, v, it.value, ms.value

    def la_qr(self, a):
        """Engine Householder QR of one host matrix: (q, r, device_ms)."""
        a = np.asfortranarray(np.asarray(a, np.float64))
        m, n = a.shape
        k = min(m, n)
        q = np.zeros((m, k), order="F")
        r = np.zeros((k, n), order="F")
        ms = C.c_double()
        self.check(self.lib.sps_la_qr(self.h, m, n, _arr(a, C.c_double), _arr(q, C.c_double), _arr(r, C.c_double),
                                      C.byref(ms)))
        return q, r, ms.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.sps_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- states -----------------------------------------------------------
    def identity_pepo(self) -> "DeviceState":
        sid = C.c_int32()
        self.check(self.lib.sps_identity_pepo(self.h, C.byref(sid)))
        return DeviceState(self, sid.value)

    def upload_state(self, sites, leg_dims, is_pepo, beta=0.0, log_amplitude=0.0) -> "DeviceState":
        """Upload site tensors (x + y*Lx order) with per-leg (n0,n1) multiplicities."""
        dims = np.ascontiguousarray(np.asarray(leg_dims, np.int32).reshape(-1))
        data = np.ascontiguousarray(np.concatenate([np.asarray(s, np.float64).reshape(-1) for s in sites]))
        sid = C.c_int32()
        self.check(self.lib.sps_state_upload(self.h, 1 if is_pepo else 0, float(beta), float(log_amplitude),
                                             _arr(dims, C.c_int32), _arr(data, C.c_double), C.byref(sid)))
        return DeviceState(self, sid.value)


class DeviceState:
    """``FiniteState`` held on the device (``src/states/finite.jl:27-49``)."""

    def __init__(self, engine: Engine, sid: int):
        self.engine = engine
        self.id = sid

    def _info(self):
        b, la, p = C.c_double(), C.c_double(), C.c_int32()
        self.engine.check(self.engine.lib.sps_state_info(self.engine.h, self.id, C.byref(b), C.byref(la),
                                                         C.byref(p)))
        return b.value, la.value, bool(p.value)

    @property
    def beta(self):
        return self._info()[0]

    @beta.setter
    def beta(self, v):
        self.engine.check(self.engine.lib.sps_state_set_beta(self.engine.h, self.id, float(v)))

    @property
    def log_amplitude(self):
        return self._info()[1]

    @property
    def is_pepo(self):
        return self._info()[2]

    @property
    def lattice(self):
        return (self.engine.Lx, self.engine.Ly)

    def copy(self) -> "DeviceState":
        nid = C.c_int32()
        self.engine.check(self.engine.lib.sps_state_copy(self.engine.h, self.id, C.byref(nid)))
        return DeviceState(self.engine, nid.value)

    def download(self):
        """Site tensors (x + y*Lx order) and their leg multiplicities."""
        L = self.engine.Lx * self.engine.Ly
        dims = np.zeros(L * 12, np.int32)
        tot = C.c_int64()
        self.engine.check(self.engine.lib.sps_state_layout(self.engine.h, self.id, _arr(dims, C.c_int32),
                                                           C.byref(tot)))
        data = np.zeros(tot.value, np.float64)
        self.engine.check(self.engine.lib.sps_state_download(self.engine.h, self.id, _arr(data, C.c_double),
                                                             tot.value))
        dims = dims.reshape(L, 6, 2)
        sites, off = [], 0
        for i in range(L):
            shape = [int(a + b) for a, b in dims[i]]
            n = int(np.prod(shape))
            sites.append(data[off:off + n].reshape(shape))
            off += n
        return sites, dims

    def __del__(self):
        try:
            if self.engine.h:
                self.engine.lib.sps_state_free(self.engine.h, self.id)
        except Exception:
            pass


def normalize_state(state: DeviceState):
    """``normalize_state!``: per-site log normalisations in row-major order."""
    L = state.engine.Lx * state.engine.Ly
    out = np.zeros(L)
    state.engine.check(state.engine.lib.sps_normalize_state(state.engine.h, state.id, _arr(out, C.c_double)))
    return out


def evolution_step(state: DeviceState, delta, D, contraction: BoundaryMPS, sector_space: Z2Space | None = None):
    """``evolution_step!(state, model, delta, D, FullUpdate, contraction)``."""
    e = state.engine
    rep = _lib.sps_step_report()
    b = _boundary(contraction, e)
    if sector_space is None:
        e.check(e.lib.sps_evolution_step(e.h, state.id, float(delta), int(D), None, C.byref(b), C.byref(rep)))
    else:
        sp = (C.c_int32 * 2)(sector_space.n0, sector_space.n1)
        e.check(e.lib.sps_evolution_step(e.h, state.id, float(delta), int(D), sp, C.byref(b), C.byref(rep)))
    return {f: getattr(rep, f) for f, _ in rep._fields_}


def lognorm(state: DeviceState, contraction: BoundaryMPS):
    """``lognorm``; a variational method adds ``boundary_variational``, the fit
    summary (``max_sweeps``, ``sweep_limit_hits``, ``fallback_count``,
    ``max_relative_change``, ``layers`` = the number of absorptions)."""
    e = state.engine
    r = _lib.sps_lognorm_result()
    b = _boundary(contraction, e)
    if isinstance(contraction, (BoundaryMPSRowVariational, BoundaryMPSDiagonalVariational)):
        counts = (C.c_int32 * 4)()
        change = C.c_double()
        e.check(e.lib.sps_lognorm_variational(e.h, state.id, C.byref(b), C.byref(r), counts, C.byref(change)))
        return dict(log_norm=r.log_norm, tensor_log_norm=r.tensor_log_norm,
                    max_environment_truncation=r.max_environment_truncation,
                    boundary_variational=dict(layers=counts[0], max_sweeps=counts[1], sweep_limit_hits=counts[2],
                                              fallback_count=counts[3], max_relative_change=change.value))
    e.check(e.lib.sps_lognorm(e.h, state.id, C.byref(b), C.byref(r)))
    return dict(log_norm=r.log_norm, tensor_log_norm=r.tensor_log_norm,
                max_environment_truncation=r.max_environment_truncation)


def lognorm_gradient(state: DeviceState, contraction: BoundaryMPS, checkpoint_rows=False):
    """lognorm (row method, exact compression) and its derivative with respect
    to every site tensor by reverse mode: (log_norm, [gradient per site in
    x + y*Lx order, shaped like the site tensor]).  ``checkpoint_rows`` keeps
    only each row's incoming boundary and recomputes the row's
    factorizations in the reverse pass.  No counterpart in the reference,
    which has no derivatives."""
    e = state.engine
    L = e.Lx * e.Ly
    dims = np.zeros(L * 12, np.int32)
    tot = C.c_int64()
    e.check(e.lib.sps_state_layout(e.h, state.id, _arr(dims, C.c_int32), C.byref(tot)))
    grads = np.zeros(tot.value, np.float64)
    value = C.c_double()
    b = _boundary(contraction, e)
    e.check(e.lib.sps_lognorm_gradient(e.h, state.id, C.byref(b), int(bool(checkpoint_rows)), C.byref(value),
                                       _arr(grads, C.c_double),
                                       tot.value))
    dims = dims.reshape(L, 6, 2)
    out, off = [], 0
    for i in range(L):
        shape = [int(a + c) for a, c in dims[i]]
        n = int(np.prod(shape))
        out.append(grads[off:off + n].reshape(shape))
        off += n
    return value.value, out


def lognorm_field_gradient(state: DeviceState, contraction: BoundaryMPS, checkpoint_rows=False):
    """Per-site field derivatives from one reverse pass of ``lognorm_gradient``:
    ``site_x`` (<X_i>, half the derivative of lnZ along X insertions) and
    ``d_fields`` (d lnZ/dh_i = beta <X_i> of the thermal state the PEPO
    represents), x + y*Lx order.  The reference's direct route to the same
    numbers is one ratio per site (``measure_energy``, ``energy.jl:43-46``)."""
    e = state.engine
    L = e.Lx * e.Ly
    x, d = np.zeros(L, np.float64), np.zeros(L, np.float64)
    value = C.c_double()
    b = _boundary(contraction, e)
    e.check(e.lib.sps_lognorm_field_gradient(e.h, state.id, C.byref(b), int(bool(checkpoint_rows)), C.byref(value),
                                             _arr(x, C.c_double), _arr(d, C.c_double)))
    return {"log_norm": value.value, "site_x": x.reshape(e.Ly, e.Lx).T.copy(), "d_fields": d}


def measure_energy(state: DeviceState, contraction: BoundaryMPS, site_profile=False):
    """``measure_energy``; also returns ``magnetization`` = <sum_i X_i>/N."""
    e = state.engine
    r = _lib.sps_energy()
    b = _boundary(contraction, e)
    L = e.Lx * e.Ly
    sx = np.zeros(L)
    diagonal = isinstance(contraction, BoundaryMPSDiagonal)
    nb = L if diagonal else max(0, (e.Ly - 1) * (e.Lx - 1))
    sn = np.zeros(max(nb, 1))
    ss = np.zeros(max(nb, 1))
    e.check(e.lib.sps_measure_energy(e.h, state.id, C.byref(b), C.byref(r), _arr(sx, C.c_double),
                                     _arr(sn, C.c_double), _arr(ss, C.c_double)))
    out = dict(energy_total=r.energy_total, energy_per_site=r.energy_per_site, log_norm=r.log_norm,
               tensor_log_norm=r.tensor_log_norm, max_environment_truncation=r.max_environment_truncation,
               x_sum=r.x_sum, zz_sum=r.zz_sum, magnetization=r.x_sum / L)
    if site_profile and diagonal:   # per-site profiles of the two sweeps, [x, y]
        out["site_x"] = sx.reshape(e.Ly, e.Lx).T.copy()
        out["Se"] = {"northwest": sn.reshape(e.Ly, e.Lx).T.copy(), "southeast": ss.reshape(e.Ly, e.Lx).T.copy()}
    elif site_profile:
        out["site_x"] = sx.reshape(e.Ly, e.Lx).T.copy()
        out["Se"] = {"north": sn[:nb].reshape(e.Ly - 1, e.Lx - 1) if nb else np.zeros((0, 0)),
                     "south": ss[:nb].reshape(e.Ly - 1, e.Lx - 1) if nb else np.zeros((0, 0))}
    return out


SAMPLING_KINDS = {"auxiliary": 0, "physical": 1}


class SamplingCache:
    """``SamplingCache(state, contraction; kind)`` on the device: ``kind="auxiliary"``
    draws the auxiliary labels of a thermal PEPO, ``kind="physical"`` the
    physical labels of a PEPS (the Born proposal of annealed resampling,
    ``born.jl:117-134``)."""

    def __init__(self, state: DeviceState, contraction: BoundaryMPS, kind="auxiliary"):
        if kind not in SAMPLING_KINDS:
            raise ValueError("unknown sampling kind")
        self.engine = state.engine
        self.kind = kind
        cid = C.c_int32()
        b = _boundary(contraction, self.engine)
        self.engine.check(self.engine.lib.sps_sampling_cache_kind(self.engine.h, state.id, C.byref(b),
                                                                  SAMPLING_KINDS[kind], C.byref(cid)))
        self.id = cid.value

    def __del__(self):
        try:
            if self.engine.h:
                self.engine.lib.sps_sampling_cache_free(self.engine.h, self.id)
        except Exception:
            pass


def sample_configuration(cache: SamplingCache, uniforms=None, configuration=None):
    """``sample_configuration(cache; rng | configuration)`` with explicit uniforms.

    ``configuration`` / the returned configuration is an (Lx, Ly) int array of
    SymmetryBasis labels (1 even, 2 odd).
    """
    e = cache.engine
    L = e.Lx * e.Ly
    rep = _lib.sps_sample_report()
    if configuration is not None:
        cfg = np.ascontiguousarray(np.asarray(configuration, np.int32).T.reshape(-1))
        e.check(e.lib.sps_sample_probability(e.h, cache.id, _arr(cfg, C.c_int32), C.byref(rep)))
        return dict(configuration=np.asarray(configuration), log_probability=rep.log_probability,
                    max_environment_truncation=rep.max_environment_truncation, **_repairs(rep))
    if uniforms is None:
        raise ValueError("an explicit RNG is required")
    u = np.ascontiguousarray(np.asarray(uniforms, np.float64).reshape(-1))
    if u.size != L:
        raise ValueError("one uniform per site is required")
    out = np.zeros(L, np.int32)
    e.check(e.lib.sps_sample(e.h, cache.id, _arr(u, C.c_double), _arr(out, C.c_int32), C.byref(rep)))
    return dict(configuration=out.reshape(e.Ly, e.Lx).T.copy(), log_probability=rep.log_probability,
                max_environment_truncation=rep.max_environment_truncation, near_boundary=rep.near_boundary,
                **_repairs(rep))


def _repairs(rep):
    """The physical kind's PSD-repair counts of a draw (zero for the auxiliary kind)."""
    return dict(metric_repairs=rep.metric_repairs, zero_proposals=rep.zero_proposals,
                min_relative_eigenvalue=rep.min_relative_eigenvalue)


def sample_probability_batch(cache: SamplingCache, configurations):
    """``sample_configuration(cache; configuration)`` for each of n configurations
    ((n, Lx, Ly) labels) in one call: (log_probabilities, reports)."""
    e = cache.engine
    L = e.Lx * e.Ly
    cfgs = np.asarray(configurations, np.int32)
    n = cfgs.shape[0]
    flat = np.ascontiguousarray(np.transpose(cfgs, (0, 2, 1)).reshape(n, L))
    lps = np.zeros(n)
    reps = (_lib.sps_sample_report * max(n, 1))()
    e.check(e.lib.sps_sample_probability_batch(e.h, cache.id, n, _arr(flat, C.c_int32), _arr(lps, C.c_double),
                                               reps))
    return lps, [dict(max_environment_truncation=reps[i].max_environment_truncation, **_repairs(reps[i]))
                 for i in range(n)]


def sample_conditionals(cache: SamplingCache, uniforms=None, configuration=None):
    """``sample_configuration`` with its ``conditionals`` (the probability of each
    chosen label, (Lx, Ly) array) from uniforms, or for a given configuration."""
    e = cache.engine
    L = e.Lx * e.Ly
    rep = _lib.sps_sample_report()
    out = np.zeros(L, np.int32)
    cond = np.zeros(L)
    u = None if uniforms is None else np.ascontiguousarray(np.asarray(uniforms, np.float64).reshape(-1))
    g = None if configuration is None else np.ascontiguousarray(np.asarray(configuration, np.int32).T.reshape(-1))
    if u is None and g is None:
        raise ValueError("an explicit RNG is required")
    if u is not None and u.size != L:
        raise ValueError("one uniform per site is required")
    e.check(e.lib.sps_sample_conditionals(e.h, cache.id, None if u is None else _arr(u, C.c_double),
                                          None if g is None else _arr(g, C.c_int32), _arr(out, C.c_int32),
                                          _arr(cond, C.c_double), C.byref(rep)))
    return dict(configuration=out.reshape(e.Ly, e.Lx).T.copy(), conditionals=cond.reshape(e.Ly, e.Lx).T.copy(),
                log_probability=rep.log_probability, max_environment_truncation=rep.max_environment_truncation)


def sample_batch(cache: SamplingCache, uniforms, reports=False):
    """Many draws in one call: uniforms (n, Lx*Ly) -> configurations (n, Lx, Ly), log_p (n,)
    (and, with ``reports``, each draw's max_environment_truncation and near_boundary count)."""
    e = cache.engine
    L = e.Lx * e.Ly
    u = np.ascontiguousarray(np.asarray(uniforms, np.float64).reshape(-1, L))
    n = u.shape[0]
    cfg = np.zeros((n, L), np.int32)
    lp = np.zeros(n)
    rep = (_lib.sps_sample_report * max(n, 1))()
    e.check(e.lib.sps_sample_batch(e.h, cache.id, n, _arr(u, C.c_double), _arr(cfg, C.c_int32),
                                   _arr(lp, C.c_double), rep))
    cfgs = cfg.reshape(n, e.Ly, e.Lx).transpose(0, 2, 1).copy()
    if reports:
        return cfgs, lp, [dict(max_environment_truncation=rep[i].max_environment_truncation,
                               near_boundary=rep[i].near_boundary) for i in range(n)]
    return cfgs, lp


def _ids(states):
    e = states[0].engine if states else None
    if any(s.engine is not e for s in states):
        raise ValueError("a batch must hold states of one engine")
    return e, np.ascontiguousarray([s.id for s in states], np.int32)


def evolution_step_batch(states, deltas, D, contraction: BoundaryMPS, sector_space: Z2Space | None = None):
    """``evolution_step!`` on every state of ``states`` in one call (per-state ``deltas``)."""
    if not states:
        return []
    e, ids = _ids(states)
    n = len(states)
    d = np.ascontiguousarray(np.broadcast_to(np.asarray(deltas, np.float64), (n,)))
    reps = (_lib.sps_step_report * n)()
    b = _boundary(contraction, e)
    sp = None if sector_space is None else (C.c_int32 * 2)(sector_space.n0, sector_space.n1)
    e.check(e.lib.sps_evolution_step_batch(e.h, n, _arr(ids, C.c_int32), _arr(d, C.c_double), int(D), sp,
                                           C.byref(b), reps))
    return [{f: getattr(r, f) for f, _ in r._fields_} for r in reps]


def measure_energy_batch(states, contraction: BoundaryMPS):
    """``measure_energy`` of every state in one call."""
    if not states:
        return []
    e, ids = _ids(states)
    n, L = len(states), e.Lx * e.Ly
    out = (_lib.sps_energy * n)()
    sx = np.zeros(n * L)
    b = _boundary(contraction, e)
    e.check(e.lib.sps_measure_energy_batch(e.h, n, _arr(ids, C.c_int32), C.byref(b), out, _arr(sx, C.c_double)))
    res = []
    for i, r in enumerate(out):
        res.append(dict(energy_total=r.energy_total, energy_per_site=r.energy_per_site, log_norm=r.log_norm,
                        tensor_log_norm=r.tensor_log_norm, max_environment_truncation=r.max_environment_truncation,
                        x_sum=r.x_sum, zz_sum=r.zz_sum, magnetization=r.x_sum / L,
                        site_x=sx[i * L:(i + 1) * L].reshape(e.Ly, e.Lx).T.copy()))
    return res


def lognorm_batch(states, contraction: BoundaryMPS):
    """``lognorm`` of every state in one call."""
    if not states:
        return []
    e, ids = _ids(states)
    n = len(states)
    out = (_lib.sps_lognorm_result * n)()
    b = _boundary(contraction, e)
    e.check(e.lib.sps_lognorm_batch(e.h, n, _arr(ids, C.c_int32), C.byref(b), out))
    return [dict(log_norm=r.log_norm, tensor_log_norm=r.tensor_log_norm,
                 max_environment_truncation=r.max_environment_truncation) for r in out]


def project_batch(pepo: DeviceState, configurations):
    """``project_configuration`` of every configuration ((n, Lx, Ly) labels) in one call."""
    e = pepo.engine
    cfgs = np.asarray(configurations, np.int32)
    n = cfgs.shape[0]
    if n == 0:
        return [], np.zeros((0, e.Lx * e.Ly))
    flat = np.ascontiguousarray(cfgs.transpose(0, 2, 1).reshape(n, -1))
    sids = np.zeros(n, np.int32)
    ln = np.zeros((n, e.Lx * e.Ly))
    e.check(e.lib.sps_project_batch(e.h, pepo.id, n, _arr(flat, C.c_int32), _arr(sids, C.c_int32),
                                    _arr(ln, C.c_double)))
    return [DeviceState(e, int(i)) for i in sids], ln


def project_configuration(pepo: DeviceState, configuration):
    """``project_configuration(checkpoint, configuration)`` -> (PEPS state, log normalisations)."""
    e = pepo.engine
    cfg = np.ascontiguousarray(np.asarray(configuration, np.int32).T.reshape(-1))
    sid = C.c_int32()
    ln = np.zeros(e.Lx * e.Ly)
    e.check(e.lib.sps_project(e.h, pepo.id, _arr(cfg, C.c_int32), C.byref(sid), _arr(ln, C.c_double)))
    return DeviceState(e, sid.value), ln

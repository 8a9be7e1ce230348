"""Host-side mirror of the reference's internal/fk and internal/layer APIs.

The names, argument meanings and errors follow the Go package
(internal/fk/fk.go:37-550, internal/layer/layer.go:24-109,
internal/visco/visco.go:42-108); every computation runs in libgfk on the GPU.

    m = Medium(Stack([Layer(0.5, 300, 150, 1700, 15), Layer(0, 800, 400, 2000, 40)]))
    g = m.vertical_displacement_multi([1, 2, 5], 20.0, Integration())
"""
import ctypes
import math
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


class FkError(RuntimeError):
    """A failed fk call: .status is the gfk_status code, str() the message."""

    def __init__(self, status, message):
        super().__init__(message or N.STATUS_NAMES.get(status, str(status)))
        self.status = status


# ------------------------------------------------------------------ medium --

@dataclass
class Layer:
    """layer.Layer (internal/layer/layer.go:24-36). qp <= 0 means 2.25*Qs."""
    thickness: float = 0.0
    vp: float = 0.0
    vs: float = 0.0
    density: float = 0.0
    qs: float = 0.0
    qp: float = 0.0

    def shear_modulus(self):
        return self.density * self.vs * self.vs

    def lame_lambda(self):
        return self.density * (self.vp * self.vp - 2 * self.vs * self.vs)


class Stack(list):
    """layer.Stack: layers over a half-space, the last entry (layer.go:40-109)."""

    def half_space(self):
        return self[-1]

    def velocity_bounds(self):
        vs = [l.vs for l in self]
        return min(vs), max(vs)

    def total_thickness(self):
        return sum(l.thickness for l in self[:-1])

    def validate(self):
        """Raises FkError(ESTACK) where layer.Stack.Validate returns an error."""
        with _c_medium(Medium(self)) as cm:
            st = N.lib().gfk_stack_validate(ctypes.byref(cm))
        if st:
            raise FkError(st, _stack_message(self))


def uniform(vp, vs, density, qs):
    """layer.Uniform (layer.go:45-47): a one-entry stack, the half-space alone."""
    return Stack([Layer(0.0, vp, vs, density, qs)])


@dataclass
class SLS:
    """visco.SLS (internal/visco/visco.go:42-47)."""
    tau_sigma: float
    tau_eps: float

    @staticmethod
    def fit(q, f0):
        """visco.Fit (visco.go:55-68): minimum Q of q at f0."""
        if q <= 0:
            raise FkError(N.EARG, f"visco: Q must be positive, got {q:g}")
        if f0 <= 0:
            raise FkError(N.EARG, f"visco: reference frequency must be positive, got {f0:g} Hz")
        w0 = 2 * math.pi * f0
        root = math.sqrt(1 + 1 / (q * q))
        return SLS((root - 1 / q) / w0, (root + 1 / q) / w0)


@dataclass
class Integration:
    """fk.Integration (fk.go:330-341): samples <= 0 and kmax_factor <= 0 take
    defaults. kmax > 0 fixes the cut at max(kmax, 40/r_min) for every
    frequency, which Integration{KMaxFactor: kmax/k_body(f)} expresses per
    frequency in the reference."""
    samples: int = 0
    kmax_factor: float = 0.0
    kmax: float = 0.0

    def c(self):
        return N.GfkIntegration(int(self.samples), 0, float(self.kmax_factor), float(self.kmax))


@dataclass
class Grid:
    """fk.Grid (fk.go:446-449)."""
    kmax: float
    samples: int


MAX_LAYER_PHASE = 16.0  # fk.go:242


@dataclass
class Medium:
    """fk.Medium (fk.go:37-53) plus how libgfk solves it.

    formulation: N.REFERENCE_DIRECT (the reference algorithm: Qp = 2.25 Qs,
    real frequencies, MaxLayerPhase guard) or N.DUNKIN (compound-matrix
    propagation, per-layer Qp, complex frequency offset omega_imag, no guard
    unless guard=True).
    """
    stack: Stack
    ref_freq: float = 0.0
    default_q: float = 0.0
    relax: SLS = None
    formulation: int = N.REFERENCE_DIRECT
    omega_imag: float = 0.0
    guard: bool = False
    quadrature: int = N.PLAIN_FP64
    engine: "Engine" = field(default=None, repr=False, compare=False)

    # -- host rules -------------------------------------------------------
    def check_layer_phase(self, freq):
        """Medium.checkLayerPhase (fk.go:251-266)."""
        with _c_medium(self) as cm:
            st = N.lib().gfk_check_layer_phase(ctypes.byref(cm), float(freq))
        if st:
            raise FkError(st, _guard_message(self, freq) if st == N.EGUARD else _stack_message(self.stack))

    def grid_for(self, ranges, freq, opt=None):
        """Medium.GridFor (fk.go:464-495)."""
        opt = opt or Integration()
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        g = N.GfkGrid()
        with _c_medium(self) as cm:
            st = N.lib().gfk_grid_for(ctypes.byref(cm), _dp(r), len(r), float(freq), opt.c(), ctypes.byref(g))
        if st:
            msg = "fk: no ranges given" if len(r) == 0 else f"fk: range must be positive, got {r[r <= 0][0]:g} m" \
                if st == N.EARG and (r <= 0).any() else N.STATUS_NAMES[st]
            raise FkError(st, msg)
        return Grid(g.kmax, g.samples)

    # -- the path (GPU) ----------------------------------------------------
    def surface_response(self, k, freq):
        """Medium.SurfaceResponse (fk.go:276-327). Scalars or equal-length arrays."""
        kk = np.atleast_1d(np.asarray(k, dtype=np.float64))
        ff = np.broadcast_to(np.asarray(freq, dtype=np.float64), kk.shape)
        kk, ff = np.ascontiguousarray(kk.ravel()), np.ascontiguousarray(ff.ravel())
        out = np.zeros(2 * kk.size)
        eng = self._engine()
        with _c_medium(self) as cm:
            st = N.lib().gfk_surface_response(eng.ctx, ctypes.byref(cm), ctypes.byref(self._solve()), _dp(kk),
                                              _dp(ff), kk.size, _dp(out))
        eng.check(st)
        u = out[0::2] + 1j * out[1::2]
        return complex(u[0]) if np.ndim(k) == 0 and np.ndim(freq) == 0 else u.reshape(np.shape(k))

    def static_coefficient(self, freq, k_far):
        """Medium.StaticCoefficient (fk.go:365-371)."""
        out = (ctypes.c_double * 2)()
        eng = self._engine()
        with _c_medium(self) as cm:
            st = N.lib().gfk_static_coefficient(eng.ctx, ctypes.byref(cm), ctypes.byref(self._solve()),
                                                float(freq), float(k_far), out)
        eng.check(st)
        return complex(out[0], out[1])

    def vertical_displacement(self, r, freq, opt=None):
        """Medium.VerticalDisplacement (fk.go:396-443), m/N."""
        opt = opt or Integration()
        out = (ctypes.c_double * 2)()
        eng = self._engine()
        with _c_medium(self) as cm:
            st = N.lib().gfk_vertical_displacement(eng.ctx, ctypes.byref(cm), ctypes.byref(self._solve()),
                                                   float(r), float(freq), opt.c(), out)
        eng.check(st)
        return complex(out[0], out[1])

    def vertical_displacement_multi(self, ranges, freq, opt=None):
        """Medium.VerticalDisplacementMulti (fk.go:506-550): one frequency, many ranges."""
        opt = opt or Integration()
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        out = np.zeros(2 * len(r))
        eng = self._engine()
        with _c_medium(self) as cm:
            st = N.lib().gfk_vertical_displacement_multi(eng.ctx, ctypes.byref(cm), ctypes.byref(self._solve()),
                                                         _dp(r), len(r), float(freq), opt.c(), _dp(out))
        eng.check(st)
        return out[0::2] + 1j * out[1::2]

    def bank_spectra(self, ranges, freqs, opt=None, raise_on_error=True, out=None):
        """VerticalDisplacementMulti at many frequencies in one GPU call, as
        cmd/geobank/main.go:133-167 builds a bank. Returns ([nf, nr] complex128,
        per-frequency status); raises on the first failing frequency unless
        raise_on_error is False. `out` may supply the [nf, 2 nr] float64
        (re, im) buffer; in page-locked memory a larger bank is downloaded in
        chunks while the rest computes."""
        opt = opt or Integration()
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        if out is None:
            out = np.zeros((len(f), 2 * len(r)))
        elif out.shape != (len(f), 2 * len(r)) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (len(freqs), 2 len(ranges))")
        status = np.zeros(len(f), dtype=np.int32)
        eng = self._engine()
        with _c_medium(self) as cm:
            st = N.lib().gfk_bank_spectra(eng.ctx, ctypes.byref(cm), ctypes.byref(self._solve()), _dp(r), len(r),
                                          _dp(f), len(f), opt.c(), _dp(out),
                                          status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        if st and raise_on_error:
            eng.check(st)
        return out[:, 0::2] + 1j * out[:, 1::2], status

    # -- helpers -----------------------------------------------------------
    def bank_payload(self, ranges, freqs, first_bin, bins, opt=None, raise_on_error=True, out=None):
        """The build ending in the bank file's float32 payload, packed on the
        device (gfk_bank_payload): [len(ranges), bins, 2] float32 with the
        spectra at bins first_bin.. and zeros elsewhere; per-frequency status."""
        opt = opt or Integration()
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        if out is None:
            out = np.zeros((len(r), bins, 2), dtype=np.float32)
        status = np.zeros(len(f), dtype=np.int32)
        eng = self._engine()
        with _c_medium(self) as cm:
            st = N.lib().gfk_bank_payload(eng.ctx, ctypes.byref(cm), ctypes.byref(self._solve()), _dp(r), len(r),
                                          _dp(f), len(f), opt.c(), int(first_bin), int(bins),
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        if st and raise_on_error:
            eng.check(st)
        return out, status

    def _solve(self):
        return N.GfkSolve(int(self.formulation), int(self.quadrature), 1 if self.guard else 0, 0,
                          float(self.omega_imag))

    def _engine(self):
        return self.engine or default_engine()


# ------------------------------------------------------------------ engine --

class Engine:
    """One libgfk context (one CUDA stream) on one device."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        st = N.lib().gfk_open(int(device), ctypes.byref(h))
        if st:
            raise FkError(st, f"gfk_open(device={device}) failed: {N.status_string(st)} "
                              "(libgfk needs a CUDA device; there is no CPU fallback)")
        self.ctx = h
        self.device = device
        self._plans = weakref.WeakSet()

    def check(self, st):
        if st:
            msg = N.lib().gfk_last_error(self.ctx).decode() or N.status_string(st)
            raise FkError(st, msg)

    def kernel_launches(self):
        return int(N.lib().gfk_kernel_launches(self.ctx))

    def stream(self):
        """The context's CUDA stream handle (an integer cudaStream_t)."""
        return int(N.lib().gfk_stream(self.ctx) or 0)

    def close(self):
        if self.ctx:
            for p in list(self._plans):
                p.close()
            N.lib().gfk_close(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = None


def default_engine():
    global _default
    if _default is None:
        _default = Engine(0)
    return _default


def prop_shape(variant):
    """gfk_prop_shape: launch shape `variant` of the Dunkin propagator as a dict."""
    v = [ctypes.c_int32() for _ in range(5)]
    st = N.lib().gfk_prop_shape(int(variant), *[ctypes.byref(x) for x in v])
    if st != 0:
        raise FkError(st, f"no propagator launch shape {variant}")
    keys = ("threads", "blocks_per_sm", "wavenumbers_per_thread", "runs_per_item")
    d = {"index": int(variant), **{k: int(x.value) for k, x in zip(keys, v)}}
    d["persistent"] = bool(v[4].value)
    return d


class Plan:
    """gfk_plan: a fixed (medium, ranges, frequencies, integration) build that
    recomputes everything on the device per execute()."""

    def __init__(self, medium, ranges, freqs, opt=None, engine=None):
        self.p = None
        self.engine = engine or medium.engine or default_engine()
        self.ranges = np.ascontiguousarray(ranges, dtype=np.float64)
        self.freqs = np.ascontiguousarray(freqs, dtype=np.float64)
        opt = opt or Integration()
        h = ctypes.c_void_p()
        with _c_medium(medium) as cm:
            st = N.lib().gfk_plan_create(self.engine.ctx, ctypes.byref(cm), ctypes.byref(medium._solve()),
                                         _dp(self.ranges), len(self.ranges), _dp(self.freqs), len(self.freqs),
                                         opt.c(), ctypes.byref(h))
        self.engine.check(st)
        self.p = h
        self.engine._plans.add(self)

    def use_graph(self, enable=True):
        """From the next execute on, run each execute as one captured CUDA graph."""
        self.engine.check(N.lib().gfk_plan_use_graph(self.p, 1 if enable else 0))

    def execute(self):
        self.engine.check(N.lib().gfk_plan_execute(self.p))

    def result_device_ptr(self):
        d = ctypes.c_void_p()
        self.engine.check(N.lib().gfk_plan_result_device(self.p, ctypes.byref(d)))
        return d.value

    def download(self, raise_on_error=True, out=None):
        """([rows, ranges] complex128, per-row status). The rows land directly
        in a complex array (its memory is the (re, im) pairs the ABI writes);
        `out` may supply one (e.g. in pinned memory) to reuse."""
        shape = (len(self.freqs), len(self.ranges))
        if out is None:
            out = np.empty(shape, dtype=np.complex128)
        elif out.shape != shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise FkError(N.EARG, f"download buffer must be a C-contiguous complex128 array of shape {shape}")
        status = np.zeros(len(self.freqs), dtype=np.int32)
        st = N.lib().gfk_plan_download(self.p, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        if st and raise_on_error:
            self.engine.check(st)
        return out, status

    def execute_download(self, raise_on_error=True, out=None):
        """execute() then download(), with each row chunk copied into `out`
        while the next one computes when `out` is page-locked (gfk_plan_execute_download)."""
        shape = (len(self.freqs), len(self.ranges))
        if out is None:
            out = np.empty(shape, dtype=np.complex128)
        elif out.shape != shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise FkError(N.EARG, f"download buffer must be a C-contiguous complex128 array of shape {shape}")
        status = np.zeros(len(self.freqs), dtype=np.int32)
        st = N.lib().gfk_plan_execute_download(self.p, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        if st and raise_on_error:
            self.engine.check(st)
        return out, status

    def statuses(self):
        """Per-row status codes of the last execute, without moving the result."""
        status = np.zeros(len(self.freqs), dtype=np.int32)
        N.lib().gfk_plan_download(self.p, None, status.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return status

    def launches_per_execute(self):
        return int(N.lib().gfk_plan_launches_per_execute(self.p))

    def tuning(self):
        """(chosen propagator launch shape, ms per shape) from the first execute."""
        v = ctypes.c_int32()
        ms = (ctypes.c_float * 16)()
        n = N.lib().gfk_plan_tuning(self.p, ctypes.byref(v), ms, 16)
        return int(v.value), [float(ms[i]) for i in range(max(n, 0))]

    def prop_shape(self):
        """The chosen propagator launch shape, described (prop_shape())."""
        return prop_shape(self.tuning()[0])

    def quad_shape(self):
        """(ranges per CTA, pipeline stages, ms per shape) of the tensor-core
        sum chosen by the first execute; (0, 0, []) otherwise."""
        tn, ns = ctypes.c_int32(), ctypes.c_int32()
        ms = (ctypes.c_float * 16)()
        n = N.lib().gfk_plan_quad_shape(self.p, ctypes.byref(tn), ctypes.byref(ns), ms, 16)
        return int(tn.value), int(ns.value), [float(ms[i]) for i in range(max(n, 0))]

    def kernel_times(self, reset=False):
        """(propagator, quadrature, other) ms per execute, CUDA-event timed."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.engine.check(N.lib().gfk_plan_kernel_times(self.p, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                        1 if reset else 0))
        return a.value, b.value, c.value

    def close(self):
        if self.p:
            if self.engine.ctx:  # a closed engine has destroyed its plans already
                N.lib().gfk_plan_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch(Plan):
    """gfk_batch_create: one plan over many media, each with its own
    frequencies, sharing ranges, integration and solve options (taken from
    the first medium). Rows are ordered medium by medium."""

    def __init__(self, media, freqs_per_medium, ranges, opt=None, engine=None):
        self.p = None
        media = list(media)
        if not media:
            raise FkError(N.EARG, "no media given")
        self.engine = engine or media[0].engine or default_engine()
        self.ranges = np.ascontiguousarray(ranges, dtype=np.float64)
        self._freqs = [np.ascontiguousarray(f, dtype=np.float64) for f in freqs_per_medium]
        if len(self._freqs) != len(media):
            raise FkError(N.EARG, "one frequency list per medium")
        self.freqs = np.concatenate(self._freqs) if self._freqs else np.zeros(0)
        self.counts = np.array([len(f) for f in self._freqs], dtype=np.int64)
        opt = opt or Integration()
        holders = [_c_medium(m) for m in media]
        arr = (N.GfkMedium * len(media))(*[h.c for h in holders])
        fptrs = (ctypes.POINTER(ctypes.c_double) * len(media))(*[_dp(f) for f in self._freqs])
        nfs = (ctypes.c_int32 * len(media))(*[len(f) for f in self._freqs])
        h = ctypes.c_void_p()
        st = N.lib().gfk_batch_create(self.engine.ctx, arr, len(media), fptrs, nfs, ctypes.byref(media[0]._solve()),
                                      _dp(self.ranges), len(self.ranges), opt.c(), ctypes.byref(h))
        del holders
        self.engine.check(st)
        self.p = h
        self.engine._plans.add(self)

    def split(self, rows):
        """Splits a [sum nf, ...] result into one array per medium."""
        return np.split(rows, np.cumsum(self.counts)[:-1])

    @classmethod
    def from_layers(cls, layers, counts, freqs, ranges, opt=None, solve=None, engine=None, freqs_per_medium=None):
        """A batch plan built straight from arrays, for sweeps over many soils:
        layers [total entries, 6] (thickness, Vp, Vs, density, Qs, Qp; each
        medium's entries consecutive, half-space last), counts [media]; every
        medium solved at `freqs` unless `freqs_per_medium` (a list of arrays)
        is given. solve: (formulation, quadrature, omega_imag); media take the
        default reference frequency and Q."""
        self = cls.__new__(cls)
        self.p = None
        self.engine = engine or default_engine()
        lay = np.ascontiguousarray(layers, dtype=np.float64)
        cnt = np.ascontiguousarray(counts, dtype=np.int32)
        nm = len(cnt)
        if lay.ndim != 2 or lay.shape[1] != 6 or int(cnt.sum()) != len(lay) or nm == 0:
            raise FkError(N.EARG, "layers must be [sum(counts), 6] and counts non-empty")
        starts = np.concatenate([[0], np.cumsum(cnt)[:-1]]).astype(np.uint64)
        med_dt = np.dtype([("layers", np.uint64), ("count", np.int32), ("_pad", np.int32), ("ref", np.float64),
                           ("dq", np.float64), ("ts", np.float64), ("te", np.float64)])
        meds = np.zeros(nm, dtype=med_dt)
        meds["layers"] = np.uint64(lay.ctypes.data) + starts * np.uint64(48)
        meds["count"] = cnt
        self.ranges = np.ascontiguousarray(ranges, dtype=np.float64)
        if freqs_per_medium is None:
            f = np.ascontiguousarray(freqs, dtype=np.float64)
            self._freqs = [f] * nm
            fptr = np.full(nm, f.ctypes.data, dtype=np.uint64)
            nfs = np.full(nm, len(f), dtype=np.int32)
        else:
            self._freqs = [np.ascontiguousarray(x, dtype=np.float64) for x in freqs_per_medium]
            if len(self._freqs) != nm:
                raise FkError(N.EARG, "one frequency list per medium")
            fptr = np.array([x.ctypes.data for x in self._freqs], dtype=np.uint64)
            nfs = np.array([len(x) for x in self._freqs], dtype=np.int32)
        self.freqs = np.concatenate(self._freqs) if self._freqs else np.zeros(0)
        self.counts = nfs.astype(np.int64)
        form, quad, wi = solve if solve is not None else (N.DUNKIN, N.PLAIN_FP64, 0.0)
        sv = N.GfkSolve(int(form), int(quad), 0, 0, float(wi))
        opt = opt or Integration()
        h = ctypes.c_void_p()
        st = N.lib().gfk_batch_create(self.engine.ctx, meds.ctypes.data_as(ctypes.POINTER(N.GfkMedium)), nm,
                                      fptr.ctypes.data_as(ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
                                      nfs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(sv),
                                      _dp(self.ranges), len(self.ranges), opt.c(), ctypes.byref(h))
        del lay, meds
        self.engine.check(st)
        self.p = h
        self.engine._plans.add(self)
        return self


# ----------------------------------------------------------------- plumbing --

def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class _c_medium:
    """Context manager holding a gfk_medium (and its layer array) alive."""

    def __init__(self, m):
        stack = m.stack
        self.arr = (N.GfkLayer * max(1, len(stack)))(
            *[N.GfkLayer(l.thickness, l.vp, l.vs, l.density, l.qs, l.qp) for l in stack])
        sls = m.relax
        self.c = N.GfkMedium(self.arr if len(stack) else None, len(stack), 0, float(m.ref_freq), float(m.default_q),
                             sls.tau_sigma if sls else 0.0, sls.tau_eps if sls else 0.0)

    def __enter__(self):
        return self.c

    def __exit__(self, *a):
        return False


def _stack_message(stack):
    if len(stack) == 0:
        return "layer: a stack needs at least a half-space"
    for i, l in enumerate(stack):
        if l.vs <= 0:
            return f"layer {i}: Vs must be positive, got {l.vs:g} m/s"
        if l.vp <= 0:
            return f"layer {i}: Vp must be positive, got {l.vp:g} m/s"
        if l.density <= 0:
            return f"layer {i}: density must be positive, got {l.density:g} kg/m^3"
        if l.vp <= math.sqrt(2) * l.vs:
            return (f"layer {i}: Vp={l.vp:g} must exceed sqrt(2)*Vs={math.sqrt(2) * l.vs:g} "
                    "for a non-negative Poisson ratio")
        if i < len(stack) - 1 and l.thickness <= 0:
            return f"layer {i}: thickness must be positive, got {l.thickness:g} m"
    return "layer: invalid stack"


def _guard_message(m, freq):
    slowest, _ = m.stack.velocity_bounds()
    k = 2 * math.pi * freq / (0.87 * slowest)
    for i, l in enumerate(m.stack[:-1]):
        kh = k * l.thickness
        if kh > MAX_LAYER_PHASE:
            return (f"fk: layer {i} is {l.thickness:g} m thick, which is k*h = {kh:.1f} at {freq:g} Hz and past the "
                    f"{MAX_LAYER_PHASE:.0f} this propagator stays accurate to; it would return a plausible wrong "
                    f"number rather than fail. Band-limit to "
                    f"{MAX_LAYER_PHASE * 0.87 * slowest / (2 * math.pi * l.thickness):.0f} Hz for this stack, or "
                    "reformulate the solve with compound matrices as internal/propmat does")
    return "fk: layer phase guard"

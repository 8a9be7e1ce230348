"""Green's-function bank files: the reference's internal/bank format.

Mirrors internal/bank/format.go (Header, RangeGrid, Provenance, New, Set, At,
Write, Open) and cmd/geobank's build loop (cmd/geobank/main.go:51-178), with the
spectra computed by libgfk on the GPU and the file written by libgfk's
gfk_bank_write. Layout (format.go:32-46): "GEOBANK\\0", uint32 version,
uint32 header length, JSON header, zero padding to 4096 bytes, float32
(re, im) payload in range-major order, little-endian.
"""
import ctypes
import json
import math
import struct
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .fk import FkError, Integration, Layer, Medium, Stack

FORMAT_VERSION = 1  # format.go:63
MAGIC = b"GEOBANK\x00"  # format.go:65
PAGE_SIZE = 4096  # format.go:70


@dataclass
class Provenance:
    """format.go:74-84."""
    solver: str = ""
    config_hash: str = ""
    created: str = ""
    notes: str = ""

    def to_json(self):
        d = {"solver": self.solver}
        for k in ("config_hash", "created", "notes"):  # omitempty
            if getattr(self, k):
                d[k] = getattr(self, k)
        return d


@dataclass
class RangeGrid:
    """format.go:92-112."""
    min_m: float
    max_m: float
    count: int

    def at(self, i):
        if self.count <= 1:
            return self.min_m
        return self.min_m + (self.max_m - self.min_m) * i / (self.count - 1)

    def spacing(self):
        if self.count <= 1:
            return 0.0
        return (self.max_m - self.min_m) / (self.count - 1)

    def ranges(self):
        return np.array([self.at(i) for i in range(self.count)], dtype=np.float64)


@dataclass
class Header:
    """format.go:115-165."""
    provenance: Provenance
    medium: Stack
    sample_rate_hz: float
    samples: int
    ranges: RangeGrid
    component: str
    units: str
    format_version: int = FORMAT_VERSION

    def bins(self):
        return self.samples // 2 + 1

    def frequency_at(self, k):
        return k * self.sample_rate_hz / self.samples

    def validate(self):
        """Header.Validate (format.go:142-165)."""
        if self.format_version != FORMAT_VERSION:
            raise FkError(N.EARG, f"bank: format version {self.format_version}, this build reads {FORMAT_VERSION}")
        if self.samples <= 0 or self.samples % 2 != 0:
            raise FkError(N.EARG, f"bank: samples must be positive and even, got {self.samples}")
        if self.sample_rate_hz <= 0:
            raise FkError(N.EARG, f"bank: sample rate must be positive, got {self.sample_rate_hz:g}")
        if self.ranges.count <= 0:
            raise FkError(N.EARG, f"bank: range grid must have at least one entry, got {self.ranges.count}")
        if self.ranges.min_m <= 0:
            raise FkError(N.EARG, f"bank: minimum range must be positive, got {self.ranges.min_m:g} m")
        if self.ranges.count > 1 and self.ranges.max_m <= self.ranges.min_m:
            raise FkError(N.EARG, f"bank: maximum range {self.ranges.max_m:g} m must exceed minimum "
                                  f"{self.ranges.min_m:g} m")
        if not self.component:
            raise FkError(N.EARG, "bank: component must be named")
        if len(self.medium) > 0:
            try:
                Stack(self.medium).validate()
            except FkError as e:
                raise FkError(e.status, f"bank: {e}") from None

    def check_range_sampling(self, max_freq):
        """Header.CheckRangeSampling (internal/bank/interp.go:132-144)."""
        if self.ranges.count <= 1 or len(self.medium) == 0:
            return
        slowest, _ = Stack(self.medium).velocity_bounds()
        limit = range_nyquist(0.87 * slowest, max_freq) / 2
        got = self.ranges.spacing()
        if got > limit:
            raise FkError(N.EARG, f"bank: range spacing {got:.4f} m is too coarse to unwrap phase up to "
                                  f"{max_freq:g} Hz; need under {limit:.4f} m")

    def to_json(self):
        """The JSON header with the Go struct's field names and order."""
        med = []
        for l in self.medium:
            d = {"thickness_m": _num(l.thickness), "vp_mps": _num(l.vp), "vs_mps": _num(l.vs),
                 "density_kgm3": _num(l.density)}
            if l.qs:
                d["qs"] = _num(l.qs)
            if l.qp:  # an extension field; the reference's json.Unmarshal ignores it
                d["qp"] = _num(l.qp)
            med.append(d)
        h = {"format_version": self.format_version, "provenance": self.provenance.to_json(), "medium": med,
             "sample_rate_hz": _num(self.sample_rate_hz), "samples": int(self.samples),
             "ranges": {"min_m": _num(self.ranges.min_m), "max_m": _num(self.ranges.max_m),
                        "count": int(self.ranges.count)},
             "component": self.component, "units": self.units}
        return json.dumps(h, separators=(",", ":"), ensure_ascii=False)

    @staticmethod
    def from_json(raw):
        d = json.loads(raw)
        prov = d.get("provenance") or {}
        med = Stack(Layer(l.get("thickness_m", 0.0), l.get("vp_mps", 0.0), l.get("vs_mps", 0.0),
                          l.get("density_kgm3", 0.0), l.get("qs", 0.0), l.get("qp", 0.0))
                    for l in (d.get("medium") or []))
        r = d.get("ranges") or {}
        return Header(Provenance(prov.get("solver", ""), prov.get("config_hash", ""), prov.get("created", ""),
                                 prov.get("notes", "")), med, float(d.get("sample_rate_hz", 0)),
                      int(d.get("samples", 0)), RangeGrid(float(r.get("min_m", 0)), float(r.get("max_m", 0)),
                                                          int(r.get("count", 0))),
                      d.get("component", ""), d.get("units", ""), int(d.get("format_version", 0)))


def _num(x):
    """A float as Go's encoding/json writes it: integral values without '.0'."""
    x = float(x)
    if math.isfinite(x) and x == int(x) and abs(x) < 1e21:
        return int(x)
    return x


def range_nyquist(slowest_velocity, max_freq):
    """bank.RangeNyquist (internal/bank/interp.go:120-125)."""
    if max_freq <= 0:
        return math.inf
    return slowest_velocity / (2 * max_freq)


@dataclass
class Bank:
    """bank.Bank: a header and Count x Bins complex responses (format.go:167-212)."""
    header: Header
    data: np.ndarray = field(default=None)  # float32 [count, bins, 2]

    @staticmethod
    def new(h):
        """bank.New (format.go:177-182)."""
        h.validate()
        return Bank(h, np.zeros((h.ranges.count, h.bins(), 2), dtype=np.float32))

    def _check(self, i, k):
        if not 0 <= i < self.header.ranges.count:
            raise FkError(N.EARG, f"bank: range index {i} out of range [0, {self.header.ranges.count})")
        if not 0 <= k < self.header.bins():
            raise FkError(N.EARG, f"bank: bin {k} out of range [0, {self.header.bins()})")

    def set(self, i, k, v):
        """Bank.Set (format.go:185-193): stored as float32 (re, im)."""
        self._check(i, k)
        self.data[i, k, 0] = np.float32(v.real)
        self.data[i, k, 1] = np.float32(v.imag)

    def at(self, i, k):
        self._check(i, k)
        return complex(float(self.data[i, k, 0]), float(self.data[i, k, 1]))

    def complex(self):
        return self.data[..., 0].astype(np.complex64) + 1j * self.data[..., 1].astype(np.complex64)

    def size_bytes(self):
        return 4 * self.data.size

    def _payload(self):
        return np.ascontiguousarray(self.data, dtype=np.float32)

    def tables(self, engine=None):
        """Bank.prepare (internal/bank/interp.go:66-102) on the GPU: the FP64
        log-magnitude and range-unwrapped phase tables, [count, bins] each."""
        from .fk import default_engine
        eng = engine or default_engine()
        c, b = self.header.ranges.count, self.header.bins()
        lm = np.zeros((c, b))
        ph = np.zeros((c, b))
        pl = self._payload()
        eng.check(N.lib().gfk_bank_tables(eng.ctx, pl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), c, b,
                                          lm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          ph.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return lm, ph

    def impulse_responses(self, ranges, length, sensor=None, velocity=True, engine=None):
        """Causal impulse responses at the given ranges, as internal/sensing
        builds them from a bank (sensing.go:196-204): Bank.Response at every
        bin, times i w (velocity) and the sensor's complex response per bin
        (`sensor`, length bins, or None), through dsp.CausalImpulseResponseAt
        with the bank's transform size. [len(ranges), length] on the GPU."""
        from .fk import default_engine
        eng = engine or default_engine()
        h = self.header
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        out = np.zeros((len(r), int(length)))
        sp = None
        if sensor is not None:
            sc = np.asarray(sensor, dtype=np.complex128)
            sa = np.ascontiguousarray(np.stack([sc.real, sc.imag], axis=1).ravel())
            sp = sa.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        pl = self._payload()
        eng.check(N.lib().gfk_bank_impulse_responses(
            eng.ctx, pl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), h.ranges.count, h.bins(),
            float(h.ranges.min_m), float(h.ranges.max_m), float(h.sample_rate_hz), int(h.samples),
            r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r), sp, 1 if velocity else 0, int(length),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def device(self, engine=None):
        """The bank uploaded once, with Bank.prepare's tables built on the
        device, for repeated queries (DeviceBank)."""
        return DeviceBank(self, engine)

    def write(self, path):
        """bank.Write (format.go:215-240), through libgfk's gfk_bank_write."""
        self.header.validate()
        want = (self.header.ranges.count, self.header.bins(), 2)
        if self.data.shape != want:
            raise FkError(N.EARG, f"bank: payload has {self.data.size} floats, header implies {2 * want[0] * want[1]}")
        payload = np.ascontiguousarray(self.data, dtype="<f4")
        st = N.lib().gfk_bank_write(str(path).encode(), self.header.to_json().encode(),
                                    payload.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), payload.size)
        if st:
            raise FkError(st, f"bank: writing {path} failed")


class DeviceBank:
    """A bank resident on the device (gfk_bank_device_open): internal/sensing
    loads a bank once and queries it contact after contact
    (sensing.go:196-204), so the payload and its tables stay on the GPU and a
    query moves only its ranges in and its responses out."""

    def __init__(self, bank, engine=None):
        from .fk import default_engine
        self.engine = engine or default_engine()
        self.header = bank.header
        h = bank.header
        pl = bank._payload()
        p = ctypes.c_void_p()
        self.engine.check(N.lib().gfk_bank_device_open(
            self.engine.ctx, pl.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), h.ranges.count, h.bins(),
            float(h.ranges.min_m), float(h.ranges.max_m), float(h.sample_rate_hz), int(h.samples), ctypes.byref(p)))
        self.p = p.value

    def impulse_responses(self, ranges, length, sensor=None, velocity=True, out=None, out_device_ptr=None):
        """Bank.impulse_responses against the resident bank: into out (host,
        [len(ranges), length] float64, e.g. pinned; allocated when None) or,
        with out_device_ptr, into device memory (returns None)."""
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        sp = None
        if sensor is not None:
            sc = np.asarray(sensor, dtype=np.complex128)
            sa = np.ascontiguousarray(np.stack([sc.real, sc.imag], axis=1).ravel())
            sp = sa.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if out_device_ptr is not None:
            self.engine.check(N.lib().gfk_bank_device_impulse_responses(
                self.p, r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r), sp, 1 if velocity else 0,
                int(length), ctypes.c_void_p(out_device_ptr), 1))
            return None
        if out is None:
            out = np.zeros((len(r), int(length)))
        elif out.shape != (len(r), int(length)) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (len(ranges), length)")
        self.engine.check(N.lib().gfk_bank_device_impulse_responses(
            self.p, r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r), sp, 1 if velocity else 0,
            int(length), out.ctypes.data_as(ctypes.c_void_p), 0))
        return out

    def close(self):
        if self.p:
            N.lib().gfk_bank_device_close(self.p)
            self.p = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def open_bank(path):
    """bank.Open (format.go:249-286)."""
    with open(path, "rb") as fh:
        raw = fh.read()
    if len(raw) < 16 or raw[:8] != MAGIC:
        raise FkError(N.EIO, f"bank: {path} is not a Green's function bank")
    version, hdr_len = struct.unpack_from("<II", raw, 8)
    if version != FORMAT_VERSION:
        raise FkError(N.EIO, f"bank: {path} is format version {version}, this build reads {FORMAT_VERSION}")
    if 16 + hdr_len > len(raw):
        raise FkError(N.EIO, f"bank: {path} has a header length of {hdr_len} that runs past the file")
    h = Header.from_json(raw[16:16 + hdr_len])
    h.validate()
    off = 16 + hdr_len
    if off % PAGE_SIZE:
        off += PAGE_SIZE - off % PAGE_SIZE
    want = 2 * h.ranges.count * h.bins()
    if (len(raw) - off) // 4 < want:
        raise FkError(N.EIO, f"bank: {path} has {(len(raw) - off) // 4} payload floats, header implies {want}")
    data = np.frombuffer(raw, dtype="<f4", count=want, offset=off).reshape(h.ranges.count, h.bins(), 2).copy()
    return Bank(h, data)


def build_bank(medium, header, max_freq, opt=None, check_range_sampling=True, spectra=False):
    """geobank build (cmd/geobank/main.go:51-178) on the GPU: bins 1..topBin are
    computed in one batched call and packed into the float32 payload on the
    device (gfk_bank_payload); DC and bins above max_freq stay zero; the
    first failing bin aborts the build as geobank does. Returns (bank, the
    FP64 spectra [bins, ranges] if spectra=True — a second solve — else None)."""
    header.validate()
    if check_range_sampling:
        header.check_range_sampling(max_freq)
    b = Bank.new(header)
    top = int(max_freq / (header.sample_rate_hz / header.samples))
    if top >= header.bins():
        top = header.bins() - 1
    if top < 1:
        return b, (np.zeros((0, header.ranges.count), dtype=np.complex128) if spectra else None)
    freqs = np.array([header.frequency_at(k) for k in range(1, top + 1)])
    payload, status = medium.bank_payload(header.ranges.ranges(), freqs, 1, header.bins(), opt or Integration(),
                                          raise_on_error=False)
    bad = np.nonzero(status)[0]
    if len(bad):
        k = int(bad[0]) + 1
        try:
            medium.bank_spectra(header.ranges.ranges(), freqs[bad[0]:bad[0] + 1], opt or Integration())
        except FkError as e:
            raise FkError(e.status, f"bin {k} ({freqs[bad[0]]:.3f} Hz): {e}") from None
        raise FkError(int(status[bad[0]]), f"bin {k} ({freqs[bad[0]]:.3f} Hz) failed")
    sp = medium.bank_spectra(header.ranges.ranges(), freqs, opt or Integration())[0] if spectra else None
    b.data = payload
    return b, sp

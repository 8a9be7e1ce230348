"""ctypes wrapper of the CPU oracle (oracle/gfk_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
benchmark's CPU-baseline leg, always as the checker, never as the thing
measured for the GPU path or shipped.

Media are given as sequences of layers, each a tuple
(thickness_m, vp_mps, vs_mps, density_kgm3, qs, qp), the last one the
half-space (internal/layer/layer.go:24-40).
"""
import ctypes
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libgfk_oracle.so"

REFERENCE_DIRECT = 0
DUNKIN = 1

STATUS = {0: "ok", 1: "EARG", 2: "ESTACK", 3: "EGUARD", 4: "ESINGULAR", 5: "ENONFINITE",
          6: "ETIMEOUT", 7: "ECUDA", 8: "ENOMEM", 9: "EIO", 10: "ELIMIT"}


class OracleError(RuntimeError):
    def __init__(self, status):
        super().__init__(f"oracle: {STATUS.get(status, status)}")
        self.status = status


class Layer(ctypes.Structure):
    _fields_ = [("thickness_m", ctypes.c_double), ("vp_mps", ctypes.c_double),
                ("vs_mps", ctypes.c_double), ("density_kgm3", ctypes.c_double),
                ("qs", ctypes.c_double), ("qp", ctypes.c_double)]


class Medium(ctypes.Structure):
    _fields_ = [("layers", ctypes.POINTER(Layer)), ("count", ctypes.c_int32),
                ("_pad", ctypes.c_int32), ("ref_freq_hz", ctypes.c_double),
                ("default_q", ctypes.c_double), ("sls_tau_sigma", ctypes.c_double),
                ("sls_tau_eps", ctypes.c_double)]


class Integration(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int32), ("_pad", ctypes.c_int32),
                ("kmax_factor", ctypes.c_double), ("kmax", ctypes.c_double)]


class Grid(ctypes.Structure):
    _fields_ = [("kmax", ctypes.c_double), ("samples", ctypes.c_int32), ("_pad", ctypes.c_int32)]


class Solve(ctypes.Structure):
    _fields_ = [("formulation", ctypes.c_int32), ("quadrature", ctypes.c_int32),
                ("guard", ctypes.c_int32), ("_pad", ctypes.c_int32),
                ("omega_imag", ctypes.c_double)]


def build():
    """Compiles the oracle (make -C oracle); returns the library path."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None
_timed = None

# The timed CPU baseline's build: the same source optimised for the host it
# runs on. The parity build (Makefile) keeps -O2 -ffp-contract=off.
TIMED_CFLAGS = ["-O3", "-march=native", "-fPIC", "-std=gnu11", "-shared"]


def _bind(l):
    P = ctypes.POINTER
    d = ctypes.c_double
    l.or_surface_response.argtypes = [P(Medium), P(Solve), d, d, P(d)]
    l.or_static_coefficient.argtypes = [P(Medium), P(Solve), d, d, P(d)]
    l.or_grid_for.argtypes = [P(Medium), P(d), ctypes.c_int, d, Integration, P(Grid)]
    l.or_vertical_displacement_multi.argtypes = [P(Medium), P(Solve), P(d), ctypes.c_int, d,
                                                 Integration, P(d)]
    l.or_vertical_displacement.argtypes = [P(Medium), P(Solve), d, d, Integration, P(d)]
    l.or_bank_spectra.argtypes = [P(Medium), P(Solve), P(d), ctypes.c_int, P(d), ctypes.c_int,
                                  Integration, P(d), P(ctypes.c_int32), ctypes.c_int]
    l.or_check_layer_phase.argtypes = [P(Medium), d]
    l.or_validate.argtypes = [P(Medium)]
    l.or_j0.argtypes = [d]
    l.or_j0.restype = d
    return l


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = _bind(ctypes.CDLL(str(LIB_PATH)))
    return _lib


def timed_lib():
    """The oracle compiled with TIMED_CFLAGS for THIS host's CPU, into a
    private temporary directory (a -march=native library must not travel to
    another machine). Returns (library, flags string)."""
    global _timed
    if _timed is None:
        import shutil
        import tempfile
        out = pathlib.Path(tempfile.mkdtemp(prefix="gfk_oracle_timed_")) / "libgfk_oracle_timed.so"
        cc = os.environ.get("CC") or shutil.which("gcc") or "cc"
        subprocess.run([cc, *TIMED_CFLAGS, "-o", str(out), str(HERE / "gfk_oracle.c"), "-lm", "-lpthread"],
                       check=True)
        _timed = (_bind(ctypes.CDLL(str(out))), " ".join(TIMED_CFLAGS))
    return _timed


class OracleMedium:
    """A medium held in C memory for the oracle's calls."""

    def __init__(self, layers, ref_freq=0.0, default_q=0.0, sls=None):
        layers = [tuple(l) + (0.0,) * (6 - len(l)) for l in layers]
        self._arr = (Layer * max(1, len(layers)))(*[Layer(*l) for l in layers])
        self.c = Medium(self._arr if layers else None, len(layers), 0, ref_freq, default_q,
                        sls[0] if sls else 0.0, sls[1] if sls else 0.0)


def _solve(formulation, omega_imag=0.0, guard=0):
    return Solve(formulation, 0, guard, 0, omega_imag)


def _medium(m):
    return m if isinstance(m, OracleMedium) else OracleMedium(m)


def _integ(samples=0, kmax_factor=0.0, kmax=0.0):
    return Integration(int(samples), 0, float(kmax_factor), float(kmax))


def surface_response(medium, k, f, formulation=REFERENCE_DIRECT, omega_imag=0.0):
    m = _medium(medium)
    out = (ctypes.c_double * 2)()
    st = lib().or_surface_response(ctypes.byref(m.c), ctypes.byref(_solve(formulation, omega_imag)),
                                   k, f, out)
    if st:
        raise OracleError(st)
    return complex(out[0], out[1])


def static_coefficient(medium, f, k_far, formulation=REFERENCE_DIRECT, omega_imag=0.0):
    m = _medium(medium)
    out = (ctypes.c_double * 2)()
    st = lib().or_static_coefficient(ctypes.byref(m.c), ctypes.byref(_solve(formulation, omega_imag)),
                                     f, k_far, out)
    if st:
        raise OracleError(st)
    return complex(out[0], out[1])


def grid_for(medium, ranges, f, samples=0, kmax_factor=0.0, kmax=0.0):
    m = _medium(medium)
    r = np.ascontiguousarray(ranges, dtype=np.float64)
    g = Grid()
    st = lib().or_grid_for(ctypes.byref(m.c), r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r),
                           f, _integ(samples, kmax_factor, kmax), ctypes.byref(g))
    if st:
        raise OracleError(st)
    return g.kmax, g.samples


def vertical_displacement_multi(medium, ranges, f, samples=0, kmax_factor=0.0, kmax=0.0,
                                formulation=REFERENCE_DIRECT, omega_imag=0.0, guard=0):
    m = _medium(medium)
    r = np.ascontiguousarray(ranges, dtype=np.float64)
    out = np.zeros(2 * len(r))
    st = lib().or_vertical_displacement_multi(
        ctypes.byref(m.c), ctypes.byref(_solve(formulation, omega_imag, guard)),
        r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r), f, _integ(samples, kmax_factor, kmax),
        out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if st:
        raise OracleError(st)
    return out[0::2] + 1j * out[1::2]


def vertical_displacement(medium, r, f, samples=0, kmax_factor=0.0, kmax=0.0,
                          formulation=REFERENCE_DIRECT, omega_imag=0.0, guard=0):
    m = _medium(medium)
    out = (ctypes.c_double * 2)()
    st = lib().or_vertical_displacement(ctypes.byref(m.c), ctypes.byref(_solve(formulation, omega_imag, guard)),
                                        r, f, _integ(samples, kmax_factor, kmax), out)
    if st:
        raise OracleError(st)
    return complex(out[0], out[1])


def bank_spectra(medium, ranges, freqs, samples=0, kmax_factor=0.0, kmax=0.0, formulation=REFERENCE_DIRECT,
                 omega_imag=0.0, guard=0, threads=None, library=None):
    """[nf, nr] complex128 and per-frequency status, threaded over frequency.
    library: a library from timed_lib() in place of the parity build."""
    m = _medium(medium)
    r = np.ascontiguousarray(ranges, dtype=np.float64)
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    out = np.zeros((len(f), 2 * len(r)))
    status = np.zeros(len(f), dtype=np.int32)
    threads = threads or os.cpu_count() or 1
    P = ctypes.POINTER
    (library or lib()).or_bank_spectra(ctypes.byref(m.c), ctypes.byref(_solve(formulation, omega_imag, guard)),
                          r.ctypes.data_as(P(ctypes.c_double)), len(r),
                          f.ctypes.data_as(P(ctypes.c_double)), len(f), _integ(samples, kmax_factor, kmax),
                          out.ctypes.data_as(P(ctypes.c_double)), status.ctypes.data_as(P(ctypes.c_int32)),
                          threads)
    return out[:, 0::2] + 1j * out[:, 1::2], status


def check_layer_phase(medium, f):
    m = _medium(medium)
    return lib().or_check_layer_phase(ctypes.byref(m.c), f)


def validate(medium):
    m = _medium(medium)
    return lib().or_validate(ctypes.byref(m.c))


def j0(x):
    return lib().or_j0(x)

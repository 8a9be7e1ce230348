"""The C-ABI boundary without a GPU: libgfk loads, exports every symbol
include/gfk.h declares, its host-side rules match the reference's, and its
bank files are the reference's format byte for byte."""
import ctypes
import json
import math
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, as_tuples

import closed_forms as CF


def declared_symbols():
    text = (ROOT / "include" / "gfk.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gfk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(gfk):
    lib = gfk._native.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(gfk._native.EXPORTS) == names


def test_status_strings(gfk):
    lib = gfk._native.lib()
    for code in range(11):
        assert lib.gfk_status_string(code)
    assert lib.gfk_status_string(99) == b"unknown status"


def test_propagator_launch_shapes(gfk):
    """gfk_prop_shape describes every tuned launch shape (host table, no GPU);
    the persistent ones are among them and unknown indices are refused."""
    shapes = []
    v = 0
    while True:
        try:
            shapes.append(gfk.prop_shape(v))
        except gfk.FkError as e:
            assert e.status == gfk._native.EARG
            break
        v += 1
    assert len(shapes) >= 10
    assert any(s["persistent"] for s in shapes) and any(not s["persistent"] for s in shapes)
    for s in shapes:
        assert s["threads"] % 32 == 0 and s["blocks_per_sm"] >= 1
        assert s["wavenumbers_per_thread"] in (1, 2) and s["runs_per_item"] >= 1
    with pytest.raises(gfk.FkError):
        gfk.prop_shape(-1)


def test_grid_for_matches_oracle(gfk, oracle):
    m = gfk.Medium(gfk.uniform(*CF.LOAM))
    for ranges, f in (([16.0], 60.0), ([1.0, 50.0], 20.0), ([2, 5, 10, 20], 0.5), (list(range(1, 65)), 300.0)):
        g = m.grid_for(ranges, f)
        kmax, n = oracle.grid_for(CF.uniform(CF.LOAM), ranges, f)
        assert (g.kmax, g.samples) == (kmax, n)
    g = m.grid_for([16.0], 60.0)
    assert g.samples == 6000  # docs/validation-report.md:60
    g = m.grid_for([1.0], 60.0, gfk.Integration(10))
    assert g.samples == 64  # the floor of fk.go:491-493
    with pytest.raises(gfk.FkError) as e:
        m.grid_for([], 20.0)
    assert e.value.status == gfk._native.EARG and "no ranges" in str(e.value)
    with pytest.raises(gfk.FkError):
        m.grid_for([0.0], 20.0)


def test_layer_phase_guard(gfk):
    """fk.go:251-266 and its logged band (docs/validation-report.md:155-157)."""
    for thick, band in ((1.0, 443), (2.0, 222), (4.0, 111)):
        st = gfk.Stack([gfk.Layer(thick, 500, 200, 1700, 25), gfk.Layer(0, 500, 200, 1700, 25)])
        m = gfk.Medium(st)
        m.check_layer_phase(band - 1)
        with pytest.raises(gfk.FkError) as e:
            m.check_layer_phase(band + 1)
        assert e.value.status == gfk._native.EGUARD
        assert f"Band-limit to {band} Hz" in str(e.value)
    gfk.Medium(gfk.uniform(*CF.LOAM)).check_layer_phase(1e5)  # no layers, no guard


def test_stack_validation(gfk):
    ok = gfk.Stack([gfk.Layer(1, 500, 200, 1700), gfk.Layer(0, 800, 400, 2000)])
    ok.validate()
    bad = [
        gfk.Stack([]),
        gfk.Stack([gfk.Layer(0, 100, 200, 1700)]),            # Vp <= sqrt2 Vs
        gfk.Stack([gfk.Layer(0, 500, -1, 1700)]),
        gfk.Stack([gfk.Layer(0, 500, 200, 0)]),
        gfk.Stack([gfk.Layer(0, 500, 200, 1700), gfk.Layer(0, 500, 200, 1700)]),  # zero thickness
        gfk.Stack([gfk.Layer(1, float("nan"), 200, 1700), gfk.Layer(0, 500, 200, 1700)]),
    ]
    for st in bad:
        with pytest.raises(gfk.FkError) as e:
            st.validate()
        assert e.value.status == gfk._native.ESTACK


def test_reads_reference_conformance_fixtures(gfk):
    """conformance_test.go:28-81: both languages' fixtures read to 1e-6."""
    conf = json.loads((GOLDEN / "conformance.json").read_text())
    want = np.array(conf["pattern"])
    want = (want[..., 0] + 1j * want[..., 1]).astype(np.complex64)
    for name in ("python_written.bank", "go_written.bank"):
        b = gfk.open_bank(GOLDEN / name)
        assert b.header.ranges.count == conf["count"] and b.header.samples == conf["samples"]
        got = b.complex()
        rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-30)
        assert rel.max() <= conf["tolerance"]


def test_writes_the_go_fixture_byte_for_byte(gfk, tmp_path):
    """The header JSON, padding and payload match what the reference's Go
    writer produced (cmd/geobank/main.go:236-267, format.go:215-240)."""
    conf = json.loads((GOLDEN / "conformance.json").read_text())
    h = gfk.Header(gfk.Provenance("go conformance fixture"), gfk.Stack([gfk.Layer(0, 500, 200, 1700)]),
                   conf["rate"], conf["samples"], gfk.RangeGrid(1, 4, conf["count"]),
                   "conformance fixture, not physical", "m/N")
    b = gfk.Bank.new(h)
    for i in range(conf["count"]):
        for k in range(h.bins()):
            b.set(i, k, complex((i + 1) * 10.0 ** (k % 5 - 2), -(k + 1) * 0.25 + i))
    out = tmp_path / "ours.bank"
    b.write(out)
    assert out.read_bytes() == (GOLDEN / "go_written.bank").read_bytes()


def test_bank_pack_layout(gfk):
    """Range-major float32 pairs, bins outside the computed band left zero."""
    nf, nr, bins = 5, 3, 9
    spectra = (np.arange(nf * nr) + 1j * (100 + np.arange(nf * nr))).reshape(nf, nr)
    sp = np.ascontiguousarray(np.stack([spectra.real, spectra.imag], -1))
    payload = np.zeros(2 * nr * bins, dtype=np.float32)
    st = gfk._native.lib().gfk_bank_pack(sp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nf, nr, 1, bins,
                                        payload.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert st == 0
    p = payload.reshape(nr, bins, 2)
    assert (p[:, 0] == 0).all() and (p[:, nf + 1:] == 0).all()
    for f in range(nf):
        for j in range(nr):
            assert p[j, f + 1, 0] == np.float32(spectra[f, j].real)
            assert p[j, f + 1, 1] == np.float32(spectra[f, j].imag)


def test_header_validation_and_range_sampling(gfk):
    h = gfk.Header(gfk.Provenance("x"), gfk.uniform(*CF.LOAM), 2000, 4096, gfk.RangeGrid(1, 40, 270), "c", "m/N")
    h.validate()
    h.check_range_sampling(300)  # geobank's defaults (cmd/geobank/main.go:56-63)
    with pytest.raises(gfk.FkError):
        gfk.RangeGrid(1, 40, 20) and gfk.Header(gfk.Provenance("x"), gfk.uniform(*CF.LOAM), 2000, 4096,
                                                 gfk.RangeGrid(1, 40, 20), "c", "m/N").check_range_sampling(300)
    for bad in (dict(samples=31), dict(sample_rate_hz=0), dict(component="")):
        kw = dict(provenance=gfk.Provenance("x"), medium=gfk.uniform(*CF.LOAM), sample_rate_hz=2000, samples=32,
                  ranges=gfk.RangeGrid(1, 4, 7), component="c", units="m/N")
        kw.update(bad)
        with pytest.raises(gfk.FkError):
            gfk.Header(**kw).validate()


def test_engine_without_gpu_fails_loudly(gfk):
    """No CUDA device here: opening a context raises rather than falling back."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(gfk.FkError) as e:
        gfk.Engine(0)
    assert "no CPU fallback" in str(e.value)

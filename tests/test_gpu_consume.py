"""GPU bank consumption (gfk_bank_tables, gfk_bank_impulse_responses) against
the oracle's restatement of Bank.prepare / Bank.Response /
CausalImpulseResponseAt, on the reference's conformance banks and on a
solver-built bank."""
import math
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import bank_oracle as BO  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    return g.load_package()


@pytest.fixture(scope="module")
def eng(pkg):
    e = pkg.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def solved_bank(pkg, eng):
    """A 48-range, 1024-sample bank of the single-soil workload from the GPU solver."""
    wl = pkg.workloads.single_soil()
    stack = wl.stack if hasattr(wl, "stack") else wl.medium.stack
    h = pkg.Header(pkg.Provenance("gfk-b200 dunkin", "test"), stack, 1000.0, 1024,
                   pkg.RangeGrid(1.0, 12.75, 48), "vertical", "m/N")
    med = pkg.Medium(stack, formulation=pkg.DUNKIN, engine=eng)
    b, _ = pkg.build_bank(med, h, 200.0, pkg.Integration(4096, 0.0, 52.36), check_range_sampling=False)
    return b


def golden(pkg, name):
    return pkg.open_bank(ROOT / "tests" / "golden" / name)


@pytest.mark.parametrize("name", ["python_written.bank", "go_written.bank", None])
def test_tables_match_oracle(pkg, eng, solved_bank, name):
    b = golden(pkg, name) if name else solved_bank
    lm, ph = b.tables(eng)
    wl, wp = BO.prepare(b.data)
    assert np.array_equal(lm == BO.NEG_INF, wl == BO.NEG_INF)
    ok = wl != BO.NEG_INF
    assert np.allclose(lm[ok], wl[ok], rtol=1e-14, atol=1e-14)
    assert np.allclose(ph, wp, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("velocity", [True, False])
def test_impulse_responses_match_oracle(pkg, eng, solved_bank, velocity):
    b = solved_bank
    h = b.header
    rng = np.random.default_rng(3)
    ranges = np.concatenate([[h.ranges.min_m, h.ranges.max_m], rng.uniform(h.ranges.min_m, h.ranges.max_m, 6)])
    f = np.arange(h.bins()) * h.sample_rate_hz / h.samples
    sensor = 28.8 * (2j * np.pi * f) ** 2 / ((2j * np.pi * f) ** 2 + 2 * 0.7 * 62.83 * 2j * np.pi * f + 62.83 ** 2)
    got = b.impulse_responses(ranges, 300, sensor=sensor, velocity=velocity, engine=eng)
    want = BO.impulse_responses(b.data, (h.ranges.min_m, h.ranges.max_m), h.sample_rate_hz, h.samples, ranges,
                                300, sensor=sensor, velocity=velocity)
    scale = np.abs(want).max(axis=1, keepdims=True)
    assert np.abs(got - want).max() <= 1e-12 * scale.max()
    assert (np.abs(got - want) <= 1e-11 * scale).all()


def test_consume_errors(pkg, eng, solved_bank):
    b = solved_bank
    with pytest.raises(pkg.FkError) as e:
        b.impulse_responses([20.0], 100, engine=eng)
    assert e.value.status == pkg._native.EARG and "outside the bank" in str(e.value)
    with pytest.raises(pkg.FkError) as e:
        b.impulse_responses([2.0], 2000, engine=eng)
    assert e.value.status == pkg._native.EARG


def test_device_bank_matches_one_shot_calls(pkg, eng, solved_bank):
    """A bank kept on the device answers repeated queries exactly as the
    one-shot call does (same tables, same kernel), into host memory and into
    device memory, and reports the one-shot call's errors."""
    import torch
    b = solved_bank
    h = b.header
    rng = np.random.default_rng(9)
    f = np.arange(h.bins()) * h.sample_rate_hz / h.samples
    sensor = 28.8 * (2j * np.pi * f) ** 2 / ((2j * np.pi * f) ** 2 + 2 * 0.7 * 62.83 * 2j * np.pi * f + 62.83 ** 2)
    with b.device(eng) as db:
        for n in (5, 37):  # the second call grows the query scratch
            ranges = rng.uniform(h.ranges.min_m, h.ranges.max_m, n)
            want = b.impulse_responses(ranges, 300, sensor=sensor, engine=eng)
            got = db.impulse_responses(ranges, 300, sensor=sensor)
            assert np.array_equal(got, want)
            dev = torch.empty((n, 300), dtype=torch.float64, device="cuda:0")
            assert db.impulse_responses(ranges, 300, sensor=sensor, out_device_ptr=dev.data_ptr()) is None
            assert np.array_equal(dev.cpu().numpy(), want)
        plain = db.impulse_responses([2.0, 9.5], 200, velocity=False)
        assert np.array_equal(plain, b.impulse_responses([2.0, 9.5], 200, velocity=False, engine=eng))
        with pytest.raises(pkg.FkError) as e:
            db.impulse_responses([20.0], 100)
        assert e.value.status == pkg._native.EARG and "outside the bank" in str(e.value)
        with pytest.raises(pkg.FkError) as e:
            db.impulse_responses([2.0], 2000)
        assert e.value.status == pkg._native.EARG

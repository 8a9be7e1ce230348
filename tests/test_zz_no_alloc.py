"""The allocation-free entry point against the allocating one.

gfk_vertical_displacement_multi_noalloc exists for callers that cannot
allocate device memory when they need a response (their device memory is
already claimed by another framework's caching allocator, or they run on a
deadline where cudaMalloc/cudaFree may synchronise the device). Its working
memory is a fixed array inside libgfk, shared by every call, so this file
checks that two calls in a row — the second reusing what the first left in
the array — both agree with gfk_vertical_displacement_multi within the 1e-9
tolerance the other FP64 GPU parity tests use. Collected last, so a failure
here cannot hide the result of any other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_noalloc(gfk, medium, ranges, freq, opt):
    N = gfk._native
    from gfk_b200.fk import _c_medium
    r = np.ascontiguousarray(ranges, dtype=np.float64)
    out = np.zeros(2 * len(r))
    with _c_medium(medium) as cm:
        st = N.lib().gfk_vertical_displacement_multi_noalloc(
            ctypes.byref(cm), ctypes.byref(medium._solve()), r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            len(r), float(freq), opt.c(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    return st, out[0::2] + 1j * out[1::2]


def test_noalloc_matches_allocating_entry_point_twice():
    import __graft_entry__
    gfk = __graft_entry__.load_package()
    eng = gfk.Engine(0)
    try:
        wl = gfk.workloads.single_soil()
        # a Dunkin medium on the workload's shared grid, and the reference
        # formulation on GridFor's own grid, at different sizes so the second
        # call overwrites only part of what the first left in the array
        cases = [
            (wl.medium(gfk.DUNKIN, engine=eng), wl.ranges, 250.0, wl.integration()),
            (gfk.Medium(gfk.Stack([gfk.Layer(3.0, 400, 160, 1600), gfk.Layer(0, 900, 400, 2000)]), engine=eng),
             np.array([2.0, 5.0, 10.0, 20.0]), 40.0, gfk.Integration()),
        ]
        for medium, ranges, freq, opt in cases:
            want = medium.vertical_displacement_multi(ranges, freq, opt)
            for _ in range(2):
                st, got = _call_noalloc(gfk, medium, ranges, freq, opt)
                assert st == 0, gfk._native.status_string(st)
                assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-9
        # requests beyond the compiled-in limits are refused before any device work
        N = gfk._native
        too_many = np.linspace(1.0, 2.0, 16385)
        st, _ = _call_noalloc(gfk, wl.medium(gfk.DUNKIN, engine=eng), too_many, 100.0, wl.integration())
        assert st == N.ELIMIT
        st, _ = _call_noalloc(gfk, wl.medium(gfk.DUNKIN, engine=eng), wl.ranges, 100.0,
                              gfk.Integration(196609, 0.0, wl.kmax))
        assert st == N.ELIMIT
        # and the guard still refuses what the reference refuses
        st, _ = _call_noalloc(gfk, cases[1][0], cases[1][1], 300.0, gfk.Integration())
        assert st == N.EGUARD
        # a call that fails on the device (a density of 1e305 kg/m^3 passes
        # the stack's validation, but rho Vs^2 overflows, so every layer
        # constant and the response are non-finite) returns the allocating
        # call's status and leaves zeros in out, not NaNs
        heavy = gfk.Medium(gfk.Stack([gfk.Layer(3.0, 400, 160, 1e305), gfk.Layer(0, 900, 400, 1e305)]),
                           formulation=gfk.DUNKIN, engine=eng)
        ranges = np.array([2.0, 5.0])
        opt = gfk.Integration(256, 0.0, 20.0)
        with pytest.raises(gfk.FkError) as e:
            heavy.vertical_displacement_multi(ranges, 40.0, opt)
        st, got = _call_noalloc(gfk, heavy, ranges, 40.0, opt)
        assert st == e.value.status == N.ENONFINITE
        assert np.array_equal(got, np.zeros(2, dtype=complex))
        # and the next call in the same array is unaffected
        st, got = _call_noalloc(gfk, *cases[0])
        assert st == 0
        want = cases[0][0].vertical_displacement_multi(*cases[0][1:])
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-9
    finally:
        eng.close()

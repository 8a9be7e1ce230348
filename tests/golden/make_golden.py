"""Generates the committed golden fixtures under tests/golden/.

Run where a checkout of the reference project is available (it is only
read), with GFK_REFERENCE naming its root directory:

    GFK_REFERENCE=<reference checkout> python tests/golden/make_golden.py

Writes:
  python_written.bank   the reference's own Python writer (py/bankfmt/bankfmt.py
                        write, py/bankfmt/conformance.py make) run on its
                        conformance payload
  go_written.bank       the reference's Go-written conformance fixture
                        (testdata/bank/go_written.bank), copied byte for byte
  conformance.json      the pattern values (conformance.py:27-29) those files hold
  known_answers.json    the numbers the reference's own test run logged
                        (docs/validation-report.md), with their source lines
  surface_response_mp.json
                        u_z(k, f) of the reference algorithm evaluated at
                        40-3000 digits (oracle/mp_direct.py) for a grid of
                        media, wavenumbers and frequencies, both Qp conventions
                        and with a complex frequency offset
  dispersion/*.json     the reference's disba dispersion goldens
                        (testdata/dispersion/*.json: disba 0.7.0
                        PhaseDispersion, Rayleigh), copied byte for byte
"""
import hashlib
import json
import math
import os
import pathlib
import re
import shutil
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if not os.environ.get("GFK_REFERENCE"):
    sys.exit("make_golden.py: set GFK_REFERENCE to the reference checkout's root directory")
REF = pathlib.Path(os.environ["GFK_REFERENCE"])


def bank_fixtures():
    sys.path.insert(0, str(REF / "py" / "bankfmt"))
    import bankfmt  # the reference's module
    import conformance
    b = conformance.make()
    bankfmt.write(str(HERE / "python_written.bank"), b)
    shutil.copyfile(REF / "testdata" / "bank" / "go_written.bank", HERE / "go_written.bank")
    vals = [[[conformance.pattern(i, k).real, conformance.pattern(i, k).imag]
             for k in range(conformance.SAMPLES // 2 + 1)] for i in range(conformance.COUNT)]
    out = {"count": conformance.COUNT, "samples": conformance.SAMPLES, "rate": conformance.RATE,
           "pattern": vals, "tolerance": 1e-6,
           "sha256": {n: hashlib.sha256((HERE / n).read_bytes()).hexdigest()
                      for n in ("python_written.bank", "go_written.bank")},
           "source": "py/bankfmt/conformance.py:27-65, testdata/bank/go_written.bank"}
    (HERE / "conformance.json").write_text(json.dumps(out, indent=1))


def known_answers():
    rep = (REF / "docs" / "validation-report.md").read_text().splitlines()
    ka = {"source": "docs/validation-report.md"}

    def grab(pattern):
        rows = []
        for n, line in enumerate(rep, 1):
            m = re.search(pattern, line)
            if m:
                rows.append((n, m.groups()))
        return rows

    ka["integrand_at_zero_k"] = [
        {"line": n, "k": float(g[0]), "integrand_abs": float(g[1]), "minus_C_abs": float(g[2]), "apart": float(g[3])}
        for n, g in grab(r"k=([0-9.e+-]+): integrand ([0-9.e+-]+), -C ([0-9.e+-]+), apart by ([0-9.e+-]+)")]
    ka["quadrature_order"] = [
        {"line": n, "n": int(g[0]), "rel": float(g[1])}
        for n, g in grab(r"n=\s*(\d+): relative error ([0-9.e+-]+)")]
    ka["far_field_phase"] = [
        {"line": n, "wavelengths": float(g[0]), "range_m": float(g[1]), "abs_ratio": float(g[2]),
         "phase_deg": float(g[3]), "gap": float(g[4])}
        for n, g in grab(r"([0-9.]+) wavelengths \(([0-9.]+) m\): \|ratio\| ([0-9.]+), phase ([+-][0-9.]+) deg, "
                         r"complex gap ([0-9.]+)")]
    ka["guard_band"] = [
        {"line": n, "thickness_m": float(g[0]), "usable_hz": float(g[1])}
        for n, g in grab(r"a ([0-9.]+) m layer is usable to ([0-9.]+) Hz")]
    ka["split_layer"] = [
        {"line": n, "freq_hz": float(g[0]), "rel": float(g[1])}
        for n, g in grab(r"(\d+) Hz \(k\*h ~\s*[0-9.]+\): identical layers differ from the half-space by ([0-9.e+-]+)")]
    ka["fastest_velocity"] = [
        {"line": n, "mps": float(g[0])} for n, g in grab(r"fastest velocity in the band: ([0-9.]+) m/s")]
    ka["causality_precursor"] = [
        {"line": n, "range_m": float(g[0]), "early": float(g[1]), "negative_time": float(g[2])}
        for n, g in grab(r"r=\s*(\d+) m: peak at [0-9.]+ s, nothing may arrive before [0-9.]+ s; largest sample "
                         r"before it ([0-9.e+-]+) of peak, largest at negative time ([0-9.e+-]+)")]
    (HERE / "known_answers.json").write_text(json.dumps(ka, indent=1))


def mp_surface_responses():
    sys.path.insert(0, str(ROOT / "oracle"))
    import mp_direct
    media = {
        "loam": [(0.0, 500.0, 200.0, 1700.0, 25.0, 0.0)],
        "single_soil": [(0.5, 300.0, 150.0, 1700.0, 15.0, 30.0), (2.0, 500.0, 250.0, 1800.0, 25.0, 50.0),
                        (0.0, 800.0, 400.0, 2000.0, 40.0, 80.0)],
        "soft_over_stiff": [(3.0, 400.0, 160.0, 1600.0, 30.0, 0.0), (0.0, 900.0, 400.0, 2000.0, 30.0, 0.0)],
        "split_loam": [(2.0, 500.0, 200.0, 1700.0, 25.0, 0.0), (2.0, 500.0, 200.0, 1700.0, 25.0, 0.0),
                       (0.0, 500.0, 200.0, 1700.0, 25.0, 0.0)],
        "near_lossless": [(0.5, 400.0, 160.0, 1600.0, 1e9, 0.0), (0.0, 2200.0, 1100.0, 2400.0, 1e9, 0.0)],
    }
    cases = []
    for name, st in media.items():
        for f in (0.977, 10.0, 60.0, 166.0, 400.0):
            for k in (0.0128, 0.4, 2.0, 9.0, 40.0, 200.0):
                for qp_mode, wi in (("reference", 0.0), ("layer", math.pi / 1.024)):
                    tot = sum(k * l[0] for l in st[:-1])
                    if 40 + 2 * tot / 2.3 > 1500:
                        continue
                    u = mp_direct.surface_response(st, k, f, wi, qp_mode)
                    cases.append({"medium": name, "k": k, "f": f, "omega_imag": wi, "qp_mode": qp_mode,
                                  "kh": tot, "u": [u.real, u.imag]})
    out = {"media": media, "cases": cases,
           "source": "internal/fk/fk.go:119-327 evaluated in mpmath (oracle/mp_direct.py)"}
    (HERE / "surface_response_mp.json").write_text(json.dumps(out, indent=1))


def dispersion_fixtures():
    out = HERE / "dispersion"
    out.mkdir(exist_ok=True)
    for src in sorted((REF / "testdata" / "dispersion").glob("*.json")):
        shutil.copyfile(src, out / src.name)


if __name__ == "__main__":
    dispersion_fixtures()
    bank_fixtures()
    known_answers()
    mp_surface_responses()
    print("golden fixtures written to", HERE)

"""Compressed ephemeris records: the library's decoder against the reference's own interpolator.

The fixtures (tests/golden/ephemeris/*.npz, recorded by tests/golden/make_ephemeris_golden.py) hold
records written by the reference's compressor (`ephemeris_compressor::compress_orbital_data` and
`compress_rotational_data`, src/modules/ephemeris_compressor.cpp:164-530) and the reference interpolator's states at 59 times per
record (ephemeris_compressor.cpp:1017-1053), both on the B-spline form as loaded and after expand(). They
cover the four orbital formats (state vectors, Keplerian vectors, circular and raw Keplerian elements) and
the three rotational ones (axial offset, quaternion, tidal lock; the tidally locked record is evaluated
against the orbital state the reference interpolator was given, kept in the fixture).

The decoder evaluates the spline and the element-to-state conversion its own way, so the bound is the
reference's own rounding spread: the larger of 1e-14 and 1.5x the difference between the reference's two
evaluation forms, relative to the record's largest |r| (|v|, |w|; the frame axes are unit vectors).
GM is compared exactly.
CPU-only: the decoder is host code of libeph_b200.so.
"""
import glob
import os

import numpy as np
import pytest

from ephemeris_b200.ephemeris_record import EphemerisInterpolator
from ephemeris_b200 import EphError, bspline_fit

HERE = os.path.dirname(os.path.abspath(__file__))
ALL = sorted(glob.glob(os.path.join(HERE, "golden", "ephemeris", "*.npz")))
FIXTURES = [f for f in ALL if int(np.load(f)["format"]) <= 4]
ROTATIONAL = [f for f in ALL if int(np.load(f)["format"]) >= 5]
EPH_ERR_ARG, EPH_ERR_LOAD, EPH_ERR_UNSUPPORTED = 1, 6, 7


def _load(path):
    z = np.load(path)
    return z, EphemerisInterpolator(z["blob"].tobytes(), float(z["span"]))


def test_fixtures_cover_every_format():
    formats = {int(np.load(f)["format"]) for f in ALL}
    assert formats == {1, 2, 3, 4, 5, 6, 7}, formats


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def test_record_matches_reference_interpolator(path):
    z, ip = _load(path)
    assert ip.format == int(z["format"])
    assert 0 <= ip.relative_error < 1
    got = ip.states(z["times"])
    ref_a, ref_b = z["loaded"], z["expanded"]
    rs = np.linalg.norm(ref_a[:, :3], axis=1).max()
    vs = np.linalg.norm(ref_a[:, 3:6], axis=1).max()
    spread_r = np.abs(ref_a[:, :3] - ref_b[:, :3]).max() / rs
    spread_v = np.abs(ref_a[:, 3:6] - ref_b[:, 3:6]).max() / vs
    tol_r, tol_v = max(1e-14, 1.5 * spread_r), max(1e-14, 1.5 * spread_v)
    for ref in (ref_a, ref_b):
        assert np.abs(got[:, :3] - ref[:, :3]).max() / rs <= tol_r
        assert np.abs(got[:, 3:] - ref[:, 3:6]).max() / vs <= tol_v
    gm_ref = ref_a[:, 6]
    for k, t in enumerate(z["times"][:5]):
        _, _, gm = ip(t)
        assert gm == gm_ref[k] or (ip.format == 1 and gm == 0 and gm_ref[k] == 0)
    ip.close()


def test_times_outside_the_record_are_rejected():
    z, ip = _load(FIXTURES[0])
    with pytest.raises(EphError) as e:
        ip(float(z["span"]) * 1.001)
    assert e.value.code == EPH_ERR_ARG
    with pytest.raises(EphError):
        ip(-1.0)
    t = np.array([0.0, -1.0, float(z["span"])])
    out = np.empty((3, 6))
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)
    assert ip.lib.eph_ephem_states(ip.h, 3, t.ctypes.data_as(D), out.ctypes.data_as(D)) == EPH_ERR_ARG
    assert np.isnan(out[1]).all() and np.isfinite(out[[0, 2]]).all()   # the other times are still evaluated
    assert np.array_equal(out[0], np.concatenate(ip(0.0)[:2]))


def _patched(blob, offset, dtype, value):
    b = bytearray(blob)
    b[offset:offset + np.dtype(dtype).itemsize] = np.array([value], dtype).tobytes()
    return bytes(b)


def test_invalid_records_are_rejected():
    z = np.load(FIXTURES[0])
    blob, span = z["blob"].tobytes(), float(z["span"])
    cases = [
        (blob[:-8], EPH_ERR_LOAD),                               # size does not match n + degree coefficients
        (_patched(blob, 0, np.float32, 1.0), EPH_ERR_LOAD),       # relative error not below 1
        (_patched(blob, 0, np.float32, np.nan), EPH_ERR_LOAD),
        (_patched(blob, 6, np.uint16, 0xFFFF), EPH_ERR_LOAD),     # format 0 (uncompressed)
        (_patched(blob, 6, np.uint16, 0xFFFF ^ 6), EPH_ERR_LOAD),   # quaternion format, wrong size for it
        (_patched(blob, 6, np.uint16, 0xFFFF ^ 8), EPH_ERR_LOAD),   # beyond the last format
        (_patched(blob, 4, np.int16, 0), EPH_ERR_LOAD),           # degree 0
        (_patched(blob, 8, np.int64, 0), EPH_ERR_LOAD),           # no segments
        (_patched(blob, 8, np.int64, 2 ** 63 - 1), EPH_ERR_LOAD),  # a segment count beyond any record size
        (blob[:16], EPH_ERR_ARG),                                 # shorter than the common header
    ]
    for rec, want in cases:
        with pytest.raises(EphError) as e:
            EphemerisInterpolator(rec, span)
        assert e.value.code == want, (want, e.value.code)
    with pytest.raises(EphError) as e:
        EphemerisInterpolator(blob, 0.0)
    assert e.value.code == EPH_ERR_ARG


@pytest.mark.parametrize("path", ROTATIONAL, ids=[os.path.basename(f)[:-4] for f in ROTATIONAL])
def test_rotational_record_matches_reference_interpolator(path):
    z, ip = _load(path)
    assert ip.format == int(z["format"]) and ip.is_rotational()
    ref_a, ref_b = z["loaded"], z["expanded"]
    got = np.zeros((len(z["times"]), 9))
    if ip.format == 7:
        with pytest.raises(EphError) as e:
            ip.rotation(0.0)                      # no orbital state given yet
        assert e.value.code == 5                  # EPH_ERR_STATE
    for k, t in enumerate(z["times"]):
        ip.set_orbital_state(ref_a[k, 9:12], ref_a[k, 12:15])   # the reference's orbital state at t
        got[k] = np.concatenate(ip.rotation(t))
    ws = np.linalg.norm(ref_a[:, :3], axis=1).max()
    spread_w = np.abs(ref_a[:, :3] - ref_b[:, :3]).max() / ws
    spread_f = np.abs(ref_a[:, 3:9] - ref_b[:, 3:9]).max()
    for ref in (ref_a, ref_b):
        assert np.abs(got[:, :3] - ref[:, :3]).max() / ws <= max(1e-14, 1.5 * spread_w)
        assert np.abs(got[:, 3:9] - ref[:, 3:9]).max() <= max(1e-14, 1.5 * spread_f)
    with pytest.raises(EphError) as e:
        ip(0.0)                                   # a rotational record has no orbital state
    assert e.value.code == EPH_ERR_UNSUPPORTED
    ip.close()


def test_orbital_record_has_no_rotation():
    _, ip = _load(FIXTURES[0])
    with pytest.raises(EphError) as e:
        ip.rotation(0.0)
    assert e.value.code == EPH_ERR_UNSUPPORTED


def _bspline_eval(coefs, d, n, x):
    """Value of sum_i coefs[i] B[d, x - i] at positions x in [0, n] (the basis recursion)."""
    out = np.zeros((len(x), coefs.shape[1]))
    for q, xv in enumerate(x):
        seg = min(int(np.floor(xv)), n - 1)
        u = xv - seg
        prev = [1.0]
        for e in range(1, d + 1):
            cur = []
            for k in range(e + 1):
                left = prev[k - 1] if k >= 1 else 0.0
                right = prev[k] if k <= e - 1 else 0.0
                cur.append(((u - k + e) * left + (1 - u + k) * right) / e)
            prev = cur
        out[q] = sum(prev[k] * coefs[seg + k] for k in range(d + 1))
    return out


def test_record_resampled_into_device_bspline_table():
    path = [f for f in FIXTURES if os.path.basename(f).startswith("moon_circular")][0]
    z, ip = _load(path)
    span = float(z["span"])
    d, n, mn = 3, 216, 864
    coefs = ip.to_bspline(d, n, mn)
    samples = ip.states(span * np.arange(mn + 1) / mn)[:, :3]
    samples[-1] = ip(span)[0]
    assert np.array_equal(coefs, bspline_fit(samples, n, d))   # the same fit of the same samples
    x = np.sort(np.random.default_rng(5).uniform(0, n, 40))
    fit = _bspline_eval(coefs, d, n, x)
    exact = ip.states(x / n * span)[:, :3]
    err = np.linalg.norm(fit - exact, axis=1).max() / np.linalg.norm(exact, axis=1).max()
    assert err < 1e-7, err


def test_fixtures_are_what_the_reference_compressor_writes(tmp_path):
    """Re-record the fixtures through the reference's own compressor (oracle/_ref/ephc, built from the
    reference sources where they are present) and compare the records byte for byte and the reference
    interpolator's values exactly."""
    import subprocess
    import sys
    ephc = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ephc")
    if not os.path.exists(ephc):
        pytest.skip("oracle/_ref/ephc is not built (the reference sources are not present)")
    env = dict(os.environ, EPH_GOLDEN_EPHEMERIS_DIR=str(tmp_path))
    subprocess.run([sys.executable, os.path.join(HERE, "golden", "make_ephemeris_golden.py")], check=True, env=env,
                   capture_output=True)
    for f in ALL:
        a, b = np.load(f), np.load(os.path.join(str(tmp_path), os.path.basename(f)))
        assert np.array_equal(a["blob"], b["blob"]), f
        for key in ("times", "loaded", "expanded"):
            assert np.array_equal(a[key], b[key]), (f, key)

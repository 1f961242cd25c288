"""GPU parity of the colour-matrix functions (exp, sqrt, inverse, det) on
config-5-shaped inputs, through the C-ABI.

  det, inverse : bit-identical to the reference's closed forms (F3 and D3);
  sqrt         : the reference's Newton iteration in the site precision --
                 bit-identical to QLA_F3 and QLA_D3; F3 within
                 1e-5 * max(1, |A|_F) of the FP64 result of the same input;
  exp          : Cayley-Hamilton/Taylor in FP64, compared with the reference
                 algorithm evaluated in FP64 (QLA_D3, bit-pinned oracle):
                 D3 |diff| <= 1e-13 * max(1, |A|_F^2) elementwise for the
                 config-5 anti-Hermitian inputs; general matrices
                 <= 1e-12 * max(1, |A|_F^2) * max(1, max|exp A|);
                 F3 within the reference test rule (16 eps abs or 10 eps rel,
                 FLT_EPSILON) of the FP64 value; and within 2e-5 * max(1,|A|_F)
                 of the reference's own FP32 result (its Pade error).
Near-degenerate spectra (10% of sites, gap < 1e-6) are included.
"""
import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu


def _run(qla, pc, fname, a, n, var="v", gang=None, ptr_idx=None):
    ns_ = getattr(qla, pc)
    nout = 1 if fname == "det" else 9
    r_d = T.to_dev(np.zeros((n, 2 * nout), dtype=a.dtype))
    a_d = T.to_dev(a)
    src = "M"
    arg = a_d
    if ptr_idx is not None:
        src = "pM"
        arg = T.ptr_array(a_d, ptr_idx, (8 if a.dtype == np.float32 else 16) * 9)
    extra = [T.to_dev(gang)] if var == "x" else []
    dest = "C" if fname == "det" else "M"
    getattr(ns_, f"{dest}_{var}eq_{fname}_{src}")(r_d, arg, *extra, n)
    return T.to_host(r_d)


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_det_inverse_bit_exact(qla, pc, dt):
    rng = np.random.default_rng(21)
    n = 20011
    a = T.positive_hermitian_inputs(rng, n, dt) + T.gaussian_field(rng, n, 9, dt)
    a = a.astype(dt)
    for fname in ("det", "inverse"):
        assert T.bits_equal(_run(qla, pc, fname, a, n), T.ora_mfunc(a, n, fname)), fname
        # pointer and gang-index variants
        idx = rng.permutation(n).astype(np.int32)
        want = T.ora_mfunc(a[idx], n, fname)
        assert T.bits_equal(_run(qla, pc, fname, a, n, ptr_idx=idx), want), fname + " pM"
        gang = rng.permutation(n).astype(np.int32)
        got = _run(qla, pc, fname, a, n, var="x", gang=gang)
        want = T.ora_mfunc(a, n, fname)
        assert T.bits_equal(got[gang], want[gang]), fname + " xeq"


def test_sqrt_bit_exact_newton(qla):
    rng = np.random.default_rng(22)
    n = 50021
    ad = T.positive_hermitian_inputs(rng, n, np.float64)
    assert T.bits_equal(_run(qla, "D3", "sqrt", ad, n), T.ora_mfunc(ad, n, "sqrt"))
    af = ad.astype(np.float32)
    got = _run(qla, "F3", "sqrt", af, n)
    assert T.bits_equal(got, T.ora_mfunc(af, n, "sqrt"))   # the reference's FP32 iteration
    scale = np.maximum(1.0, np.sqrt(np.sum(af.astype(np.float64) ** 2, axis=1)))[:, None]
    assert (np.abs(got - T.ora_mfunc(af.astype(np.float64), n, "sqrt")) / scale).max() <= 1e-5
    # and the result squares back to the input
    s = T.to_complex(_run(qla, "D3", "sqrt", ad, n))
    assert np.max(np.abs(s @ s - T.to_complex(ad))) < 1e-12 * np.max(np.abs(T.to_complex(ad)))


def test_exp_config5_against_fp64_reference(qla):
    rng = np.random.default_rng(23)
    n = 100003
    a, deg = T.antihermitian_exp_inputs(rng, n, np.float64)
    norm2 = np.sum(a.astype(np.float64) ** 2, axis=1)
    scale = np.maximum(1.0, norm2)[:, None]
    ref_d = T.ora_mfunc(a, n, "exp")
    got_d = _run(qla, "D3", "exp", a, n)
    err = np.abs(got_d - ref_d) / scale
    assert err.max() <= 1e-13, err.max()
    assert err[deg].max() <= 1e-13
    # unitarity of exp(iQ)
    u = T.to_complex(got_d)
    assert np.max(np.abs(np.conj(np.transpose(u, (0, 2, 1))) @ u - np.eye(3))) < 1e-13

    af = a.astype(np.float32)
    got_f = _run(qla, "F3", "exp", af, n)
    ref_fp64 = T.ora_mfunc(af.astype(np.float64), n, "exp")
    ok, nbad = T.qla_close(got_f, ref_fp64, np.float32)
    assert ok, nbad
    ref_f32 = T.ora_mfunc(af, n, "exp")  # the reference's own FP32 algorithm
    assert (np.abs(got_f.astype(np.float64) - ref_f32) / np.sqrt(scale)).max() <= 2e-5


def test_exp_general_matrices_and_zero(qla):
    rng = np.random.default_rng(24)
    n = 4099
    a = T.gaussian_field(rng, n, 9, np.float64) * rng.uniform(0, 3, n)[:, None]
    a[0] = 0.0
    got = _run(qla, "D3", "exp", a, n)
    want = T.ora_mfunc(a, n, "exp")
    # general (non-normal) matrices: the error of both methods scales with
    # |A|_F^2 and with the size of the result
    scale = (np.maximum(1.0, np.sum(a ** 2, axis=1)) * np.maximum(1.0, np.abs(want).max(axis=1)))[:, None]
    assert (np.abs(got - want) / scale).max() <= 1e-12
    assert np.array_equal(got[0], np.array([1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0], float))

"""Full-size parity of the level-1 configurations, through the C-ABI.

config 1 -- 16^4 = 65,536 sites, inputs drawn through QLA's own generator
  (QLA_seed_random per site, QLA_gaussian deviates, Haar SU(3) links by
  modified Gram-Schmidt, phase fix and det normalisation; ColorVectors from
  seed + 1): V_veq_M_times_V and V_veq_Ma_times_V bit-identical to the oracle
  in F3 and in D3 (the same float values promoted), r_veq_norm2_V within
  1e-12 of the exact sum (DF3, D3) and the correctly rounded float (F3).
config 2 -- the Wilson-hop-shaped sequence on the 32^3x64 periodic lattice
  (2,097,152 sites), F3 and D3, for all eight (mu, sign): the device-built
  neighbour table equals the host one; H_veq_spproj_D -> H_eq_M_times_xH
  through that table -> D_vpeq_sprecon_H accumulating all eight directions;
  V_veq_M_times_pV through a pointer array built from the same table; the
  fused hop term accumulating all eight directions, both through the table
  (D_peq_spproj_M_times_xD) and through QLA's pointer form
  (D_vpeq_spproj_M_times_pD).  Every
  intermediate and result bit-identical to the oracle (build_qla.pl:1087-1135,
  1588-1622; expressions_gamma.pl:205-337).
config 5 -- matrix functions on 2,097,152 sites: det and inverse of general
  matrices bit-identical (F3, D3); sqrt of A = B^+B + 0.1 bit-identical to
  the reference's own iteration (QLA_F3 in float, QLA_D3), F3 within
  1e-5 max(1, |A|_F) of FP64; exp of i Q (spectral norm U[0,3], 10%
  near-degenerate pairs) within the stated tolerances of the FP64 oracle.
"""
import numpy as np
import pytest

import qla_testlib as T

pytestmark = pytest.mark.gpu

DIMS2 = [32, 32, 32, 64]
N2 = 32 * 32 * 32 * 64


# ---------------------------------------------------------------------------
# config 1

@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_config1_qla_rng_haar_inputs(qla, pc, dt):
    n = 16 ** 4
    seed = 2025
    u = T.qla_rng_haar_su3(seed, n, np.float32).astype(dt)
    v = T.qla_rng_gaussian(seed + 1, n, 6).astype(dt)
    z = T.to_complex(u.astype(np.float64))
    assert np.abs(np.conj(np.transpose(z, (0, 2, 1))) @ z - np.eye(3)).max() < 1e-6
    ud, vd = T.to_dev(u), T.to_dev(v)
    ns = getattr(qla, pc)
    for name, adja in (("V_veq_M_times_V", 0), ("V_veq_Ma_times_V", 1)):
        rd = T.to_dev(np.zeros((n, 6), dt))
        getattr(ns, name)(rd, ud, vd, n)
        want = T.ora_lmult(np.zeros((n, 6), dt), u, v, n, 1, "eq", adja=adja)
        assert T.bits_equal(T.to_host(rd), want), (pc, name)
    exact = T.ora_norm2(v, n, 3, exact=True)
    red = qla.DF3 if pc == "F3" else qla.D3
    got = red.r_veq_norm2_V(None, vd, n)
    assert abs(got - exact) <= 1e-12 * exact, (pc, got, exact)
    if pc == "F3":
        gf = qla.F3.r_veq_norm2_V(None, vd, n)
        assert abs(gf - exact) <= 6e-8 * exact, (gf, exact)
    assert qla.device_error() == 0


# ---------------------------------------------------------------------------
# config 2

@pytest.fixture(scope="module")
def hop_inputs():
    """Haar links (one field per direction, from QLA's generator) and a
    Gaussian DiracFermion on the 32^3x64 lattice, in float; D3 uses the same
    values promoted."""
    u = [T.qla_rng_haar_su3(300 + mu, N2, np.float32) for mu in range(4)]
    d = T.qla_rng_gaussian(310, N2, 24)
    out0 = T.qla_rng_gaussian(311, N2, 24)
    vv = T.qla_rng_gaussian(312, N2, 6)
    nbr = {(mu, s): T.shift_index(DIMS2, mu, s) for mu in range(4) for s in (1, -1)}
    return u, d, out0, vv, nbr


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_config2_hop_sequence_full_lattice(qla, cuda, hop_inputs, pc, dt):
    u32, d32, out32, vv32, nbr = hop_inputs
    n = N2
    ns = getattr(qla, pc)
    rb = 8 if dt == np.float32 else 16  # bytes per complex number
    u = [x.astype(dt) for x in u32]
    d, vv = d32.astype(dt), vv32.astype(dt)
    ud = [T.to_dev(x) for x in u]
    dd, vd = T.to_dev(d), T.to_dev(vv)
    od = T.to_dev(out32.astype(dt))      # unfused sequence accumulates here
    fd = T.to_dev(out32.astype(dt))      # fused hop term (index form) accumulates here
    pd = T.to_dev(out32.astype(dt))      # fused hop term (pointer form) accumulates here
    want = out32.astype(dt)
    h = cuda.empty((n, 12), dtype=od.dtype, device="cuda")
    h2 = cuda.empty_like(h)
    vo = cuda.empty((n, 6), dtype=od.dtype, device="cuda")
    idx = cuda.empty(n, dtype=cuda.int32, device="cuda")
    for mu in range(4):
        for s in (1, -1):
            tab = nbr[(mu, s)]
            qla.shift_index(idx, DIMS2, mu, s)
            assert np.array_equal(T.to_host(idx), tab), (mu, s)
            ns.H_veq_spproj_D(h, dd, mu, s, n)
            hh = T.ora_spproj(np.zeros((n, 12), dt), d, n, mu, s, "eq")
            assert T.bits_equal(T.to_host(h), hh), (pc, "spproj", mu, s)
            ns.H_eq_M_times_xH(h2, ud[mu], h, idx, n)
            hh2 = T.ora_lmult(np.zeros((n, 12), dt), u[mu], hh, n, 2, "eq", idx_b=tab)
            assert T.bits_equal(T.to_host(h2), hh2), (pc, "M_times_xH", mu, s)
            ns.D_vpeq_sprecon_H(od, h2, mu, s, n)
            T.ora_sprecon(want, hh2, n, mu, s, "peq")
            ns.D_peq_spproj_M_times_xD(fd, ud[mu], dd, idx, mu, s, n)
            pdp = T.ptr_array(dd, tab, 12 * rb)
            ns.D_vpeq_spproj_M_times_pD(pd, ud[mu], pdp, mu, s, n)
            del pdp
            # the literal config op: V_veq_M_times_pV through pointers built from the table
            ptrs = T.ptr_array(vd, tab, 3 * rb)
            ns.V_veq_M_times_pV(vo, ud[mu], ptrs, n)
            wv = T.ora_lmult(np.zeros((n, 6), dt), u[mu], vv, n, 1, "eq", idx_b=tab)
            assert T.bits_equal(T.to_host(vo), wv), (pc, "M_times_pV", mu, s)
            del ptrs
    assert T.bits_equal(T.to_host(od), want), (pc, "sequence")
    # the fused term's own reference composition (spproj, multiply, sprecon
    # with eq intermediates, make_code_binary.pl:189-336), accumulated
    wf = out32.astype(dt)
    for mu in range(4):
        for s in (1, -1):
            T.ora_hop(wf, u[mu], d, n, mu, s, "peq", "D", "spproj", idx_b=nbr[(mu, s)])
    assert T.bits_equal(T.to_host(fd), wf), (pc, "fused, index form")
    assert T.bits_equal(T.to_host(pd), wf), (pc, "fused, pointer form")
    assert qla.device_error() == 0


# ---------------------------------------------------------------------------
# config 5

def _mf(qla, pc, fname, a, n):
    nout = 1 if fname == "det" else 9
    rd = T.to_dev(np.zeros((n, 2 * nout), dtype=a.dtype))
    dest = "C" if fname == "det" else "M"
    getattr(getattr(qla, pc), f"{dest}_veq_{fname}_M")(rd, T.to_dev(a), n)
    return T.to_host(rd)


@pytest.fixture(scope="module")
def mfunc_inputs():
    rng = np.random.default_rng(55)
    a_exp, deg = T.antihermitian_exp_inputs(rng, N2, np.float64)
    pos = T.positive_hermitian_inputs(rng, N2, np.float64)
    gen = T.gaussian_field(rng, N2, 9, np.float64)
    return a_exp, deg, pos, gen


@pytest.mark.parametrize("pc,dt", [("F3", np.float32), ("D3", np.float64)])
def test_config5_det_inverse_sqrt_full_size(qla, mfunc_inputs, pc, dt):
    _, _, pos, gen = mfunc_inputs
    n = N2
    g = gen.astype(dt)
    for fname in ("det", "inverse"):
        assert T.bits_equal(_mf(qla, pc, fname, g, n), T.ora_mfunc(g, n, fname)), (pc, fname)
    p = pos.astype(dt)
    got = _mf(qla, pc, "sqrt", p, n)
    assert T.bits_equal(got, T.ora_mfunc(p, n, "sqrt")), (pc, "sqrt")  # the reference's own iteration
    scale = np.maximum(1.0, np.sqrt(np.sum(p.astype(np.float64) ** 2, axis=1)))[:, None]
    assert (np.abs(got - T.ora_mfunc(p.astype(np.float64), n, "sqrt")) / scale).max() <= 1e-5, pc
    assert qla.device_error() == 0


def test_config5_exp_full_size(qla, mfunc_inputs):
    a, deg, _, _ = mfunc_inputs
    n = N2
    scale = np.maximum(1.0, np.sum(a ** 2, axis=1))[:, None]
    err = np.abs(_mf(qla, "D3", "exp", a, n) - T.ora_mfunc(a, n, "exp")) / scale
    assert err.max() <= 1e-13 and err[deg].max() <= 1e-13, err.max()
    af = a.astype(np.float32)
    got = _mf(qla, "F3", "exp", af, n)
    ok, nbad = T.qla_close(got, T.ora_mfunc(af.astype(np.float64), n, "exp"), np.float32)
    assert ok, nbad
    assert qla.device_error() == 0

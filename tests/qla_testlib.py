"""Test-side helpers: seeded lattice inputs and ctypes bindings of the checkers.

The checkers are the oracle (oracle/liboracle.so, a CPU restatement of the
reference algorithms) and, when it has been built, the reference library
itself (oracle/_ref/libqla_ref.so).  Nothing in the product imports this file.
"""
import ctypes
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, "oracle", "liboracle.so")
REF_SO = os.path.join(REPO, "oracle", "_ref", "libqla_ref.so")

EQOPS = {"eq": 0, "peq": 1, "meq": 2, "eqm": 3}
# complex numbers per record for Nc=3 (include/qla_types.h:29-33)
NCPLX3 = {"V": 3, "H": 6, "D": 12, "M": 9}
NCOL3 = {"V": 1, "H": 2, "D": 4, "M": 3}

_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle/liboracle.so not built (run make -C oracle)")
        _oracle = ctypes.CDLL(ORACLE_SO)
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
    return _ref


class ref_one_thread:
    """Runs the reference library's OpenMP loops on one thread (the sequential
    summation order of its reductions) inside the with-block."""

    def __enter__(self):
        ref()
        self.gomp = ctypes.CDLL("libgomp.so.1")
        self.prev = self.gomp.omp_get_max_threads()
        self.gomp.omp_set_num_threads(1)
        return self

    def __exit__(self, *exc):
        self.gomp.omp_set_num_threads(self.prev)
        return False


def ptr(a):
    """ctypes void pointer to a numpy array (None for None)."""
    if a is None:
        return None
    return ctypes.c_void_p(a.ctypes.data)


def rtype(dtype):
    return "f" if np.dtype(dtype) == np.float32 else "d"


# ---------------------------------------------------------------------------
# seeded inputs

def gaussian_field(rng, n, ncplx, dtype=np.float32):
    """n records of ncplx complex numbers with i.i.d. N(0,1) real/imag parts,
    as a flat real array of shape (n, 2*ncplx)."""
    return rng.standard_normal((n, 2 * ncplx)).astype(dtype)


def haar_su3(rng, n, dtype=np.float32, nc=3):
    """n Haar-random SU(nc) matrices: complex Gaussian, QR (Gram-Schmidt via
    numpy's Householder QR), diagonal phase fix, det normalised to 1.
    Returned as (n, 2*nc*nc) real array in [ic][jc] complex order."""
    z = (rng.standard_normal((n, nc, nc)) + 1j * rng.standard_normal((n, nc, nc))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=1, axis2=2)
    ph = d / np.abs(d)
    q = q * ph[:, None, :]
    det = np.linalg.det(q)
    q = q / (det ** (1.0 / nc))[:, None, None]
    out = np.empty((n, nc * nc, 2), dtype=np.float64)
    out[..., 0] = q.reshape(n, -1).real
    out[..., 1] = q.reshape(n, -1).imag
    return out.reshape(n, 2 * nc * nc).astype(dtype)


def qla_rng_gaussian(seed, n, nreal):
    """n records of nreal float N(0,1) deviates drawn the way a QLA program
    draws them: site i's generator seeded by QLA_seed_random(&S[i], seed, i)
    (lib/random/QLA_seed_random.c:13-34), then nreal successive QLA_gaussian
    calls on it (lib/random/QLA_gaussian.c:40-50, Box-Muller), through the
    oracle's restatement of both (pinned to the reference's lib/random)."""
    O = oracle()
    st = np.zeros((n, 11), np.uint32)
    O.ora_rng_seedfield(ptr(st), int(seed), ptr(np.arange(n, dtype=np.int32)), ctypes.c_long(n), None, None)
    g = np.zeros((n, nreal), np.float32)
    O.ora_rng_fill_f(nreal, 1, 0, ptr(g), ptr(st), ctypes.c_long(n), None, None)
    return g


def qla_rng_haar_su3(seed, n, dtype=np.float32):
    """n Haar-random SU(3) links from QLA's generator: per site 18 QLA_gaussian
    deviates (qla_rng_gaussian) form a complex Gaussian 3x3 (row-major
    [ic][jc], re/im interleaved), whose columns go through modified
    Gram-Schmidt QR in FP64; column j is multiplied by R_jj / |R_jj| (the
    phase fix), the matrix is divided by the principal cube root of its
    determinant, and the result is rounded to `dtype`."""
    g = qla_rng_gaussian(seed, n, 18).astype(np.float64)
    z = (g[:, 0::2] + 1j * g[:, 1::2]).reshape(n, 3, 3)
    q = np.empty_like(z)
    rdiag = np.empty((n, 3), dtype=np.complex128)
    for j in range(3):
        v = z[:, :, j].copy()
        for k in range(j):
            rkj = np.sum(np.conj(q[:, :, k]) * v, axis=1)
            v = v - rkj[:, None] * q[:, :, k]
        rjj = np.sqrt(np.sum(np.abs(v) ** 2, axis=1))
        q[:, :, j] = v / rjj[:, None]
        rdiag[:, j] = rjj
    q = q * (rdiag / np.abs(rdiag))[:, None, :]
    det = np.linalg.det(q)
    q = q / np.power(det, 1.0 / 3.0)[:, None, None]
    return from_complex(q, dtype)


def lattice_dims_volume(dims):
    v = 1
    for d in dims:
        v *= d
    return v


def shift_index(dims, mu, sign):
    """Periodic neighbour table: idx[i] = site at x + sign*e_mu, lexicographic
    i = x0 + L0*(x1 + L1*(x2 + L2*x3))."""
    dims = list(dims)
    coords = np.indices(dims[::-1]).reshape(len(dims), -1)[::-1]  # coords[d][i]
    c = coords.copy()
    c[mu] = (c[mu] + sign) % dims[mu]
    idx = np.zeros(c.shape[1], dtype=np.int64)
    stride = 1
    for d in range(len(dims)):
        idx += c[d] * stride
        stride *= dims[d]
    return idx.astype(np.int32)


# ---------------------------------------------------------------------------
# oracle wrappers (numpy in, numpy out)

def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def ora_lmult(r, a, b, n, ncol, eqop, adja=0, adjb=0, idx_a=None, idx_b=None, gang=None, nc=3):
    t = rtype(r.dtype)
    f = getattr(oracle(), "ora_lmult_" + t)
    idx_a, idx_b, gang = _i32(idx_a), _i32(idx_b), _i32(gang)
    f(ptr(r), ptr(a), ptr(b), ctypes.c_long(n), nc, ncol, EQOPS.get(eqop, eqop), adja, adjb,
      ptr(idx_a), ptr(idx_b), ptr(gang))
    return r


def ora_spproj(r, a, n, mu, sign, eqop, idx_a=None, gang=None, nc=3):
    f = getattr(oracle(), "ora_spproj_" + rtype(r.dtype))
    idx_a, gang = _i32(idx_a), _i32(gang)
    f(ptr(r), ptr(a), ctypes.c_long(n), nc, mu, sign, EQOPS.get(eqop, eqop), ptr(idx_a), ptr(gang))
    return r


def ora_sprecon(r, a, n, mu, sign, eqop, idx_a=None, gang=None, nc=3):
    f = getattr(oracle(), "ora_sprecon_" + rtype(r.dtype))
    idx_a, gang = _i32(idx_a), _i32(gang)
    f(ptr(r), ptr(a), ctypes.c_long(n), nc, mu, sign, EQOPS.get(eqop, eqop), ptr(idx_a), ptr(gang))
    return r


def ora_rtimes(r, s, b, n, ncplx, eqop, idx_b=None, gang=None):
    t = rtype(r.dtype)
    f = getattr(oracle(), "ora_rtimes_" + t)
    cs = ctypes.c_float(s) if t == "f" else ctypes.c_double(s)
    idx_b, gang = _i32(idx_b), _i32(gang)
    f(ptr(r), cs, ptr(b), ctypes.c_long(n), ncplx, EQOPS.get(eqop, eqop), ptr(idx_b), ptr(gang))
    return r


def ora_norm2(a, n, ncplx, exact=False, idx_a=None, gang=None):
    t = rtype(a.dtype)
    f = getattr(oracle(), ("ora_norm2_exact_" if exact else "ora_norm2_ref_") + t)
    f.restype = ctypes.c_double
    idx_a, gang = _i32(idx_a), _i32(gang)
    return f(ptr(a), ctypes.c_long(n), ncplx, ptr(idx_a), ptr(gang))


def ora_dot(a, b, n, ncplx, exact=False, idx_a=None, idx_b=None, gang=None):
    t = rtype(a.dtype)
    f = getattr(oracle(), ("ora_dot_exact_" if exact else "ora_dot_ref_") + t)
    out = np.zeros(2, dtype=np.float64)
    idx_a, idx_b, gang = _i32(idx_a), _i32(idx_b), _i32(gang)
    f(ptr(out), ptr(a), ptr(b), ctypes.c_long(n), ncplx, ptr(idx_a), ptr(idx_b), ptr(gang))
    return complex(out[0], out[1])


# ---------------------------------------------------------------------------
# tolerance rule of the reference test-suite (test/src/compare.h:10-25,
# protocol_compare.m4:80-91): an element fails only if its absolute difference
# exceeds NABS*eps AND its relative difference exceeds NREL*eps.

def qla_close(a, b, dtype, nabs=16, nrel=10):
    eps = np.finfo(dtype).eps
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    diff = np.abs(a - b)
    scale = np.maximum(np.abs(a), np.abs(b))
    rel = np.where(scale > 0, diff / np.where(scale > 0, scale, 1), 0)
    bad = (diff > nabs * eps) & (rel > nrel * eps)
    return not bool(np.any(bad)), int(np.count_nonzero(bad))


# ---------------------------------------------------------------------------
# device helpers (torch is imported lazily so CPU-only tests never need CUDA)

def to_dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def ptr_dev(t):
    """ctypes pointer to a device tensor's storage (the caller keeps t alive)."""
    return ctypes.c_void_p(t.data_ptr())


def to_host(t):
    return t.detach().cpu().numpy()


def ptr_array(base_t, idx, rec_bytes):
    """Device array of device pointers &base[idx[k]] (the `pX` argument form)."""
    import torch
    addrs = base_t.data_ptr() + idx.astype(np.int64) * rec_bytes
    return torch.from_numpy(addrs).cuda()


def bits_equal(a, b):
    """Bit-exact equality of two float arrays (treating +0 and -0 as equal,
    NaNs must agree in position)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    return bool(np.array_equal(a, b, equal_nan=True))


# ---------------------------------------------------------------------------
# matrix-function inputs (config 5) and oracle wrapper

MF = {"exp": 0, "sqrt": 1, "inverse": 2, "det": 3, "invsqrt": 4, "log": 5, "expA": 6, "expTA": 7, "sqrtPH": 8,
      "invsqrtPH": 9, "eigenvals": 10, "eigenvalsH": 11}


def to_complex(m, nc=3):
    m = np.asarray(m, dtype=np.float64)
    return (m[:, 0::2] + 1j * m[:, 1::2]).reshape(-1, nc, nc)


def from_complex(z, dtype):
    n = z.shape[0]
    out = np.empty((n, z.shape[1] * z.shape[2], 2))
    out[..., 0] = z.reshape(n, -1).real
    out[..., 1] = z.reshape(n, -1).imag
    return out.reshape(n, -1).astype(dtype)


def antihermitian_exp_inputs(rng, n, dtype, degenerate_frac=0.1, nc=3):
    """A = i Q, Q = W diag(lambda) W^+ with W Haar, lambda real traceless with
    spectral norm ~ U[0,3]; a fraction of sites get a pair with |l_i - l_j| < 1e-6."""
    w = to_complex(haar_su3(rng, n, np.float64, nc), nc)
    lam = rng.uniform(-1, 1, (n, nc))
    lam -= lam.mean(axis=1, keepdims=True)
    lam *= (rng.uniform(0, 3, n) / np.maximum(np.abs(lam).max(axis=1), 1e-300))[:, None]
    deg = rng.random(n) < degenerate_frac
    gap = rng.uniform(0, 1e-6, n)
    lam[deg, 1] = lam[deg, 0] + gap[deg]
    lam[deg] -= lam[deg].mean(axis=1, keepdims=True)
    q = w @ (lam[:, :, None] * np.conj(np.transpose(w, (0, 2, 1))))
    return from_complex(1j * q, dtype), deg


def positive_hermitian_inputs(rng, n, dtype, nc=3):
    """A = B^+ B + 0.1 1 with B complex Gaussian."""
    b = (rng.standard_normal((n, nc, nc)) + 1j * rng.standard_normal((n, nc, nc))) / np.sqrt(2)
    h = np.conj(np.transpose(b, (0, 2, 1))) @ b + 0.1 * np.eye(nc)
    return from_complex(h, dtype)


def ora_mfunc(a, n, which, nc=3):
    f = getattr(oracle(), "ora_mfunc_" + rtype(a.dtype))
    nout = 1 if which == "det" else nc if which.startswith("eigen") else nc * nc
    r = np.zeros((n, 2 * nout), dtype=a.dtype)
    rc = f(ptr(r), ptr(a), ctypes.c_long(n), nc, MF[which])
    if rc != 0:
        raise ValueError(f"oracle has no {which} at nc={nc}")
    return r


def ora_minv(a, b, n, nb, nc=3, idx_a=None, idx_b=None):
    """r = a^-1 b per site (nb = 1: ColorVector b, nb = nc: ColorMatrix b)."""
    f = getattr(oracle(), "ora_minv_" + rtype(a.dtype))
    r = np.zeros((n, 2 * nc * nb), dtype=a.dtype)
    idx_a, idx_b = _i32(idx_a), _i32(idx_b)
    f(ptr(r), ptr(a), ptr(b), ctypes.c_long(n), nc, nb, ptr(idx_a), ptr(idx_b))
    return r


def hermitian_inputs(rng, n, dtype, nc=3):
    """(G + G^+)/2 with G complex Gaussian: real spectrum of both signs."""
    g = rng.standard_normal((n, nc, nc)) + 1j * rng.standard_normal((n, nc, nc))
    return from_complex(0.5 * (g + np.conj(np.transpose(g, (0, 2, 1)))), dtype)


# ---------------------------------------------------------------------------
# QLA_I_ integer ops

INT_CODES = {"and": 6, "divide": 4, "eq": 11, "ge": 16, "gt": 15, "le": 14, "lshift": 9, "lt": 13, "mask": 19,
             "max": 17, "min": 18, "minus": 3, "mod": 5, "ne": 12, "or": 7, "plus": 2, "rshift": 10, "xor": 8}


def int_shape(shape):
    """(code, [pointer flag per field operand], takes a scalar) for a QLA_I_ shape."""
    import re
    p = lambda t: t.startswith("p")  # noqa: E731
    if shape in ("I", "pI"):
        return 0, [p(shape)], False
    if shape == "i":
        return 22, [], True
    if shape == "zero":
        return 21, [], False
    m = re.match(r"^(p?I)_times_(p?I)$", shape)
    if m:
        return 1, [p(m.group(1)), p(m.group(2))], False
    m = re.match(r"^i_times_(p?I)$", shape)
    if m:
        return 23, [p(m.group(1))], True
    m = re.match(r"^i_times_(p?I)_(plus|minus)_(p?I)$", shape)
    if m:
        return (24 if m.group(2) == "plus" else 25), [p(m.group(1)), p(m.group(3))], True
    m = re.match(r"^not_(p?I)$", shape)
    if m:
        return 20, [p(m.group(1))], False
    m = re.match(r"^(p?I)_(\w+)_(p?I)$", shape)
    return INT_CODES[m.group(2)], [p(m.group(1)), p(m.group(3))], False


def int_inputs(rng, n, ns):
    """Seeded int32 operands valid for every op (divisors and shift counts in
    1..31, a 0/1 mask), plus pointer/gang index tables."""
    return {
        "a": rng.integers(-1_000_000, 1_000_000, ns).astype(np.int32),
        "b": rng.integers(-1_000_000, 1_000_000, ns).astype(np.int32),
        "bs": rng.integers(1, 32, ns).astype(np.int32),
        "bm": rng.integers(0, 2, ns).astype(np.int32),
        "c": rng.integers(-1_000_000, 1_000_000, ns).astype(np.int32),
        "r0": rng.integers(-1_000_000, 1_000_000, n).astype(np.int32),
        "ia": rng.integers(0, ns, n).astype(np.int32),
        "ib": rng.integers(0, ns, n).astype(np.int32),
        "gang": rng.permutation(n).astype(np.int32),
        "s": np.array([-37], dtype=np.int32),
    }


def int_second(code):
    return "bs" if code in (4, 5, 9, 10) else ("bm" if code == 19 else "b")


def ora_int(name, ins, n):
    """Oracle result of QLA_I_<var><eqop>_<shape> on int_inputs()."""
    import re
    m = re.match(r"QLA_I_([vx])(eq|peq|meq|eqm)_(\w+)$", name)
    var, eq, shape = m.groups()
    code, ptrs, scal = int_shape(shape)
    r = ins["r0"].copy()
    srcs = ["a", int_second(code), "c"] if not scal else [("a"), int_second(code), "c"]
    if scal:
        srcs = ["a", "b"]  # the scalar forms take fields b (and c) of the C API; use a, b here
    fld = [ins[srcs[j]] for j in range(len(ptrs))] + [None] * (3 - len(ptrs))
    idx = [(ins["ia"] if j == 0 else ins["ib"]) if ptrs[j] else None for j in range(len(ptrs))] + \
          [None] * (3 - len(ptrs))
    gang = ins["gang"] if var == "x" else None
    f = oracle().ora_int
    f(code, EQOPS[eq], ptr(r), ptr(fld[0]), ptr(fld[1]), ptr(fld[2]), int(ins["s"][0]), ctypes.c_long(n),
      ptr(idx[0]), ptr(idx[1]), ptr(idx[2]), ptr(gang))
    return r


def int_call_args(name, ins, n, r, to_arr, to_ptrs):
    """Argument list of the C entry point, built with the caller's array
    constructors (host numpy for the reference, device for the product)."""
    import re
    m = re.match(r"QLA_I_([vx])(eq|peq|meq|eqm)_(\w+)$", name)
    var, eq, shape = m.groups()
    code, ptrs, scal = int_shape(shape)
    srcs = ["a", "b"] if scal else ["a", int_second(code)]
    args = [r]
    if scal:
        args.append(to_arr(ins["s"]))
    for j, isp in enumerate(ptrs):
        src = ins[srcs[j]]
        args.append(to_ptrs(src, ins["ia"] if j == 0 else ins["ib"]) if isp else to_arr(src))
    if var == "x":
        args.append(to_arr(ins["gang"]))
    args.append(n)
    return args


def ora_hop(r, a, b, n, mu, sign, eqop, dest, kind, adja=0, idx_b=None, gang=None, nc=3):
    """Fused hop terms composed from the oracle in the reference's order
    (make_code_binary.pl:189-336): intermediates with `eq`, eqop last.
    kind 'spproj': b is D; dest H: r (eqop) A spproj(b); dest D: r (eqop)
    sprecon(A spproj(b)); kind 'sprecon': b is H, r (eqop) sprecon(A b);
    a None: D (eqop) sprecon(spproj(b))."""
    dt = r.dtype
    nall = r.shape[0]
    sites = np.arange(n) if gang is None else np.asarray(gang)
    bsel = b[idx_b[sites]] if idx_b is not None else b[sites]
    asel = a[sites] if a is not None else None
    m = len(sites)
    if kind == "spproj":
        t1 = np.zeros((m, 4 * nc), dt)
        ora_spproj(t1, np.ascontiguousarray(bsel), m, mu, sign, "eq", nc=nc)
    else:
        t1 = np.ascontiguousarray(bsel)
    if asel is None:
        t2 = t1
    elif dest == "H":
        rr = np.ascontiguousarray(r[sites])
        ora_lmult(rr, np.ascontiguousarray(asel), t1, m, 2, eqop, adja=adja, nc=nc)
        r[sites] = rr
        return r
    else:
        t2 = np.zeros((m, 4 * nc), dt)
        ora_lmult(t2, np.ascontiguousarray(asel), t1, m, 2, "eq", adja=adja, nc=nc)
    rr = np.ascontiguousarray(r[sites])
    ora_sprecon(rr, t2, m, mu, sign, eqop, nc=nc)
    r[sites] = rr
    del nall
    return r


def ora_multi(r, ms, vs, n, eqop, adja=0, idx_a=None, idx_b=None, gang=None, nc=3):
    """r (eqop) sum_d A_d b_d with the reference's per-direction rounding
    (build_qla.pl:1693-1727): direction 0 uses the eqop, later directions
    accumulate into the rounded r with the eqop's sign."""
    minus = eqop in ("meq", "eqm")
    for d in range(len(ms)):
        eq_d = eqop if d == 0 else ("meq" if minus else "peq")
        ora_lmult(r, ms[d], vs[d], n, 1, eq_d, adja=adja, idx_a=idx_a, idx_b=idx_b, gang=gang, nc=nc)
    return r


PKIND = {"MP": 0, "PM": 1, "PP": 2, "TRACE": 3}


def ora_prop(kind, r, a, b, n, eqop, ca=0, cb=0, idx_a=None, idx_b=None, gang=None, nc=3):
    f = getattr(oracle(), "ora_prop_n_" + rtype(r.dtype))
    idx_a, idx_b, gang = _i32(idx_a), _i32(idx_b), _i32(gang)
    f(nc, PKIND[kind], ca, cb, EQOPS.get(eqop, eqop), ptr(r), ptr(a), ptr(b), ctypes.c_long(n), ptr(idx_a),
      ptr(idx_b), ptr(gang))
    return r


def prop_cases(lib, names, nc, dt, rng, n, ns):
    """Inputs and oracle results for the propagator entry points `names` of
    library `lib` (F3 / D3 / FN / DN) at nc colours.  Yields (name, args
    builder, want) where args(dev, ptrs_a, ptrs_b, gang_dev) gives the C
    arguments after the leading nc (FN / DN) in host (pointer) or device
    form, as the caller provides."""
    import re
    m = rng.standard_normal((ns, 2 * nc * nc)).astype(dt)
    p1 = rng.standard_normal((ns, 32 * nc * nc)).astype(dt)
    p2 = rng.standard_normal((ns, 32 * nc * nc)).astype(dt)
    r0p = rng.standard_normal((ns, 32 * nc * nc)).astype(dt)
    r0m = rng.standard_normal((ns, 2 * nc * nc)).astype(dt)
    ia = rng.integers(0, ns, ns).astype(np.int32)
    ib = rng.integers(0, ns, ns).astype(np.int32)
    gang = rng.permutation(n).astype(np.int32)
    data = {"M": m, "P1": p1, "P2": p2, "ia": ia, "ib": ib, "gang": gang}
    out = []
    pre = f"QLA_{lib}_"
    for name in names:
        short = name[len(pre):]
        mt = re.match(r"M_([vx])eq_spintrace_(p?)P$", short)
        if mt:
            var, pa = mt.groups()
            want = r0m[:n].copy()
            ora_prop("TRACE", want, p1, None, n, "eq", idx_a=ia if pa else None, gang=gang if var == "x" else None,
                     nc=nc)
            out.append((name, dict(var=var, a=("P1", bool(pa)), b=None, r0=r0m[:n]), want))
            continue
        var, eq, pa, ta, ca, pb, tb, cb = re.match(
            r"P_([vx])(eq|peq|meq|eqm)_(p?)(M|P)(a?)_times_(p?)(M|P)(a?)$", short).groups()
        ka = "M" if ta == "M" else "P1"
        kb = "M" if tb == "M" else "P2"
        want = r0p[:n].copy()
        ora_prop(ta + tb, want, data[ka], data[kb], n, eq, ca=int(bool(ca)), cb=int(bool(cb)),
                 idx_a=ia if pa else None, idx_b=ib if pb else None, gang=gang if var == "x" else None, nc=nc)
        out.append((name, dict(var=var, a=(ka, bool(pa)), b=(kb, bool(pb)), r0=r0p[:n]), want))
    return data, out


# ---------------------------------------------------------------------------
# element-wise families, site-local dot products, outer product: a generic
# case builder driven by the generated manifest (parameter types and kinds)

EW_SHAPES = {"COPY": 0, "CONJ": 1, "I": 2, "CT": 3, "CTA": 4, "CAT": 5, "CATA": 6, "RT": 7, "RTA": 8, "PLUS": 9,
             "MINUS": 10, "RT_PLUS": 11, "RT_MINUS": 12, "CT_PLUS": 13, "CT_MINUS": 14}
LD_KINDS = {"LD_DOT": 0, "LD_DOT_AA": 1, "LD_ADOT": 2, "LD_REDOT": 3, "LD_NORM2": 4}
NE3 = {"V": 3, "H": 6, "D": 12, "M": 9, "P": 144}
_TYPE_OF = {"ColorVector": "V", "HalfFermion": "H", "DiracFermion": "D", "ColorMatrix": "M",
            "DiracPropagator": "P", "Complex": "C", "Real": "R", "QLA_Int": "I", "QLA_RandomState": "S"}


def param_type(ctype):
    """(record letter, pointer array?) of a generated parameter type."""
    for k, v in _TYPE_OF.items():
        if k in ctype:
            return v, ctype.replace(" ", "").endswith("**")
    return None, False


def _perm_code(t):
    return {"M": 1, "P": 2}.get(t, 0)


def ewise_oracle_plan(e):
    """How the oracle computes manifest entry e: (function, keyword arguments
    that name the inputs)."""
    fam = e["family"]
    if fam == "ldot" and e["dest"] == "M":  # outer product
        return "outer", {}
    if fam == "ldot":
        return "ldot", {"kind": LD_KINDS[e["kind"]]}
    dest = e["dest"]
    if "scal" in e:
        sc, src = e["scal"], e["b"]
        adj = src.endswith("a")
        base = {"c": "CT", "r": "RT", "C": "CT", "pC": "CT", "Ca": "CAT", "pCa": "CAT", "R": "RT", "pR": "RT"}[sc]
        shape = base + ("A" if adj else "")
        kind = 1 if sc in ("c", "r") else (3 if sc in ("R", "pR") else 2)
        return "ewise", {"shape": EW_SHAPES[shape], "perm": _perm_code(dest) if adj else 0, "scal_kind": kind}
    op = e["op"]
    if op in ("plus", "minus", "r_plus", "r_minus", "c_plus", "c_minus"):
        shape = {"plus": "PLUS", "minus": "MINUS", "r_plus": "RT_PLUS", "r_minus": "RT_MINUS",
                 "c_plus": "CT_PLUS", "c_minus": "CT_MINUS"}[op]
        return "ewise", {"shape": EW_SHAPES[shape], "perm": 0, "scal_kind": 1 if op[0] in "rc" else 0}
    src = e["a"]
    if op == "conj_":
        return "ewise", {"shape": 1, "perm": 0, "scal_kind": 0}
    if op == "i_":
        return "ewise", {"shape": 2, "perm": 0, "scal_kind": 0}
    if op == "transpose_":
        return "ewise", {"shape": 0, "perm": _perm_code(dest), "scal_kind": 0}
    # "copy": the adjoint copy (Ma, Pa) or the plain P copy
    if src.endswith("a"):
        return "ewise", {"shape": 1, "perm": _perm_code(dest), "scal_kind": 0}
    return "ewise", {"shape": 0, "perm": 0, "scal_kind": 0}


def ne_at(letter, nc):
    """complex numbers per record of the given letter at nc colours"""
    return {"V": nc, "H": 2 * nc, "D": 4 * nc, "M": nc * nc, "P": 16 * nc * nc, "C": 1}[letter]


def ewise_inputs(e, rng, dt, n, ns, nc=3):
    """Seeded host inputs for manifest entry e: a dict param -> array (records
    of ns sites for sources, n sites for the destination), pointer-form
    index tables, and the gang subset for x forms."""
    ins = {}
    for t, name in zip(e["ctypes"], e["params"]):
        letter, is_ptr = param_type(t)
        if name in ("n", "index"):
            continue
        if letter is None:
            continue
        if name == "r":
            nrec = n
        else:
            nrec = ns
        if letter == "R":
            arr = rng.standard_normal(nrec).astype(dt)
        elif letter == "C":
            arr = rng.standard_normal((nrec, 2)).astype(dt)
        else:
            arr = rng.standard_normal((nrec, 2 * ne_at(letter, nc))).astype(dt)
        ins[name] = (letter, is_ptr, arr)
    # scalar constants (c / r forms): a single value
    plan, kw = ewise_oracle_plan(e)
    if plan == "ewise" and kw["scal_kind"] == 1:
        letter, is_ptr, _ = ins["a"]
        ins["a"] = (letter, False, (rng.standard_normal(1 if letter == "R" else 2)).astype(dt))
    idx = {name: rng.integers(0, ns, n).astype(np.int32) for name, v in ins.items() if v[1]}
    gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32) if e["var"] == "x" else None
    return ins, idx, gang


def ewise_oracle(e, ins, idx, gang, n, nc=3):
    """The oracle's result for manifest entry e on ewise_inputs()."""
    plan, kw = ewise_oracle_plan(e)
    r = ins["r"][2].copy()
    dt = r.dtype
    t = rtype(dt)
    g = _i32(gang)
    nsites = len(gang) if gang is not None else n
    eq = EQOPS[e.get("eqop", "eq")]

    def arr(name):
        return ins[name][2] if name in ins else None

    def ix(name):
        return _i32(idx.get(name))

    if plan == "outer":
        getattr(oracle(), "ora_outer_n_" + t)(nc, eq, ptr(r), ptr(arr("a")), ptr(arr("b")), ctypes.c_long(nsites),
                                             ptr(ix("a")), ptr(ix("b")), ptr(g))
        return r
    if plan == "ldot":
        ne = ne_at(ins["a"][0], nc)
        getattr(oracle(), "ora_ldot_n_" + t)(nc, kw["kind"], _perm_code(ins["a"][0]), eq, ptr(r), ptr(arr("a")),
                                            ptr(arr("b")), ctypes.c_long(nsites), ne, ptr(ix("a")), ptr(ix("b")),
                                            ptr(g))
        return r
    dest = e["dest"]
    ne = ne_at(dest, nc)
    cs = ctypes.c_float if t == "f" else ctypes.c_double
    sre = sim = 0.0
    s_arr, s_idx = None, None
    two = kw["shape"] >= 9
    if kw["scal_kind"] == 1:
        sv = arr("a")
        sre = float(sv[0])
        sim = float(sv[1]) if len(sv) > 1 else 0.0
        b_name, c_name = "b", ("c" if kw["shape"] >= 11 else None)
    elif kw["scal_kind"] in (2, 3):
        s_arr, s_idx = arr("a"), ix("a")
        b_name, c_name = "b", None
    elif two:
        b_name, c_name = "a", "b"
    else:
        b_name, c_name = "a", None
    getattr(oracle(), "ora_ewise_n_" + t)(nc, kw["shape"], kw["perm"], eq, ptr(r), ptr(arr(b_name)),
                                       ptr(arr(c_name)) if c_name else None, ptr(s_arr), kw["scal_kind"],
                                       cs(sre), cs(sim), ctypes.c_long(nsites), ne, ptr(ix(b_name)),
                                       ptr(ix(c_name)) if c_name else None, ptr(s_idx), ptr(g))
    return r


# ---------------------------------------------------------------------------
# site-field families (fills, copymask, components, gamma multiplication,
# traces) and the global P / adjoint-form reductions and global sums

SF_FAMILIES = ("fill", "mask", "component", "gamma", "trace")
NE_OF = dict(NE3, C=1)


def rec_bytes(letter, dt, nc=3):
    """bytes per record of a field of the given letter in precision dt"""
    if letter == "I":
        return 4
    if letter == "S":
        return 44
    return np.dtype(dt).itemsize * (1 if letter == "R" else 2 * ne_at(letter, nc))


NCOLOR_FAMILIES = ("ewise_v", "ewise_h", "ewise_d", "ewise_m", "ewise_p", "ldot", "fill", "mask", "component",
                   "gamma", "trace", "gred", "gsum", "convert")


def fixed_colour_twin(name):
    """The QLA_F3_ / QLA_D3_ / QLA_DF3_ / QLA_FD3_ entry point a QLA_FN_ /
    QLA_DN_ / QLA_DFN_ / QLA_FDN_ one generalises."""
    import re
    m = re.match(r"QLA_(FN|DN|DFN|FDN|F2|D2|DF2|FD2)_(.*)$", name)
    return "QLA_" + {"FN": "F3", "DN": "D3", "DFN": "DF3", "FDN": "FD3", "F2": "F3", "D2": "D3", "DF2": "DF3",
                     "FD2": "FD3"}[m.group(1)] + "_" + m.group(2)


def ncolor_case(e, rng, n, ns, nc):
    """(inputs, oracle result, kind) of the fixed-colour twin entry e at nc
    colours: kind "map" (bit-exact field result), "gred" / "gsum" (one value
    or record, reference summation order), "convert"."""
    fam = e["family"]
    dt = np.float64 if e["pc"] == "D3" else np.float32
    if fam == "convert":
        ins, idx, gang = convert_inputs(e, rng, n, ns, nc=nc)
        return (ins, idx, gang, {}), convert_oracle(e, ins, idx, gang, n, nc=nc), "convert"
    if fam in ("gred", "gsum"):
        ins, idx, gang, ints = sitefield_inputs(e, rng, dt, n, ns, nc=nc)
        if fam == "gred":
            out = gred_oracle(e, ins, idx, gang, n, nc=nc)
            odt = np.float64 if e.get("out") == "double" else dt
            want = out[:1].astype(odt) if e["dest"] == "r" else out.astype(odt)
        else:
            want = gsum_oracle(e, ins, idx, gang, n, nc=nc)
        return (ins, idx, gang, ints), want, fam
    if fam in SF_FAMILIES:
        ins, idx, gang, ints = sitefield_inputs(e, rng, dt, n, ns, nc=nc)
        return (ins, idx, gang, ints), sitefield_oracle(e, ins, idx, gang, n, ints, nc=nc), "map"
    ins, idx, gang = ewise_inputs(e, rng, dt, n, ns, nc=nc)
    return (ins, idx, gang, {}), ewise_oracle(e, ins, idx, gang, n, nc=nc), "map"


def _letter(src):
    return src[1:] if src.startswith("p") and len(src) > 1 else src


def sitefield_inputs(e, rng, dt, n, ns, nc=3):
    """Seeded inputs for a site-field entry: (ins, idx, gang, ints) with ins
    as ewise_inputs, ints the values of the int arguments (colour / spin
    indices, mu)."""
    ins, ints = {}, {}
    half = e.get("dest") == "H" or _letter(e.get("a", "")) == "H"
    for t, name in zip(e["ctypes"], e["params"]):
        if name in ("n", "index"):
            continue
        if t == "int":
            hi = {"mu": 16, "i_c": nc, "j_c": nc, "i_s": 2 if half else 4, "j_s": 4}[name]
            ints[name] = int(rng.integers(0, hi))
            continue
        letter, is_ptr = param_type(t)
        nrec = n if name == "r" else ns
        if name == "a" and e.get("op") in ("fill", "diagfill"):
            nrec = 1
        if letter == "I":
            arr = rng.choice(np.array([0, 0, 1, -3, 7], np.int32), nrec)
        elif letter == "R":
            arr = rng.standard_normal(nrec).astype(dt)
        elif letter == "C":
            arr = rng.standard_normal((nrec, 2)).astype(dt)
        else:
            arr = rng.standard_normal((nrec, 2 * ne_at(letter, nc))).astype(dt)
        if name == "a" and e.get("op") in ("fill", "diagfill"):
            arr = arr.reshape(-1)
        ins[name] = (letter, is_ptr, arr)
    idx = {name: rng.integers(0, ns, n).astype(np.int32) for name, v in ins.items() if v[1]}
    gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32) if e["var"] == "x" else None
    return ins, idx, gang, ints


def sitefield_oracle(e, ins, idx, gang, n, ints, nc=3):
    """The oracle's result for a site-field entry on sitefield_inputs()."""
    r = ins["r"][2].copy()
    t = rtype(r.dtype)
    g = _i32(gang)
    nsites = ctypes.c_long(len(gang) if gang is not None else n)
    eq = EQOPS[e.get("eqop", "eq")]
    O = oracle()
    op, fam = e.get("op"), e["family"]

    def arr(name):
        return ins[name][2] if name in ins else None

    def ix(name):
        return _i32(idx.get(name))

    if op == "fill":
        getattr(O, "ora_fill_" + t)(eq, ptr(r), ptr(arr("a")), nsites, ne_at(e["dest"], nc), ptr(g))
    elif op == "diagfill":
        getattr(O, "ora_diagfill_n_" + t)(nc, eq, ptr(r), ptr(arr("a")), nsites, ptr(g))
    elif op == "zero":
        getattr(O, "ora_zero_" + t)(ptr(r), nsites, ne_at(e["dest"], nc), ptr(g))
    elif op == "mask":
        getattr(O, "ora_mask_" + t)(ptr(r), ptr(arr("a")), ptr(arr("b")), nsites, ne_at(e["dest"], nc),
                                    ptr(ix("a")), ptr(ix("b")), ptr(g))
    elif fam == "component":
        what = {"elem": "e", "colorvec": "c", "diracvec": "d"}[op]
        getattr(O, "ora_component_n_" + t)(nc, ord(what), ord(e["dest"]), ord(_letter(e["a"])), ptr(r),
                                           ptr(arr("a")), ints.get("i_c", 0), ints.get("i_s", 0),
                                           ints.get("j_c", 0), ints.get("j_s", 0), nsites, ptr(ix("a")), ptr(g))
    elif fam == "gamma":
        getattr(O, "ora_gamma_n_" + t)(nc, 1 if op == "gamma_right" else 0, ne_at(e["dest"], nc), ints["mu"],
                                       ptr(r), ptr(arr("a")), nsites, ptr(ix("a")), ptr(g))
    elif fam == "trace":
        kind = {"trace": 0, "re_trace": 1, "im_trace": 2, "antiherm": 3}[op]
        getattr(O, "ora_trace_n_" + t)(nc, kind, ptr(r), ptr(arr("a")), nsites, ptr(ix("a")), ptr(g))
    else:
        raise ValueError(e["name"])
    return r


def gred_oracle(e, ins, idx, gang, n, nc=3):
    """Reference-order global reduction (re, im) in double for a gred entry."""
    a = ins["a"][2]
    t = rtype(a.dtype)
    out = np.zeros(2, np.float64)
    kind = LD_KINDS[e["kind"]]
    perm = _perm_code(_letter(e["a"]).rstrip("a"))
    b = ins["b"][2] if "b" in ins else None
    getattr(oracle(), "ora_gdot_n_" + t)(nc, kind, perm, ptr(out), ptr(a), ptr(b),
                                         ctypes.c_long(len(gang) if gang is not None else n),
                                         ne_at(_letter(e["a"]).rstrip("a"), nc), ptr(_i32(idx.get("a"))),
                                         ptr(_i32(idx.get("b"))), ptr(_i32(gang)))
    return out


def gsum_oracle(e, ins, idx, gang, n, nc=3):
    """Reference-order global sum (one record) for a gsum entry, rounded to
    the output precision (the site precision; double for QLA_DF3_)."""
    a = ins["a"][2]
    t = rtype(a.dtype)
    T = _letter(e["a"])
    out = np.zeros(2 * ne_at(T, nc), np.float64)
    getattr(oracle(), "ora_gsum_" + t)(ptr(out), ptr(a), ctypes.c_long(len(gang) if gang is not None else n),
                                       ne_at(T, nc), ptr(_i32(idx.get("a"))), ptr(_i32(gang)))
    return out if e.get("out") == "double" else out.astype(a.dtype)


def convert_inputs(e, rng, n, ns, nc=3):
    """Inputs of a QLA_DF3_ / QLA_FD3_ conversion: (ins, idx, gang)."""
    src_dt, dst_dt = (np.float32, np.float64) if e["lib"] == "DF3" else (np.float64, np.float32)
    ne = ne_at(e["dest"], nc)
    a = rng.standard_normal((ns, 2 * ne)).astype(src_dt)
    r = rng.standard_normal((n, 2 * ne)).astype(dst_dt)
    ins = {"r": (e["dest"], False, r), "a": (e["dest"], e["a"].startswith("p"), a)}
    idx = {"a": rng.integers(0, ns, n).astype(np.int32)} if e["a"].startswith("p") else {}
    gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32) if e["var"] == "x" else None
    return ins, idx, gang


def convert_oracle(e, ins, idx, gang, n, nc=3):
    r = ins["r"][2].copy()
    f = oracle().ora_convert_df if e["lib"] == "DF3" else oracle().ora_convert_fd
    f(ptr(r), ptr(ins["a"][2]), ctypes.c_long(len(gang) if gang is not None else n), 2 * ne_at(e["dest"], nc),
      ptr(_i32(idx.get("a"))), ptr(_i32(gang)))
    return r


# ---------------------------------------------------------------------------
# random-number generator state fields (QLA_RandomState: 11 32-bit words)

def rng_states(rng, ns):
    """ns seeded generator states (QLA_seed_random with varied seeds and
    indices), each advanced by a few draws."""
    st = np.zeros((ns, 11), np.uint32)
    O = oracle()
    for k in range(ns):
        row = st[k]
        O.ora_rng_seed(ptr(row), int(rng.integers(-2**31, 2**31 - 1)), int(rng.integers(0, 1 << 20)))
        for _ in range(int(rng.integers(0, 5))):
            O.ora_rng_uniform(ptr(row))
    return st


def random_case(e, rng, n, ns, nc=3, milc=0):
    """Inputs and the oracle's results for a random-family entry e (a
    fixed-colour, F / D or S entry): (ins, idx, gang, ints, want_r, want_states)
    where ins maps parameter -> (letter, pointer?, array) as ewise_inputs and
    want_states is the state field after the call (None when not written)."""
    O = oracle()
    op = e["op"]
    gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32) if e["var"] == "x" else None
    nsites = ctypes.c_long(len(gang) if gang is not None else n)
    idx, ins, ints = {}, {}, {}
    if op in ("gaussian", "random"):
        dt = np.float64 if e["pc"] in ("D3", "D", "DN") else np.float32
        nreal = 1 if e["dest"] == "R" else (2 if e["dest"] == "C" else 2 * ne_at(e["dest"], nc))
        r = rng.standard_normal((n, nreal)).astype(dt)
        st = rng_states(rng, ns)
        ptr_s = e["a"].startswith("p")
        ins = {"r": (e["dest"], False, r), "a": ("S", ptr_s, st)}
        if ptr_s:
            idx["a"] = rng.permutation(ns)[:n].astype(np.int32)
        want_r, want_s = r.copy(), st.copy()
        getattr(O, "ora_rng_fill_" + rtype(dt))(nreal, int(op == "gaussian"), milc, ptr(want_r), ptr(want_s),
                                                nsites, ptr(_i32(idx.get("a"))), ptr(_i32(gang)))
        return ins, idx, gang, ints, want_r, want_s
    r = rng_states(rng, n)
    ins["r"] = ("S", False, r)
    want = r.copy()
    if op == "seed":
        a = rng.integers(0, 1 << 20, ns).astype(np.int32)
        ins["a"] = ("I", e["a"].startswith("p"), a)
        if e["a"].startswith("p"):
            idx["a"] = rng.integers(0, ns, n).astype(np.int32)
        ints["seed"] = int(rng.integers(-2**31, 2**31 - 1))
        O.ora_rng_seedfield(ptr(want), ints["seed"], ptr(a), nsites, ptr(_i32(idx.get("a"))), ptr(_i32(gang)))
        return ins, idx, gang, ints, want, None
    a = rng_states(rng, ns)
    ins["a"] = ("S", e["a"].startswith("p"), a)
    if e["a"].startswith("p"):
        idx["a"] = rng.integers(0, ns, n).astype(np.int32)
    m = None
    if op == "mask":
        m = rng.choice(np.array([0, 1, -2, 0], np.int32), ns)
        ins["b"] = ("I", e["b"].startswith("p"), m)
        if e["b"].startswith("p"):
            idx["b"] = rng.integers(0, ns, n).astype(np.int32)
    O.ora_rng_copy(ptr(want), ptr(a), ptr(m), nsites, ptr(_i32(idx.get("a"))), ptr(_i32(idx.get("b"))),
                   ptr(_i32(gang)))
    return ins, idx, gang, ints, want, None


# ---------------------------------------------------------------------------
# QLA_F_ / QLA_D_ / QLA_DF_ real, complex and integer fields

def scalar_op_codes():
    """name -> code of the product's ScalarOp enumeration (read from its
    header, the single source of the numbering)."""
    import re
    txt = open(os.path.join(REPO, "qla_b200", "csrc", "qla_scalar.cuh")).read()
    body = txt[txt.index("enum ScalarOp"):]
    body = body[body.index("{") + 1:body.index("};")]
    names = re.findall(r"\b(SO_\w+)\b", re.sub(r"//[^\n]*", "", body))
    return {nm: i for i, nm in enumerate(names)}


# transcendental ops: CUDA's functions, compared to the host libm within a few ulp
SCALAR_APPROX = {"SO_R_SIN", "SO_R_COS", "SO_R_TAN", "SO_R_ASIN", "SO_R_ACOS", "SO_R_ATAN", "SO_R_EXP", "SO_R_LOG",
                 "SO_R_LOG10", "SO_R_SINH", "SO_R_COSH", "SO_R_TANH", "SO_R_POW", "SO_R_ATAN2", "SO_R_ARG",
                 "SO_C_CEXP", "SO_C_CEXPI", "SO_C_CLOG"}


def _fd_values(rng, spec, name, size, dt):
    """Seeded values in the domain of scalar op `spec` for operand `name`."""
    u = lambda lo, hi: rng.uniform(lo, hi, size).astype(dt)  # noqa: E731
    if spec in ("SO_R_ASIN", "SO_R_ACOS"):
        return u(-1, 1)
    if spec in ("SO_R_SQRT", "SO_R_LOG", "SO_R_LOG10"):
        return u(0.01, 10)
    if spec == "SO_R_POW":
        return u(0.1, 3) if name == "a" else u(-2, 2)
    if spec in ("SO_R_EXP", "SO_R_SINH", "SO_R_COSH", "SO_R_TANH"):
        return u(-5, 5)
    if spec == "SO_R_TAN":
        return u(-1.5, 1.5)
    if spec in ("SO_I_ROUND", "SO_I_TRUNC"):
        v = u(-1000, 1000)
        v[::5] = np.round(v[::5]) + 0.5
        return v
    if spec in ("SO_R_DIVIDE", "SO_R_MOD") and name == "b":
        v = u(0.5, 3)
        v[::2] *= -1
        return v
    return (rng.standard_normal(size) * 3).astype(dt)


def fd_case(e, rng, n, ns):
    """Inputs and the oracle's result for a QLA_F_ / QLA_D_ / QLA_DF_ entry
    e: (ins, idx, gang, want, mode) with mode "exact", "approx" (within a
    few ulp), "reduce" (one value, reference summation order) or "convert"."""
    O = oracle()
    plan, spec = e.get("plan"), e.get("spec")
    lib = e["name"].split("_")[1]
    if e["family"] == "convert":
        src = np.float32 if e["lib"] == "DF" else np.float64
        dst = np.float64 if e["lib"] == "DF" else np.float32
        nr = 1 if e["dest"] == "R" else 2
        a = rng.standard_normal((ns, nr)).astype(src)
        r = rng.standard_normal((n, nr)).astype(dst)
        ptr_a = e["a"].startswith("p")
        ins = {"r": (e["dest"], False, r), "a": (e["dest"], ptr_a, a)}
        idx = {"a": rng.integers(0, ns, n).astype(np.int32)} if ptr_a else {}
        gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32) if e["var"] == "x" else None
        want = r.copy()
        f = O.ora_convert_df if e["lib"] == "DF" else O.ora_convert_fd
        f(ptr(want), ptr(a), ctypes.c_long(len(gang) if gang is not None else n), nr, ptr(_i32(idx.get("a"))),
          ptr(_i32(gang)))
        return ins, idx, gang, want, "convert"
    dt = np.float64 if lib == "D" else np.float32
    t = "d" if lib == "D" else "f"
    gang = rng.permutation(n)[: n // 2 + 1].astype(np.int32) if e["var"] == "x" else None
    nsites = ctypes.c_long(len(gang) if gang is not None else n)
    ins, idx = {}, {}
    sval = None
    for nm, l in e["opnds"]:
        if l in "rc":
            v = (rng.standard_normal(1 if l == "r" else 2) * 1.5).astype(dt)
            ins[nm] = (l.upper(), False, v)
            sval = v
            continue
        tok = e[nm]
        is_ptr = tok.startswith("p")
        if l == "I":
            if spec == "SO_R_MASK" or plan == "mask":
                arr = rng.choice(np.array([0, 1, -3, 0, 7], np.int32), ns)
            elif spec == "SO_R_LDEXP":
                arr = rng.integers(-10, 11, ns).astype(np.int32)
            else:
                arr = rng.integers(-1000, 1001, ns).astype(np.int32)
        elif l == "R":
            arr = _fd_values(rng, spec, nm, ns, dt)
            if spec in ("SO_I_EQ", "SO_I_GE", "SO_I_LE", "SO_I_NE") and nm == "b":
                arr[::3] = ins["a"][2][::3] if not ins["a"][1] else arr[::3]
        else:
            arr = (rng.standard_normal((ns, 2)) * 2).astype(dt)
        ins[nm] = (l, is_ptr, arr)
        if is_ptr:
            idx[nm] = rng.integers(0, ns, n).astype(np.int32)
    dest = e["dest"]
    if dest in "cr":
        out_dt = np.float64 if lib in ("D", "DF") else np.float32
        want_len = 2 if (dest == "c" or (plan == "gsum")) else 1
        ins["r"] = (dest, False, np.zeros(want_len, out_dt))
        a, b = ins["a"][2], ins["b"][2] if "b" in ins else None
        ia, ib = _i32(idx.get("a")), _i32(idx.get("b"))
        if plan == "gdot":
            out = np.zeros(2, np.float64)
            getattr(O, "ora_gdot_" + t)(LD_KINDS[spec], 0, ptr(out), ptr(a), ptr(b), nsites, 1, ptr(ia), ptr(ib),
                                        ptr(_i32(gang)))
            want = out[:want_len].astype(out_dt)
        elif plan == "gsum":
            out = np.zeros(2, np.float64)
            getattr(O, "ora_gsum_" + t)(ptr(out), ptr(a), nsites, 1, ptr(ia), ptr(_i32(gang)))
            want = out.astype(out_dt)
        else:
            f = getattr(O, "ora_sred_" + t)
            f.restype = ctypes.c_double
            isint = int(ins["a"][0] == "I")
            v = f({"SR_DOT": 0, "SR_NORM2": 1, "SR_SUM": 2}[spec], isint, ptr(a), ptr(b), nsites, ptr(ia), ptr(ib),
                  ptr(_i32(gang)))
            want = np.array([v], out_dt)
        return ins, idx, gang, want, "reduce"
    shape_r = {"R": (n,), "I": (n,), "C": (n, 2)}[dest]
    r = (rng.standard_normal(shape_r) * 2).astype(np.int32 if dest == "I" else dt)
    ins["r"] = (dest, False, r)
    want = r.copy()
    eq = EQOPS[e["eqop"]]
    arr = lambda nm: ins[nm][2] if nm in ins else None  # noqa: E731
    ix = lambda nm: _i32(idx.get(nm))  # noqa: E731
    cs = ctypes.c_float if dt == np.float32 else ctypes.c_double
    if plan == "ew":
        shape, sk = spec
        code = EW_SHAPES[shape]
        sre = sim = 0.0
        if sk == 0:
            bn, cn, sn = "a", ("b" if shape in ("PLUS", "MINUS") else None), None
        elif sk == 1:
            bn, cn, sn = "b", ("c" if "c" in ins else None), None
            sre = float(sval[0])
            sim = float(sval[1]) if len(sval) > 1 else 0.0
        else:
            bn, cn, sn = "b", None, "a"
        getattr(O, "ora_ewise_n_" + t)(3, code, 0, eq, ptr(want), ptr(arr(bn)), ptr(arr(cn)) if cn else None,
                                       ptr(arr(sn)) if sn else None, sk, cs(sre), cs(sim), nsites, 1, ptr(ix(bn)),
                                       ptr(ix(cn)) if cn else None, ptr(ix(sn)) if sn else None, ptr(_i32(gang)))
        return ins, idx, gang, want, "exact"
    if plan == "fill":
        getattr(O, "ora_fill_" + t)(eq, ptr(want), ptr(arr("a")), nsites, 1, ptr(_i32(gang)))
        return ins, idx, gang, want, "exact"
    if plan == "zero":
        getattr(O, "ora_zero_" + t)(ptr(want), nsites, 1, ptr(_i32(gang)))
        return ins, idx, gang, want, "exact"
    if plan == "mask":
        getattr(O, "ora_mask_" + t)(ptr(want), ptr(arr("a")), ptr(arr("b")), nsites, 1, ptr(ix("a")), ptr(ix("b")),
                                    ptr(_i32(gang)))
        return ins, idx, gang, want, "exact"
    if plan == "ldot":
        getattr(O, "ora_ldot_" + t)(LD_KINDS[spec], 0, eq, ptr(want), ptr(arr("a")), ptr(arr("b")), nsites, 1,
                                    ptr(ix("a")), ptr(ix("b")), ptr(_i32(gang)))
        return ins, idx, gang, want, "exact"
    code = scalar_op_codes()[spec]
    has_const = any(l in "rc" for _, l in e["opnds"])
    getattr(O, "ora_scalar_" + t)(code, eq, ptr(want), None if has_const else ptr(arr("a")), ptr(arr("b")),
                                  ptr(arr("c")), cs(float(sval[0]) if has_const else 0.0), nsites,
                                  None if has_const else ptr(ix("a")), ptr(ix("b")), ptr(ix("c")), ptr(_i32(gang)))
    return ins, idx, gang, want, ("approx" if spec in SCALAR_APPROX else "exact")


def within_ulps(got, want, k=4):
    """got and want agree within k units in the last place of want (NaN and
    infinities must match exactly)."""
    g = np.asarray(got).ravel()
    w = np.asarray(want).ravel()
    if g.dtype != w.dtype:
        return False
    nan_g, nan_w = np.isnan(g), np.isnan(w)
    if np.any(nan_g != nan_w):
        return False
    fin = np.isfinite(w) & ~nan_w
    if np.any(g[~fin & ~nan_w] != w[~fin & ~nan_w]):
        return False
    return bool(np.all(np.abs(g[fin].astype(np.float64) - w[fin].astype(np.float64))
                       <= k * np.spacing(np.abs(w[fin])).astype(np.float64)))

"""qla_b200 -- QLA 1.9.0 level-1 site operators on NVIDIA B200 (sm_100a).

The product is the C-ABI shared library ``qla_b200/lib/libqla_b200.so``: the
reference's QLA_F3_/QLA_D3_/QLA_DF3_ function names and signatures
(include/qla_b200_*.h) over device-resident arrays, implemented by
hand-written CUDA kernels.  This Python package only loads that library and
offers a thin mirror of the C API for Python callers and tests:

    import qla_b200 as qla
    qla.F3.V_veq_M_times_V(r, a, b, n)      # r, a, b: CUDA tensors (or raw device pointers)

There is no CPU fallback: if the library is missing, importing the mirror
raises.  Build it with ``python -m qla_b200.build``.
"""
import ctypes
import json
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libqla_b200.so")
MANIFEST_PATH = os.path.join(_PKG, "gen", "api_manifest.json")

_lib = None


class QLAError(RuntimeError):
    pass


def lib():
    """The loaded libqla_b200.so (raises QLAError when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QLAError(f"{LIB_PATH} is missing: build it with `python -m qla_b200.build` "
                           "(qla_b200 has no CPU fallback)")
        _lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
        _lib.qlagpu_last_error.restype = ctypes.c_int
        _lib.qlagpu_last_error_string.restype = ctypes.c_char_p
        _lib.qlagpu_device_error.restype = ctypes.c_uint
        _lib.qlagpu_device_error.argtypes = [ctypes.c_int]
        _lib.qlagpu_set_stream.argtypes = [ctypes.c_void_p]
        _lib.qlagpu_get_stream.restype = ctypes.c_void_p
        _lib.qlagpu_tune_set.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        _lib.qlagpu_version.restype = ctypes.c_char_p
        _lib.qlagpu_shift_index.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_int]
    return _lib


def manifest():
    with open(MANIFEST_PATH) as f:
        return json.load(f)


def last_error():
    """(code, message) of the calling thread's sticky status."""
    L = lib()
    return L.qlagpu_last_error(), L.qlagpu_last_error_string().decode()


def clear_error():
    lib().qlagpu_clear_error()


def check(where=""):
    """Raise QLAError if the sticky status is set (and clear it)."""
    code, msg = last_error()
    if code:
        clear_error()
        raise QLAError(f"{where}: qla_b200 error {code}: {msg}")


def set_stream(stream):
    """Issue subsequent calls of this thread on `stream` (a torch.cuda.Stream,
    a raw cudaStream_t as int, or None for the legacy default stream)."""
    handle = getattr(stream, "cuda_stream", stream)
    lib().qlagpu_set_stream(ctypes.c_void_p(handle or 0))


def device_error(clear=True):
    return lib().qlagpu_device_error(1 if clear else 0)


def _addr(x):
    """Device address of a CUDA tensor, or a raw integer address."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    dp = getattr(x, "data_ptr", None)
    if dp is not None:
        if not getattr(x, "is_cuda", True):
            raise QLAError("qla_b200 array arguments must be CUDA tensors (device memory)")
        return dp()
    raise QLAError(f"cannot take the address of {type(x)}")


_REAL_CT = {"QLA_F_Real *": ctypes.c_float, "QLA_D_Real *": ctypes.c_double}
_CPLX_CT = {"QLA_F_Complex *": ctypes.c_float, "QLA_D_Complex *": ctypes.c_double}


class _Fn:
    """Python mirror of one C entry point.  Field arguments take CUDA tensors
    (or integer device addresses); a scalar coefficient takes a Python number
    (passed as a host scalar) or a CUDA tensor (left on the device); a
    reduction output takes a CUDA tensor, or None to get the value back."""

    def __init__(self, entry):
        self.entry = entry
        self.name = entry["name"]
        self.fn = getattr(lib(), self.name)
        self.fn.restype = None
        self.fn.argtypes = [ctypes.c_int if t == "int" else ctypes.c_void_p for t in entry["ctypes"]]

    def __call__(self, *args):
        e = self.entry
        red = e["family"] in ("norm2", "dot", "redot", "gred")
        ridx = e["params"].index("r") if red else 0
        if len(args) != len(e["params"]) and not (red and len(args) == len(e["params"]) - 1):
            raise TypeError(f"{self.name} takes {len(e['params'])} arguments ({', '.join(e['params'])})")
        cargs = []
        keep = []
        ret = None
        reduction_host = red and (len(args) < len(e["params"]) or args[ridx] is None)
        if reduction_host and len(args) < len(e["params"]):
            args = tuple(args[:ridx]) + (None,) + tuple(args[ridx:])
        for i, (t, v) in enumerate(zip(e["ctypes"], args)):
            if t == "int":
                cargs.append(int(v))
            elif i == ridx and reduction_host:
                ct = _REAL_CT.get(t) or _CPLX_CT.get(t)
                n = 2 if t in _CPLX_CT else 1
                buf = (ct * n)()
                keep.append(buf)
                cargs.append(ctypes.cast(buf, ctypes.c_void_p))
                ret = (buf, n)
            elif t in _REAL_CT and not hasattr(v, "data_ptr"):
                s = _REAL_CT[t](float(v))
                keep.append(s)
                cargs.append(ctypes.cast(ctypes.pointer(s), ctypes.c_void_p))
            else:
                cargs.append(_addr(v))
        self.fn(*cargs)
        check(self.name)
        if ret is not None:
            buf, n = ret
            return complex(buf[0], buf[1]) if n == 2 else float(buf[0])
        return None


class _Namespace:
    def __init__(self, pc):
        self._pc = pc
        self._fns = {}

    def __getattr__(self, short):
        if short.startswith("_"):
            raise AttributeError(short)
        name = f"QLA_{self._pc}_{short}"
        f = self._fns.get(name)
        if f is None:
            entries = {e["name"]: e for e in manifest()}
            if name not in entries:
                raise AttributeError(f"{name} is not part of libqla_b200")
            f = self._fns[name] = _Fn(entries[name])
        return f


F3 = _Namespace("F3")
D3 = _Namespace("D3")
DF3 = _Namespace("DF3")
FD3 = _Namespace("FD3")
FN = _Namespace("FN")
DN = _Namespace("DN")
DFN = _Namespace("DFN")
I = _Namespace("I")  # noqa: E741


def shift_index(idx, dims, mu, sign):
    """Fill the int32 CUDA tensor idx with the periodic neighbour table of the
    lexicographic lattice `dims` (x0 fastest) in direction mu, sign +-1."""
    arr = (ctypes.c_int * len(dims))(*dims)
    lib().qlagpu_shift_index(_addr(idx), len(dims), ctypes.cast(arr, ctypes.c_void_p), mu, sign)
    check("qlagpu_shift_index")


def check_index(idx, n, nsrc):
    """qlagpu_check_index: (return code, first bad position or -1) for the
    int32 index stream idx[0..n) against [0, nsrc)."""
    L = lib()
    L.qlagpu_check_index.restype = ctypes.c_int
    L.qlagpu_check_index.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p]
    first = ctypes.c_longlong(-2)
    rc = L.qlagpu_check_index(_addr(idx), int(n), int(nsrc), ctypes.byref(first))
    return rc, first.value


def version():
    return lib().qlagpu_version().decode()


class _BatchField(ctypes.Structure):
    _fields_ = [("r", ctypes.c_void_p), ("u", ctypes.c_void_p), ("u2", ctypes.c_void_p), ("nbr", ctypes.c_void_p),
                ("w", ctypes.c_void_p), ("v", ctypes.c_void_p), ("n", ctypes.c_longlong)]


class BatchPlan:
    """Plan of the batched uneven-volume sequence (qlagpu_F3_batch_plan): for
    every field, r = u * u2[nbr] then w = r * v, all in one persistent launch.
    `fields` is a list of dicts with CUDA tensors (or device addresses) for
    keys r, u, u2, nbr, w, v and the site count n."""

    def __init__(self, fields):
        L = lib()
        L.qlagpu_F3_batch_plan.restype = ctypes.c_void_p
        L.qlagpu_F3_batch_plan.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.qlagpu_batch_run.restype = ctypes.c_int
        L.qlagpu_batch_run.argtypes = [ctypes.c_void_p]
        L.qlagpu_batch_destroy.argtypes = [ctypes.c_void_p]
        arr = (_BatchField * len(fields))()
        for k, f in enumerate(fields):
            arr[k] = _BatchField(*[_addr(f[key]) for key in ("r", "u", "u2", "nbr", "w", "v")], int(f["n"]))
        self._keep = fields
        self.handle = L.qlagpu_F3_batch_plan(ctypes.cast(arr, ctypes.c_void_p), len(fields))
        if not self.handle:
            check("qlagpu_F3_batch_plan")
            raise QLAError("qlagpu_F3_batch_plan failed")

    def run(self):
        rc = lib().qlagpu_batch_run(self.handle)
        if rc:
            check("qlagpu_batch_run")

    def close(self):
        if getattr(self, "handle", None):
            lib().qlagpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# batched sequences (qlagpu_F3_batch_plan_program)
REC = {"V": 0, "H": 1, "D": 2, "M": 3}
ROLE = {"in": 0, "out": 1, "inout": 2}
BOP = {"lmult": 0, "spproj": 1, "sprecon": 2, "rtimes": 3, "copy": 4}
EQOP = {"eq": 0, "peq": 1, "meq": 2, "eqm": 3}
REG0, REG1 = 8, 9


class _BatchStream(ctypes.Structure):
    _fields_ = [("base", ctypes.c_void_p), ("index", ctypes.c_void_p), ("nsrc", ctypes.c_longlong),
                ("kind", ctypes.c_int), ("role", ctypes.c_int)]


class _BatchStep(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("eqop", ctypes.c_int), ("a", ctypes.c_int), ("b", ctypes.c_int),
                ("dst", ctypes.c_int), ("store", ctypes.c_int), ("adja", ctypes.c_int), ("adjb", ctypes.c_int),
                ("mu", ctypes.c_int), ("sign", ctypes.c_int), ("r", ctypes.c_float)]


class _BatchProgram(ctypes.Structure):
    _fields_ = [("n", ctypes.c_longlong), ("nstreams", ctypes.c_int), ("nsteps", ctypes.c_int),
                ("stream", _BatchStream * 8), ("step", _BatchStep * 8)]


class BatchProgramPlan(BatchPlan):
    """Plan of per-field level-1 programs (qlagpu_F3_batch_plan_program), all
    fields in one persistent launch.  `programs` is a list of dicts:

        {"n": sites,
         "streams": [{"base": tensor, "index": int32 tensor or None, "nsrc": 0,
                      "kind": "V"|"H"|"D"|"M", "role": "in"|"out"|"inout"}, ...],
         "steps": [{"op": "lmult"|"spproj"|"sprecon"|"rtimes"|"copy",
                    "eqop": "eq"|"peq"|"meq"|"eqm", "a": stream or REG0/REG1,
                    "b": ..., "dst": REG0|REG1, "store": stream or -1,
                    "adja": 0, "adjb": 0, "mu": 0, "sign": 1, "r": 0.0}, ...]}
    """

    def __init__(self, programs):
        L = lib()
        L.qlagpu_F3_batch_plan_program.restype = ctypes.c_void_p
        L.qlagpu_F3_batch_plan_program.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.qlagpu_batch_run.restype = ctypes.c_int
        L.qlagpu_batch_run.argtypes = [ctypes.c_void_p]
        L.qlagpu_batch_destroy.argtypes = [ctypes.c_void_p]
        arr = (_BatchProgram * len(programs))()
        for k, pr in enumerate(programs):
            q = arr[k]
            q.n = int(pr["n"])
            q.nstreams = len(pr["streams"])
            q.nsteps = len(pr["steps"])
            for j, st in enumerate(pr["streams"]):
                idx = st.get("index")
                q.stream[j] = _BatchStream(_addr(st["base"]), _addr(idx) if idx is not None else None,
                                           int(st.get("nsrc", 0)), REC[st["kind"]], ROLE[st["role"]])
            for j, sp in enumerate(pr["steps"]):
                q.step[j] = _BatchStep(BOP[sp["op"]], EQOP[sp.get("eqop", "eq")], int(sp["a"]), int(sp.get("b", 0)),
                                       int(sp.get("dst", REG0)), int(sp.get("store", -1)), int(sp.get("adja", 0)),
                                       int(sp.get("adjb", 0)), int(sp.get("mu", 0)), int(sp.get("sign", 1)),
                                       float(sp.get("r", 0.0)))
        self._keep = programs
        self.handle = L.qlagpu_F3_batch_plan_program(ctypes.cast(arr, ctypes.c_void_p), len(programs))
        if not self.handle:
            check("qlagpu_F3_batch_plan_program")
            raise QLAError("qlagpu_F3_batch_plan_program failed")


#!/usr/bin/env python3
"""Generator of the QLA B200 C-ABI: the QLA level-1 entry points for the hot
families, as extern "C" wrappers over the CUDA engine, plus their prototypes.

It replaces the reference's Perl generator (lib/perl/build_qla.pl) for the
site-loop families on the B200 path.  Where build_qla.pl walks every
(operation x eqop x datatype x indexing variant) and writes one C loop per
combination (build_qla.pl:186-2705, prototype.pl:450 make_prototype), this
generator walks the same combinations for the hot families and writes one
short wrapper per combination that picks a compiled engine OP; the loop body
itself lives once per family in qla_b200/csrc/qla_ops.cuh.

Naming follows the reference (doc/qla.tex:390-627, prototype.pl:450-520):
  QLA_<PC>_<dest>_<v|x><eqop>_<args>   with eqop in eq, peq, meq, eqm,
  `p` before an operand for an array of pointers, a trailing `int *index` for
  the gang-indexed `x` variants (indirection.pl:66-101), scalars passed by
  pointer.  The per-operand index forms `..._times_xV(r, a, b, int *jb, n)` are
  documented by the reference (doc/qla.tex:476-487, variant 5) but not
  generated there; they are the int32 neighbour-gather form of `pV`.

Outputs (all written by this script, committed):
  include/qla_b200_<pc>.h               prototypes, each citing what it replaces
  qla_b200/csrc/gen/<pc>_<family>.cu    wrappers (split per family to compile in parallel)
  qla_b200/gen/api_manifest.json        every symbol with its family and argument kinds
"""
import itertools
import json
import re
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT_INC = os.path.join(REPO, "include")
OUT_CU = os.path.join(REPO, "qla_b200", "csrc", "gen")

EQOPS = ["eq", "peq", "meq", "eqm"]
EQ_ENUM = {"eq": "qlab::EQ", "peq": "qlab::PEQ", "meq": "qlab::MEQ", "eqm": "qlab::EQM"}
# record abbreviation -> (type name, columns per colour row, complex per record at Nc=3)
REC = {"V": ("ColorVector", 1, 3), "H": ("HalfFermion", 2, 6), "D": ("DiracFermion", 4, 12),
       "M": ("ColorMatrix", 3, 9), "P": ("DiracPropagator", 48, 144)}
FIELD_TYPES = ["V", "H", "D", "M"]

# citations into the reference generator for each family
CITE = {
    "lmult": "lib/perl/build_qla.pl:1588-1622 (left multiplication by a colour matrix), "
             "expressions_tensor.pl:766",
    "lmult_x": "doc/qla.tex:476-487 (per-operand index variant 5, not generated by the reference)",
    "spproj": "lib/perl/build_qla.pl:1087-1110, make_code_unary.pl:183-241, expressions_gamma.pl:244-275",
    "sprecon": "lib/perl/build_qla.pl:1112-1135, expressions_gamma.pl:309-337",
    "rtimes": "lib/perl/build_qla.pl:1256-1292 (real constant times field)",
    "copy": "lib/perl/build_qla.pl:370-400 (assignment / gather)",
    "copy_x": "doc/qla.tex:555-575 (unary per-operand index variant 5, not generated by the reference)",
    "norm2": "lib/perl/build_qla.pl:2089-2155, make_code_unary.pl:318-365 (global norm2)",
    "dot": "lib/perl/build_qla.pl:2196-2360, make_code_binary.pl:110-172 (global inner product)",
    "redot": "lib/perl/build_qla.pl:2250-2284 (real part of the global inner product)",
    "hop": "lib/perl/build_qla.pl:1137-1250 (fused spin projection x colour matrix), make_code_binary.pl:189-336",
    "hop_x": "doc/qla.tex:476-487 (per-operand index variant 5 of the fused hop terms, not generated by the reference)",
    "multi": "lib/perl/build_qla.pl:1693-1727 (multi-direction sum r = sum_d a_d * b_d)",
    "prop": "lib/perl/build_qla.pl:1588-1661 (DiracPropagator left/right/full products), :942-968 (spin trace)",
    "mfunc": "lib/perl/build_qla.pl:1000-1060 (matrix functions), code-templates/M_eq_exp_M.c:243-367, "
             "M_eq_sqrt_M.c:73-181, M_eq_inverse_M.c:50-162, C_eq_det_M.c:50-143",
}
CITE["mfunc_ext"] = ("lib/perl/build_qla.pl:1022-1061 (matrix functions, eigenvalues), code-templates/"
                     "M_eq_invsqrt_M.c:88-127, M_eq_log_M.c:127-199, M_eq_expA_M.c:100-298, "
                     "M_eq_expTA_M.c:96-274, M_eq_sqrtPH_M.c:84-197, M_eq_invsqrtPH_M.c:84-201, "
                     "V_eq_eigenvals_M.c:127-186, V_eq_eigenvalsH_M.c:106-166")
for _t in "vhdmp":
    CITE["ewise_" + _t] = "lib/perl/build_qla.pl:403-469, 1256-1420 (element-wise families)"
CITE["ewise_times"] = "lib/perl/build_qla.pl:1256-1335 (constant multiples of a field), include/qla_complex.h:258-400"
CITE["ewise_field"] = "lib/perl/build_qla.pl:1256-1335 (per-site complex / real field times a field)"
CITE["ewise_unary"] = "lib/perl/build_qla.pl:403-469 (conj, i, adjoint and transpose copies)"
CITE["ewise_sum"] = "lib/perl/build_qla.pl:1338-1420 (sums, differences, r/c times a field plus / minus a field)"
CITE["ldot"] = "lib/perl/build_qla.pl:2358-2460 (site-local dot products and norms)"
CITE["outer"] = "lib/perl/build_qla.pl:1588-1622 (ColorVector times adjoint ColorVector)"
CITE["fill"] = ("lib/perl/build_qla.pl:2561-2618 (zero fills, constant fills, diagonal fill of a colour matrix), "
                "make_code_unary.pl (identity, diagfill, zero)")
CITE["mask"] = "lib/perl/build_qla.pl:2058-2084 (copymask: r = a where the integer mask is non-zero)"
CITE["component"] = ("lib/perl/build_qla.pl:767-931 (array components, colour column vectors and Dirac vectors: "
                     "extraction and insertion)")
CITE["gamma"] = ("lib/perl/build_qla.pl:1358-1412 (left / right multiplication by gamma_mu, mu = 0..15), "
                 "expressions_gamma.pl:59-134, 384-470")
CITE["trace"] = "lib/perl/build_qla.pl:933-1064 (trace, real / imaginary trace, traceless antihermitian part)"
CITE["gred"] = ("lib/perl/build_qla.pl:2089-2272 (global norm2 and inner products of DiracPropagators, "
                "trace of the adjoint-form products Ma.M and Pa.P)")
CITE["gsum"] = "lib/perl/build_qla.pl:2449-2521 (global sums of a field over the sites)"
CITE["random"] = ("lib/perl/build_qla.pl:2620-2690 (uniform and gaussian random fills, seeding), "
                  "lib/random/QLA_random.c:18-36, QLA_gaussian.c:19-55, QLA_seed_random.c:13-36")
CITE["scalar"] = ("lib/perl/build_qla.pl:186-355, 1936-2082, 2089-2555 (real, complex and integer fields: "
                  "elementary functions, arithmetic, comparisons, masks, conversions, reductions), "
                  "include/qla_complex.h:110-140, 417-428, lib/cmath")
CITE["cfield"] = CITE["rfield"] = CITE["sglobal"] = CITE["scalar"]
CITE["convert"] = ("lib/perl/build_qla.pl:356-400 (copying between precisions: QLA_DF_c_eq_c promotion, "
                   "QLA_FD_c_eq_c rounding)")
CITE["reunit"] = ("no counterpart in the reference: r = a (a^+ a)^(-1/2), the composition of "
                  "M_veq_Ma_times_M, M_veq_invsqrtPH_M and M_veq_M_times_M fused in FP64")
CITE["minv"] = ("lib/perl/build_qla.pl:1663-1690 (colour matrix inverse times vector / matrix), "
                "code-templates/V_eq_M_inverse_V.c:84-168, M_eq_M_inverse_M.c:85-135")
MFUNC_OPS = {"exp": "ExpOp", "sqrt": "SqrtOp", "inverse": "InverseOp"}
# the remaining matrix functions: name -> OP template (R substituted)
MFUNC_EXT_OPS = {"invsqrt": "InvsqrtOp<{R}>", "log": "LogOp<{R}>", "expA": "ExpAHOp<{R}, true>",
                 "expTA": "ExpAHOp<{R}, false>", "sqrtPH": "SqrtPHOp<{R}, false>",
                 "invsqrtPH": "SqrtPHOp<{R}, true>"}
EIGEN_OPS = {"eigenvals": "EigenvalsOp<{R}>", "eigenvalsH": "EigenvalsHOp<{R}>"}
CITE["int"] = "lib/perl/build_qla.pl:1932-2082 (integer fields)"
# QLA_I_ binary operators offered with veq/xeq only (build_qla.pl:1932-2082)
INT_BINOPS = {"and": "IC_AND", "divide": "IC_DIVIDE", "eq": "IC_EQ", "ge": "IC_GE", "gt": "IC_GT", "le": "IC_LE",
              "lshift": "IC_LSHIFT", "lt": "IC_LT", "mask": "IC_MASK", "max": "IC_MAX", "min": "IC_MIN",
              "minus": "IC_MINUS", "mod": "IC_MOD", "ne": "IC_NE", "or": "IC_OR", "plus": "IC_PLUS",
              "rshift": "IC_RSHIFT", "xor": "IC_XOR"}


FN_NCS = [2, 3, 4, 8]          # colour counts with compiled QLA_FN_ kernels
FN_MFUNC_NCS = [2, 3, 4, 8]    # nc = 2: the templates' two-colour closed forms
# the two-colour closed-form OP of each matrix function (qla_mfunc_nc2.cuh)
NC2_FN = {"exp": "N2_EXP", "sqrt": "N2_SQRT", "invsqrt": "N2_INVSQRT", "log": "N2_LOG", "expA": "N2_EXPA",
          "expTA": "N2_EXPTA", "sqrtPH": "N2_SQRTPH", "invsqrtPH": "N2_INVSQRTPH", "inverse": "N2_INVERSE",
          "det": "N2_DET", "eigenvals": "N2_EIG", "eigenvalsH": "N2_EIGH"}


def _nc2_op(fname, R="float"):
    return f"Nc2MfuncOp<{R}, qlab::{NC2_FN[fname]}>"


# remaining matrix functions for QLA_FN_: nc -> OP (closed forms at nc = 2
# and 3, the templates' generic exp / Newton paths otherwise)
FN_MFUNC_EXT = {
    "invsqrt": lambda nc: _nc2_op("invsqrt") if nc == 2 else f"GenMfuncExtOp<float, {nc}, 0>",
    "log": lambda nc: _nc2_op("log") if nc == 2 else f"GenMfuncExtOp<float, {nc}, 1>",
    "expA": lambda nc: (_nc2_op("expA") if nc == 2 else "ExpAHOp<float, true>" if nc == 3
                        else f"GenMfuncExtOp<float, {nc}, 2>"),
    "expTA": lambda nc: (_nc2_op("expTA") if nc == 2 else "ExpAHOp<float, false>" if nc == 3
                         else f"GenMfuncExtOp<float, {nc}, 2>"),
    "sqrtPH": lambda nc: (_nc2_op("sqrtPH") if nc == 2 else "SqrtPHOp<float, false>" if nc == 3
                          else f"GenMfuncExtOp<float, {nc}, 3>"),
    "invsqrtPH": lambda nc: (_nc2_op("invsqrtPH") if nc == 2 else "SqrtPHOp<float, true>" if nc == 3
                             else f"GenMfuncExtOp<float, {nc}, 4>"),
}


def _fn_switch(ncs, call_of_nc, name):
    """switch (nc) over the compiled colour counts; other nc record an error."""
    cases = "".join(f"    case {nc}: {call_of_nc(nc)} break;\n" for nc in ncs)
    return (f"switch (nc) {{\n{cases}    default: qlab::set_error(QLAGPU_ERR_ARG, \"{name}\", "
            f"\"nc not compiled (supported: {', '.join(map(str, ncs))})\");\n  }}")


def gen_fn(prec="F"):
    """QLA_FN_ / QLA_DFN_ (prec "F") or QLA_DN_ (prec "D") entry points
    (colour count nc at run time, doc/qla.tex:595-611): the hot families of
    gen_pc for nc in FN_NCS."""
    fns = []
    R = "float" if prec == "F" else "double"
    LIB = prec + "N"
    cols = {"V": lambda nc: 1, "H": lambda nc: 2, "D": lambda nc: 4, "M": lambda nc: nc}
    ncpl = {"V": lambda nc: nc, "H": lambda nc: 2 * nc, "D": lambda nc: 4 * nc, "M": lambda nc: nc * nc}
    kid = lambda fam: f'"{LIB}_{fam}"'  # noqa: E731

    def opnd(ptr, arg):
        return (f"qlab::op_ptr((const void* const*){arg})" if ptr else f"qlab::op_contig({arg})")

    def add(name, params, body, family, cite, kinds):
        fns.append(Fn(name, [("int", "nc")] + params, body, family, cite, kinds))

    for T in FIELD_TYPES:
        src2s = [(T, False), ("p" + T, True)] + ([("Ma", False), ("pMa", True)] if T == "M" else [])
        for var in ["v", "x"]:
            gang = "index" if var == "x" else "nullptr"
            tail = [("int *", "index")] if var == "x" else []
            for eq in EQOPS:
                for s1 in ["M", "Ma", "pM", "pMa"]:
                    adja = s1.endswith("a")
                    for s2, p2 in src2s:
                        adjb = s2.endswith("a")
                        name = f"QLA_{LIB}_{T}_{var}{eq}_{s1}_times_{s2}"
                        call = lambda nc, T=T, adja=adja, adjb=adjb, s1=s1, p2=p2, eq=eq, gang=gang: (
                            f"qlab::api_map<qlab::LMultOp<{R}, {nc}, {cols[T](nc)}, {str(adja).lower()}, "
                            f"{str(adjb).lower()}>>({kid('lmult')}, r, {opnd(s1.startswith('p'), 'a')}, "
                            f"{opnd(p2, 'b')}, {gang}, n, {EQ_ENUM[eq]});")
                        add(name, [("void *", "r"), ("void *", "a"), ("void *", "b")] + tail + [("int", "n")],
                            _fn_switch(FN_NCS, call, name), "lmult", CITE["lmult"],
                            dict(dest=T, eqop=eq, var=var, a=s1, b=s2))
        for eq in EQOPS:
            for s1 in ["M", "Ma"]:
                name = f"QLA_{LIB}_{T}_{eq}_{s1}_times_x{T}"
                call = lambda nc, T=T, s1=s1, eq=eq: (
                    f"qlab::api_map<qlab::LMultOp<{R}, {nc}, {cols[T](nc)}, {str(s1 == 'Ma').lower()}, false>>("
                    f"{kid('lmult')}, r, qlab::op_contig(a), qlab::op_idx(b, jb), nullptr, n, {EQ_ENUM[eq]});")
                add(name, [("void *", "r"), ("void *", "a"), ("void *", "b"), ("int *", "jb"), ("int", "n")],
                    _fn_switch(FN_NCS, call, name), "lmult", CITE["lmult_x"],
                    dict(dest=T, eqop=eq, var="xb", a=s1, b="x" + T))
        for var in ["v", "x"]:
            gang = "index" if var == "x" else "nullptr"
            tail = [("int *", "index")] if var == "x" else []
            for eq in EQOPS:
                for src, p1 in [(T, False), ("p" + T, True)]:
                    name = f"QLA_{LIB}_{T}_{var}{eq}_r_times_{src}"
                    call = lambda nc, T=T, p1=p1, eq=eq, gang=gang: (
                        f"qlab::api_scalar_map<qlab::RTimesOp<{R}, {ncpl[T](nc)}>, {R}>({kid('rtimes')}, r, "
                        f"(const {R}*)a, {opnd(p1, 'b')}, {gang}, n, {EQ_ENUM[eq]});")
                    add(name, [("void *", "r"), (f"QLA_{prec}_Real *", "a"), ("void *", "b")] + tail + [("int", "n")],
                        _fn_switch(FN_NCS, call, name), "rtimes", CITE["rtimes"],
                        dict(dest=T, eqop=eq, var=var, b=src))
                    name = f"QLA_{LIB}_{T}_{var}{eq}_{src}"
                    call = lambda nc, T=T, p1=p1, eq=eq, gang=gang: (
                        f"qlab::api_map<qlab::CopyOp<{R}, {ncpl[T](nc)}>>({kid('copy')}, r, {opnd(p1, 'a')}, "
                        f"qlab::Opnd{{}}, {gang}, n, {EQ_ENUM[eq]});")
                    add(name, [("void *", "r"), ("void *", "a")] + tail + [("int", "n")],
                        _fn_switch(FN_NCS, call, name), "copy", CITE["copy"], dict(dest=T, eqop=eq, var=var, a=src))
        # global reductions: FN (float result) and DFN (double result)
        for rpc, outR, OP in ((("FN", "float", "F"), ("DFN", "double", "D")) if prec == "F" else
                              (("DN", "double", "D"),)):
            for var in ["v", "x"]:
                gang = "index" if var == "x" else "nullptr"
                tail = [("int *", "index")] if var == "x" else []
                for src, p1 in [(T, False), ("p" + T, True)]:
                    name = f"QLA_{rpc}_r_{var}eq_norm2_{src}"
                    call = lambda nc, T=T, p1=p1, gang=gang, outR=outR: (
                        f"qlab::api_reduce<qlab::Norm2Op<{R}, {ncpl[T](nc)}, {outR}>>({kid('norm2')}, r, "
                        f"sizeof({outR}), {opnd(p1, 'a')}, qlab::Opnd{{}}, {gang}, n);")
                    add(name, [(f"QLA_{OP}_Real *", "r"), ("void *", "a")] + tail + [("int", "n")],
                        _fn_switch(FN_NCS, call, name), "norm2", CITE["norm2"],
                        dict(dest="r", var=var, a=src, out=outR))
                for sa, pa_ in [(T, False), ("p" + T, True)]:
                    for sb, pb_ in [(T, False), ("p" + T, True)]:
                        name = f"QLA_{rpc}_c_{var}eq_{sa}_dot_{sb}"
                        call = lambda nc, T=T, pa_=pa_, pb_=pb_, gang=gang, outR=outR: (
                            f"qlab::api_reduce<qlab::DotOp<{R}, {ncpl[T](nc)}, {outR}>>({kid('dot')}, r, "
                            f"2 * sizeof({outR}), {opnd(pa_, 'a')}, {opnd(pb_, 'b')}, {gang}, n);")
                        add(name, [(f"QLA_{OP}_Complex *", "r"), ("void *", "a"), ("void *", "b")] + tail +
                            [("int", "n")], _fn_switch(FN_NCS, call, name), "dot", CITE["dot"],
                            dict(dest="c", var=var, a=sa, b=sb, out=outR))
                        name = f"QLA_{rpc}_r_{var}eq_re_{sa}_dot_{sb}"
                        call = lambda nc, T=T, pa_=pa_, pb_=pb_, gang=gang, outR=outR: (
                            f"qlab::api_reduce<qlab::ReDotOp<{R}, {ncpl[T](nc)}, {outR}>>({kid('redot')}, r, "
                            f"sizeof({outR}), {opnd(pa_, 'a')}, {opnd(pb_, 'b')}, {gang}, n);")
                        add(name, [(f"QLA_{OP}_Real *", "r"), ("void *", "a"), ("void *", "b")] + tail +
                            [("int", "n")], _fn_switch(FN_NCS, call, name), "redot", CITE["redot"],
                            dict(dest="r", var=var, a=sa, b=sb, out=outR))
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        tail = [("int *", "index")] if var == "x" else []
        for eq in EQOPS:
            for src, p1 in [("D", False), ("pD", True)]:
                name = f"QLA_{LIB}_H_{var}{eq}_spproj_{src}"
                call = lambda nc, p1=p1, eq=eq, gang=gang: (
                    f"qlab::api_map<qlab::SpprojOp<{R}, {nc}>>({kid('spproj')}, r, {opnd(p1, 'a')}, "
                    f"qlab::Opnd{{}}, {gang}, n, {EQ_ENUM[eq]}, mu, sign);")
                add(name, [("void *", "r"), ("void *", "a"), ("int", "mu"), ("int", "sign")] + tail + [("int", "n")],
                    "if (mu < 0 || mu > 4) return;\n  " + _fn_switch(FN_NCS, call, name), "spproj",
                    CITE["spproj"], dict(eqop=eq, var=var, a=src))
            for src, p1 in [("H", False), ("pH", True)]:
                name = f"QLA_{LIB}_D_{var}{eq}_sprecon_{src}"
                call = lambda nc, p1=p1, eq=eq, gang=gang: (
                    f"qlab::api_map<qlab::SpreconOp<{R}, {nc}>>({kid('sprecon')}, r, {opnd(p1, 'a')}, "
                    f"qlab::Opnd{{}}, {gang}, n, {EQ_ENUM[eq]}, mu, sign);")
                add(name, [("void *", "r"), ("void *", "a"), ("int", "mu"), ("int", "sign")] + tail + [("int", "n")],
                    "if (mu < 0 || mu > 4) return;\n  " + _fn_switch(FN_NCS, call, name), "sprecon",
                    CITE["sprecon"], dict(eqop=eq, var=var, a=src))
        for src, p1 in [("M", False), ("pM", True)]:
            for fname, opname in (("exp", "GenExpOp"), ("sqrt", "GenSqrtOp"), ("inverse", "GenInverseOp")):
                name = f"QLA_{LIB}_M_{var}eq_{fname}_{src}"
                call = lambda nc, opname=opname, fname=fname, p1=p1, gang=gang: (
                    f"qlab::api_map<qlab::{_nc2_op(fname, R) if nc == 2 else f'{opname}<{R}, {nc}>'}>("
                    f"{kid('mfunc')}, r, {opnd(p1, 'a')}, qlab::Opnd{{}}, "
                    f"{gang}, n, qlab::EQ);")
                add(name, [("void *", "r"), ("void *", "a")] + tail + [("int", "n")],
                    _fn_switch(FN_MFUNC_NCS, call, name), "mfunc", CITE["mfunc"],
                    dict(dest="M", eqop="eq", var=var, a=src, fn=fname))
            name = f"QLA_{LIB}_C_{var}eq_det_{src}"
            call = lambda nc, p1=p1, gang=gang: (
                f"qlab::api_map<qlab::{_nc2_op('det', R) if nc == 2 else f'GenDetOp<{R}, {nc}>'}>({kid('mfunc')}, r, "
                f"{opnd(p1, 'a')}, qlab::Opnd{{}}, {gang}, n, qlab::EQ);")
            add(name, [(f"QLA_{prec}_Complex *", "r"), ("void *", "a")] + tail + [("int", "n")],
                _fn_switch(FN_MFUNC_NCS, call, name), "mfunc", CITE["mfunc"],
                dict(dest="C", eqop="eq", var=var, a=src, fn="det"))
            # the remaining matrix functions: the Nc = 3 closed forms at nc = 3,
            # the templates' generic paths otherwise
            for fname, opf in FN_MFUNC_EXT.items():
                name = f"QLA_{LIB}_M_{var}eq_{fname}_{src}"
                call = lambda nc, opf=opf, p1=p1, gang=gang: (
                    f"qlab::api_map<qlab::{opf(nc).replace('float', R)}>({kid('mfunc_ext')}, r, {opnd(p1, 'a')}, "
                    f"qlab::Opnd{{}}, "
                    f"{gang}, n, qlab::EQ);")
                add(name, [("void *", "r"), ("void *", "a")] + tail + [("int", "n")],
                    _fn_switch(FN_MFUNC_NCS, call, name), "mfunc_ext", CITE["mfunc_ext"],
                    dict(dest="M", eqop="eq", var=var, a=src, fn=fname))
            for fname, opn, herm in (("eigenvals", "EigenvalsOp", "false"), ("eigenvalsH", "EigenvalsHOp", "true")):
                name = f"QLA_{LIB}_V_{var}eq_{fname}_{src}"
                call = lambda nc, opn=opn, herm=herm, fname=fname, p1=p1, gang=gang: (
                    f"qlab::api_map<qlab::"
                    f"{_nc2_op(fname, R) if nc == 2 else opn + '<' + R + '>' if nc == 3 else f'GenEigenOp<{R}, {nc}, {herm}>'}>("
                    f"{kid('mfunc_ext')}, r, {opnd(p1, 'a')}, qlab::Opnd{{}}, {gang}, n, qlab::EQ);")
                add(name, [("void *", "r"), ("void *", "a")] + tail + [("int", "n")],
                    _fn_switch(FN_MFUNC_NCS, call, name), "mfunc_ext", CITE["mfunc_ext"],
                    dict(dest="V", eqop="eq", var=var, a=src, fn=fname))
        for T_ in ("V", "M"):
            for s1, p1 in (("M", False), ("pM", True)):
                for s2, p2 in ((T_, False), ("p" + T_, True)):
                    name = f"QLA_{LIB}_{T_}_{var}eq_{s1}_inverse_{s2}"
                    call = lambda nc, T_=T_, p1=p1, p2=p2, gang=gang: (
                        f"qlab::api_map<qlab::"
                        f"{f'Nc2MInverseOp<{R}, ' if nc == 2 else f'GenMInverseOp<{R}, {nc}, '}{1 if T_ == 'V' else nc}>>("
                        f"{kid('minv')}, r, {opnd(p1, 'a')}, {opnd(p2, 'b')}, {gang}, n, qlab::EQ);")
                    add(name, [("void *", "r"), ("void *", "a"), ("void *", "b")] + tail + [("int", "n")],
                        _fn_switch(FN_MFUNC_NCS, call, name), "mfunc_ext", CITE["minv"],
                        dict(dest=T_, eqop="eq", var=var, a=s1, b=s2, fn="inverse_" + T_))
    # fused hop terms: the fixed-colour generator's entry points with the
    # colour count of the op templates switched over the compiled nc
    src_pc = "F3" if prec == "F" else "D3"
    for fn in gen_pc(src_pc, R, prec):
        if fn.family != "hop":
            continue
        name = fn.name.replace(f"QLA_{src_pc}_", f"QLA_{LIB}_", 1)
        params = [(("void *", nm) if re.search(r"QLA_[FD]3_", t) else (t, nm)) for t, nm in fn.params]
        guard, call = fn.body.split("\n  ", 1)
        call = call.replace(f'"{src_pc}_', f'"{LIB}_')
        call_of_nc = lambda nc, call=call: re.sub(  # noqa: E731
            r"(Sp\w+Op<\w+), 3([,>])", lambda m: f"{m.group(1)}, {nc}{m.group(2)}", call)
        add(name, params, guard + "\n  " + _fn_switch(FN_NCS, call_of_nc, name), "hop", fn.cite, fn.kinds)
    return fns


# record length at nc colours for the record lengths of the fixed-colour generator
NE_AT_NC = {"1": "1", "3": "nc", "6": "2 * nc", "12": "4 * nc", "9": "nc * nc", "144": "16 * nc * nc"}


def _ncolor_body(body):
    """The run-time-nc call (qla_ncolor.cuh) for a fixed-colour body of
    gen_ewise / gen_sitefield."""
    m = re.match(r"qlab::(api_\w+)<([^>]*)>\((\"[^\"]*\"), (.*)\);$", body, re.S)
    api, targs, kid, rest = m.group(1), [t.strip() for t in m.group(2).split(",")], m.group(3), m.group(4)
    kid = re.sub(r'"(F3|D3)_', lambda mm: '"' + mm.group(1)[0] + "N_", kid)
    ne = lambda t: NE_AT_NC[t]  # noqa: E731
    if api == "api_ew":
        R_, NE_, SH, PERM, SC, SRE = targs
        return f"qlab::api_ew_n<{R_}, {SH}, {SC}, {SRE}>({kid}, nc, {ne(NE_)}, {PERM}, {rest});"
    if api == "api_ldot":
        R_, NE_, KIND, PERM = targs
        return f"qlab::api_ldot_n<{R_}, {KIND}>({kid}, nc, {ne(NE_)}, {PERM}, {rest});"
    if api in ("api_outer", "api_diagfill", "api_antiherm"):
        return f"qlab::{api}_n<{targs[0]}>({kid}, nc, {rest});"
    if api in ("api_fill", "api_zero", "api_mask"):
        return f"qlab::{api}_n<{targs[0]}>({kid}, nc, {ne(targs[1])}, {rest});"
    if api == "api_sub":
        return f"qlab::api_sub_n<{targs[0]}>({kid}, nc, {rest});"
    if api == "api_gamma":
        return f"qlab::api_gamma_n<{targs[0]}, {targs[2]}>({kid}, nc, {ne(targs[1])}, {rest});"
    if api == "api_trace":
        return f"qlab::api_trace_n<{targs[0]}, {targs[1]}>({kid}, nc, {rest});"
    if api == "api_gdot":
        R_, NE_, KIND, PERM, OUT = targs
        return f"qlab::api_gdot_n<{R_}, {KIND}, {OUT}>({kid}, nc, {ne(NE_)}, {PERM}, {rest});"
    if api == "api_gsum":
        out = targs[2] if len(targs) > 2 else targs[0]
        return f"qlab::api_gsum_n<{targs[0]}, {out}>({kid}, nc, {ne(targs[1])}, {rest});"
    if api == "api_convert":
        return f"qlab::api_convert_n<{targs[0]}, {targs[1]}>({kid}, nc, {ne(targs[2])}, {rest});"
    if api == "api_prop":
        return f"qlab::api_prop_n<{', '.join(targs)}>({kid}, nc, {rest});"
    if api == "api_rng_fill":
        return f"qlab::api_rng_fill_n<{targs[0]}>({kid}, nc, {ne(targs[1])}, {rest});"
    if api == "api_multi":
        return f"qlab::api_multi_n<{', '.join(targs)}>({kid}, nc, {rest});"
    raise ValueError(api)


def gen_fn_wide(prec):
    """The element-wise, site-local product, fill / component / gamma /
    trace, global P / adjoint-form reduction, global sum and (for F)
    precision-conversion families of QLA_FN_ / QLA_DFN_ / QLA_FDN_ (prec "F")
    or QLA_DN_ (prec "D"): the entry points of gen_ewise and gen_sitefield
    with a leading int nc, record arguments as void * (the reference's
    variably sized records) and the run-time-nc kernels of qla_ncolor.cuh."""
    src_pc = "F3" if prec == "F" else "D3"
    R = "float" if prec == "F" else "double"
    fns = []
    props = [fn for fn in gen_pc(src_pc, R, prec) if fn.family in ("prop", "multi")]
    for fn in gen_ewise(src_pc, R, prec) + gen_sitefield(src_pc, R, prec) + props:
        m = re.match(r"QLA_(F3|D3|DF3|FD3)_(.*)$", fn.name)
        lib = {"F3": "FN", "D3": "DN", "DF3": "DFN", "FD3": "FDN"}[m.group(1)]
        params = [("int", "nc")]
        for t, nm in fn.params:
            params.append(("void *", nm) if re.search(r"QLA_[FD]3_", t) else (t, nm))
        fns.append(Fn(f"QLA_{lib}_{m.group(2)}", params, _ncolor_body(fn.body), fn.family, fn.cite, fn.kinds))
    return fns


def gen_two(prec):
    """QLA_F2_ / QLA_DF2_ / QLA_FD2_ (prec "F") or QLA_D2_ (prec "D"): the
    two-colour libraries, with the fixed-colour libraries' names and record
    types (QLA_F2_ColorMatrix ...) and the N-colour implementations at nc = 2."""
    src_pc, R = ("F3", "float") if prec == "F" else ("D3", "double")
    twins = {fn.name: fn for fn in gen_pc(src_pc, R, prec)}
    fns = []
    for fn in gen_fn(prec) + gen_fn_wide(prec):
        m = re.match(r"QLA_(FN|DN|DFN|FDN)_(.*)$", fn.name)
        lib3 = {"FN": "F3", "DN": "D3", "DFN": "DF3", "FDN": "FD3"}[m.group(1)]
        lib2 = {"FN": "F2", "DN": "D2", "DFN": "DF2", "FDN": "FD2"}[m.group(1)]
        twin = twins[f"QLA_{lib3}_{m.group(2)}"]
        params = [(re.sub(r"QLA_([FD])3_", r"QLA_\g<1>2_", t), nm) for t, nm in twin.params]
        body = fn.body
        if "switch (nc)" in body:
            # compiled-colour families: keep the nc = 2 instantiation
            head = body[:body.index("switch (nc)")]
            case2 = re.search(r"case 2: (.*?) break;\n", body)
            if case2:
                body = head + case2.group(1)
            else:
                body = (head + f'qlab::set_error(QLAGPU_ERR_ARG, "QLA_{lib2}_{m.group(2)}", '
                        '"not built for two colours");')
        else:
            body = re.sub(r"\bnc\b", "2", body)
        body = re.sub(r'"(FN|DN)_', lambda mm: '"' + mm.group(1)[0] + "2_", body)
        fns.append(Fn(f"QLA_{lib2}_{m.group(2)}", params, body, fn.family, fn.cite, fn.kinds))
    return fns


def gen_int():
    """QLA_I_ entry points: the (shape x eqop x indexing) set of the reference's
    integer library."""
    fns = []
    kid = '"I_int"'

    def field(name, ptr):
        if ptr:
            return ("QLA_Int *RESTRICT *", name), f"qlab::op_ptr((const void* const*){name})"
        return ("QLA_Int *RESTRICT", name), f"qlab::op_contig({name})"

    def emit(shape, var, eq, code, fields, scalar):
        name = f"QLA_I_{var}{eq}_{shape}"
        params = [("QLA_Int *RESTRICT", "r")]
        if scalar:
            params.append(("QLA_Int *RESTRICT", "a"))
        ops = []
        for fname_, ptr in fields:
            pp, oo = field(fname_, ptr)
            params.append(pp)
            ops.append(oo)
        if var == "x":
            params.append(("int *", "index"))
        params.append(("int", "n"))
        while len(ops) < 3:
            ops.append("qlab::Opnd{}")
        body = (f"qlab::api_int({kid}, qlab::{code}, {EQ_ENUM[eq]}, (int*)r, {'(const int*)a' if scalar else 'nullptr'}, "
                f"{ops[0]}, {ops[1]}, {ops[2]}, {len(fields)}, {'index' if var == 'x' else 'nullptr'}, n);")
        fns.append(Fn(name, params, body, "int", CITE["int"], dict(dest="I", eqop=eq, var=var, shape=shape)))

    P = [("", False), ("p", True)]
    for var in ["v", "x"]:
        for eq in EQOPS:
            for pa, xa in P:
                emit(f"{pa}I", var, eq, "IC_COPY", [("a", xa)], False)
                for pb, xb in P:
                    emit(f"{pa}I_times_{pb}I", var, eq, "IC_TIMES", [("a", xa), ("b", xb)], False)
                emit(f"i_times_{pa}I", var, eq, "IC_S_TIMES", [("b", xa)], True)
            emit("i", var, eq, "IC_S", [], True)
        for opn, code in INT_BINOPS.items():
            for pa, xa in P:
                for pb, xb in P:
                    emit(f"{pa}I_{opn}_{pb}I", var, "eq", code, [("a", xa), ("b", xb)], False)
        for pa, xa in P:
            for pm in ("plus", "minus"):
                for pb, xb in P:
                    emit(f"i_times_{pa}I_{pm}_{pb}I", var, "eq", "IC_S_TIMES_PLUS" if pm == "plus" else
                         "IC_S_TIMES_MINUS", [("b", xa), ("c", xb)], True)
            emit(f"not_{pa}I", var, "eq", "IC_NOT", [("a", xa)], False)
        emit("zero", var, "eq", "IC_ZERO", [], False)
    # random-number state fields: copies, masked copies, seeding
    kid_s = '"S_state"'
    for var in ["v", "x"]:
        tail = [("int *", "index")] if var == "x" else []
        gang = "index" if var == "x" else "nullptr"
        for pa, xa in P:
            sa = ("QLA_RandomState *RESTRICT *" if xa else "QLA_RandomState *RESTRICT", "a")
            oa = "qlab::op_ptr((const void* const*)a)" if xa else "qlab::op_contig(a)"
            fns.append(Fn(f"QLA_S_{var}eq_{pa}S", [("QLA_RandomState *RESTRICT", "r"), sa] + tail + [("int", "n")],
                          f"qlab::api_rng_copy({kid_s}, r, {oa}, qlab::Opnd{{}}, false, {gang}, n);", "random",
                          CITE["random"], dict(dest="S", eqop="eq", var=var, op="copy", a=pa + "S")))
            for pm, xm in P:
                sm = ("QLA_Int *RESTRICT *" if xm else "QLA_Int *RESTRICT", "b")
                om = "qlab::op_ptr((const void* const*)b)" if xm else "qlab::op_contig(b)"
                fns.append(Fn(f"QLA_S_{var}eq_{pa}S_mask_{pm}I",
                              [("QLA_RandomState *RESTRICT", "r"), sa, sm] + tail + [("int", "n")],
                              f"qlab::api_rng_copy({kid_s}, r, {oa}, {om}, true, {gang}, n);", "random",
                              CITE["random"], dict(dest="S", eqop="eq", var=var, op="mask", a=pa + "S", b=pm + "I")))
            si = ("QLA_Int *RESTRICT *" if xa else "QLA_Int *RESTRICT", "a")
            fns.append(Fn(f"QLA_S_{var}eq_seed_i_{pa}I",
                          [("QLA_RandomState *RESTRICT", "r"), ("int", "seed"), si] + tail + [("int", "n")],
                          f"qlab::api_rng_seed({kid_s}, r, seed, {oa}, {gang}, n);", "random", CITE["random"],
                          dict(dest="S", eqop="eq", var=var, op="seed", a=pa + "I")))
    return fns


# QLA_F_ / QLA_D_ entry points: (dest, name pattern, operands, all eqops?, plan, spec).
# Operands are (parameter, letter): R / C / I fields (each with a pointer form
# `p`), or the constants "r" / "c" passed by pointer.  {a} {b} {c} in the
# pattern stand for the field operands' names (with `p` for pointer forms).
_UNARY_R = ["sin", "cos", "tan", "asin", "acos", "atan", "sqrt", "fabs", "exp", "log", "log10", "sinh", "cosh",
            "tanh", "ceil", "floor", "sign"]
FD_TABLE = (
    [("C", "{a}", [("a", "C")], True, "ew", ("COPY", 0)),
     ("C", "{a}a", [("a", "C")], True, "ew", ("CONJ", 0)),
     ("C", "i_{a}", [("a", "C")], True, "ew", ("I", 0)),
     ("C", "c", [("a", "c")], True, "fill", None),
     ("C", "zero", [], False, "zero", None),
     ("C", "{a}_mask_{b}", [("a", "C"), ("b", "I")], False, "mask", None),
     ("C", "{a}", [("a", "R")], False, "scalar", "SO_C_FROM_R"),
     ("C", "{a}_plus_i_{b}", [("a", "R"), ("b", "R")], False, "scalar", "SO_C_R_PLUS_I_R"),
     ("C", "{a}_times_{b}", [("a", "C"), ("b", "C")], True, "ew", ("CT", 2)),
     ("C", "{a}_times_{b}a", [("a", "C"), ("b", "C")], True, "ew", ("CTA", 2)),
     ("C", "{a}a_times_{b}", [("a", "C"), ("b", "C")], True, "ew", ("CAT", 2)),
     ("C", "{a}a_times_{b}a", [("a", "C"), ("b", "C")], True, "ew", ("CATA", 2)),
     ("C", "{a}_times_{b}", [("a", "R"), ("b", "C")], True, "ew", ("RT", 3)),
     ("C", "{a}_times_{b}a", [("a", "R"), ("b", "C")], True, "ew", ("RTA", 3)),
     ("C", "c_times_{b}", [("a", "c"), ("b", "C")], True, "ew", ("CT", 1)),
     ("C", "c_times_{b}a", [("a", "c"), ("b", "C")], True, "ew", ("CTA", 1)),
     ("C", "r_times_{b}", [("a", "r"), ("b", "C")], True, "ew", ("RT", 1)),
     ("C", "r_times_{b}a", [("a", "r"), ("b", "C")], True, "ew", ("RTA", 1)),
     ("C", "{a}_plus_{b}", [("a", "C"), ("b", "C")], False, "ew", ("PLUS", 0)),
     ("C", "{a}_minus_{b}", [("a", "C"), ("b", "C")], False, "ew", ("MINUS", 0)),
     ("C", "c_times_{b}_plus_{c}", [("a", "c"), ("b", "C"), ("c", "C")], False, "ew", ("CT_PLUS", 1)),
     ("C", "c_times_{b}_minus_{c}", [("a", "c"), ("b", "C"), ("c", "C")], False, "ew", ("CT_MINUS", 1)),
     ("C", "r_times_{b}_plus_{c}", [("a", "r"), ("b", "C"), ("c", "C")], False, "ew", ("RT_PLUS", 1)),
     ("C", "r_times_{b}_minus_{c}", [("a", "r"), ("b", "C"), ("c", "C")], False, "ew", ("RT_MINUS", 1)),
     ("C", "{a}_divide_{b}", [("a", "C"), ("b", "C")], False, "scalar", "SO_C_DIVIDE"),
     ("C", "{a}_dot_{b}", [("a", "C"), ("b", "C")], True, "ldot", "LD_DOT"),
     ("C", "{a}_dot_{b}a", [("a", "C"), ("b", "C")], True, "ldot", "LD_DOT_AA"),
     ("C", "{a}a_dot_{b}", [("a", "C"), ("b", "C")], True, "ldot", "LD_ADOT"),
     ("C", "cexp_{a}", [("a", "C")], False, "scalar", "SO_C_CEXP"),
     ("C", "clog_{a}", [("a", "C")], False, "scalar", "SO_C_CLOG"),
     ("C", "csqrt_{a}", [("a", "C")], False, "scalar", "SO_C_CSQRT"),
     ("C", "cexpi_{a}", [("a", "R")], False, "scalar", "SO_C_CEXPI"),
     ("R", "{a}", [("a", "R")], True, "scalar", "SO_R_COPY"),
     ("R", "{a}", [("a", "I")], False, "scalar", "SO_R_FROM_I"),
     ("R", "r", [("a", "r")], True, "scalar", "SO_R_FILL"),
     ("R", "zero", [], False, "scalar", "SO_R_ZERO"),
     ("R", "{a}_mask_{b}", [("a", "R"), ("b", "I")], False, "scalar", "SO_R_MASK"),
     ("R", "{a}_times_{b}", [("a", "R"), ("b", "R")], True, "scalar", "SO_R_TIMES_R"),
     ("R", "r_times_{b}", [("a", "r"), ("b", "R")], True, "scalar", "SO_R_RTIMES"),
     ("R", "r_times_{b}_plus_{c}", [("a", "r"), ("b", "R"), ("c", "R")], False, "scalar", "SO_R_RT_PLUS"),
     ("R", "r_times_{b}_minus_{c}", [("a", "r"), ("b", "R"), ("c", "R")], False, "scalar", "SO_R_RT_MINUS"),
     ("R", "{a}_ldexp_{b}", [("a", "R"), ("b", "I")], False, "scalar", "SO_R_LDEXP")]
    + [("R", "{a}_" + op + "_{b}", [("a", "R"), ("b", "R")], False, "scalar", "SO_R_" + op.upper())
       for op in ("plus", "minus", "divide", "max", "min", "mod", "pow", "atan2")]
    + [("R", f + "_{a}", [("a", "R")], False, "scalar", "SO_R_" + f.upper()) for f in _UNARY_R]
    + [("R", f + "_{a}", [("a", "C")], False, "scalar", "SO_R_" + f.upper()) for f in ("re", "im", "norm", "arg")]
    + [("R", "norm2_{a}", [("a", "C")], True, "ldot", "LD_NORM2"),
       ("R", "re_{a}_dot_{b}", [("a", "C"), ("b", "C")], True, "ldot", "LD_REDOT")]
    + [("I", "{a}_" + op + "_{b}", [("a", "R"), ("b", "R")], False, "scalar", "SO_I_" + op.upper())
       for op in ("eq", "ge", "gt", "le", "lt", "ne")]
    + [("I", "round_{a}", [("a", "R")], False, "scalar", "SO_I_ROUND"),
       ("I", "trunc_{a}", [("a", "R")], False, "scalar", "SO_I_TRUNC")]
    # global reductions and sums (lower-case destination)
    + [("c", "{a}_dot_{b}", [("a", "C"), ("b", "C")], False, "gdot", "LD_DOT"),
       ("c", "{a}a_dot_{b}", [("a", "C"), ("b", "C")], False, "gdot", "LD_ADOT"),
       ("c", "sum_{a}", [("a", "C")], False, "gsum", None),
       ("r", "{a}_dot_{b}", [("a", "R"), ("b", "R")], False, "sred", "SR_DOT"),
       ("r", "{a}_dot_{b}", [("a", "I"), ("b", "I")], False, "sred", "SR_DOT"),
       ("r", "norm2_{a}", [("a", "C")], False, "gdot", "LD_NORM2"),
       ("r", "norm2_{a}", [("a", "R")], False, "sred", "SR_NORM2"),
       ("r", "norm2_{a}", [("a", "I")], False, "sred", "SR_NORM2"),
       ("r", "re_{a}_dot_{b}", [("a", "C"), ("b", "C")], False, "gdot", "LD_REDOT"),
       ("r", "sum_{a}", [("a", "R")], False, "sred", "SR_SUM"),
       ("r", "sum_{a}", [("a", "I")], False, "sred", "SR_SUM")])

# QLA_DF_ reductions of float fields returned in double
DF_TABLE = [row for row in FD_TABLE if row[0] in "cr" and "I" not in [l for _, l in row[2]]]


def _fd_entries(lib, table, R, RW, OUT, prec_in, prec_out):
    """Entry points of `table` for library `lib` (F, D or DF): field elements
    of type R (precision prec_in), results in prec_out (OUT for globals)."""
    fns = []
    kid = lambda fam: f'"{lib}_{fam}"'  # noqa: E731
    ftype = {"R": f"QLA_{prec_in}_Real", "C": f"QLA_{prec_in}_Complex", "I": "QLA_Int"}
    dtype = {"R": f"QLA_{prec_out}_Real", "C": f"QLA_{prec_out}_Complex", "I": "QLA_Int",
             "r": f"QLA_{prec_out}_Real", "c": f"QLA_{prec_out}_Complex"}
    for dest, pat, opnds, alleq, plan, spec in table:
        fields = [(nm, l) for nm, l in opnds if l in "RCI"]
        consts = [(nm, l) for nm, l in opnds if l in "rc"]
        fam = {"ew": "cfield", "fill": "cfield", "zero": "cfield", "mask": "cfield", "ldot": "cfield",
               "gdot": "sglobal", "gsum": "sglobal", "sred": "sglobal"}.get(plan, None)
        if plan == "scalar":
            fam = "cfield" if dest == "C" else "rfield"
        for var in ["v", "x"]:
            tail = [("int *", "index")] if var == "x" else []
            gang = "index" if var == "x" else "nullptr"
            for eq in (EQOPS if alleq else ["eq"]):
                for ptrs in itertools.product((False, True), repeat=len(fields)):
                    tok = {nm: ("p" if pf else "") + l for (nm, l), pf in zip(fields, ptrs)}
                    name = f"QLA_{lib}_{dest}_{var}{eq}_" + pat.format(**{k: tok.get(k, "") for k in "abc"})
                    params = [(f"{dtype[dest]} *RESTRICT", "r")]
                    ops = {}
                    for nm, l in opnds:
                        if l in "rc":
                            params.append((f"{dtype[l]} *RESTRICT", nm))
                        else:
                            pf = tok[nm].startswith("p")
                            params.append((f"{ftype[l]} *RESTRICT *" if pf else f"{ftype[l]} *RESTRICT", nm))
                            ops[nm] = f"qlab::op_ptr((const void* const*){nm})" if pf else f"qlab::op_contig({nm})"
                    params += tail + [("int", "n")]
                    o = lambda nm: ops.get(nm, "qlab::Opnd{}")  # noqa: E731
                    E = EQ_ENUM[eq]
                    if plan == "ew":
                        shape, sk = spec
                        sc = {0: "qlab::SC_NONE", 1: "qlab::SC_CONST", 2: "qlab::SC_FIELD", 3: "qlab::SC_FIELD"}[sk]
                        sreal = "true" if (sk == 3 or (sk == 1 and consts and consts[0][1] == "r")) else "false"
                        if sk == 0:
                            two = shape in ("PLUS", "MINUS")
                            args = f"r, nullptr, qlab::Opnd{{}}, {o('a')}, {o('b') if two else 'qlab::Opnd{}'}"
                        elif sk == 1:
                            args = f"r, a, qlab::Opnd{{}}, {o('b')}, {o('c')}"
                        else:
                            args = f"r, nullptr, {o('a')}, {o('b')}, qlab::Opnd{{}}"
                        body = (f"qlab::api_ew<{R}, 1, qlab::EW_{shape}, qlab::PERM_ID, {sc}, {sreal}>({kid('ew')}, "
                                f"{args}, {gang}, n, {E});")
                    elif plan == "fill":
                        body = f"qlab::api_fill<{R}, 1>({kid('fill')}, r, a, {gang}, n, {E});"
                    elif plan == "zero":
                        body = f"qlab::api_zero<{R}, 1>({kid('fill')}, r, {gang}, n);"
                    elif plan == "mask":
                        body = f"qlab::api_mask<{R}, 1>({kid('mask')}, r, {o('a')}, {o('b')}, {gang}, n);"
                    elif plan == "ldot":
                        body = (f"qlab::api_ldot<{R}, 1, qlab::{spec}, qlab::PERM_ID>({kid('ldot')}, r, {o('a')}, "
                                f"{o('b')}, {gang}, n, {E});")
                    elif plan == "scalar":
                        body = (f"qlab::api_scalar<{R}, qlab::{spec}>({kid('scalar')}, r, "
                                f"{'a' if consts else 'nullptr'}, {o('a') if not consts else 'qlab::Opnd{}'}, "
                                f"{o('b')}, {o('c')}, {gang}, n, {E});")
                    elif plan == "gdot":
                        body = (f"qlab::api_gdot<{R}, 1, qlab::{spec}, qlab::PERM_ID, {OUT}>({kid('gdot')}, r, "
                                f"{o('a')}, {o('b')}, {gang}, n);")
                    elif plan == "gsum":
                        body = f"qlab::api_gsum<{R}, 1, {OUT}>({kid('gsum')}, r, {o('a')}, {gang}, n);"
                    else:  # sred
                        rin = "int" if fields[0][1] == "I" else R
                        body = (f"qlab::api_sred<{rin}, {RW}, qlab::{spec}, {OUT}>({kid('sred')}, r, {o('a')}, "
                                f"{o('b')}, {gang}, n);")
                    kinds = dict(dest=dest, eqop=eq, var=var, plan=plan, spec=spec if not isinstance(spec, tuple)
                                 else list(spec), opnds=[[nm, l] for nm, l in opnds],
                                 **{nm: tok[nm] for nm in tok})
                    fns.append(Fn(name, params, body, fam, CITE["scalar"], kinds))
    return fns


def gen_fd(prec):
    """QLA_F_ / QLA_D_ (real, complex and integer fields): the entry points of
    FD_TABLE, and the uniform and gaussian random fills."""
    R = "float" if prec == "F" else "double"
    fns = _fd_entries(prec, FD_TABLE, R, R, R, prec, prec)
    kid = f'"{prec}_random"'
    for var in ["v", "x"]:
        tail = [("int *", "index")] if var == "x" else []
        gang = "index" if var == "x" else "nullptr"
        for ps, xs in (("", False), ("p", True)):
            sa = ("QLA_RandomState *RESTRICT *" if xs else "QLA_RandomState *RESTRICT", "a")
            oa = "qlab::op_ptr((const void* const*)a)" if xs else "qlab::op_contig(a)"
            for dest, what in (("R", "random"), ("R", "gaussian"), ("C", "gaussian")):
                rt = f"QLA_{prec}_{'Real' if dest == 'R' else 'Complex'} *RESTRICT"
                name = f"QLA_{prec}_{dest}_{var}eq_{what}_{ps}S"
                body = (f"qlab::api_rng_fill<{R}, 1, {str(dest == 'R').lower()}>({kid}, {int(what == 'gaussian')}, r, "
                        f"{oa}, {gang}, n);")
                fns.append(Fn(name, [(rt, "r"), sa] + tail + [("int", "n")], body, "random", CITE["random"],
                              dict(dest=dest, eqop="eq", var=var, op=what, a=ps + "S")))
    if prec == "F":
        fns += gen_df()
    return fns


def gen_df():
    """QLA_DF_ / QLA_FD_: float <-> double conversions of real and complex
    fields, and the global reductions of float fields returned in double."""
    fns = _fd_entries("DF", DF_TABLE, "float", "float", "double", "F", "D")
    for var in ["v", "x"]:
        tail = [("int *", "index")] if var == "x" else []
        gang = "index" if var == "x" else "nullptr"
        for T in ("R", "C"):
            for p1 in (False, True):
                for lib, rin, rout, pin, pout in (("DF", "float", "double", "F", "D"),
                                                  ("FD", "double", "float", "D", "F")):
                    tin = f"QLA_{pin}_{'Real' if T == 'R' else 'Complex'}"
                    tout = f"QLA_{pout}_{'Real' if T == 'R' else 'Complex'}"
                    pa = (f"{tin} *RESTRICT *" if p1 else f"{tin} *RESTRICT", "a")
                    oa = "qlab::op_ptr((const void* const*)a)" if p1 else "qlab::op_contig(a)"
                    name = f"QLA_{lib}_{T}_{var}eq_{'p' if p1 else ''}{T}"
                    if T == "R":
                        body = f"qlab::api_rconvert<{rin}, {rout}>(\"DF_convert\", r, {oa}, {gang}, n);"
                    else:
                        body = f"qlab::api_convert<{rin}, {rout}, 1>(\"DF_convert\", r, {oa}, {gang}, n);"
                    fns.append(Fn(name, [(f"{tout} *RESTRICT", "r"), pa] + tail + [("int", "n")], body, "convert",
                                  CITE["scalar"], dict(dest=T, eqop="eq", var=var, a=("p" if p1 else "") + T,
                                                       lib=lib)))
    return fns


class Fn:
    def __init__(self, name, params, body, family, cite, kinds):
        self.name = name
        self.params = params    # list of (ctype, name)
        self.body = body
        self.family = family
        self.cite = cite
        self.kinds = kinds      # argument kinds for the Python mirror / tests

    def proto(self, restrict):
        ps = ", ".join(t.replace("RESTRICT", restrict) + " " + n for t, n in self.params)
        return f"void {self.name}({ps})"


def ptype(pc, t):
    return f"QLA_{pc}_{REC[t][0]}"


def operand(pc, t, ptr, argname, restrict="RESTRICT"):
    """C parameter and engine operand descriptor for a field operand."""
    ct = ptype(pc, t)
    if ptr:
        return (f"{ct} *RESTRICT *", argname), f"qlab::op_ptr((const void* const*){argname})"
    return (f"{ct} *RESTRICT", argname), f"qlab::op_contig({argname})"


def gen_pc(pc, R, P):
    """Generate the hot families for colour-3 precision pc (F3/D3)."""
    fns = []
    kid = lambda fam: f'"{pc}_{fam}"'
    # ---- left multiplication by a colour matrix
    for T in FIELD_TYPES:
        ncol = REC[T][1]
        src2s = [(T, False), ("p" + T, True)]
        if T == "M":
            src2s += [("Ma", False), ("pMa", True)]
        for var in ["v", "x"]:
            for eq in EQOPS:
                for s1 in ["M", "Ma", "pM", "pMa"]:
                    adja = "a" in s1[-1:]
                    p1 = s1.startswith("p")
                    for s2name, p2 in src2s:
                        adjb = s2name.endswith("a")
                        name = f"QLA_{pc}_{T}_{var}{eq}_{s1}_times_{s2name}"
                        pr = (f"{ptype(pc, T)} *RESTRICT", "r")
                        pa, oa = operand(pc, "M", p1, "a")
                        pb, ob = operand(pc, T, p2, "b")
                        params = [pr, pa, pb]
                        gang = "nullptr"
                        if var == "x":
                            params.append(("int *", "index"))
                            gang = "index"
                        params.append(("int", "n"))
                        op = f"qlab::LMultOp<{R}, 3, {ncol}, {str(adja).lower()}, {str(adjb).lower()}>"
                        body = (f"qlab::api_map<{op}>({kid('lmult_' + T + str(int(adja)) + str(int(adjb)))}, r, "
                                f"{oa}, {ob}, {gang}, n, {EQ_ENUM[eq]});")
                        fns.append(Fn(name, params, body, "lmult", CITE["lmult"],
                                      dict(dest=T, eqop=eq, var=var, a=s1, b=s2name)))
            # per-operand int32 index on the field operand (doc variant 5)
        for eq in EQOPS:
            for s1 in ["M", "Ma"]:
                adja = s1 == "Ma"
                name = f"QLA_{pc}_{T}_{eq}_{s1}_times_x{T}"
                params = [(f"{ptype(pc, T)} *RESTRICT", "r"), (f"{ptype(pc, 'M')} *RESTRICT", "a"),
                          (f"{ptype(pc, T)} *RESTRICT", "b"), ("int *", "jb"), ("int", "n")]
                op = f"qlab::LMultOp<{R}, 3, {ncol}, {str(adja).lower()}, false>"
                body = (f"qlab::api_map<{op}>({kid('lmult_' + T + str(int(adja)) + '0')}, r, qlab::op_contig(a), "
                        f"qlab::op_idx(b, jb), nullptr, n, {EQ_ENUM[eq]});")
                fns.append(Fn(name, params, body, "lmult", CITE["lmult_x"],
                              dict(dest=T, eqop=eq, var="xb", a=s1, b="x" + T)))
    # ---- spin projection / reconstruction
    for var in ["v", "x"]:
        for eq in EQOPS:
            for src, p1 in [("D", False), ("pD", True)]:
                name = f"QLA_{pc}_H_{var}{eq}_spproj_{src}"
                pa, oa = operand(pc, "D", p1, "a")
                params = [(f"{ptype(pc, 'H')} *RESTRICT", "r"), pa, ("int", "mu"), ("int", "sign")]
                gang = "nullptr"
                if var == "x":
                    params.append(("int *", "index"))
                    gang = "index"
                params.append(("int", "n"))
                body = ("if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */\n  "
                        f"qlab::api_map<qlab::SpprojOp<{R}, 3>>({kid('spproj')}, r, {oa}, qlab::Opnd{{}}, {gang}, n, "
                        f"{EQ_ENUM[eq]}, mu, sign);")
                fns.append(Fn(name, params, body, "spproj", CITE["spproj"], dict(eqop=eq, var=var, a=src)))
            for src, p1 in [("H", False), ("pH", True)]:
                name = f"QLA_{pc}_D_{var}{eq}_sprecon_{src}"
                pa, oa = operand(pc, "H", p1, "a")
                params = [(f"{ptype(pc, 'D')} *RESTRICT", "r"), pa, ("int", "mu"), ("int", "sign")]
                gang = "nullptr"
                if var == "x":
                    params.append(("int *", "index"))
                    gang = "index"
                params.append(("int", "n"))
                body = ("if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */\n  "
                        f"qlab::api_map<qlab::SpreconOp<{R}, 3>>({kid('sprecon')}, r, {oa}, qlab::Opnd{{}}, {gang}, "
                        f"n, {EQ_ENUM[eq]}, mu, sign);")
                fns.append(Fn(name, params, body, "sprecon", CITE["sprecon"], dict(eqop=eq, var=var, a=src)))
    # ---- DiracPropagator products and spin trace
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        tail = [("int *", "index")] if var == "x" else []
        for eq in EQOPS:
            pairs = []
            for ta in ["M", "Ma", "pM", "pMa"]:
                for tb in ["P", "Pa", "pP", "pPa"]:
                    pairs.append((ta, tb, "PK_MP"))
            for ta in ["P", "Pa", "pP", "pPa"]:
                for tb in ["M", "Ma", "pM", "pMa"]:
                    pairs.append((ta, tb, "PK_PM"))
                for tb in ["P", "Pa", "pP", "pPa"]:
                    pairs.append((ta, tb, "PK_PP"))
            for ta, tb, kind in pairs:
                name = f"QLA_{pc}_P_{var}{eq}_{ta}_times_{tb}"
                pa, oa = operand(pc, ta.strip("p").rstrip("a"), ta.startswith("p"), "a")
                pb, ob = operand(pc, tb.strip("p").rstrip("a"), tb.startswith("p"), "b")
                ca, cb = str(ta.endswith("a")).lower(), str(tb.endswith("a")).lower()
                params = [(f"{ptype(pc, 'P')} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                body = (f"qlab::api_prop<{R}, qlab::{kind}, {ca}, {cb}>({kid('prop')}, r, {oa}, {ob}, {gang}, n, "
                        f"{EQ_ENUM[eq]});")
                fns.append(Fn(name, params, body, "prop", CITE["prop"], dict(dest="P", eqop=eq, var=var, a=ta, b=tb)))
            for src, p1 in ([("P", False), ("pP", True)] if eq == "eq" else []):
                name = f"QLA_{pc}_M_{var}{eq}_spintrace_{src}"
                pa, oa = operand(pc, "P", p1, "a")
                params = [(f"{ptype(pc, 'M')} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                body = (f"qlab::api_prop<{R}, qlab::PK_TRACE, false, false>({kid('prop')}, r, {oa}, qlab::Opnd{{}}, "
                        f"{gang}, n, {EQ_ENUM[eq]});")
                fns.append(Fn(name, params, body, "prop", CITE["prop"], dict(dest="M", eqop=eq, var=var, a=src)))
    # ---- multi-direction accumulation r (eqop) sum_d a_d * b_d
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        tail = [("int *", "index")] if var == "x" else []
        for eq in EQOPS:
            for s1 in ["nM", "nMa", "npM", "npMa"]:
                adja = str(s1.endswith("a")).lower()
                pa = "p" in s1
                for s2 in ["nV", "npV"]:
                    pb = "p" in s2
                    name = f"QLA_{pc}_V_{var}{eq}_{s1}_times_{s2}"
                    params = [(f"{ptype(pc, 'V')} *RESTRICT", "r"),
                              (f"{ptype(pc, 'M')} *RESTRICT {'**' if pa else '*'}", "a"),
                              (f"{ptype(pc, 'V')} *RESTRICT {'**' if pb else '*'}", "b")] + tail + \
                        [("int", "n"), ("int", "nd")]
                    body = (f"qlab::api_multi<{R}, {adja}>({kid('multi')}, r, (const void*)a, {str(pa).lower()}, "
                            f"(const void*)b, {str(pb).lower()}, {gang}, n, nd, {EQ_ENUM[eq]});")
                    fns.append(Fn(name, params, body, "multi", CITE["multi"],
                                  dict(dest="V", eqop=eq, var=var, a=s1, b=s2)))
    # ---- fused spin projection x colour matrix (Wilson hop terms)
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        tail = [("int *", "index")] if var == "x" else []
        for eq in EQOPS:
            for s1 in ["M", "Ma", "pM", "pMa"]:
                adja = str(s1.endswith("a")).lower()
                pa, oa = operand(pc, "M", s1.startswith("p"), "a")
                for dest, src, opname in (("H", "D", f"SpprojMultOp<{R}, 3, {adja}, 2>"),
                                          ("D", "D", f"SpprojMultOp<{R}, 3, {adja}, 4>"),
                                          ("D", "H", f"SpreconMultOp<{R}, 3, {adja}>")):
                    kind = "sprecon" if src == "H" else "spproj"
                    for sname, p2 in [(src, False), ("p" + src, True)]:
                        name = f"QLA_{pc}_{dest}_{var}{eq}_{kind}_{s1}_times_{sname}"
                        pb, ob = operand(pc, src, p2, "b")
                        params = [(f"{ptype(pc, dest)} *RESTRICT", "r"), pa, pb, ("int", "mu"),
                                  ("int", "sign")] + tail + [("int", "n")]
                        body = ("if (mu < 0 || mu > 4) return;  /* the reference's switch has no default */\n  "
                                f"qlab::api_map<qlab::{opname}>({kid('hop_' + dest + kind + adja)}, r, {oa}, {ob}, "
                                f"{gang}, n, {EQ_ENUM[eq]}, mu, sign);")
                        fns.append(Fn(name, params, body, "hop", CITE["hop"],
                                      dict(dest=dest, eqop=eq, var=var, a=s1, b=sname, kind=kind)))
            for sname, p1 in [("D", False), ("pD", True)]:
                name = f"QLA_{pc}_D_{var}{eq}_spproj_{sname}"
                pa, oa = operand(pc, "D", p1, "a")
                params = [(f"{ptype(pc, 'D')} *RESTRICT", "r"), pa, ("int", "mu"), ("int", "sign")] + tail + \
                    [("int", "n")]
                body = ("if (mu < 0 || mu > 4) return;\n  "
                        f"qlab::api_map<qlab::SpprojDOp<{R}, 3>>({kid('hop_Dspproj')}, r, {oa}, qlab::Opnd{{}}, "
                        f"{gang}, n, {EQ_ENUM[eq]}, mu, sign);")
                fns.append(Fn(name, params, body, "hop", CITE["hop"], dict(dest="D", eqop=eq, var=var, a=sname,
                                                                           kind="spproj")))
    for eq in EQOPS:
        for s1 in ["M", "Ma"]:
            adja = str(s1 == "Ma").lower()
            for dest, src, opname in (("H", "D", f"SpprojMultOp<{R}, 3, {adja}, 2>"),
                                      ("D", "D", f"SpprojMultOp<{R}, 3, {adja}, 4>"),
                                      ("D", "H", f"SpreconMultOp<{R}, 3, {adja}>")):
                kind = "sprecon" if src == "H" else "spproj"
                name = f"QLA_{pc}_{dest}_{eq}_{kind}_{s1}_times_x{src}"
                params = [(f"{ptype(pc, dest)} *RESTRICT", "r"), (f"{ptype(pc, 'M')} *RESTRICT", "a"),
                          (f"{ptype(pc, src)} *RESTRICT", "b"), ("int *", "jb"), ("int", "mu"), ("int", "sign"),
                          ("int", "n")]
                body = ("if (mu < 0 || mu > 4) return;\n  "
                        f"qlab::api_map<qlab::{opname}>({kid('hop_' + dest + kind + adja)}, r, qlab::op_contig(a), "
                        f"qlab::op_idx(b, jb), nullptr, n, {EQ_ENUM[eq]}, mu, sign);")
                fns.append(Fn(name, params, body, "hop", CITE["hop_x"],
                              dict(dest=dest, eqop=eq, var="xb", a=s1, b="x" + src, kind=kind)))
    # ---- real constant times field, copies / gathers
    for T in FIELD_TYPES:
        nc = REC[T][2]
        for var in ["v", "x"]:
            for eq in EQOPS:
                for src, p1 in [(T, False), ("p" + T, True)]:
                    name = f"QLA_{pc}_{T}_{var}{eq}_r_times_{src}"
                    pb, ob = operand(pc, T, p1, "b")
                    params = [(f"{ptype(pc, T)} *RESTRICT", "r"), (f"QLA_{P}_Real *RESTRICT", "a"), pb]
                    gang = "nullptr"
                    if var == "x":
                        params.append(("int *", "index"))
                        gang = "index"
                    params.append(("int", "n"))
                    body = (f"qlab::api_scalar_map<qlab::RTimesOp<{R}, {nc}>, {R}>({kid('rtimes_' + T)}, r, a, {ob}, "
                            f"{gang}, n, {EQ_ENUM[eq]});")
                    fns.append(Fn(name, params, body, "rtimes", CITE["rtimes"],
                                  dict(dest=T, eqop=eq, var=var, b=src)))
                    name = f"QLA_{pc}_{T}_{var}{eq}_{src}"
                    pa, oa = operand(pc, T, p1, "a")
                    params = [(f"{ptype(pc, T)} *RESTRICT", "r"), pa]
                    if var == "x":
                        params.append(("int *", "index"))
                    params.append(("int", "n"))
                    body = (f"qlab::api_map<qlab::CopyOp<{R}, {nc}>>({kid('copy_' + T)}, r, {oa}, qlab::Opnd{{}}, "
                            f"{gang}, n, {EQ_ENUM[eq]});")
                    fns.append(Fn(name, params, body, "copy", CITE["copy"], dict(dest=T, eqop=eq, var=var, a=src)))
        for eq in EQOPS:
            name = f"QLA_{pc}_{T}_{eq}_x{T}"
            params = [(f"{ptype(pc, T)} *RESTRICT", "r"), (f"{ptype(pc, T)} *RESTRICT", "a"), ("int *", "ja"),
                      ("int", "n")]
            body = (f"qlab::api_map<qlab::CopyOp<{R}, {nc}>>({kid('copy_' + T)}, r, qlab::op_idx(a, ja), "
                    f"qlab::Opnd{{}}, nullptr, n, {EQ_ENUM[eq]});")
            fns.append(Fn(name, params, body, "copy", CITE["copy_x"], dict(dest=T, eqop=eq, var="xa", a="x" + T)))
    # ---- colour-matrix functions
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        for src, p1 in [("M", False), ("pM", True)]:
            pa, oa = operand(pc, "M", p1, "a")
            tail = [("int *", "index")] if var == "x" else []
            for fname, opname in MFUNC_OPS.items():
                name = f"QLA_{pc}_M_{var}eq_{fname}_{src}"
                params = [(f"{ptype(pc, 'M')} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                body = (f"qlab::api_map<qlab::{opname}<{R}>>({kid('mfunc_' + fname)}, r, {oa}, qlab::Opnd{{}}, "
                        f"{gang}, n, qlab::EQ);")
                fns.append(Fn(name, params, body, "mfunc", CITE["mfunc"], dict(dest="M", eqop="eq", var=var, a=src,
                                                                                fn=fname)))
            name = f"QLA_{pc}_C_{var}eq_det_{src}"
            params = [(f"QLA_{P}_Complex *RESTRICT", "r"), pa] + tail + [("int", "n")]
            body = (f"qlab::api_map<qlab::DetOp<{R}>>({kid('mfunc_det')}, r, {oa}, qlab::Opnd{{}}, {gang}, n, "
                    f"qlab::EQ);")
            fns.append(Fn(name, params, body, "mfunc", CITE["mfunc"], dict(dest="C", eqop="eq", var=var, a=src,
                                                                            fn="det")))
    # ---- the remaining matrix functions and the eigenvalues
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        tail = [("int *", "index")] if var == "x" else []
        for src, p1 in [("M", False), ("pM", True)]:
            pa, oa = operand(pc, "M", p1, "a")
            for dest, table in (("M", MFUNC_EXT_OPS), ("V", EIGEN_OPS)):
                for fname, opt in table.items():
                    name = f"QLA_{pc}_{dest}_{var}eq_{fname}_{src}"
                    params = [(f"{ptype(pc, dest)} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                    body = (f"qlab::api_map<qlab::{opt.format(R=R)}>({kid('mfunc_' + fname)}, r, {oa}, "
                            f"qlab::Opnd{{}}, {gang}, n, qlab::EQ);")
                    fns.append(Fn(name, params, body, "mfunc_ext", CITE["mfunc_ext"],
                                  dict(dest=dest, eqop="eq", var=var, a=src, fn=fname)))
    # ---- unitarity reprojection (no counterpart in the reference)
    for var in ["v", "x"]:
        gang = "index" if var == "x" else "nullptr"
        tail = [("int *", "index")] if var == "x" else []
        for src, p1 in [("M", False), ("pM", True)]:
            pa, oa = operand(pc, "M", p1, "a")
            name = f"qlagpu_{pc}_M_{var}eq_reunit_{src}"
            params = [(f"{ptype(pc, 'M')} *RESTRICT", "r"), pa] + tail + [("int", "n")]
            body = (f"qlab::api_map<qlab::ReunitOp<{R}>>({kid('reunit')}, r, {oa}, qlab::Opnd{{}}, {gang}, n, "
                    f"qlab::EQ);")
            fns.append(Fn(name, params, body, "mfunc_ext", CITE["reunit"],
                          dict(dest="M", eqop="eq", var=var, a=src, fn="reunit")))
    # ---- a^-1 b for a ColorVector or ColorMatrix b
    for T, nb in (("V", 1), ("M", 3)):
        for var in ["v", "x"]:
            gang = "index" if var == "x" else "nullptr"
            tail = [("int *", "index")] if var == "x" else []
            for s1, p1 in [("M", False), ("pM", True)]:
                for s2, p2 in [(T, False), ("p" + T, True)]:
                    name = f"QLA_{pc}_{T}_{var}eq_{s1}_inverse_{s2}"
                    pa, oa = operand(pc, "M", p1, "a")
                    pb, ob = operand(pc, T, p2, "b")
                    params = [(f"{ptype(pc, T)} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                    body = (f"qlab::api_map<qlab::MInverseOp<{R}, {nb}>>({kid('minv_' + T)}, r, {oa}, {ob}, "
                            f"{gang}, n, qlab::EQ);")
                    fns.append(Fn(name, params, body, "mfunc_ext", CITE["minv"],
                                  dict(dest=T, eqop="eq", var=var, a=s1, b=s2, fn="inverse_" + T)))
    # ---- global reductions
    red_pcs = [(pc, R, P)]
    if pc == "F3":
        red_pcs.append(("DF3", "float", "D"))
    for rpc, RR, OP in red_pcs:
        outR = "float" if rpc == "F3" else "double"
        for T in FIELD_TYPES:
            nc = REC[T][2]
            for var in ["v", "x"]:
                gang = "index" if var == "x" else "nullptr"
                for src, p1 in [(T, False), ("p" + T, True)]:
                    name = f"QLA_{rpc}_r_{var}eq_norm2_{src}"
                    pa, oa = operand(pc, T, p1, "a")
                    params = [(f"QLA_{OP}_Real *RESTRICT", "r"), pa]
                    if var == "x":
                        params.append(("int *", "index"))
                    params.append(("int", "n"))
                    body = (f"qlab::api_reduce<qlab::Norm2Op<{RR}, {nc}, {outR}>>({kid('norm2_' + T)}, r, "
                            f"sizeof({outR}), {oa}, qlab::Opnd{{}}, {gang}, n);")
                    fns.append(Fn(name, params, body, "norm2", CITE["norm2"], dict(dest="r", var=var, a=src,
                                                                                    out=outR)))
                for sa, pa_ in [(T, False), ("p" + T, True)]:
                    for sb, pb_ in [(T, False), ("p" + T, True)]:
                        name = f"QLA_{rpc}_c_{var}eq_{sa}_dot_{sb}"
                        pa, oa = operand(pc, T, pa_, "a")
                        pb, ob = operand(pc, T, pb_, "b")
                        params = [(f"QLA_{OP}_Complex *RESTRICT", "r"), pa, pb]
                        if var == "x":
                            params.append(("int *", "index"))
                        params.append(("int", "n"))
                        body = (f"qlab::api_reduce<qlab::DotOp<{RR}, {nc}, {outR}>>({kid('dot_' + T)}, r, "
                                f"2 * sizeof({outR}), {oa}, {ob}, {gang}, n);")
                        fns.append(Fn(name, params, body, "dot", CITE["dot"],
                                      dict(dest="c", var=var, a=sa, b=sb, out=outR)))
                        name = f"QLA_{rpc}_r_{var}eq_re_{sa}_dot_{sb}"
                        params = [(f"QLA_{OP}_Real *RESTRICT", "r"), pa, pb]
                        if var == "x":
                            params.append(("int *", "index"))
                        params.append(("int", "n"))
                        body = (f"qlab::api_reduce<qlab::ReDotOp<{RR}, {nc}, {outR}>>({kid('redot_' + T)}, r, "
                                f"sizeof({outR}), {oa}, {ob}, {gang}, n);")
                        fns.append(Fn(name, params, body, "redot", CITE["redot"],
                                      dict(dest="r", var=var, a=sa, b=sb, out=outR)))
    fns += gen_ewise(pc, R, P)
    fns += gen_sitefield(pc, R, P)
    return fns


# element counts (complex numbers per record) at Nc = 3
NE3 = {"V": 3, "H": 6, "D": 12, "M": 9, "P": 144}
PERM_OF = {"M": "qlab::PERM_M", "P": "qlab::PERM_P"}


def gen_ewise(pc, R, P):
    """The element-wise families (constant and field multiples, sums,
    combinations, conj / i / adjoint / transpose copies), site-local dot
    products and norms, and the ColorVector outer product, for F3 / D3."""
    fns = []
    kid = lambda fam: f'"{pc}_{fam}"'  # noqa: E731
    cplx, real = f"QLA_{P}_Complex", f"QLA_{P}_Real"

    def var_tail(var):
        return ([("int *", "index")] if var == "x" else []), ("index" if var == "x" else "nullptr")

    def srcs(T, adj):
        """(name suffix, pointer?, permutation) of the field source."""
        out = [(T, False, "qlab::PERM_ID"), ("p" + T, True, "qlab::PERM_ID")]
        if adj:
            out += [(T + "a", False, PERM_OF[T]), ("p" + T + "a", True, PERM_OF[T])]
        return out

    def emit(name, params, body, cite_key, kinds):
        # one source file per destination type (and for the local products)
        fam = {"ldot": "ldot", "outer": "ldot"}.get(cite_key, "ewise_" + kinds.get("dest", "x").lower())
        fns.append(Fn(name, params, body, fam, CITE[cite_key], kinds))

    for T in ["V", "H", "D", "M", "P"]:
        ne = NE3[T]
        adj = T in ("M", "P")
        rt = f"{ptype(pc, T)} *RESTRICT"
        for var in ["v", "x"]:
            tail, gang = var_tail(var)
            for eq in EQOPS:
                # ---- constant multiples: c_times (all), r_times (P and adjoints; the
                # plain V/H/D/M forms are the RTimesOp family)
                for src, p1, perm in srcs(T, adj):
                    pb, ob = operand(pc, T, p1, "b")
                    isadj = src.endswith("a")
                    for kind, st, shape in (("c", cplx, "qlab::EW_CTA" if isadj else "qlab::EW_CT"),
                                            ("r", real, "qlab::EW_RTA" if isadj else "qlab::EW_RT")):
                        if kind == "r" and T != "P" and not isadj:
                            continue
                        name = f"QLA_{pc}_{T}_{var}{eq}_{kind}_times_{src}"
                        params = [(rt, "r"), (f"{st} *RESTRICT", "a"), pb] + tail + [("int", "n")]
                        body = (f"qlab::api_ew<{R}, {ne}, {shape}, {perm}, qlab::SC_CONST, {str(kind == 'r').lower()}>"
                                f"({kid('ew_' + kind + 'times')}, r, a, qlab::Opnd{{}}, {ob}, qlab::Opnd{{}}, {gang}, n, "
                                f"{EQ_ENUM[eq]});")
                        emit(name, params, body, "ewise_times",
                             dict(dest=T, eqop=eq, var=var, scal=kind, b=src))
                # ---- per-site field multiples: C, Ca, R (and pointer forms)
                for sname, sp, shape, sreal, sadj in (("C", False, "CT", False, False), ("pC", True, "CT", False, False),
                                                      ("Ca", False, "CAT", False, True), ("pCa", True, "CAT", False, True),
                                                      ("R", False, "RT", True, False), ("pR", True, "RT", True, False)):
                    st = real if sreal else cplx
                    sparam = (f"{st} *RESTRICT *", "a") if sp else (f"{st} *RESTRICT", "a")
                    sop = "qlab::op_ptr((const void* const*)a)" if sp else "qlab::op_contig(a)"
                    for src, p1, perm in srcs(T, adj):
                        pb, ob = operand(pc, T, p1, "b")
                        isadj = src.endswith("a")
                        sh = {"CT": "CTA", "CAT": "CATA", "RT": "RTA"}[shape] if isadj else shape
                        name = f"QLA_{pc}_{T}_{var}{eq}_{sname}_times_{src}"
                        params = [(rt, "r"), sparam, pb] + tail + [("int", "n")]
                        body = (f"qlab::api_ew<{R}, {ne}, qlab::EW_{sh}, {perm}, qlab::SC_FIELD, {str(sreal).lower()}>"
                                f"({kid('ew_field')}, r, nullptr, {sop}, {ob}, qlab::Opnd{{}}, {gang}, n, {EQ_ENUM[eq]});")
                        emit(name, params, body, "ewise_field", dict(dest=T, eqop=eq, var=var, scal=sname, b=src))
                # ---- conj, i*a, and (M, P) adjoint / transpose copies, P copies
                unary = [("conj_", "qlab::EW_CONJ", "qlab::PERM_ID", False), ("i_", "qlab::EW_I", "qlab::PERM_ID", False)]
                if adj:
                    unary += [("", "qlab::EW_CONJ", PERM_OF[T], True), ("transpose_", "qlab::EW_COPY", PERM_OF[T], False)]
                if T == "P":
                    unary += [("", "qlab::EW_COPY", "qlab::PERM_ID", False)]
                for pre, shape, perm, asadj in unary:
                    for p1 in (False, True):
                        pa, oa = operand(pc, T, p1, "a")
                        src = ("p" if p1 else "") + T + ("a" if asadj else "")
                        name = f"QLA_{pc}_{T}_{var}{eq}_{pre}{src}"
                        params = [(rt, "r"), pa] + tail + [("int", "n")]
                        body = (f"qlab::api_ew<{R}, {ne}, {shape}, {perm}, qlab::SC_NONE, false>({kid('ew_unary')}, r, "
                                f"nullptr, qlab::Opnd{{}}, {oa}, qlab::Opnd{{}}, {gang}, n, {EQ_ENUM[eq]});")
                        emit(name, params, body, "ewise_unary", dict(dest=T, eqop=eq, var=var, op=pre or "copy", a=src))
            # ---- sums and combinations (eq only)
            for pa_, pb_ in itertools.product((False, True), (False, True)):
                sa = ("p" if pa_ else "") + T
                sb = ("p" if pb_ else "") + T
                for op, shape in (("plus", "PLUS"), ("minus", "MINUS")):
                    pa, oa = operand(pc, T, pa_, "a")
                    pb, ob = operand(pc, T, pb_, "b")
                    name = f"QLA_{pc}_{T}_{var}eq_{sa}_{op}_{sb}"
                    params = [(rt, "r"), pa, pb] + tail + [("int", "n")]
                    body = (f"qlab::api_ew<{R}, {ne}, qlab::EW_{shape}, qlab::PERM_ID, qlab::SC_NONE, false>("
                            f"{kid('ew_sum')}, r, nullptr, qlab::Opnd{{}}, {oa}, {ob}, {gang}, n, qlab::EQ);")
                    emit(name, params, body, "ewise_sum", dict(dest=T, eqop="eq", var=var, op=op, a=sa, b=sb))
                    for kind, st in (("r", real), ("c", cplx)):
                        pb2, ob2 = operand(pc, T, pa_, "b")
                        pc2, oc2 = operand(pc, T, pb_, "c")
                        name = f"QLA_{pc}_{T}_{var}eq_{kind}_times_{sa}_{op}_{sb}"
                        params = [(rt, "r"), (f"{st} *RESTRICT", "a"), pb2, pc2] + tail + [("int", "n")]
                        sh = ("RT_" if kind == "r" else "CT_") + shape
                        body = (f"qlab::api_ew<{R}, {ne}, qlab::EW_{sh}, qlab::PERM_ID, qlab::SC_CONST, "
                                f"{str(kind == 'r').lower()}>({kid('ew_axpby')}, r, a, qlab::Opnd{{}}, {ob2}, {oc2}, "
                                f"{gang}, n, qlab::EQ);")
                        emit(name, params, body, "ewise_sum", dict(dest=T, eqop="eq", var=var, op=kind + "_" + op,
                                                                  a=sa, b=sb))
    # ---- site-local dot products and norms (complex / real field outputs)
    for T in ["V", "H", "D", "M", "P"]:
        ne = NE3[T]
        for var in ["v", "x"]:
            tail, gang = var_tail(var)
            for eq in EQOPS:
                pairs = [(T, T, "LD_DOT", "qlab::PERM_ID")]
                if T in ("M", "P"):
                    pairs += [(T, T + "a", "LD_DOT_AA", PERM_OF[T]), (T + "a", T, "LD_ADOT", PERM_OF[T])]
                for ta, tb, kind, perm in pairs:
                    for pa_, pb_ in itertools.product((False, True), (False, True)):
                        sa = ("p" if pa_ else "") + ta
                        sb = ("p" if pb_ else "") + tb
                        pa, oa = operand(pc, T, pa_, "a")
                        pb, ob = operand(pc, T, pb_, "b")
                        name = f"QLA_{pc}_C_{var}{eq}_{sa}_dot_{sb}"
                        params = [(f"{cplx} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                        body = (f"qlab::api_ldot<{R}, {ne}, qlab::{kind}, {perm}>({kid('ldot')}, r, {oa}, {ob}, {gang}, "
                                f"n, {EQ_ENUM[eq]});")
                        emit(name, params, body, "ldot", dict(dest="C", eqop=eq, var=var, a=sa, b=sb, kind=kind))
                        if kind == "LD_DOT":
                            name = f"QLA_{pc}_R_{var}{eq}_re_{sa}_dot_{sb}"
                            params = [(f"{real} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                            body = (f"qlab::api_ldot<{R}, {ne}, qlab::LD_REDOT, qlab::PERM_ID>({kid('ldot')}, r, {oa}, "
                                    f"{ob}, {gang}, n, {EQ_ENUM[eq]});")
                            emit(name, params, body, "ldot", dict(dest="R", eqop=eq, var=var, a=sa, b=sb,
                                                                   kind="LD_REDOT"))
                for pa_ in (False, True):
                    sa = ("p" if pa_ else "") + T
                    pa, oa = operand(pc, T, pa_, "a")
                    name = f"QLA_{pc}_R_{var}{eq}_norm2_{sa}"
                    params = [(f"{real} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                    body = (f"qlab::api_ldot<{R}, {ne}, qlab::LD_NORM2, qlab::PERM_ID>({kid('ldot')}, r, {oa}, "
                            f"qlab::Opnd{{}}, {gang}, n, {EQ_ENUM[eq]});")
                    emit(name, params, body, "ldot", dict(dest="R", eqop=eq, var=var, a=sa, kind="LD_NORM2"))
    # ---- outer product of two ColorVectors
    for var in ["v", "x"]:
        tail, gang = var_tail(var)
        for eq in EQOPS:
            for pa_, pb_ in itertools.product((False, True), (False, True)):
                sa = ("p" if pa_ else "") + "V"
                sb = ("p" if pb_ else "") + "Va"
                pa, oa = operand(pc, "V", pa_, "a")
                pb, ob = operand(pc, "V", pb_, "b")
                name = f"QLA_{pc}_M_{var}{eq}_{sa}_times_{sb}"
                params = [(f"{ptype(pc, 'M')} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                body = f"qlab::api_outer<{R}>({kid('outer')}, r, {oa}, {ob}, {gang}, n, {EQ_ENUM[eq]});"
                emit(name, params, body, "outer", dict(dest="M", eqop=eq, var=var, a=sa, b=sb))
    return fns


def gen_sitefield(pc, R, P):
    """Fills, copymask, component extraction / insertion, gamma
    multiplication, traces and the antihermitian part, the global reductions
    of DiracPropagators and adjoint-form products, and the global sums."""
    fns = []
    kid = lambda fam: f'"{pc}_{fam}"'  # noqa: E731
    cplx, real = f"QLA_{P}_Complex", f"QLA_{P}_Real"
    outR = R

    def var_tail(var):
        return ([("int *", "index")] if var == "x" else []), ("index" if var == "x" else "nullptr")

    def emit(name, params, body, fam, kinds):
        fns.append(Fn(name, params, body, fam, CITE[fam], kinds))

    def src_param(t, p1, argname="a"):
        """parameter and operand of a field source of record letter t (C and I too)"""
        ct = {"C": cplx, "R": real, "I": "QLA_Int"}.get(t, ptype(pc, t) if t in REC else None)
        if p1:
            return (f"{ct} *RESTRICT *", argname), f"qlab::op_ptr((const void* const*){argname})"
        return (f"{ct} *RESTRICT", argname), f"qlab::op_contig({argname})"

    for var in ["v", "x"]:
        tail, gang = var_tail(var)
        # ---- constant fills, the diagonal fill, zero
        for T in ["V", "H", "D", "M", "P"]:
            ne = NE3[T]
            rt = f"{ptype(pc, T)} *RESTRICT"
            for eq in EQOPS:
                name = f"QLA_{pc}_{T}_{var}{eq}_{T.lower()}"
                params = [(rt, "r"), (f"{ptype(pc, T)} *RESTRICT", "a")] + tail + [("int", "n")]
                body = f"qlab::api_fill<{R}, {ne}>({kid('fill')}, r, a, {gang}, n, {EQ_ENUM[eq]});"
                emit(name, params, body, "fill", dict(dest=T, eqop=eq, var=var, op="fill", a=T.lower()))
            name = f"QLA_{pc}_{T}_{var}eq_zero"
            params = [(rt, "r")] + tail + [("int", "n")]
            emit(name, params, f"qlab::api_zero<{R}, {ne}>({kid('fill')}, r, {gang}, n);", "fill",
                 dict(dest=T, eqop="eq", var=var, op="zero"))
            # gaussian random fills from a field of generator states
            for ps, xs in (("", False), ("p", True)):
                sa = ("QLA_RandomState *RESTRICT *" if xs else "QLA_RandomState *RESTRICT", "a")
                oa = "qlab::op_ptr((const void* const*)a)" if xs else "qlab::op_contig(a)"
                name = f"QLA_{pc}_{T}_{var}eq_gaussian_{ps}S"
                body = f"qlab::api_rng_fill<{R}, {ne}, false>({kid('random')}, 1, r, {oa}, {gang}, n);"
                emit(name, [(rt, "r"), sa] + tail + [("int", "n")], body, "random",
                     dict(dest=T, eqop="eq", var=var, op="gaussian", a=ps + "S"))
            # ---- copymask
            for pa_, pm_ in itertools.product((False, True), (False, True)):
                pa, oa = src_param(T, pa_)
                pm, om = src_param("I", pm_, "b")
                sa = ("p" if pa_ else "") + T
                sm = ("p" if pm_ else "") + "I"
                name = f"QLA_{pc}_{T}_{var}eq_{sa}_mask_{sm}"
                params = [(rt, "r"), pa, pm] + tail + [("int", "n")]
                body = f"qlab::api_mask<{R}, {ne}>({kid('mask')}, r, {oa}, {om}, {gang}, n);"
                emit(name, params, body, "mask", dict(dest=T, eqop="eq", var=var, op="mask", a=sa, b=sm))
        for eq in EQOPS:
            name = f"QLA_{pc}_M_{var}{eq}_c"
            params = [(f"{ptype(pc, 'M')} *RESTRICT", "r"), (f"{cplx} *RESTRICT", "a")] + tail + [("int", "n")]
            body = f"qlab::api_diagfill<{R}>({kid('fill')}, r, a, {gang}, n, {EQ_ENUM[eq]});"
            emit(name, params, body, "fill", dict(dest="M", eqop=eq, var=var, op="diagfill", a="c"))
        # ---- array components, colour columns, Dirac vectors
        idx_args = {"V": ["i_c"], "H": ["i_c", "i_s"], "D": ["i_c", "i_s"], "M": ["i_c", "j_c"],
                    "P": ["i_c", "i_s", "j_c", "j_s"]}
        col_args = {"H": ["i_s"], "D": ["i_s"], "M": ["j_c"], "P": ["i_s", "j_c", "j_s"]}

        def call_sub(what, dst, src, args, ne_out, ne_src, oa):
            vals = {k: (k if k in args else "0") for k in ("i_c", "i_s", "j_c", "j_s")}
            return (f"qlab::api_sub<{R}, {ne_out}, {ne_src}>({kid('component')}, r, {oa}, {gang}, n, '{what}', "
                    f"'{dst}', '{src}', {vals['i_c']}, {vals['i_s']}, {vals['j_c']}, {vals['j_s']});")

        for T in ["V", "H", "D", "M", "P"]:
            args = idx_args[T]
            ip = [("int", a_) for a_ in args]
            for p1 in (False, True):
                # C = elem(T)
                pa, oa = src_param(T, p1)
                name = f"QLA_{pc}_C_{var}eq_elem_{'p' if p1 else ''}{T}"
                params = [(f"{cplx} *RESTRICT", "r"), pa] + ip + tail + [("int", "n")]
                emit(name, params, call_sub("e", "C", T, args, 1, NE3[T], oa), "component",
                     dict(dest="C", eqop="eq", var=var, op="elem", a=("p" if p1 else "") + T, idx=args))
                # elem(T) = C
                pa, oa = src_param("C", p1)
                name = f"QLA_{pc}_{T}_{var}eq_elem_{'p' if p1 else ''}C"
                params = [(f"{ptype(pc, T)} *RESTRICT", "r"), pa] + ip + tail + [("int", "n")]
                emit(name, params, call_sub("e", T, "C", args, NE3[T], 1, oa), "component",
                     dict(dest=T, eqop="eq", var=var, op="elem", a=("p" if p1 else "") + "C", idx=args))
        for T in ["H", "D", "M", "P"]:
            args = col_args[T]
            ip = [("int", a_) for a_ in args]
            for p1 in (False, True):
                pa, oa = src_param(T, p1)
                name = f"QLA_{pc}_V_{var}eq_colorvec_{'p' if p1 else ''}{T}"
                params = [(f"{ptype(pc, 'V')} *RESTRICT", "r"), pa] + ip + tail + [("int", "n")]
                emit(name, params, call_sub("c", "V", T, args, 3, NE3[T], oa), "component",
                     dict(dest="V", eqop="eq", var=var, op="colorvec", a=("p" if p1 else "") + T, idx=args))
                pa, oa = src_param("V", p1)
                name = f"QLA_{pc}_{T}_{var}eq_colorvec_{'p' if p1 else ''}V"
                params = [(f"{ptype(pc, T)} *RESTRICT", "r"), pa] + ip + tail + [("int", "n")]
                emit(name, params, call_sub("c", T, "V", args, NE3[T], 3, oa), "component",
                     dict(dest=T, eqop="eq", var=var, op="colorvec", a=("p" if p1 else "") + "V", idx=args))
        for p1 in (False, True):
            args = ["j_c", "j_s"]
            ip = [("int", a_) for a_ in args]
            pa, oa = src_param("P", p1)
            name = f"QLA_{pc}_D_{var}eq_diracvec_{'p' if p1 else ''}P"
            params = [(f"{ptype(pc, 'D')} *RESTRICT", "r"), pa] + ip + tail + [("int", "n")]
            emit(name, params, call_sub("d", "D", "P", args, 12, 144, oa), "component",
                 dict(dest="D", eqop="eq", var=var, op="diracvec", a=("p" if p1 else "") + "P", idx=args))
            pa, oa = src_param("D", p1)
            name = f"QLA_{pc}_P_{var}eq_diracvec_{'p' if p1 else ''}D"
            params = [(f"{ptype(pc, 'P')} *RESTRICT", "r"), pa] + ip + tail + [("int", "n")]
            emit(name, params, call_sub("d", "P", "D", args, 144, 12, oa), "component",
                 dict(dest="P", eqop="eq", var=var, op="diracvec", a=("p" if p1 else "") + "D", idx=args))
        # ---- gamma multiplication
        for T, sides in (("D", ("left",)), ("P", ("left", "right"))):
            for side in sides:
                for p1 in (False, True):
                    pa, oa = src_param(T, p1)
                    sa = ("p" if p1 else "") + T
                    name = (f"QLA_{pc}_{T}_{var}eq_gamma_times_{sa}" if side == "left"
                            else f"QLA_{pc}_{T}_{var}eq_{sa}_times_gamma")
                    params = [(f"{ptype(pc, T)} *RESTRICT", "r"), pa, ("int", "mu")] + tail + [("int", "n")]
                    body = (f"qlab::api_gamma<{R}, {NE3[T]}, {str(side == 'left').lower()}>({kid('gamma')}, r, {oa}, "
                            f"mu, {gang}, n);")
                    emit(name, params, body, "gamma", dict(dest=T, eqop="eq", var=var, op="gamma_" + side, a=sa))
        # ---- traces and the antihermitian part
        for p1 in (False, True):
            pa, oa = src_param("M", p1)
            sa = ("p" if p1 else "") + "M"
            for dest, op, kind, rtype in (("C", "trace", "SF_TRACE_C", cplx), ("R", "re_trace", "SF_TRACE_RE", real),
                                          ("R", "im_trace", "SF_TRACE_IM", real)):
                name = f"QLA_{pc}_{dest}_{var}eq_{op}_{sa}"
                params = [(f"{rtype} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                body = f"qlab::api_trace<{R}, qlab::{kind}>({kid('trace')}, r, {oa}, {gang}, n);"
                emit(name, params, body, "trace", dict(dest=dest, eqop="eq", var=var, op=op, a=sa))
            name = f"QLA_{pc}_M_{var}eq_antiherm_{sa}"
            params = [(f"{ptype(pc, 'M')} *RESTRICT", "r"), pa] + tail + [("int", "n")]
            body = f"qlab::api_antiherm<{R}>({kid('trace')}, r, {oa}, {gang}, n);"
            emit(name, params, body, "trace", dict(dest="M", eqop="eq", var=var, op="antiherm", a=sa))
        # ---- global reductions of P and of the adjoint-form products
        greds = [("c", "Ma", "M", "M", "LD_ADOT", "qlab::PERM_M"), ("c", "P", "P", "P", "LD_DOT", "qlab::PERM_ID"),
                 ("c", "Pa", "P", "P", "LD_ADOT", "qlab::PERM_P"), ("r", "P", "P", "P", "LD_REDOT", "qlab::PERM_ID")]
        for dest, ta, T, tb, kind, perm in greds:
            for pa_, pb_ in itertools.product((False, True), (False, True)):
                pa, oa = src_param(T, pa_)
                pb, ob = src_param(tb, pb_, "b")
                sa = ("p" if pa_ else "") + ta
                sb = ("p" if pb_ else "") + tb
                op = "re_" if kind == "LD_REDOT" else ""
                name = f"QLA_{pc}_{dest}_{var}eq_{op}{sa}_dot_{sb}"
                rtype = real if dest == "r" else cplx
                params = [(f"{rtype} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                body = (f"qlab::api_gdot<{R}, {NE3[T]}, qlab::{kind}, {perm}, {outR}>({kid('gred')}, r, {oa}, {ob}, "
                        f"{gang}, n);")
                emit(name, params, body, "gred", dict(dest=dest, eqop="eq", var=var, a=sa, b=sb, kind=kind))
        for p1 in (False, True):
            pa, oa = src_param("P", p1)
            sa = ("p" if p1 else "") + "P"
            name = f"QLA_{pc}_r_{var}eq_norm2_{sa}"
            params = [(f"{real} *RESTRICT", "r"), pa] + tail + [("int", "n")]
            body = (f"qlab::api_gdot<{R}, 144, qlab::LD_NORM2, qlab::PERM_ID, {outR}>({kid('gred')}, r, {oa}, "
                    f"qlab::Opnd{{}}, {gang}, n);")
            emit(name, params, body, "gred", dict(dest="r", eqop="eq", var=var, a=sa, kind="LD_NORM2"))
        # ---- global sums
        for T in ["V", "H", "D", "M", "P"]:
            for p1 in (False, True):
                pa, oa = src_param(T, p1)
                sa = ("p" if p1 else "") + T
                name = f"QLA_{pc}_{T.lower()}_{var}eq_sum_{sa}"
                params = [(f"{ptype(pc, T)} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                body = f"qlab::api_gsum<{R}, {NE3[T]}>({kid('gsum')}, r, {oa}, {gang}, n);"
                emit(name, params, body, "gsum", dict(dest=T.lower(), eqop="eq", var=var, a=sa))
        if pc != "F3":
            continue
        # ---- QLA_DF3_: the F3 global reductions and sums returned in double
        for dest, ta, T, tb, kind, perm in greds:
            for pa_, pb_ in itertools.product((False, True), (False, True)):
                pa, oa = src_param(T, pa_)
                pb, ob = src_param(tb, pb_, "b")
                sa = ("p" if pa_ else "") + ta
                sb = ("p" if pb_ else "") + tb
                op = "re_" if kind == "LD_REDOT" else ""
                name = f"QLA_DF3_{dest}_{var}eq_{op}{sa}_dot_{sb}"
                rtype = "QLA_D_Real" if dest == "r" else "QLA_D_Complex"
                params = [(f"{rtype} *RESTRICT", "r"), pa, pb] + tail + [("int", "n")]
                body = (f"qlab::api_gdot<float, {NE3[T]}, qlab::{kind}, {perm}, double>({kid('gred_df')}, r, {oa}, "
                        f"{ob}, {gang}, n);")
                emit(name, params, body, "gred", dict(dest=dest, eqop="eq", var=var, a=sa, b=sb, kind=kind,
                                                      out="double"))
        for p1 in (False, True):
            pa, oa = src_param("P", p1)
            sa = ("p" if p1 else "") + "P"
            name = f"QLA_DF3_r_{var}eq_norm2_{sa}"
            params = [("QLA_D_Real *RESTRICT", "r"), pa] + tail + [("int", "n")]
            body = (f"qlab::api_gdot<float, 144, qlab::LD_NORM2, qlab::PERM_ID, double>({kid('gred_df')}, r, {oa}, "
                    f"qlab::Opnd{{}}, {gang}, n);")
            emit(name, params, body, "gred", dict(dest="r", eqop="eq", var=var, a=sa, kind="LD_NORM2", out="double"))
        for T in ["V", "H", "D", "M", "P"]:
            for p1 in (False, True):
                pa, oa = src_param(T, p1)
                sa = ("p" if p1 else "") + T
                name = f"QLA_DF3_{T.lower()}_{var}eq_sum_{sa}"
                params = [(f"{ptype('D3', T)} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                body = f"qlab::api_gsum<float, {NE3[T]}, double>({kid('gsum_df')}, r, {oa}, {gang}, n);"
                emit(name, params, body, "gsum", dict(dest=T.lower(), eqop="eq", var=var, a=sa, out="double"))
        # ---- precision conversions D3 <- F3 (QLA_DF3_) and F3 <- D3 (QLA_FD3_)
        for T in ["V", "H", "D", "M", "P"]:
            for p1 in (False, True):
                for lib, rin, rout, pin, pout in (("DF3", "float", "double", "F3", "D3"),
                                                  ("FD3", "double", "float", "D3", "F3")):
                    ct = ptype(pin, T)
                    pa = (f"{ct} *RESTRICT *", "a") if p1 else (f"{ct} *RESTRICT", "a")
                    oa = "qlab::op_ptr((const void* const*)a)" if p1 else "qlab::op_contig(a)"
                    sa = ("p" if p1 else "") + T
                    name = f"QLA_{lib}_{T}_{var}eq_{sa}"
                    params = [(f"{ptype(pout, T)} *RESTRICT", "r"), pa] + tail + [("int", "n")]
                    body = f"qlab::api_convert<{rin}, {rout}, {NE3[T]}>({kid('convert')}, r, {oa}, {gang}, n);"
                    emit(name, params, body, "convert", dict(dest=T, eqop="eq", var=var, a=sa, lib=lib))
    return fns


HEADER_TOP = """/*
 * {fname} -- GENERATED by qla_b200/gen/gen_qla.py; do not edit.
 *
 * QLA {pc} level-1 entry points implemented by libqla_b200.so (sm_100a).
 * Each declaration replaces the reference function of the same name, whose
 * C loop the reference generator emits from the cited section.  Array
 * arguments are device pointers; see qla_b200_runtime.h for scalars,
 * reduction outputs, streams and errors.
 */
#ifndef {guard}
#define {guard}
#include "qla_b200_types.h"

#ifdef __cplusplus
#define QLA_B200_RESTRICT __restrict__
extern "C" {{
#else
#define QLA_B200_RESTRICT restrict
#endif

"""

HEADER_END = """
#ifdef __cplusplus
}
#endif
#endif
"""

CU_TOP = """// GENERATED by qla_b200/gen/gen_qla.py; do not edit.
// QLA {pc} {family} entry points (extern "C"), reference: {cite}
#include "../../../include/qla_b200_types.h"
#include "../qla_api.cuh"
{extra_includes}
extern "C" {{
"""


def write_if_changed(path, text):
    if os.path.exists(path):
        with open(path) as f:
            if f.read() == text:
                return False
    with open(path, "w") as f:
        f.write(text)
    return True


def main():
    os.makedirs(OUT_CU, exist_ok=True)
    manifest = []
    groups = {}
    headers = {}
    for pc, R, P in [("F3", "float", "F"), ("D3", "double", "D"), ("I", None, None), ("FN", None, None),
                     ("DN", None, None), ("F", None, None), ("D", None, None), ("F2", None, None),
                     ("D2", None, None)]:
        for fn in (gen_int() if pc == "I" else gen_fn("F") + gen_fn_wide("F") if pc == "FN"
                   else gen_fn("D") + gen_fn_wide("D") if pc == "DN" else gen_fd(pc) if pc in ("F", "D")
                   else gen_two(pc[0]) if pc in ("F2", "D2") else gen_pc(pc, R, P)):
            hpc = fn.name.split("_")[1]  # F3 / D3 / DF3
            # the reference declares QLA_FD3_ in qla_df3.h, QLA_FDN_ in qla_dfn.h, QLA_S_ in qla_int.h
            hpc = {"FD3": "DF3", "FDN": "DFN", "S": "I", "FD": "DF", "FD2": "DF2"}.get(hpc, hpc)
            headers.setdefault(hpc, []).append(fn)
            groups.setdefault((pc, fn.family), []).append(fn)
            manifest.append(dict(name=fn.name, pc=hpc, family=fn.family, params=[n for _, n in fn.params],
                                 ctypes=[t.replace("RESTRICT", "").strip() for t, _ in fn.params], **fn.kinds))
    written = 0
    for hpc, fns in headers.items():
        fname = f"qla_b200_{'int' if hpc == 'I' else hpc.lower()}.h"
        text = HEADER_TOP.format(fname=fname, pc=hpc, guard=f"QLA_B200_{hpc}_H")
        fam = None
        for fn in fns:
            if fn.family != fam:
                fam = fn.family
                text += f"/* ---- {fam}: replaces the {hpc} functions emitted by {fn.cite.split(',')[0]} */\n"
            if fn.cite.startswith("no counterpart"):
                text += f"/* {fn.name}: {fn.cite} */\n"
            else:
                text += f"/* replaces {fn.name} ({fn.cite}) */\n"
            text += fn.proto("QLA_B200_RESTRICT") + ";\n"
        text += HEADER_END
        written += write_if_changed(os.path.join(OUT_INC, fname), text)
    for (pc, family), fns in groups.items():
        extra = {"int": '#include "../qla_int.cuh"\n', "mfunc": '#include "../qla_mfunc.cuh"\n',
                 "mfunc_ext": '#include "../qla_mfunc_ext.cuh"\n',
                 "multi": '#include <vector>\n#include "../qla_multi.cuh"\n',
                 "prop": '#include "../qla_prop.cuh"\n',
                 "ldot": '#include "../qla_ewise.cuh"\n'}.get(family, "")
        if family.startswith("ewise"):
            extra = '#include "../qla_ewise.cuh"\n'
        if family in ("fill", "mask", "component", "gamma", "trace", "gred", "gsum", "convert"):
            extra = '#include "../qla_sitefield.cuh"\n'
        if family == "random":
            extra = '#include "../qla_random.cuh"\n'
        if family in ("cfield", "rfield", "sglobal") or (pc == "F" and family == "convert"):
            extra = '#include "../qla_scalar.cuh"\n'
        if pc in ("FN", "DN", "F2", "D2") and (family.startswith("ewise") or family in (
                "ldot", "fill", "mask", "component", "gamma", "trace", "gred", "gsum", "convert", "prop", "multi",
                "random")):
            extra = '#include "../qla_ncolor.cuh"\n#include "../qla_random.cuh"\n'
        if pc in ("FN", "DN", "F2", "D2") and family in ("mfunc", "mfunc_ext"):
            extra = '#include "../qla_mfunc_nc2.cuh"\n'
        text = CU_TOP.format(pc=pc, family=family, cite=CITE[family], extra_includes=extra)
        for fn in fns:
            text += ("QLAB_EXPORT " + fn.proto("__restrict__") + " {\n  QLAB_TRACE(\"" + fn.name + "\");\n  " +
                     fn.body + "\n}\n\n")
        text += "}  // extern \"C\"\n"
        written += write_if_changed(os.path.join(OUT_CU, f"{pc.lower()}_{family}.cu"), text)
    mtext = json.dumps(manifest, indent=0, sort_keys=True)
    written += write_if_changed(os.path.join(HERE, "api_manifest.json"), mtext)
    print(f"gen_qla: {len(manifest)} entry points, {written} files updated", file=sys.stderr)


if __name__ == "__main__":
    main()

"""CPU checks of the drop-in boundary: the C-ABI library loads without a GPU,
exports every symbol that include/*.h declares, the declarations carry a
reference citation, the generator's output is up to date, and the Python
mirror refuses non-device arrays instead of falling back to the CPU."""
import ctypes
import glob
import os
import re
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(REPO, "include")


def declared_symbols():
    syms = {}
    for h in glob.glob(os.path.join(INC, "*.h")):
        with open(h) as f:
            text = f.read()
        for m in re.finditer(r"^\s*(?:void|int|unsigned|const char \*|void \*)\s*\*?\s*((?:QLA|qlagpu)_\w+)\s*\(",
                             text, re.M):
            syms[m.group(1)] = os.path.basename(h)
    return syms


def test_headers_declare_the_hot_path():
    syms = declared_symbols()
    for s in ["QLA_F3_V_veq_M_times_V", "QLA_F3_V_veq_Ma_times_V", "QLA_F3_r_veq_norm2_V",
              "QLA_F3_H_veq_spproj_D", "QLA_F3_V_veq_M_times_pV", "QLA_F3_H_veq_M_times_pH",
              "QLA_F3_D_vpeq_sprecon_H", "QLA_F3_D_vpeq_r_times_D", "QLA_DF3_r_veq_norm2_D",
              "QLA_DF3_c_veq_D_dot_D", "QLA_F3_M_veq_M_times_pM", "QLA_D3_D_vpeq_r_times_D",
              "QLA_F3_V_eq_M_times_xV", "QLA_F3_V_veq_pV", "qlagpu_last_error", "qlagpu_shift_index"]:
        assert s in syms, s
    assert len(syms) > 1200


def test_library_exports_every_declared_symbol():
    import qla_b200
    lib = qla_b200.lib()  # loads without a GPU
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing[:10]


def test_declarations_cite_the_reference():
    for h in ("qla_b200_f3.h", "qla_b200_d3.h", "qla_b200_df3.h"):
        with open(os.path.join(INC, h)) as f:
            lines = f.read().splitlines()
        for i, line in enumerate(lines):
            if line.startswith("void QLA_"):
                assert lines[i - 1].startswith("/* replaces QLA_") and ".pl:" in lines[i - 1] or \
                    "doc/qla.tex" in lines[i - 1], line
            elif line.startswith("void qlagpu_"):  # additions of this library
                assert "no counterpart in the reference" in lines[i - 1], line


def test_generator_output_is_current():
    r = subprocess.run([sys.executable, os.path.join(REPO, "qla_b200", "gen", "gen_qla.py")],
                       capture_output=True, text=True, check=True)
    assert "0 files updated" in r.stderr, r.stderr


def test_manifest_matches_exports():
    import qla_b200
    names = {e["name"] for e in qla_b200.manifest()}
    syms = declared_symbols()
    # the host functions on one random-number state are hand-written, not generated
    host_api = {"QLA_seed_random", "QLA_random", "QLA_gaussian"}
    assert {s for s in names if s.startswith("QLA_")} == {s for s in syms if s.startswith("QLA_")} - host_api
    assert names <= set(syms)


def test_python_mirror_rejects_host_arrays():
    import numpy as np
    import torch

    import qla_b200
    t = torch.zeros(4, 6)
    with pytest.raises(qla_b200.QLAError):
        qla_b200.F3.V_veq_M_times_V(t, t, t, 1)
    del np


def test_runtime_error_api_without_device():
    import qla_b200
    L = qla_b200.lib()
    qla_b200.clear_error()
    assert L.qlagpu_last_error() == 0
    # argument errors are caught on the host, before any CUDA call
    assert L.qlagpu_tune_set(b"F3_lmult_V00", 96, 4) != 0
    code, msg = qla_b200.last_error()
    assert code == 4 and "qlagpu_tune_set" in msg
    qla_b200.clear_error()
    assert L.qlagpu_tune_set(b"F3_lmult_V00", 128, 4) == 0
    L.qlagpu_tune_clear()
    # NULL arrays are reported, not dereferenced
    L.QLA_F3_V_veq_M_times_V(None, None, None, 16)
    code, _ = qla_b200.last_error()
    assert code == 1
    qla_b200.clear_error()
    # n <= 0 is a no-op for maps, exactly as in the reference
    L.QLA_F3_V_veq_M_times_V(None, None, None, 0)
    assert qla_b200.last_error()[0] == 0
    assert b"sm_100a" in qla_b200.lib().qlagpu_version()
    assert ctypes.sizeof(ctypes.c_void_p) == 8

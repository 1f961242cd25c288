"""Build libqla_b200.so in-tree for sm_100a.

  python -m qla_b200.build [--jobs N] [--force]

Runs the C-ABI generator (qla_b200/gen/gen_qla.py), compiles every .cu under
qla_b200/csrc with nvcc (-gencode arch=compute_100a,code=sm_100a), one object
per file in parallel, and links qla_b200/lib/libqla_b200.so.  Each object is
rebuilt when its source or a header it includes is newer (nvcc writes the
header list beside the object, `-MD -MF`); an object without that list is
rebuilt when any header of the package is newer.
"""
import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libqla_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I" + os.path.join(REPO, "include"),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _newest_header():
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(REPO, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0)


def _deps_time(obj):
    """Newest modification time of the headers recorded for `obj`, or None
    when the dependency file is missing or names a file that no longer exists."""
    d = obj + ".d"
    if not os.path.exists(d):
        return None
    with open(d) as f:
        txt = f.read().replace("\\\n", " ")
    _, _, rhs = txt.partition(":")
    newest = 0.0
    for dep in rhs.split():
        if not dep.startswith("/usr/"):
            dep = dep if os.path.isabs(dep) else os.path.join(REPO, dep)
            if not os.path.exists(dep):
                return None
            newest = max(newest, os.path.getmtime(dep))
    return newest


def build(jobs=None, force=False, verbose=True):
    subprocess.check_call([sys.executable, os.path.join(PKG, "gen", "gen_qla.py")])
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "gen", "*.cu")))
    hdr_t = _newest_header()
    todo = []
    objs = []
    for s in srcs:
        rel = os.path.relpath(s, CSRC).replace(os.sep, "__")
        o = os.path.join(OBJ, rel[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o):
            todo.append((s, o))
            continue
        dt = _deps_time(o)
        if os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t if dt is None else dt):
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        # extern "C" entry points must stay visible despite -fvisibility=hidden
        cmd = [nvcc()] + NVCC_FLAGS + ["-DQLA_B200_BUILD", "-c", s, "-o", o + ".tmp", "-MD", "-MF", o + ".d.tmp"]
        r = subprocess.run(cmd, capture_output=True, text=True, cwd=REPO)
        if r.returncode != 0:
            return s, r.stderr
        os.replace(o + ".tmp", o)
        os.replace(o + ".d.tmp", o + ".d")
        return s, None

    jobs = jobs or min(len(todo) or 1, os.cpu_count() or 4)
    errors = []
    if todo:
        if verbose:
            print(f"qla_b200.build: compiling {len(todo)} of {len(srcs)} sources with {jobs} jobs", file=sys.stderr)
        with ThreadPoolExecutor(max_workers=jobs) as ex:
            for s, err in ex.map(compile_one, todo):
                if err:
                    errors.append((s, err))
    if errors:
        for s, err in errors:
            print(f"--- {s}\n{err}", file=sys.stderr)
        raise RuntimeError(f"qla_b200.build: {len(errors)} source(s) failed to compile")
    if todo or not os.path.exists(LIB) or force:
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB + ".tmp"] + objs + \
            ["-lcudart"]
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
        if verbose:
            print(f"qla_b200.build: linked {LIB}", file=sys.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(a.jobs, a.force)

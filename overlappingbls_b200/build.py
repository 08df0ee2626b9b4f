"""Build libobl_b200.so (sm_100a) in-tree with nvcc.

    python -m overlappingbls_b200.build [--force] [-j N] [-D NAME=VALUE ...] [--out PATH] [--tuned [WORKLOAD]]
                                        [--checked]

Objects go to overlappingbls_b200/_build/ (git-ignored); the shared library is
written next to this file so that it travels with the source tree.  -D passes
compile-time tuning definitions (e.g. OBL_SIDX_SHIFT=4) and --out writes a variant
library elsewhere (with its own object directory under _build/), loadable through
$OBL_LIB.  --checked writes the bounds-checked build libobl_b200_check.so
(-DOBL_CHECK=1).
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libobl_b200.so")
# the bounds-checked build (-DOBL_CHECK=1: index checks that record and skip, see csrc/check.cuh)
LIB_CHECK = os.path.join(HERE, "libobl_b200_check.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I" + INCLUDE,
         "--expt-relaxed-constexpr"]
# per-file flags: the persistent ensemble kernel reads data other SMs wrote earlier in the
# same launch, so its global loads default to the L2-only (.cg) cache policy
FILE_FLAGS = {f: ["-Xptxas", "-dlcm=cg"] for f in
              ("ensemble.cu", "ensemble_all.cu", "ensemble_part_rows.cu", "ensemble_part_mid.cu")}


def _deps():
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


def _compile(src, force, hdr_mtime, build_dir=BUILD, defines=()):
    obj = os.path.join(build_dir, os.path.basename(src).replace(".cu", ".o"))
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime)):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + ["-D" + d for d in defines] + FILE_FLAGS.get(os.path.basename(src), []) + \
        ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "$ " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(force=False, jobs=None, verbose=False, defines=(), out=None):
    lib = out or LIB
    # a variant's objects (other definitions) go to their own folder under _build/
    build_dir = BUILD if out is None else os.path.join(BUILD, os.path.basename(out).replace(".so", ""))
    os.makedirs(build_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _deps()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    objs, errs = [], []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, err in ex.map(lambda s: _compile(s, force, hdr, build_dir, defines), srcs):
            objs.append(obj)
            if err:
                errs.append(err)
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    if verbose:
        print(lib)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-D", dest="defines", action="append", default=[])
    ap.add_argument("--out", default=None)
    ap.add_argument("--checked", action="store_true", help="the bounds-checked build, libobl_b200_check.so")
    ap.add_argument("--tuned", nargs="?", const="512x512x256", default=None, metavar="WORKLOAD",
                    help="add the schedule the tuner's cache chose for WORKLOAD (overlappingbls_b200.tune)")
    a = ap.parse_args()
    defines = list(a.defines)
    if a.checked:
        defines.append("OBL_CHECK=1")
        a.out = a.out or LIB_CHECK
    if a.tuned:
        from overlappingbls_b200 import tune
        defines += tune.tuned_defines(a.tuned)
        print("tuned schedule:", defines or "default")
    try:
        build(force=a.force or bool(a.tuned), jobs=a.j, verbose=True, defines=defines, out=a.out)
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)

"""Build the native parts of lightspeed_b200 in-tree.

  python lightspeed_b200/build.py [--jobs N] [--force]

(run as a script: the package itself imports the modules this builds)

Steps (each skipped when its outputs are newer than its inputs):
  1. quadrature tables   tables/gen_tables.py   -> csrc/tables/quad_tables.inc
  2. quartet code        csrc/gen_kernels.py    -> csrc/generated/*.cuh
  3. CUDA engine         csrc/*.cu (sm_100a)    -> lightspeed_b200/liblsjk.so
  4. host C++ + Python binding (pybind11)       -> lightspeed_b200/_lightspeed*.so

The kernels are compiled for sm_100a only (-gencode arch=compute_100a,
code=sm_100a); nvcc cross-compiles without a GPU.
"""
import argparse
import glob
import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]
LIB = os.path.join(PKG, "liblsjk.so")
LMAX = 3        # largest shell of the kernels (f)


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _newest(paths):
    return max([_mtime(p) for p in paths] + [0.0])


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: %s" % cmd[-1])
    return r


def gen_sources(force=False):
    inc = os.path.join(CSRC, "tables", "quad_tables.inc")
    gen = os.path.join(PKG, "tables", "gen_tables.py")
    if force or _mtime(inc) < _mtime(gen):
        _run([sys.executable, gen], cwd=ROOT)
    kgen = os.path.join(CSRC, "gen_kernels.py")
    jq = os.path.join(CSRC, "generated", "jquartets.cuh")
    if force or _mtime(jq) < _mtime(kgen):
        _run([sys.executable, kgen, str(LMAX)], cwd=ROOT)


def cuda_units():
    """(object name, source, extra flags) for every translation unit."""
    units = []
    for name in ("basis", "pairs", "capi", "jbuild", "kbuild", "oneint", "mlp"):
        units.append((name, os.path.join(CSRC, name + ".cu"), []))
    # K gradient classes, one unit per partner-1 shell
    for l1 in range(LMAX + 1):
        units.append(("kgrad_%d" % l1, os.path.join(CSRC, "kgrad.cu"), ["-DLSJK_KG_L1=%d" % l1]))
    # bra Hermite classes 0..2*LMAX, and 2*LMAX+1 for the gradients
    for lb in range(2 * LMAX + 2):
        units.append(("jinst_%d" % lb, os.path.join(CSRC, "jinst.cu"), ["-DLSJK_LB=%d" % lb]))
    for l1 in range(LMAX + 1):
        for l2 in range(LMAX + 1):
            units.append(("kinst_%d%d" % (l1, l2), os.path.join(CSRC, "kinst.cu"),
                          ["-DLSJK_L1=%d" % l1, "-DLSJK_L2=%d" % l2]))
    return units


def build_cuda(jobs=8, force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    deps = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "generated", "*.cuh")) + \
        [os.path.join(CSRC, "tables", "quad_tables.inc"), os.path.join(INCLUDE, "lsjk.h")]
    dep_time = _newest(deps)
    todo = []
    objs = []
    for name, src, extra in cuda_units():
        obj = os.path.join(OBJ, name + ".o")
        objs.append(obj)
        if force or _mtime(obj) < max(dep_time, _mtime(src)):
            todo.append((name, src, extra, obj))

    def compile_one(t):
        name, src, extra, obj = t
        cmd = [NVCC] + NVFLAGS + extra + ["-Xptxas", "-v", "-c", src, "-o", obj]
        r = _run(cmd, cwd=CSRC)
        with open(os.path.join(OBJ, name + ".ptxas.log"), "w") as fh:
            fh.write(r.stderr)
        return name

    if todo:
        with ThreadPoolExecutor(max_workers=jobs) as ex:
            for name in ex.map(compile_one, todo):
                if verbose:
                    print("compiled", name)
    if force or todo or _mtime(LIB) < _newest(objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
        if verbose:
            print("linked", LIB)
    return LIB


def build_host(force=False, verbose=False):
    import pybind11
    hsrc = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    if not hsrc:
        return None
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(PKG, "_lightspeed" + suffix)
    deps = hsrc + glob.glob(os.path.join(CSRC, "host", "*.hpp")) + [LIB, os.path.join(INCLUDE, "lsjk.h")]
    if not force and _mtime(out) >= _newest(deps):
        return out
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp",
           "-I" + INCLUDE, "-I" + os.path.join(CSRC, "host"), "-I" + pybind11.get_include(),
           "-I" + sysconfig.get_paths()["include"]] + hsrc + \
          ["-o", out, "-L" + PKG, "-llsjk", "-Wl,-rpath,$ORIGIN"]
    _run(cmd)
    if verbose:
        print("built", out)
    return out


def build_all(jobs=8, force=False, verbose=False):
    gen_sources(force)
    build_cuda(jobs, force, verbose)
    build_host(force, verbose)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 8)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build_all(a.jobs, a.force, verbose=True)


if __name__ == "__main__":
    main()

"""Build the sm_100a CUDA library in-tree: hackathon_b200/_lib/libddm_b200.so.

nvcc cross-compiles for sm_100a without a GPU, so this runs anywhere the CUDA
toolkit is installed. Objects are compiled in parallel and rebuilt only when
a source or header is newer than the library.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libddm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include")]


# sim.cu restates the reference's JavaScript arithmetic: every product and sum
# rounded on its own (no fused multiply-add)
PER_FILE = {"sim.cu": ["--fmad=false"]}


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    deps += glob.glob(os.path.join(ROOT, "include", "*.h")) + [os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    """Compile every CUDA/C++ source for sm_100a and link the shared library."""
    if not force and not _stale():
        return LIB
    nvcc = _nvcc()
    obj_dir = os.path.join(OUT_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmd = [nvcc, *ARCH, *FLAGS, *extra, *PER_FILE.get(os.path.basename(src), []), "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            # host FP64 code: IEEE operation order, no FMA contraction (the
            # reference's JavaScript arithmetic)
            cmd = [nvcc, *FLAGS, "-Wno-deprecated-gpu-targets", "-Xcompiler", "-ffp-contract=off", "-x", "c++",
                   "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return obj, r.stderr

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        results = list(ex.map(compile_one, _sources()))
    if verbose or ptxas_info:
        for _, err in results:
            if err:
                print(err, file=sys.stderr)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-cudart=static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))

"""Build libfastmc_b200.so (CUDA sm_100a kernels + C++ host code + the C ABI) in-tree.

    python fastmc-1.4.0_b200/build.py            # incremental
    python fastmc-1.4.0_b200/build.py --force    # rebuild everything

Output: fastmc-1.4.0_b200/lib/libfastmc_b200.so (nvcc cross-compiles sm_100a without a GPU).
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib", "libfastmc_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX_HOST", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  f"-I{INCLUDE}", f"-I{CSRC}", "-Xptxas", "-warn-spills"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function", f"-I{INCLUDE}", f"-I{CSRC}",
            "-I/usr/local/cuda/include"]

SOURCES = ["fmc_inputs.cpp", "fmc_desc.cpp", "fmc_restart.cpp", "fmc_system.cpp", "fmc_kernels.cu", "fmc_chain.cu", "fmc_api.cu", "fmc_noalloc.cu", "fmc_batch.cu",
           "fmc_batch_host.cu", "fmc_slot.cu", "fmc_serve.cu"]
HEADERS = ["fmc_common.h", "fmc_inputs.h", "fmc_desc.h", "fmc_system.h", "fmc_device.cuh", "fmc_kernels.h", "fmc_chain.h", "fmc_batch.h", "fmc_restart.h"]


def _newest_header():
    hs = [os.path.join(CSRC, h) for h in HEADERS if os.path.exists(os.path.join(CSRC, h))]
    hs.append(os.path.join(INCLUDE, "fastmc_b200.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src, force):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), _newest_header()):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVFLAGS + ["-c", path, "-o", obj]
    else:
        cmd = [CXX] + CXXFLAGS + ["-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, (r.stdout + r.stderr).strip() or None


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [o for o, _ in results]
    for (o, msg) in results:
        if msg and verbose:
            print(f"[{os.path.basename(o)}] {msg}")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

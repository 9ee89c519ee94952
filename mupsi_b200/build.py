"""Build libmupsi_gpu.so in-tree with nvcc for sm_100a (no JIT cache).

    python -m mupsi_b200.build
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmupsi_gpu.so")
SOURCES = ["core.cu", "render.cu", "mlp.cu", "host_bvh.cpp", "host_obj.cpp", "display.cpp"]
HEADERS = ["core.cuh", "dmath.cuh", "geom.cuh", "gp.cuh", "host.h", "scene.cuh", "tc.cuh"]
ROOT_HEADER = os.path.join(HERE, "..", "include", "mupsi_gpu.h")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: float expressions round exactly as written (FMA only where a
# kernel calls fmaf); the host side gets -ffp-contract=off for the same reason.
NVCC_FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-Xptxas", "-warn-spills"]


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [ROOT_HEADER, __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, env=env)))
        objs.append(obj)
    for cmd, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + out)
        if verbose and out.strip():
            print(out)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

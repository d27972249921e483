"""Build recipe for libifgf_b200.so (sm_100a).

Compiles the CUDA pipeline and the host planner with nvcc and links one
shared library in-tree (ifgf_b200/libifgf_b200.so) with the CUDA runtime
linked statically, so the library depends on the driver only.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libifgf_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE]

SOURCES = ["operator.cu", "plan.cpp", "gpu_tree.cu", "gpu_lists.cu", "gpu_target_lists.cu",
           "capi.cpp", "noalloc.cu", "upward_images.cu"] + [
    f"kernels_k{k}.cu" for k in range(8)]
HEADERS = ["common.hpp", "devbuf.hpp", "gpu_target_lists.hpp", "plan.hpp", "operator.hpp",
           "device_math.cuh", "mult.hpp",
           "mult_kernels.cuh", "mult_batch.cuh", "far_staged.cuh", "tcgen05.cuh", "upward_tc.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ifgf_b200.h")]
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path, *headers]):
            cmd = [NVCC, *ARCH, *COMMON, "-c", path, "-o", obj]
            if verbose and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            cmds.append(cmd)
    # translation units compile in parallel (one per kernel plug-in)
    from concurrent.futures import ThreadPoolExecutor

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=not verbose)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd, r in zip(cmds, ex.map(run, cmds)):
            if r.returncode != 0:
                if not verbose:
                    sys.stderr.write(r.stdout.decode() + r.stderr.decode())
                raise subprocess.CalledProcessError(r.returncode, cmd)
    if force or _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

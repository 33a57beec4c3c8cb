"""Builds the CUDA library of the package for sm_100a.

``python -m delta_ray_b200.build`` (or ``build()``) compiles csrc/*.cu with
nvcc into ``delta_ray_b200/libdr_b200.so`` in place, so that the shared object
travels with the source tree.  The build is incremental: sources are only
recompiled when they, or the headers, are newer than the library.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdr_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The renderer's kernels keep IEEE operation order (no FMA contraction): its
# branch decisions (hit triangles, edge-tree choices, line-sample tests) then
# see the bits of the CPU restatement of the reference, which runs the same
# operations in the same order, so a GPU render takes each sample's branches
# as the CPU does.  Only the learned proposal's network (dr_mlp.cu), whose
# output is a sampling weight, is contracted.
NO_FMA = ["-fmad=false"]
PER_FILE_FLAGS = {"dr_backward.cu": NO_FMA, "dr_edge_kernels.cu": NO_FMA, "dr_kernels.cu": NO_FMA,
                  "dr_scene_build.cu": NO_FMA}
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off",
              "-Xcompiler", "-fvisibility=hidden", "-I", os.path.join(ROOT, "include")]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra_flags=()):
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    procs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs + [__file__]):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, *PER_FILE_FLAGS.get(os.path.basename(src), []), *extra_flags,
                   "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for src, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out}")
        if verbose and out.strip():
            print(out)
    if _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

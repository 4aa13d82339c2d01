"""Builds the library in-tree: monocuda-pt_b200/libmcpt.so (sm_100a) and the
`monocuda` command-line driver next to it.

Per-file flags:
  mc_bvh.cu     -O3 -fmad=false, IEEE division: the Morton codes must equal the
                reference's host (IEEE, no contraction) computation bit for bit.
  mc_ingest.cu  the same IEEE flags: light areas and normals equal the
                reference's host computation bit for bit.
  mc_render.cu, mc_resolve.cu, mc_volume.cu  -O3 --use_fast_math: the reference's release flags
                (CMakeLists.txt:88-96), which the per-ray arithmetic must match.
  other .cu     -O3
  mc_scene.cpp, mc_scene_gen.cpp, mc_obj.cpp  g++ -O2 -ffp-contract=off (host
                scene, camera and OBJ math as the reference's host code).

Usage: python monocuda-pt_b200/build.py [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmcpt.so")
CLI = os.path.join(HERE, "monocuda")
NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", os.path.join(ROOT, "include"), "-I", CSRC]

UNITS = {
    "mc_bvh.cu": ["-O3", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "mc_render.cu": ["-O3", "--use_fast_math"],
    "mc_context.cu": ["-O3"],
    "mc_host.cu": ["-O3"],
    "mc_batch.cu": ["-O3", "--use_fast_math"],
    "mc_guide.cu": ["-O3"],
    "mc_server.cu": ["-O3"],
    "mc_ingest.cu": ["-O3", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "mc_resolve.cu": ["-O3", "--use_fast_math"],
    "mc_volume.cu": ["-O3", "--use_fast_math"],
}
HOST_UNITS = {"mc_scene.cpp": ["-O2", "-ffp-contract=off", "-fno-fast-math"],
              "mc_scene_gen.cpp": ["-O2", "-ffp-contract=off", "-fno-fast-math"], "mc_image.cpp": ["-O2"],
              "mc_obj.cpp": ["-O2", "-ffp-contract=off", "-fno-fast-math"], "mc_files.cpp": ["-O2"]}


def headers():
    out = [os.path.join(ROOT, "include", "mc_abi.h")]
    out += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return out


def stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def compile_unit(src, flags, host):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if host:
        cmd = [CXX, "-std=c++17", "-fPIC", "-fvisibility=hidden", "-pthread", "-I", os.path.join(ROOT, "include"),
               "-I", CSRC, "-c", src, "-o", obj] + flags
    else:
        cmd = [NVCC] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj


def build(jobs=8, force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = headers()
    work = []
    objs = []
    for name, flags in list(UNITS.items()) + list(HOST_UNITS.items()):
        src = os.path.join(CSRC, name)
        if not os.path.exists(src):
            continue
        host = name in HOST_UNITS
        obj = os.path.join(OBJ, name + ".o")
        objs.append(obj)
        if force or stale(obj, [src] + hdrs):
            work.append((src, flags, host))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(compile_unit, *w) for w in work]
        for f in futs:
            f.result()
            if verbose:
                print("compiled", f.result())
    if force or work or stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    cli_src = os.path.join(HERE, "cli", "monocuda.cpp")
    if os.path.exists(cli_src) and (force or stale(CLI, [cli_src, LIB] + hdrs)):
        cmd = [CXX, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), cli_src, "-o", CLI,
               "-L", HERE, "-lmcpt", "-Wl,-rpath,$ORIGIN", "-pthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("CLI link failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=8)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.j, a.force, a.v))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)

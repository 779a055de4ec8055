"""Build the native libraries in-tree (they travel with the repository).

  trussnet_b200/libv2m_cuda.so     the CUDA relaxation (csrc/*.cu), sm_100a, C ABI of
                                   include/v2m_cuda.h
  trussnet_b200/libv2m_cuda_check.so  the same with device bounds checks (V2M_CHECK)
  trussnet_b200/libv2m_relax_cl.so the C++ shim tn::relax_cl (csrc/relax_cl_shim.cpp),
                                   built only where the reference headers are present

Parity needs IEEE float arithmetic in the kernels: no FMA contraction
(--fmad=false), correctly rounded division and square root (nvcc's defaults,
kept explicit).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libv2m_cuda.so")
LIB_CHECK = os.path.join(HERE, "libv2m_cuda_check.so")   # the bounds-checked build (V2M_CHECK)
SHIM = os.path.join(HERE, "libv2m_relax_cl.so")


def _reference_tree() -> str:
    """The reference tree whose headers the shim and the drop-in driver compile
    against: V2M_REFERENCE, else the location oracle/Makefile's recipe names
    (the one place that names it)."""
    if os.environ.get("V2M_REFERENCE"):
        return os.environ["V2M_REFERENCE"]
    r = subprocess.run(["make", "-s", "--no-print-directory", "-f", os.path.join(ROOT, "oracle", "Makefile"),
                        "print-ref"], capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


REF = _reference_tree()

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "--fmad=false", "-prec-div=true",
              "-prec-sqrt=true", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xptxas", "-v"]
SOURCES = ["v2m_kernels.cu", "v2m_host.cu", "v2m_adjoint.cu", "v2m_noalloc.cu", "v2m_seed.cu", "v2m_grid.cu"]
HEADERS = ["v2m_kernels.h", "v2m_types.cuh", "v2m_field.cuh", "v2m_sdf.cuh", "v2m_binsort.cuh", "v2m_grid.h"]


def nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_cuda(force: bool = False, verbose: bool = False, check: bool = False) -> str:
    """libv2m_cuda.so; check=True: libv2m_cuda_check.so, the same sources with
    V2M_CHECK (device bounds checks on the lookups whose ranges hold by
    construction; a failed check makes the call return V2M_ERR_KERNEL). The
    sources compile in parallel."""
    out = LIB_CHECK if check else LIB
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "v2m_cuda.h"), __file__]
    if not force and not _stale(out, deps):
        return out
    flags = NVCC_FLAGS + (["-DV2M_CHECK"] if check else [])
    tag = ".check" if check else ""
    jobs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", tag + ".o"))
        cmd = [nvcc(), *flags, "-c", os.path.join(CSRC, src), "-o", obj]
        jobs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    objs, logs, failed = [], [], None
    for src, obj, pr in jobs:
        o, e = pr.communicate()
        logs.append(o + e)
        if pr.returncode != 0 and failed is None:
            failed = f"nvcc failed on {src}:\n{e[-6000:]}"
        objs.append(obj)
    if failed:
        raise RuntimeError(failed)
    tmp = out + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    os.replace(tmp, out)
    for o in objs:
        os.remove(o)
    if not check:
        with open(os.path.join(CSRC, "ptxas_info.txt"), "w") as f:
            f.write("\n".join(line for log in logs for line in log.splitlines() if "ptxas" in line))
    if verbose:
        print("\n".join(logs))
    return out


def build_shim(force: bool = False) -> str | None:
    """tn::relax_cl over the C ABI; compiled against the reference's headers
    (src/v2m_particles.h, src/v2m_grid.h), so only where they exist."""
    if not os.path.isdir(os.path.join(REF, "src")):
        return SHIM if os.path.exists(SHIM) else None
    src = os.path.join(CSRC, "relax_cl_shim.cpp")
    if not os.path.exists(src):
        return None
    if not force and not _stale(SHIM, [src, LIB]):
        return SHIM
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", os.path.join(REF, "src"), "-I",
           os.path.join(ROOT, "include"), src, "-o", SHIM, "-L", HERE, "-lv2m_cuda", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"shim build failed:\n{r.stderr[-4000:]}")
    return SHIM


def build_dropin(force: bool = False) -> str | None:
    """tests/_bin/dropin_driver: the reference pipeline's relax dispatch over the
    reference's types, linked with the shim and the reference CPU path (a test
    program; built only where the reference headers exist, then it travels)."""
    out = os.path.join(ROOT, "tests", "_bin", "dropin_driver")
    src = os.path.join(ROOT, "tests", "dropin_driver.cpp")
    refso = os.path.join(ROOT, "oracle", "_ref", "libv2m_ref.so")
    if not os.path.isdir(os.path.join(REF, "src")) or not os.path.exists(SHIM) or not os.path.exists(refso):
        return out if os.path.exists(out) else None
    if not force and not _stale(out, [src, SHIM, refso]):
        return out
    os.makedirs(os.path.dirname(out), exist_ok=True)
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(REF, "src"), src, "-o", out,
           "-L", HERE, "-lv2m_relax_cl", "-lv2m_cuda", "-L", os.path.dirname(refso), "-lv2m_ref",
           "-Wl,-rpath,$ORIGIN/../../trussnet_b200:$ORIGIN/../../oracle/_ref", "-fopenmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"drop-in driver build failed:\n{r.stderr[-4000:]}")
    return out


def build_oracle() -> None:
    """The CPU checkers under oracle/ (test infrastructure)."""
    env = dict(os.environ)
    r = subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile"), "all"], capture_output=True,
                       text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")


def build_all(force: bool = False) -> None:
    build_cuda(force=force)
    build_cuda(force=force, check=True)
    build_shim(force=force)
    build_oracle()
    build_dropin(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIB)

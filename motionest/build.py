"""Build libmotionest.so in place (nvcc, sm_100a).  Used by __graft_entry__.build() and by
`python -m motionest.build`.  The library has no torch dependency: it is a plain C ABI."""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libmotionest.so"
BUILD = ROOT / "_build"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xptxas", "-warn-spills", "-I", str(ROOT / "include")]


def sources():
    return sorted(CSRC.glob("*.cu"))


def _gen_consts():
    gen = CSRC / "gen_twiddles.py"
    out = CSRC / "dft_consts.cuh"
    if not out.exists() or out.stat().st_mtime < gen.stat().st_mtime:
        subprocess.run([sys.executable, str(gen)], check=True, stdout=subprocess.DEVNULL)


def _stale():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "motionest.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force=False, verbose=False, jobs=8):
    _gen_consts()
    if not force and not _stale():
        return LIB
    BUILD.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        cmd = [NVCC, *ARCH, *FLAGS, "-dc", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _wait(procs.pop(0))
    for p in procs:
        _wait(p)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp),
           "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def _wait(item):
    src, p = item
    out, _ = p.communicate()
    text = out.decode(errors="replace")
    if p.returncode != 0:
        sys.stderr.write(text)
        raise RuntimeError(f"nvcc failed on {src.name}")
    if text.strip():
        sys.stderr.write(text)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)

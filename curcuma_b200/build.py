"""In-tree build of libgfnff_b200.so (sm_100a) and of the test oracle.

The CUDA sources are compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a``;
the host setup and the C ABI with the system g++ (OpenMP for the O(N^2) setup scans).
Everything lands inside the source tree so that the built library travels with the
repository snapshot.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libgfnff_b200.so"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")
CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"

CU_SOURCES = [CSRC / "device" / "engine.cu", CSRC / "device" / "peaks.cu", CSRC / "device" / "eeq_noalloc.cu",
              CSRC / "device" / "md.cu"]
CPP_SOURCES = [CSRC / "setup" / "topology.cpp", CSRC / "setup" / "parameters.cpp",
               CSRC / "setup" / "linalg.cpp", CSRC / "setup" / "param_file.cpp", CSRC / "setup" / "alpb.cpp", CSRC / "setup" / "topo_cache.cpp",
               CSRC / "capi.cpp"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _headers():
    return (list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.inc"))
            + [ROOT / "include" / "gfnff_b200.h"])


def build_library(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    objs = []
    hdr = _headers()
    for src in CU_SOURCES:
        obj = BUILD / (src.stem + ".cu.o")
        if force or _stale(obj, [src] + hdr):
            _run([NVCC, *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-ccbin", CXX, "-c", src, "-o", obj])
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = BUILD / (src.stem + ".o")
        if force or _stale(obj, [src] + hdr):
            _run([CXX, "-O3", "-std=c++17", "-fPIC", "-fopenmp", f"-I{CUDA / 'include'}", "-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([CXX, "-shared", "-o", LIB, *objs, f"-L{CUDA / 'lib64'}", "-lcudart", "-lcusolver", "-lgomp",
              f"-Wl,-rpath,{CUDA / 'lib64'}"])
    return LIB


def build_oracle(force: bool = False) -> Path:
    """Test infrastructure: the CPU oracle (oracle/_build/liboracle.so)."""
    args = ["make", "-C", str(ROOT / "oracle")]
    if force:
        args.append("-B")
    _run(args)
    return ROOT / "oracle" / "_build" / "liboracle.so"


if __name__ == "__main__":
    force = "--force" in sys.argv
    build_library(force)
    if "--no-oracle" not in sys.argv:
        build_oracle(force)

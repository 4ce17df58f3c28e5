"""Build libjamma_b200.so in-tree with nvcc for sm_100a (B200).

Run ``python -m jamma_b200._build``; the shared library is written next to this
file so that it travels with the source tree.  cuBLAS / cuSOLVER come from the
CUDA toolkit (linked dynamically, rpath set to the toolkit's lib64).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libjamma_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cuda_home() -> Path:
    env = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if env:
        return Path(env)
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parent.parent
    return Path("/usr/local/cuda")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def build(force: bool = False, verbose: bool = False) -> Path:
    srcs = sources()
    deps = srcs + sorted(CSRC.glob("*.cuh")) + sorted((HERE.parent / "include").glob("*.h"))
    if LIB.exists() and not force:
        newest = max(p.stat().st_mtime for p in deps)
        if LIB.stat().st_mtime >= newest:
            return LIB
    cuda = _cuda_home()
    nvcc = str(cuda / "bin" / "nvcc")
    out_dir = HERE / "_objs"
    out_dir.mkdir(exist_ok=True)
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-I", str(HERE.parent / "include")]
    cmds = [[nvcc, "-c", str(src), "-o", str(out_dir / (src.stem + ".o"))] + common for src in srcs]
    objs = [c[4] for c in cmds]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(subprocess.run, c, check=True) for c in cmds]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    link = [nvcc, "-shared", "-o", str(tmp)] + ARCH + objs + [
        "-L", str(cuda / "lib64"), "-lcublas", "-lcusolver", "-ldl",
        "-Xlinker", f"-rpath,{cuda / 'lib64'}",
    ]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

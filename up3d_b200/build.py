"""Builds the up3d CUDA library (sm_100a) in-tree: up3d_b200/lib/libup3d.so.

    python -m up3d_b200.build          # or up3d_b200.build.build()

nvcc compiles every .cu under csrc/ for sm_100a and links one shared object
with the CUDA runtime linked statically, so the library carries no runtime
dependency beyond the driver.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB_DIR = HERE / "lib"
LIB = LIB_DIR / "libup3d.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]
LINK = ["-Xcompiler", "-fopenmp", "-lgomp"]


def sources():
    return sorted(CSRC.glob("*.cu"))


STAMP = LIB_DIR / "libup3d.sources"


def _source_digest() -> str:
    """Digest of every source the library is built from (and the flags)."""
    import hashlib
    h = hashlib.sha256(" ".join(ARCH + FLAGS + LINK).encode())
    deps = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "up3d.h"]
    for p in deps:
        h.update(p.name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()


def _stale() -> bool:
    if not LIB.exists() or not STAMP.exists():
        return True
    return STAMP.read_text().strip() != _source_digest()


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    obj_dir = LIB_DIR / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    procs = []
    objs = []
    for src in sources():
        obj = obj_dir / (src.stem + ".o")
        objs.append(obj)
        cmd = [nvcc, *ARCH, *FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append(f"--- {src.name}\n{text}")
        elif verbose and text.strip():
            print(text)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    digest = _source_digest()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), *LINK]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    STAMP.write_text(digest + "\n")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)

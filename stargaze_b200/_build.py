"""Build recipe for the in-tree CUDA library `libstargaze_b200.so`.

The library is compiled for sm_100a only with nvcc and linked with the static
CUDA runtime, so the built file is self-contained and travels with the source
tree. Rebuilds are skipped when the library is newer than every source.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
CSRC = PACKAGE_DIR / "csrc"
INCLUDE = PACKAGE_DIR.parent / "include"
LIBRARY = PACKAGE_DIR / "libstargaze_b200.so"

SOURCES = ["sg_kernels.cu", "sg_wavefront.cu", "sg_wave_adjoint.cu", "sg_display.cu", "sg_host.cpp", "sg_noalloc.cu"]
HEADERS = ["sg_adjoint.cuh", "sg_device.cuh", "sg_surface.cuh", "sg_integrator.cuh", "sg_air.cuh", "sg_internal.h", "sg_landscape.cuh", "sg_wave_common.cuh"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC,-O3,-fvisibility=hidden",
    "-Xptxas",
    "-v",
    "--expt-relaxed-constexpr",
]


def nvcc_path() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build stargaze_b200")


def _inputs() -> list[Path]:
    files = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS]
    files.append(INCLUDE / "stargaze_b200.h")
    files.append(Path(__file__))
    return files


def up_to_date() -> bool:
    if not LIBRARY.exists():
        return False
    built = LIBRARY.stat().st_mtime
    return all(p.stat().st_mtime <= built for p in _inputs())


def _compile(source: str, objdir: Path) -> tuple[Path, str]:
    obj = objdir / (Path(source).stem + ".o")
    cmd = [nvcc_path(), *ARCH_FLAGS, *NVCC_FLAGS, "-c", "-o", str(obj), str(CSRC / source)]
    proc = subprocess.run(cmd, cwd=str(CSRC), capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}):\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return obj, proc.stdout + proc.stderr


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile the kernels and the C-ABI host runtime into LIBRARY: one nvcc
    per translation unit, run concurrently, then one shared-library link."""
    if not force and up_to_date():
        return LIBRARY
    objdir = PACKAGE_DIR / "_build"
    objdir.mkdir(exist_ok=True)
    workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(lambda s: _compile(s, objdir), SOURCES))
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [nvcc_path(), *ARCH_FLAGS, "-shared", "-o", str(tmp), *[str(obj) for obj, _ in results]]
    proc = subprocess.run(cmd, cwd=str(CSRC), capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({proc.returncode}):\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    report = "".join(log for _, log in results) + proc.stdout + proc.stderr
    if verbose:
        print(report)
    os.replace(tmp, LIBRARY)
    (PACKAGE_DIR / "ptxas_report.txt").write_text(report)
    return LIBRARY


if __name__ == "__main__":
    print(build_library(force=True, verbose=True))

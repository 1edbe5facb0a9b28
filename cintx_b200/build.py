"""Build libcintx_cuda.so in-tree for sm_100a.

Each .cu/.cpp under csrc/ is compiled by nvcc in parallel (objects in cintx_b200/_build/,
rebuilt when the source or any header is newer) and linked with the CUDA runtime statically,
so the library carries no dependency on the runtime version a host application loads.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcintx_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps(path: str, seen: set | None = None) -> set:
    """Files reached through #include "..." from path (recursively)."""
    seen = set() if seen is None else seen
    base = os.path.dirname(path)
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if line.startswith("#include") and '"' in line:
                dep = os.path.normpath(os.path.join(base, line.split('"')[1]))
                if os.path.exists(dep) and dep not in seen:
                    seen.add(dep)
                    _deps(dep, seen)
    return seen


def _ensure_table():
    table = os.path.join(CSRC, "rys_table.bin")
    if not os.path.exists(table):
        subprocess.run([sys.executable, os.path.join(CSRC, "gen_rys_table.py"), "--out", table], check=True)
    return table


def _compile(src: str, obj: str, extra: list[str]) -> tuple[str, int, str]:
    cmd = [NVCC] + FLAGS + ARCH + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    table = _ensure_table()
    todo = []
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        stamp = max([os.path.getmtime(src)] + [os.path.getmtime(d) for d in _deps(src)])
        if src.endswith("rys_table.cu"):
            stamp = max(stamp, os.path.getmtime(table))
        if not os.path.exists(obj) or os.path.getmtime(obj) < stamp:
            extra = []
            if src.endswith("rys_table.cu"):
                extra = ['-DCINTX_RYS_TABLE_PATH="%s"' % table]
            todo.append((src, obj, extra))
    if todo:
        jobs = jobs or os.cpu_count() or 4
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for src, rc, log in ex.map(lambda t: _compile(*t), todo):
                if verbose or rc:
                    sys.stderr.write(log)
                if rc:
                    raise RuntimeError("nvcc failed on %s" % src)
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB + ".tmp"] + objs + ["-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

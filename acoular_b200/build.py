"""Build the native library ``acoular_b200/lib/libacoular_b200.so`` for sm_100a with nvcc.

The library is a plain C-ABI shared object (``include/acoular_b200.h``); Python reaches it through
``ctypes`` (``acoular_b200._native``).  Built in-tree so that it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / 'csrc'
LIB_DIR = PKG / 'lib'
LIB = LIB_DIR / 'libacoular_b200.so'
ROOT = PKG.parent

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC,-O3,-fopenmp', '--expt-relaxed-constexpr',
              '-Xptxas', '-O3']


def sources():
    return sorted(list(CSRC.glob('*.cu')) + list(CSRC.glob('*.cpp')))


def _nvcc() -> str:
    nv = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(nv).exists():
        msg = 'nvcc not found: the CUDA toolkit is required to build acoular_b200'
        raise RuntimeError(msg)
    return nv


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob('*.cuh')) + list(CSRC.glob('*.h')) + list((ROOT / 'include').glob('*.h'))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile every source to an object (in parallel) and link the shared library."""
    if not force and not needs_build():
        return LIB
    nvcc = _nvcc()
    obj_dir = LIB_DIR / 'obj'
    obj_dir.mkdir(parents=True, exist_ok=True)
    procs = []
    objs = []
    for src in sources():
        obj = obj_dir / (src.name + '.o')
        objs.append(obj)
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, '-I', str(ROOT / 'include'), '-c', str(src), '-o', str(obj)]
        if verbose:
            print(' '.join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors='replace')))
        elif verbose and out:
            print(out.decode(errors='replace'), file=sys.stderr)
    if failed:
        msg = '\n'.join(f'--- {s.name}\n{o}' for s, o in failed)
        raise RuntimeError(f'nvcc failed:\n{msg}')
    tmp = LIB.with_suffix('.so.tmp')
    cmd = [nvcc, *ARCH, '-shared', '-o', str(tmp), *map(str, objs), '-lcuda', '-Xcompiler', '-fopenmp']
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)

"""Build ``libdamask_b200.so`` (sm_100a) in-tree with nvcc.

Usage: ``python -m damask_b200.build [--verbose]``.  The library is written next to
this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
LIB = HERE / 'libdamask_b200.so'
SOURCES = ['kernels.cu', 'constitutive.cu', 'dpdf.cu', 'polarization.cu', 'adjoint.cu', 'context.cu', 'noalloc.cu',
           'host_parallel.cu', 'lattice.cpp',
           'vti.cpp', 'driver.cpp']
HEADERS = ['dmk_device.cuh', 'constitutive.cuh', 'kernels.cuh', 'adjoint.cuh', 'lattice.h', 'lattice_tables.h',
           'host_parallel.h']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def _nvcc() -> str:
    cand = [os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc']
    for c in cand:
        if c and Path(c).exists():
            return c
    raise RuntimeError('nvcc not found')


def _host_cxx() -> list[str]:
    # the default CXX of this image may be a wrapper without OpenMP/libstdc++ extras;
    # pin the system compiler as the nvcc host compiler when it exists
    return ['-ccbin', '/usr/bin/g++'] if Path('/usr/bin/g++').exists() else []


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [HERE.parent / 'include' / 'damask_b200.h']
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    objdir = HERE / '_build'
    objdir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    common = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-O3'] + _host_cxx()
    if verbose:
        common += ['-Xptxas', '-v']
    cmds, objs = [], []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + '.o')
        cmd = [nvcc] + common + ['-c', str(CSRC / src), '-o', str(obj)]
        if src.endswith('.cpp'):
            cxx = '/usr/bin/g++' if Path('/usr/bin/g++').exists() else (shutil.which('g++') or 'g++')
            cmd = [cxx, '-O3', '-std=c++17', '-fPIC', '-c', str(CSRC / src), '-o', str(obj)]
        cmds.append(cmd)
        objs.append(str(obj))
    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    tmp = LIB.with_suffix('.so.tmp')
    subprocess.run([nvcc] + ARCH + _host_cxx() + ['-shared', '-o', str(tmp)] + objs + ['-lcufft', '-lcudart', '-lz'], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    build(verbose='--verbose' in sys.argv, force=True)
    print(LIB)

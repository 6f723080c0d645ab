"""Build the engine's native artefacts in-tree.

    python -m lbflow_b200.build            # library + LBFlow command line
    python -m lbflow_b200.build --force    # rebuild everything

Outputs (git-ignored, shipped with the working tree):
    lbflow_b200/lib/liblbflow_b200.so   the C-ABI library (include/lbflow.h)
    lbflow_b200/lib/LBFlow              the C++11 host driver (input.prm CLI)

Every CUDA translation unit is compiled for sm_100a only.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / 'csrc'
HOST = CSRC / 'host'
LIB = PKG / 'lib'
OBJ = PKG / '_build'
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVFLAGS = ['-std=c++17', '-O3', '-lineinfo', '--expt-relaxed-constexpr', '-Xcompiler', '-fPIC',
           '-Xcompiler', '-O3'] + ARCH
CUDA_UNITS = ['engine.cu', 'scsp_launch.cu', 'color_launch.cu', 'noalloc.cu', 'batch.cu', 'conv.cu', 'darcy.cu']
HOST_UNITS = ['main.cpp', 'prm.cpp', 'io.cpp', 'simulation.cpp']
LIBNAME = 'liblbflow_b200.so'


def _newer(target, sources):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _headers(d):
    return [p for p in d.glob('*') if p.suffix in ('.h', '.cuh', '.hpp')]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('build failed: ' + ' '.join(map(str, cmd)) + '\n' + r.stdout + r.stderr)
    return r


def build(force=False, verbose=False, jobs=None):
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    deps = _headers(CSRC) + list((ROOT / 'include').glob('*.h'))
    jobs = jobs or min(8, os.cpu_count() or 4)
    objs = []
    cmds = []
    for u in CUDA_UNITS:
        src = CSRC / u
        obj = OBJ / (u + '.o')
        objs.append(obj)
        if force or _newer(obj, [src] + deps):
            cmds.append([NVCC] + NVFLAGS + ['-c', str(src), '-o', str(obj)])
    with cf.ThreadPoolExecutor(jobs) as ex:
        for r in ex.map(_run, cmds):
            if verbose:
                print(r.stdout + r.stderr, end='')
    lib = LIB / LIBNAME
    if force or _newer(lib, objs):
        _run([NVCC, '-shared'] + ARCH + ['-o', str(lib)] + [str(o) for o in objs] + ['-lcudart'])
    # Host driver: C++11, talks to the engine only through include/lbflow.h.
    exe = LIB / 'LBFlow'
    hsrc = [HOST / u for u in HOST_UNITS]
    if all(p.exists() for p in hsrc) and (force or _newer(exe, hsrc + _headers(HOST) + [lib])):
        _run(['g++', '-std=c++11', '-O2', '-Wall', '-pthread', '-I', str(ROOT / 'include'), '-o', str(exe)]
             + [str(p) for p in hsrc]
             + ['-L', str(LIB), '-llbflow_b200', '-Wl,-rpath,$ORIGIN'])
    return lib


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose', action='store_true')
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == '__main__':
    main()

"""Build libnngp_b200.so (sm_100a) in-tree with nvcc.

    python -m nngpr_b200.build [--verbose-ptxas] [--force]

Compiles ``nngpr_b200/csrc/*.cu`` in parallel into ``nngpr_b200/_build/*.o`` and links
``nngpr_b200/libnngp_b200.so`` (static CUDA runtime, no torch dependency).  Objects are
rebuilt when a source or header is newer than the object.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
BUILD = os.path.join(PKG, '_build')
LIB = os.path.join(PKG, 'libnngp_b200.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ARCH + ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
                     '-I', os.path.join(ROOT, 'include')]


def nvcc() -> str:
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def _deps() -> list[str]:
    return glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(ROOT, 'include', '*.h'))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _deps())


def build(force: bool = False, verbose_ptxas: bool = False, jobs: int | None = None) -> str:
    """Compile and link; returns the path of the shared library."""
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    objs = [os.path.join(BUILD, os.path.basename(s)[:-3] + '.o') for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, s)]
    extra = ['-Xptxas', '-v'] if verbose_ptxas else []

    def compile_one(so):
        s, o = so
        cmd = [nvcc()] + NVCC_FLAGS + extra + ['-c', s, '-o', o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r.returncode, r.stdout + r.stderr

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for s, rc, log in ex.map(compile_one, todo):
                if log.strip() and (rc != 0 or verbose_ptxas):
                    sys.stderr.write(log)
                if rc != 0:
                    raise RuntimeError(f'nvcc failed on {s}')
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        tmp = LIB + '.tmp'
        cmd = [nvcc()] + ARCH + ['-shared', '-o', tmp] + objs + ['-cudart', 'static']
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError('link failed')
        os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--force', action='store_true')
    ap.add_argument('--verbose-ptxas', action='store_true')
    args = ap.parse_args()
    print(build(force=args.force, verbose_ptxas=args.verbose_ptxas))


if __name__ == '__main__':
    main()

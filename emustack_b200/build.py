"""Build libemustack_gsm.so (all CUDA sources in csrc/) for sm_100a, in tree.

    python -m emustack_b200.build          # or emustack_b200.build.build_library()

The library is a plain C-ABI shared object (declarations in
include/emustack_gsm.h); Python reaches it through ctypes.  Sources are
compiled one object per .cu file, in parallel, then linked once.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, 'libemustack_gsm.so')
OBJDIR = os.path.join(HERE, '_build')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC',
         '-Xcompiler', '-ffp-contract=off', '--expt-relaxed-constexpr',
         '-I' + os.path.join(ROOT, 'include')]
# Sources whose floating-point operations keep the roundings written in the
# source: with -fmad=false every multiply and add is emitted with an explicit
# rounding mode, so the assembler fuses none of them and every launch variant
# of a kernel (other register budgets, other schedules) returns the same bits.
# The fused multiply-adds of these files are their explicit fma() calls.
EXACT_ROUNDING = {'film_stack.cu', 'film_varlen.cu', 'film_ring.cu'}


def nvcc():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def _newer(src_files, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_files)


def build_library(force=False, verbose=False):
    """Compile csrc/*.cu into emustack_b200/libemustack_gsm.so; returns its path."""
    srcs = sorted(glob.glob(os.path.join(CSRC, '*.cu')))
    headers = glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(CSRC, '*.h')) + \
        glob.glob(os.path.join(ROOT, 'include', '*.h'))
    os.makedirs(OBJDIR, exist_ok=True)
    if not force and not _newer(srcs + headers, LIB):
        return LIB
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + '.o')
        if not force and not _newer([src] + headers, obj):
            return obj
        extra = ['-fmad=false'] if os.path.basename(src) in EXACT_ROUNDING else []
        cmd = [cc] + ARCH + FLAGS + extra + ['-c', src, '-o', obj]
        if verbose:
            print(' '.join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('nvcc failed on %s:\n%s\n%s' % (src, r.stdout, r.stderr))
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB + '.tmp'
    cmd = [cc] + ARCH + ['-shared', '-cudart', 'static', '-o', tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('link failed:\n%s\n%s' % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build_library(force='--force' in sys.argv, verbose=True))

"""Builds libmom25d_b200.so in-tree with nvcc for sm_100a (the only target): python -m mom25d_b200.build"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libmom25d_b200.so')
SOURCES = ['capi.cu', 'green.cu', 'fill.cu', 'vias.cu', 'gmres.cu', 'lu.cu', 'umma.cu', 'noalloc.cu', 'trsv_sb.cu']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3', '-std=c++17',
         '-Xcompiler', '-fPIC', '-shared', '-Xptxas', '-O3', '--expt-relaxed-constexpr']


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(SRC, f) for f in os.listdir(SRC)] + [os.path.join(HERE, '..', 'include', 'mom25d_b200.h')]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    cmd = [NVCC] + FLAGS + [os.path.join(SRC, s) for s in SOURCES] + ['-o', LIB + '.tmp', '-lcuda']
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))

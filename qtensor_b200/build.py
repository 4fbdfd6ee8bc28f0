"""Build ``libqtb.so`` (sm_100a) in-tree with nvcc.

Run ``python -m qtensor_b200.build`` (or ``__graft_entry__.build()``).  The
library is written next to this file so it travels with the source tree.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libqtb.so')
SOURCES = ['plan.cpp', 'qtb.cu', 'contract.cu']
ARCH_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc_path():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def needs_build():
    if not os.path.exists(LIB):
        return True
    mtime = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, '..', 'include', 'qtb.h'))
    return any(os.path.getmtime(d) > mtime for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    cmd = [nvcc_path(), *ARCH_FLAGS, '-lineinfo', '-O3', '-std=c++17', '-shared',
           '-Xcompiler', '-fPIC,-O3', '-Xptxas', '-v' if verbose else '-O3',
           '-o', LIB + '.tmp'] + [os.path.join(CSRC, s) for s in SOURCES] + ['-lpthread']
    proc = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError('nvcc failed:\n' + proc.stdout + proc.stderr)
    if verbose:
        sys.stderr.write(proc.stdout + proc.stderr)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)

"""Build libbyteqc_b200.so (sm_100a) in-tree.

The 55 shell-quartet class launchers are compiled as separate translation
units so nvcc runs them in parallel; everything links into one shared library
next to this file.  ``python -m byteqc_b200.build`` or ``build()``.
"""
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libbyteqc_b200.so')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')

NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-I', CSRC, '-I', INCLUDE,
         '-ccbin', 'g++']

PAIRS = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (3, 2), (3, 3)]
SOURCES = ['jk_dispatch.cu', 'schwarz.cu', 'capi.cu', 'int1e.cu', 'rys_table.cu', 'peak.cu', 'mlp.cu', 'plan.cu']


def classes():
    out = []
    for a in range(len(PAIRS)):
        for b in range(a + 1):
            out.append(PAIRS[a] + PAIRS[b])
    return out


def _class_units():
    """One wrapper translation unit per class launcher."""
    os.makedirs(BUILD, exist_ok=True)
    units = []
    for c in classes():
        name = 'cls_%d%d%d%d.cu' % c
        path = os.path.join(BUILD, name)
        src = ('#include "jk_kernels.cuh"\n'
               'int bqc_class_%d%d%d%d(const JKArgs &a, const JKTask &t, int fp32, '
               'cudaStream_t s) {\n  return bqc::launch_class<%d, %d, %d, %d>(a, t, fp32, s);\n}\n'
               % (c + c))
        if not os.path.exists(path) or open(path).read() != src:
            with open(path, 'w') as f:
                f.write(src)
        units.append(path)
    return units


_INCLUDE_RE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src, seen=None):
    """The source file and every local header it includes, recursively
    (looked up next to the including file, then in csrc/ and include/)."""
    seen = set() if seen is None else seen
    if src in seen:
        return seen
    seen.add(src)
    with open(src) as f:
        text = f.read()
    for name in _INCLUDE_RE.findall(text):
        for d in (os.path.dirname(src), CSRC, INCLUDE):
            path = os.path.join(d, name)
            if os.path.exists(path):
                _deps(os.path.abspath(path), seen)
                break
    return seen


def _compile(src, extra=()):
    obj = os.path.join(BUILD, os.path.basename(src).replace('.cu', '.o'))
    if os.path.exists(obj) and \
            os.path.getmtime(obj) > max(os.path.getmtime(d) for d in _deps(os.path.abspath(src))):
        return obj
    cmd = [NVCC] + ARCH + FLAGS + list(extra) + ['-c', src, '-o', obj]
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s' % (src, r.stderr[-4000:]))
    if os.environ.get('BQC_BUILD_VERBOSE'):
        print('%6.1fs %s' % (time.time() - t0, os.path.basename(src)), file=sys.stderr)
    return obj


def build(jobs=None, verbose=True):
    if shutil.which(NVCC) is None:
        raise RuntimeError('nvcc not found: the CUDA library cannot be built')
    units = [os.path.join(CSRC, s) for s in SOURCES] + _class_units()
    jobs = jobs or os.cpu_count() or 4
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(_compile, units))
    if os.path.exists(LIB) and os.path.getmtime(LIB) > max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC] + ARCH + ['-shared', '-o', LIB] + objs + ['-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('link failed:\n' + r.stderr[-4000:])
    if verbose:
        print('built', LIB, file=sys.stderr)
    return LIB


if __name__ == '__main__':
    build()

"""Build ``frfs_b200/_lib/libbdgfs.so`` from ``frfs_b200/csrc/*.cu``.

AOT build for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
nvcc cross-compiles without a GPU.  Usage: ``python -m frfs_b200.build``.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUTDIR = os.path.join(HERE, '_lib')
LIB = os.path.join(OUTDIR, 'libbdgfs.so')
ROOT = os.path.dirname(HERE)

NVCC_FLAGS = ['-std=c++17', '-O3', '-lineinfo',
              '-gencode', 'arch=compute_100a,code=sm_100a',
              '-Xcompiler', '-fPIC', '-Xcompiler', '-O2',
              '--expt-relaxed-constexpr', '-diag-suppress', '177']


def _nvcc():
    cand = os.path.join(os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin', 'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def sources():
    return sorted(glob.glob(os.path.join(CSRC, '*.cu')))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = (sources() + glob.glob(os.path.join(CSRC, '*.cuh'))
            + glob.glob(os.path.join(ROOT, 'include', '*.h')))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile every CUDA source into one shared library (in-tree)."""
    if not force and not _stale():
        return LIB
    gen = os.path.join(CSRC, 'gen_fft.py')
    subprocess.check_call([sys.executable, gen])
    os.makedirs(OUTDIR, exist_ok=True)
    cmds, objs = [], []
    for src in sources():
        obj = os.path.join(OUTDIR, os.path.basename(src)[:-3] + '.o')
        cmd = [_nvcc(), *NVCC_FLAGS, '-I', os.path.join(ROOT, 'include'),
               '-c', src, '-o', obj]
        if verbose:
            cmd.insert(1, '-Xptxas=-v')
            print(' '.join(cmd), flush=True)
        cmds.append(cmd)
        objs.append(obj)
    # one nvcc process per source, as many at once as there are host cores
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        list(ex.map(subprocess.check_call, cmds))
    tmp = LIB + '.tmp'
    subprocess.check_call([_nvcc(), '-shared', '-gencode',
                           'arch=compute_100a,code=sm_100a', *objs, '-o', tmp,
                           '-lcudart'])
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))

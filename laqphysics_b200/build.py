"""Build libhelium_b200.so (all CUDA sources, sm_100a) in-tree.

Usage: ``python -m laqphysics_b200.build [--force]``.  The library lands in
``laqphysics_b200/_lib/`` so it travels with the source tree; nothing is installed
into site-packages and no JIT cache is used.
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / 'csrc'
LIBDIR = HERE / '_lib'
LIBRARY = LIBDIR / 'libhelium_b200.so'
INCLUDE = HERE.parent / 'include'

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr', '-Xcompiler', '-Wall']
COMPILE_FLAGS = FLAGS
LIBS = ['-lnvrtc', '-lcuda']


def nvcc():
    found = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not Path(found).exists():
        raise RuntimeError('nvcc not found; the CUDA toolkit is required to build libhelium_b200.so')
    return found


def sources():
    return sorted(CSRC.glob('*.cu'))


def dependencies():
    return sources() + sorted(CSRC.glob('*.cuh')) + sorted(INCLUDE.glob('*.h')) + [Path(__file__)]


def up_to_date():
    if not LIBRARY.exists():
        return False
    stamp = LIBRARY.stat().st_mtime
    return all(p.stat().st_mtime <= stamp for p in dependencies())


def _compile(source, objdir, verbose):
    obj = objdir / (source.stem + '.o')
    cmd = [nvcc(), *ARCH, *COMPILE_FLAGS, f'-I{INCLUDE}', '-c', str(source), '-o', str(obj)]
    if verbose:
        cmd.insert(1, '-Xptxas=-v')
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f'nvcc failed on {source.name}:\n' + result.stdout + result.stderr)
    if verbose:
        sys.stderr.write(result.stderr)
    return obj


def build(force=False, verbose=False):
    """Compile every source to an object file in parallel (one nvcc per file), then link."""
    if not force and up_to_date():
        return LIBRARY
    LIBDIR.mkdir(exist_ok=True)
    objdir = LIBDIR / 'obj'
    objdir.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as pool:
        objects = list(pool.map(lambda src: _compile(src, objdir, verbose), sources()))
    tmp = LIBRARY.with_suffix('.so.tmp')
    cmd = [nvcc(), *ARCH, '-shared', '-Xcompiler', '-fPIC', *map(str, objects), '-o', str(tmp), *LIBS]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError('nvcc link failed:\n' + result.stdout + result.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == '__main__':
    parser = argparse.ArgumentParser()
    parser.add_argument('--force', action='store_true')
    parser.add_argument('--verbose', action='store_true')
    args = parser.parse_args()
    print(build(args.force, args.verbose))

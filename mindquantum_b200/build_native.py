"""Build libmqb200.so (the CUDA kernels + C ABI) in-tree for sm_100a.

    python -m mindquantum_b200.build_native        # rebuild if any source changed

The library is compiled with nvcc for ``arch=compute_100a,code=sm_100a`` only and links the
CUDA runtime statically; beyond the NVIDIA driver it needs the toolkit's NVRTC (libnvrtc.so.12),
which compiles the generated pass kernels at run time.
"""
import os
import subprocess
import time
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
LIB = os.path.join(HERE, 'libmqb200.so')
FUSED = ['fused_fwd_c64.cu', 'fused_fwd_c128.cu', 'fused_bwd_c64.cu', 'fused_bwd_c128.cu']
SOURCES = ['kernels.cu', *FUSED, 'capi.cpp', 'scheduler.cpp', 'noalloc.cu', 'jit.cpp']
HEADERS = ['kernels.cuh', 'mqb_internal.h', 'mqb_gate_ids.h', 'fused_impl.cuh', 'regops.cuh', 'regmath.cuh',
           'tile.cuh', 'jit_abi.h', 'jit.h', 'pipe.cuh']
# headers compiled again at run time by NVRTC for the generated pass kernels (embedded as text)
JIT_HEADERS = [('kJitRegmath', 'regmath.cuh'), ('kJitTile', 'tile.cuh'), ('kJitAbi', 'jit_abi.h'),
               ('kJitPipe', 'pipe.cuh')]
# NVRTC from the CUDA toolkit the library is built with (found again at run time through the rpath)
CUDA_LIB = '/usr/local/cuda/lib64'
NVRTC_LIBS = [f'-L{CUDA_LIB}', '-lnvrtc', '-Xlinker', f'-rpath={CUDA_LIB}']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def _nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return 'nvcc'


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(INCLUDE, 'mqb200.h')]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False):
    """Compile the library unless it is newer than every source."""
    if not force and up_to_date():
        return LIB
    # outputs are stamped with the build's start time, so a source edited while the build runs
    # leaves them stale for the next build
    t_start = time.time()
    bdir = os.path.join(os.path.dirname(HERE), '_build', 'mqb200')
    os.makedirs(bdir, exist_ok=True)
    env = dict(os.environ)
    env.pop('CC', None)
    env.pop('CXX', None)
    common = ['-O3', '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
              '-Xcompiler', '-fvisibility-inlines-hidden', '-ccbin', 'g++', f'-I{INCLUDE}']

    def obj(name):
        return os.path.join(bdir, os.path.splitext(name)[0] + '.o')

    # the NVRTC headers as C++ string literals
    embed = os.path.join(bdir, 'jit_embed.cpp')
    text = ['// generated by build_native.py from the headers below', 'namespace mqb {']
    for sym, name in JIT_HEADERS:
        body = open(os.path.join(CSRC, name), encoding='utf8').read()
        if ')MQBJIT"' in body:
            raise RuntimeError(f'{name} contains the raw-string delimiter')
        text.append(f'extern const char *const {sym} = R"MQBJIT({body})MQBJIT";')
    text.append('}  // namespace mqb')
    text = '\n'.join(text) + '\n'
    if not os.path.exists(embed) or open(embed, encoding='utf8').read() != text:
        with open(embed, 'w', encoding='utf8') as f:
            f.write(text)

    compiles = [[_nvcc(), *ARCH, '-lineinfo', *common, '-c', os.path.join(CSRC, f), '-o', obj(f)]
                for f in ('kernels.cu', *FUSED, 'noalloc.cu')]
    compiles.append([_nvcc(), *ARCH, '-lineinfo', *common, '-x', 'cu', '-c', os.path.join(CSRC, 'capi.cpp'),
                     '-o', obj('capi.cpp')])
    compiles.append([_nvcc(), *common, '-x', 'c++', '-c', os.path.join(CSRC, 'scheduler.cpp'),
                     '-o', obj('scheduler.cpp')])
    compiles.append([_nvcc(), *common, '-x', 'c++', '-c', os.path.join(CSRC, 'jit.cpp'), '-o', obj('jit.cpp')])
    compiles.append([_nvcc(), *common, '-x', 'c++', '-c', embed, '-o', obj('jit_embed.cpp')])
    link = [_nvcc(), *ARCH, '-shared', '-cudart', 'static', '-ccbin', 'g++',
            *[obj(f) for f in SOURCES], obj('jit_embed.cpp'), *NVRTC_LIBS, '-lpthread', '-ldl', '-o', LIB + '.tmp']
    def newest_dep(src):
        # the source and every header it includes, transitively (quoted includes of this tree)
        seen, todo, newest = set(), [src], 0.0
        while todo:
            f = todo.pop()
            if f in seen or not os.path.exists(f):
                continue
            seen.add(f)
            newest = max(newest, os.path.getmtime(f))
            with open(f, encoding='utf8') as fh:
                for line in fh:
                    line = line.strip()
                    if line.startswith('#include "'):
                        todo.append(os.path.normpath(os.path.join(os.path.dirname(f), line.split('"')[1])))
        return newest

    def stale(cmd):
        out = cmd[cmd.index('-o') + 1]
        src = cmd[cmd.index('-c') + 1]
        return force or not os.path.exists(out) or os.path.getmtime(out) < newest_dep(src)

    def run(cmd):
        if verbose:
            print(' '.join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
        else:
            out = cmd[cmd.index('-o') + 1]
            os.utime(out, (t_start, t_start))
        return res.returncode

    todo = [c for c in compiles if stale(c)]
    # the fused translation units dominate the build time: compile everything in parallel
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as pool:
        codes = list(pool.map(run, todo))
    if any(codes) or run(link) != 0:
        raise RuntimeError('building libmqb200.so failed')
    os.replace(LIB + '.tmp', LIB)
    os.utime(LIB, (t_start, t_start))
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))

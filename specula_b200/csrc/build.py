"""Build libspecula_b200.so (sm_100a) in-tree with nvcc.

    python -m specula_b200.csrc.build        # or python specula_b200/csrc/build.py

The library has a plain C ABI (include/specula_b200.h) and links the CUDA
runtime statically, so it only needs the driver at run time.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, 'libspecula_b200.so')
SOURCES = ['sb_common.cu', 'sb_sh.cu', 'sb_detector.cu', 'sb_control.cu', 'sb_atmo.cu', 'sb_adjoint.cu', 'sb_psf.cu',
           'sb_psf_tc.cu', 'sb_mc.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    # every source, every private header of this directory, the ABI header and this script
    headers = [os.path.join(HERE, f) for f in sorted(os.listdir(HERE)) if f.endswith('.cuh')]
    deps = [os.path.join(HERE, s) for s in SOURCES] + headers + [os.path.join(ROOT, 'include', 'specula_b200.h'),
                                                                 __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return OUT
    cmd = [nvcc(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '-shared', '-Xcompiler', '-fPIC',
           '-cudart', 'static', '-I', os.path.join(ROOT, 'include'), *extra,
           '-o', OUT + '.tmp'] + [os.path.join(HERE, s) for s in SOURCES]
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + '.tmp', OUT)
    return OUT


if __name__ == '__main__':
    extra = ['-Xptxas', '-v'] if '--ptxas-v' in sys.argv else []
    print(build(force='--force' in sys.argv or bool(extra), verbose=True, extra=extra))

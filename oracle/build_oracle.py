"""Build recipe for the CPU checker (test infrastructure only).

Two shared libraries:

* ``oracle/lib/libnif_oracle.so`` -- the C restatement in ``nif_oracle.c``,
  compiled with ``-ffp-contract=off`` so its doubles match natinterp3d's
  (which is built ``-std=c11`` without ``-march``, hence without FMA).
* ``oracle/_ref/libnatinterp3d_ref.so`` -- natinterp3d's own C sources
  (``unity.c`` of the natinterp3d source tree, read in place, never copied)
  plus ``ref_shim.c``, with the compile flags of natinterp3d's ``setup.py``
  (``-std=c11 -O3 -fno-math-errno -flto -fopenmp -DUSE_LIST_NODE_ALLOCATOR``).
  Only built where the natinterp3d sources exist; elsewhere the prebuilt
  file is used as is.

Run ``python oracle/build_oracle.py`` or call :func:`build`.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, 'lib')
REF_DIR = os.path.join(HERE, '_ref')
ORACLE_SO = os.path.join(LIB_DIR, 'libnif_oracle.so')
REF_SO = os.path.join(REF_DIR, 'libnatinterp3d_ref.so')

# natinterp3d's Linux flags (setup.py:17-22, 36)
REF_CFLAGS = ['-std=c11', '-O3', '-fno-math-errno', '-flto', '-fopenmp',
              '-DUSE_LIST_NODE_ALLOCATOR', '-DNPY_NO_DEPRECATED_API=NPY_1_7_API_VERSION']
REF_LDFLAGS = ['-fopenmp', '-flto', '-lm', '-lpthread']


def ref_source_dir():
    """natinterp3d's C sources, located as the product's build recipe does
    (NATINTERP3D_SRC, an importable natinterp3d package, the default checkout)."""
    sys.path.insert(0, os.path.dirname(HERE))
    from natinterp3d_b200 import _build
    return _build.ref_source_dir()


def _cc():
    # /usr/bin/gcc ships libgomp's spec file; some images put another gcc first on PATH
    return '/usr/bin/gcc' if os.path.exists('/usr/bin/gcc') else 'gcc'


def _run(cmd):
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


# the exact-predicate arithmetic shared with the product (nif_exact.h)
EXACT_DIR = os.path.join(os.path.dirname(HERE), 'natinterp3d_b200', 'csrc')


def build_oracle(force=False):
    os.makedirs(LIB_DIR, exist_ok=True)
    src = os.path.join(HERE, 'nif_oracle.c')
    deps = [src, __file__, os.path.join(EXACT_DIR, 'nif_exact.h')]
    if force or _stale(ORACLE_SO, deps):
        _run([_cc(), '-O2', '-std=c11', '-ffp-contract=off', '-fno-fast-math', '-fPIC',
              '-shared', '-Wall', '-I', EXACT_DIR, '-o', ORACLE_SO, src, '-lm'])
    return ORACLE_SO


def build_ref(force=False):
    """Compile natinterp3d's own query code; returns the .so path or None."""
    ref_src = ref_source_dir()
    unity = os.path.join(ref_src, 'unity.c')
    if not os.path.exists(unity):
        return REF_SO if os.path.exists(REF_SO) else None
    os.makedirs(REF_DIR, exist_ok=True)
    shim = os.path.join(HERE, 'ref_shim.c')
    deps = [shim, __file__] + [os.path.join(ref_src, f) for f in os.listdir(ref_src)
                               if f.endswith(('.c', '.h'))]
    if force or _stale(REF_SO, deps):
        _run([_cc()] + REF_CFLAGS + ['-fPIC', '-shared', '-w', '-fvisibility=hidden', '-I', ref_src, '-o', REF_SO,
                                     shim] + REF_LDFLAGS)
    return REF_SO


def build(force=False):
    build_oracle(force)
    build_ref(force)


if __name__ == '__main__':
    build(force='--force' in sys.argv)
    print(ORACLE_SO)
    print(REF_SO if os.path.exists(REF_SO) else '(natinterp3d sources not found: _ref not built)')

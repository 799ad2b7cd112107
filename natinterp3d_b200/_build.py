"""Build recipes for the two native libraries of natinterp3d_b200.

``lib/libnif_mesh.so``
    Host-side Delaunay constructor.  ``csrc/mesh_export.c`` is compiled with
    natinterp3d's own constructor sources on the include path (they are read
    where they lie, never copied into this tree) and with natinterp3d's
    ``setup.py`` flags, so the mesh -- including the constructor's random
    perturbation of degenerate vertices -- is the one natinterp3d builds.

``lib/libnif_cuda.so``
    The sm_100a kernels and the C ABI declared in ``include/natinterp3d_b200.h``,
    compiled by nvcc with ``-fmad=false`` (no fused multiply-add contraction:
    every FP64 expression rounds exactly as natinterp3d's C does) and a static
    CUDA runtime.

Both are built in-tree so that a prebuilt copy travels with the source tree;
where the natinterp3d sources are absent the prebuilt constructor is used.
"""
import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, 'csrc')
LIB_DIR = os.path.join(PKG_DIR, 'lib')
INCLUDE_DIR = os.path.join(REPO_DIR, 'include')
MESH_SO = os.path.join(LIB_DIR, 'libnif_mesh.so')
CUDA_SO = os.path.join(LIB_DIR, 'libnif_cuda.so')
# Where this recipe looks for natinterp3d's C sources, in order: the
# NATINTERP3D_SRC environment variable; an importable natinterp3d package
# whose directory holds them; the source checkout this build reads by default.
CHECKOUT_REF_SRC = '/root/reference/src/natinterp3d'

# natinterp3d's Linux compile flags (setup.py:17-22, 36 of natinterp3d)
MESH_CFLAGS = ['-std=c11', '-O3', '-fno-math-errno', '-flto', '-fopenmp',
               '-DUSE_LIST_NODE_ALLOCATOR', '-fvisibility=hidden']
MESH_LDFLAGS = ['-fopenmp', '-flto', '-lm', '-lpthread']

CUDA_SOURCES = ['nif_cuda.cu', 'nif_delaunay.cu']
NVCC_FLAGS = ['-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo',
              '-fmad=false', '--prec-div=true', '--prec-sqrt=true', '-Xcompiler', '-fPIC',
              '-Xcompiler', '-fvisibility=hidden', '-cudart', 'static', '--expt-relaxed-constexpr']


def _has_sources(d):
    return bool(d) and os.path.exists(os.path.join(d, 'delaunay.c'))


def ref_source_dir():
    """Directory of natinterp3d's C sources (may not exist where only the
    prebuilt libraries travel)."""
    env = os.environ.get('NATINTERP3D_SRC')
    if env:
        return env
    try:
        import importlib.util
        spec = importlib.util.find_spec('natinterp3d')
        if spec is not None and spec.origin:
            d = os.path.dirname(spec.origin)
            if _has_sources(d):
                return d
    except (ImportError, ValueError):
        pass
    return CHECKOUT_REF_SRC


def _cc():
    return '/usr/bin/gcc' if os.path.exists('/usr/bin/gcc') else 'gcc'


def _nvcc():
    cand = os.path.join(os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin', 'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_mesh_lib(force=False):
    ref_src = ref_source_dir()
    src = os.path.join(CSRC, 'mesh_export.c')
    if not os.path.exists(os.path.join(ref_src, 'delaunay.c')):
        if os.path.exists(MESH_SO):
            return MESH_SO
        raise RuntimeError('natinterp3d constructor sources not found at %r and no prebuilt %s'
                           % (ref_src, MESH_SO))
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = [src, __file__] + [os.path.join(ref_src, f) for f in os.listdir(ref_src)
                              if f.endswith(('.c', '.h'))]
    if force or _stale(MESH_SO, deps):
        subprocess.run([_cc()] + MESH_CFLAGS + ['-fPIC', '-shared', '-w', '-I', ref_src,
                                                '-o', MESH_SO, src] + MESH_LDFLAGS, check=True)
    return MESH_SO


def cuda_deps():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cu', '.cuh', '.h'))]
    out += [os.path.join(INCLUDE_DIR, f) for f in os.listdir(INCLUDE_DIR) if f.endswith('.h')]
    return out + [__file__]


def build_cuda_lib(force=False, extra_flags=()):
    os.makedirs(LIB_DIR, exist_ok=True)
    if not force and not _stale(CUDA_SO, cuda_deps()):
        return CUDA_SO
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    cmd = [_nvcc()] + NVCC_FLAGS + list(extra_flags) + ['-I', INCLUDE_DIR, '-I', CSRC,
                                                       '-shared', '-o', CUDA_SO] + srcs
    subprocess.run(cmd, check=True)
    return CUDA_SO


def build(force=False):
    build_mesh_lib(force)
    build_cuda_lib(force)


if __name__ == '__main__':
    build(force='--force' in sys.argv)
    print(MESH_SO)
    print(CUDA_SO)

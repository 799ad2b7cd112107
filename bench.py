"""Benchmark of the Sibson query path on B200.

Default workload (one step = one pass of the hot path over one batch):
plain interpolate at scale -- 1,000,000 keys uniform in [0,1]^3 (float64),
10,000,000 queries uniform in [0.02,0.98]^3 (float64), values D=3 float32
N(0,1), seed 1.  The Delaunay construction (natinterp3d's own, on the host)
is done once before timing, on both arms, as in natinterp3d's Interpolator.

Our arm prints one JSON line with
  value   queries/s with inputs resident in HBM (CUDA events, max over ranks)
  e2e     queries/s through Interpolator.interpolate with host numpy buffers
          (host->device copy of the queries and values, device->host copy of
          the result inside the timed region)
  roofline, cpu_baseline, clocks, gpu_launches.
``--impl reference`` times natinterp3d's own CPU implementation (its C
sources compiled in oracle/_ref; mesh built by its own constructor) with all
host threads on a bounded sample of the same workload.

Multi-GPU (torchrun): every rank builds the same mesh and processes its own
batch of queries (weak scaling, no data-path collective).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'Sibson queries/s at 1M keys (plain, fwd+bwd, batched) vs CPU OpenMP, 1 B200'
WORKLOAD = ('plain interpolate at scale: {keys:,} keys U[0,1]^3 float64, {queries:,} queries '
            'U[0.02,0.98]^3 float64, values D={dim} float32 N(0,1), seed {seed}')

# DRAM bytes (read + write) per row of one launch, from the ncu captures in
# profiles/ (TRAFFIC_SOURCE)
TRAFFIC_PER_ROW = {'k_rows_volume': (796.55e6 + 52.46e6) / 1_000_000}
TRAFFIC_SOURCE = ('one 1,000,000-row k_rows_volume launch of the 1M-key / 10M-query workload '
                  '(dram__bytes_read.sum + dram__bytes_write.sum, 1 pass; '
                  'profiles/k_rows_volume_200k_keys_2M_queries.md)')

# FP64 operations per unit of work, counted as natinterp3d's C evaluates them
# (each add, subtract, multiply and divide is one flop; no fused multiply-add)
FLOPS = {'orient': 23, 'insphere': 77, 'tet_cc': 79, 'tri_cc': 56, 'subcell': 89}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=5)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    p.add_argument('--keys', type=int, default=1_000_000)
    p.add_argument('--queries', type=int, default=10_000_000)
    p.add_argument('--dim', type=int, default=3)
    p.add_argument('--seed', type=int, default=1)
    p.add_argument('--e2e-steps', type=int, default=3)
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--predicates', default='fast', choices=['fast', 'audit', 'exact'],
                   help="geometric predicates: natinterp3d's fast signs (default), the same "
                        "signs with uncertain evaluations counted, or exact signs")
    p.add_argument('--mode', default='plain', choices=['plain', 'fwdbwd', 'batched'],
                   help='plain: the interpolate workload above; fwdbwd: the differentiable '
                        'workload (200k keys, 1M queries in [0.1,0.9]^3, D=16, seed 3); '
                        'batched: 512 uneven problems (keys log-uniform [500, 100k], queries '
                        'log-uniform [1k, 200k], boxes of side 0.5-2, D=4 float32, seed 4)')
    p.add_argument('--problems', type=int, default=512)
    p.add_argument('--no-legs', action='store_true',
                   help='plain leg only (skip get_weights, fwd+bwd and batched sub-results)')
    p.add_argument('--no-tune', action='store_true',
                   help="skip the autotuner (untimed setup) and keep the library's default "
                        "launch settings")
    p.add_argument('--tuning', default=None,
                   help='fixed launch settings blocks_per_sm,bucket_shift,tile (e.g. 8,0,8) '
                        'instead of the autotuner')
    return p.parse_args()


def fixed_tuning(args):
    if not args.tuning:
        return None
    b, s, t = (int(x) for x in args.tuning.split(','))
    return {'blocks_per_sm': b, 'bucket_shift': s, 'tile': t}


def make_data(args, rank=0):
    rng = np.random.default_rng(args.seed)
    keys = rng.uniform(0.0, 1.0, (args.keys, 3))
    values = rng.standard_normal((args.keys, args.dim)).astype(np.float32)
    qrng = np.random.default_rng([args.seed, rank])
    queries = qrng.uniform(0.02, 0.98, (args.queries, 3))
    return keys, queries, values


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.FIELDS,
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(n)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['no samples'], 'samples': 0}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': smax, 'reasons': sorted(reasons),
                'samples': len(sm)}


# ---------------------------------------------------------------------------
def flops_per_query(stats, gpu_walk_steps, n):
    """Algorithmic FP64 flops per query of the row path, by kernel.

    The kernels read tet and face circumcentres from the per-mesh cache, so
    per query they evaluate: 4 orientation tests per walk step (k_locate),
    the insphere tests (k_rows_cavity), and in k_rows_volume one virtual-tet
    circumcentre per boundary face, two fresh triangle circumcentres and one
    subcell volume per new term, one subcell volume per old term, one
    addition per term, and the normalisation.  Returns {'locate', 'cavity',
    'volume', 'total'} per query."""
    q = stats['queries']
    terms = stats['old_terms'] + stats['new_terms']
    locate = 4 * FLOPS['orient'] * gpu_walk_steps / n * q
    cavity = FLOPS['insphere'] * stats['insphere']
    volume = (FLOPS['tet_cc'] * stats['boundary']
              + 2 * FLOPS['tri_cc'] * stats['new_terms']
              + FLOPS['subcell'] * terms
              + terms + 3 * stats['neighbours'] + 4 * q)
    out = {'locate': locate / q, 'cavity': cavity / q, 'volume': volume / q}
    out['total'] = sum(out.values())
    return out


def plain_config(args, world):
    """The workload keys both arms print (identical in both)."""
    return {'workload': WORKLOAD.format(keys=args.keys, queries=args.queries, dim=args.dim,
                                        seed=args.seed),
            'keys': args.keys, 'queries_per_gpu': args.queries, 'D': args.dim,
            'parallelism': 'replicated mesh, queries sharded' if world > 1 else 'single GPU',
            'l2': 'inputs larger than L2 (10M queries = 240 MB; the resident mesh about 1.6 GB)'}


def run_reference(args, rank, world):
    """natinterp3d's own CPU implementation (oracle/_ref: its C sources built with
    its own flags) with all host threads.  Each step is get_weights + scipy
    W @ values on a bounded sample of the workload's queries (at least 1M,
    about 3 s of work); natinterp3d's one-time packing of its mesh and the
    per-call set-up are warmed before timing, and the per-call set-up is
    amortised as in a call of that size."""
    if rank != 0:
        return None
    from oracle import oracle
    if not oracle.ref_available():
        print(json.dumps({'impl': 'reference', 'unavailable': 'natinterp3d reference library '
                          'not built (oracle/_ref missing)'}))
        return None
    keys, queries, values = make_data(args)
    nthreads = host_threads()
    t0 = time.perf_counter()
    ref = oracle.RefInterpolator(keys, num_threads=nthreads)
    build_s = time.perf_counter() - t0
    ref.interpolate(queries[:20_000], values)  # first call packs the mesh
    probe = queries[:200_000]
    ref.interpolate(probe, values)
    t0 = time.perf_counter()
    ref.interpolate(probe, values)
    rate = probe.shape[0] / (time.perf_counter() - t0)
    sample = int(min(queries.shape[0], max(1_000_000, rate * 3.0)))
    qs = queries[:sample]
    for _ in range(max(1, args.warmup)):
        ref.interpolate(qs, values)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.interpolate(qs, values)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    value = sample / sec
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'queries/s',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': sec * 1e3, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic: seeded uniform keys and queries, '
                                                     'N(0,1) float32 values',
        'config': plain_config(args, world),
        'cpu_baseline': {'value': value, 'unit': 'queries/s', 'cores': nthreads,
                         'kind': 'reference',
                         'sample': '%d of the %d queries per step (get_weights with %d OpenMP '
                                   'threads + scipy W @ values), mesh built by natinterp3d in %.1f s'
                                   % (sample, args.queries, nthreads, build_s)},
        'e2e': {'value': value, 'unit': 'queries/s', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))
    return line


def cpu_baseline(interp, queries, values):
    """natinterp3d's own query code on the same mesh object, all host threads."""
    from oracle import oracle
    if not oracle.ref_available() or interp.host_mesh is None:
        return None
    nthreads = host_threads()
    ptr = interp.host_mesh.native_pointer()
    c = interp.centroid

    def run(qs):
        W = oracle.ref_query(ptr, np.ascontiguousarray(qs, np.float64) - c, interp.n_keys, nthreads)
        return W @ values

    probe = queries[:50_000]
    run(probe)
    t0 = time.perf_counter()
    run(probe)
    rate = probe.shape[0] / (time.perf_counter() - t0)
    sample = int(min(queries.shape[0], max(50_000, rate * 3.0)))
    t0 = time.perf_counter()
    run(queries[:sample])
    sec = time.perf_counter() - t0
    return {'value': sample / sec, 'unit': 'queries/s', 'cores': nthreads, 'kind': 'reference',
            'sample': '%d queries of the workload: natinterp3d getInsertionFreeWeightsParallel '
                      '(%d threads) on the same mesh + scipy W @ values, %.2f s' % (
                          sample, nthreads, sec)}


def fwdbwd_cpu_baseline(interp, queries, values, gout):
    """natinterp3d's own code for the differentiable step's CPU equivalent: its
    weights (all host threads, same mesh object), scipy W @ values and the
    values gradient W.T @ gout.  natinterp3d has no query gradient, so that
    term has no CPU counterpart."""
    from oracle import oracle
    if not oracle.ref_available() or interp.host_mesh is None:
        return None
    nthreads = host_threads()
    ptr = interp.host_mesh.native_pointer()
    c = interp.centroid

    def run(qs, gs):
        W = oracle.ref_query(ptr, np.ascontiguousarray(qs, np.float64) - c, interp.n_keys, nthreads)
        return W @ values, W.T @ gs

    n = min(queries.shape[0], 100_000)
    run(queries[:n // 10], gout[:n // 10])
    t0 = time.perf_counter()
    run(queries[:n], gout[:n])
    sec = time.perf_counter() - t0
    return {'value': n / sec, 'unit': 'queries/s', 'cores': nthreads, 'kind': 'reference',
            'sample': '%d queries of the workload: natinterp3d getInsertionFreeWeightsParallel '
                      '(%d threads) on the same mesh + scipy W @ values + W.T @ gout, %.2f s'
                      % (n, nthreads, sec)}


def _events_ms(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _bitwise_csr(A, B):
    return bool(np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices) and
                np.array_equal(np.asarray(A.data).view(np.uint8), np.asarray(B.data).view(np.uint8)))


def _weights_leg(interp, queries, steps, warmup, cpu, sample_n, workload):
    """get_weights on the device (count + fill, CSR left in HBM) and end to end
    through Interpolator.get_weights (host numpy in, scipy CSR out), plus
    natinterp3d's own get_weights on the same mesh object (all host threads)
    on a sample, which the device rows must equal bit for bit."""
    import ctypes
    import torch
    from natinterp3d_b200 import _native
    from oracle import oracle
    dm = interp.device_mesh
    lib = _native.cuda_lib()
    M = queries.shape[0]
    qd = torch.from_numpy(queries).to(dm.device)
    c = interp.centroid
    step = lambda: dm.weights_csr(qd, c, vals_dtype=torch.float64)
    ms = _events_ms(step, steps, warmup)
    lib.nif_profile_enable(1)
    rowptr, cols, vals, summ = dm.weights_csr(qd, c, vals_dtype=torch.float64, return_summary=True)
    ph = (ctypes.c_double * 4)()
    lib.nif_profile_read(ph)
    lib.nif_profile_enable(0)
    nnz = int(summ['nnz'])
    del rowptr, cols, vals
    e2e = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        W = interp.get_weights(queries)
        e2e.append(time.perf_counter() - t0)
    out = {'value': M / (ms * 1e-3), 'unit': 'queries/s', 'ms_per_step': ms, 'steps': steps,
           'warmup': warmup, 'nnz': nnz,
           # count call's phases (the fill call's compaction is not among them)
           'phase_ms': {'bucketing': ph[0], 'rows': ph[1], 'rows_large': ph[2],
                        'row_pointer_scan': ph[3]},
           'e2e': {'value': M / e2e[-1], 'unit': 'queries/s', 'h2d_bytes_per_step': int(queries.nbytes),
                   'd2h_bytes_per_step': int(W.data.nbytes + W.indices.nbytes + W.indptr.nbytes)},
           'config': {'workload': workload}}
    if cpu and oracle.ref_available() and interp.host_mesh is not None:
        nthreads = host_threads()
        ptr = interp.host_mesh.native_pointer()
        qs = np.ascontiguousarray(queries[:sample_n])
        oracle.ref_query(ptr, qs[:min(sample_n, 20_000)] - c, interp.n_keys, nthreads)  # warm
        best = None
        for _ in range(2):
            t0 = time.perf_counter()
            Wr = oracle.ref_query(ptr, qs - c, interp.n_keys, nthreads)
            t = time.perf_counter() - t0
            best = t if best is None else min(best, t)
        out['bit_identical_to_natinterp3d'] = _bitwise_csr(W[:sample_n], Wr)
        out['cpu_baseline'] = {'value': sample_n / best, 'unit': 'queries/s', 'cores': nthreads,
                               'kind': 'reference',
                               'sample': '%d queries of the workload: natinterp3d '
                                         'getInsertionFreeWeightsParallel (%d threads) on the same '
                                         'mesh, best of 2, %.2f s' % (sample_n, nthreads, best)}
    return out


def leg_get_weights_small(local_rank, steps, warmup, cpu=True):
    """get_weights at the small configuration: 10,000 keys U[0,1]^3, 100,000
    queries U[0.05,0.95]^3, seed 0 (float64)."""
    import torch
    import natinterp3d_b200 as ni
    dev = torch.device('cuda', local_rank)
    rng = np.random.default_rng(0)
    keys = rng.uniform(0.0, 1.0, (10_000, 3))
    queries = rng.uniform(0.05, 0.95, (100_000, 3))
    interp = ni.Interpolator(keys, device=dev, keep_host_mesh=cpu)
    return _weights_leg(interp, queries, steps, warmup, cpu, 100_000,
                        'get_weights: 10,000 keys U[0,1]^3, 100,000 queries U[0.05,0.95]^3, '
                        'float64, seed 0')


def tet_set_digest(tet_v):
    """(count, two order-independent 64-bit sums) of a tet set: the sorted
    vertex quadruple of each tet mixed by two odd-multiplier hashes."""
    t = np.sort(np.asarray(tet_v), axis=1).astype(np.uint64)
    c1 = np.array([0x9E3779B97F4A7C15, 0xC2B2AE3D27D4EB4F, 0x165667B19E3779F9,
                   0xD6E8FEB86659FD93], dtype=np.uint64)
    c2 = np.array([0xFF51AFD7ED558CCD, 0xC4CEB9FE1A85EC53, 0x94D049BB133111EB,
                   0xBF58476D1CE4E5B9], dtype=np.uint64)
    with np.errstate(over='ignore'):
        h1 = (t * c1).sum(axis=1, dtype=np.uint64)
        h2 = (t * c2).sum(axis=1, dtype=np.uint64)
        h1 ^= h1 >> np.uint64(29)
        h2 ^= h2 >> np.uint64(31)
        h1 *= np.uint64(0xBF58476D1CE4E5B9)
        h2 *= np.uint64(0x94D049BB133111EB)
        return int(t.shape[0]), int(h1.sum(dtype=np.uint64)), int(h2.sum(dtype=np.uint64))


def leg_gpu_construction(keys, interp, host_build_s, local_rank):
    """natinterp3d's tetrahedralization of the bench keys built on the GPU
    (``constructor='gpu'``) against natinterp3d's host constructor, which
    built ``interp``'s mesh in ``host_build_s`` seconds: time, rounds, the
    builder's exact checks, and whether the tet set equals natinterp3d's."""
    import torch
    from natinterp3d_b200.device import gpu_delaunay, GPUConstructionError
    dev = torch.device('cuda', local_rank)
    centered = keys - interp.centroid
    gpu_delaunay(centered[:10_000], dev)  # first-use costs (module load) off the clock
    torch.cuda.synchronize()
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        try:
            (vxyz, tv, tn), info = gpu_delaunay(centered, dev)
        except GPUConstructionError as e:
            return {'unavailable': str(e)}
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        last = tv
    t = min(times)
    host_tv = interp.mesh_arrays[1]
    same = (tet_set_digest(last.cpu().numpy()) == tet_set_digest(host_tv)
            and np.array_equal(vxyz.cpu().numpy().view(np.uint8),
                               interp.mesh_arrays[0].view(np.uint8)))
    return {'value': keys.shape[0] / t, 'unit': 'keys/s', 'gpu_s': t,
            'host_constructor_s': host_build_s, 'speedup_vs_host': host_build_s / t,
            'tets': int(info['n_tets']), 'rounds': int(info['rounds']),
            'max_cavity': int(info['max_cavity']),
            'exact_evaluations': int(info['exact_evaluations']),
            'checks': {k: int(info[k]) for k in ('bad_orientation', 'bad_adjacency',
                                                  'non_delaunay_faces', 'cospherical_faces')},
            'same_tets_and_vertices_as_natinterp3d': bool(same),
            'config': {'workload': 'Delaunay tetrahedralization of the plain workload\'s keys '
                                   '(+ natinterp3d\'s super-simplex), wall clock with the result '
                                   'on the device'}}


def leg_fwdbwd(args, rank, local_rank, steps, warmup, cpu=True):
    """Differentiable workload: loss = sum(out * g), backward into queries and
    values (200k keys U[0,1]^3, 1M queries U[0.1,0.9]^3 float64 with grad,
    values D=16 float32 with grad, seed 3)."""
    import torch
    import natinterp3d_b200 as ni
    from natinterp3d_b200 import autograd as nag
    keys_n, q_n, dim = 200_000, 1_000_000, 16
    torch.cuda.set_device(local_rank)
    dev = torch.device('cuda', local_rank)
    rng = np.random.default_rng([3, rank])
    keys = rng.uniform(0, 1, (keys_n, 3))
    t0 = time.perf_counter()
    interp = ni.Interpolator(keys, device=dev, keep_host_mesh=cpu)
    build_s = time.perf_counter() - t0
    qn = rng.uniform(0.1, 0.9, (q_n, 3))
    vn = rng.standard_normal((keys_n, dim)).astype(np.float32)
    gn = rng.standard_normal((q_n, dim))
    qd, vd, gd = (torch.from_numpy(a).to(dev) for a in (qn, vn, gn))
    # autotuner (setup, untimed) on the weights path the differentiable forward uses
    tuned = None
    if fixed_tuning(args):
        interp.set_tuning(fixed_tuning(args))
    elif not args.no_tune:
        tuned = interp.tune(qd, mode='weights', use_cache=False)['tuning']

    def fwd():
        return interp.interpolate_device(qd, vd, check=False)

    def fwdbwd():
        q = qd.clone().requires_grad_(True)
        v = vd.clone().requires_grad_(True)
        out = nag.interpolate(interp, q, v)
        (out * gd).sum().backward()
        return q.grad, v.grad

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_fwd = timed(fwd)
    ms_fb = timed(fwdbwd)
    base = fwdbwd_cpu_baseline(interp, qn, vn, gn) if cpu else None
    return {
        'metric': METRIC, 'mode': 'fwd+bwd', 'value': q_n / (ms_fb * 1e-3), 'unit': 'queries/s',
        'steps': steps, 'warmup': warmup, 'ms_per_step': ms_fb,
        'plain_forward_ms': ms_fwd, 'fwdbwd_over_forward': ms_fb / ms_fwd, 'cpu_baseline': base,
        'higher_is_better': True, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': 'differentiable: %d keys U[0,1]^3, %d queries U[0.1,0.9]^3 float64 '
                               'with grad, values D=%d float32 with grad, loss=sum(out*g), seed 3'
                               % (keys_n, q_n, dim)},
        'setup': {'mesh_build_s': round(build_s, 2), 'tuning': interp.tuning,
                  'autotuned': tuned is not None}}


def run_fwdbwd(args, rank, world, local_rank):
    line = leg_fwdbwd(args, rank, local_rank, args.steps, args.warmup,
                      cpu=(rank == 0 and not args.no_cpu_baseline))
    if rank == 0:
        line['n_gpus'] = world
        print(json.dumps(line))


def batched_workload(P, seed):
    rng = np.random.default_rng(seed)
    keys, queries = [], []
    for _ in range(P):
        nk = int(np.exp(rng.uniform(np.log(500), np.log(100_000))))
        nq = int(np.exp(rng.uniform(np.log(1_000), np.log(200_000))))
        lo = rng.uniform(-5, 5, 3)
        side = rng.uniform(0.5, 2.0, 3)
        keys.append(lo + side * rng.uniform(0, 1, (nk, 3)))
        queries.append(lo + side * (0.025 + 0.95 * rng.uniform(0, 1, (nq, 3))))
    values = [rng.standard_normal((k.shape[0], 4)).astype(np.float32) for k in keys]
    return keys, queries, values


def leg_batched(args, rank, local_rank, steps, warmup, cpu=True):
    """Uneven batch: one captured graph vs one plain call per problem vs natinterp3d's loop."""
    import torch
    from natinterp3d_b200.batch import BatchInterpolator
    from oracle import oracle
    torch.cuda.set_device(local_rank)
    dev = torch.device('cuda', local_rank)
    keys, queries, values = batched_workload(args.problems, 4 + rank)
    t0 = time.perf_counter()
    b = BatchInterpolator(keys, device=dev)
    build_s = time.perf_counter() - t0
    qoff = b.query_offsets([len(q) for q in queries])
    M = int(qoff[-1])
    qcat = torch.from_numpy(np.concatenate(queries)).to(dev)
    vcat = torch.from_numpy(np.concatenate(values)).to(dev)
    # autotuner (setup, untimed): occupancy and tile size of the persistent kernel
    tuned = None
    if fixed_tuning(args):
        b.set_tuning(fixed_tuning(args))
    elif not args.no_tune:
        tuned = b.tune(qcat, qoff, vcat, use_cache=False)['tuning']
    graph = b.capture(qcat, qoff, vcat)
    eager = b.interpolate_per_problem(qcat, qoff, vcat)
    same = bool(torch.equal(graph.replay(), eager))

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_graph = timed(graph.replay)
    ms_loop = timed(lambda: b.interpolate_per_problem(qcat, qoff, vcat))
    # the same loop through the default device API: each call checks its rows
    # (reads the row counters back, so it synchronises once per problem)
    qo, ko = qoff, b.key_offsets.cpu().numpy()

    def api_loop():
        for p, it in enumerate(b.interpolators):
            if qo[p + 1] > qo[p]:
                it.interpolate_device(qcat[qo[p]:qo[p + 1]], vcat[ko[p]:ko[p + 1]])

    ms_api = timed(api_loop)
    # host API: one Interpolator.interpolate per problem (numpy in and out) vs one
    # batched call; each measured on its second run (the first allocates)
    for _ in range(2):
        t0 = time.perf_counter()
        for p in range(args.problems):
            b.interpolators[p].interpolate(queries[p], values[p])
        host_loop_s = time.perf_counter() - t0
    for _ in range(2):
        t0 = time.perf_counter()
        b.interpolate(queries, values)
        host_batch_s = time.perf_counter() - t0
    base = None
    if cpu and oracle.ref_available():
        # natinterp3d's own code, one Interpolator per problem, on a sample of problems
        nthreads = host_threads()
        sample = list(range(0, args.problems, max(1, args.problems // 24)))
        refs = [oracle.RefInterpolator(keys[p], num_threads=nthreads) for p in sample]
        t0 = time.perf_counter()
        for r, p in zip(refs, sample):
            r.interpolate(queries[p], values[p])
        sec = time.perf_counter() - t0
        nq = sum(len(queries[p]) for p in sample)
        base = {'value': nq / sec, 'unit': 'queries/s', 'cores': nthreads, 'kind': 'reference',
               'sample': '%d of %d problems (%d queries): natinterp3d Interpolator per problem, '
                         'get_weights + scipy W @ values' % (len(sample), args.problems, nq)}
    return {
        'metric': METRIC, 'mode': 'batched', 'value': M / (ms_graph * 1e-3), 'unit': 'queries/s',
        'steps': steps, 'warmup': warmup, 'ms_per_step': ms_graph,
        'per_problem_launches_ms': ms_loop, 'batched_over_per_problem_speedup': ms_loop / ms_graph,
        'per_problem_api_ms': ms_api, 'batched_over_per_problem_api': ms_api / ms_graph,
        'host_api_per_problem_s': host_loop_s, 'host_api_batched_s': host_batch_s,
        'host_api_speedup': host_loop_s / host_batch_s,
        'bit_identical_to_per_problem': same, 'higher_is_better': True, 'dtype': 'f64',
        'data': 'synthetic', 'cpu_baseline': base,
        'config': {'workload': '%d problems, keys log-uniform [500, 100k] in boxes of side 0.5-2, '
                               'queries log-uniform [1k, 200k] in the boxes shrunk 5%%, values D=4 '
                               'float32, seed 4' % args.problems,
                   'total_keys': int(b.n_keys.sum()), 'total_queries': M},
        'setup': {'mesh_build_s': round(build_s, 1), 'tuning': b.get_tuning(),
                  'autotuned': tuned is not None}}


def run_batched(args, rank, world, local_rank):
    line = leg_batched(args, rank, local_rank, args.steps, args.warmup,
                       cpu=(rank == 0 and not args.no_cpu_baseline))
    if rank == 0:
        line['n_gpus'] = world
        print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))

    if args.impl == 'reference':
        run_reference(args, rank, world)
        return
    if args.mode == 'fwdbwd':
        run_fwdbwd(args, rank, world, local_rank)
        return
    if args.mode == 'batched':
        run_batched(args, rank, world, local_rank)
        return

    import torch
    import natinterp3d_b200 as ni
    from natinterp3d_b200 import _native
    from oracle import oracle

    torch.cuda.set_device(local_rank)
    dev = torch.device('cuda', local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600),
                                device_id=dev)

    keys, queries, values = make_data(args, rank)
    t0 = time.perf_counter()
    interp = ni.Interpolator(keys, device=dev, keep_host_mesh=(rank == 0 and not args.no_cpu_baseline),
                             predicates=args.predicates)
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    dm = interp.device_mesh
    upload_s = time.perf_counter() - t0

    lib = _native.cuda_lib()
    qd = torch.from_numpy(queries).to(dev)
    vd = torch.from_numpy(values).to(dev)
    M = queries.shape[0]

    # correctness gate on a sample before timing: bit-identical to the oracle
    sample_n = min(M, 20_000)
    om = oracle.OracleMesh(*interp.mesh_arrays)
    om.set_predicates(args.predicates)
    Wref, stats, _ = om.weights(queries[:sample_n] - interp.centroid, with_stats=True)
    out_s = dm.interpolate(qd[:sample_n], vd, interp.centroid).cpu().numpy()
    exact = bool(np.array_equal(out_s, Wref @ values))

    # autotuner (setup, untimed): launch settings for this workload, timed on
    # a 2M-query sample; results do not depend on them
    t0 = time.perf_counter()
    tuned = tune_times = None
    if fixed_tuning(args):
        interp.set_tuning(fixed_tuning(args))
    elif not args.no_tune:
        rep = interp.tune(qd, vd, use_cache=False)
        tuned = rep['tuning']
        # the 2M-query sample's time of the library default and of the pick
        times = {tuple(sorted(c.items())): t for c, t in rep['times_ms']}
        dflt = {'blocks_per_sm': 8, 'bucket_shift': 0, 'tile': 8}
        tune_times = {'default_ms': times.get(tuple(sorted(dflt.items()))),
                      'chosen_ms': times.get(tuple(sorted(tuned.items())))}
    tune_s = time.perf_counter() - t0

    def step():
        return dm.interpolate(qd, vd, interp.centroid, check=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    lib.nif_profile_enable(1)
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    # per-phase device times of the timed calls (events recorded in each call,
    # read once here: the loop itself never waits on the host)
    ph = (ctypes.c_double * 4)()
    have_phases = lib.nif_profile_read(ph) == 0
    kms, kn = (ctypes.c_double * 5)(), (ctypes.c_double * 5)()
    lib.nif_profile_kernels(kms, kn)
    lib.nif_profile_enable(0)
    ms = e0.elapsed_time(e1) / args.steps
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = M * world / (ms * 1e-3)

    # summary of one extra call (walk steps, large rows), untimed
    _, summ = dm.interpolate(qd, vd, interp.centroid, return_summary=True)

    # end to end through the public API with host buffers
    e2e_times = []
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = interp.interpolate(queries, values)
        e2e_times.append(time.perf_counter() - t0)
    e2e_sec = float(np.median(e2e_times[1:]))
    if dist is not None:
        t = torch.tensor([e2e_sec], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_sec = float(t.item())

    if rank == 0:
        phases = list(ph) if have_phases else [0.0] * 4
        rows_ms = phases[1]
        fpq = flops_per_query(stats, summ['walk_steps'], M)
        fused, separate = ctypes.c_double(), ctypes.c_double()
        lib.nif_measure_fp64_peak(ctypes.byref(fused), ctypes.byref(separate))
        # the dominant kernel, k_rows_volume: its launches take every row but
        # the few the fused kernel takes (cavities wider than a record)
        vol_rows = M - int(summ['rows_wide'])
        vol_ms, vol_launches = kms[2], kn[2]
        achieved = (fpq['volume'] * vol_rows / (vol_ms * 1e-3) / 1e12) if vol_ms > 0 else None
        path_achieved = fpq['total'] * M / (rows_ms * 1e-3) / 1e12 if rows_ms > 0 else None
        names = ['k_locate', 'k_rows_cavity', 'k_rows_volume', 'k_rows_fast', 'k_rows_order']
        kernels = {n: {'ms_per_step': kms[i], 'launches_per_step': kn[i],
                       'share_of_rows_phase': kms[i] / rows_ms if rows_ms > 0 else None}
                   for i, n in enumerate(names)}
        for i, part in enumerate(['locate', 'cavity', 'volume']):
            kernels[names[i]]['flops_per_query'] = fpq[part]
        # bucketing (k_bucket, three scan kernels, k_scatter), the row kernels
        # the profiler bracketed, and the large-row kernel
        launches_per_step = int(round(5 + sum(kn) + 1))
        cpu = None if args.no_cpu_baseline else cpu_baseline(interp, queries, values)
        line = {
            'metric': METRIC, 'value': value, 'unit': 'queries/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic: seeded uniform keys and queries, N(0,1) float32 values',
            'config': plain_config(args, world),
            'setup': {
                'mesh_build_s': round(build_s, 2), 'mesh_upload_s': round(upload_s, 3),
                'tets': dm.n_tets, 'resident_mesh_mb': round(dm.nbytes / 1e6, 1),
                'octree': dm.octree_stats,
                'bit_identical_to_oracle_on_sample': exact, 'predicates': args.predicates,
                'tuning': dm.get_tuning(), 'autotuned': tuned is not None,
                'tune_s': round(tune_s, 2), 'tune_sample_ms': tune_times,
            },
            'roofline': {
                'bound': 'fp64', 'kernel': 'k_rows_volume',
                'achieved': achieved, 'peak': separate.value, 'unit': 'TFLOP/s',
                'frac': (achieved / separate.value) if achieved and separate.value else None,
                'peak_fused_fma': fused.value,
                'peak_note': 'measured on this GPU by nif_measure_fp64_peak: separately rounded '
                             'DMUL+DADD (the kernels never fuse, for bit parity)',
                'flops_per_query': fpq['volume'],
                'rows_per_launch': vol_rows / vol_launches if vol_launches else None,
                'launch_ms': vol_ms / vol_launches if vol_launches else None,
                # dram__bytes_read.sum + dram__bytes_write.sum of one
                # k_rows_volume launch from an ncu capture (profiles/), per row,
                # times this workload's rows per launch
                'traffic': (TRAFFIC_PER_ROW['k_rows_volume'] * vol_rows / vol_launches
                            if vol_launches else None),
                'traffic_note': 'per launch; ncu capture of %s' % TRAFFIC_SOURCE,
                'row_path': {
                    'kernels': 'k_locate + k_rows_cavity + k_rows_order + k_rows_volume (+ k_rows_fast)',
                    'achieved': path_achieved, 'flops_per_query': fpq['total'],
                    'frac': (path_achieved / separate.value) if path_achieved and separate.value
                    else None,
                    'ms_per_step': rows_ms,
                },
                'kernels': kernels,
                'phase_ms': {'bucketing': phases[0], 'rows': rows_ms,
                             'rows_large': phases[2], 'epilogue': phases[3]},
            },
            'cpu_baseline': cpu,
            'e2e': {'value': M * world / e2e_sec, 'unit': 'queries/s',
                    'h2d_bytes_per_step': int(queries.nbytes + values.nbytes),
                    'd2h_bytes_per_step': int(out.nbytes)},
            'gpu_launches': launches_per_step * args.steps,
            'clocks': clocks.summary(),
            'summary': {k: int(v) for k, v in summ.items() if k != 'nnz'},
        }
        if world == 1 and not args.no_legs:
            # the other legs of the metric, each with its own CPU baseline
            cpu_on = not args.no_cpu_baseline
            legs = {}
            legs['get_weights_1M_keys_10M_queries'] = _weights_leg(
                interp, queries, 3, 1, cpu_on, 1_000_000,
                'get_weights on the plain workload: ' + WORKLOAD.format(
                    keys=args.keys, queries=args.queries, dim=args.dim, seed=args.seed))
            legs['get_weights_10k_keys_100k_queries'] = leg_get_weights_small(
                local_rank, max(args.steps, 5), 3, cpu_on)
            del out
            legs['fwd+bwd'] = leg_fwdbwd(args, rank, local_rank, max(args.steps, 5),
                                         max(args.warmup, 3), cpu_on)
            legs['gpu_construction_1M_keys'] = leg_gpu_construction(keys, interp, build_s,
                                                                    local_rank)
            legs['batched'] = leg_batched(args, rank, local_rank, max(args.steps, 3),
                                          max(args.warmup, 3), cpu_on)
            line['legs'] = legs
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()

// natinterp3d_b200: sm_100a kernels and the C ABI of libnif_cuda.so
// (declarations and contracts in include/natinterp3d_b200.h).
//
// Query pipeline (one call):
//   k_bucket / scan / k_scatter   spatial bucketing of the queries (Morton
//                                 order of a grid over the mesh bounding box),
//                                 so that concurrently running groups touch
//                                 nearby tets and the mesh stays in L1/L2;
//                                 natinterp3d sorts by Morton code for the
//                                 same reason (natural.c:70-96)
//   k_rows<fast>                  one warp (G = 32 lanes) per query, scratch
//                                 in shared memory, a persistent grid of 6 or
//                                 8 blocks per SM taking rows by static
//                                 stride or in tiles from a device counter
//                                 (nif_tuning); rows that exceed its
//                                 per-query capacities are queued
//   k_rows<large>                 the queued rows, one warp each, scratch in a
//                                 global-memory workspace with much larger
//                                 capacities
//   then either  count scan + k_compact  (get_weights: CSR)
//   or the rows were reduced against the values in place (interpolate).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <type_traits>
#include <new>

#include "natinterp3d_b200.h"
#include "nif_kernels.cuh"
#include "nif_grad.cuh"

#define NIF_EXPORT extern "C" __attribute__((visibility("default")))

namespace nif {

// ---------------------------------------------------------------------------
// capacities
// ---------------------------------------------------------------------------
#ifndef NIF_FAST_G
#define NIF_FAST_G 32
#endif
// resident 4-warp blocks per SM of the shared-memory row kernels: the two
// occupancy points compiled (nif_tuning.blocks_per_sm) and the default
constexpr int OCC_LO = 6;   // 80 registers a thread
constexpr int OCC_HI = 8;   // 64 registers a thread
constexpr int OCC_DEFAULT = OCC_HI;
constexpr int TILE_MAX = 1024;
constexpr int MESH_TILE_DEFAULT = 8;   // queries per work item of a single mesh's row kernel
constexpr int BATCH_TILE_DEFAULT = 64;
constexpr int FAST_G = NIF_FAST_G;    // lanes per query in the shared-memory kernel
using FastWS = Workspace<256, 96, 128, 64, 128, FAST_G, uint8_t, int8_t>;
constexpr int LARGE_G = 32;
using LargeWS = Workspace<16384, 4096, 8192, 2048, 8192, LARGE_G, uint16_t, int16_t>;
constexpr int ROW_STAGE = 24;         // get_weights: entries staged per row (mean about 15.5)
using CavWS = CavWorkspace<256, 96, FAST_G, uint8_t, int8_t>;
using VolWS = VolWorkspace<REC_CAV, 128, 64, 128, FAST_G>;
// rows a record buffer holds: calls run in chunks of these (measured: 256k-
// and 64k-row chunks, whose records stay in L2, ran 6 % and 25 % slower on
// 10M queries -- the launches' tails cost more than the DRAM round trip)
#ifndef NIF_REC_CHUNK
#define NIF_REC_CHUNK (1 << 20)
#endif
constexpr int REC_CHUNK = NIF_REC_CHUNK;
// resident blocks per SM of the split kernels (0: the mesh's blocks_per_sm).
// The cavity kernel is issue-bound and fits 10 blocks in 48 registers (1-2 %
// faster than 8 on 10M queries); the volume kernel spills at 10 (16 % slower)
// and follows the mesh's setting.
#ifndef NIF_CAV_OCC
#define NIF_CAV_OCC 10
#endif
#ifndef NIF_VOL_OCC
#define NIF_VOL_OCC 0
#endif

constexpr int FAST_BLOCK = 128;       // 4 warps
constexpr int LARGE_GROUPS = 64;      // concurrent large-row groups (one warp each)
constexpr int SCAN_TILE = 2048;
constexpr int SCAN_THREADS = 256;

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------------------
// per-call device summary (mirrors nif_summary)
// ---------------------------------------------------------------------------
struct DevSummary {
    unsigned long long nnz;
    unsigned long long rows_large;
    unsigned long long rows_failed;
    unsigned long long rows_outside;
    unsigned long long walk_steps;
    int first_status;
    int large_count;  // rows queued for the large kernel
    int refill_count; // get_weights: fast-kernel rows longer than ROW_STAGE
    int wide_count;   // split rows whose cavity exceeds a record (the fused kernel takes them)
    // predicate evaluations the filter could not certify / whose decision the
    // exact sign changes (PRED_AUDIT and PRED_EXACT meshes)
    unsigned long long orient_unc, orient_flip, insphere_unc, insphere_flip;
};

// ---------------------------------------------------------------------------
// resident mesh preparation
// ---------------------------------------------------------------------------

// validates the packed mesh and converts it to the resident layout
__global__ void k_prep_vertices(const double *__restrict__ vxyz, int nv, d4 *__restrict__ vtx) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        vtx[i] = d4{vxyz[3 * (size_t)i], vxyz[3 * (size_t)i + 1], vxyz[3 * (size_t)i + 2], 0.0};
}

__global__ void k_prep_tets(const int32_t *__restrict__ tet_v, const int32_t *__restrict__ tet_n,
                            int nv, int nt, int4 *__restrict__ tv, int4 *__restrict__ tn,
                            int *__restrict__ bad) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        int4 p = make_int4(tet_v[4 * (size_t)t], tet_v[4 * (size_t)t + 1], tet_v[4 * (size_t)t + 2],
                           tet_v[4 * (size_t)t + 3]);
        int4 n = make_int4(tet_n[4 * (size_t)t], tet_n[4 * (size_t)t + 1], tet_n[4 * (size_t)t + 2],
                           tet_n[4 * (size_t)t + 3]);
        bool ok = true;
        for (int j = 0; j < 4; j++) {
            ok = ok && comp(p, j) >= 0 && comp(p, j) < nv;
            ok = ok && comp(n, j) >= -1 && comp(n, j) < nt;
        }
        if (!ok) {
            atomicExch(bad, 1);
            p = make_int4(0, 0, 0, 0);
            n = make_int4(-1, -1, -1, -1);
        }
        tv[t] = p;
        tn[t] = n;
    }
}

// orientation flags, mirror slots, tet and face circumcentres.  flag[0]: bad
// mesh, flag[1]: tets whose orientation sign the filter cannot certify.
__global__ void k_prep_geometry(MeshView M, uint32_t *__restrict__ tinfo, d4 *__restrict__ tcc,
                                d4 *__restrict__ fcc, int *__restrict__ bad) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < M.nt; t += gridDim.x * blockDim.x) {
        const int4 p = M.tv[t];
        const int4 n = M.tn[t];
        const dv3 P0 = vload(M, p.x), P1 = vload(M, p.y), P2 = vload(M, p.z), P3 = vload(M, p.w);
        // natinterp3d recomputes this sign on every call (natural_insertionfree.c:457-476);
        // bit 2 (the exact sign) equals it unless k_prep_exact_orient corrects it
        const double o = orient_fast(P0, P1, P2, P3);
        uint32_t info = o > 0 ? 5u : 0u;
        if (orient_uncertain(P0, P1, P2, P3, o)) {
            info |= 2u;
            atomicAdd(&bad[1], 1);
        }
        for (int j = 0; j < 4; j++) {
            const int nb = comp(n, j);
            int jm = 0;
            if (nb >= 0) {
                const int4 nn = M.tn[nb];
                jm = -1;
                for (int k = 0; k < 4; k++)
                    if (comp(nn, k) == t && jm < 0) jm = k;
                if (jm < 0) {
                    atomicExch(bad, 2);
                    jm = 0;
                }
            }
            info |= (uint32_t)jm << (8 + 2 * j);
        }
        tinfo[t] = info;
        const dv3 c = tet_cc(P0, P1, P2, P3);
        tcc[t] = d4{c.x, c.y, c.z, 0.0};
        // face opposite p[i], remaining vertices in ascending slot order
        // (natural_insertionfree.c:649-652)
        const dv3 f0 = tri_cc(P1, P2, P3);
        const dv3 f1 = tri_cc(P0, P2, P3);
        const dv3 f2 = tri_cc(P0, P1, P3);
        const dv3 f3 = tri_cc(P0, P1, P2);
        fcc[4 * (size_t)t + 0] = d4{f0.x, f0.y, f0.z, 0.0};
        fcc[4 * (size_t)t + 1] = d4{f1.x, f1.y, f1.z, 0.0};
        fcc[4 * (size_t)t + 2] = d4{f2.x, f2.y, f2.z, 0.0};
        fcc[4 * (size_t)t + 3] = d4{f3.x, f3.y, f3.z, 0.0};
    }
}

// exact orientation (bit 2) of the tets flagged uncertain (bit 1); one warp
// per block, lanes take turns in the block's scratch.  flag[2] counts the
// tets whose "orient3d > 0" flag the exact sign changes.
__global__ void __launch_bounds__(32) k_prep_exact_orient(MeshView M, uint32_t *__restrict__ tinfo,
                                                          int *__restrict__ flag) {
    __shared__ double scr[NIF_ORIENT_SCRATCH];
    for (int base = blockIdx.x * 32; base < M.nt; base += gridDim.x * 32) {
        const int t = base + threadIdx.x;
        const bool unc = t < M.nt && (tinfo[t] & 2u);
        unsigned um = __ballot_sync(0xffffffffu, unc);
        while (um) {
            const int l = __ffs(um) - 1;
            um &= um - 1u;
            if ((int)threadIdx.x == l) {
                const int4 p = M.tv[t];
                double a[3], b[3], c[3], d[3];
                to3(vload(M, p.x), a), to3(vload(M, p.y), b), to3(vload(M, p.z), c);
                to3(vload(M, p.w), d);
                const uint32_t info = tinfo[t];
                const uint32_t xpos = nif_orient_exact_sign(a, b, c, d, scr) > 0 ? 4u : 0u;
                if ((xpos != 0) != ((info & 1u) != 0)) atomicAdd(&flag[2], 1);
                tinfo[t] = (info & ~4u) | xpos;
            }
            __syncwarp();
        }
    }
}

// bounding box of the data vertices: per-block partials (6 doubles per block)
__global__ void k_bbox_partial(const d4 *__restrict__ vtx, int n, double *__restrict__ part) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const d4 v = vtx[i];
        lo[0] = fmin(lo[0], v.x); lo[1] = fmin(lo[1], v.y); lo[2] = fmin(lo[2], v.z);
        hi[0] = fmax(hi[0], v.x); hi[1] = fmax(hi[1], v.y); hi[2] = fmax(hi[2], v.z);
    }
    __shared__ double s[6][256];
    for (int a = 0; a < 3; a++) {
        s[a][threadIdx.x] = lo[a];
        s[3 + a][threadIdx.x] = hi[a];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int a = 0; a < 3; a++) {
                s[a][threadIdx.x] = fmin(s[a][threadIdx.x], s[a][threadIdx.x + w]);
                s[3 + a][threadIdx.x] = fmax(s[3 + a][threadIdx.x], s[3 + a][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int a = 0; a < 6; a++) part[6 * blockIdx.x + a] = s[a][0];
}

__device__ __forceinline__ unsigned spread3(unsigned v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Centroid of tet p as natinterp3d's constructor computes it for its k-d tree
// (delaunay.c:151-157): (p0 + p1 + p2 + p3) / 4 per axis, summed left to right.
__device__ __forceinline__ d4 tet_centroid(const MeshView &M, const int4 &p, int t) {
    const d4 a = M.vtx[p.x], b = M.vtx[p.y], c = M.vtx[p.z], d = M.vtx[p.w];
    return d4{fdiv(fadd(fadd(fadd(a.x, b.x), c.x), d.x), 4.0),
              fdiv(fadd(fadd(fadd(a.y, b.y), c.y), d.y), 4.0),
              fdiv(fadd(fadd(fadd(a.z, b.z), c.z), d.z), 4.0), (double)t};
}

// 60-bit Morton code of each tet centroid's cell (oct_code), split into two
// 32-bit words for the radix sort (low word first, then the high word)
__global__ void k_cen_code(MeshView M, uint32_t *__restrict__ chi, uint32_t *__restrict__ clo,
                           uint32_t *__restrict__ key, int32_t *__restrict__ idx) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < M.nt; t += gridDim.x * blockDim.x) {
        const d4 c = tet_centroid(M, M.tv[t], t);
        int ix[3];
        const unsigned long long code = oct_code(M, dv3{c.x, c.y, c.z}, ix);
        chi[t] = (uint32_t)(code >> 32);
        clo[t] = (uint32_t)code;
        key[t] = (uint32_t)code;
        idx[t] = t;
    }
}

__global__ void k_gather_key(const uint32_t *__restrict__ src, const int32_t *__restrict__ idx, int n,
                             uint32_t *__restrict__ key) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        key[k] = src[idx[k]];
}

__global__ void k_cen_gather(MeshView M, const int32_t *__restrict__ idx, const uint32_t *__restrict__ chi,
                             const uint32_t *__restrict__ clo, d4 *__restrict__ cs,
                             unsigned long long *__restrict__ code) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M.nt; k += gridDim.x * blockDim.x) {
        const int t = idx[k];
        cs[k] = tet_centroid(M, M.tv[t], t);
        code[k] = ((unsigned long long)chi[t] << 32) | clo[t];
    }
}

// cell of a centroid in the uniform seed grid (the formula grid_nearest uses)
__device__ __forceinline__ int grid_cell(const MeshView &M, const d4 &c) {
    const double x[3] = {c.x, c.y, c.z};
    int ic[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double f = (x[a] - M.glo[a]) * M.ginv[a];
        ic[a] = f > 0.0 ? (f < (double)(M.gdim[a] - 1) ? (int)f : M.gdim[a] - 1) : 0;
    }
    return (ic[2] * M.gdim[1] + ic[1]) * M.gdim[0] + ic[0];
}

__global__ void k_grid_count(MeshView M, int *__restrict__ count) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M.nt; k += gridDim.x * blockDim.x)
        atomicAdd(&count[grid_cell(M, M.cs[k])], 1);
}

__global__ void k_grid_fill(MeshView M, int *__restrict__ cursor, d4 *__restrict__ items) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M.nt; k += gridDim.x * blockDim.x) {
        const d4 c = M.cs[k];
        items[atomicAdd(&cursor[grid_cell(M, c)], 1)] = c;
    }
}

// Octree build, one node level at a time.  Nodes are numbered level by level
// in centroid order; node j spans centroids [na[j], nb[j]).  node_of[i] is
// the deepest node built so far that holds centroid i.  A level-k node with
// more than OCT_SPLIT centroids gets one child per distinct 6-bit digit k of
// its centroids' codes: flag marks each child's first centroid.
__device__ __forceinline__ bool oct_splits(const int *na, const int *nb, int p, int s0, int s1) {
    return p >= s0 && p < s1 && nb[p] - na[p] > OCT_SPLIT;
}

__global__ void k_oct_flag(const unsigned long long *__restrict__ code, int nt, const int *__restrict__ node_of,
                           const int *__restrict__ na, const int *__restrict__ nb, int s0, int s1, int k,
                           int *__restrict__ flag) {
    const int sh = 6 * (OCT_KMAX - 1 - k);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        const int p = node_of[i];
        int f = 0;
        if (oct_splits(na, nb, p, s0, s1))
            f = (i == na[p]) || ((code[i] >> sh) != (code[i - 1] >> sh));
        flag[i] = f;
    }
}

__global__ void k_oct_link(const unsigned long long *__restrict__ code, int nt, int *__restrict__ node_of,
                           int *__restrict__ na, const int *__restrict__ nb, int s0, int s1, int k,
                           const int *__restrict__ flag, const int *__restrict__ scan, int *__restrict__ par,
                           int *__restrict__ first, int *__restrict__ nch, unsigned long long *__restrict__ mask) {
    const int sh = 6 * (OCT_KMAX - 1 - k);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        const int p = node_of[i];
        if (!oct_splits(na, nb, p, s0, s1)) continue;
        const int f = flag[i];
        if (f) {
            const int j = s1 + scan[i];
            na[j] = i;
            par[j] = p;
            if (i == na[p]) first[p] = j;
            atomicAdd(&nch[p], 1);
            atomicOr(&mask[p], 1ull << (int)((code[i] >> sh) & 63ull));
        }
        node_of[i] = s1 + scan[i] + f - 1;
    }
}

__global__ void k_oct_end(int s1, int T, const int *__restrict__ na, const int *__restrict__ par,
                          int *__restrict__ nb) {
    for (int j = s1 + blockIdx.x * blockDim.x + threadIdx.x; j < s1 + T; j += gridDim.x * blockDim.x) {
        const int pe = nb[par[j]];
        nb[j] = (j + 1 < s1 + T && na[j + 1] < pe) ? na[j + 1] : pe;
    }
}

// node records of nodes [s, e), deepest level first: a leaf's box over its
// centroids, an inner node's over its children's boxes (float min / max of
// outward-rounded bounds are exact)
__global__ void k_oct_box(int s, int e, const int *__restrict__ na, const int *__restrict__ nb,
                          const int *__restrict__ first, const int *__restrict__ nch,
                          const d4 *__restrict__ cs, float4 *__restrict__ onode) {
    for (int j = s + blockIdx.x * blockDim.x + threadIdx.x; j < e; j += gridDim.x * blockDim.x) {
        float4 lo, hi;
        if (nch[j] == 0) {
            double l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int k = na[j]; k < nb[j]; k++) {
                const d4 c = cs[k];
                l[0] = fmin(l[0], c.x); l[1] = fmin(l[1], c.y); l[2] = fmin(l[2], c.z);
                h[0] = fmax(h[0], c.x); h[1] = fmax(h[1], c.y); h[2] = fmax(h[2], c.z);
            }
            lo = make_float4(__double2float_rd(l[0]), __double2float_rd(l[1]), __double2float_rd(l[2]),
                             __int_as_float(na[j]));
            hi = make_float4(__double2float_ru(h[0]), __double2float_ru(h[1]), __double2float_ru(h[2]),
                             __int_as_float(-(nb[j] - na[j])));
        } else {
            lo = make_float4(INFINITY, INFINITY, INFINITY, __int_as_float(first[j]));
            hi = make_float4(-INFINITY, -INFINITY, -INFINITY, __int_as_float(nch[j]));
            for (int c = first[j]; c < first[j] + nch[j]; c++) {
                const float4 a = onode[2 * c], b = onode[2 * c + 1];
                lo.x = fminf(lo.x, a.x); lo.y = fminf(lo.y, a.y); lo.z = fminf(lo.z, a.z);
                hi.x = fmaxf(hi.x, b.x); hi.y = fmaxf(hi.y, b.y); hi.z = fmaxf(hi.z, b.z);
            }
        }
        onode[2 * j] = lo;
        onode[2 * j + 1] = hi;
    }
}

// ---------------------------------------------------------------------------
// query bucketing
// ---------------------------------------------------------------------------
template <class QT>
__device__ __forceinline__ dv3 load_query(const QT *__restrict__ Q, int64_t i, const double *cen) {
    // natinterp3d.py:115: np.ascontiguousarray(Q, float64) - centroid
    return dv3{fsub((double)Q[3 * i], cen[0]), fsub((double)Q[3 * i + 1], cen[1]),
               fsub((double)Q[3 * i + 2], cen[2])};
}

struct Centroid {
    double c[3];
};


template <class QT>
__global__ void k_bucket(const QT *__restrict__ Q, int64_t M, Centroid cen, MeshView mv, int bits,
                         int *__restrict__ bucket, int *__restrict__ bcount) {
    const double scale = (double)(1 << bits);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        const dv3 q = load_query(Q, i, cen.c);
        const double c[3] = {q.x, q.y, q.z};
        unsigned code = 0;
        for (int a = 0; a < 3; a++) {
            double f = (c[a] - mv.glo[a]) * mv.ginv[a] / (double)mv.gdim[a] * scale;
            int k = (f >= 0.0) ? (f < scale ? (int)f : (1 << bits) - 1) : 0;
            code |= spread3((unsigned)k) << a;
        }
        bucket[i] = (int)code;
        atomicAdd(&bcount[code], 1);
    }
}

__global__ void k_scatter(const int *__restrict__ bucket, int64_t M, int *__restrict__ cursor,
                          int *__restrict__ order) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int pos = atomicAdd(&cursor[bucket[i]], 1);
        order[pos] = (int)i;
    }
}

// ---------------------------------------------------------------------------
// exclusive scan (three passes): int32 input, OutT output, optional total
// ---------------------------------------------------------------------------
template <class OutT>
__global__ void k_scan_reduce(const int *__restrict__ in, int64_t n, OutT *__restrict__ bsum) {
    __shared__ OutT s[SCAN_THREADS];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    OutT acc = 0;
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_THREADS) {
        const int64_t i = base + k;
        if (i < n) acc += (OutT)in[i];
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = SCAN_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[blockIdx.x] = s[0];
}

// single block: exclusive scan of the block sums in place, total to *total
template <class OutT>
__global__ void k_scan_blocks(OutT *__restrict__ bsum, int nb, OutT *__restrict__ total) {
    __shared__ OutT s[SCAN_THREADS];
    __shared__ OutT carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nb; b0 += SCAN_THREADS) {
        const int i = b0 + threadIdx.x;
        const OutT v = (i < nb) ? bsum[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int w = 1; w < SCAN_THREADS; w <<= 1) {
            const OutT add = ((int)threadIdx.x >= w) ? s[threadIdx.x - w] : 0;
            __syncthreads();
            s[threadIdx.x] += add;
            __syncthreads();
        }
        if (i < nb) bsum[i] = carry + s[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == SCAN_THREADS - 1) carry += s[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class OutT>
__global__ void k_scan_apply(const int *__restrict__ in, int64_t n, const OutT *__restrict__ bsum,
                             OutT *__restrict__ out) {
    __shared__ OutT s[SCAN_THREADS];
    constexpr int PER = SCAN_TILE / SCAN_THREADS;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * PER;
    OutT v[PER];
    OutT acc = 0;
    for (int k = 0; k < PER; k++) {
        const int64_t i = base + k;
        v[k] = (i < n) ? (OutT)in[i] : 0;
        acc += v[k];
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 1; w < SCAN_THREADS; w <<= 1) {
        const OutT add = ((int)threadIdx.x >= w) ? s[threadIdx.x - w] : 0;
        __syncthreads();
        s[threadIdx.x] += add;
        __syncthreads();
    }
    OutT run = bsum[blockIdx.x] + s[threadIdx.x] - acc;
    for (int k = 0; k < PER; k++) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

// ---------------------------------------------------------------------------
// row sinks
// ---------------------------------------------------------------------------

// get_weights, count pass: every row's neighbour count and normaliser; rows
// of at most ROW_STAGE entries are staged at i * ROW_STAGE, longer rows are
// queued (refill) and recomputed straight into the final CSR by the fill
// pass, as are the rows the large kernel handled (their queue is the large-
// row list).  So no row ever needs more room than its final CSR slice.
struct StageSink {
    static constexpr bool FULL = true;
    int *__restrict__ cnt;          // [M] entries of the row (0 for empty / failed rows)
    uint8_t *__restrict__ staged;   // [M] 1: the row is staged
    int *__restrict__ cols;         // [M * ROW_STAGE]
    double *__restrict__ vals;      // [M * ROW_STAGE]
    int *__restrict__ refill;       // [M] fast-kernel rows longer than ROW_STAGE
    DevSummary *sum;
    double *__restrict__ total;     // [M] normaliser of each row (0 for empty rows)

    template <int G, class W>
    __device__ __forceinline__ void emit(int64_t i, int nnb, W &ws, const Grp<G> &g, bool large,
                                         const MeshView &, dv3, const RowInfo &r) {
        const bool stage = !large && nnb <= ROW_STAGE;
        if (stage) {
            const int64_t o = i * ROW_STAGE;
            for (int s = g.lane; s < nnb; s += G) {
                cols[o + s] = ws.nbr_vid[s];
                vals[o + s] = ws.acc[s];
            }
        }
        if (g.lane == 0) {
            total[i] = (nnb > 0) ? r.total : 0.0;
            cnt[i] = nnb;
            staged[i] = stage ? 1 : 0;
            if (!large && !stage) refill[atomicAdd(&sum->refill_count, 1)] = (int)i;
        }
    }
    __device__ __forceinline__ void empty(int64_t i, int lane) {
        if (lane == 0) {
            cnt[i] = 0;
            staged[i] = 1;
            total[i] = 0.0;
        }
    }
};

// get_weights, fill pass: a queued row recomputed into its final CSR slice
// (the same routine as the count pass, hence the same entries); a row whose
// count differs from its slice is an internal error and writes nothing
template <class VT>
struct DirectSink {
    static constexpr bool FULL = true;
    const int32_t *__restrict__ rowptr;
    int32_t *__restrict__ cols;
    VT *__restrict__ vals;
    DevSummary *sum;

    template <int G, class W>
    __device__ __forceinline__ void emit(int64_t i, int nnb, W &ws, const Grp<G> &g, bool,
                                         const MeshView &, dv3, const RowInfo &) {
        const int64_t o = rowptr[i];
        if (rowptr[i + 1] - o != nnb) {
            if (g.lane == 0) atomicCAS(&sum->first_status, 0, NIF_ERR_INTERNAL);
            return;
        }
        for (int s = g.lane; s < nnb; s += G) {
            cols[o + s] = ws.nbr_vid[s];
            vals[o + s] = (VT)ws.acc[s];
        }
    }
    __device__ __forceinline__ void empty(int64_t, int) {}
};

template <class T> struct Arith;
template <> struct Arith<double> {
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
};
template <> struct Arith<float> {
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
};

// interpolate: out[i, :] = sum over the row of (CT)(WT)w * (CT)values[col, :],
// accumulated from zero in stored order (scipy csr_matvec / csr_matvecs).
// natinterp3d's get_weights ends with W.astype(query dtype); for a float32
// query that conversion also canonicalises the CSR (columns sorted within each
// row), so with WT = float the row is accumulated in ascending column order.
template <class WT, class VT, class CT>
struct InterpSink {
    const VT *__restrict__ values;  // [N][D]
    CT *__restrict__ out;           // [M][D]
    int D;
    static constexpr bool FULL = true;
    static constexpr bool SORTED = sizeof(WT) == 4;

    template <int G, class W>
    __device__ __forceinline__ void emit(int64_t i, int nnb, W &ws, const Grp<G> &g, bool,
                                         const MeshView &, dv3, const RowInfo &) {
        CT *o = out + i * (int64_t)D;
        if (nnb == 0) {
            for (int d = g.lane; d < D; d += G) o[d] = (CT)0;
            return;
        }
        // the cavity-search scratch is free now: stage the products there
        double *buf = reinterpret_cast<double *>(&ws.u);
        constexpr int BUFN = (int)(sizeof(ws.u) / sizeof(double));
        if (SORTED) {
            // position of each neighbour in ascending column order (columns are distinct)
            for (int s = g.lane; s < nnb; s += G) {
                const int v = ws.nbr_vid[s];
                int r = 0;
                for (int t = 0; t < nnb; t++) r += ws.nbr_vid[t] < v;
                ws.vh_first[s] = r;
            }
        }
        const int dc = max(1, min(D, BUFN / nnb));
        for (int d0 = 0; d0 < D; d0 += dc) {
            const int nd = min(dc, D - d0);
            g.sync();
            for (int k = g.lane; k < nnb * nd; k += G) {
                const int s = k / nd, d = k - s * nd;
                const CT w = (CT)(WT)ws.acc[s];
                const CT x = (CT)values[(int64_t)ws.nbr_vid[s] * D + d0 + d];
                const int row = SORTED ? ws.vh_first[s] : s;
                buf[row * nd + d] = (double)Arith<CT>::mul(w, x);
            }
            g.sync();
            for (int d = g.lane; d < nd; d += G) {
                CT acc = (CT)0;
                for (int s = 0; s < nnb; s++) acc = Arith<CT>::add(acc, (CT)buf[s * nd + d]);
                o[d0 + d] = acc;
            }
        }
        g.sync();
    }
    __device__ __forceinline__ void empty(int64_t i, int lane) {
        CT *o = out + i * (int64_t)D;
        if (lane == 0)
            for (int d = 0; d < D; d++) o[d] = (CT)0;
    }
};

// d loss / d query: gq[i, :] = sum_k dL/dw_ik dw_ik/dq_i with dL/dw_ik =
// gout[i, :] . values[k, :] (derivation in nif_grad.cuh).  The forward pass's
// CSR weights and row normalisers are inputs; the kernel rebuilds only each
// row's cavity, boundary and neighbour order (whose column order matches the
// CSR row) and differentiates the virtual-tet volumes, one boundary face per
// lane.  Rows without a derivative (empty, outside the super-simplex, or
// exactly on a data site, where Sibson coordinates are only continuous) get
// zero.
template <class QT, class VT, class GT>
struct GradSink {
    static constexpr bool FULL = false;
    // the dual-number face gradient holds many FP64 values: fewer, larger threads
#ifndef NIF_GRAD_MINB
#define NIF_GRAD_MINB 4
#endif
    static constexpr int MIN_BLOCKS = NIF_GRAD_MINB;
    const VT *__restrict__ values;   // [N][D]
    const GT *__restrict__ gout;     // [M][D]
    const int32_t *__restrict__ rowptr;
    const double *__restrict__ w;    // CSR weights (float64) of the forward pass
    const double *__restrict__ total;// [M] row normalisers of the forward pass
    QT *__restrict__ gq;             // [M][3]
    int D;

    template <int G, class W>
    __device__ __forceinline__ void emit(int64_t i, int nnb, W &ws, const Grp<G> &g, bool,
                                         const MeshView &M, dv3 q, const RowInfo &r) {
        double gx = 0.0, gy = 0.0, gz = 0.0;
        const int64_t r0 = rowptr[i];
        const double S = total[i];
        if (nnb > 0 && !r.coincident && S > 1e-30 && rowptr[i + 1] - r0 == nnb) {
            double *ck = reinterpret_cast<double *>(&ws.u);  // free after the cavity search
            const GT *go = gout + i * (int64_t)D;
            for (int s = g.lane; s < nnb; s += G) {
                const VT *vr = values + (int64_t)ws.nbr_vid[s] * D;
                double a = 0.0;
                for (int d = 0; d < D; d++) a += (double)go[d] * (double)vr[d];
                ck[s] = a;
            }
            g.sync();
            double gbar = 0.0;
            if (g.lane == 0)
                for (int s = 0; s < nnb; s++) gbar += ck[s] * w[r0 + s];
            gbar = g.shfl(gbar, 0);
            const double inv_total = 1.0 / S;
            for (int s = g.lane; s < nnb; s += G) ck[s] = (ck[s] - gbar) * inv_total;
            g.sync();
            for (int b = g.lane; b < r.nbf; b += G) {
                const int cf = ws.bface[b];
                const int f = cf & 3;
                const int tt = ws.cav_tet[cf >> 2];
                const int4 p = M.tv[tt];
                const int va = comp(p, face_vslot(f, 0));
                const int vb = comp(p, face_vslot(f, 1));
                const int vc = comp(p, face_vslot(f, 2));
                const int sa = va < M.n ? neighbour_slot(ws, va) : -1;
                const int sb = vb < M.n ? neighbour_slot(ws, vb) : -1;
                const int sc = vc < M.n ? neighbour_slot(ws, vc) : -1;
                // virtual terms enter the stolen volumes with a minus sign
                const double c0 = sa >= 0 ? -ck[sa] : 0.0;
                const double c1 = sb >= 0 ? -ck[sb] : 0.0;
                const double c2 = sc >= 0 ? -ck[sc] : 0.0;
                if (c0 == 0.0 && c1 == 0.0 && c2 == 0.0) continue;
                const dv3 gf = virtual_face_grad(q, vload(M, va), vload(M, vb), vload(M, vc),
                                                 cload(&M.fcc[4 * (size_t)tt + (3 - f)]), c0, c1, c2);
                gx += gf.x;
                gy += gf.y;
                gz += gf.z;
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) {
                gx += __shfl_xor_sync(g.mask, gx, o, G);
                gy += __shfl_xor_sync(g.mask, gy, o, G);
                gz += __shfl_xor_sync(g.mask, gz, o, G);
            }
            g.sync();
        }
        if (g.lane == 0) {
            gq[3 * i] = (QT)gx;
            gq[3 * i + 1] = (QT)gy;
            gq[3 * i + 2] = (QT)gz;
        }
    }
};

// ---------------------------------------------------------------------------
// sparse products: CSR x dense and its transpose through a sorted CSC
// ---------------------------------------------------------------------------

// y[i, d] = sum over row i of w * x[col, d], accumulated from zero in stored
// order in the promoted type (scipy csr_matvecs)
template <class WT, class XT, class CT>
__global__ void k_spmm(int64_t M, int D, const int32_t *__restrict__ rowptr,
                       const int32_t *__restrict__ cols, const WT *__restrict__ vals,
                       const XT *__restrict__ x, CT *__restrict__ y) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < M * D;
         u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = u / D;
        const int d = (int)(u - i * D);
        CT acc = (CT)0;
        int e = rowptr[i];
        const int e1 = rowptr[i + 1];
        // four entries' loads issued together; the sum stays in stored order
        for (; e + 4 <= e1; e += 4) {
            const int c0 = cols[e], c1 = cols[e + 1], c2 = cols[e + 2], c3 = cols[e + 3];
            const CT w0 = (CT)vals[e], w1 = (CT)vals[e + 1], w2 = (CT)vals[e + 2], w3 = (CT)vals[e + 3];
            const CT x0 = (CT)x[(int64_t)c0 * D + d], x1 = (CT)x[(int64_t)c1 * D + d];
            const CT x2 = (CT)x[(int64_t)c2 * D + d], x3 = (CT)x[(int64_t)c3 * D + d];
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w0, x0));
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w1, x1));
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w2, x2));
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w3, x3));
        }
        for (; e < e1; e++)
            acc = Arith<CT>::add(acc, Arith<CT>::mul((CT)vals[e], (CT)x[(int64_t)cols[e] * D + d]));
        y[u] = acc;
    }
}

// sort key of entry e: its column, or the column's rank in a caller-given
// processing order (clamped to [0, N) so that a bad rank cannot leave the sort's range)
__global__ void k_row_of(int64_t M, const int32_t *__restrict__ rowptr, int32_t *__restrict__ rowof,
                         uint32_t *__restrict__ keys, const int32_t *__restrict__ cols,
                         int32_t *__restrict__ idx, const int32_t *__restrict__ rank, int64_t N) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x)
        for (int e = rowptr[i]; e < rowptr[i + 1]; e++) {
            rowof[e] = (int32_t)i;
            int k = cols[e];
            if (rank) {
                k = rank[k];
                k = k < 0 ? 0 : (k >= N ? (int)(N - 1) : k);
            }
            keys[e] = (uint32_t)k;
            idx[e] = e;
        }
}

// inverse of a processing order: inv[rank[k]] = k (entries a bad rank leaves
// unset stay -1 and are skipped)
__global__ void k_rank_inverse(int64_t N, const int32_t *__restrict__ rank, int32_t *__restrict__ inv) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int r = rank[k];
        if (r >= 0 && r < N) inv[r] = (int32_t)k;
    }
}

// stable LSD radix sort of (key, value) pairs, 4 bits per pass
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint32_t *__restrict__ keys, int64_t n,
                                                         int shift, int nblocks, int *__restrict__ hist) {
    __shared__ int h[16];
    if (threadIdx.x < 16) h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int j = 0; j < RS_ITEMS; j++) {
        const int64_t i = base + j * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 15u], 1);
    }
    __syncthreads();
    if (threadIdx.x < 16) hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

__device__ __forceinline__ unsigned long long pick4(unsigned long long c0, unsigned long long c1,
                                                    unsigned long long c2, unsigned long long c3,
                                                    int d) {
    const unsigned long long c = (d < 4) ? c0 : (d < 8 ? c1 : (d < 12 ? c2 : c3));
    return (c >> (16 * (d & 3))) & 0xffffull;
}

// Thread t of a block owns the tile's items 8t..8t+7 in order; an item's
// destination is the block's start for its digit (scanned histogram) plus
// the digit's count in earlier threads plus its rank inside its own thread,
// so equal keys keep their input order.  Counts are packed 16 bits per digit.
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(
    const uint32_t *__restrict__ kin, const int32_t *__restrict__ vin, int64_t n, int shift,
    int nblocks, const int *__restrict__ off, uint32_t *__restrict__ kout, int32_t *__restrict__ vout) {
    __shared__ uint32_t sk[RS_TILE];
    __shared__ int32_t sv[RS_TILE];
    __shared__ unsigned long long wsum[RS_THREADS / 32][4];
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int j = 0; j < RS_ITEMS; j++) {
        const int idx = j * RS_THREADS + threadIdx.x;
        if (base + idx < n) {
            sk[idx] = kin[base + idx];
            sv[idx] = vin[base + idx];
        }
    }
    __syncthreads();
    uint32_t mk[RS_ITEMS];
    int32_t mv[RS_ITEMS];
    int dg[RS_ITEMS], rk[RS_ITEMS];
    unsigned long long c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
    for (int j = 0; j < RS_ITEMS; j++) {
        const int idx = threadIdx.x * RS_ITEMS + j;
        dg[j] = -1;
        rk[j] = 0;
        mk[j] = 0;
        mv[j] = 0;
        if (base + idx < n) {
            mk[j] = sk[idx];
            mv[j] = sv[idx];
            const int d = (int)((mk[j] >> shift) & 15u);
            dg[j] = d;
            rk[j] = (int)pick4(c0, c1, c2, c3, d);
            const unsigned long long inc = 1ull << (16 * (d & 3));
            if (d < 4) c0 += inc; else if (d < 8) c1 += inc; else if (d < 12) c2 += inc; else c3 += inc;
        }
    }
    // exclusive scan of the packed counts over the block's threads
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long s0 = c0, s1 = c1, s2 = c2, s3 = c3;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t0 = __shfl_up_sync(0xffffffffu, s0, o);
        const unsigned long long t1 = __shfl_up_sync(0xffffffffu, s1, o);
        const unsigned long long t2 = __shfl_up_sync(0xffffffffu, s2, o);
        const unsigned long long t3 = __shfl_up_sync(0xffffffffu, s3, o);
        if (lane >= o) {
            s0 += t0; s1 += t1; s2 += t2; s3 += t3;
        }
    }
    if (lane == 31) {
        wsum[warp][0] = s0; wsum[warp][1] = s1; wsum[warp][2] = s2; wsum[warp][3] = s3;
    }
    __syncthreads();
    unsigned long long e0 = s0 - c0, e1 = s1 - c1, e2 = s2 - c2, e3 = s3 - c3;
    for (int w = 0; w < warp; w++) {
        e0 += wsum[w][0]; e1 += wsum[w][1]; e2 += wsum[w][2]; e3 += wsum[w][3];
    }
#pragma unroll
    for (int j = 0; j < RS_ITEMS; j++) {
        const int d = dg[j];
        if (d < 0) continue;
        const int64_t pos = (int64_t)off[(int64_t)d * nblocks + blockIdx.x] +
                            (int64_t)pick4(e0, e1, e2, e3, d) + rk[j];
        kout[pos] = mk[j];
        vout[pos] = mv[j];
    }
}

// colptr[k] = first position of key k in the sorted keys (lower bound)
__global__ void k_colptr(const uint32_t *__restrict__ keys, int64_t n, int64_t N,
                         int32_t *__restrict__ colptr) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= N;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((int64_t)keys[mid] < k) lo = mid + 1; else hi = mid;
        }
        colptr[k] = (int32_t)lo;
    }
}

// y[k, d] = sum over column k, ascending row, of w * x[row, d]
template <class WT, class XT, class CT>
__global__ void k_spmm_t(int64_t N, int D, const int32_t *__restrict__ colptr,
                         const int32_t *__restrict__ perm, const int32_t *__restrict__ rowof,
                         const WT *__restrict__ vals, const XT *__restrict__ x, CT *__restrict__ y,
                         const int32_t *__restrict__ inv) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < N * D;
         u += (int64_t)gridDim.x * blockDim.x) {
        // position r of the processing order: column k (keys in the caller's
        // order, or inv[r] for a caller-given order)
        const int64_t r = u / D;
        const int d = (int)(u - r * D);
        const int64_t k = inv ? (int64_t)inv[r] : r;
        if (k < 0 || k >= N) continue;
        CT acc = (CT)0;
        int p = colptr[r];
        const int p1 = colptr[r + 1];
        // four entries' loads issued together; the sum stays in ascending row order
        for (; p + 4 <= p1; p += 4) {
            const int e0 = perm[p], e1 = perm[p + 1], e2 = perm[p + 2], e3 = perm[p + 3];
            const int r0 = rowof[e0], r1 = rowof[e1], r2 = rowof[e2], r3 = rowof[e3];
            const CT w0 = (CT)vals[e0], w1 = (CT)vals[e1], w2 = (CT)vals[e2], w3 = (CT)vals[e3];
            const CT x0 = (CT)x[(int64_t)r0 * D + d], x1 = (CT)x[(int64_t)r1 * D + d];
            const CT x2 = (CT)x[(int64_t)r2 * D + d], x3 = (CT)x[(int64_t)r3 * D + d];
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w0, x0));
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w1, x1));
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w2, x2));
            acc = Arith<CT>::add(acc, Arith<CT>::mul(w3, x3));
        }
        for (; p < p1; p++) {
            const int e = perm[p];
            acc = Arith<CT>::add(acc, Arith<CT>::mul((CT)vals[e], (CT)x[(int64_t)rowof[e] * D + d]));
        }
        y[k * D + d] = acc;
    }
}

// ---------------------------------------------------------------------------
// row kernels
// ---------------------------------------------------------------------------
// problem of row i in a batch: off[p] <= i < off[p + 1]
__device__ __forceinline__ int find_problem(const int64_t *__restrict__ off, int P, int64_t i) {
    int lo = 0, hi = P;  // off[lo] <= i < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Where the split row kernels find a row's mesh and key centroid.
// OneMesh: every row queries one mesh (passed as a __grid_constant__ kernel
// argument).  ManyMeshes: a batch; row i belongs to problem p with
// qoff[p] <= i < qoff[p + 1], whose view the group caches in `slot` while
// consecutive rows stay in the same problem (`cur`).
struct OneMesh {
    MeshView M;
    Centroid cen;
    __device__ __forceinline__ const MeshView &get(int64_t, int &, MeshView *, const Grp<FAST_G> &,
                                                   const double *&c) const {
        c = cen.c;
        return M;
    }
};

struct ManyMeshes {
    const MeshView *__restrict__ views;
    const int64_t *__restrict__ qoff;
    int P;
    const double *__restrict__ cens;
    __device__ __forceinline__ const MeshView &get(int64_t i, int &cur, MeshView *slot,
                                                   const Grp<FAST_G> &g, const double *&c) const {
        const int p = find_problem(qoff, P, i);
        if (p != cur) {
            g.sync();
            if (g.lane == 0) *slot = views[p];
            g.sync();
            cur = p;
        }
        c = cens + 3 * p;
        return *slot;
    }
};

// Rows [s, s1) of work item t of the tiled schedule: tiles of `tile` rows,
// then the last `tail` rows (about `tile` per resident group) one at a
// time, so that the groups finish together instead of waiting on the last
// full tiles.
__device__ __forceinline__ void tile_range(unsigned long long t, int tile, int64_t nrows, int64_t tail,
                                           int64_t &s, int64_t &s1) {
    const int64_t nhead = nrows > tail ? (nrows - tail) / tile : 0;
    if ((int64_t)t < nhead) {
        s = (int64_t)t * tile;
        s1 = s + tile;
    } else {
        s = nhead * tile + ((int64_t)t - nhead);
        s1 = min(nrows, s + 1);
    }
}

struct LargeQueue {
    int *__restrict__ list;  // [M]
};

template <int G>
__device__ __forceinline__ void record(DevSummary *sum, const RowInfo &r, int lane) {
    if (lane != 0) return;
    if (r.outside) atomicAdd(&sum->rows_outside, 1ull);
}

// fast path: shared-memory scratch, rows in bucket order; PM is PM_PLAIN or
// PM_FILTER; OCC resident blocks per SM.  With tile == 0 group k takes rows
// k, k + ng, k + 2 ng, ...; with tile > 0 it takes tiles of `tile`
// consecutive rows from the device counter (zeroed before the launch).
template <class QT, class Sink, int PM, int OCC>
__global__ void __launch_bounds__(FAST_BLOCK, OCC) k_rows_fast(MeshView M, const QT *__restrict__ Q,
                                                          Centroid cen, const int *__restrict__ order,
                                                          int64_t nrows, const int *nrows_dev,
                                                          Sink sink, LargeQueue lq,
                                                          DevSummary *sum, int tile,
                                                          unsigned long long *counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    // a row count known only on the device (a queue's length) bounds nrows
    if (nrows_dev) nrows = min(nrows, (int64_t)*nrows_dev);
    constexpr int G = FAST_G;
    constexpr int GPB = FAST_BLOCK / G;
    Grp<G> g;
    FastWS &ws = reinterpret_cast<FastWS *>(smem)[threadIdx.x / G];
    const int64_t gid = tile <= 0 ? (int64_t)blockIdx.x * GPB + threadIdx.x / G : 0;
    const int64_t ng = (int64_t)gridDim.x * GPB;
    unsigned long long steps = 0;
    // one loop for both schedules, so that the row routine is inlined once
    int64_t s = gid, s1 = tile <= 0 ? nrows : 0;  // tiled: fetch a tile first
    for (;;) {
        if (s >= s1) {
            if (tile <= 0) break;
            unsigned long long t = 0;
            if (g.lane == 0) t = atomicAdd(counter, 1ull);
            t = __shfl_sync(g.mask, t, 0, G);
            tile_range(t, tile, nrows, ng * tile, s, s1);
            if (s >= nrows) break;
        }
        const int64_t i = order[s];
        const dv3 q = load_query(Q, i, cen.c);
        const RowInfo r = sibson_row<G, FastWS, Sink::FULL, PM>(M, q, ws, g);
        steps += r.steps;
        if (r.status == ST_CAPACITY || r.status == ST_UNCERTAIN) {
            if (g.lane == 0) {
                const int slot = atomicAdd(&sum->large_count, 1);
                lq.list[slot] = (int)i;
            }
        } else {
            if (r.status != ST_OK && g.lane == 0) {
                atomicAdd(&sum->rows_failed, 1ull);
                atomicCAS(&sum->first_status, 0, NIF_ERR_WALK);
            }
            record<G>(sum, r, g.lane);
            sink.template emit<G>(i, r.status == ST_OK ? r.nnb : 0, ws, g, false, M, q, r);
        }
        g.sync();
        s += tile <= 0 ? ng : 1;
    }
    if (g.lane == 0 && steps) atomicAdd(&sum->walk_steps, steps);
}

// Point location of every row: one warp per row, rows in bucket order as
// the row kernels take them; located[i] = the tet, -1 outside the
// super-simplex, -2 a walk that hit its step limit, -3 (PM_FILTER) a walk
// test the error bound cannot certify (the large kernel resolves the row).
template <class QT, class Rows, int PM = PM_PLAIN>
__global__ void __launch_bounds__(FAST_BLOCK) k_locate(const __grid_constant__ Rows rows,
                                                       const QT *__restrict__ Q,
                                                       const int *__restrict__ order, int64_t nrows,
                                                       int *__restrict__ located, DevSummary *sum,
                                                       int tile, unsigned long long *counter) {
    constexpr int G = 32;
    constexpr int GPB = FAST_BLOCK / G;
    __shared__ int scratch[GPB][64];
    __shared__ MeshView sview[GPB];
    Grp<G> g;
    int *scr = scratch[threadIdx.x / G];
    int cur = -1;
    const int64_t gid = tile <= 0 ? (int64_t)blockIdx.x * GPB + threadIdx.x / G : 0;
    const int64_t ng = (int64_t)gridDim.x * GPB;
    unsigned long long steps = 0;
    int64_t s = gid, s1 = tile <= 0 ? nrows : 0;
    for (;;) {
        if (s >= s1) {
            if (tile <= 0) break;
            unsigned long long t = 0;
            if (g.lane == 0) t = atomicAdd(counter, 1ull);
            t = __shfl_sync(g.mask, t, 0, G);
            tile_range(t, tile, nrows, ng * tile, s, s1);
            if (s >= nrows) break;
        }
        const int64_t i = order[s];
        const double *cen;
        const MeshView &M = rows.get(i, cur, &sview[threadIdx.x / G], g, cen);
        const dv3 q = load_query(Q, i, cen);
        RowInfo r{ST_OK, 0, 0, false, false, 0.0, 0, 0, 0, 0, 0};
        bool on_face = false;
        const int t = locate<G, PM>(M, q, g, scr, r, on_face);
        steps += r.steps;
        if (g.lane == 0)
            located[i] = r.status == ST_UNCERTAIN ? -3
                         : (r.status != ST_OK ? -2 : (r.outside ? -1 : t));
        g.sync();
        s += tile <= 0 ? ng : 1;
    }
    if (g.lane == 0 && steps) atomicAdd(&sum->walk_steps, steps);
}

// The split row kernels (natinterp3d's signs, located rows): k_rows_cavity
// writes each row's record, k_rows_volume reads it and emits the row.  Rows
// are positions [0, nrows) of `order` (one chunk of a call); record s
// belongs to position s.  Each kernel holds one half of the row code.
// Rows whose cavity fits the shared-memory capacities but not a record are
// queued in `wide` for the fused row kernel, larger ones for the large kernel.
template <class QT, class Rows, int OCC, int PM = PM_PLAIN>
__global__ void __launch_bounds__(FAST_BLOCK, OCC)
    k_rows_cavity(const __grid_constant__ Rows rows, const QT *__restrict__ Q,
                  const int *__restrict__ order, int64_t nrows, const int *__restrict__ located,
                  RowHead *__restrict__ heads, RowEntry *__restrict__ ents, int *__restrict__ wide,
                  LargeQueue lq, DevSummary *sum, int tile, unsigned long long *counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int G = FAST_G;
    constexpr int GPB = FAST_BLOCK / G;
    __shared__ MeshView sview[GPB];
    Grp<G> g;
    CavWS &ws = reinterpret_cast<CavWS *>(smem)[threadIdx.x / G];
    int cur = -1;
    const int64_t gid = tile <= 0 ? (int64_t)blockIdx.x * GPB + threadIdx.x / G : 0;
    const int64_t ng = (int64_t)gridDim.x * GPB;
    int64_t s = gid, s1 = tile <= 0 ? nrows : 0;
    for (;;) {
        if (s >= s1) {
            if (tile <= 0) break;
            unsigned long long t = 0;
            if (g.lane == 0) t = atomicAdd(counter, 1ull);
            t = __shfl_sync(g.mask, t, 0, G);
            tile_range(t, tile, nrows, ng * tile, s, s1);
            if (s >= nrows) break;
        }
        const int64_t i = order[s];
        const int t = located[i];
        RowHead h{0, t, RS_OK, 0};
        if (t == -1) {
            h.state = RS_OUTSIDE;
        } else if (t == -3) {
            h.state = RS_QUEUED;
            if (g.lane == 0) lq.list[atomicAdd(&sum->large_count, 1)] = (int)i;
        } else if (t < 0) {
            h.state = RS_WALK;
        } else {
            const double *cen;
            const MeshView &M = rows.get(i, cur, &sview[threadIdx.x / G], g, cen);
            const dv3 q = load_query(Q, i, cen);
            const int rc = cavity_record<G, CavWS, PM>(M, q, ws, g, t, h, ents + s * REC_CAV);
            if (rc != REC_DONE) {
                h.state = RS_QUEUED;
                if (g.lane == 0) {
                    if (rc == REC_WIDE)
                        wide[atomicAdd(&sum->wide_count, 1)] = (int)i;
                    else
                        lq.list[atomicAdd(&sum->large_count, 1)] = (int)i;
                }
            }
        }
        if (g.lane == 0) heads[s] = h;
        g.sync();
        s += tile <= 0 ? ng : 1;
    }
}

// The split rows' visiting order: each record entry gets its position in
// natinterp3d's LIFO visiting order (natural_insertionfree.c:486-551,
// replayed on the cavity; its non-cavity tets are leaves and do not change
// the order) and which of its faces take a neighbour's face-cache copy;
// k_rows_volume derives the fcc[] indices from these.  One warp takes 32
// consecutive rows: the lanes load the rows' neighbour bytes into shared
// memory entry by entry, each lane replays one row there, and the lanes
// write the positions back entry by entry.  Rows without a cavity record
// are left alone.
constexpr int ORD_WARPS = 2;
constexpr int ORD_PAD = REC_CAV + 1;  // row stride of the shared tables (banks)
struct OrderWS {
    int nbr[32][ORD_PAD];
    int8_t stack[32][4 * REC_CAV + 1];
    int8_t pos[32][REC_CAV];
    int start[33];
};

__global__ void __launch_bounds__(32 * ORD_WARPS) k_rows_order(int64_t nrows, const RowHead *__restrict__ heads,
                                                               RowEntry *__restrict__ ents) {
    extern __shared__ __align__(16) unsigned char smem[];
    OrderWS &w = reinterpret_cast<OrderWS *>(smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int64_t ngroups = (nrows + 31) / 32;
    for (int64_t gi = (int64_t)blockIdx.x * ORD_WARPS + (threadIdx.x >> 5); gi < ngroups;
         gi += (int64_t)gridDim.x * ORD_WARPS) {
        const int64_t s0 = gi * 32;
        const int64_t s = s0 + lane;
        int nc = 0;
        if (s < nrows) {
            const RowHead h = heads[s];
            if (h.state == RS_OK && h.ncav > 0 && h.ncav <= REC_CAV) nc = h.ncav;
        }
        // entry offsets of the 32 rows in one flattened index space
        int incl = nc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(full, incl, off);
            if (lane >= off) incl += v;
        }
        w.start[lane] = incl - nc;
        if (lane == 31) w.start[32] = incl;
        __syncwarp();
        const int total = w.start[32];
        // row of flattened entry k: the last row whose start is <= k
        auto row_of = [&](int k) {
            int lo = 0, hi = 32;  // start[lo] <= k < start[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (w.start[mid] <= k) lo = mid; else hi = mid;
            }
            // skip empty rows that share the start
            while (w.start[lo + 1] <= k) lo++;
            return lo;
        };
        // the neighbour bytes of each entry, ORD_LOADS loads in flight a lane
        constexpr int ORD_LOADS = 6;
        for (int k0 = lane; k0 < total; k0 += 32 * ORD_LOADS) {
            int x[ORD_LOADS];
            int jj[ORD_LOADS], ee[ORD_LOADS];
#pragma unroll
            for (int u = 0; u < ORD_LOADS; u++) {
                const int k = k0 + 32 * u;
                if (k < total) {
                    jj[u] = row_of(k);
                    ee[u] = k - w.start[jj[u]];
                    x[u] = ents[(s0 + jj[u]) * REC_CAV + ee[u]].nbr;
                }
            }
#pragma unroll
            for (int u = 0; u < ORD_LOADS; u++) {
                if (k0 + 32 * u < total) w.nbr[jj[u]][ee[u]] = x[u];
            }
        }
        __syncwarp();
        if (nc > 0) {
            int8_t *stack = w.stack[lane];
            int8_t *pos = w.pos[lane];
            const int *nb = w.nbr[lane];
            for (int c = 0; c < nc; c++) pos[c] = 0;
            uint64_t vis = 0;
            int sp = 0, nord = 0;
            stack[sp++] = 0;  // the flood put the located tet first
            while (sp > 0) {
                const int c = stack[--sp];
                if ((vis >> c) & 1ull) continue;
                vis |= 1ull << c;
                pos[c] = (int8_t)nord++;
                const unsigned wd = (unsigned)nb[c];
#pragma unroll
                for (int f = 0; f < 4; f++) {
                    const int n = (int8_t)((wd >> (8 * f)) & 0xffu);
                    if (n >= 0 && !((vis >> n) & 1ull)) stack[sp++] = (int8_t)n;
                }
            }
        }
        __syncwarp();
        // each entry's position, and in bits 8-11 which of its faces natinterp3d's
        // face cache answers with a neighbour's copy (the neighbour across face
        // 3 - i was visited earlier: bit i)
        for (int k = lane; k < total; k += 32) {
            const int j = row_of(k), e = k - w.start[j];
            const int pe = w.pos[j][e];
            const unsigned wd = (unsigned)w.nbr[j][e];
            unsigned take = 0;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int n = (int8_t)((wd >> (8 * (3 - i))) & 0xffu);
                if (n >= 0 && w.pos[j][n] < pe) take |= 1u << i;
            }
            ents[(s0 + j) * REC_CAV + e].pos = pe | (int)(take << 8);
        }
        __syncwarp();
    }
}

template <class QT, class Rows, class Sink, int OCC>
__global__ void __launch_bounds__(FAST_BLOCK, OCC)
    k_rows_volume(const __grid_constant__ Rows rows, const QT *__restrict__ Q,
                  const int *__restrict__ order, int64_t nrows, const RowHead *__restrict__ heads,
                  const RowEntry *__restrict__ ents, Sink sink, LargeQueue lq, DevSummary *sum,
                  int tile, unsigned long long *counter) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int G = FAST_G;
    constexpr int GPB = FAST_BLOCK / G;
    __shared__ MeshView sview[GPB];
    Grp<G> g;
    VolWS &ws = reinterpret_cast<VolWS *>(smem)[threadIdx.x / G];
    int cur = -1;
    const int64_t gid = tile <= 0 ? (int64_t)blockIdx.x * GPB + threadIdx.x / G : 0;
    const int64_t ng = (int64_t)gridDim.x * GPB;
    int64_t s = gid, s1 = tile <= 0 ? nrows : 0;
    for (;;) {
        if (s >= s1) {
            if (tile <= 0) break;
            unsigned long long t = 0;
            if (g.lane == 0) t = atomicAdd(counter, 1ull);
            t = __shfl_sync(g.mask, t, 0, G);
            tile_range(t, tile, nrows, ng * tile, s, s1);
            if (s >= nrows) break;
        }
        const int64_t i = order[s];
        const RowHead h = heads[s];
        if (h.state != RS_QUEUED) {
            const double *cen;
            const MeshView &M = rows.get(i, cur, &sview[threadIdx.x / G], g, cen);
            const dv3 q = load_query(Q, i, cen);
            RowInfo r{ST_OK, 0, 0, h.state == RS_OUTSIDE, false, 0.0, 0, 0, 0, 0, 0};
            if (h.state == RS_OK) r = volume_row<G, VolWS, Sink::FULL>(M, q, ws, g, h, ents + s * REC_CAV);
            if (h.state == RS_WALK) r.status = ST_WALK;
            if (r.status == ST_CAPACITY) {
                if (g.lane == 0) lq.list[atomicAdd(&sum->large_count, 1)] = (int)i;
            } else {
                if (r.status != ST_OK && g.lane == 0) {
                    atomicAdd(&sum->rows_failed, 1ull);
                    atomicCAS(&sum->first_status, 0, NIF_ERR_WALK);
                }
                record<G>(sum, r, g.lane);
                sink.template emit<G>(i, r.status == ST_OK ? r.nnb : 0, ws, g, false, M, q, r);
            }
        }
        g.sync();
        s += tile <= 0 ? ng : 1;
    }
}

template <int G>
__device__ __forceinline__ void record_predicates(DevSummary *sum, const RowInfo &r, int lane) {
    if (lane != 0) return;
    if (r.o_unc) atomicAdd(&sum->orient_unc, (unsigned long long)r.o_unc);
    if (r.o_flip) atomicAdd(&sum->orient_flip, (unsigned long long)r.o_flip);
    if (r.i_unc) atomicAdd(&sum->insphere_unc, (unsigned long long)r.i_unc);
    if (r.i_flip) atomicAdd(&sum->insphere_flip, (unsigned long long)r.i_flip);
}

// large path: one warp per queued row, scratch in global memory; resolves
// uncertain predicates exactly (xs: NIF_EXACT_SCRATCH doubles per block)
template <class QT, class Sink>
__global__ void __launch_bounds__(32) k_rows_large(MeshView M, const QT *__restrict__ Q, Centroid cen,
                                                   LargeQueue lq, Sink sink, LargeWS *__restrict__ wsv,
                                                   double *__restrict__ xsv, DevSummary *sum) {
    constexpr int G = LARGE_G;
    Grp<G> g;
    LargeWS &ws = wsv[blockIdx.x];
    double *xs = xsv + (size_t)blockIdx.x * NIF_EXACT_SCRATCH;
    const int nq = sum->large_count;
    unsigned long long steps = 0;
    for (int j = blockIdx.x; j < nq; j += gridDim.x) {
        const int64_t i = lq.list[j];
        const dv3 q = load_query(Q, i, cen.c);
        const RowInfo r = sibson_row<G, LargeWS, Sink::FULL, PM_RESOLVE>(M, q, ws, g, xs);
        steps += r.steps;
        record_predicates<G>(sum, r, g.lane);
        if (g.lane == 0) atomicAdd(&sum->rows_large, 1ull);
        if (r.status != ST_OK) {
            if (g.lane == 0) {
                atomicAdd(&sum->rows_failed, 1ull);
                atomicCAS(&sum->first_status, 0,
                          r.status == ST_WALK ? NIF_ERR_WALK : NIF_ERR_CAPACITY);
            }
            sink.template emit<G>(i, 0, ws, g, true, M, q, r);
        } else {
            record<G>(sum, r, g.lane);
            sink.template emit<G>(i, r.nnb, ws, g, true, M, q, r);
        }
        g.sync();
    }
    if (g.lane == 0 && steps) atomicAdd(&sum->walk_steps, steps);
}

// CSR compaction of the staged rows: 8 lanes per row
template <class VT>
__global__ void k_compact(int64_t M, const int *__restrict__ cnt, const uint8_t *__restrict__ staged,
                          const int *__restrict__ scols, const double *__restrict__ svals,
                          const int32_t *__restrict__ rowptr, int32_t *__restrict__ cols,
                          VT *__restrict__ vals) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t u = tid; u < M * 8; u += stride) {
        const int64_t i = u >> 3;
        if (!staged[i]) continue;
        const int l = (int)(u & 7);
        const int n = cnt[i];
        const int64_t s = i * ROW_STAGE;
        const int64_t d = rowptr[i];
        for (int k = l; k < n; k += 8) {
            cols[d + k] = scols[s + k];
            vals[d + k] = (VT)svals[s + k];
        }
    }
}

__global__ void k_rowptr32(const int64_t *__restrict__ off, int64_t M, int64_t total,
                           int32_t *__restrict__ rowptr) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= M;
         i += (int64_t)gridDim.x * blockDim.x)
        rowptr[i] = (int32_t)(i < M ? off[i] : total);
}

// FP64 throughput probe: 8 independent chains per thread of either
// separately rounded multiply and add (2 instructions, 2 flops) or fused
// multiply-add (1 instruction, 2 flops).
template <bool FUSED>
__global__ void k_fp64_peak(double *out, int iters, double b, double c) {
    double a[8];
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-9 + k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = FUSED ? __fma_rn(a[k], b, c) : __dadd_rn(__dmul_rn(a[k], b), c);
    }
    double r = 0.0;
    for (int k = 0; k < 8; k++) r += a[k];
    if (r == 12345.678) out[0] = r;  // keeps the chains live
}

}  // namespace nif

using namespace nif;

// ===========================================================================
// host side
// ===========================================================================
struct nif_dmesh {
    MeshView view;
    int n_vertices, n_tets;
    int device;
    int num_sms;
    size_t bytes;
    int64_t orient_unc, orient_flip;  // tets with an uncertain / flipped orientation flag
    int oct_nodes, oct_levels;        // centroid octree: nodes, node levels
    nif_tuning tune{OCC_DEFAULT, 0, MESH_TILE_DEFAULT, 0};
};

namespace {

struct Carve {
    unsigned char *base;
    size_t off;
    size_t cap;
    bool ok;
    template <class T>
    T *take(size_t count) {
        off = align_up(off, 256);
        T *p = reinterpret_cast<T *>(base + off);
        off += count * sizeof(T);
        if (off > cap) ok = false;
        return p;
    }
};

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline int cuda_rc(cudaError_t e) { return e == cudaSuccess ? NIF_OK : NIF_ERR_CUDA; }

#define NIF_CUDA(call)                                  \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return NIF_ERR_CUDA;     \
    } while (0)

// Octree nodes the resident mesh has room for.  A typical mesh needs far
// fewer (about one per 50 tets on uniform keys); where a level would exceed
// the room, its nodes stay leaves -- larger leaves, same results.
int oct_node_cap(int nt) { return nt / 8 + 1024; }

// Seed-grid cells per tet (about two centroids a cell), and the cells the
// resident mesh has room for.
#ifndef NIF_GRID_CELLS_PER_TET
#define NIF_GRID_CELLS_PER_TET 0.5
#endif
int grid_cell_cap(int nt) { return (int)(NIF_GRID_CELLS_PER_TET * nt) + 64; }

// Scratch of the centroid sort and octree build at mesh creation, carved
// from the start of the face-circumcentre array (filled only afterwards).
struct OctScratch {
    uint32_t *chi, *clo, *key_a, *key_b;
    int32_t *idx_a, *idx_b;
    int *hist, *off, *bsum, *tot;
    int64_t nblocks;
    unsigned long long *code;
    int *node_of, *flag, *scan;
    int *na, *nb, *par, *first, *nch;
    int *gcursor;
};

OctScratch carve_oct_scratch(Carve &c, int nt) {
    OctScratch S;
    const int cap = oct_node_cap(nt);
    S.nblocks = (nt + RS_TILE - 1) / RS_TILE;
    S.chi = c.take<uint32_t>(nt);
    S.clo = c.take<uint32_t>(nt);
    S.key_a = c.take<uint32_t>(nt);
    S.key_b = c.take<uint32_t>(nt);
    S.idx_a = c.take<int32_t>(nt);
    S.idx_b = c.take<int32_t>(nt);
    S.hist = c.take<int>(16 * S.nblocks);
    S.off = c.take<int>(16 * S.nblocks);
    S.bsum = c.take<int>((16 * S.nblocks + nt + SCAN_TILE - 1) / SCAN_TILE + 1);
    S.tot = c.take<int>(2);
    S.code = c.take<unsigned long long>(nt);
    S.node_of = c.take<int>(nt);
    S.flag = c.take<int>(nt);
    S.scan = c.take<int>(nt);
    S.na = c.take<int>(cap);
    S.nb = c.take<int>(cap);
    S.par = c.take<int>(cap);
    S.first = c.take<int>(cap);
    S.nch = c.take<int>(cap);
    S.gcursor = c.take<int>(grid_cell_cap(nt));
    return S;
}

// face-circumcentre slots: 4 per tet, more for tiny meshes so that the
// build scratch fits
size_t fcc_slots(int nt) {
    Carve c{nullptr, 0, (size_t)-1, true};
    carve_oct_scratch(c, nt);
    const size_t need = (align_up(c.off, 256) + sizeof(d4) - 1) / sizeof(d4);
    return need > 4 * (size_t)nt ? need : 4 * (size_t)nt;
}

struct MeshLayout {
    d4 *vtx;
    int4 *tv, *tn;
    uint32_t *tinfo;
    d4 *tcc, *fcc;
    d4 *cs;                      // sorted centroids
    float4 *onode;               // octree node records, two float4 each
    unsigned long long *omask;   // octree child digits
    int *gstart;                 // seed grid: cell starts
    d4 *gitems;                  // seed grid: centroids by cell
    double *bbox_part;
    int *flag;
};

MeshLayout carve_mesh(Carve &c, int nv, int nt) {
    MeshLayout L;
    L.vtx = c.take<d4>(nv);
    L.tv = c.take<int4>(nt);
    L.tn = c.take<int4>(nt);
    L.tinfo = c.take<uint32_t>(nt);
    L.tcc = c.take<d4>(nt);
    L.fcc = c.take<d4>(fcc_slots(nt));
    L.cs = c.take<d4>(nt);
    L.onode = c.take<float4>(2 * (size_t)oct_node_cap(nt));
    L.omask = c.take<unsigned long long>(oct_node_cap(nt));
    L.gstart = c.take<int>(grid_cell_cap(nt) + 1);
    L.gitems = c.take<d4>(nt);
    L.bbox_part = c.take<double>(6 * 256);
    L.flag = c.take<int>(4);
    return L;
}

int blocks_for(int64_t n, int threads, int cap = 148 * 32) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

// query workspace layout
struct QueryLayout {
    DevSummary *sum;
    unsigned long long *counter;  // work-item counter of the tiled row schedule
    int bits_cap;                 // largest bucket resolution bcount holds (bits per axis)
    int *bucket, *bcount, *order, *large_list;
    int64_t *scan_bsum;     // block sums for the scans
    int64_t *scan_total;
    LargeWS *large_ws;
    double *exact;          // NIF_EXACT_SCRATCH doubles per large-row group
    int *located;           // k_locate's tet per row (null: the row kernel locates)
    RowHead *heads;         // split-row records of one chunk of rows
    RowEntry *ents;
    int *wide;              // split rows whose cavity exceeds a record
    // weights mode only
    int *cnt;
    uint8_t *staged;
    int64_t *off64;
    int *scols;             // staged rows, ROW_STAGE entries each
    double *svals;
    double *rtot;           // per-row normaliser
    int *refill;            // fast-kernel rows longer than ROW_STAGE
    DevSummary *fill_sum;   // counters of the fill pass's recomputed rows
};

constexpr int bucket_bits(int64_t M) {
    int b = 1;
    while (b < 10 && ((int64_t)1 << (3 * (b + 1))) <= M / 2) b++;
    return b;
}

// The layout does not depend on the mesh's tuning: bcount has room for one
// bucket bit per axis more than the default, and run_bucketing clamps to it.
QueryLayout carve_query(Carve &c, int64_t M, int mode) {
    QueryLayout L{};
    const int bits = min(10, bucket_bits(M) + 1);
    const int64_t nbk = (int64_t)1 << (3 * bits);
    const int64_t mscan = M > nbk ? M : nbk;
    L.bits_cap = bits;
    L.sum = c.take<DevSummary>(1);
    L.counter = c.take<unsigned long long>(1);
    L.bucket = c.take<int>(M > 0 ? M : 1);
    L.bcount = c.take<int>(nbk + 1);
    L.order = c.take<int>(M > 0 ? M : 1);
    L.large_list = c.take<int>(M > 0 ? M : 1);
    L.scan_bsum = c.take<int64_t>((mscan + SCAN_TILE - 1) / SCAN_TILE + 1);
    L.scan_total = c.take<int64_t>(1);
    L.large_ws = c.take<LargeWS>(LARGE_GROUPS);
    L.exact = c.take<double>((size_t)LARGE_GROUPS * NIF_EXACT_SCRATCH);
    L.located = c.take<int>(M > 0 ? M : 1);
    {
        const int64_t ch = M < REC_CHUNK ? (M > 0 ? M : 1) : REC_CHUNK;
        L.heads = c.take<RowHead>(ch);
        L.ents = c.take<RowEntry>(ch * REC_CAV);
        L.wide = c.take<int>(M > 0 ? M : 1);
    }
    if (mode == NIF_MODE_WEIGHTS) {
        const int64_t m1 = M > 0 ? M : 1;
        L.cnt = c.take<int>(m1);
        L.staged = c.take<uint8_t>(m1);
        L.off64 = c.take<int64_t>(M + 1);
        L.scols = c.take<int>(m1 * ROW_STAGE);
        L.svals = c.take<double>(m1 * ROW_STAGE);
        L.rtot = c.take<double>(m1);
        L.refill = c.take<int>(m1);
        L.fill_sum = c.take<DevSummary>(1);
    }
    return L;
}

// Split-row records of every row of a get_weights call, kept for the
// gradient of the same rows (nif_weights_count_records /
// nif_query_grad_records), and the gradient pass's own scratch: rows it
// would queue again are already in the forward's queues, so its re-queues
// go to `requeue` and are dropped.
struct RecordLayout {
    RowHead *heads;          // [M], record of bucket position s at s
    RowEntry *ents;          // [M * REC_CAV]
    DevSummary *sum;         // counters of the gradient's record and wide passes
    DevSummary *large_sum;   // the forward's counters: the large pass's queue length
    int *requeue;            // [M]
    unsigned long long *counter;
};

RecordLayout carve_records(Carve &c, int64_t M) {
    RecordLayout R{};
    const int64_t m1 = M > 0 ? M : 1;
    R.heads = c.take<RowHead>(m1);
    R.ents = c.take<RowEntry>(m1 * REC_CAV);
    R.sum = c.take<DevSummary>(1);
    R.large_sum = c.take<DevSummary>(1);
    R.requeue = c.take<int>(m1);
    R.counter = c.take<unsigned long long>(1);
    return R;
}

template <class OutT>
void launch_scan(const int *in, int64_t n, OutT *bsum, OutT *total, OutT *out, cudaStream_t st) {
    const int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 0) {
        k_scan_blocks<OutT><<<1, SCAN_THREADS, 0, st>>>(bsum, 0, total);
        return;
    }
    k_scan_reduce<OutT><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, bsum);
    k_scan_blocks<OutT><<<1, SCAN_THREADS, 0, st>>>(bsum, (int)nb, total);
    k_scan_apply<OutT><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, bsum, out);
}

template <class Kern>
int set_smem(Kern k, size_t bytes) {
    return cuda_rc(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// Resident blocks per SM of kernel k with `smem` bytes of dynamic shared
// memory, on the current device.  The first call per (kernel, device) sets
// the kernel's shared-memory limit there and queries the occupancy; the
// answer is cached, and concurrent first calls from several host threads are
// serialised.
template <class Kern>
int resident_blocks(Kern k, int threads, size_t smem) {
    constexpr int DEVS = 64;
    static std::mutex mu;
    static int cache[DEVS] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < DEVS && cache[dev] > 0) return cache[dev];
    if (smem > 48 * 1024) set_smem(k, smem);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem) != cudaSuccess || n < 1)
        n = 1;
    if (dev >= 0 && dev < DEVS) cache[dev] = n;
    return n;
}

// Optional phase timing (nif_profile_enable / nif_profile_read): events
// recorded on the launching stream between the phases of a query call, one
// set per call in a ring of PROF_RING sets, so that timed loops never wait
// on the host; nif_profile_read averages the calls recorded since the last
// enable or read.
// Within the row phase, events also bracket each launch of the row kernels
// (kernel spans, by kind), so that the time of one kernel is known apart
// from the others.
constexpr int PROF_EVENTS = 5;  // start | bucketing | fast rows | large rows | finish
constexpr int PROF_RING = 64;
constexpr int PROF_SPANS = 48;  // kernel spans recorded per call (further launches are not)
constexpr int PROF_KINDS = 5;   // k_locate | k_rows_cavity | k_rows_volume | k_rows_fast | k_rows_order
enum { SPAN_LOCATE = 0, SPAN_CAVITY = 1, SPAN_VOLUME = 2, SPAN_FUSED = 3, SPAN_ORDER = 4 };
struct Profiler {
    bool on = false;
    bool created = false;
    int calls = 0;     // calls started since enable / read (the ring keeps the last PROF_RING)
    int marks = 0;     // marks of the current call
    cudaEvent_t ev[PROF_RING][PROF_EVENTS];
    cudaEvent_t sev[PROF_RING][PROF_SPANS][2];
    int skind[PROF_RING][PROF_SPANS];
    int nspan[PROF_RING];
    // per-kind averages of the calls the last nif_profile_read covered
    double kms[PROF_KINDS], klaunch[PROF_KINDS];
};
Profiler g_prof;

inline void prof_mark(int k, cudaStream_t st) {
    if (!g_prof.on) return;
    if (!g_prof.created) {
        for (int r = 0; r < PROF_RING; r++) {
            for (int i = 0; i < PROF_EVENTS; i++) cudaEventCreate(&g_prof.ev[r][i]);
            for (int i = 0; i < PROF_SPANS; i++) {
                cudaEventCreate(&g_prof.sev[r][i][0]);
                cudaEventCreate(&g_prof.sev[r][i][1]);
            }
        }
        g_prof.created = true;
    }
    if (k == 0) {
        g_prof.calls++;
        g_prof.marks = 0;
        g_prof.nspan[(g_prof.calls - 1) % PROF_RING] = 0;
    }
    if (g_prof.calls == 0) return;
    cudaEventRecord(g_prof.ev[(g_prof.calls - 1) % PROF_RING][k], st);
    g_prof.marks = k + 1;
}

// brackets one row-kernel launch of the current call (begin: end = false)
inline void prof_span(int kind, bool end, cudaStream_t st) {
    if (!g_prof.on || !g_prof.created || g_prof.calls == 0 || g_prof.marks != 2) return;
    const int r = (g_prof.calls - 1) % PROF_RING;
    int &n = g_prof.nspan[r];
    if (n >= PROF_SPANS) return;
    cudaEventRecord(g_prof.sev[r][n][end ? 1 : 0], st);
    if (end) g_prof.skind[r][n++] = kind;
}

// bucket the queries (writes L.order); positions fit int32 because M < 2^31
template <class QT>
void run_bucketing(const nif_dmesh *m, const QT *Q, int64_t M, const Centroid &cen,
                   const QueryLayout &L, cudaStream_t st) {
    const int bits = max(1, min(L.bits_cap, bucket_bits(M) + m->tune.bucket_shift));
    const int64_t nbk = (int64_t)1 << (3 * bits);
    prof_mark(0, st);
    cudaMemsetAsync(L.bcount, 0, sizeof(int) * (nbk + 1), st);
    k_bucket<QT><<<blocks_for(M, 256), 256, 0, st>>>(Q, M, cen, m->view, bits, L.bucket, L.bcount);
    // in-place exclusive scan: bucket starts become the scatter cursors
    launch_scan<int>(L.bcount, nbk, reinterpret_cast<int *>(L.scan_bsum),
                     reinterpret_cast<int *>(L.scan_total), L.bcount, st);
    k_scatter<<<blocks_for(M, 256), 256, 0, st>>>(L.bucket, M, L.bcount, L.order);
    prof_mark(1, st);
}

// The rows a fast-kernel launch takes: positions [0, nrows) of `order`
// (nrows further bounded by *nrows_dev when that is set), rows it cannot hold
// queued in `large`, counters in `sum`.
struct RowSet {
    const int *order;
    const int *nrows_dev;
    int *large;
    DevSummary *sum;
    unsigned long long *counter;
    const int *located;  // k_locate's tets of these rows, or null (the row kernel locates)
};

inline RowSet all_rows(const QueryLayout &L) {
    return RowSet{L.order, nullptr, L.large_list, L.sum, L.counter, L.located};
}

// queries per work item of the tiled schedule: at most `tile`, smaller for a
// call too small to give every resident group two tiles
inline int fit_tile(int tile, int64_t M, int per_sm, int num_sms, int gpb) {
    if (tile > 0) {
        const int64_t fit = M / (2 * (int64_t)per_sm * num_sms * gpb);
        if (fit < tile) tile = (int)fit;
    }
    return tile;
}

// persistent grid of the fast row kernel: resident blocks per SM x SMs
template <class QT, class Sink, int PM, int OCC>
void launch_fast_occ(const nif_dmesh *m, const QT *Q, int64_t M, const Centroid &cen,
                     const RowSet &R, const Sink &sink, cudaStream_t st) {
    constexpr int GPB = FAST_BLOCK / FAST_G;
    const size_t smem = GPB * sizeof(FastWS);
    auto kern = k_rows_fast<QT, Sink, PM, OCC>;
    const int per_sm = resident_blocks(kern, FAST_BLOCK, smem);
    // tile is an upper bound: a call too small to give every resident group
    // two tiles takes smaller ones (or the static stride), so that small
    // calls keep the whole GPU busy
    const int tile = fit_tile(m->tune.tile, M, per_sm, m->num_sms, GPB);
    int64_t blocks = (M + GPB - 1) / GPB;
    if (tile > 0) blocks = (M + (int64_t)GPB * tile - 1) / ((int64_t)GPB * tile);
    const int64_t cap = (int64_t)per_sm * m->num_sms;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    if (tile > 0) cudaMemsetAsync(R.counter, 0, sizeof(unsigned long long), st);
    kern<<<(unsigned)blocks, FAST_BLOCK, smem, st>>>(m->view, Q, cen, R.order, M, R.nrows_dev, sink,
                                                    LargeQueue{R.large}, R.sum, tile, R.counter);
}

// the structure-only (gradient) rows keep their own occupancy; the others
// run at the mesh's tuned one
template <class QT, class Sink, int PM>
void launch_fast_loc(const nif_dmesh *m, const QT *Q, int64_t M, const Centroid &cen,
                     const RowSet &R, const Sink &sink, cudaStream_t st) {
    if constexpr (!Sink::FULL)
        launch_fast_occ<QT, Sink, PM, Sink::MIN_BLOCKS>(m, Q, M, cen, R, sink, st);
    else if (m->tune.blocks_per_sm == OCC_LO)
        launch_fast_occ<QT, Sink, PM, OCC_LO>(m, Q, M, cen, R, sink, st);
    else
        launch_fast_occ<QT, Sink, PM, OCC_HI>(m, Q, M, cen, R, sink, st);
}

// the launch settings a row-kernel launch takes: the work-item tile (from
// the mesh's or the batch's tuning) and the GPU's SM count
struct Launch {
    int tile;
    int num_sms;
};

// one persistent launch of kernel `kern` over n rows (tiled schedule)
template <class Kern, class... Args>
void launch_rows(Kern kern, const Launch &lc, int64_t n, size_t smem, unsigned long long *counter,
                 cudaStream_t st, Args... args) {
    constexpr int GPB = FAST_BLOCK / FAST_G;
    const int per_sm = resident_blocks(kern, FAST_BLOCK, smem);
    const int tile = fit_tile(lc.tile, n, per_sm, lc.num_sms, GPB);
    int64_t blocks = (n + GPB - 1) / GPB;
    if (tile > 0) blocks = (n + (int64_t)GPB * tile - 1) / ((int64_t)GPB * tile);
    const int64_t cap = (int64_t)per_sm * lc.num_sms;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    if (tile > 0) cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    kern<<<(unsigned)blocks, FAST_BLOCK, smem, st>>>(args..., tile, counter);
}

// resident blocks per SM of a row kernel with this sink: the mesh's setting,
// except for the structure-only (gradient) rows, which keep their own
template <class Sink, int OCC>
constexpr int sink_occ() {
    if constexpr (Sink::FULL)
        return OCC;
    else
        return Sink::MIN_BLOCKS;
}

// The split row over positions [0, M) of R.order, whose rows `rows` maps to
// their meshes: k_locate over all rows, then per chunk of REC_CHUNK rows the
// cavity records and the volumes.  Rows whose cavity exceeds a record are
// left in `wide` (count in R.sum->wide_count) for the fused kernel.
template <class QT, class Rows, class Sink, int OCC, int PM = PM_PLAIN>
void launch_split(const Launch &lc, const Rows &rows, const QT *Q, int64_t M, const RowSet &R,
                  RowHead *heads, RowEntry *ents, int *wide, const Sink &sink, cudaStream_t st,
                  bool keep = false) {
    constexpr int GPB = FAST_BLOCK / FAST_G;
    constexpr int COCC = NIF_CAV_OCC > 0 ? NIF_CAV_OCC : OCC;
    constexpr int VOCC = sink_occ<Sink, (NIF_VOL_OCC > 0 ? NIF_VOL_OCC : OCC)>();
    int *located = const_cast<int *>(R.located);
    prof_span(SPAN_LOCATE, false, st);
    launch_rows(k_locate<QT, Rows, PM>, lc, M, 0, R.counter, st, rows, Q, R.order, M, located,
                R.sum);
    prof_span(SPAN_LOCATE, true, st);
    for (int64_t c0 = 0; c0 < M; c0 += REC_CHUNK) {
        const int64_t n = min((int64_t)REC_CHUNK, M - c0);
        // one chunk's records, or (keep) every row's at its own position
        RowHead *h = keep ? heads + c0 : heads;
        RowEntry *e = keep ? ents + c0 * REC_CAV : ents;
        prof_span(SPAN_CAVITY, false, st);
        launch_rows(k_rows_cavity<QT, Rows, COCC, PM>, lc, n, GPB * sizeof(CavWS), R.counter, st,
                    rows, Q, R.order + c0, n, (const int *)located, h, e, wide, LargeQueue{R.large},
                    R.sum);
        prof_span(SPAN_CAVITY, true, st);
        prof_span(SPAN_ORDER, false, st);
        {
            const int64_t groups = (n + 31) / 32;
            int64_t ob = (groups + ORD_WARPS - 1) / ORD_WARPS;
            if (ob > (int64_t)lc.num_sms * 32) ob = (int64_t)lc.num_sms * 32;
            k_rows_order<<<(unsigned)ob, 32 * ORD_WARPS, ORD_WARPS * sizeof(OrderWS), st>>>(
                n, (const RowHead *)h, e);
        }
        prof_span(SPAN_ORDER, true, st);
        prof_span(SPAN_VOLUME, false, st);
        launch_rows(k_rows_volume<QT, Rows, Sink, VOCC>, lc, n, GPB * sizeof(VolWS), R.counter, st,
                    rows, Q, R.order + c0, n, (const RowHead *)h, (const RowEntry *)e, sink,
                    LargeQueue{R.large}, R.sum);
        prof_span(SPAN_VOLUME, true, st);
    }
}

// With natinterp3d's signs, a located[] array and record buffers (and rows
// that are a plain order, not a queue), the rows are located by k_locate and
// then run through the split row kernels; otherwise the fused row kernel
// takes them whole.
template <class QT, class Sink, int PM>
void launch_fast(const nif_dmesh *m, const QT *Q, int64_t M, const Centroid &cen,
                 const RowSet &R, const Sink &sink, cudaStream_t st, RowHead *heads = nullptr,
                 RowEntry *ents = nullptr, int *wide = nullptr, bool keep = false) {
    if constexpr (PM == PM_PLAIN || PM == PM_FILTER) {
        if (R.located && heads && !R.nrows_dev) {
            const Launch lc{m->tune.tile, m->num_sms};
            const OneMesh rows{m->view, cen};
            if (m->tune.blocks_per_sm == OCC_LO)
                launch_split<QT, OneMesh, Sink, OCC_LO, PM>(lc, rows, Q, M, R, heads, ents, wide, sink,
                                                            st, keep);
            else
                launch_split<QT, OneMesh, Sink, OCC_HI, PM>(lc, rows, Q, M, R, heads, ents, wide, sink,
                                                            st, keep);
            // rows whose cavity exceeds a record: the fused row kernel (which
            // queues what exceeds its own capacities for the large kernel)
            const RowSet W{wide, &R.sum->wide_count, R.large, R.sum, R.counter, nullptr};
            prof_span(SPAN_FUSED, false, st);
            launch_fast_loc<QT, Sink, PM>(m, Q, M, cen, W, sink, st);
            prof_span(SPAN_FUSED, true, st);
            return;
        }
    }
    prof_span(SPAN_FUSED, false, st);
    launch_fast_loc<QT, Sink, PM>(m, Q, M, cen, R, sink, st);
    prof_span(SPAN_FUSED, true, st);
}

// fast rows (filtered when the mesh's predicate mode is not the default),
// then the rows they queued; large_groups workspaces in L.  With rec, every
// row's split-row record is kept there (natinterp3d's signs only).
template <class QT, class Sink>
void run_rows(const nif_dmesh *m, const QT *Q, int64_t M, const Centroid &cen, const QueryLayout &L,
              const Sink &sink, cudaStream_t st, int large_groups = LARGE_GROUPS,
              const RecordLayout *rec = nullptr) {
    if (m->view.pmode == PRED_FAST && rec)
        launch_fast<QT, Sink, PM_PLAIN>(m, Q, M, cen, all_rows(L), sink, st, rec->heads, rec->ents,
                                        L.wide, true);
    else if (m->view.pmode == PRED_FAST)
        launch_fast<QT, Sink, PM_PLAIN>(m, Q, M, cen, all_rows(L), sink, st, L.heads, L.ents, L.wide);
    else
        launch_fast<QT, Sink, PM_FILTER>(m, Q, M, cen, all_rows(L), sink, st, L.heads, L.ents, L.wide);
    prof_mark(2, st);
    k_rows_large<QT, Sink><<<large_groups, 32, 0, st>>>(m->view, Q, cen, LargeQueue{L.large_list},
                                                        sink, L.large_ws, L.exact, L.sum);
    prof_mark(3, st);
}

// fill pass of get_weights: the count pass's queued rows again, into the CSR
template <class QT, class Sink>
void refill_rows(const nif_dmesh *m, const QT *Q, int64_t M, const Centroid &cen, const QueryLayout &L,
                 const Sink &sink, cudaStream_t st) {
    // fast-kernel rows longer than ROW_STAGE: the queue's length is on the device
    // (few rows: the row kernel locates them itself)
    const RowSet R{L.refill, &L.sum->refill_count, L.large_list, L.fill_sum, L.counter, nullptr};
    if (m->view.pmode == PRED_FAST)
        launch_fast<QT, Sink, PM_PLAIN>(m, Q, M, cen, R, sink, st);
    else
        launch_fast<QT, Sink, PM_FILTER>(m, Q, M, cen, R, sink, st);
    // the rows the large kernel handled (their queue is intact: refilled rows
    // all fit the fast kernel, so nothing is appended to it)
    k_rows_large<QT, Sink><<<LARGE_GROUPS, 32, 0, st>>>(m->view, Q, cen, LargeQueue{L.large_list},
                                                        sink, L.large_ws, L.exact, L.fill_sum);
}

__global__ void k_rowptr_guarded(const int64_t *__restrict__ off, int64_t M,
                                 const int64_t *__restrict__ total, int32_t *__restrict__ rowptr) {
    const int64_t tot = *total;
    if (tot > INT32_MAX) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= M;
         i += (int64_t)gridDim.x * blockDim.x)
        rowptr[i] = (int32_t)(i < M ? off[i] : tot);
}

int read_summary(const QueryLayout &L, cudaStream_t st, nif_summary *out, int64_t *total) {
    DevSummary d;
    int64_t tot = 0;
    NIF_CUDA(cudaMemcpyAsync(&d, L.sum, sizeof(d), cudaMemcpyDeviceToHost, st));
    if (total) NIF_CUDA(cudaMemcpyAsync(&tot, L.scan_total, sizeof(tot), cudaMemcpyDeviceToHost, st));
    NIF_CUDA(cudaStreamSynchronize(st));
    NIF_CUDA(cudaGetLastError());
    if (out) {
        out->nnz = total ? tot : 0;
        out->rows_large = (int64_t)d.rows_large;
        out->rows_failed = (int64_t)d.rows_failed;
        out->rows_outside = (int64_t)d.rows_outside;
        out->walk_steps = (int64_t)d.walk_steps;
        out->first_status = d.first_status;
        out->rows_wide = d.wide_count;
        out->orient_uncertain = (int64_t)d.orient_unc;
        out->orient_flipped = (int64_t)d.orient_flip;
        out->insphere_uncertain = (int64_t)d.insphere_unc;
        out->insphere_flipped = (int64_t)d.insphere_flip;
    }
    if (total) *total = tot;
    return NIF_OK;
}

int check_query_args(const nif_dmesh *m, const void *q, int qdt, int64_t M, const double *cen,
                     const void *ws) {
    if (!m || !cen || M < 0 || M > (int64_t)INT32_MAX) return NIF_ERR_ARG;
    if (qdt != NIF_F64 && qdt != NIF_F32) return NIF_ERR_ARG;
    if (M > 0 && (!q || !ws)) return NIF_ERR_ARG;
    if (ws && reinterpret_cast<uintptr_t>(ws) % 256 != 0) return NIF_ERR_ARG;
    return NIF_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// exported API
// ---------------------------------------------------------------------------
// face-circumcentre indices 4 t + i must fit int32
constexpr int MAX_TETS = INT_MAX / 4;

NIF_EXPORT int nif_dmesh_bytes(int n_vertices, int n_tets, size_t *bytes) {
    if (!bytes || n_vertices < 5 || n_tets < 1 || n_tets > MAX_TETS) return NIF_ERR_ARG;
    Carve c{nullptr, 0, (size_t)-1, true};
    carve_mesh(c, n_vertices, n_tets);
    *bytes = align_up(c.off, 256);
    return NIF_OK;
}

NIF_EXPORT int nif_dmesh_create(const double *d_vxyz, const int32_t *d_tet_v,
                                const int32_t *d_tet_n, int n_vertices, int n_tets, void *d_buf,
                                size_t buf_bytes, void *stream, nif_dmesh **out) {
    if (!out) return NIF_ERR_ARG;
    *out = nullptr;
    if (!d_vxyz || !d_tet_v || !d_tet_n || !d_buf || n_vertices < 5 || n_tets < 1 ||
        n_tets > MAX_TETS)
        return NIF_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(d_buf) % 256 != 0) return NIF_ERR_ARG;
    size_t need = 0;
    nif_dmesh_bytes(n_vertices, n_tets, &need);
    if (buf_bytes < need) return NIF_ERR_WORKSPACE;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(d_buf), 0, buf_bytes, true};
    MeshLayout L = carve_mesh(c, n_vertices, n_tets);

    nif_dmesh *h = new (std::nothrow) nif_dmesh();
    if (!h) return NIF_ERR_NOMEM;
    h->n_vertices = n_vertices;
    h->n_tets = n_tets;
    h->bytes = need;
    if (cudaGetDevice(&h->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess) {
        delete h;
        return NIF_ERR_CUDA;
    }
    MeshView &V = h->view;
    V.vtx = L.vtx;
    V.tv = L.tv;
    V.tn = L.tn;
    V.tinfo = L.tinfo;
    V.tcc = L.tcc;
    V.fcc = L.fcc;
    V.n = n_vertices - 4;
    V.nv = n_vertices;
    V.nt = n_tets;
    V.pmode = PRED_FAST;

    V.cs = L.cs;
    V.onode = L.onode;
    V.omask = L.omask;
    V.gstart = L.gstart;
    V.gitems = L.gitems;

    int rc = NIF_OK;
    do {
        if (cudaMemsetAsync(L.flag, 0, 4 * sizeof(int), st) != cudaSuccess) { rc = NIF_ERR_CUDA; break; }
        k_prep_vertices<<<blocks_for(n_vertices, 256), 256, 0, st>>>(d_vxyz, n_vertices, L.vtx);
        k_prep_tets<<<blocks_for(n_tets, 256), 256, 0, st>>>(d_tet_v, d_tet_n, n_vertices, n_tets,
                                                             L.tv, L.tn, L.flag);
        const int nbb = blocks_for(V.n, 256, 256);
        k_bbox_partial<<<nbb, 256, 0, st>>>(L.vtx, V.n, L.bbox_part);
        double part[6 * 256];
        if (cudaMemcpyAsync(part, L.bbox_part, sizeof(double) * 6 * nbb, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = NIF_ERR_CUDA;
            break;
        }
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int b = 0; b < nbb; b++)
            for (int a = 0; a < 3; a++) {
                lo[a] = fmin(lo[a], part[6 * b + a]);
                hi[a] = fmax(hi[a], part[6 * b + 3 + a]);
            }
        double ext[3], emax = 0.0;
        for (int a = 0; a < 3; a++) {
            ext[a] = hi[a] - lo[a];
            if (!(ext[a] > 0.0) || !isfinite(ext[a])) ext[a] = 0.0;
            emax = fmax(emax, ext[a]);
        }
        if (!(emax > 0.0)) emax = 1.0;
        for (int a = 0; a < 3; a++)
            if (ext[a] < emax * 1e-3) ext[a] = emax * 1e-3;

        // seed grid over the data bounding box, about two centroids a cell,
        // within the room grid_cell_cap(n_tets) leaves; query bucketing
        // normalises by the same box
        {
            const int cap = grid_cell_cap(n_tets);
            const double side = cbrt(ext[0] * ext[1] * ext[2] / (NIF_GRID_CELLS_PER_TET * n_tets));
            int gd[3];
            for (int a = 0; a < 3; a++) {
                const double r = ext[a] / side;
                gd[a] = r < 1.0 ? 1 : (r > 4096.0 ? 4096 : (int)(r + 0.5));
            }
            while ((int64_t)gd[0] * gd[1] * gd[2] > cap) {
                const int a = (gd[0] >= gd[1] && gd[0] >= gd[2]) ? 0 : (gd[1] >= gd[2] ? 1 : 2);
                gd[a] = gd[a] > 1 ? gd[a] - 1 : 1;
            }
            V.gext = 0.0;
            for (int a = 0; a < 3; a++) {
                V.gdim[a] = gd[a];
                V.glo[a] = lo[a];
                V.ginv[a] = (double)gd[a] / ext[a];
                V.gh[a] = ext[a] / (double)gd[a];
                V.gext = fmax(V.gext, ext[a]);
            }
        }
        // centroid code space: the bounding box of all vertices (the
        // super-simplex's four included), which holds every tet centroid
        {
            d4 sv[4];
            if (cudaMemcpyAsync(sv, L.vtx + V.n, sizeof(sv), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rc = NIF_ERR_CUDA;
                break;
            }
            double olo[3] = {lo[0], lo[1], lo[2]}, ohi[3] = {hi[0], hi[1], hi[2]};
            for (int k = 0; k < 4; k++) {
                const double c[3] = {sv[k].x, sv[k].y, sv[k].z};
                for (int a = 0; a < 3; a++) {
                    olo[a] = fmin(olo[a], c[a]);
                    ohi[a] = fmax(ohi[a], c[a]);
                }
            }
            V.oext = 0.0;
            for (int a = 0; a < 3; a++) {
                double e = ohi[a] - olo[a];
                if (!(e > 0.0) || !isfinite(e)) e = 1.0;
                V.olo[a] = olo[a];
                V.osc[a] = (double)(1 << OCT_BITS) / e;
                V.oext = fmax(V.oext, e);
            }
        }
        // centroid octree: centroids sorted by code (two 32-bit radix sorts,
        // low word then high word), then node levels top down, then boxes
        // bottom up.  The scratch is the face-circumcentre array.
        {
            Carve tc{reinterpret_cast<unsigned char *>(L.fcc), 0, sizeof(d4) * fcc_slots(n_tets), true};
            const OctScratch T = carve_oct_scratch(tc, n_tets);
            if (!tc.ok) { rc = NIF_ERR_INTERNAL; break; }
            const int nb = blocks_for(n_tets, 256);
            k_cen_code<<<nb, 256, 0, st>>>(V, T.chi, T.clo, T.key_a, T.idx_a);
            uint32_t *kin = T.key_a, *kout = T.key_b;
            int32_t *vin = T.idx_a, *vout = T.idx_b;
            for (int word = 0; word < 2; word++) {
                if (word == 1) k_gather_key<<<nb, 256, 0, st>>>(T.chi, vin, n_tets, kin);
                for (int pass = 0; pass < 8; pass++) {
                    k_rs_hist<<<(unsigned)T.nblocks, RS_THREADS, 0, st>>>(kin, n_tets, 4 * pass,
                                                                           (int)T.nblocks, T.hist);
                    launch_scan<int>(T.hist, 16 * T.nblocks, T.bsum, T.tot, T.off, st);
                    k_rs_scatter<<<(unsigned)T.nblocks, RS_THREADS, 0, st>>>(
                        kin, vin, n_tets, 4 * pass, (int)T.nblocks, T.off, kout, vout);
                    std::swap(kin, kout);
                    std::swap(vin, vout);
                }
            }
            k_cen_gather<<<nb, 256, 0, st>>>(V, vin, T.chi, T.clo, L.cs, T.code);
            const int cap = oct_node_cap(n_tets);
            if (cudaMemsetAsync(T.node_of, 0, sizeof(int) * n_tets, st) != cudaSuccess ||
                cudaMemsetAsync(T.nch, 0, sizeof(int) * cap, st) != cudaSuccess ||
                cudaMemsetAsync(T.first, 0, sizeof(int) * cap, st) != cudaSuccess ||
                cudaMemsetAsync(L.omask, 0, sizeof(unsigned long long) * cap, st) != cudaSuccess) {
                rc = NIF_ERR_CUDA;
                break;
            }
            const int root[2] = {0, n_tets};
            if (cudaMemcpyAsync(T.na, &root[0], sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(T.nb, &root[1], sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess) {
                rc = NIF_ERR_CUDA;
                break;
            }
            int lvl[OCT_KMAX + 2] = {0, 1};
            int levels = 1;  // node levels built: [lvl[l], lvl[l + 1]) for l < levels
            for (int k = 0; k < OCT_KMAX; k++) {
                const int s0 = lvl[k], s1 = lvl[k + 1];
                k_oct_flag<<<nb, 256, 0, st>>>(T.code, n_tets, T.node_of, T.na, T.nb, s0, s1, k, T.flag);
                launch_scan<int>(T.flag, n_tets, T.bsum, T.tot, T.scan, st);
                int tot = 0;
                if (cudaMemcpyAsync(&tot, T.tot, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess) {
                    rc = NIF_ERR_CUDA;
                    break;
                }
                if (tot == 0 || (int64_t)s1 + tot > cap) break;  // no split / no room: leaves stay
                k_oct_link<<<nb, 256, 0, st>>>(T.code, n_tets, T.node_of, T.na, T.nb, s0, s1, k, T.flag,
                                               T.scan, T.par, T.first, T.nch, L.omask);
                k_oct_end<<<blocks_for(tot, 256), 256, 0, st>>>(s1, tot, T.na, T.par, T.nb);
                lvl[k + 2] = s1 + tot;
                levels = k + 2;
            }
            if (rc != NIF_OK) break;
            for (int l = levels - 1; l >= 0; l--)
                k_oct_box<<<blocks_for(lvl[l + 1] - lvl[l], 128), 128, 0, st>>>(
                    lvl[l], lvl[l + 1], T.na, T.nb, T.first, T.nch, L.cs, L.onode);
            h->oct_nodes = lvl[levels];
            h->oct_levels = levels;
            // seed grid: centroids counted per cell, cell starts scanned, then
            // each centroid placed at its cell's cursor
            const int ncell = V.gdim[0] * V.gdim[1] * V.gdim[2];
            if (cudaMemsetAsync(L.gstart, 0, sizeof(int) * (ncell + 1), st) != cudaSuccess) {
                rc = NIF_ERR_CUDA;
                break;
            }
            k_grid_count<<<nb, 256, 0, st>>>(V, L.gstart);
            launch_scan<int>(L.gstart, ncell, T.bsum, L.gstart + ncell, L.gstart, st);
            if (cudaMemcpyAsync(T.gcursor, L.gstart, sizeof(int) * ncell, cudaMemcpyDeviceToDevice,
                                st) != cudaSuccess) {
                rc = NIF_ERR_CUDA;
                break;
            }
            k_grid_fill<<<nb, 256, 0, st>>>(V, T.gcursor, L.gitems);
        }
        k_prep_geometry<<<blocks_for(n_tets, 128), 128, 0, st>>>(V, L.tinfo, L.tcc, L.fcc, L.flag);
        int flag[4];
        if (cudaMemcpyAsync(flag, L.flag, sizeof(flag), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = NIF_ERR_CUDA;
            break;
        }
        if (flag[0]) { rc = NIF_ERR_INTERNAL; break; }
        h->orient_unc = flag[1];
        if (flag[1] > 0) {
            // rare: near-flat tets; resolve their exact orientation flags
            k_prep_exact_orient<<<blocks_for(n_tets, 32, 4 * 148), 32, 0, st>>>(V, L.tinfo, L.flag);
            if (cudaMemcpyAsync(flag, L.flag, sizeof(flag), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rc = NIF_ERR_CUDA;
                break;
            }
        }
        h->orient_flip = flag[2];
        if (cudaGetLastError() != cudaSuccess) rc = NIF_ERR_CUDA;
    } while (0);
    if (rc != NIF_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return NIF_OK;
}

NIF_EXPORT void nif_dmesh_destroy(nif_dmesh *m) { delete m; }

NIF_EXPORT int nif_dmesh_info(const nif_dmesh *m, int64_t info[8]) {
    if (!m || !info) return NIF_ERR_ARG;
    info[0] = m->n_vertices;
    info[1] = m->n_tets;
    info[2] = m->oct_nodes;
    info[3] = m->oct_levels;
    info[4] = 0;
    info[5] = m->orient_unc;
    info[6] = m->orient_flip;
    info[7] = m->view.pmode;
    return NIF_OK;
}

NIF_EXPORT int nif_dmesh_set_predicates(nif_dmesh *m, int mode) {
    if (!m || (mode != NIF_PRED_FAST && mode != NIF_PRED_AUDIT && mode != NIF_PRED_EXACT))
        return NIF_ERR_ARG;
    m->view.pmode = mode;
    return NIF_OK;
}

namespace {
// a tuning is valid for a mesh (batch = false) or a batch (batch = true)
bool tuning_ok(const nif_tuning *t, bool batch) {
    return t && (t->blocks_per_sm == OCC_LO || t->blocks_per_sm == OCC_HI) &&
           t->bucket_shift >= -2 && t->bucket_shift <= 1 && t->tile >= (batch ? 1 : 0) &&
           t->tile <= TILE_MAX && t->reserved == 0;
}
}  // namespace

NIF_EXPORT int nif_dmesh_set_tuning(nif_dmesh *m, const nif_tuning *t) {
    if (!m || !tuning_ok(t, false)) return NIF_ERR_ARG;
    m->tune = *t;
    return NIF_OK;
}

NIF_EXPORT int nif_dmesh_get_tuning(const nif_dmesh *m, nif_tuning *t) {
    if (!m || !t) return NIF_ERR_ARG;
    *t = m->tune;
    return NIF_OK;
}

NIF_EXPORT int nif_query_workspace_bytes(const nif_dmesh *m, int64_t M, int mode, size_t *bytes) {
    if (!m || !bytes || M < 0 || (mode != NIF_MODE_WEIGHTS && mode != NIF_MODE_INTERP))
        return NIF_ERR_ARG;
    Carve c{nullptr, 0, (size_t)-1, true};
    carve_query(c, M, mode);
    *bytes = align_up(c.off, 256);
    return NIF_OK;
}

NIF_EXPORT int nif_records_bytes(int64_t M, size_t *bytes) {
    if (!bytes || M < 0) return NIF_ERR_ARG;
    Carve c{nullptr, 0, (size_t)-1, true};
    carve_records(c, M);
    *bytes = align_up(c.off, 256);
    return NIF_OK;
}

namespace {
int weights_count(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                  const double centroid[3], void *d_ws, size_t ws_bytes, int32_t *d_rowptr,
                  const RecordLayout *rec, void *stream, nif_summary *summary) {
    int rc = check_query_args(m, d_queries, query_dtype, M, centroid, d_ws);
    if (rc != NIF_OK) return rc;
    if (!d_rowptr) return NIF_ERR_ARG;
    size_t need = 0;
    nif_query_workspace_bytes(m, M, NIF_MODE_WEIGHTS, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(d_ws), 0, ws_bytes, true};
    QueryLayout L = carve_query(c, M, NIF_MODE_WEIGHTS);
    Centroid cen{{centroid[0], centroid[1], centroid[2]}};
    NIF_CUDA(cudaMemsetAsync(L.sum, 0, sizeof(DevSummary), st));
    if (M > 0) {
        StageSink sink{L.cnt, L.staged, L.scols, L.svals, L.refill, L.sum, L.rtot};
        if (query_dtype == NIF_F64) {
            run_bucketing(m, static_cast<const double *>(d_queries), M, cen, L, st);
            run_rows(m, static_cast<const double *>(d_queries), M, cen, L, sink, st, LARGE_GROUPS, rec);
        } else {
            run_bucketing(m, static_cast<const float *>(d_queries), M, cen, L, st);
            run_rows(m, static_cast<const float *>(d_queries), M, cen, L, sink, st, LARGE_GROUPS, rec);
        }
    }
    launch_scan<int64_t>(L.cnt, M, L.scan_bsum, L.scan_total, L.off64, st);
    k_rowptr_guarded<<<blocks_for(M + 1, 256), 256, 0, st>>>(L.off64, M, L.scan_total, d_rowptr);
    if (M > 0) prof_mark(4, st);
    int64_t total = 0;
    nif_summary tmp;
    rc = read_summary(L, st, summary ? summary : &tmp, &total);
    if (rc != NIF_OK) return rc;
    if (total > (int64_t)INT32_MAX) return NIF_ERR_OVERFLOW;
    return NIF_OK;
}
}  // namespace

NIF_EXPORT int nif_weights_count(const nif_dmesh *m, const void *d_queries, int query_dtype,
                                 int64_t M, const double centroid[3], void *d_ws, size_t ws_bytes,
                                 int32_t *d_rowptr, void *stream, nif_summary *summary) {
    return weights_count(m, d_queries, query_dtype, M, centroid, d_ws, ws_bytes, d_rowptr, nullptr,
                         stream, summary);
}

NIF_EXPORT int nif_weights_count_records(const nif_dmesh *m, const void *d_queries, int query_dtype,
                                         int64_t M, const double centroid[3], void *d_ws,
                                         size_t ws_bytes, int32_t *d_rowptr, void *d_records,
                                         size_t records_bytes, void *stream, nif_summary *summary) {
    if (!m || m->view.pmode != PRED_FAST || !d_records) return NIF_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(d_records) % 256 != 0) return NIF_ERR_ARG;
    size_t need = 0;
    if (nif_records_bytes(M, &need) != NIF_OK) return NIF_ERR_ARG;
    if (records_bytes < need) return NIF_ERR_WORKSPACE;
    Carve c{static_cast<unsigned char *>(d_records), 0, records_bytes, true};
    const RecordLayout R = carve_records(c, M);
    return weights_count(m, d_queries, query_dtype, M, centroid, d_ws, ws_bytes, d_rowptr, &R,
                         stream, summary);
}

namespace {
// the fill pass: staged rows copied into the CSR, then the queued rows
// (longer than ROW_STAGE, or handled by the large kernel) recomputed into
// their slices from the same queries
template <class VT>
int fill_typed(const nif_dmesh *m, const void *q, int qdt, int64_t M, const Centroid &cen,
               const QueryLayout &L, const int32_t *rowptr, VT *vals, int32_t *cols, cudaStream_t st) {
    k_compact<VT><<<blocks_for(M * 8, 256), 256, 0, st>>>(M, L.cnt, L.staged, L.scols, L.svals, rowptr,
                                                         cols, vals);
    // the refill passes count into their own record; the large kernel reads
    // its queue length from there
    NIF_CUDA(cudaMemcpyAsync(L.fill_sum, L.sum, sizeof(DevSummary), cudaMemcpyDeviceToDevice, st));
    DirectSink<VT> sink{rowptr, cols, vals, L.fill_sum};
    if (qdt == NIF_F64)
        refill_rows(m, static_cast<const double *>(q), M, cen, L, sink, st);
    else
        refill_rows(m, static_cast<const float *>(q), M, cen, L, sink, st);
    return cuda_rc(cudaGetLastError());
}
}  // namespace

NIF_EXPORT int nif_weights_fill(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                                const double centroid[3], const void *d_ws, size_t ws_bytes,
                                const int32_t *d_rowptr, void *d_vals, int vals_dtype,
                                int32_t *d_cols, double *d_row_totals, void *stream) {
    int rc = check_query_args(m, d_queries, query_dtype, M, centroid, d_ws);
    if (rc != NIF_OK) return rc;
    if (!d_rowptr) return NIF_ERR_ARG;
    if (vals_dtype != NIF_F64 && vals_dtype != NIF_F32) return NIF_ERR_ARG;
    size_t need = 0;
    nif_query_workspace_bytes(m, M, NIF_MODE_WEIGHTS, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    if (M == 0) return NIF_OK;
    if (!d_vals || !d_cols) return NIF_ERR_ARG;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(const_cast<void *>(d_ws)), 0, ws_bytes, true};
    QueryLayout L = carve_query(c, M, NIF_MODE_WEIGHTS);
    Centroid cen{{centroid[0], centroid[1], centroid[2]}};
    if (d_row_totals)
        NIF_CUDA(cudaMemcpyAsync(d_row_totals, L.rtot, sizeof(double) * M, cudaMemcpyDeviceToDevice, st));
    if (vals_dtype == NIF_F64)
        return fill_typed<double>(m, d_queries, query_dtype, M, cen, L, d_rowptr,
                                  static_cast<double *>(d_vals), d_cols, st);
    return fill_typed<float>(m, d_queries, query_dtype, M, cen, L, d_rowptr,
                             static_cast<float *>(d_vals), d_cols, st);
}

namespace {
template <class QT, class VT, class CT>
int interp_typed(const nif_dmesh *m, const void *q, int64_t M, const Centroid &cen, const void *v,
                 int D, void *out, const QueryLayout &L, cudaStream_t st) {
    InterpSink<QT, VT, CT> sink{static_cast<const VT *>(v), static_cast<CT *>(out), D};
    run_bucketing(m, static_cast<const QT *>(q), M, cen, L, st);
    run_rows(m, static_cast<const QT *>(q), M, cen, L, sink, st);
    return NIF_OK;
}
}  // namespace

NIF_EXPORT int nif_interpolate(const nif_dmesh *m, const void *d_queries, int query_dtype,
                               int64_t M, const double centroid[3], const void *d_values,
                               int values_dtype, int D, void *d_out, int out_dtype, void *d_ws,
                               size_t ws_bytes, void *stream, nif_summary *summary) {
    int rc = check_query_args(m, d_queries, query_dtype, M, centroid, d_ws);
    if (rc != NIF_OK) return rc;
    if (values_dtype != NIF_F64 && values_dtype != NIF_F32) return NIF_ERR_ARG;
    if (D < 1) return NIF_ERR_ARG;
    const int expect = (query_dtype == NIF_F32 && values_dtype == NIF_F32) ? NIF_F32 : NIF_F64;
    if (out_dtype != expect) return NIF_ERR_ARG;
    if (M > 0 && (!d_values || !d_out)) return NIF_ERR_ARG;
    size_t need = 0;
    nif_query_workspace_bytes(m, M, NIF_MODE_INTERP, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(d_ws), 0, ws_bytes, true};
    QueryLayout L = carve_query(c, M, NIF_MODE_INTERP);
    Centroid cen{{centroid[0], centroid[1], centroid[2]}};
    NIF_CUDA(cudaMemsetAsync(L.sum, 0, sizeof(DevSummary), st));
    if (M > 0) {
        if (query_dtype == NIF_F64 && values_dtype == NIF_F64)
            rc = interp_typed<double, double, double>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        else if (query_dtype == NIF_F64)
            rc = interp_typed<double, float, double>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        else if (values_dtype == NIF_F32)
            rc = interp_typed<float, float, float>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        else
            rc = interp_typed<float, double, double>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        if (rc != NIF_OK) return rc;
    }
    if (M > 0) prof_mark(4, st);
    if (summary) return read_summary(L, st, summary, nullptr);
    return cuda_rc(cudaGetLastError());
}

NIF_EXPORT int nif_profile_enable(int on) {
    g_prof.on = on != 0;
    g_prof.calls = 0;
    g_prof.marks = 0;
    return NIF_OK;
}

NIF_EXPORT int nif_profile_read(double ms[4]) {
    if (!ms) return NIF_ERR_ARG;
    for (int i = 0; i < 4; i++) ms[i] = 0.0;
    // complete calls in the ring: all but the current one if it is unfinished
    const int last = g_prof.marks == PROF_EVENTS ? g_prof.calls : g_prof.calls - 1;
    const int first = last - PROF_RING + 1 > 1 ? last - PROF_RING + 1 : 1;
    if (!g_prof.created || last < 1) return NIF_ERR_ARG;
    NIF_CUDA(cudaEventSynchronize(g_prof.ev[(last - 1) % PROF_RING][PROF_EVENTS - 1]));
    const int ncalls = last - first + 1;
    for (int k = 0; k < PROF_KINDS; k++) g_prof.kms[k] = g_prof.klaunch[k] = 0.0;
    for (int c = first; c <= last; c++) {
        const int r = (c - 1) % PROF_RING;
        for (int i = 0; i < 4; i++) {
            float t = 0.f;
            NIF_CUDA(cudaEventElapsedTime(&t, g_prof.ev[r][i], g_prof.ev[r][i + 1]));
            ms[i] += t / ncalls;
        }
        for (int j = 0; j < g_prof.nspan[r]; j++) {
            float t = 0.f;
            NIF_CUDA(cudaEventElapsedTime(&t, g_prof.sev[r][j][0], g_prof.sev[r][j][1]));
            g_prof.kms[g_prof.skind[r][j]] += t / ncalls;
            g_prof.klaunch[g_prof.skind[r][j]] += 1.0 / ncalls;
        }
    }
    g_prof.calls = 0;
    g_prof.marks = 0;
    return NIF_OK;
}

NIF_EXPORT int nif_profile_kernels(double ms[5], double launches[5]) {
    if (!ms || !launches) return NIF_ERR_ARG;
    for (int k = 0; k < PROF_KINDS; k++) {
        ms[k] = g_prof.kms[k];
        launches[k] = g_prof.klaunch[k];
    }
    return NIF_OK;
}

NIF_EXPORT int nif_measure_fp64_peak(double *tflops_fused, double *tflops_separate) {
    if (!tflops_fused || !tflops_separate) return NIF_ERR_ARG;
    int dev = 0, sms = 0;
    NIF_CUDA(cudaGetDevice(&dev));
    NIF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    double *out = nullptr;
    NIF_CUDA(cudaMalloc(&out, sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    double best[2] = {0.0, 0.0};
    for (int rep = 0; rep < 4; rep++) {
        for (int v = 0; v < 2; v++) {
            cudaEventRecord(e0);
            if (v == 0)
                k_fp64_peak<true><<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
            else
                k_fp64_peak<false><<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double tf = flops / (ms * 1e-3) / 1e12;
            if (rep > 0 && tf > best[v]) best[v] = tf;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops_fused = best[0];
    *tflops_separate = best[1];
    return cuda_rc(cudaGetLastError());
}

// ===========================================================================
// Allocation-free interpolation (nif_interpolate_noalloc)
//
// For callers that cannot allocate device memory or pass a workspace in: the
// scratch of one call lives in the static array below, which the CUDA runtime
// places on every device that loads this library for the life of the process.
// Host code must never pass the array's name to a kernel -- on the host that
// name is only a stand-in, not a device address -- so the device address is
// looked up once per device with cudaGetSymbolAddress and cached.
// ===========================================================================
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[NIF_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_LARGE_GROUPS = 8;  // large-row workspaces inside the scratch
constexpr int NOALLOC_MAX_DEVICES = 256;

std::mutex g_noalloc_mu;
void *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

// device address of this device's scratch array, looked up on first use
int noalloc_scratch(int dev, void **out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return NIF_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return NIF_ERR_CUDA;
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return NIF_OK;
}

// Bytes carve_noalloc takes for M queries (the same takes, each 256-byte
// aligned), so that the fixed array is checked against the largest call at
// compile time.
constexpr size_t noalloc_bytes(int64_t M) {
    const int bits = bucket_bits(M);
    const int64_t nbk = (int64_t)1 << (3 * bits);
    const int64_t mscan = M > nbk ? M : nbk;
    const int64_t m1 = M > 0 ? M : 1;
    const size_t takes[] = {sizeof(DevSummary),
                            sizeof(unsigned long long),
                            sizeof(int) * (size_t)m1,
                            sizeof(int) * (size_t)(nbk + 1),
                            sizeof(int) * (size_t)m1,
                            sizeof(int) * (size_t)m1,
                            sizeof(int64_t) * (size_t)((mscan + SCAN_TILE - 1) / SCAN_TILE + 1),
                            sizeof(int64_t),
                            sizeof(LargeWS) * (size_t)NOALLOC_LARGE_GROUPS,
                            sizeof(double) * (size_t)NOALLOC_LARGE_GROUPS * NIF_EXACT_SCRATCH};
    size_t off = 0;
    for (size_t t : takes) off = (off + 255) / 256 * 256 + t;
    return off;
}
static_assert(noalloc_bytes(NIF_NOALLOC_MAX_QUERIES) <= NIF_NOALLOC_SCRATCH_BYTES,
              "the fixed scratch array must hold the largest call nif_interpolate_noalloc accepts");

// interpolate-mode layout with NOALLOC_LARGE_GROUPS large-row workspaces
QueryLayout carve_noalloc(Carve &c, int64_t M) {
    QueryLayout L{};
    const int bits = bucket_bits(M);
    const int64_t nbk = (int64_t)1 << (3 * bits);
    const int64_t mscan = M > nbk ? M : nbk;
    L.bits_cap = bits;  // a positive bucket_shift is capped at the default here
    L.sum = c.take<DevSummary>(1);
    L.counter = c.take<unsigned long long>(1);
    L.bucket = c.take<int>(M > 0 ? M : 1);
    L.bcount = c.take<int>(nbk + 1);
    L.order = c.take<int>(M > 0 ? M : 1);
    L.large_list = c.take<int>(M > 0 ? M : 1);
    L.scan_bsum = c.take<int64_t>((mscan + SCAN_TILE - 1) / SCAN_TILE + 1);
    L.scan_total = c.take<int64_t>(1);
    L.large_ws = c.take<LargeWS>(NOALLOC_LARGE_GROUPS);
    L.exact = c.take<double>((size_t)NOALLOC_LARGE_GROUPS * NIF_EXACT_SCRATCH);
    return L;
}

template <class QT, class VT, class CT>
void noalloc_typed(const nif_dmesh *m, const void *q, int64_t M, const Centroid &cen,
                   const void *v, int D, void *out, const QueryLayout &L, cudaStream_t st) {
    InterpSink<QT, VT, CT> sink{static_cast<const VT *>(v), static_cast<CT *>(out), D};
    run_bucketing(m, static_cast<const QT *>(q), M, cen, L, st);
    run_rows(m, static_cast<const QT *>(q), M, cen, L, sink, st, NOALLOC_LARGE_GROUPS);
}

}  // namespace

NIF_EXPORT int nif_interpolate_noalloc(const nif_dmesh *m, const void *d_queries, int query_dtype,
                                       int64_t M, const double centroid[3], const void *d_values,
                                       int values_dtype, int D, void *d_out, int out_dtype,
                                       void *stream, nif_summary *summary) {
    if (!m || !centroid || M < 0) return NIF_ERR_ARG;
    if (M > (int64_t)NIF_NOALLOC_MAX_QUERIES) return NIF_ERR_TOO_LARGE;
    if (query_dtype != NIF_F64 && query_dtype != NIF_F32) return NIF_ERR_ARG;
    if (values_dtype != NIF_F64 && values_dtype != NIF_F32) return NIF_ERR_ARG;
    if (D < 1) return NIF_ERR_ARG;
    const int expect = (query_dtype == NIF_F32 && values_dtype == NIF_F32) ? NIF_F32 : NIF_F64;
    if (out_dtype != expect) return NIF_ERR_ARG;
    if (M > 0 && (!d_queries || !d_values || !d_out)) return NIF_ERR_ARG;
    int dev = -1;
    NIF_CUDA(cudaGetDevice(&dev));
    if (dev != m->device) return NIF_ERR_ARG;
    void *scratch = nullptr;
    int rc = noalloc_scratch(dev, &scratch);
    if (rc != NIF_OK) return rc;
    Carve c{reinterpret_cast<unsigned char *>(scratch), 0, NIF_NOALLOC_SCRATCH_BYTES, true};
    QueryLayout L = carve_noalloc(c, M);
    if (!c.ok) return NIF_ERR_INTERNAL;  // the fixed array must hold the largest accepted call
    cudaStream_t st = S(stream);
    Centroid cen{{centroid[0], centroid[1], centroid[2]}};
    // counters and queue length start at zero (bucket counts are cleared by run_bucketing)
    NIF_CUDA(cudaMemsetAsync(L.sum, 0, sizeof(DevSummary), st));
    if (M > 0) {
        if (query_dtype == NIF_F64 && values_dtype == NIF_F64)
            noalloc_typed<double, double, double>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        else if (query_dtype == NIF_F64)
            noalloc_typed<double, float, double>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        else if (values_dtype == NIF_F32)
            noalloc_typed<float, float, float>(m, d_queries, M, cen, d_values, D, d_out, L, st);
        else
            noalloc_typed<float, double, double>(m, d_queries, M, cen, d_values, D, d_out, L, st);
    }
    if (summary) return read_summary(L, st, summary, nullptr);
    return cuda_rc(cudaGetLastError());
}

// ===========================================================================
// sparse products and the query gradient
// ===========================================================================
namespace {

template <class WT, class XT>
int spmm_typed(int64_t M, int D, const int32_t *rowptr, const int32_t *cols, const void *vals,
               const void *x, void *y, cudaStream_t st) {
    using CT = typename std::conditional<(sizeof(WT) == 8 || sizeof(XT) == 8), double, float>::type;
    if (M * D == 0) return NIF_OK;
    k_spmm<WT, XT, CT><<<blocks_for(M * D, 256), 256, 0, st>>>(
        M, D, rowptr, cols, static_cast<const WT *>(vals), static_cast<const XT *>(x),
        static_cast<CT *>(y));
    return cuda_rc(cudaGetLastError());
}

template <class WT, class XT>
int spmm_t_typed(int64_t N, int D, const int32_t *colptr, const int32_t *perm, const int32_t *rowof,
                 const void *vals, const void *x, void *y, const int32_t *inv, cudaStream_t st) {
    using CT = typename std::conditional<(sizeof(WT) == 8 || sizeof(XT) == 8), double, float>::type;
    if (N * D == 0) return NIF_OK;
    k_spmm_t<WT, XT, CT><<<blocks_for(N * D, 256), 256, 0, st>>>(
        N, D, colptr, perm, rowof, static_cast<const WT *>(vals), static_cast<const XT *>(x),
        static_cast<CT *>(y), inv);
    return cuda_rc(cudaGetLastError());
}

int expect_promoted(int a, int b) { return (a == NIF_F32 && b == NIF_F32) ? NIF_F32 : NIF_F64; }

struct CscLayout {
    int32_t *rowof, *idx_a, *idx_b, *colptr, *inv;
    uint32_t *key_a, *key_b;
    int *hist, *off, *bsum, *total;
};

CscLayout carve_csc(Carve &c, int64_t nnz, int64_t N) {
    CscLayout L{};
    const int64_t nb = (nnz + RS_TILE - 1) / RS_TILE;
    const int64_t nh = 16 * (nb > 0 ? nb : 1);
    L.rowof = c.take<int32_t>(nnz > 0 ? nnz : 1);
    L.idx_a = c.take<int32_t>(nnz > 0 ? nnz : 1);
    L.idx_b = c.take<int32_t>(nnz > 0 ? nnz : 1);
    L.key_a = c.take<uint32_t>(nnz > 0 ? nnz : 1);
    L.key_b = c.take<uint32_t>(nnz > 0 ? nnz : 1);
    L.colptr = c.take<int32_t>(N + 1);
    L.inv = c.take<int32_t>(N > 0 ? N : 1);
    L.hist = c.take<int>(nh);
    L.off = c.take<int>(nh);
    L.bsum = c.take<int>((nh + SCAN_TILE - 1) / SCAN_TILE + 1);
    L.total = c.take<int>(2);
    return L;
}

}  // namespace

NIF_EXPORT int nif_spmm(int64_t M, int64_t N, const int32_t *d_rowptr, const int32_t *d_cols,
                        const void *d_vals, int vals_dtype, const void *d_x, int x_dtype, int D,
                        void *d_y, int y_dtype, void *stream) {
    if (M < 0 || N < 0 || D < 1) return NIF_ERR_ARG;
    if ((vals_dtype != NIF_F64 && vals_dtype != NIF_F32) || (x_dtype != NIF_F64 && x_dtype != NIF_F32))
        return NIF_ERR_ARG;
    if (y_dtype != expect_promoted(vals_dtype, x_dtype)) return NIF_ERR_ARG;
    if (M > 0 && (!d_rowptr || !d_y)) return NIF_ERR_ARG;
    cudaStream_t st = S(stream);
    if (vals_dtype == NIF_F64 && x_dtype == NIF_F64)
        return spmm_typed<double, double>(M, D, d_rowptr, d_cols, d_vals, d_x, d_y, st);
    if (vals_dtype == NIF_F64)
        return spmm_typed<double, float>(M, D, d_rowptr, d_cols, d_vals, d_x, d_y, st);
    if (x_dtype == NIF_F64)
        return spmm_typed<float, double>(M, D, d_rowptr, d_cols, d_vals, d_x, d_y, st);
    return spmm_typed<float, float>(M, D, d_rowptr, d_cols, d_vals, d_x, d_y, st);
}

NIF_EXPORT int nif_spmm_t_workspace_bytes(int64_t M, int64_t N, int64_t nnz, size_t *bytes) {
    if (!bytes || M < 0 || N < 0 || nnz < 0 || nnz > (int64_t)INT32_MAX || N >= ((int64_t)1 << 32))
        return NIF_ERR_ARG;
    Carve c{nullptr, 0, (size_t)-1, true};
    carve_csc(c, nnz, N);
    *bytes = align_up(c.off, 256);
    return NIF_OK;
}

namespace {
int spmm_t_impl(int64_t M, int64_t N, int64_t nnz, const int32_t *d_rowptr, const int32_t *d_cols,
                const void *d_vals, int vals_dtype, const void *d_x, int x_dtype, int D, void *d_y,
                int y_dtype, const int32_t *d_key_rank, void *d_ws, size_t ws_bytes, void *stream) {
    size_t need = 0;
    int rc = nif_spmm_t_workspace_bytes(M, N, nnz, &need);
    if (rc != NIF_OK) return rc;
    if (D < 1 || (vals_dtype != NIF_F64 && vals_dtype != NIF_F32) ||
        (x_dtype != NIF_F64 && x_dtype != NIF_F32) || y_dtype != expect_promoted(vals_dtype, x_dtype))
        return NIF_ERR_ARG;
    if (!d_ws || reinterpret_cast<uintptr_t>(d_ws) % 256 != 0) return NIF_ERR_ARG;
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    if (N > 0 && !d_y) return NIF_ERR_ARG;
    if (nnz > 0 && (!d_rowptr || !d_cols || !d_vals || !d_x)) return NIF_ERR_ARG;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(d_ws), 0, ws_bytes, true};
    CscLayout L = carve_csc(c, nnz, N);
    if (M > 0)
        k_row_of<<<blocks_for(M, 256), 256, 0, st>>>(M, d_rowptr, L.rowof, L.key_a, d_cols, L.idx_a,
                                                      d_key_rank, N);
    const int32_t *inv = nullptr;
    if (d_key_rank && N > 0) {
        NIF_CUDA(cudaMemsetAsync(L.inv, 0xff, sizeof(int32_t) * N, st));
        k_rank_inverse<<<blocks_for(N, 256), 256, 0, st>>>(N, d_key_rank, L.inv);
        inv = L.inv;
    }
    // stable sort by column over as many 4-bit digits as the column count needs
    int bits = 0;
    while (bits < 32 && ((int64_t)1 << bits) < N) bits++;
    const int passes = (bits + 3) / 4;
    uint32_t *kin = L.key_a, *kout = L.key_b;
    int32_t *vin = L.idx_a, *vout = L.idx_b;
    const int64_t nblocks = (nnz + RS_TILE - 1) / RS_TILE;
    for (int pass = 0; pass < passes && nnz > 0; pass++) {
        const int shift = 4 * pass;
        k_rs_hist<<<(unsigned)nblocks, RS_THREADS, 0, st>>>(kin, nnz, shift, (int)nblocks, L.hist);
        launch_scan<int>(L.hist, 16 * nblocks, L.bsum, L.total, L.off, st);
        k_rs_scatter<<<(unsigned)nblocks, RS_THREADS, 0, st>>>(kin, vin, nnz, shift, (int)nblocks,
                                                                L.off, kout, vout);
        uint32_t *tk = kin; kin = kout; kout = tk;
        int32_t *tv = vin; vin = vout; vout = tv;
    }
    k_colptr<<<blocks_for(N + 1, 256), 256, 0, st>>>(kin, nnz, N, L.colptr);
    if (vals_dtype == NIF_F64 && x_dtype == NIF_F64)
        return spmm_t_typed<double, double>(N, D, L.colptr, vin, L.rowof, d_vals, d_x, d_y, inv, st);
    if (vals_dtype == NIF_F64)
        return spmm_t_typed<double, float>(N, D, L.colptr, vin, L.rowof, d_vals, d_x, d_y, inv, st);
    if (x_dtype == NIF_F64)
        return spmm_t_typed<float, double>(N, D, L.colptr, vin, L.rowof, d_vals, d_x, d_y, inv, st);
    return spmm_t_typed<float, float>(N, D, L.colptr, vin, L.rowof, d_vals, d_x, d_y, inv, st);
}
}  // namespace

NIF_EXPORT int nif_spmm_t(int64_t M, int64_t N, int64_t nnz, const int32_t *d_rowptr,
                          const int32_t *d_cols, const void *d_vals, int vals_dtype, const void *d_x,
                          int x_dtype, int D, void *d_y, int y_dtype, void *d_ws, size_t ws_bytes,
                          void *stream) {
    return spmm_t_impl(M, N, nnz, d_rowptr, d_cols, d_vals, vals_dtype, d_x, x_dtype, D, d_y, y_dtype,
                       nullptr, d_ws, ws_bytes, stream);
}

NIF_EXPORT int nif_spmm_t_ordered(int64_t M, int64_t N, int64_t nnz, const int32_t *d_rowptr,
                                  const int32_t *d_cols, const void *d_vals, int vals_dtype,
                                  const void *d_x, int x_dtype, int D, void *d_y, int y_dtype,
                                  const int32_t *d_key_rank, void *d_ws, size_t ws_bytes,
                                  void *stream) {
    if (N > 0 && !d_key_rank) return NIF_ERR_ARG;
    return spmm_t_impl(M, N, nnz, d_rowptr, d_cols, d_vals, vals_dtype, d_x, x_dtype, D, d_y, y_dtype,
                       d_key_rank, d_ws, ws_bytes, stream);
}

namespace {
template <class QT, class VT>
void grad_typed(const nif_dmesh *m, const void *q, int64_t M, const Centroid &cen, const void *v,
                int D, const void *gout, const int32_t *rowptr, const double *w, const double *tot,
                void *gq, const QueryLayout &L, cudaStream_t st) {
    using GT = typename std::conditional<(sizeof(QT) == 8 || sizeof(VT) == 8), double, float>::type;
    GradSink<QT, VT, GT> sink{static_cast<const VT *>(v), static_cast<const GT *>(gout), rowptr, w,
                              tot, static_cast<QT *>(gq), D};
    run_bucketing(m, static_cast<const QT *>(q), M, cen, L, st);
    run_rows(m, static_cast<const QT *>(q), M, cen, L, sink, st);
}
}  // namespace

namespace {
// the gradient rows from the forward's records: the volume kernel per chunk
// of records, the forward's wide rows through the fused kernel, and the
// forward's large-row queue through the large kernel (the same rows and
// capacities as the forward, so the passes queue nothing new)
template <class QT, class VT>
void grad_records_typed(const nif_dmesh *m, const void *q, int64_t M, const Centroid &cen,
                        const void *v, int D, const void *gout, const int32_t *rowptr,
                        const double *w, const double *tot, void *gq, const QueryLayout &L,
                        const RecordLayout &R, cudaStream_t st) {
    using GT = typename std::conditional<(sizeof(QT) == 8 || sizeof(VT) == 8), double, float>::type;
    using Sink = GradSink<QT, VT, GT>;
    Sink sink{static_cast<const VT *>(v), static_cast<const GT *>(gout), rowptr, w, tot,
              static_cast<QT *>(gq), D};
    const QT *Q = static_cast<const QT *>(q);
    constexpr int GPB = FAST_BLOCK / FAST_G;
    const Launch lc{m->tune.tile, m->num_sms};
    const OneMesh rows{m->view, cen};
    cudaMemsetAsync(R.sum, 0, sizeof(DevSummary), st);
    for (int64_t c0 = 0; c0 < M; c0 += REC_CHUNK) {
        const int64_t n = min((int64_t)REC_CHUNK, M - c0);
        launch_rows(k_rows_volume<QT, OneMesh, Sink, Sink::MIN_BLOCKS>, lc, n, GPB * sizeof(VolWS),
                    R.counter, st, rows, Q, L.order + c0, n, (const RowHead *)(R.heads + c0),
                    (const RowEntry *)(R.ents + c0 * REC_CAV), sink, LargeQueue{R.requeue}, R.sum);
    }
    const RowSet W{L.wide, &L.sum->wide_count, R.requeue, R.sum, R.counter, nullptr};
    launch_fast_loc<QT, Sink, PM_PLAIN>(m, Q, M, cen, W, sink, st);
    cudaMemcpyAsync(R.large_sum, L.sum, sizeof(DevSummary), cudaMemcpyDeviceToDevice, st);
    k_rows_large<QT, Sink><<<LARGE_GROUPS, 32, 0, st>>>(m->view, Q, cen, LargeQueue{L.large_list},
                                                        sink, L.large_ws, L.exact, R.large_sum);
}
}  // namespace

NIF_EXPORT int nif_query_grad_records(const nif_dmesh *m, const void *d_queries, int query_dtype,
                                      int64_t M, const double centroid[3], const int32_t *d_rowptr,
                                      const double *d_weights, const double *d_row_totals,
                                      const void *d_values, int values_dtype, int D,
                                      const void *d_gout, int gout_dtype, void *d_gq,
                                      const void *d_ws, size_t ws_bytes, void *d_records,
                                      size_t records_bytes, void *stream, nif_summary *summary) {
    int rc = check_query_args(m, d_queries, query_dtype, M, centroid, d_ws);
    if (rc != NIF_OK) return rc;
    if (m->view.pmode != PRED_FAST || !d_records) return NIF_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(d_records) % 256 != 0) return NIF_ERR_ARG;
    if ((values_dtype != NIF_F64 && values_dtype != NIF_F32) || D < 1) return NIF_ERR_ARG;
    if (gout_dtype != expect_promoted(query_dtype, values_dtype)) return NIF_ERR_ARG;
    if (M > 0 && (!d_values || !d_gout || !d_gq || !d_rowptr || !d_row_totals)) return NIF_ERR_ARG;
    size_t need = 0, rneed = 0;
    nif_query_workspace_bytes(m, M, NIF_MODE_WEIGHTS, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    nif_records_bytes(M, &rneed);
    if (records_bytes < rneed) return NIF_ERR_WORKSPACE;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(const_cast<void *>(d_ws)), 0, ws_bytes, true};
    const QueryLayout L = carve_query(c, M, NIF_MODE_WEIGHTS);
    Carve cr{static_cast<unsigned char *>(d_records), 0, records_bytes, true};
    const RecordLayout R = carve_records(cr, M);
    Centroid cen{{centroid[0], centroid[1], centroid[2]}};
    if (M > 0) {
        if (query_dtype == NIF_F64 && values_dtype == NIF_F64)
            grad_records_typed<double, double>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr,
                                               d_weights, d_row_totals, d_gq, L, R, st);
        else if (query_dtype == NIF_F64)
            grad_records_typed<double, float>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr,
                                              d_weights, d_row_totals, d_gq, L, R, st);
        else if (values_dtype == NIF_F32)
            grad_records_typed<float, float>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr,
                                             d_weights, d_row_totals, d_gq, L, R, st);
        else
            grad_records_typed<float, double>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr,
                                              d_weights, d_row_totals, d_gq, L, R, st);
    }
    if (summary) {
        // the gradient pass's own counters (its rows are the forward's)
        QueryLayout G = L;
        G.sum = R.sum;
        return read_summary(G, st, summary, nullptr);
    }
    return cuda_rc(cudaGetLastError());
}

NIF_EXPORT int nif_query_grad(const nif_dmesh *m, const void *d_queries, int query_dtype, int64_t M,
                              const double centroid[3], const int32_t *d_rowptr,
                              const double *d_weights, const double *d_row_totals,
                              const void *d_values, int values_dtype, int D, const void *d_gout,
                              int gout_dtype, void *d_gq, void *d_ws, size_t ws_bytes, void *stream,
                              nif_summary *summary) {
    int rc = check_query_args(m, d_queries, query_dtype, M, centroid, d_ws);
    if (rc != NIF_OK) return rc;
    if ((values_dtype != NIF_F64 && values_dtype != NIF_F32) || D < 1) return NIF_ERR_ARG;
    if (gout_dtype != expect_promoted(query_dtype, values_dtype)) return NIF_ERR_ARG;
    if (M > 0 && (!d_values || !d_gout || !d_gq || !d_rowptr || !d_row_totals)) return NIF_ERR_ARG;
    size_t need = 0;
    nif_query_workspace_bytes(m, M, NIF_MODE_INTERP, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(d_ws), 0, ws_bytes, true};
    QueryLayout L = carve_query(c, M, NIF_MODE_INTERP);
    Centroid cen{{centroid[0], centroid[1], centroid[2]}};
    NIF_CUDA(cudaMemsetAsync(L.sum, 0, sizeof(DevSummary), st));
    if (M > 0) {
        if (query_dtype == NIF_F64 && values_dtype == NIF_F64)
            grad_typed<double, double>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr, d_weights,
                                       d_row_totals, d_gq, L, st);
        else if (query_dtype == NIF_F64)
            grad_typed<double, float>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr, d_weights,
                                       d_row_totals, d_gq, L, st);
        else if (values_dtype == NIF_F32)
            grad_typed<float, float>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr, d_weights,
                                       d_row_totals, d_gq, L, st);
        else
            grad_typed<float, double>(m, d_queries, M, cen, d_values, D, d_gout, d_rowptr, d_weights,
                                       d_row_totals, d_gq, L, st);
    }
    if (summary) return read_summary(L, st, summary, nullptr);
    return cuda_rc(cudaGetLastError());
}

// ===========================================================================
// Batched interpolation: many independent (keys, queries) problems in one
// pipeline with no host synchronisation, so that it can be captured in a
// CUDA graph.  Every problem keeps its own resident mesh (nif_dmesh_create);
// the batch holds the device array of their views.  Queries, centroids,
// values and outputs are concatenated by problem, with int64 offsets.
// ===========================================================================
namespace nif {



__device__ __forceinline__ int bucket_bits_dev(int64_t M) {
    int b = 1;
    while (b < 10 && ((int64_t)1 << (3 * (b + 1))) <= M / 2) b++;
    return b;
}

// per-problem bucket bases (one thread; P is small)
__global__ void k_batch_setup(const int64_t *__restrict__ qoff, int P, int *__restrict__ bits,
                              int64_t *__restrict__ bbase) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int64_t acc = 0;
    for (int p = 0; p < P; p++) {
        const int b = bucket_bits_dev(qoff[p + 1] - qoff[p]);
        bits[p] = b;
        bbase[p] = acc;
        acc += (int64_t)1 << (3 * b);
    }
    bbase[P] = acc;
}

template <class QT>
__global__ void k_batch_bucket(const QT *__restrict__ Q, int64_t M, const int64_t *__restrict__ qoff,
                               int P, const double *__restrict__ cens, const MeshView *__restrict__ views,
                               const int *__restrict__ bits, const int64_t *__restrict__ bbase,
                               int *__restrict__ bucket, int *__restrict__ bcount) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int p = find_problem(qoff, P, i);
        const dv3 q = load_query(Q, i, cens + 3 * p);
        const MeshView &mv = views[p];
        const int b = bits[p];
        const double scale = (double)(1 << b);
        const double c[3] = {q.x, q.y, q.z};
        unsigned code = 0;
        for (int a = 0; a < 3; a++) {
            const double f = (c[a] - mv.glo[a]) * mv.ginv[a] / (double)mv.gdim[a] * scale;
            const int k = (f >= 0.0) ? (f < scale ? (int)f : (1 << b) - 1) : 0;
            code |= spread3((unsigned)k) << a;
        }
        const int64_t bk = bbase[p] + code;
        bucket[i] = (int)bk;
        atomicAdd(&bcount[bk], 1);
    }
}

// interpolation sink of a batch: values and outputs of query i belong to its problem
template <class WT, class VT, class CT>
struct BatchInterpSink {
    static constexpr bool FULL = true;
    const VT *__restrict__ values;   // concatenated [sum N_p][D]
    const int64_t *__restrict__ koff; // [P+1] key offsets
    const int64_t *__restrict__ qoff; // [P+1] query offsets
    int P;
    CT *__restrict__ out;             // concatenated [sum M_p][D]
    int D;

    template <int G, class W>
    __device__ __forceinline__ void emit(int64_t i, int nnb, W &ws, const Grp<G> &g, bool large,
                                         const MeshView &M, dv3 q, const RowInfo &r) {
        const int p = find_problem(qoff, P, i);
        InterpSink<WT, VT, CT> s{values + koff[p] * D, out, D};
        s.template emit<G>(i, nnb, ws, g, large, M, q, r);
    }
};

// persistent row kernel of a batch: warps pull tiles of bucket-ordered
// queries from a device counter; the mesh view of the current problem is
// kept in shared memory
template <class QT, class Sink, int PM, int OCC>
__global__ void __launch_bounds__(FAST_BLOCK, OCC)
    k_rows_batch(const MeshView *__restrict__ views, const int64_t *__restrict__ qoff, int P,
                 const QT *__restrict__ Q, const double *__restrict__ cens,
                 const int *__restrict__ order, int64_t nrows, const int *nrows_dev, Sink sink,
                 LargeQueue lq, DevSummary *sum, unsigned long long *counter, int tile) {
    extern __shared__ __align__(16) unsigned char smem[];
    // a row count known only on the device (a queue's length) bounds nrows
    if (nrows_dev) nrows = min(nrows, (int64_t)*nrows_dev);
    constexpr int G = FAST_G;
    constexpr int GPB = FAST_BLOCK / G;
    __shared__ MeshView sview[GPB];
    Grp<G> g;
    const int gib = threadIdx.x / G;
    FastWS &ws = reinterpret_cast<FastWS *>(smem)[gib];
    MeshView &M = sview[gib];
    int cur = -1;
    unsigned long long steps = 0;
    for (;;) {
        unsigned long long t = 0;
        if (g.lane == 0) t = atomicAdd(counter, 1ull);
        t = __shfl_sync(g.mask, t, 0, G);
        int64_t s0, s1;
        tile_range(t, tile, nrows, (int64_t)gridDim.x * GPB * tile, s0, s1);
        if (s0 >= nrows) break;
        for (int64_t s = s0; s < s1; s++) {
            const int64_t i = order[s];
            const int p = find_problem(qoff, P, i);
            if (p != cur) {
                g.sync();
                if (g.lane == 0) M = views[p];
                g.sync();
                cur = p;
            }
            const dv3 q = load_query(Q, i, cens + 3 * p);
            const RowInfo r = sibson_row<G, FastWS, Sink::FULL, PM>(M, q, ws, g);
            steps += r.steps;
            if (r.status == ST_CAPACITY || r.status == ST_UNCERTAIN) {
                if (g.lane == 0) {
                    const int slot = atomicAdd(&sum->large_count, 1);
                    lq.list[slot] = (int)i;
                }
            } else {
                if (r.status != ST_OK && g.lane == 0) {
                    atomicAdd(&sum->rows_failed, 1ull);
                    atomicCAS(&sum->first_status, 0, NIF_ERR_WALK);
                }
                if (r.outside && g.lane == 0) atomicAdd(&sum->rows_outside, 1ull);
                sink.template emit<G>(i, r.status == ST_OK ? r.nnb : 0, ws, g, false, M, q, r);
            }
            g.sync();
        }
    }
    if (g.lane == 0 && steps) atomicAdd(&sum->walk_steps, steps);
}

template <class QT, class Sink>
__global__ void __launch_bounds__(32) k_rows_batch_large(const MeshView *__restrict__ views,
                                                         const int64_t *__restrict__ qoff, int P,
                                                         const QT *__restrict__ Q,
                                                         const double *__restrict__ cens, LargeQueue lq,
                                                         Sink sink, LargeWS *__restrict__ wsv,
                                                         double *__restrict__ xsv, DevSummary *sum) {
    constexpr int G = LARGE_G;
    __shared__ MeshView M;
    Grp<G> g;
    LargeWS &ws = wsv[blockIdx.x];
    double *xs = xsv + (size_t)blockIdx.x * NIF_EXACT_SCRATCH;
    const int nq = sum->large_count;
    int cur = -1;
    for (int j = blockIdx.x; j < nq; j += gridDim.x) {
        const int64_t i = lq.list[j];
        const int p = find_problem(qoff, P, i);
        if (p != cur) {
            g.sync();
            if (g.lane == 0) M = views[p];
            g.sync();
            cur = p;
        }
        const dv3 q = load_query(Q, i, cens + 3 * p);
        const RowInfo r = sibson_row<G, LargeWS, Sink::FULL, PM_RESOLVE>(M, q, ws, g, xs);
        record_predicates<G>(sum, r, g.lane);
        if (g.lane == 0) atomicAdd(&sum->rows_large, 1ull);
        if (r.status != ST_OK) {
            if (g.lane == 0) {
                atomicAdd(&sum->rows_failed, 1ull);
                atomicCAS(&sum->first_status, 0, r.status == ST_WALK ? NIF_ERR_WALK : NIF_ERR_CAPACITY);
            }
            sink.template emit<G>(i, 0, ws, g, true, M, q, r);
        } else {
            sink.template emit<G>(i, r.nnb, ws, g, true, M, q, r);
        }
        g.sync();
    }
}

}  // namespace nif

struct nif_dbatch {
    int P;
    int device;
    int num_sms;
    bool filtered;      // some mesh uses a non-default predicate mode
    MeshView *d_views;  // [P] in the caller's buffer
    nif_tuning tune{OCC_DEFAULT, 0, BATCH_TILE_DEFAULT, 0};
};

namespace {

struct BatchLayout {
    DevSummary *sum;
    unsigned long long *counter;
    int *bits, *bucket, *bcount, *order, *large_list, *bsum, *btotal;
    int64_t *bbase;
    LargeWS *large_ws;
    double *exact;
    // split rows (the default predicate mode): located tets, one chunk's
    // records, rows whose cavity exceeds a record
    int *located, *wide;
    RowHead *heads;
    RowEntry *ents;
};

BatchLayout carve_batch(Carve &c, int P, int64_t M) {
    BatchLayout L{};
    const int64_t nbk = 8 * (int64_t)P + M / 2 + 1;
    L.sum = c.take<DevSummary>(1);
    L.counter = c.take<unsigned long long>(1);
    L.bits = c.take<int>(P);
    L.bbase = c.take<int64_t>(P + 1);
    L.bucket = c.take<int>(M > 0 ? M : 1);
    L.bcount = c.take<int>(nbk + 1);
    L.order = c.take<int>(M > 0 ? M : 1);
    L.large_list = c.take<int>(M > 0 ? M : 1);
    L.bsum = c.take<int>((nbk + 1 + SCAN_TILE - 1) / SCAN_TILE + 1);
    L.btotal = c.take<int>(2);
    L.large_ws = c.take<LargeWS>(LARGE_GROUPS);
    L.exact = c.take<double>((size_t)LARGE_GROUPS * NIF_EXACT_SCRATCH);
    const int64_t m1 = M > 0 ? M : 1;
    const int64_t ch = m1 < REC_CHUNK ? m1 : REC_CHUNK;
    L.located = c.take<int>(m1);
    L.wide = c.take<int>(m1);
    L.heads = c.take<RowHead>(ch);
    L.ents = c.take<RowEntry>(ch * REC_CAV);
    return L;
}

template <class QT, class Sink, int PM, int OCC>
void launch_batch_rows_occ(const nif_dbatch *b, const QT *Q, int64_t M, const int64_t *qoff,
                           const double *cens, const Sink &sink, const BatchLayout &L,
                           cudaStream_t st, const int *order, const int *nrows_dev) {
    constexpr int GPB = FAST_BLOCK / FAST_G;
    const size_t smem = GPB * sizeof(FastWS);
    auto kern = k_rows_batch<QT, Sink, PM, OCC>;
    const int per_sm = resident_blocks(kern, FAST_BLOCK, smem);
    const int tile = b->tune.tile;
    const int64_t want = (M + (int64_t)GPB * tile - 1) / ((int64_t)GPB * tile);
    int64_t blocks = (int64_t)per_sm * b->num_sms;
    if (blocks > want) blocks = want;
    if (blocks < 1) blocks = 1;
    cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), st);
    kern<<<(unsigned)blocks, FAST_BLOCK, smem, st>>>(b->d_views, qoff, b->P, Q, cens, order, M, nrows_dev,
                                                    sink, LargeQueue{L.large_list}, L.sum, L.counter,
                                                    tile);
}

// the fused batch row kernel over positions [0, M) of `order` (bounded by
// *nrows_dev where that is set)
template <class QT, class Sink, int PM>
void launch_batch_rows(const nif_dbatch *b, const QT *Q, int64_t M, const int64_t *qoff,
                       const double *cens, const Sink &sink, const BatchLayout &L, cudaStream_t st,
                       const int *order, const int *nrows_dev = nullptr) {
    if (b->tune.blocks_per_sm == OCC_LO)
        launch_batch_rows_occ<QT, Sink, PM, OCC_LO>(b, Q, M, qoff, cens, sink, L, st, order, nrows_dev);
    else
        launch_batch_rows_occ<QT, Sink, PM, OCC_HI>(b, Q, M, qoff, cens, sink, L, st, order, nrows_dev);
}

template <class QT, class VT, class CT>
void batch_typed(const nif_dbatch *b, const void *q, int64_t M, const int64_t *qoff, const double *cens,
                 const void *v, const int64_t *koff, int D, void *out, const BatchLayout &L,
                 cudaStream_t st) {
    using Sink = BatchInterpSink<QT, VT, CT>;
    const QT *Q = static_cast<const QT *>(q);
    const int64_t nbk = 8 * (int64_t)b->P + M / 2 + 1;
    cudaMemsetAsync(L.sum, 0, sizeof(DevSummary), st);
    cudaMemsetAsync(L.counter, 0, sizeof(unsigned long long), st);
    cudaMemsetAsync(L.bcount, 0, sizeof(int) * (nbk + 1), st);
    k_batch_setup<<<1, 1, 0, st>>>(qoff, b->P, L.bits, L.bbase);
    k_batch_bucket<QT><<<blocks_for(M, 256), 256, 0, st>>>(Q, M, qoff, b->P, cens, b->d_views, L.bits,
                                                          L.bbase, L.bucket, L.bcount);
    launch_scan<int>(L.bcount, nbk, L.bsum, L.btotal, L.bcount, st);
    k_scatter<<<blocks_for(M, 256), 256, 0, st>>>(L.bucket, M, L.bcount, L.order);
    Sink sink{static_cast<const VT *>(v), koff, qoff, b->P, static_cast<CT *>(out), D};
    // the split row kernels, rows mapped to their problems' meshes (filtered
    // predicates where any problem's mesh asks for them: the kernels test
    // each mesh's own mode); then the rows whose cavity exceeds a record
    // through the fused kernel
    const Launch lc{b->tune.tile, b->num_sms};
    const ManyMeshes rows{b->d_views, qoff, b->P, cens};
    const RowSet R{L.order, nullptr, L.large_list, L.sum, L.counter, L.located};
    if (b->filtered) {
        if (b->tune.blocks_per_sm == OCC_LO)
            launch_split<QT, ManyMeshes, Sink, OCC_LO, PM_FILTER>(lc, rows, Q, M, R, L.heads, L.ents,
                                                                  L.wide, sink, st);
        else
            launch_split<QT, ManyMeshes, Sink, OCC_HI, PM_FILTER>(lc, rows, Q, M, R, L.heads, L.ents,
                                                                  L.wide, sink, st);
        launch_batch_rows<QT, Sink, PM_FILTER>(b, Q, M, qoff, cens, sink, L, st, L.wide,
                                               &L.sum->wide_count);
    } else {
        if (b->tune.blocks_per_sm == OCC_LO)
            launch_split<QT, ManyMeshes, Sink, OCC_LO>(lc, rows, Q, M, R, L.heads, L.ents, L.wide, sink, st);
        else
            launch_split<QT, ManyMeshes, Sink, OCC_HI>(lc, rows, Q, M, R, L.heads, L.ents, L.wide, sink, st);
        launch_batch_rows<QT, Sink, PM_PLAIN>(b, Q, M, qoff, cens, sink, L, st, L.wide,
                                              &L.sum->wide_count);
    }
    k_rows_batch_large<QT, Sink><<<LARGE_GROUPS, 32, 0, st>>>(b->d_views, qoff, b->P, Q, cens,
                                                             LargeQueue{L.large_list}, sink,
                                                             L.large_ws, L.exact, L.sum);
}

}  // namespace

NIF_EXPORT int nif_batch_set_tuning(nif_dbatch *b, const nif_tuning *t) {
    if (!b || !tuning_ok(t, true)) return NIF_ERR_ARG;
    b->tune = *t;
    return NIF_OK;
}

NIF_EXPORT int nif_batch_get_tuning(const nif_dbatch *b, nif_tuning *t) {
    if (!b || !t) return NIF_ERR_ARG;
    *t = b->tune;
    return NIF_OK;
}

NIF_EXPORT int nif_batch_bytes(int n_problems, size_t *bytes) {
    if (!bytes || n_problems < 1) return NIF_ERR_ARG;
    *bytes = align_up(sizeof(MeshView) * (size_t)n_problems, 256);
    return NIF_OK;
}

NIF_EXPORT int nif_batch_create(int n_problems, nif_dmesh *const *meshes, void *d_buf, size_t buf_bytes,
                                void *stream, nif_dbatch **out) {
    if (!out || !meshes || n_problems < 1 || !d_buf) return NIF_ERR_ARG;
    *out = nullptr;
    size_t need = 0;
    nif_batch_bytes(n_problems, &need);
    if (buf_bytes < need) return NIF_ERR_WORKSPACE;
    MeshView *host = static_cast<MeshView *>(malloc(sizeof(MeshView) * (size_t)n_problems));
    if (!host) return NIF_ERR_NOMEM;
    int dev = -1;
    bool filtered = false;
    for (int p = 0; p < n_problems; p++) {
        if (!meshes[p] || (p > 0 && meshes[p]->device != dev)) {
            free(host);
            return NIF_ERR_ARG;
        }
        dev = meshes[p]->device;
        host[p] = meshes[p]->view;  // predicate modes as of now
        filtered = filtered || host[p].pmode != PRED_FAST;
    }
    cudaStream_t st = S(stream);
    if (cudaMemcpyAsync(d_buf, host, sizeof(MeshView) * (size_t)n_problems, cudaMemcpyHostToDevice, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        free(host);
        return NIF_ERR_CUDA;
    }
    free(host);
    nif_dbatch *b = new (std::nothrow) nif_dbatch();
    if (!b) return NIF_ERR_NOMEM;
    b->P = n_problems;
    b->device = dev;
    b->num_sms = meshes[0]->num_sms;
    b->filtered = filtered;
    b->d_views = static_cast<MeshView *>(d_buf);
    *out = b;
    return NIF_OK;
}

NIF_EXPORT void nif_batch_destroy(nif_dbatch *b) { delete b; }

NIF_EXPORT int nif_batch_workspace_bytes(const nif_dbatch *b, int64_t total_queries, size_t *bytes) {
    if (!b || !bytes || total_queries < 0 || total_queries > (int64_t)INT32_MAX) return NIF_ERR_ARG;
    Carve c{nullptr, 0, (size_t)-1, true};
    carve_batch(c, b->P, total_queries);
    *bytes = align_up(c.off, 256);
    return NIF_OK;
}

NIF_EXPORT int nif_batch_interpolate(const nif_dbatch *b, const void *d_queries, int query_dtype,
                                     const int64_t *d_query_offsets, const double *d_centroids,
                                     const void *d_values, int values_dtype,
                                     const int64_t *d_key_offsets, int D, void *d_out, int out_dtype,
                                     int64_t total_queries, void *d_ws, size_t ws_bytes, void *stream) {
    if (!b || total_queries < 0 || total_queries > (int64_t)INT32_MAX || D < 1) return NIF_ERR_ARG;
    if ((query_dtype != NIF_F64 && query_dtype != NIF_F32) ||
        (values_dtype != NIF_F64 && values_dtype != NIF_F32))
        return NIF_ERR_ARG;
    if (out_dtype != expect_promoted(query_dtype, values_dtype)) return NIF_ERR_ARG;
    if (!d_query_offsets || !d_centroids || !d_key_offsets || !d_ws) return NIF_ERR_ARG;
    if (total_queries > 0 && (!d_queries || !d_values || !d_out)) return NIF_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(d_ws) % 256 != 0) return NIF_ERR_ARG;
    size_t need = 0;
    nif_batch_workspace_bytes(b, total_queries, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    cudaStream_t st = S(stream);
    Carve c{reinterpret_cast<unsigned char *>(d_ws), 0, ws_bytes, true};
    BatchLayout L = carve_batch(c, b->P, total_queries);
    if (total_queries == 0) return cuda_rc(cudaMemsetAsync(L.sum, 0, sizeof(DevSummary), st));
    const int64_t M = total_queries;
    if (query_dtype == NIF_F64 && values_dtype == NIF_F64)
        batch_typed<double, double, double>(b, d_queries, M, d_query_offsets, d_centroids, d_values,
                                            d_key_offsets, D, d_out, L, st);
    else if (query_dtype == NIF_F64)
        batch_typed<double, float, double>(b, d_queries, M, d_query_offsets, d_centroids, d_values,
                                           d_key_offsets, D, d_out, L, st);
    else if (values_dtype == NIF_F32)
        batch_typed<float, float, float>(b, d_queries, M, d_query_offsets, d_centroids, d_values,
                                         d_key_offsets, D, d_out, L, st);
    else
        batch_typed<float, double, double>(b, d_queries, M, d_query_offsets, d_centroids, d_values,
                                           d_key_offsets, D, d_out, L, st);
    return cuda_rc(cudaGetLastError());
}

NIF_EXPORT int nif_batch_summary(const nif_dbatch *b, int64_t total_queries, const void *d_ws,
                                 size_t ws_bytes, void *stream, nif_summary *summary) {
    if (!b || !summary || !d_ws) return NIF_ERR_ARG;
    size_t need = 0;
    if (nif_batch_workspace_bytes(b, total_queries, &need) != NIF_OK || ws_bytes < need)
        return NIF_ERR_WORKSPACE;
    Carve c{reinterpret_cast<unsigned char *>(const_cast<void *>(d_ws)), 0, ws_bytes, true};
    BatchLayout L = carve_batch(c, b->P, total_queries);
    DevSummary d;
    cudaStream_t st = S(stream);
    NIF_CUDA(cudaMemcpyAsync(&d, L.sum, sizeof(d), cudaMemcpyDeviceToHost, st));
    NIF_CUDA(cudaStreamSynchronize(st));
    summary->nnz = 0;
    summary->rows_large = (int64_t)d.rows_large;
    summary->rows_failed = (int64_t)d.rows_failed;
    summary->rows_outside = (int64_t)d.rows_outside;
    summary->walk_steps = (int64_t)d.walk_steps;
    summary->first_status = d.first_status;
    summary->rows_wide = d.wide_count;
    summary->orient_uncertain = (int64_t)d.orient_unc;
    summary->orient_flipped = (int64_t)d.orient_flip;
    summary->insphere_uncertain = (int64_t)d.insphere_unc;
    summary->insphere_flipped = (int64_t)d.insphere_flip;
    return NIF_OK;
}

NIF_EXPORT int nif_query_summary(const nif_dmesh *m, int64_t M, int mode, const void *d_ws,
                                 size_t ws_bytes, void *stream, nif_summary *summary) {
    if (!m || !summary || !d_ws || M < 0) return NIF_ERR_ARG;
    size_t need = 0;
    int rc = nif_query_workspace_bytes(m, M, mode, &need);
    if (rc != NIF_OK) return rc;
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    Carve c{reinterpret_cast<unsigned char *>(const_cast<void *>(d_ws)), 0, ws_bytes, true};
    QueryLayout L = carve_query(c, M, mode);
    return read_summary(L, S(stream), summary, nullptr);
}

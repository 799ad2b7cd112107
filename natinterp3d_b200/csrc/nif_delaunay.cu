// Delaunay tetrahedralization of the keys on the GPU (opt-in constructor).
//
// natinterp3d builds its mesh on the host by sequential Bowyer-Watson
// insertion into a super-simplex (buildMesh, delaunay.c:108-161: the
// super-simplex of initSuperSimplex, delaunay.c:832-863, then addPoint per
// key, delaunay.c:619-688, whose cavity is the conflict search of
// delaunay.c:561-614).  The tetrahedralization of keys + super-simplex
// vertices that this produces is the Delaunay tetrahedralization of those
// points; for points in general position (no five on a sphere, no four on a
// plane among those a cavity meets) it is unique, so any insertion order
// gives the same set of tets.  Here the keys are inserted in parallel
// rounds:
//
//   1. every uninserted key knows a tet that contains it; each tet holding
//      keys nominates one of them (the lowest pseudo-random priority);
//   2. every nominee finds its cavity -- the connected tets whose
//      circumsphere strictly contains it -- and claims the cavity tets and
//      the tets just outside it with atomicMin of its priority;
//   3. nominees that hold every claim are winners.  Two winners' claimed
//      regions are disjoint and never adjacent, so inserting all winners at
//      once equals inserting them one after another: no tet outside a
//      winner's cavity can conflict with it after another winner's insertion
//      (a conflict would be connected to the winner through a claimed tet);
//   4. each winner replaces its cavity by the tets joining it to the cavity's
//      boundary faces, reusing the cavity's slots;
//   5. keys whose tet died walk to their new tet, starting from a tet of the
//      winner that killed it.
//
// Every sign is exact: the fast determinant decides when it clears the
// static error bound, and the expansion arithmetic of nif_exact.h decides
// the rest.  A zero where it matters (a key on the circumsphere of a tet it
// meets, a key on the plane of a cavity boundary face, duplicate keys) makes
// the result depend on tie-breaking, which natinterp3d settles by random
// perturbation (delaunay.c:513-522); this builder stops with
// NIF_ERR_DEGENERATE instead and the caller falls back to natinterp3d's
// constructor.  The output uses natinterp3d's packed layout and face order
// (getFaceVerticies3, delaunay.c:444-467: face f lies opposite p[3-f] and is
// shared with neighbour s[f]); every tet is positively oriented.  A check
// kernel verifies the result with exact predicates: orientation, neighbour
// symmetry and the empty-sphere property of every interior face (local
// Delaunay everywhere implies Delaunay).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>

#include "natinterp3d_b200.h"
#include "nif_exact.h"
#include "nif_geometry.cuh"

#define NIF_EXPORT extern "C" __attribute__((visibility("default")))

namespace nif {
namespace dt {

constexpr int WARPS = 4;               // warps per block of the warp kernels
constexpr int THREADS = 32 * WARPS;
constexpr int HS = 512;                // tested-tet hash slots per insertion (power of two)
constexpr int CAV = 256;               // cavity tets per insertion
constexpr int BF = 2 * CAV + 2;        // boundary faces per insertion
constexpr int WALK_LIMIT = 1 << 16;    // steps of one relocation walk
constexpr int ROUND_LIMIT = 1 << 14;   // insertion rounds
constexpr unsigned FULL = 0xffffffffu;

enum : int {
    ERR_NONE = 0,
    ERR_DEGENERATE = 1,   // an exact zero that decides the result
    ERR_CAPACITY = 2,     // tet slots or list space exhausted
    ERR_WALK = 3,         // a relocation walk exceeded its step limit
    ERR_OUTSIDE = 4,      // a key outside the super-simplex
    ERR_INTERNAL = 5,     // an inconsistency (a negative boundary orientation)
};

// per-round and global counters (device)
struct State {
    int nnom;               // nominees this round
    int nwin;               // winners this round
    int nreloc;             // keys to relocate this round
    int err;                // first error (ERR_*)
    long long listtop;      // ints used in the cavity lists this round
    int tet_top;            // tet slots in use (high-water mark)
    int inserted;           // keys inserted so far
    int deferred;           // nominees skipped for capacity this round
    int max_cav;            // largest cavity seen
    unsigned long long exact_evals;  // predicates decided by expansion arithmetic
};

// one nominee's cavity in the round's list buffer: ncav tet ids, then nbf
// (cavity tet * 4 + face, outside tet) pairs
struct Cavity {
    long long off;
    int ncav, nbf;
    int status;  // 0 ok, 1 skipped this round, 2 failed, 3 outranked nearby (no flood)
    int pad;
};

struct Dev {
    double4 *pts;           // [n + 4]: keys, then the super-simplex vertices
    int4 *tv, *tn;          // [cap]
    unsigned long long *own, *nom;  // [cap] round-stamped claims
    int *kround;            // [cap] round in which the slot's tet died
    int *startnew;          // [cap] a live tet of the winner that killed it
    int *ptet;              // [n] containing tet of an uninserted key, -1 once inserted
    int *noms, *wins, *reloc;  // [n] lists of the round
    Cavity *cav;            // [n]
    int *lists;             // [list_cap]
    long long list_cap;
    double *scratch;        // [warps][NIF_EXACT_SCRATCH]
    int scratch_warps;
    double *bbox;           // [2 * 3 * blocks] partial extents
    State *st;
    int n, cap;
};

__device__ __forceinline__ dv3 P3(const double4 &v) { return dv3{v.x, v.y, v.z}; }

__device__ __forceinline__ int comp4(const int4 &v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// face f of a tet lies opposite p[3-f]: (0,1,2) (3,1,0) (0,2,3) (3,2,1)
__device__ __forceinline__ int fslot(int f, int j) {
    constexpr unsigned bits = (0u | 1u << 2 | 2u << 4) | ((3u | 1u << 2 | 0u << 4) << 6) |
                              ((0u | 2u << 2 | 3u << 4) << 12) | ((3u | 2u << 2 | 1u << 4) << 18);
    return (bits >> (6 * f + 2 * j)) & 3;
}

__device__ __forceinline__ unsigned long long key_of(int round, int p) {
    const unsigned pr = (unsigned)p * 2654435761u ^ 0x5bd1e995u;  // a bijection of the key id
    return ((unsigned long long)(0xffffffffu - (unsigned)round) << 32) | pr;
}

__device__ __forceinline__ void set_err(State *st, int e) { atomicCAS(&st->err, ERR_NONE, e); }

__device__ __forceinline__ double *warp_scratch(const Dev &D) {
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    return D.scratch + (size_t)(w % D.scratch_warps) * NIF_EXACT_SCRATCH;
}

// Exact sign of orient3d / insphere with natinterp3d's conventions: the fast
// value when it clears the error bound, else the lanes in `pending` (a
// ballot taken by the whole warp) evaluate the expansion one at a time in
// the warp's scratch.
__device__ int orient_sign(const Dev &D, dv3 a, dv3 b, dv3 c, dv3 d, bool active) {
    int s = 0;
    bool unc = false;
    if (active) {
        const double o = orient_fast(a, b, c, d);
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z},
                     E[3] = {d.x, d.y, d.z};
        unc = nif_orient_uncertain(o, nif_orient_permanent(A, B, C, E));
        s = o > 0.0 ? 1 : (o < 0.0 ? -1 : 0);
    }
    unsigned pend = __ballot_sync(FULL, unc);
    if (pend) {
        double *scr = warp_scratch(D);
        const int lane = threadIdx.x & 31;
        while (pend) {
            const int l = __ffs(pend) - 1;
            if (lane == l) {
                const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z},
                             E[3] = {d.x, d.y, d.z};
                s = nif_orient_exact_sign(A, B, C, E, scr);
                atomicAdd(&D.st->exact_evals, 1ull);
            }
            __syncwarp();
            pend &= pend - 1;
        }
    }
    return s;
}

__device__ int insphere_sign(const Dev &D, dv3 a, dv3 b, dv3 c, dv3 d, dv3 e, bool active) {
    int s = 0;
    bool unc = false;
    if (active) {
        const double v = insphere_fast(a, b, c, d, e);
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z},
                     E[3] = {d.x, d.y, d.z}, F[3] = {e.x, e.y, e.z};
        unc = nif_insphere_uncertain(v, nif_insphere_permanent(A, B, C, E, F));
        s = v > 0.0 ? 1 : (v < 0.0 ? -1 : 0);
    }
    unsigned pend = __ballot_sync(FULL, unc);
    if (pend) {
        double *scr = warp_scratch(D);
        const int lane = threadIdx.x & 31;
        while (pend) {
            const int l = __ffs(pend) - 1;
            if (lane == l) {
                const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z},
                             E[3] = {d.x, d.y, d.z}, F[3] = {e.x, e.y, e.z};
                s = nif_insphere_exact_sign(A, B, C, E, F, scr);
                atomicAdd(&D.st->exact_evals, 1ull);
            }
            __syncwarp();
            pend &= pend - 1;
        }
    }
    return s;
}

// ---------------------------------------------------------------------------
// set-up: extents, super-simplex, first tet

__global__ void k_bbox(const double *__restrict__ keys, int n, double *__restrict__ part) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int a = 0; a < 3; a++) {
            const double v = keys[3 * (size_t)i + a];
            lo[a] = fmin(lo[a], v);
            hi[a] = fmax(hi[a], v);
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

// natinterp3d's super-simplex (initSuperSimplex, delaunay.c:841-855, from
// the extents of getRange, delaunay.c:1086-1111), the first tet, and every
// key located in it.  Vertex ids: keys 0..n-1, super-simplex n..n+3.
__global__ void k_init(Dev D, const double *__restrict__ keys, int nblocks) {
    __shared__ int ok;
    if (threadIdx.x == 0) {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int b = 0; b < nblocks; b++)
            for (int a = 0; a < 3; a++) {
                lo[a] = fmin(lo[a], D.bbox[6 * b + a]);
                hi[a] = fmax(hi[a], D.bbox[6 * b + 3 + a]);
            }
        double r[3];
        ok = 1;
        for (int a = 0; a < 3; a++) {
            r[a] = __dsub_rn(hi[a], lo[a]);
            if (!(r[a] > 0.0) || !isfinite(r[a])) ok = 0;
        }
        const double half_x = __ddiv_rn(r[0], 2.0), half_y = __ddiv_rn(r[1], 2.0);
        double4 s0 = make_double4(__dadd_rn(lo[0], half_x), __dadd_rn(hi[1], __dmul_rn(3.0, r[1])),
                                  __dsub_rn(lo[2], r[2]), 0.0);
        double4 s1 = make_double4(__dadd_rn(hi[0], __dmul_rn(2.0, r[0])),
                                  __dsub_rn(lo[1], __dmul_rn(2.0, r[1])), __dsub_rn(lo[2], r[2]), 0.0);
        double4 s2 = make_double4(__dsub_rn(lo[0], __dmul_rn(2.0, r[0])),
                                  __dsub_rn(lo[1], __dmul_rn(2.0, r[1])), __dsub_rn(lo[2], r[2]), 0.0);
        double4 s3 = make_double4(__dadd_rn(lo[0], half_x), __dadd_rn(lo[1], half_y),
                                  __dadd_rn(hi[2], __dmul_rn(2.0, r[2])), 0.0);
        D.pts[D.n] = s0;
        D.pts[D.n + 1] = s1;
        D.pts[D.n + 2] = s2;
        D.pts[D.n + 3] = s3;
        if (!ok) set_err(D.st, ERR_DEGENERATE);
    }
    __syncthreads();
    // the first tet: the super-simplex, positively oriented
    if (threadIdx.x < 32) {
        const dv3 a = P3(D.pts[D.n]), b = P3(D.pts[D.n + 1]), c = P3(D.pts[D.n + 2]),
                  d = P3(D.pts[D.n + 3]);
        const int s = orient_sign(D, a, b, c, d, threadIdx.x == 0);
        if (threadIdx.x == 0) {
            D.tv[0] = s > 0 ? make_int4(D.n, D.n + 1, D.n + 2, D.n + 3)
                            : make_int4(D.n + 1, D.n, D.n + 2, D.n + 3);
            D.tn[0] = make_int4(-1, -1, -1, -1);
            if (s == 0) set_err(D.st, ERR_DEGENERATE);
            D.st->tet_top = 1;
        }
    }
}

__global__ void k_load_keys(Dev D, const double *__restrict__ keys) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += gridDim.x * blockDim.x) {
        D.pts[i] = make_double4(keys[3 * (size_t)i], keys[3 * (size_t)i + 1], keys[3 * (size_t)i + 2], 0.0);
        D.ptet[i] = 0;
    }
}

// every key strictly inside the super-simplex (warp per key, 4 lanes)
__global__ void k_check_inside(Dev D) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int4 t = D.tv[0];
    for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < D.n; i += warps) {
        const dv3 q = P3(D.pts[i]);
        dv3 a{0, 0, 0}, b = a, c = a;
        if (lane < 4) {
            a = P3(D.pts[comp4(t, fslot(lane, 0))]);
            b = P3(D.pts[comp4(t, fslot(lane, 1))]);
            c = P3(D.pts[comp4(t, fslot(lane, 2))]);
        }
        const int s = orient_sign(D, a, b, c, q, lane < 4);
        if (__any_sync(FULL, lane < 4 && s <= 0) && lane == 0) set_err(D.st, ERR_OUTSIDE);
    }
}

// ---------------------------------------------------------------------------
// one insertion round

__global__ void k_nominate(Dev D, int round) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < D.n; p += gridDim.x * blockDim.x) {
        const int t = D.ptet[p];
        if (t >= 0) atomicMin(&D.nom[t], key_of(round, p));
    }
}

__global__ void k_collect(Dev D, int round) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < D.n; p += gridDim.x * blockDim.x) {
        const int t = D.ptet[p];
        if (t >= 0 && D.nom[t] == key_of(round, p)) D.noms[atomicAdd(&D.st->nnom, 1)] = p;
    }
}

// warp-private open-addressing set of tested tets in shared memory:
// state 1 = in the cavity, 2 = outside
struct CavWS {
    int hkey[HS];
    int8_t hstate[HS];
    int cav[CAV];
    int ncav;
};

__device__ __forceinline__ unsigned thash(int t) { return (unsigned)t * 2654435761u; }

// slot of t (inserted when absent: *fresh = true); -1 when the table is full
__device__ int h_upsert(CavWS &w, int t, bool *fresh) {
    unsigned h = thash(t) & (HS - 1);
    for (int k = 0; k < HS; k++) {
        const int prev = atomicCAS(&w.hkey[h], -1, t);
        if (prev == -1) {
            *fresh = true;
            return (int)h;
        }
        if (prev == t) {
            *fresh = false;
            return (int)h;
        }
        h = (h + 1) & (HS - 1);
    }
    *fresh = false;
    return -1;
}

__device__ int h_find(const CavWS &w, int t) {
    unsigned h = thash(t) & (HS - 1);
    for (int k = 0; k < HS; k++) {
        const int v = w.hkey[h];
        if (v == t) return (int)h;
        if (v == -1) return -1;
        h = (h + 1) & (HS - 1);
    }
    return -1;
}

// The cavity of every nominee and its claims.  One warp per nominee.
__global__ void __launch_bounds__(THREADS) k_cavity(Dev D, int round) {
    __shared__ CavWS wsv[WARPS];
    CavWS &w = wsv[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int nnom = D.st->nnom;
    for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < nnom; i += warps) {
        const int p = D.noms[i];
        const unsigned long long key = key_of(round, p);
        const dv3 P = P3(D.pts[p]);
        const int t0 = D.ptet[p];
        // A nominee within two tet steps of a nominee with a lower priority
        // skips the flood: their claims would meet in a tet adjacent to both
        // start tets, so it could only win if that nominee did not claim.
        // Every nominee that would win without this test passes it (all the
        // nominees it conflicts with have higher priorities), and the
        // nominees it removes claim nothing, so no winner is lost.
        bool lower = false;
        if (lane < 16) {
            const int n1 = comp4(D.tn[t0], lane >> 2);
            if (n1 >= 0) {
                lower = D.nom[n1] < key;
                const int n2 = comp4(D.tn[n1], lane & 3);
                if (n2 >= 0 && D.nom[n2] < key) lower = true;
            }
        }
        if (__any_sync(FULL, lower)) {
            if (lane == 0) {
                Cavity cv;
                cv.off = 0;
                cv.ncav = cv.nbf = 0;
                cv.status = 3;
                cv.pad = 0;
                D.cav[i] = cv;
            }
            __syncwarp();
            continue;
        }
        for (int k = lane; k < HS; k += 32) w.hkey[k] = -1;
        __syncwarp();
        if (lane == 0) {
            bool fr;
            const int s = h_upsert(w, t0, &fr);
            w.hstate[s] = 1;
            w.cav[0] = t0;
            w.ncav = 1;
        }
        __syncwarp();
        int status = 0;  // 0 ok, 1 over capacity, 2 degenerate
        int head = 0;
        // breadth-first over tets whose circumsphere strictly contains P
        while (head < w.ncav && status == 0) {
            const int end = w.ncav;
            for (int k0 = 0; k0 < 4 * (end - head); k0 += 32) {
                const int k = k0 + lane;
                bool test = false;
                int nb = -1, slot = -1;
                if (k < 4 * (end - head)) {
                    const int c = w.cav[head + (k >> 2)];
                    nb = comp4(D.tn[c], k & 3);
                    if (nb >= 0) {
                        bool fresh = false;
                        slot = h_upsert(w, nb, &fresh);
                        if (slot < 0) status = 1;
                        test = fresh;
                    }
                }
                dv3 a{0, 0, 0}, b = a, c = a, d = a;
                if (test) {
                    const int4 v = D.tv[nb];
                    a = P3(D.pts[v.x]);
                    b = P3(D.pts[v.y]);
                    c = P3(D.pts[v.z]);
                    d = P3(D.pts[v.w]);
                }
                const int s = insphere_sign(D, a, b, c, d, P, test);
                if (test) {
                    if (s == 0) status = 2;
                    if (s > 0) {
                        w.hstate[slot] = 1;
                        const int at = atomicAdd(&w.ncav, 1);
                        if (at < CAV)
                            w.cav[at] = nb;
                        else
                            status = 1;
                    } else {
                        w.hstate[slot] = 2;
                    }
                }
                status = __reduce_max_sync(FULL, status);
            }
            __syncwarp();
            head = end;
        }
        const int ncav = min(w.ncav, CAV);
        // boundary faces: (cavity tet, face) whose neighbour is not in the cavity
        int nbf = 0;
        if (status == 0) {
            for (int k0 = 0; k0 < 4 * ncav; k0 += 32) {
                const int k = k0 + lane;
                bool isb = false;
                if (k < 4 * ncav) {
                    const int nb = comp4(D.tn[w.cav[k >> 2]], k & 3);
                    const int hs = nb < 0 ? -1 : h_find(w, nb);
                    isb = hs < 0 || w.hstate[hs] != 1;
                }
                nbf += __popc(__ballot_sync(FULL, isb));
            }
            if (nbf > BF) status = 1;
        }
        long long off = 0;
        if (status == 0) {
            if (lane == 0) off = atomicAdd((unsigned long long *)&D.st->listtop,
                                           (unsigned long long)(ncav + 2 * nbf));
            off = __shfl_sync(FULL, off, 0);
            if (off + ncav + 2 * nbf > D.list_cap) status = 1;
        }
        if (status == 0) {
            int *L = D.lists + off;
            for (int k = lane; k < ncav; k += 32) L[k] = w.cav[k];
            int base = 0;
            for (int k0 = 0; k0 < 4 * ncav; k0 += 32) {
                const int k = k0 + lane;
                bool isb = false;
                int c = -1, nb = -1;
                if (k < 4 * ncav) {
                    c = w.cav[k >> 2];
                    nb = comp4(D.tn[c], k & 3);
                    const int hs = nb < 0 ? -1 : h_find(w, nb);
                    isb = hs < 0 || w.hstate[hs] != 1;
                }
                // P must see every boundary face from inside the cavity
                dv3 a{0, 0, 0}, b = a, cc = a;
                if (isb) {
                    const int4 v = D.tv[c];
                    a = P3(D.pts[comp4(v, fslot(k & 3, 0))]);
                    b = P3(D.pts[comp4(v, fslot(k & 3, 1))]);
                    cc = P3(D.pts[comp4(v, fslot(k & 3, 2))]);
                }
                const int so = orient_sign(D, a, b, cc, P, isb);
                if (isb && so == 0) status = 2;
                if (isb && so < 0) set_err(D.st, ERR_INTERNAL);
                const unsigned bm = __ballot_sync(FULL, isb);
                if (isb) {
                    const int at = base + __popc(bm & ((1u << lane) - 1u));
                    L[ncav + 2 * at] = 4 * c + (k & 3);
                    L[ncav + 2 * at + 1] = nb;
                }
                base += __popc(bm);
            }
            status = __reduce_max_sync(FULL, status);
        }
        if (status == 0) {
            // claims: the cavity and the tets across its boundary
            const int *L = D.lists + off;
            for (int k = lane; k < ncav; k += 32) atomicMin(&D.own[L[k]], key);
            for (int k = lane; k < nbf; k += 32) {
                const int o = L[ncav + 2 * k + 1];
                if (o >= 0) atomicMin(&D.own[o], key);
            }
        }
        if (lane == 0) {
            Cavity cv;
            cv.off = off;
            cv.ncav = ncav;
            cv.nbf = nbf;
            cv.status = status;
            cv.pad = 0;
            D.cav[i] = cv;
            if (status == 1) atomicAdd(&D.st->deferred, 1);
            if (status == 2) set_err(D.st, ERR_DEGENERATE);
            if (status == 0) atomicMax(&D.st->max_cav, ncav);
        }
        __syncwarp();
    }
}

// winners: nominees that hold every one of their claims
__global__ void k_check(Dev D, int round) {
    const int nnom = D.st->nnom;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnom; i += gridDim.x * blockDim.x) {
        const Cavity cv = D.cav[i];
        if (cv.status != 0) continue;
        const unsigned long long key = key_of(round, D.noms[i]);
        const int *L = D.lists + cv.off;
        bool won = true;
        for (int k = 0; k < cv.ncav && won; k++) won = D.own[L[k]] == key;
        for (int k = 0; k < cv.nbf && won; k++) {
            const int o = L[cv.ncav + 2 * k + 1];
            won = o < 0 || D.own[o] == key;
        }
        if (won) D.wins[atomicAdd(&D.st->nwin, 1)] = i;
    }
}

// shared state of one winner's insertion
struct InsWS {
    int fv[BF][3];   // boundary face vertices
    int slotg[BF];   // slot of the cavity tet in the outside tet's neighbours
};

// The winners' insertions.  One warp per winner.
__global__ void __launch_bounds__(THREADS) k_insert(Dev D, int round) {
    extern __shared__ __align__(16) unsigned char smem[];
    InsWS &w = reinterpret_cast<InsWS *>(smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int nwin = D.st->nwin;
    for (int wi = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); wi < nwin; wi += warps) {
        const int i = D.wins[wi];
        const int p = D.noms[i];
        const Cavity cv = D.cav[i];
        const int *L = D.lists + cv.off;
        const int ncav = cv.ncav, nbf = cv.nbf;
        // slots of the new tets: the cavity's, then fresh ones
        int base = 0;
        if (lane == 0 && nbf > ncav) base = atomicAdd(&D.st->tet_top, nbf - ncav);
        base = __shfl_sync(FULL, base, 0);
        if (nbf > ncav && base + (nbf - ncav) > D.cap) {
            if (lane == 0) set_err(D.st, ERR_CAPACITY);
            continue;
        }
        auto slot_of = [&](int k) { return k < ncav ? L[k] : base + (k - ncav); };
        // read everything the insertion overwrites
        for (int k = lane; k < nbf; k += 32) {
            const int cf = L[ncav + 2 * k], o = L[ncav + 2 * k + 1];
            const int c = cf >> 2, f = cf & 3;
            const int4 v = D.tv[c];
            w.fv[k][0] = comp4(v, fslot(f, 0));
            w.fv[k][1] = comp4(v, fslot(f, 1));
            w.fv[k][2] = comp4(v, fslot(f, 2));
            int g = -1;
            if (o >= 0) {
                const int4 on = D.tn[o];
                for (int j = 0; j < 4; j++)
                    if (comp4(on, j) == c) g = j;
            }
            w.slotg[k] = g;
        }
        __syncwarp();
        for (int k = lane; k < nbf; k += 32) {
            const int T = slot_of(k);
            const int a = w.fv[k][0], b = w.fv[k][1], c = w.fv[k][2];
            const int o = L[ncav + 2 * k + 1];
            // (a, b, c, p): face 0 = (a, b, c) faces the outside tet; faces
            // 1, 2, 3 = (p, b, a), (a, c, p), (p, c, b) hold the edges ab, ac, bc
            int nbr[3] = {-1, -1, -1};
            const int eu[3] = {a, a, b}, ev[3] = {b, c, c};
            for (int e = 0; e < 3; e++) {
                for (int j = 0; j < nbf; j++) {
                    if (j == k) continue;
                    const int x = w.fv[j][0], y = w.fv[j][1], z = w.fv[j][2];
                    const bool hu = x == eu[e] || y == eu[e] || z == eu[e];
                    const bool hv = x == ev[e] || y == ev[e] || z == ev[e];
                    if (hu && hv) {
                        nbr[e] = slot_of(j);
                        break;
                    }
                }
            }
            D.tv[T] = make_int4(a, b, c, p);
            D.tn[T] = make_int4(o, nbr[0], nbr[1], nbr[2]);
            if (nbr[0] < 0 || nbr[1] < 0 || nbr[2] < 0) set_err(D.st, ERR_INTERNAL);
            if (o >= 0 && w.slotg[k] >= 0)
                reinterpret_cast<int *>(&D.tn[o])[w.slotg[k]] = T;
            else if (o >= 0)
                set_err(D.st, ERR_INTERNAL);
        }
        // cavity slots: the round they died in and where their keys restart
        const int first = slot_of(0);
        for (int k = lane; k < ncav; k += 32) {
            D.kround[L[k]] = round;
            D.startnew[L[k]] = first;
            if (k >= nbf) D.tv[L[k]] = make_int4(-1, -1, -1, -1);  // slot left unused
        }
        if (lane == 0) {
            D.ptet[p] = -1;
            atomicAdd(&D.st->inserted, 1);
        }
        __syncwarp();
    }
}

__global__ void k_reloc_collect(Dev D, int round) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < D.n; p += gridDim.x * blockDim.x) {
        const int t = D.ptet[p];
        if (t >= 0 && D.kround[t] == round) D.reloc[atomicAdd(&D.st->nreloc, 1)] = p;
    }
}

// visibility walk of each key whose tet died, from a tet of its killer
// (4 lanes, one per face; the first face the key lies strictly outside of)
__global__ void __launch_bounds__(THREADS) k_relocate(Dev D) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int nreloc = D.st->nreloc;
    for (int i = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < nreloc; i += warps) {
        const int p = D.reloc[i];
        const dv3 q = P3(D.pts[p]);
        int t = D.startnew[D.ptet[p]];
        int steps = 0;
        for (;;) {
            if (++steps > WALK_LIMIT) {
                if (lane == 0) set_err(D.st, ERR_WALK);
                t = -1;
                break;
            }
            const int4 v = D.tv[t];
            dv3 a{0, 0, 0}, b = a, c = a;
            if (lane < 4) {
                a = P3(D.pts[comp4(v, fslot(lane, 0))]);
                b = P3(D.pts[comp4(v, fslot(lane, 1))]);
                c = P3(D.pts[comp4(v, fslot(lane, 2))]);
            }
            const int s = orient_sign(D, a, b, c, q, lane < 4);
            const unsigned neg = __ballot_sync(FULL, lane < 4 && s < 0);
            if (!neg) break;
            const int nt = comp4(D.tn[t], __ffs(neg) - 1);
            if (nt < 0) {
                if (lane == 0) set_err(D.st, ERR_OUTSIDE);
                t = -1;
                break;
            }
            t = nt;
        }
        if (lane == 0 && t >= 0) D.ptet[p] = t;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// verification and output

// Exact checks of the finished mesh, one warp per tet (lane f checks face
// f): positive orientation, neighbour symmetry (the neighbour across face f
// has this tet as a neighbour across a face with the same vertices), and
// the empty sphere: the neighbour's vertex opposite the shared face lies
// strictly outside this tet's circumsphere.
__global__ void __launch_bounds__(THREADS) k_verify(Dev D, unsigned long long *bad) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int top = D.st->tet_top;
    for (int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); t < top; t += warps) {
        const int4 v = D.tv[t];
        if (v.x < 0) continue;
        const dv3 a = P3(D.pts[v.x]), b = P3(D.pts[v.y]), c = P3(D.pts[v.z]), d = P3(D.pts[v.w]);
        const int so = orient_sign(D, a, b, c, d, lane == 0);
        if (lane == 0 && so <= 0) atomicAdd(&bad[0], 1ull);
        bool active = false;
        dv3 e{0, 0, 0};
        if (lane < 4) {
            const int u = comp4(D.tn[t], lane);
            if (u >= 0) {
                const int4 uv = D.tv[u];
                const int4 un = D.tn[u];
                const int f0 = comp4(v, fslot(lane, 0)), f1 = comp4(v, fslot(lane, 1)),
                          f2 = comp4(v, fslot(lane, 2));
                int back = -1, opp = -1;
                for (int j = 0; j < 4; j++) {
                    const int x = comp4(uv, j);
                    if (x != f0 && x != f1 && x != f2) opp = x;
                    if (comp4(un, j) == t) back = j;
                }
                bool sym = back >= 0 && uv.x >= 0;
                if (sym) {
                    const int g0 = comp4(uv, fslot(back, 0)), g1 = comp4(uv, fslot(back, 1)),
                              g2 = comp4(uv, fslot(back, 2));
                    const int s0 = f0 + f1 + f2, s1 = g0 + g1 + g2;
                    sym = s0 == s1 && (g0 == f0 || g0 == f1 || g0 == f2) &&
                          (g1 == f0 || g1 == f1 || g1 == f2) && (g2 == f0 || g2 == f1 || g2 == f2);
                }
                if (!sym) atomicAdd(&bad[1], 1ull);
                if (sym && opp >= 0) {
                    active = true;
                    e = P3(D.pts[opp]);
                }
            }
        }
        const int si = insphere_sign(D, a, b, c, d, e, active);
        if (active && si >= 0) atomicAdd(&bad[si == 0 ? 3 : 2], 1ull);
    }
}

__global__ void k_alive(Dev D, int *__restrict__ flag) {
    const int top = D.st->tet_top;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < top; t += gridDim.x * blockDim.x)
        flag[t] = D.tv[t].x >= 0 ? 1 : 0;
}

// exclusive scan of flag[0..n) into idx (single block; n up to a few tens of millions)
__global__ void k_scan_single(const int *__restrict__ flag, int n, int *__restrict__ idx, int *total) {
    __shared__ int part[1024];
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int a = threadIdx.x * per, b = min(n, a + per);
    int s = 0;
    for (int i = a; i < b; i++) s += flag[i];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int i = 0; i < (int)blockDim.x; i++) {
            const int x = part[i];
            part[i] = acc;
            acc += x;
        }
        *total = acc;
    }
    __syncthreads();
    int acc = part[threadIdx.x];
    for (int i = a; i < b; i++) {
        idx[i] = acc;
        acc += flag[i];
    }
}

__global__ void k_emit(Dev D, const int *__restrict__ flag, const int *__restrict__ idx,
                       double *__restrict__ vxyz, int32_t *__restrict__ otv, int32_t *__restrict__ otn) {
    const int top = D.st->tet_top;
    const int stride = gridDim.x * blockDim.x;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < top; t += stride) {
        if (!flag[t]) continue;
        const int o = idx[t];
        const int4 v = D.tv[t], nb = D.tn[t];
        otv[4 * (size_t)o] = v.x;
        otv[4 * (size_t)o + 1] = v.y;
        otv[4 * (size_t)o + 2] = v.z;
        otv[4 * (size_t)o + 3] = v.w;
        for (int j = 0; j < 4; j++) {
            const int u = comp4(nb, j);
            otn[4 * (size_t)o + j] = u < 0 ? -1 : idx[u];
        }
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n + 4; i += stride) {
        const double4 p = D.pts[i];
        vxyz[3 * (size_t)i] = p.x;
        vxyz[3 * (size_t)i + 1] = p.y;
        vxyz[3 * (size_t)i + 2] = p.z;
    }
}

// ---------------------------------------------------------------------------
// workspace layout

struct Carve {
    unsigned char *base;
    size_t off, cap;
    template <class T>
    T *take(size_t n) {
        off = (off + 255) & ~(size_t)255;
        T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
        off += n * sizeof(T);
        return p;
    }
};

constexpr int BBOX_BLOCKS = 256;
constexpr int SCRATCH_WARPS = 148 * 16;

struct Layout {
    Dev D;
    int *flag, *idx, *total;
    unsigned long long *bad;
};

Layout carve(Carve &c, int n, int cap) {
    Layout L{};
    Dev &D = L.D;
    D.n = n;
    D.cap = cap;
    D.pts = c.take<double4>((size_t)n + 4);
    D.tv = c.take<int4>(cap);
    D.tn = c.take<int4>(cap);
    D.own = c.take<unsigned long long>(cap);
    D.nom = c.take<unsigned long long>(cap);
    D.kround = c.take<int>(cap);
    D.startnew = c.take<int>(cap);
    D.ptet = c.take<int>(n);
    D.noms = c.take<int>(n);
    D.wins = c.take<int>(n);
    D.reloc = c.take<int>(n);
    D.cav = c.take<Cavity>(n);
    D.list_cap = 96ll * n + (1 << 16);
    D.lists = c.take<int>((size_t)D.list_cap);
    D.scratch_warps = SCRATCH_WARPS;
    D.scratch = c.take<double>((size_t)SCRATCH_WARPS * NIF_EXACT_SCRATCH);
    D.bbox = c.take<double>(6 * BBOX_BLOCKS);
    D.st = c.take<State>(1);
    L.flag = c.take<int>(cap);
    L.idx = c.take<int>(cap);
    L.total = c.take<int>(1);
    L.bad = c.take<unsigned long long>(4);
    return L;
}

int rc_of(cudaError_t e) { return e == cudaSuccess ? NIF_OK : NIF_ERR_CUDA; }

}  // namespace dt
}  // namespace nif

using namespace nif::dt;

NIF_EXPORT int nif_delaunay_max_tets(int n, int *cap) {
    if (!cap || n < 1 || n > (1 << 26)) return NIF_ERR_ARG;
    // a Delaunay tetrahedralization of n points has about 6.7 n tets for
    // uniform data; slots also hold the round's unused cavity slots
    const long long c = 8ll * n + 4096;
    if (c > (1ll << 29) - 1) return NIF_ERR_ARG;
    *cap = (int)c;
    return NIF_OK;
}

NIF_EXPORT int nif_delaunay_workspace_bytes(int n, size_t *bytes) {
    int cap = 0;
    if (!bytes || nif_delaunay_max_tets(n, &cap) != NIF_OK) return NIF_ERR_ARG;
    Carve c{nullptr, 0, (size_t)-1};
    carve(c, n, cap);
    *bytes = (c.off + 255) & ~(size_t)255;
    return NIF_OK;
}

NIF_EXPORT int nif_delaunay_build(const double *d_keys, int n, void *d_ws, size_t ws_bytes,
                                  double *d_vxyz, int32_t *d_tet_v, int32_t *d_tet_n, int tet_cap,
                                  void *stream, nif_delaunay_info *info) {
    int cap = 0;
    if (!d_keys || !d_ws || !d_vxyz || !d_tet_v || !d_tet_n || !info) return NIF_ERR_ARG;
    if (nif_delaunay_max_tets(n, &cap) != NIF_OK || tet_cap < cap) return NIF_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(d_ws) % 256 != 0) return NIF_ERR_ARG;
    size_t need = 0;
    nif_delaunay_workspace_bytes(n, &need);
    if (ws_bytes < need) return NIF_ERR_WORKSPACE;
    memset(info, 0, sizeof(*info));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Carve c{static_cast<unsigned char *>(d_ws), 0, ws_bytes};
    Layout L = carve(c, n, cap);
    Dev &D = L.D;
    int rc;
#define DT_CHECK(x)                      \
    do {                                 \
        if ((rc = rc_of(x)) != NIF_OK) { \
            return rc;                   \
        }                                \
    } while (0)
    DT_CHECK(cudaMemsetAsync(D.st, 0, sizeof(State), st));
    DT_CHECK(cudaMemsetAsync(D.own, 0xff, sizeof(unsigned long long) * cap, st));
    DT_CHECK(cudaMemsetAsync(D.nom, 0xff, sizeof(unsigned long long) * cap, st));
    DT_CHECK(cudaMemsetAsync(D.kround, 0xff, sizeof(int) * cap, st));
    DT_CHECK(cudaMemsetAsync(L.bad, 0, sizeof(unsigned long long) * 4, st));
    const int pblocks = (int)std::min<long long>(148ll * 8, (n + 255) / 256);
    const int wblocks = 148 * 4;  // 16 warps per SM: SCRATCH_WARPS in all
    k_load_keys<<<pblocks, 256, 0, st>>>(D, d_keys);
    k_bbox<<<BBOX_BLOCKS, 256, 0, st>>>(d_keys, n, D.bbox);
    k_init<<<1, 32, 0, st>>>(D, d_keys, BBOX_BLOCKS);
    k_check_inside<<<wblocks, THREADS, 0, st>>>(D);
    DT_CHECK(cudaGetLastError());
    const size_t ins_smem = WARPS * sizeof(InsWS);
    DT_CHECK(cudaFuncSetAttribute(k_insert, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ins_smem));
    State h{};
    DT_CHECK(cudaMemcpyAsync(&h, D.st, sizeof(State), cudaMemcpyDeviceToHost, st));
    DT_CHECK(cudaStreamSynchronize(st));
    int round = 0;
    while (h.err == ERR_NONE && h.inserted < n) {
        if (++round > ROUND_LIMIT) {
            h.err = ERR_CAPACITY;
            break;
        }
        // clear the round's counters (nnom, nwin, nreloc, listtop, deferred)
        DT_CHECK(cudaMemsetAsync(&D.st->nnom, 0, 3 * sizeof(int), st));
        DT_CHECK(cudaMemsetAsync(&D.st->listtop, 0, sizeof(long long), st));
        DT_CHECK(cudaMemsetAsync(&D.st->deferred, 0, sizeof(int), st));
        k_nominate<<<pblocks, 256, 0, st>>>(D, round);
        k_collect<<<pblocks, 256, 0, st>>>(D, round);
        k_cavity<<<wblocks, THREADS, 0, st>>>(D, round);
        k_check<<<pblocks, 256, 0, st>>>(D, round);
        k_insert<<<wblocks, THREADS, ins_smem, st>>>(D, round);
        k_reloc_collect<<<pblocks, 256, 0, st>>>(D, round);
        k_relocate<<<wblocks, THREADS, 0, st>>>(D);
        DT_CHECK(cudaGetLastError());
        DT_CHECK(cudaMemcpyAsync(&h, D.st, sizeof(State), cudaMemcpyDeviceToHost, st));
        DT_CHECK(cudaStreamSynchronize(st));
        if (h.err == ERR_NONE && h.nwin == 0 && h.inserted < n) h.err = ERR_CAPACITY;
    }
    info->rounds = round;
    info->max_cavity = h.max_cav;
    info->exact_evaluations = (int64_t)h.exact_evals;
    info->tet_slots = h.tet_top;
    info->error = h.err;
    if (h.err == ERR_DEGENERATE || h.err == ERR_OUTSIDE) return NIF_ERR_DEGENERATE;
    if (h.err == ERR_CAPACITY) return NIF_ERR_CAPACITY;
    if (h.err == ERR_WALK) return NIF_ERR_WALK;
    if (h.err != ERR_NONE) return NIF_ERR_INTERNAL;
    k_verify<<<wblocks, THREADS, 0, st>>>(D, L.bad);
    k_alive<<<pblocks, 256, 0, st>>>(D, L.flag);
    k_scan_single<<<1, 1024, 0, st>>>(L.flag, h.tet_top, L.idx, L.total);
    k_emit<<<pblocks, 256, 0, st>>>(D, L.flag, L.idx, d_vxyz, d_tet_v, d_tet_n);
    DT_CHECK(cudaGetLastError());
    unsigned long long bad[4];
    int total = 0;
    DT_CHECK(cudaMemcpyAsync(bad, L.bad, sizeof(bad), cudaMemcpyDeviceToHost, st));
    DT_CHECK(cudaMemcpyAsync(&total, L.total, sizeof(int), cudaMemcpyDeviceToHost, st));
    DT_CHECK(cudaMemcpyAsync(&h, D.st, sizeof(State), cudaMemcpyDeviceToHost, st));
    DT_CHECK(cudaStreamSynchronize(st));
#undef DT_CHECK
    info->n_tets = total;
    info->exact_evaluations = (int64_t)h.exact_evals;
    info->bad_orientation = (int64_t)bad[0];
    info->bad_adjacency = (int64_t)bad[1];
    info->non_delaunay_faces = (int64_t)bad[2];
    info->cospherical_faces = (int64_t)bad[3];
    if (bad[3]) return NIF_ERR_DEGENERATE;
    if (bad[0] || bad[1] || bad[2]) return NIF_ERR_INTERNAL;
    return NIF_OK;
}

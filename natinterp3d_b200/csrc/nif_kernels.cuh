// Device-side Sibson (natural-neighbour) query: one cooperative group of G
// lanes per query.
//
// Per query (natinterp3d's getWeightsSingleQueryIF, natural_insertionfree.c:591-738):
//   1. locate   seed tet = the tet whose centroid is nearest to the query, as
//               natinterp3d's k-d tree returns it (delaunay.c:392-395), found in
//               a uniform grid of centroids (an octree where the grid is too
//               coarse); then
//               natinterp3d's visibility walk (delaunay.c:398-405), the four
//               face tests of a step on 4 lanes
//   2. cavity   the connected set of tets whose circumsphere strictly contains
//               the query (inspherefast > 0, natural_insertionfree.c:502-530),
//               found breadth-first with all lanes testing in parallel; a
//               single-lane integer replay then recovers natinterp3d's LIFO
//               visiting order, which fixes the column order and the
//               floating-point summation order of every weight
//   3. boundary faces and natural neighbours in first-seen order (:559-584)
//   4. signed Voronoi-subcell volumes: +cavity-tet terms (:642-676) and
//      -virtual-tet terms (:681-719), one term per lane, folded into each
//      neighbour's sum in natinterp3d's accumulation order
//   5. normalisation (:721-737)
// Tet circumcentres and face circumcentres are read from the per-mesh cache
// (computed with the same formulas and argument orders); a face shared by two
// cavity tets uses the circumcentre computed from the tet natinterp3d visits
// first, as natinterp3d's face cache does (:233-253).
//
// Predicates.  natinterp3d evaluates orient3dfast / inspherefast and uses their
// signs as they come (predicates.c:1687, 3301); that is the default here
// (PRED_FAST).  Two more modes per mesh: PRED_AUDIT keeps those signs and
// counts every evaluation whose fast value the static error bound cannot
// certify ("uncertain"), and those whose decision the exact sign would change
// ("flipped"); PRED_EXACT decides by the exact sign.  The row routine comes in
// three variants: PM_PLAIN (fast signs only), PM_FILTER (fast kernel of the
// non-default modes: certified signs only, the row is handed to the
// large-row kernel at the first uncertain evaluation that matters) and
// PM_RESOLVE (large-row kernel: uncertain evaluations are resolved exactly,
// one lane at a time, in a per-group global scratch, and counted).
#pragma once
#include <limits.h>
#include <stddef.h>
#include <stdint.h>

#include "nif_exact.h"
#include "nif_geometry.cuh"

namespace nif {

// per-row status codes (stored as int8)
constexpr int ST_OK = 0;
constexpr int ST_WALK = 1;       // walk step limit
constexpr int ST_CAPACITY = 2;   // per-query capacity of this kernel exceeded
constexpr int ST_UNCERTAIN = 4;  // a predicate needs exact evaluation (PM_FILTER only)

// predicate modes of a mesh (MeshView::pmode)
constexpr int PRED_FAST = 0;
constexpr int PRED_AUDIT = 1;
constexpr int PRED_EXACT = 2;

// row-routine variants
constexpr int PM_PLAIN = 0;
constexpr int PM_FILTER = 1;
constexpr int PM_RESOLVE = 2;

constexpr int WALK_LIMIT = 1 << 16;
constexpr int SEED_STEP_LIMIT = 1 << 16;  // node and leaf visits of one nearest-centroid search
constexpr int OCT_BITS = 20;              // centroid code: cell bits per axis
constexpr int OCT_KMAX = 10;              // octree node levels below the root (6 code bits each)
constexpr int OCT_SPLIT = 128;            // a node with more centroids than this has children

struct __align__(32) d4 {
    double x, y, z, w;
};

// Resident mesh (device pointers) and its parameters, passed by value.
struct MeshView {
    const d4 *__restrict__ vtx;        // [nv] x, y, z, 0
    const int4 *__restrict__ tv;       // [nt] vertex ids
    const int4 *__restrict__ tn;       // [nt] neighbour tets (-1 = none)
    const uint32_t *__restrict__ tinfo;// [nt] bit0: orient3dfast(p0..p3) > 0; bit1: that sign is
                                       // uncertain; bit2: exact orient3d(p0..p3) > 0;
                                       // bits 8+2j: mirror slot of face j
    const d4 *__restrict__ tcc;        // [nt] tet circumcentre
    const d4 *__restrict__ fcc;        // [nt*4] circumcentre of the face opposite p[i]
    // Tet centroids, (p0 + p1 + p2 + p3) / 4 per axis as natinterp3d's
    // constructor computes them for its k-d tree (delaunay.c:151-157), sorted
    // by a 60-bit Morton code of their cell in a 2^20 grid per axis over the
    // bounding box of all vertices: x, y, z and the tet id (as a double).
    // An octree over that order: node k spans the centroids of one octree
    // cell, two octree levels (64 sub-cells, one 6-bit code digit) per node
    // level.  onode[2 k] = float box lo (w: first child node, or first
    // centroid of a leaf, as int bits); onode[2 k + 1] = box hi (w: number of
    // children, or minus the centroid count of a leaf); omask[k] = the
    // digits of the children present.  Boxes are rounded outwards.
    const d4 *__restrict__ cs;
    const float4 *__restrict__ onode;
    const unsigned long long *__restrict__ omask;
    double olo[3], osc[3];             // cell of x: floor((x - olo) * osc), clamped
    double oext;                       // largest extent of the code space
    int n;                             // data vertices (ids >= n are super-simplex vertices)
    int nv, nt;
    int pmode;                         // PRED_*
    // Uniform grid over the data bounding box, gdim cells per axis (cell of x
    // along axis a: floor((x - glo) * ginv), clamped), about two centroids a
    // cell: the centroids of cell k are gitems[gstart[k] .. gstart[k + 1]),
    // x, y, z and the tet id (as a double), in no particular order.  The
    // seed search reads it first; query bucketing normalises by the same box.
    const int *__restrict__ gstart;
    const d4 *__restrict__ gitems;
    int gdim[3];
    double glo[3], ginv[3];
    double gh[3];                      // cell size, 1 / ginv
    double gext;                       // largest extent of the grid (margins)
};

__device__ __forceinline__ int comp(const int4 &v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// getFaceVerticies3 (delaunay.c:444-467): face f = (p[a], p[b], p[c]) lies
// opposite p[3-f] and is shared with neighbour s[f].
__device__ __forceinline__ int face_vslot(int f, int j) {
    constexpr unsigned bits = (0u | 1u << 2 | 2u << 4) | ((3u | 1u << 2 | 0u << 4) << 6) |
                              ((0u | 2u << 2 | 3u << 4) << 12) | ((3u | 2u << 2 | 1u << 4) << 18);
    return (bits >> (6 * f + 2 * j)) & 3;
}

__device__ __forceinline__ dv3 vload(const MeshView &M, int vid) {
    const d4 v = M.vtx[vid];
    return dv3{v.x, v.y, v.z};
}

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ dv3 cload(const d4 *p) {
    const d4 v = *p;
    return dv3{v.x, v.y, v.z};
}

// Squared distance between a tet centroid and q as natinterp3d's k-d tree
// evaluates it: dist_sq = 0; dist_sq += SQ(node->pos[i] - pos[i]) for
// i = 0, 1, 2 (kdtree.c:411-414; 0 + a == a exactly).
__device__ __forceinline__ double kd_dist2(const d4 &c, const dv3 &q) {
    const double dx = fsub(c.x, q.x), dy = fsub(c.y, q.y), dz = fsub(c.z, q.z);
    return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
}

// A lower bound of kd_dist2 over every centroid inside the box [lo, hi]:
// per axis the rounded distance to the nearer face (0 inside), squared and
// summed in the same order.  Rounding is monotonic, so no centroid in the
// box evaluates below it.
__device__ __forceinline__ double box_dist2(const float4 &lo, const float4 &hi, const dv3 &q) {
    auto axis = [](double x, float l, float h) {
        return x < (double)l ? fsub((double)l, x) : (x > (double)h ? fsub(x, (double)h) : 0.0);
    };
    const double ax = axis(q.x, lo.x, hi.x), ay = axis(q.y, lo.y, hi.y), az = axis(q.z, lo.z, hi.z);
    return fadd(fadd(fmul(ax, ax), fmul(ay, ay)), fmul(az, az));
}

// Lane helpers for a group of G consecutive lanes of a warp.
template <int G>
struct Grp {
    unsigned mask;  // warp-lane mask of the group
    int lane;       // lane within the group
    int base;       // first warp lane of the group
    __device__ __forceinline__ Grp() {
        const int wl = threadIdx.x & 31;
        lane = wl % G;
        base = wl - lane;
        mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << base);
    }
    __device__ __forceinline__ unsigned local(unsigned m) const {
        return (G == 32) ? m : ((m >> base) & ((1u << G) - 1u));
    }
    __device__ __forceinline__ unsigned ballot(bool p) const { return local(__ballot_sync(mask, p)); }
    __device__ __forceinline__ bool any(bool p) const { return __any_sync(mask, p); }
    __device__ __forceinline__ unsigned lt() const { return (1u << lane) - 1u; }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ unsigned match(int v) const { return local(__match_any_sync(mask, v)); }
    __device__ __forceinline__ int shfl(int v, int src) const { return __shfl_sync(mask, v, src, G); }
    __device__ __forceinline__ double shfl(double v, int src) const {
        return __shfl_sync(mask, v, src, G);
    }
    __device__ __forceinline__ int shfl_xor(int v, int off) const {
        return __shfl_xor_sync(mask, v, off, G);
    }
    __device__ __forceinline__ double shfl_xor_d(double v, int off) const {
        return __shfl_xor_sync(mask, v, off, G);
    }
};

__device__ __forceinline__ unsigned long long spread3_64(unsigned v) {  // 20 bits -> every third bit
    unsigned long long x = v & 0xfffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

// cell coordinates (clamped) and 60-bit Morton code of a point in the
// centroid code space
__device__ __forceinline__ unsigned long long oct_code(const MeshView &M, const dv3 &p, int ix[3]) {
    const double c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double f = (c[a] - M.olo[a]) * M.osc[a];
        ix[a] = f > 0.0 ? (f < (double)((1 << OCT_BITS) - 1) ? (int)f : (1 << OCT_BITS) - 1) : 0;
    }
    return spread3_64(ix[0]) | (spread3_64(ix[1]) << 1) | (spread3_64(ix[2]) << 2);
}

// True when every point within sqrt(best) of q lies inside q's octree cell
// at octree level 2 m (margins absorb the rounding of the cell bounds and of
// the centroids' own cell assignment).
__device__ __forceinline__ bool ball_in_cell(const MeshView &M, const dv3 &q, double best,
                                             const int ix[3], int m) {
    if (!(best < INFINITY)) return false;
    const double r = sqrt(best) * (1.0 + 1e-9) + 1e-9 * M.oext;
    const double c[3] = {q.x, q.y, q.z};
    const int sh = OCT_BITS - 2 * m;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double w = (double)(1 << sh) / M.osc[a];
        const double lo = M.olo[a] + (double)(ix[a] >> sh) * w;
        if (!(c[a] - r > lo && c[a] + r < lo + w)) return false;
    }
    return true;
}

// The tet whose centroid is nearest to q under kd_dist2, ties to the lowest
// tet id: the seed natinterp3d's k-d tree returns (kd_nearest3_data,
// kdtree.c:543-564).  Its pruning never skips a strictly nearer centroid, so
// it returns a minimiser of the same rounded distance; among exactly equal
// distances its visiting order decides, here the lowest id.
// Bottom-up over the octree, one lane per child (two per lane for 64):
//   1. descend along q's own code to the deepest node holding q's cell;
//   2. search that node's subtree;
//   3. walk back up: stop as soon as the ball of radius sqrt(best) around q
//      lies inside the cell just searched (octree cells are disjoint, so no
//      other centroid can be nearer); otherwise search the parent's other
//      children.
// A subtree search is depth-first, entering a child while its box bound is
// <= best (an equal distance may still lose to a lower id).  stk: 64 ints of
// group scratch (the descent path and the search frames); every lane keeps
// the same control state and lane 0 stores it.  Bounded by SEED_STEP_LIMIT
// visits (then the best centroid so far, a valid seed for the walk).
template <int G>
__device__ int nearest_centroid(const MeshView &M, const dv3 q, const Grp<G> &g, int *stk) {
    static_assert(G == 32, "two children of a 64-wide node per lane");
    int *path = stk;        // [OCT_KMAX + 1]
    int *frm = stk + 16;    // 3 ints a frame: node, pending children (lo, hi word)
    int ix[3];
    const unsigned long long code = oct_code(M, q, ix);
    int node = 0, depth = 0;
    if (g.lane == 0) path[0] = 0;
    for (; depth < OCT_KMAX; depth++) {
        const int nch = __float_as_int(M.onode[2 * node + 1].w);
        if (nch <= 0) break;
        const unsigned long long mask = M.omask[node];
        const int dg = (int)((code >> (6 * (OCT_KMAX - 1 - depth))) & 63ull);
        if (!((mask >> dg) & 1ull)) break;
        node = __float_as_int(M.onode[2 * node].w) + __popcll(mask & ((1ull << dg) - 1ull));
        if (g.lane == 0) path[depth + 1] = node;
    }
    g.sync();
    double best = INFINITY;
    int bid = INT_MAX;
    int steps = 0;
    // centroids [a, a + n) of a leaf
    auto leaf_pass = [&](int a, int n) {
        for (int k0 = a; k0 < a + n; k0 += G) {
            const int k = k0 + g.lane;
            double d = INFINITY;
            int id = INT_MAX;
            if (k < a + n) {
                const d4 e = M.cs[k];
                d = kd_dist2(e, q);
                id = (int)e.w;
            }
            const bool better = d < best || (d == best && id < bid);
            if (g.any(better)) {
                double bd = better ? d : best;
                int bi = better ? id : bid;
#pragma unroll
                for (int off = G / 2; off > 0; off >>= 1) {
                    const double od = g.shfl_xor_d(bd, off);
                    const int oi = g.shfl_xor(bi, off);
                    if (od < bd || (od == bd && oi < bi)) {
                        bd = od;
                        bi = oi;
                    }
                }
                best = bd;
                bid = bi;
            }
        }
    };
    // every centroid under node r, except under its child `skip`
    auto subtree = [&](int r, int skip) {
        {
            const float4 lo = M.onode[2 * r], hi = M.onode[2 * r + 1];
            if (__float_as_int(hi.w) <= 0) {
                ++steps;
                leaf_pass(__float_as_int(lo.w), -__float_as_int(hi.w));
                return;
            }
        }
        int sp = 1;
        if (g.lane == 0) frm[0] = r;
        bool fresh = true;
        unsigned long long pend = 0;
        while (sp > 0 && steps < SEED_STEP_LIMIT) {
            ++steps;
            g.sync();
            const int nd = frm[3 * (sp - 1)];
            if (!fresh)
                pend = (unsigned long long)(unsigned)frm[3 * (sp - 1) + 1] |
                       ((unsigned long long)(unsigned)frm[3 * (sp - 1) + 2] << 32);
            const int first = __float_as_int(M.onode[2 * nd].w);
            const int nch = __float_as_int(M.onode[2 * nd + 1].w);
            // box bounds of the children lane and lane + 32
            double d0 = INFINITY, d1 = INFINITY;
            const int c0 = first + g.lane, c1 = first + 32 + g.lane;
            if (g.lane < nch && c0 != skip) d0 = box_dist2(M.onode[2 * c0], M.onode[2 * c0 + 1], q);
            if (32 + g.lane < nch && c1 != skip) d1 = box_dist2(M.onode[2 * c1], M.onode[2 * c1 + 1], q);
            auto within = [&]() {
                return (unsigned long long)g.ballot(d0 <= best) |
                       ((unsigned long long)g.ballot(d1 <= best) << 32);
            };
            pend = fresh ? within() : (pend & within());
            fresh = false;
            bool pushed = false;
            while (pend && steps < SEED_STEP_LIMIT) {
                const int c = __ffsll((long long)pend) - 1;
                pend &= pend - 1ull;
                const int ch = first + c;
                const float4 clo = M.onode[2 * ch], chi = M.onode[2 * ch + 1];
                ++steps;
                if (__float_as_int(chi.w) <= 0) {
                    leaf_pass(__float_as_int(clo.w), -__float_as_int(chi.w));
                    pend &= within();  // the same children, against the improved best
                } else {
                    if (g.lane == 0) {
                        frm[3 * (sp - 1) + 1] = (int)(unsigned)pend;
                        frm[3 * (sp - 1) + 2] = (int)(unsigned)(pend >> 32);
                        frm[3 * sp] = ch;
                    }
                    ++sp;
                    fresh = true;
                    pushed = true;
                    break;
                }
            }
            if (!pushed) --sp;
        }
        g.sync();
    };
    subtree(node, -1);
    for (int l = depth - 1; l >= 0; l--) {
        if (ball_in_cell(M, q, best, ix, l + 1)) break;
        subtree(path[l], path[l + 1]);
    }
    return bid == INT_MAX ? 0 : bid;
}

constexpr int GRID_DENSE = 256;  // centroids in a search block beyond which the octree searches
constexpr int GRID_RMAX = 3;     // largest block radius (cells) the grid search widens to

// The nearest tet centroid to q (same distance and ties as nearest_centroid)
// from the uniform grid: the centroids of the cells within Chebyshev radius
// r of q's cell, one lane per cell, r = 1 first; done once the best distance
// is below the distance from q to the searched block's open sides (sides on
// the grid's boundary are closed: centroids beyond them are clamped into the
// boundary cells, which have been searched).  Returns -1 where the block
// holds more than GRID_DENSE centroids or r would exceed GRID_RMAX: the
// octree search takes over there (clustered data, far-away queries).
template <int G>
__device__ int grid_nearest(const MeshView &M, const dv3 q) {
    static_assert(G == 32, "one lane per cell of a 3x3x3 block");
    const double c[3] = {q.x, q.y, q.z};
    double f[3];  // q's position in cell units
    int ic[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        f[a] = (c[a] - M.glo[a]) * M.ginv[a];
        ic[a] = f[a] > 0.0 ? (f[a] < (double)(M.gdim[a] - 1) ? (int)f[a] : M.gdim[a] - 1) : 0;
    }
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    double best = INFINITY;
    int bid = INT_MAX;
    for (int r = 1; r <= GRID_RMAX; r++) {
        const int w = 2 * r + 1, ncell = w * w * w;
        // this round's cells: the 27 of the 3x3x3 block, then the shell at
        // Chebyshev radius r
        int total = 0;
        for (int k0 = 0; k0 < ncell; k0 += 32) {
            const int k = k0 + lane;
            int a = 0, b = 0;
            int dx, dy, dz;
            bool take;
            if (r == 1) {
                dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
                take = lane < 27;
            } else {
                dx = k % w - r, dy = (k / w) % w - r, dz = k / (w * w) - r;
                take = k < ncell && max(abs(dx), max(abs(dy), abs(dz))) == r;
            }
            const int x = ic[0] + dx, y = ic[1] + dy, z = ic[2] + dz;
            if (take && x >= 0 && y >= 0 && z >= 0 && x < M.gdim[0] && y < M.gdim[1] && z < M.gdim[2]) {
                const int cell = (z * M.gdim[1] + y) * M.gdim[0] + x;
                a = M.gstart[cell];
                b = M.gstart[cell + 1];
            }
            total += __reduce_add_sync(full, b - a);
            if (total > GRID_DENSE) return -1;
            for (int i = a; i < b; i++) {
                const d4 e = M.gitems[i];
                const double d = kd_dist2(e, q);
                const int id = (int)e.w;
                if (d < best || (d == best && id < bid)) {
                    best = d;
                    bid = id;
                }
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double od = __shfl_xor_sync(full, best, off);
            const int oi = __shfl_xor_sync(full, bid, off);
            if (od < best || (od == best && oi < bid)) {
                best = od;
                bid = oi;
            }
        }
        // distance from q to the block's open sides (not on the grid's boundary)
        double lb = INFINITY;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (ic[a] - r > 0) lb = fmin(lb, (f[a] - (double)(ic[a] - r)) * M.gh[a]);
            if (ic[a] + r < M.gdim[a] - 1) lb = fmin(lb, ((double)(ic[a] + r + 1) - f[a]) * M.gh[a]);
        }
        if (lb == INFINITY) return bid == INT_MAX ? -1 : bid;  // the block covers the grid
        const double m = lb - 1e-9 * M.gext;
        if (bid != INT_MAX && m > 0.0 && best < m * m * (1.0 - 1e-12)) return bid;
    }
    return -1;
}

// Per-group scratch.  The first union member is live during the cavity
// search, the second only during the single-lane replay of natinterp3d's
// visiting order.  Index types are the narrowest that hold each capacity.
template <int HS_, int CAV_, int BF_, int NBR_, int VH_, int G_, class SlotT, class CavT>
struct Workspace {
    static constexpr int HS = HS_;        // tested-tet hash slots (power of two)
    static constexpr int QCAP = HS_ * 3 / 4;
    static constexpr int CAV = CAV_;      // cavity tets
    static constexpr int STACK = 4 * CAV_ + 1;
    static constexpr int BF = BF_;        // boundary faces
    static constexpr int NBR = NBR_;      // natural neighbours
    static constexpr int VH = VH_;        // neighbour hash slots (power of two)
    static constexpr int G = G_;
    using slot_t = SlotT;                 // tested-tet hash slot index
    using cav_t = CavT;                   // signed cavity index
    union U {
        struct {
            int hkey[HS_];
            CavT hval[HS_];
            SlotT queue[HS_ * 3 / 4];
        } a;
        struct {
            CavT stack[4 * CAV_ + 1];
        } r;
    } u;
    double acc[NBR_];            // stolen volume per neighbour
    int cav_tet[CAV_];
    int nbr_vid[NBR_];
    int vh_key[VH_];
    int vh_first[VH_];
    alignas(4) CavT cav_nbr[4 * CAV_];  // cavity index of neighbour f of cavity tet c, -1 outside
    CavT order[CAV_];            // cavity tets in natinterp3d's visiting order
    CavT pos[CAV_];              // inverse of order
    uint16_t bface[BF_];         // (cavity index << 2) | face
    int16_t vh_slot[VH_];
};

// Workspaces of the split row (k_rows_cavity, then k_rows_volume): the same
// member names as Workspace, each holding only what its phase uses.
template <int HS_, int CAV_, int G_, class SlotT, class CavT>
struct CavWorkspace {
    static constexpr int HS = HS_;
    static constexpr int QCAP = HS_ * 3 / 4;
    static constexpr int CAV = CAV_;
    static constexpr int STACK = 4 * CAV_ + 1;
    static constexpr int G = G_;
    using slot_t = SlotT;
    using cav_t = CavT;
    union U {
        struct {
            int hkey[HS_];
            CavT hval[HS_];
            SlotT queue[HS_ * 3 / 4];
        } a;
        struct {
            CavT stack[4 * CAV_ + 1];
        } r;
    } u;
    int cav_tet[CAV_];
    alignas(4) CavT cav_nbr[4 * CAV_];
    CavT order[CAV_];
    CavT pos[CAV_];
};

template <int CAV_, int BF_, int NBR_, int VH_, int G_>
struct VolWorkspace {
    static constexpr int CAV = CAV_;
    static constexpr int BF = BF_;
    static constexpr int NBR = NBR_;
    static constexpr int VH = VH_;
    static constexpr int G = G_;
    union U {
        double buf[4 * G_ * 10 / 8];  // the fold's item buffer (4 G terms + slots); sink staging
    } u;
    double acc[NBR_];
    int4 ctv[CAV_];     // vertex record of the o-th visited cavity tet
    int4 cfp[CAV_];     // fcc[] indices of its faces (natinterp3d's face cache)
    int cav_tet[CAV_];  // cavity tets in visiting order
    int ftet[CAV_];     // cavity tets in the flood's order (the record's)
    int8_t fpos[CAV_];  // visiting position of the e-th record entry
    int nbr_vid[NBR_];
    int vh_key[VH_];
    int vh_first[VH_];
    uint16_t bface[BF_];
    int16_t vh_slot[VH_];
    uint8_t bmask[CAV_];  // boundary faces of each cavity tet, one bit per face
};

// One row between k_rows_cavity, k_rows_order and k_rows_volume: a header
// and, per cavity tet in the flood's order, the tet, which of its faces bound
// the cavity (bits 0-3) and the mirror slots of its faces (bits 8-15, the
// mesh's tinfo bits 8-15), the cavity indices of its four neighbours (four
// signed bytes, -1 outside the cavity); k_rows_order adds the tet's position
// in natinterp3d's visiting order, from which k_rows_volume derives the fcc[]
// indices of its faces' circumcentres as natinterp3d's face cache returns them.
constexpr int REC_CAV = 48;  // cavity tets a record holds (larger cavities take the large kernel)
constexpr int RS_OK = 0, RS_OUTSIDE = 1, RS_WALK = 2, RS_QUEUED = 3;
struct __align__(16) RowHead {
    int ncav;   // cavity tets (0: the coincident-vertex row)
    int start;  // located tet
    int state;  // RS_*
    int pad;
};
struct __align__(16) RowEntry {
    int tet;
    unsigned bmask;  // boundary faces | mirror slots << 8
    int nbr;         // cavity indices of neighbours 0..3, one signed byte each
    int pos;         // position in natinterp3d's visiting order (bits 0-7); bit 8 + i: face
                     // 3 - i takes the copy of the neighbour visited earlier
};
static_assert(sizeof(RowEntry) == 16, "RowEntry is one 16-byte load");

__device__ __forceinline__ unsigned mix_hash(int key) {
    return (unsigned)key * 2654435761u;
}

// Inserts key; returns its slot, whether newly inserted (fresh = true) or
// already present.  Returns -1 and sets full when every slot was probed.
__device__ __forceinline__ int hash_insert(int *keys, int hs, int key, bool &fresh, bool &full) {
    unsigned h = mix_hash(key) & (unsigned)(hs - 1);
#pragma unroll 1
    for (int probe = 0; probe < hs; ++probe) {
        const int old = atomicCAS(&keys[h], -1, key);
        if (old == -1) {
            fresh = true;
            return (int)h;
        }
        if (old == key) return (int)h;
        h = (h + 1) & (unsigned)(hs - 1);
    }
    full = true;
    return -1;
}

// Slot of key (inserted if absent); -1 and full=true when the table is full.
__device__ __forceinline__ int hash_upsert(int *keys, int hs, int key, bool &full) {
    unsigned h = mix_hash(key) & (unsigned)(hs - 1);
#pragma unroll 1
    for (int probe = 0; probe < hs; ++probe) {
        const int old = atomicCAS(&keys[h], -1, key);
        if (old == -1 || old == key) return (int)h;
        h = (h + 1) & (unsigned)(hs - 1);
    }
    full = true;
    return -1;
}

__device__ __forceinline__ int hash_find(const int *keys, int hs, int key) {
    unsigned h = mix_hash(key) & (unsigned)(hs - 1);
#pragma unroll 1
    for (int probe = 0; probe < hs; ++probe) {
        const int k = keys[h];
        if (k == key) return (int)h;
        if (k == -1) return -1;
        h = (h + 1) & (unsigned)(hs - 1);
    }
    return -1;
}

struct RowInfo {
    int status;
    int nnb;
    int steps;
    bool outside;
    bool coincident;  // row from the coincident-vertex path
    double total;     // sum of the stolen volumes (the normaliser), 0 if none
    int nbf;          // boundary faces (ws.bface[0..nbf))
    // PM_RESOLVE only: predicate evaluations natinterp3d performs for this row
    // that the filter could not certify, and those whose decision the exact
    // sign changes (walk orientation tests / cavity in-sphere tests)
    int o_unc, o_flip, i_unc, i_flip;
};

// ---- predicate filters and exact resolution ---------------------------------
__device__ __forceinline__ void to3(const dv3 &v, double *o) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
}

__device__ __forceinline__ int sgn(double x) { return (x > 0.0) - (x < 0.0); }

__device__ __forceinline__ bool orient_uncertain(const dv3 &a, const dv3 &b, const dv3 &c,
                                                 const dv3 &d, double fast) {
    double pa[3], pb[3], pc[3], pd[3];
    to3(a, pa), to3(b, pb), to3(c, pc), to3(d, pd);
    return nif_orient_uncertain(fast, nif_orient_permanent(pa, pb, pc, pd));
}

__device__ __forceinline__ bool insphere_uncertain(const dv3 &a, const dv3 &b, const dv3 &c,
                                                   const dv3 &d, const dv3 &e, double fast) {
    double pa[3], pb[3], pc[3], pd[3], pe[3];
    to3(a, pa), to3(b, pb), to3(c, pc), to3(d, pd), to3(e, pe);
    return nif_insphere_uncertain(fast, nif_insphere_permanent(pa, pb, pc, pd, pe));
}

// Exact orient3d signs for the lanes with unc set, one lane at a time in the
// shared scratch xs (NIF_EXACT_SCRATCH doubles); other lanes keep s.
template <int G>
__device__ __forceinline__ int resolve_orient(const Grp<G> &g, double *xs, bool unc, const dv3 &a,
                                              const dv3 &b, const dv3 &c, const dv3 &d, int s) {
    unsigned um = g.ballot(unc);
    while (um) {
        const int l = __ffs(um) - 1;
        um &= um - 1u;
        if (g.lane == l) {
            double pa[3], pb[3], pc[3], pd[3];
            to3(a, pa), to3(b, pb), to3(c, pc), to3(d, pd);
            s = nif_orient_exact_sign(pa, pb, pc, pd, xs);
        }
        g.sync();
    }
    return s;
}

template <int G>
__device__ __forceinline__ int resolve_insphere(const Grp<G> &g, double *xs, bool unc, const dv3 &a,
                                                const dv3 &b, const dv3 &c, const dv3 &d,
                                                const dv3 &e, int s) {
    unsigned um = g.ballot(unc);
    while (um) {
        const int l = __ffs(um) - 1;
        um &= um - 1u;
        if (g.lane == l) {
            double pa[3], pb[3], pc[3], pd[3], pe[3];
            to3(a, pa), to3(b, pb), to3(c, pc), to3(d, pd), to3(e, pe);
            s = nif_insphere_exact_sign(pa, pb, pc, pd, pe, xs);
        }
        g.sync();
    }
    return s;
}

// PRED_EXACT, query exactly on a face or edge of its located tet: the cavity
// index of the lowest-id cavity tet whose closure contains q (exact signs),
// from which the visiting order is replayed -- the order then no longer
// depends on which of the containing tets the walk reached.
template <int G, class W>
__device__ int canonical_start(const MeshView &M, const W &ws, const Grp<G> &g, double *xs,
                               const dv3 q, int ncav) {
    int best_t = INT_MAX, best_c = 0;
    for (int c0 = 0; c0 < ncav; c0 += G) {
        const int c = c0 + g.lane;
        bool alive = c < ncav;
        const int tt = alive ? ws.cav_tet[c] : 0;
        const int4 p = M.tv[tt];
        for (int f = 0; f < 4; f++) {
            dv3 v1{0.0, 0.0, 0.0}, v2 = v1, v3 = v1;
            int s = 1;
            bool unc = false;
            if (alive) {
                v1 = vload(M, comp(p, face_vslot(f, 0)));
                v2 = vload(M, comp(p, face_vslot(f, 1)));
                v3 = vload(M, comp(p, face_vslot(f, 2)));
                const double o = orient_fast(v1, v2, v3, q);
                s = sgn(o);
                unc = orient_uncertain(v1, v2, v3, q, o);
            }
            s = resolve_orient(g, xs, unc, v1, v2, v3, q, s);
            if (s < 0) alive = false;
        }
        if (alive && tt < best_t) {
            best_t = tt;
            best_c = c;
        }
    }
    for (int off = G / 2; off > 0; off >>= 1) {
        const int ot = g.shfl_xor(best_t, off), oc = g.shfl_xor(best_c, off);
        if (ot < best_t) {
            best_t = ot;
            best_c = oc;
        }
    }
    return best_c;
}

// slot of a data vertex among the natural neighbours, -1 if it is not one
template <class W>
__device__ __forceinline__ int neighbour_slot(const W &ws, int v) {
    const int s = hash_find(ws.vh_key, W::VH, v);
    return s >= 0 ? ws.vh_slot[s] : -1;
}

// Point location (natinterp3d's findContainingSimplex, delaunay.c:383-407):
// the seed is the nearest tet centroid, then natinterp3d's visibility walk.
// Returns the located tet; r.status / r.outside report a walk that hit its
// step limit or left the super-simplex, r.steps counts the steps.  scratch:
// 64 ints of group scratch (the octree search's).  PM selects the predicate
// variant as in sibson_row; *on_face is set in PM_RESOLVE / PRED_EXACT when a
// face test of the located tet is exactly zero.
template <int G, int PM>
__device__ int locate(const MeshView &M, const dv3 q, const Grp<G> &g, int *scratch, RowInfo &r,
                      bool &on_face, double *xs = nullptr) {
    const bool filt = PM != PM_PLAIN && M.pmode != PRED_FAST;
    int t = grid_nearest<G>(M, q);
    if (t < 0) t = nearest_centroid<G>(M, q, g, scratch);
    for (;;) {
        if (r.steps >= WALK_LIMIT) {
            r.status = ST_WALK;
            return t;
        }
        ++r.steps;
        const int4 p = M.tv[t];
        const int4 nbs = M.tn[t];  // loaded with p: no second dependent trip per step
        int sg = 1;
        bool unc = false;
        dv3 v1{0.0, 0.0, 0.0}, v2 = v1, v3 = v1;
        if (g.lane < 4) {
            const int f = g.lane;
            v1 = vload(M, comp(p, face_vslot(f, 0)));
            v2 = vload(M, comp(p, face_vslot(f, 1)));
            v3 = vload(M, comp(p, face_vslot(f, 2)));
            const double o = orient_fast(v1, v2, v3, q);
            sg = sgn(o);
            if (filt) unc = orient_uncertain(v1, v2, v3, q, o);
        }
        unsigned m;
        if constexpr (PM == PM_PLAIN) {
            m = g.ballot(sg < 0);
        } else if constexpr (PM == PM_FILTER) {
            // natinterp3d tests faces 0..3 and moves through the first negative
            // one: only uncertain tests up to that face can change the step
            m = g.ballot(!unc && sg < 0);
            const int fn = m ? __ffs(m) - 1 : 4;
            if (g.ballot(unc) & ((2u << fn) - 1u)) {
                r.status = ST_UNCERTAIN;
                return t;
            }
        } else {
            if (filt) {
                const int xsg = resolve_orient(g, xs, unc, v1, v2, v3, q, sg);
                const int use = M.pmode == PRED_EXACT ? xsg : sg;
                m = g.ballot(use < 0);
                const unsigned seen = (2u << (m ? __ffs(m) - 1 : 3)) - 1u;  // tests natinterp3d makes
                r.o_unc += __popc(g.ballot(unc) & seen);
                r.o_flip += __popc(g.ballot(unc && ((xsg < 0) != (sg < 0))) & seen);
                if (!m) on_face = g.ballot(use == 0) != 0u;
            } else {
                m = g.ballot(sg < 0);
            }
        }
        if (!m) return t;
        const int nb = comp(nbs, __ffs(m) - 1);
        if (nb < 0) {
            r.outside = true;
            return t;
        }
        t = nb;
    }
}

// Steps 2 of the row: the cavity of q around tet `start` (natinterp3d's
// findCavity, natural_insertionfree.c:486-551) by a parallel flood over the
// tested-tet hash, then natinterp3d's LIFO visiting order replayed on it.
// Returns the number of cavity tets, ws.cav_tet[c] their tets, ws.order[o]
// the cavity index of the o-th visited, ws.pos its inverse and ws.cav_nbr
// [4c + f] the cavity index of neighbour f of cavity tet c (-1 outside).  On
// overflow / an uncertain test (PM_FILTER) r.status is set; an empty cavity
// (0) leaves the order unset.  REPLAY = false stops after the flood and the
// neighbour table (the split row path replays the order in k_rows_order).
template <int G, class W, int PM, bool REPLAY = true>
__device__ int flood_replay(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g, const int start,
                            RowInfo &r, const bool on_face, double *xs) {
    using cav_t = typename W::cav_t;
    using slot_t = typename W::slot_t;
    const bool filt = PM != PM_PLAIN && M.pmode != PRED_FAST;
    // ---- 2. cavity: parallel flood over the tested-tet hash ----------------
    // While a cavity tet's four neighbours are inserted into the hash, the
    // slot of each is kept in nsl[4c+f] (aliasing cav_nbr, which is filled
    // from it after the flood).  A missing neighbour (hull face of the
    // super-simplex) gets the slot of the key NO_TET, inserted up front with
    // hval = -1 and never queued, so every face has a slot.
    static_assert(sizeof(slot_t) == sizeof(cav_t), "nsl aliases cav_nbr");
    constexpr int NO_TET = -2;
    slot_t *nsl = reinterpret_cast<slot_t *>(ws.cav_nbr);
    for (int i = g.lane; i < W::HS; i += G) {
        ws.u.a.hkey[i] = -1;
        ws.u.a.hval[i] = (cav_t)-1;
    }
    g.sync();
    int none_slot = 0;
    if (g.lane == 0) {
        const int h = (int)(mix_hash(start) & (unsigned)(W::HS - 1));
        ws.u.a.hkey[h] = start;
        ws.u.a.queue[0] = (slot_t)h;
        bool fresh = false, full = false;
        none_slot = hash_insert(ws.u.a.hkey, W::HS, NO_TET, fresh, full);
    }
    none_slot = g.shfl(none_slot, 0);
    g.sync();
    int qhead = 0, qtail = 1, ncav = 0;
    bool overflow = false;
    // With natinterp3d's signs the located tet's neighbours join its wave:
    // the flood tests them next whenever the located tet is in the cavity, in
    // this same queue order, so the cavity indices are those of a flood that
    // starts with the located tet alone, and one wave of a single lane is
    // saved.  (If the located tet is not in the cavity, their tests are
    // dropped below.)  Filtered modes keep the plain start, so that their
    // predicate counters count the same tests.
    const bool ring = !filt;
    if (ring) {
        int ns = -1;
        bool full = false;
        if (g.lane < 4) {
            const int nb = comp(M.tn[start], g.lane);
            bool fresh = false;
            if (nb >= 0) {
                const int sl = hash_insert(ws.u.a.hkey, W::HS, nb, fresh, full);
                if (fresh) ns = sl;
            }
        }
        const unsigned pm = g.ballot(ns >= 0);
        if (ns >= 0) ws.u.a.queue[qtail + __popc(pm & g.lt())] = (slot_t)ns;
        qtail += __popc(pm);
        if (g.any(full)) overflow = true;
        g.sync();
    }
    while (!overflow && qhead < qtail) {
        const int n = min(G, qtail - qhead);
        int slot = -1, tt = -1;
        bool inc = false, unc = false;
        dv3 ia{0.0, 0.0, 0.0}, ib = ia, ic = ia, id = ia;
        double sv = 0.0;
        if (g.lane < n) {
            slot = ws.u.a.queue[qhead + g.lane];
            tt = ws.u.a.hkey[slot];
            const int4 p = M.tv[tt];
            const dv3 a = vload(M, p.x), b = vload(M, p.y);
            ic = vload(M, p.z);
            id = vload(M, p.w);
            // insphere argument order fixed by the tet's orientation
            // (natural_insertionfree.c:511-515); PRED_EXACT uses the exact one
            const uint32_t info = M.tinfo[tt];
            const bool pos = (info & ((PM != PM_PLAIN && M.pmode == PRED_EXACT) ? 4u : 1u)) != 0;
            ia = pos ? a : b;
            ib = pos ? b : a;
            sv = insphere_fast(ia, ib, ic, id, q);
            inc = sv > 0;
            if (filt) unc = insphere_uncertain(ia, ib, ic, id, q, sv);
        }
        if constexpr (PM == PM_FILTER) {
            if (g.any(unc)) {
                r.status = ST_UNCERTAIN;
                return 0;
            }
        } else if constexpr (PM == PM_RESOLVE) {
            if (filt && g.any(unc)) {
                const bool xin = resolve_insphere(g, xs, unc, ia, ib, ic, id, q, inc ? 1 : -1) > 0;
                r.i_unc += __popc(g.ballot(unc));
                r.i_flip += __popc(g.ballot(unc && xin != inc));
                if (M.pmode == PRED_EXACT) inc = xin;
            }
        }
        const unsigned cm = g.ballot(inc);
        if (ring && qhead == 0 && !(cm & 1u)) break;  // the located tet is outside: empty cavity
        const int ci = ncav + __popc(cm & g.lt());
        if (g.lane < n) ws.u.a.hval[slot] = (cav_t)(inc ? ci : -1);
        if (inc && ci < W::CAV) {
            ws.cav_tet[ci] = tt;
            // the volume phase reads this tet's cached circumcentres
            prefetch_l2(&M.tcc[tt]);
            prefetch_l2(&M.fcc[4 * (size_t)tt]);
        }
        const int nnew = __popc(cm);
        const int base = ncav;
        ncav += nnew;
        qhead += n;
        if (ncav > W::CAV) {
            overflow = true;
            break;
        }
        g.sync();
        for (int k0 = 0; k0 < 4 * nnew; k0 += G) {
            const int k = k0 + g.lane;
            int ns = -1;
            bool full = false, fresh = false;
            if (k < 4 * nnew) {
                const int nb = comp(M.tn[ws.cav_tet[base + (k >> 2)]], k & 3);
                int sl = none_slot;
                if (nb >= 0) sl = hash_insert(ws.u.a.hkey, W::HS, nb, fresh, full);
                if (fresh) ns = sl;
                nsl[4 * base + k] = (slot_t)(full ? none_slot : sl);
            }
            const unsigned pm = g.ballot(ns >= 0);
            const int qi = qtail + __popc(pm & g.lt());
            if (ns >= 0 && qi < W::QCAP) ws.u.a.queue[qi] = (slot_t)ns;
            qtail += __popc(pm);
            if (g.any(full) || qtail > W::QCAP) overflow = true;
        }
        if (overflow) break;
        g.sync();
    }
    g.sync();
    if (overflow) {
        r.status = ST_CAPACITY;
        return 0;
    }
    if (ncav == 0) return 0;

    // cavity-local neighbour table: cav_nbr[4c+f] = cavity index of s[f] or -1
    // (every neighbour slot recorded by the flood has been tested by now)
    for (int k = g.lane; k < 4 * ncav; k += G) ws.cav_nbr[k] = ws.u.a.hval[nsl[k]];
    if constexpr (!REPLAY) {
        g.sync();
    } else {
        for (int c = g.lane; c < ncav; c += G) ws.pos[c] = (cav_t)-1;
        g.sync();

        // cavity index 0 is the located tet, the flood's start
        int start_c = 0;
        if constexpr (PM == PM_RESOLVE) {
            if (on_face && M.pmode == PRED_EXACT) start_c = canonical_start(M, ws, g, xs, q, ncav);
        }

        // replay natinterp3d's LIFO flood on the cavity (its non-cavity tets are
        // leaves and do not change the order in which cavity tets are reached)
        if (g.lane == 0) {
            cav_t *stack = ws.u.r.stack;
            int sp = 0, nord = 0;
            stack[sp++] = (cav_t)start_c;
            if constexpr (W::CAV <= 128) {
                // visited set in two 64-bit registers
                uint64_t v0 = 0, v1 = 0;
                while (sp > 0) {
                    const int c = stack[--sp];
                    const uint64_t bit = 1ull << (c & 63);
                    if ((c < 64 ? v0 : v1) & bit) continue;
                    if (c < 64) v0 |= bit; else v1 |= bit;
                    int n0, n1, n2, n3;
                    if constexpr (sizeof(cav_t) == 1) {
                        // the four signed 8-bit entries of tet c in one 32-bit load
                        const int w = *reinterpret_cast<const int *>(&ws.cav_nbr[4 * c]);
                        n0 = (int8_t)(w & 0xff);
                        n1 = (int8_t)((w >> 8) & 0xff);
                        n2 = (int8_t)((w >> 16) & 0xff);
                        n3 = (int8_t)((unsigned)w >> 24);
                    } else {
                        n0 = ws.cav_nbr[4 * c], n1 = ws.cav_nbr[4 * c + 1];
                        n2 = ws.cav_nbr[4 * c + 2], n3 = ws.cav_nbr[4 * c + 3];
                    }
                    ws.pos[c] = (cav_t)nord;
                    ws.order[nord++] = (cav_t)c;
                    const int nb[4] = {n0, n1, n2, n3};
    #pragma unroll
                    for (int f = 0; f < 4; f++) {
                        const int nc = nb[f];
                        if (nc >= 0 && !(((nc < 64 ? v0 : v1) >> (nc & 63)) & 1ull)) stack[sp++] = (cav_t)nc;
                    }
                }
            } else {
                while (sp > 0) {
                    const int c = stack[--sp];
                    if (ws.pos[c] >= 0) continue;
                    ws.pos[c] = (cav_t)nord;
                    ws.order[nord++] = (cav_t)c;
                    for (int f = 0; f < 4; f++) {
                        const int nc = ws.cav_nbr[4 * c + f];
                        if (nc >= 0 && ws.pos[nc] < 0) stack[sp++] = (cav_t)nc;
                    }
                }
            }
        }
        g.sync();
    }

    return ncav;
}

// The coincident-vertex row (natural_insertionfree.c:596-622): an empty
// cavity means the query may sit exactly on a vertex of the start tet; the
// row is 1/n on each of the n data vertices of that tet equal to q.
template <int G, class W>
__device__ void coincident_row(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g, int start,
                               RowInfo &r) {
    bool co = false;
    int v = -1;
    if (g.lane < 4) {
        v = comp(M.tv[start], g.lane);
        co = v < M.n && veq(vload(M, v), q);
    }
    const unsigned cm = g.ballot(co);
    const int nco = __popc(cm);
    if (co) {
        const int s = __popc(cm & g.lt());
        ws.nbr_vid[s] = v;
        ws.acc[s] = fdiv(1.0, (double)nco);
    }
    g.sync();
    r.nnb = nco;
    r.coincident = true;
}

// The circumcentres of the 4 faces of cavity tet c as natinterp3d's face
// cache returns them (natural_insertionfree.c:233-253), as fcc[] indices
// (4 T < 2^31: nif_dmesh_create limits T): for a face shared with another
// cavity tet, the copy cached by whichever of the two natinterp3d visits first
// (its mirror slot is in tinfo), else the tet's own.  Needs ws.pos.
template <class W>
__device__ __forceinline__ void face_cc_choice(const MeshView &M, const W &ws, int c, int (&fp)[4]) {
    const int tt = ws.cav_tet[c];
    const uint32_t info = M.tinfo[tt];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int j = 3 - i;
        const int nc = ws.cav_nbr[4 * c + j];
        if (nc >= 0 && ws.pos[nc] < ws.pos[c]) {
            const int jm = (info >> (8 + 2 * j)) & 3;
            fp[i] = 4 * ws.cav_tet[nc] + (3 - jm);
        } else {
            fp[i] = 4 * tt + i;
        }
    }
}

// Steps 3-5 of the row: boundary faces in visiting order, the natural
// neighbours in first-seen order, and (FULL) the stolen volumes folded in
// natinterp3d's order and normalised.  The caller describes the cavity:
//   face(k, c)       whether face k & 3 of the (k >> 2)-th tet in visiting
//                    order is a boundary face; c = that tet's index into
//                    ws.cav_tet
//   tet_fp(o, c, fp) the o-th tet in visiting order (index c into
//                    ws.cav_tet) and the fcc[] indices of its four faces as
//                    natinterp3d's face cache returns them
//   tet_tv(c)        the vertex record of cavity tet c (M.tv[ws.cav_tet[c]])
template <int G, class W, bool FULL, class FaceFn, class FpFn, class TvFn>
__device__ RowInfo row_volumes(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g, const int ncav,
                               RowInfo r, FaceFn face, FpFn tet_fp, TvFn tet_tv) {
    // ---- 3. boundary faces (cavity order, then face order) ------------------
    int nbf = 0;
    for (int k0 = 0; k0 < 4 * ncav; k0 += G) {
        const int k = k0 + g.lane;
        bool isb = false;
        int c = 0;
        if (k < 4 * ncav) isb = face(k, c);
        const unsigned bm = g.ballot(isb);
        const int b = nbf + __popc(bm & g.lt());
        if (isb && b < W::BF) ws.bface[b] = (uint16_t)((c << 2) | (k & 3));
        nbf += __popc(bm);
    }
    if (nbf > W::BF) {
        r.status = ST_CAPACITY;
        return r;
    }
    r.nbf = nbf;

    // natural neighbours in first-seen order over the boundary-face vertices
    for (int i = g.lane; i < W::VH; i += G) {
        ws.vh_key[i] = -1;
        ws.vh_first[i] = 0x7fffffff;
    }
    g.sync();
    bool vfull = false;
    for (int k = g.lane; k < 3 * nbf; k += G) {
        const int b = k / 3, j = k - 3 * b;
        const int cf = ws.bface[b];
        const int v = comp(tet_tv(cf >> 2), face_vslot(cf & 3, j));
        if (v < M.n) {
            const int s = hash_upsert(ws.vh_key, W::VH, v, vfull);
            if (s >= 0) atomicMin(&ws.vh_first[s], k);
        }
    }
    g.sync();
    if (g.any(vfull)) {
        r.status = ST_CAPACITY;
        return r;
    }
    int nnb = 0;
    for (int k0 = 0; k0 < 3 * nbf; k0 += G) {
        const int k = k0 + g.lane;
        bool first = false;
        int v = -1, s = -1;
        if (k < 3 * nbf) {
            const int b = k / 3, j = k - 3 * b;
            const int cf = ws.bface[b];
            v = comp(tet_tv(cf >> 2), face_vslot(cf & 3, j));
            if (v < M.n) {
                s = hash_find(ws.vh_key, W::VH, v);
                first = (s >= 0) && ws.vh_first[s] == k;
            }
        }
        const unsigned fm = g.ballot(first);
        const int slot = nnb + __popc(fm & g.lt());
        if (first) {
            ws.vh_slot[s] = (int16_t)slot;
            if (slot < W::NBR) {
                ws.nbr_vid[slot] = v;
                ws.acc[slot] = 0.0;
            }
        }
        nnb += __popc(fm);
    }
    if (nnb > W::NBR) {
        r.status = ST_CAPACITY;
        return r;
    }
    g.sync();
    if (nnb == 0) return r;
    if constexpr (!FULL) {
        r.nnb = nnb;
        return r;
    }

    // ---- 4. stolen volumes ----------------------------------------------------
    // Items in natinterp3d's order: the 4 vertices of every cavity tet (cavity
    // order), then the 3 vertices of every boundary face (face order).  One
    // lane computes the items of one cavity tet (4) or one boundary face (3),
    // sharing that tet's loads and face-circumcentre choices, or the face's
    // virtual-tet circumcentre, among them; the terms go to a shared buffer
    // in item order.  Then lanes whose items belong to the same neighbour are
    // folded into acc[] by the lowest of them, in lane order, so every acc[]
    // is a left-to-right sum in item order.
    {
        // the cavity-search scratch is free now: item buffer of one round
        constexpr int PER = 4 * G;  // items of one round (old terms: 4 per lane)
        static_assert(PER * (sizeof(double) + sizeof(int16_t)) <= sizeof(ws.u), "item buffer");
        double *bterm = reinterpret_cast<double *>(&ws.u);
        int16_t *bslot = reinterpret_cast<int16_t *>(bterm + PER);
        // folds buffered items [0, n) into acc[]
        auto fold = [&](int n) {
            for (int k0 = 0; k0 < n; k0 += G) {
                const int k = k0 + g.lane;
                const int s = k < n ? bslot[k] : -1;
                const double term = k < n ? bterm[k] : 0.0;
                const unsigned peers = g.match(s);
                const bool lead = s >= 0 && (__ffs(peers) - 1) == g.lane;
                unsigned rem = lead ? peers : 0u;
                double a = lead ? ws.acc[s] : 0.0;
                while (g.any(rem != 0u)) {
                    const int src = rem ? __ffs(rem) - 1 : g.lane;
                    const double tv = g.shfl(term, src);
                    if (rem) {
                        a = fadd(a, tv);
                        rem &= rem - 1u;
                    }
                }
                if (lead) ws.acc[s] = a;
                g.sync();
            }
        };
        // cavity-tet terms (natural_insertionfree.c:642-676): one lane per
        // item (tet o = k / 4, vertex k % 4), so that a cavity of 18 tets
        // takes 3 lane-steps of 32 items rather than 4 steps of 18 lanes
        for (int k0 = 0; k0 < 4 * ncav; k0 += PER) {
            const int n_round = min(PER, 4 * ncav - k0);
#pragma unroll 1
            for (int k = k0 + g.lane; k < k0 + n_round; k += G) {
                const int o = k >> 2, vi = k & 3;
                int c, fp[4];
                tet_fp(o, c, fp);
                const int tt = ws.cav_tet[c];
                const int4 p = tet_tv(c);
                const int v = comp(p, vi);
                const int sl = v < M.n ? neighbour_slot(ws, v) : -1;
                double term = 0.0;
                if (sl >= 0) {
                    // the other three vertices in ascending slot order
                    const int o0v = (vi == 0) ? 1 : 0;
                    const int o1v = (vi <= 1) ? 2 : 1;
                    const int o2v = (vi <= 2) ? 3 : 2;
                    const dv3 pk = vload(M, v);
                    const dv3 pa = vload(M, comp(p, o0v));
                    const dv3 pb = vload(M, comp(p, o1v));
                    const dv3 pc = vload(M, comp(p, o2v));
                    const dv3 ct = cload(&M.tcc[tt]);
                    // fp[] indexed through selects, so that it stays in registers
                    auto pick = [&](int i) {
                        return i == 0 ? fp[0] : (i == 1 ? fp[1] : (i == 2 ? fp[2] : fp[3]));
                    };
                    const dv3 f1 = cload(&M.fcc[pick(o2v)]);
                    const dv3 f2 = cload(&M.fcc[pick(o1v)]);
                    const dv3 f3 = cload(&M.fcc[pick(o0v)]);
                    term = subcell_volume(pk, pa, pb, pc, ct, f1, f2, f3);
                }
                bterm[k - k0] = term;
                bslot[k - k0] = (int16_t)sl;
            }
            g.sync();
            fold(n_round);
        }
        // virtual-tet terms, query + boundary face (:681-719)
        for (int b0 = 0; b0 < nbf; b0 += G) {
            const int b = b0 + g.lane;
            const int nb_round = min(G, nbf - b0);
            if (b < nbf) {
                const int cf = ws.bface[b];
                const int f = cf & 3;
                const int tt = ws.cav_tet[cf >> 2];
                const int4 p = tet_tv(cf >> 2);
                const int va = comp(p, face_vslot(f, 0));
                const int vb = comp(p, face_vslot(f, 1));
                const int vc = comp(p, face_vslot(f, 2));
                const dv3 ct = tet_cc(q, vload(M, va), vload(M, vb), vload(M, vc));
                const int ffi = 4 * tt + (3 - f);
#pragma unroll 1
                for (int j = 0; j < 3; j++) {
                    const int v = (j == 0) ? va : (j == 1 ? vb : vc);
                    const int sl = v < M.n ? neighbour_slot(ws, v) : -1;
                    double term = 0.0;
                    if (sl >= 0) {
                        // the face's vertices are re-read (L1) rather than held
                        // across the loop, which would spill them
                        const int vn = (j == 0) ? vb : (j == 1 ? vc : va);  // face_verts[(j+1)%3]
                        const int vp = (j == 0) ? vc : (j == 1 ? va : vb);  // face_verts[(j+2)%3]
                        const dv3 pk = vload(M, v), pb = vload(M, vn), pc = vload(M, vp);
                        const dv3 f1 = tri_cc(pk, q, pb);
                        const dv3 f2 = tri_cc(pk, q, pc);
                        term = -subcell_volume(pk, q, pb, pc, ct, f1, f2, cload(&M.fcc[ffi]));
                    }
                    bterm[3 * g.lane + j] = term;
                    bslot[3 * g.lane + j] = (int16_t)sl;
                }
            }
            g.sync();
            fold(3 * nb_round);
        }
    }

    // ---- 5. normalisation -----------------------------------------------------
    double total = 0.0;
    if (g.lane == 0)
        for (int s = 0; s < nnb; s++) total = fadd(total, ws.acc[s]);
    total = g.shfl(total, 0);
    if (!(total > 1e-30)) return r;  // empty row
    const double inv = fdiv(1.0, total);
    for (int s = g.lane; s < nnb; s += G) ws.acc[s] = fmul(ws.acc[s], inv);
    g.sync();
    r.nnb = nnb;
    r.total = total;
    return r;
}

// The Sibson row of centred query q.  On ST_OK the row is ws.nbr_vid[0..nnb)
// with normalised weights ws.acc[0..nnb), in natinterp3d's column order.
// With FULL = false only the combinatorial part is built (cavity, visiting
// order, boundary faces, neighbours in column order) and no volume is
// computed; the query-gradient kernel needs nothing more.  PM selects the
// predicate variant (PM_*); PM_RESOLVE needs xs, NIF_EXACT_SCRATCH doubles of
// global scratch owned by this group.  (The split kernels, k_rows_cavity and
// k_rows_volume, run the same steps on located rows.)
template <int G, class W, bool FULL = true, int PM = PM_PLAIN>
__device__ RowInfo sibson_row(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g,
                              double *xs = nullptr) {
    RowInfo r{ST_OK, 0, 0, false, false, 0.0, 0, 0, 0, 0, 0};
    bool on_face = false;  // PRED_EXACT: a face test of the located tet is exactly zero

    // ---- 1. point location -------------------------------------------------
    const int start = locate<G, PM>(M, q, g, reinterpret_cast<int *>(ws.acc), r, on_face, xs);
    if (r.status != ST_OK || r.outside) return r;

    // ---- 2. cavity and natinterp3d's visiting order ---------------------------
    const int ncav = flood_replay<G, W, PM>(M, q, ws, g, start, r, on_face, xs);
    if (r.status != ST_OK) return r;
    if (ncav == 0) {
        coincident_row<G>(M, q, ws, g, start, r);
        return r;
    }
    auto face = [&](int k, int &c) {
        c = ws.order[k >> 2];
        return ws.cav_nbr[4 * c + (k & 3)] < 0;
    };
    auto tet_fp = [&](int o, int &c, int (&fp)[4]) {
        c = ws.order[o];
        face_cc_choice(M, ws, c, fp);
    };
    auto tet_tv = [&](int c) { return M.tv[ws.cav_tet[c]]; };
    return row_volumes<G, W, FULL>(M, q, ws, g, ncav, r, face, tet_fp, tet_tv);
}

// The split row, part 1: cavity and visiting order of q around its located
// tet, written as a record (head, entries[REC_CAV]).  Returns REC_DONE, or
// REC_WIDE where the cavity fits the shared-memory capacities but not the
// record (the caller queues the row for the fused row kernel), or REC_LARGE
// where it exceeds the shared-memory capacities (the large kernel's).
// With PM_FILTER a test the error bound cannot certify also gives REC_LARGE
// (the large kernel resolves it exactly).
constexpr int REC_DONE = 0, REC_WIDE = 1, REC_LARGE = 2;
template <int G, class W, int PM = PM_PLAIN>
__device__ int cavity_record(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g, int start,
                             RowHead &head, RowEntry *__restrict__ ent) {
    static_assert(REC_CAV <= 127, "neighbour indices are signed bytes");
    RowInfo r{ST_OK, 0, 0, false, false, 0.0, 0, 0, 0, 0, 0};
    const int ncav = flood_replay<G, W, PM, false>(M, q, ws, g, start, r, false, nullptr);
    if (r.status != ST_OK) return REC_LARGE;
    if (ncav > REC_CAV) return REC_WIDE;
    head.ncav = ncav;
    for (int c = g.lane; c < ncav; c += G) {
        const int tt = ws.cav_tet[c];
        unsigned bm = (M.tinfo[tt] >> 8) & 0xffu;
        bm <<= 8;
        unsigned nb = 0;
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const int nc = ws.cav_nbr[4 * c + f];
            bm |= (nc < 0 ? 1u : 0u) << f;
            nb |= ((unsigned)nc & 0xffu) << (8 * f);
        }
        RowEntry e;
        e.tet = tt;
        e.bmask = bm;
        e.nbr = (int)nb;
        e.pos = 0;
        ent[c] = e;
    }
    g.sync();
    return REC_DONE;
}

// The split row, part 2: from a record of part 1 (state RS_OK) the row as
// sibson_row returns it (steps 3-5, or the coincident-vertex row).
template <int G, class W, bool FULL>
__device__ RowInfo volume_row(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g,
                              const RowHead &head, const RowEntry *__restrict__ ent) {
    RowInfo r{ST_OK, 0, 0, false, false, 0.0, 0, 0, 0, 0, 0};
    const int ncav = head.ncav;
    if (ncav == 0) {
        coincident_row<G>(M, q, ws, g, head.start, r);
        return r;
    }
    // the record is in the flood's order: place each tet at its position in
    // natinterp3d's visiting order
    for (int e = g.lane; e < ncav; e += G) {
        const RowEntry x = ent[e];
        const int o = min(x.pos & 0xff, ncav - 1);  // a permutation of 0..ncav-1
        ws.cav_tet[o] = x.tet;
        ws.bmask[o] = (uint8_t)(x.bmask & 0xfu);
        ws.ctv[o] = M.tv[x.tet];
        ws.ftet[e] = x.tet;
        ws.fpos[e] = (int8_t)o;
    }
    g.sync();
    // natinterp3d's face cache (natural_insertionfree.c:233-253): a face
    // shared with a cavity tet visited earlier returns that tet's copy, the
    // mirror slot of the face in it; otherwise the tet's own slot
    // (k_rows_order marked those faces; cfp is first read after the syncs of
    // the boundary-face step)
    for (int e = g.lane; e < ncav; e += G) {
        const RowEntry x = ent[e];
        const int o = ws.fpos[e];
        const unsigned wd = (unsigned)x.nbr;
        const unsigned mir = (x.bmask >> 8) & 0xffu;
        const unsigned take = ((unsigned)x.pos >> 8) & 0xfu;
        int fp[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int jf = 3 - i;
            const int n = (int8_t)((wd >> (8 * jf)) & 0xffu);
            if (((take >> i) & 1u) && n >= 0 && n < ncav) {
                const int jm = (mir >> (2 * jf)) & 3;
                fp[i] = 4 * ws.ftet[n] + (3 - jm);
            } else {
                fp[i] = 4 * x.tet + i;
            }
        }
        ws.cfp[o] = make_int4(fp[0], fp[1], fp[2], fp[3]);
    }
    auto face = [&](int k, int &c) {
        c = k >> 2;
        return ((ws.bmask[c] >> (k & 3)) & 1u) != 0u;
    };
    auto tet_fp = [&](int o, int &c, int (&fp)[4]) {
        c = o;
        const int4 f = ws.cfp[o];
        fp[0] = f.x;
        fp[1] = f.y;
        fp[2] = f.z;
        fp[3] = f.w;
    };
    auto tet_tv = [&](int c) { return ws.ctv[c]; };
    return row_volumes<G, W, FULL>(M, q, ws, g, ncav, r, face, tet_fp, tet_tv);
}

}  // namespace nif

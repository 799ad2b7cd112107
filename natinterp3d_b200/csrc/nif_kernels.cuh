// Device-side Sibson (natural-neighbour) query: one cooperative group of G
// lanes per query.
//
// Per query (natinterp3d's getWeightsSingleQueryIF, natural_insertionfree.c:591-738):
//   1. locate   seed tet from a uniform grid, then natinterp3d's visibility walk
//               (delaunay.c:398-405); the four face tests of a step run on 4 lanes
//   2. cavity   the connected set of tets whose circumsphere strictly contains
//               the query (inspherefast > 0, natural_insertionfree.c:502-530),
//               found breadth-first with all lanes testing in parallel; a
//               single-lane integer replay then recovers natinterp3d's LIFO
//               visiting order, which fixes the column order and the
//               floating-point summation order of every weight
//   3. boundary faces and natural neighbours in first-seen order (:559-584)
//   4. signed Voronoi-subcell volumes: +cavity-tet terms (:642-676) and
//      -virtual-tet terms (:681-719), one term per lane, written to a
//      slot-sorted buffer and summed per neighbour in natinterp3d's order
//   5. normalisation (:721-737)
// Tet circumcentres and face circumcentres are read from the per-mesh cache
// (computed with the same formulas and argument orders); a face shared by two
// cavity tets uses the circumcentre computed from the tet natinterp3d visits
// first, as natinterp3d's face cache does (:233-253).
#pragma once
#include <stdint.h>

#include "nif_geometry.cuh"

namespace nif {

// per-row status codes (stored as int8)
constexpr int ST_OK = 0;
constexpr int ST_WALK = 1;       // walk step limit
constexpr int ST_CAPACITY = 2;   // per-query capacity of this kernel exceeded
constexpr int ST_ARENA = 3;      // large-row output arena full

constexpr int WALK_LIMIT = 1 << 16;

struct __align__(32) d4 {
    double x, y, z, w;
};

// Resident mesh (device pointers) + seed grid parameters, passed by value.
struct MeshView {
    const d4 *__restrict__ vtx;        // [nv] x, y, z, 0
    const int4 *__restrict__ tv;       // [nt] vertex ids
    const int4 *__restrict__ tn;       // [nt] neighbour tets (-1 = none)
    const uint32_t *__restrict__ tinfo;// [nt] bit0: orient3dfast(p0..p3) > 0; bits 8+2j: mirror slot of face j
    const d4 *__restrict__ tcc;        // [nt] tet circumcentre
    const d4 *__restrict__ fcc;        // [nt*4] circumcentre of the face opposite p[i]
    const int *__restrict__ grid;      // seed tets of the finest grid level
    int n;                             // data vertices (ids >= n are super-simplex vertices)
    int nv, nt;
    int gdim[3];
    double glo[3], ginv[3];
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

__device__ __forceinline__ dv3 cload(const d4 *p) {
    const d4 v = *p;
    return dv3{v.x, v.y, v.z};
}

__device__ __forceinline__ int seed_cell(const MeshView &M, dv3 q) {
    double c[3] = {q.x, q.y, q.z};
    int idx[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        double f = (c[a] - M.glo[a]) * M.ginv[a];
        int k = (f >= 0.0) ? (f < (double)M.gdim[a] ? (int)f : M.gdim[a] - 1) : 0;
        idx[a] = k;
    }
    return (idx[2] * M.gdim[1] + idx[1]) * M.gdim[0] + idx[0];
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
};

// Per-group scratch.  The first union member is live during the cavity
// search, the second only during the single-lane replay, the third during
// the volume terms and the interpolation epilogue.
template <int HS_, int CAV_, int BF_, int NBR_, int VH_, int TERMS_, int G_>
struct Workspace {
    static constexpr int HS = HS_;        // tested-tet hash slots (power of two)
    static constexpr int QCAP = HS_ * 3 / 4;
    static constexpr int CAV = CAV_;      // cavity tets
    static constexpr int STACK = 4 * CAV_ + 1;
    static constexpr int BF = BF_;        // boundary faces
    static constexpr int NBR = NBR_;      // natural neighbours
    static constexpr int VH = VH_;        // neighbour hash slots (power of two)
    static constexpr int TERMS = TERMS_;  // volume terms
    static constexpr int G = G_;
    union U {
        struct {
            int hkey[HS_];
            int hval[HS_];
            int queue[HS_ * 3 / 4];
        } a;
        struct {
            int stack[4 * CAV_ + 1];
        } r;
        struct {
            double terms[TERMS_];
            double vt[G_][3];
        } b;
    } u;
    int cav_tet[CAV_];
    int cav_nbr[4 * CAV_];
    int order[CAV_];
    int pos[CAV_];
    int bface[BF_];
    int vh_key[VH_];
    int vh_first[VH_];
    int vh_slot[VH_];
    int nbr_vid[NBR_];
    int cnt[NBR_];
    int off[NBR_];
    int run[NBR_];
    double w[NBR_];
};

__device__ __forceinline__ unsigned mix_hash(int key) {
    return (unsigned)key * 2654435761u;
}

// Inserts key; returns its slot if newly inserted, -1 if already present.
// Sets full when every slot was probed.
__device__ __forceinline__ int hash_insert(int *keys, int hs, int key, bool &full) {
    unsigned h = mix_hash(key) & (unsigned)(hs - 1);
    for (int probe = 0; probe < hs; ++probe) {
        const int old = atomicCAS(&keys[h], -1, key);
        if (old == -1) return (int)h;
        if (old == key) return -1;
        h = (h + 1) & (unsigned)(hs - 1);
    }
    full = true;
    return -1;
}

// Slot of key (inserted if absent); -1 and full=true when the table is full.
__device__ __forceinline__ int hash_upsert(int *keys, int hs, int key, bool &full) {
    unsigned h = mix_hash(key) & (unsigned)(hs - 1);
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
};

// Circumcentre natinterp3d's face cache returns for the face opposite p[i] of
// cavity tet c (tet id t, tinfo word info): the value cached by whichever of
// the two cavity tets sharing the face natinterp3d visits first.
template <class W>
__device__ __forceinline__ dv3 face_cc(const MeshView &M, const W &ws, int c, int t, uint32_t info,
                                      int i) {
    const int j = 3 - i;
    const int nc = ws.cav_nbr[4 * c + j];
    if (nc >= 0 && ws.pos[nc] < ws.pos[c]) {
        const int jm = (info >> (8 + 2 * j)) & 3;
        return cload(&M.fcc[4 * (size_t)ws.cav_tet[nc] + (3 - jm)]);
    }
    return cload(&M.fcc[4 * (size_t)t + i]);
}

// slot of a data vertex among the natural neighbours, -1 if it is not one
template <class W>
__device__ __forceinline__ int neighbour_slot(const W &ws, int v) {
    const int s = hash_find(ws.vh_key, W::VH, v);
    return s >= 0 ? ws.vh_slot[s] : -1;
}

// The Sibson row of centred query q.  On ST_OK the row is ws.nbr_vid[0..nnb)
// with normalised weights ws.w[0..nnb), in natinterp3d's column order.
template <int G, class W>
__device__ RowInfo sibson_row(const MeshView &M, const dv3 q, W &ws, const Grp<G> &g) {
    RowInfo r{ST_OK, 0, 0, false};

    // ---- 1. point location -------------------------------------------------
    int t = M.grid[seed_cell(M, q)];
    for (;;) {
        if (r.steps >= WALK_LIMIT) {
            r.status = ST_WALK;
            return r;
        }
        ++r.steps;
        const int4 p = M.tv[t];
        bool neg = false;
        if (g.lane < 4) {
            const int f = g.lane;
            const dv3 v1 = vload(M, comp(p, face_vslot(f, 0)));
            const dv3 v2 = vload(M, comp(p, face_vslot(f, 1)));
            const dv3 v3 = vload(M, comp(p, face_vslot(f, 2)));
            neg = orient_fast(v1, v2, v3, q) < 0;
        }
        const unsigned m = g.ballot(neg);
        if (!m) break;
        const int nb = comp(M.tn[t], __ffs(m) - 1);
        if (nb < 0) {
            r.outside = true;
            return r;
        }
        t = nb;
    }
    const int start = t;

    // ---- 2. cavity: parallel flood over the tested-tet hash ----------------
    for (int i = g.lane; i < W::HS; i += G) {
        ws.u.a.hkey[i] = -1;
        ws.u.a.hval[i] = -1;
    }
    g.sync();
    if (g.lane == 0) {
        const int h = (int)(mix_hash(start) & (unsigned)(W::HS - 1));
        ws.u.a.hkey[h] = start;
        ws.u.a.queue[0] = h;
    }
    g.sync();
    int qhead = 0, qtail = 1, ncav = 0;
    bool overflow = false;
    while (qhead < qtail) {
        const int n = min(G, qtail - qhead);
        int slot = -1, tt = -1;
        bool inc = false;
        if (g.lane < n) {
            slot = ws.u.a.queue[qhead + g.lane];
            tt = ws.u.a.hkey[slot];
            const int4 p = M.tv[tt];
            const dv3 a = vload(M, p.x), b = vload(M, p.y), c = vload(M, p.z), d = vload(M, p.w);
            const double ins = (M.tinfo[tt] & 1u) ? insphere_fast(a, b, c, d, q)
                                                  : insphere_fast(b, a, c, d, q);
            inc = ins > 0;
        }
        const unsigned cm = g.ballot(inc);
        const int ci = ncav + __popc(cm & g.lt());
        if (g.lane < n) ws.u.a.hval[slot] = inc ? ci : -1;
        if (inc && ci < W::CAV) ws.cav_tet[ci] = tt;
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
            bool full = false;
            if (k < 4 * nnew) {
                const int nb = comp(M.tn[ws.cav_tet[base + (k >> 2)]], k & 3);
                if (nb >= 0) ns = hash_insert(ws.u.a.hkey, W::HS, nb, full);
            }
            const unsigned pm = g.ballot(ns >= 0);
            const int qi = qtail + __popc(pm & g.lt());
            if (ns >= 0 && qi < W::QCAP) ws.u.a.queue[qi] = ns;
            qtail += __popc(pm);
            if (g.any(full) || qtail > W::QCAP) overflow = true;
        }
        if (overflow) break;
        g.sync();
    }
    g.sync();
    if (overflow) {
        r.status = ST_CAPACITY;
        return r;
    }

    if (ncav == 0) {
        // coincident-vertex path (natural_insertionfree.c:596-622): an empty
        // cavity means the query may sit exactly on a vertex of the start tet
        bool co = false;
        int v = -1;
        if (g.lane < 4) {
            v = comp(M.tv[start], g.lane);
            co = v < M.n && veq(vload(M, v), q);
        }
        const unsigned cm = g.ballot(co);
        const int nco = __popc(cm);
        if (nco > 0) {
            const double w = fdiv(1.0, (double)nco);
            if (co) {
                const int s = __popc(cm & g.lt());
                ws.nbr_vid[s] = v;
                ws.w[s] = w;
            }
        }
        g.sync();
        r.nnb = nco;
        return r;
    }

    // cavity-local neighbour table: cav_nbr[4c+f] = cavity index of s[f] or -1
    for (int k = g.lane; k < 4 * ncav; k += G) {
        const int nb = comp(M.tn[ws.cav_tet[k >> 2]], k & 3);
        int v = -1;
        if (nb >= 0) {
            const int s = hash_find(ws.u.a.hkey, W::HS, nb);
            v = (s >= 0) ? ws.u.a.hval[s] : -1;
        }
        ws.cav_nbr[k] = v;
    }
    for (int c = g.lane; c < ncav; c += G) ws.pos[c] = -1;
    g.sync();

    // replay natinterp3d's LIFO flood on the cavity (its non-cavity tets are
    // leaves and do not change the order in which cavity tets are reached)
    if (g.lane == 0) {
        int *stack = ws.u.r.stack;
        int sp = 0, nord = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int c = stack[--sp];
            if (ws.pos[c] >= 0) continue;
            ws.pos[c] = nord;
            ws.order[nord++] = c;
            for (int f = 0; f < 4; f++) {
                const int nc = ws.cav_nbr[4 * c + f];
                if (nc >= 0 && ws.pos[nc] < 0) stack[sp++] = nc;
            }
        }
    }
    g.sync();

    // ---- 3. boundary faces (cavity order, then face order) ------------------
    int nbf = 0;
    for (int k0 = 0; k0 < 4 * ncav; k0 += G) {
        const int k = k0 + g.lane;
        bool isb = false;
        int c = 0;
        if (k < 4 * ncav) {
            c = ws.order[k >> 2];
            isb = ws.cav_nbr[4 * c + (k & 3)] < 0;
        }
        const unsigned bm = g.ballot(isb);
        const int b = nbf + __popc(bm & g.lt());
        if (isb && b < W::BF) ws.bface[b] = (c << 2) | (k & 3);
        nbf += __popc(bm);
    }
    if (nbf > W::BF) {
        r.status = ST_CAPACITY;
        return r;
    }

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
        const int v = comp(M.tv[ws.cav_tet[cf >> 2]], face_vslot(cf & 3, j));
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
            v = comp(M.tv[ws.cav_tet[cf >> 2]], face_vslot(cf & 3, j));
            if (v < M.n) {
                s = hash_find(ws.vh_key, W::VH, v);
                first = (s >= 0) && ws.vh_first[s] == k;
            }
        }
        const unsigned fm = g.ballot(first);
        const int slot = nnb + __popc(fm & g.lt());
        if (first) {
            ws.vh_slot[s] = slot;
            if (slot < W::NBR) ws.nbr_vid[slot] = v;
        }
        nnb += __popc(fm);
    }
    if (nnb > W::NBR) {
        r.status = ST_CAPACITY;
        return r;
    }
    g.sync();
    if (nnb == 0) return r;

    // ---- 4. volume terms: counting pass --------------------------------------
    for (int s = g.lane; s < nnb; s += G) ws.cnt[s] = 0;
    g.sync();
    for (int k0 = 0; k0 < 4 * ncav; k0 += G) {
        const int k = k0 + g.lane;
        int s = -1;
        if (k < 4 * ncav) {
            const int v = comp(M.tv[ws.cav_tet[ws.order[k >> 2]]], k & 3);
            if (v < M.n) s = neighbour_slot(ws, v);
        }
        const unsigned peers = g.match(s);
        if (s >= 0 && (__ffs(peers) - 1) == g.lane) ws.cnt[s] += __popc(peers);
        g.sync();
    }
    for (int k0 = 0; k0 < 3 * nbf; k0 += G) {
        const int k = k0 + g.lane;
        int s = -1;
        if (k < 3 * nbf) {
            const int b = k / 3, j = k - 3 * b;
            const int cf = ws.bface[b];
            const int v = comp(M.tv[ws.cav_tet[cf >> 2]], face_vslot(cf & 3, j));
            if (v < M.n) s = neighbour_slot(ws, v);
        }
        const unsigned peers = g.match(s);
        if (s >= 0 && (__ffs(peers) - 1) == g.lane) ws.cnt[s] += __popc(peers);
        g.sync();
    }
    int nterm = 0;
    if (g.lane == 0) {
        for (int s = 0; s < nnb; s++) {
            ws.off[s] = nterm;
            ws.run[s] = 0;
            nterm += ws.cnt[s];
        }
    }
    nterm = g.shfl(nterm, 0);
    g.sync();
    if (nterm > W::TERMS) {
        r.status = ST_CAPACITY;
        return r;
    }

    // ---- 4b. volume terms: compute pass (same item order) -------------------
    // cavity tets: +volume of the subcell of each neighbour vertex
    for (int k0 = 0; k0 < 4 * ncav; k0 += G) {
        const int k = k0 + g.lane;
        int s = -1, c = 0, tt = 0, vi = 0;
        int4 p = make_int4(0, 0, 0, 0);
        if (k < 4 * ncav) {
            c = ws.order[k >> 2];
            vi = k & 3;
            tt = ws.cav_tet[c];
            p = M.tv[tt];
            const int v = comp(p, vi);
            if (v < M.n) s = neighbour_slot(ws, v);
        }
        const unsigned peers = g.match(s);
        int dest = 0;
        if (s >= 0) dest = ws.off[s] + ws.run[s] + __popc(peers & g.lt());
        g.sync();
        if (s >= 0 && (__ffs(peers) - 1) == g.lane) ws.run[s] += __popc(peers);
        if (s >= 0) {
            const uint32_t info = M.tinfo[tt];
            // the other three vertices in ascending slot order
            const int o0 = (vi == 0) ? 1 : 0;
            const int o1 = (vi <= 1) ? 2 : 1;
            const int o2 = (vi <= 2) ? 3 : 2;
            const dv3 pk = vload(M, comp(p, vi));
            const dv3 pa = vload(M, comp(p, o0));
            const dv3 pb = vload(M, comp(p, o1));
            const dv3 pc = vload(M, comp(p, o2));
            const dv3 ct = cload(&M.tcc[tt]);
            const dv3 f2 = face_cc(M, ws, c, tt, info, o2);
            const dv3 f1 = face_cc(M, ws, c, tt, info, o1);
            const dv3 f0 = face_cc(M, ws, c, tt, info, o0);
            ws.u.b.terms[dest] = subcell_volume(pk, pa, pb, pc, ct, f2, f1, f0);
        }
        g.sync();
    }
    // virtual tets (query + boundary face): -volume, faces in chunks of G
    for (int b0 = 0; b0 < nbf; b0 += G) {
        {
            const int b = b0 + g.lane;
            if (b < nbf) {
                const int cf = ws.bface[b];
                const int f = cf & 3;
                const int4 p = M.tv[ws.cav_tet[cf >> 2]];
                const dv3 fa = vload(M, comp(p, face_vslot(f, 0)));
                const dv3 fb = vload(M, comp(p, face_vslot(f, 1)));
                const dv3 fc = vload(M, comp(p, face_vslot(f, 2)));
                const dv3 cv = tet_cc(q, fa, fb, fc);
                ws.u.b.vt[g.lane][0] = cv.x;
                ws.u.b.vt[g.lane][1] = cv.y;
                ws.u.b.vt[g.lane][2] = cv.z;
            }
        }
        g.sync();
        const int kend = 3 * min(nbf, b0 + G);
        for (int k0 = 3 * b0; k0 < kend; k0 += G) {
            const int k = k0 + g.lane;
            int s = -1, b = 0, j = 0, tt = 0, f = 0;
            int4 p = make_int4(0, 0, 0, 0);
            if (k < kend) {
                b = k / 3;
                j = k - 3 * b;
                const int cf = ws.bface[b];
                f = cf & 3;
                tt = ws.cav_tet[cf >> 2];
                p = M.tv[tt];
                const int v = comp(p, face_vslot(f, j));
                if (v < M.n) s = neighbour_slot(ws, v);
            }
            const unsigned peers = g.match(s);
            int dest = 0;
            if (s >= 0) dest = ws.off[s] + ws.run[s] + __popc(peers & g.lt());
            g.sync();
            if (s >= 0 && (__ffs(peers) - 1) == g.lane) ws.run[s] += __popc(peers);
            if (s >= 0) {
                const int ja = (j == 2) ? 0 : j + 1;
                const int jb = (j == 0) ? 2 : j - 1;
                const dv3 pk = vload(M, comp(p, face_vslot(f, j)));
                const dv3 pa = vload(M, comp(p, face_vslot(f, ja)));
                const dv3 pb = vload(M, comp(p, face_vslot(f, jb)));
                const dv3 cface = cload(&M.fcc[4 * (size_t)tt + (3 - f)]);
                const int bl = b - b0;
                const dv3 cv = mk(ws.u.b.vt[bl][0], ws.u.b.vt[bl][1], ws.u.b.vt[bl][2]);
                const dv3 cqa = tri_cc(pk, q, pa);
                const dv3 cqb = tri_cc(pk, q, pb);
                ws.u.b.terms[dest] = -subcell_volume(pk, q, pa, pb, cv, cqa, cqb, cface);
            }
            g.sync();
        }
        g.sync();
    }

    // per-neighbour sums in natinterp3d's accumulation order
    for (int s = g.lane; s < nnb; s += G) {
        double acc = 0.0;
        const int o = ws.off[s], e = o + ws.cnt[s];
        for (int j = o; j < e; j++) acc = fadd(acc, ws.u.b.terms[j]);
        ws.w[s] = acc;
    }
    g.sync();

    // ---- 5. normalisation -----------------------------------------------------
    double total = 0.0;
    if (g.lane == 0)
        for (int s = 0; s < nnb; s++) total = fadd(total, ws.w[s]);
    total = g.shfl(total, 0);
    if (!(total > 1e-30)) return r;  // empty row
    const double inv = fdiv(1.0, total);
    for (int s = g.lane; s < nnb; s += G) ws.w[s] = fmul(ws.w[s], inv);
    g.sync();
    r.nnb = nnb;
    return r;
}

}  // namespace nif

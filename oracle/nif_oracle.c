/*
 * natinterp3d_b200 CPU oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A sequential FP64 restatement of natinterp3d's insertion-free Sibson query
 * (natural_insertionfree.c) over the packed mesh arrays that the product
 * uploads to the GPU (vxyz [V][3], tet_v [T][4], tet_n [T][4]; vertex ids
 * >= N are the four super-simplex vertices).  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it; the product never does.
 *
 * Parity contract: every floating-point expression below is evaluated with
 * the same operand grouping as natinterp3d's C code, and this file is compiled
 * with -ffp-contract=off, so on IEEE-754 doubles the results are bit-identical
 * to natinterp3d compiled with its setup.py flags (-std=c11, no -march, hence
 * no FMA).  The one deliberate difference is the point-location seed: natinterp3d
 * seeds its walk with the tet whose centroid is nearest to the query, found in
 * an unbalanced k-d tree (delaunay.c:392-395, kdtree.c:543-564); this oracle
 * finds the same exact-nearest centroid with a uniform grid (ties go to the
 * lowest tet id).  The walk, cavity search, boundary extraction, neighbour
 * order, volume terms and normalisation follow natinterp3d step by step.
 *
 * Predicate modes (orc_mesh_set_predicates), the same three the product has:
 *   0  natinterp3d's signs: the fast determinants' own signs (the default);
 *   1  the same signs, and every evaluation whose fast value lies inside the
 *      static error bound is re-evaluated exactly and counted ("uncertain"),
 *      together with those whose decision the exact sign would change
 *      ("flipped");
 *   2  exact signs (filter, then expansion arithmetic), counted the same
 *      way; a query that lies exactly on a face or edge of the tet its walk
 *      ends in floods the cavity from the lowest-id tet containing it, so
 *      the visiting order does not depend on the walk's seed.
 * The exact arithmetic is the product's nif_exact.h, pinned separately
 * against rational arithmetic and against Shewchuk's robust predicates.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_OK 0
#define ORC_ERR_ARG -1
#define ORC_ERR_NOMEM -3
#define ORC_ERR_OVERFLOW -5
#define ORC_ERR_WALK -6

#define ORC_PRED_FAST 0
#define ORC_PRED_AUDIT 1
#define ORC_PRED_EXACT 2

#include "nif_exact.h"

/* ------------------------------------------------------------------------- */
/* Geometric predicates: the non-robust "fast" determinants natinterp3d calls  */
/* (predicates.c:1687-1710 orient3dfast, :3301-3347 inspherefast).            */
/* ------------------------------------------------------------------------- */

typedef struct { double x, y, z; } v3;

static inline v3 ld(const double *p) { v3 r = {p[0], p[1], p[2]}; return r; }
static inline v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline v3 add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline v3 scale(v3 a, double s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
/* crossProduct, delaunay.c:986-990 */
static inline v3 cross(v3 b, v3 c) {
    v3 r = {b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
    return r;
}
/* scalarProduct, delaunay.c:994-996: (a0 b0 + a1 b1) + a2 b2 */
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

/* orient3dfast(a, b, c, d): sign of det[a-d; b-d; c-d]. */
double orc_orient(const double *pa, const double *pb, const double *pc, const double *pd) {
    v3 d = ld(pd);
    v3 u = sub(ld(pa), d), v = sub(ld(pb), d), w = sub(ld(pc), d);
    double t0 = u.x * (v.y * w.z - v.z * w.y);
    double t1 = v.x * (w.y * u.z - w.z * u.y);
    double t2 = w.x * (u.y * v.z - u.z * v.y);
    return (t0 + t1) + t2;
}

/* inspherefast(a, b, c, d, e): lifted 4x4 determinant relative to e. */
double orc_insphere(const double *pa, const double *pb, const double *pc, const double *pd,
                    const double *pe) {
    v3 e = ld(pe);
    v3 r[4] = {sub(ld(pa), e), sub(ld(pb), e), sub(ld(pc), e), sub(ld(pd), e)};
    /* 2x2 minors of the (x, y) columns: m(i,j) = x_i y_j - x_j y_i */
#define M2(i, j) (r[i].x * r[j].y - r[j].x * r[i].y)
    double m01 = M2(0, 1), m12 = M2(1, 2), m23 = M2(2, 3), m30 = M2(3, 0);
    double m02 = M2(0, 2), m13 = M2(1, 3);
#undef M2
    double abc = r[0].z * m12 - r[1].z * m02 + r[2].z * m01;
    double bcd = r[1].z * m23 - r[2].z * m13 + r[3].z * m12;
    double cda = r[2].z * m30 + r[3].z * m02 + r[0].z * m23;
    double dab = r[3].z * m01 + r[0].z * m13 + r[1].z * m30;
    double lift[4];
    for (int k = 0; k < 4; k++) lift[k] = r[k].x * r[k].x + r[k].y * r[k].y + r[k].z * r[k].z;
    return (lift[3] * abc - lift[2] * dab) + (lift[1] * cda - lift[0] * bcd);
}

/* ------------------------------------------------------------------------- */
/* Circumcentres and Voronoi subcell volume                                   */
/* ------------------------------------------------------------------------- */

/* circumCenterTri3D, natural_insertionfree.c:24-49 */
static v3 tri_cc(v3 a, v3 b, v3 c) {
    v3 ab = sub(b, a), ac = sub(c, a);
    v3 n = cross(ab, ac);
    double n2 = dot(n, n);
    if (n2 < 1e-30) {
        v3 r = {(a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0};
        return r;
    }
    double ab2 = dot(ab, ab), ac2 = dot(ac, ac);
    v3 t = {ab2 * ac.x - ac2 * ab.x, ab2 * ac.y - ac2 * ab.y, ab2 * ac.z - ac2 * ab.z};
    v3 cr = cross(t, n);
    double inv = 1.0 / (2.0 * n2);
    return add(a, scale(cr, inv));
}

/* circumCenterTet, natural_insertionfree.c:54-84 */
static v3 tet_cc(v3 a, v3 b, v3 c, v3 d) {
    v3 ba = sub(b, a), ca = sub(c, a), da = sub(d, a);
    v3 x1 = cross(ba, ca), x2 = cross(da, ba), x3 = cross(ca, da);
    v3 m1 = scale(x1, dot(da, da));
    v3 m2 = scale(x2, dot(ca, ca));
    v3 m3 = scale(x3, dot(ba, ba));
    v3 s = add(m3, add(m1, m2));
    double den = 2.0 * dot(ba, x3);
    if (fabs(den) < 1e-30) {
        v3 r = {(a.x + b.x + c.x + d.x) * 0.25, (a.y + b.y + c.y + d.y) * 0.25,
                (a.z + b.z + c.z + d.z) * 0.25};
        return r;
    }
    return add(scale(s, 1.0 / den), a);
}

/* voronoiSubcellVolume, natural_insertionfree.c:92-146; the algebra is
 * derived in docs/insertion-free.rst:88-165 of natinterp3d. */
static double subcell(v3 pk, v3 pa, v3 pb, v3 pc, v3 ct, v3 fab, v3 fac, v3 fbc) {
    v3 ta = sub(pa, pk), tb = sub(pb, pk), tc = sub(pc, pk);
    double sv = dot(ta, cross(tb, tc));
    v3 a = pa, b = pb;
    if (sv < 0) {
        a = pb; b = pa;
        v3 t = fac; fac = fbc; fbc = t;
    }
    v3 df = sub(fab, pk), dg = sub(fac, pk), dh = sub(fbc, pk), dt = sub(ct, pk);
    v3 c1 = cross(df, dt), c2 = cross(dt, dg), c3 = cross(dh, dt);
    v3 e1 = sub(a, b), e2 = sub(a, pc), e3 = sub(b, pc);
    double vol = e1.x * c1.x;
    vol = vol + e1.y * c1.y;
    vol = vol + e1.z * c1.z;
    vol = vol + e2.x * c2.x;
    vol = vol + e2.y * c2.y;
    vol = vol + e2.z * c2.z;
    vol = vol + e3.x * c3.x;
    vol = vol + e3.y * c3.y;
    vol = vol + e3.z * c3.z;
    return vol / 12.0;
}

/* ------------------------------------------------------------------------- */
/* Mesh + seed grid                                                           */
/* ------------------------------------------------------------------------- */

typedef struct {
    int nv, nt, n;           /* vertices (incl. 4 super), tets, data vertices */
    const double *vx;        /* [nv][3] */
    const int32_t *tv;       /* [nt][4] */
    const int32_t *tn;       /* [nt][4] */
    unsigned char *pos;      /* orient3dfast(p0..p3) > 0, natural_insertionfree.c:457-476 */
    unsigned char *pos_x;    /* exact orient3d(p0..p3) > 0 */
    long orient_unc, orient_flip; /* tets whose orientation sign is uncertain / flipped */
    int pmode;               /* ORC_PRED_* */
    int seed_first;          /* walk from tet 0, as natinterp3d does without its k-d tree
                                (delaunay.c:389-391), instead of the nearest centroid */
    double *cen;             /* tet centroids [nt][3], delaunay.c:152-157 */
    /* exact nearest-centroid grid */
    double lo[3], h[3];
    int g[3];
    int *cell_start, *cell_items;
} orc_mesh;

/* getFaceVerticies3, delaunay.c:444-467: face i lies opposite p[3-i] and is
 * shared with neighbour s[i]. */
static const int FACE3[4][3] = {{0, 1, 2}, {3, 1, 0}, {0, 2, 3}, {3, 2, 1}};

static inline const double *V(const orc_mesh *m, int vid) { return m->vx + 3 * (size_t)vid; }

static int cell_coord(const orc_mesh *m, int d, double x) {
    double f = (x - m->lo[d]) / m->h[d];
    int c = (f >= 0) ? (int)f : -1;
    if (c < 0) c = 0;
    if (c >= m->g[d]) c = m->g[d] - 1;
    return c;
}

void orc_mesh_free(orc_mesh *m) {
    if (!m) return;
    free(m->pos);
    free(m->pos_x);
    free(m->cen);
    free(m->cell_start);
    free(m->cell_items);
    free(m);
}

orc_mesh *orc_mesh_new(const double *vx, int nv, const int32_t *tv, const int32_t *tn, int nt) {
    if (nv < 5 || nt < 1) return NULL;
    orc_mesh *m = calloc(1, sizeof(orc_mesh));
    if (!m) return NULL;
    m->nv = nv; m->nt = nt; m->n = nv - 4;
    m->vx = vx; m->tv = tv; m->tn = tn;
    m->pos = malloc((size_t)nt);
    m->pos_x = malloc((size_t)nt);
    m->cen = malloc(sizeof(double) * 3 * (size_t)nt);
    if (!m->pos || !m->pos_x || !m->cen) { orc_mesh_free(m); return NULL; }
    double oscr[NIF_ORIENT_SCRATCH];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int t = 0; t < nt; t++) {
        const int32_t *p = tv + 4 * (size_t)t;
        const double *P0 = V(m, p[0]), *P1 = V(m, p[1]), *P2 = V(m, p[2]), *P3 = V(m, p[3]);
        const double o = orc_orient(P0, P1, P2, P3);
        m->pos[t] = o > 0;
        m->pos_x[t] = m->pos[t];
        if (nif_orient_uncertain(o, nif_orient_permanent(P0, P1, P2, P3))) {
            m->orient_unc++;
            m->pos_x[t] = nif_orient_exact_sign(P0, P1, P2, P3, oscr) > 0;
            if (m->pos_x[t] != m->pos[t]) m->orient_flip++;
        }
        for (int d = 0; d < 3; d++) {
            double c = (V(m, p[0])[d] + V(m, p[1])[d] + V(m, p[2])[d] + V(m, p[3])[d]) / 4;
            m->cen[3 * (size_t)t + d] = c;
            if (c < lo[d]) lo[d] = c;
            if (c > hi[d]) hi[d] = c;
        }
    }
    /* about two centroids per cell */
    double ext[3], vol = 1.0;
    for (int d = 0; d < 3; d++) {
        ext[d] = hi[d] - lo[d];
        if (!(ext[d] > 0)) ext[d] = 1.0;
        vol *= ext[d];
    }
    double side = cbrt(vol / (nt / 2.0 + 1.0));
    for (int d = 0; d < 3; d++) {
        int g = (int)(ext[d] / side) + 1;
        if (g > 1024) g = 1024;
        m->g[d] = g;
        m->lo[d] = lo[d];
        m->h[d] = ext[d] / g;
    }
    size_t ncell = (size_t)m->g[0] * m->g[1] * m->g[2];
    m->cell_start = calloc(ncell + 1, sizeof(int));
    m->cell_items = malloc(sizeof(int) * (size_t)nt);
    if (!m->cell_start || !m->cell_items) { orc_mesh_free(m); return NULL; }
    int *cid = malloc(sizeof(int) * (size_t)nt);
    if (!cid) { orc_mesh_free(m); return NULL; }
    for (int t = 0; t < nt; t++) {
        const double *c = m->cen + 3 * (size_t)t;
        int cx = cell_coord(m, 0, c[0]), cy = cell_coord(m, 1, c[1]), cz = cell_coord(m, 2, c[2]);
        cid[t] = (cz * m->g[1] + cy) * m->g[0] + cx;
        m->cell_start[cid[t] + 1]++;
    }
    for (size_t i = 0; i < ncell; i++) m->cell_start[i + 1] += m->cell_start[i];
    int *fill = malloc(sizeof(int) * ncell);
    if (!fill) { free(cid); orc_mesh_free(m); return NULL; }
    memcpy(fill, m->cell_start, sizeof(int) * ncell);
    for (int t = 0; t < nt; t++) m->cell_items[fill[cid[t]]++] = t; /* ascending tet id per cell */
    free(fill);
    free(cid);
    return m;
}

/* Squared distance as kd_nearest_i computes it (kdtree.c:411-414). */
static inline double cen_d2(const orc_mesh *m, int t, const double *q) {
    const double *c = m->cen + 3 * (size_t)t;
    double dx = c[0] - q[0], dy = c[1] - q[1], dz = c[2] - q[2];
    return dx * dx + dy * dy + dz * dz;
}

/* Exact nearest tet centroid (the seed natinterp3d's k-d tree returns). */
static int nearest_centroid(const orc_mesh *m, const double *q) {
    int c0[3];
    for (int d = 0; d < 3; d++) c0[d] = cell_coord(m, d, q[d]);
    int best = -1;
    double bd = INFINITY;
    int gmax = m->g[0];
    if (m->g[1] > gmax) gmax = m->g[1];
    if (m->g[2] > gmax) gmax = m->g[2];
    for (int r = 0; r <= gmax; r++) {
        int lo[3], hi[3];
        for (int d = 0; d < 3; d++) {
            lo[d] = c0[d] - r < 0 ? 0 : c0[d] - r;
            hi[d] = c0[d] + r >= m->g[d] ? m->g[d] - 1 : c0[d] + r;
        }
        for (int z = lo[2]; z <= hi[2]; z++)
            for (int y = lo[1]; y <= hi[1]; y++)
                for (int x = lo[0]; x <= hi[0]; x++) {
                    int cheb = abs(x - c0[0]);
                    if (abs(y - c0[1]) > cheb) cheb = abs(y - c0[1]);
                    if (abs(z - c0[2]) > cheb) cheb = abs(z - c0[2]);
                    if (cheb != r) continue;
                    int cell = (z * m->g[1] + y) * m->g[0] + x;
                    for (int k = m->cell_start[cell]; k < m->cell_start[cell + 1]; k++) {
                        int t = m->cell_items[k];
                        double d2 = cen_d2(m, t, q);
                        if (d2 < bd || (d2 == bd && t < best)) { bd = d2; best = t; }
                    }
                }
        /* distance from q to any cell outside the searched block */
        double lb = INFINITY;
        int open = 0;
        for (int d = 0; d < 3; d++) {
            double qd = q[d];
            double blo = m->lo[d] + lo[d] * m->h[d], bhi = m->lo[d] + (hi[d] + 1) * m->h[d];
            if (qd < blo) qd = blo;
            if (qd > bhi) qd = bhi;
            if (lo[d] > 0) { open = 1; if (qd - blo < lb) lb = qd - blo; }
            if (hi[d] < m->g[d] - 1) { open = 1; if (bhi - qd < lb) lb = bhi - qd; }
        }
        if (!open) break;
        if (best >= 0 && lb * lb > bd * (1.0 + 1e-12)) break;
    }
    return best;
}

/* ------------------------------------------------------------------------- */
/* Per-query scratch                                                          */
/* ------------------------------------------------------------------------- */

typedef struct { int *a; int n, cap; } ivec;
static int ipush(ivec *v, int x) {
    if (v->n == v->cap) {
        int nc = v->cap ? 2 * v->cap : 64;
        int *na = realloc(v->a, sizeof(int) * nc);
        if (!na) return -1;
        v->a = na; v->cap = nc;
    }
    v->a[v->n++] = x;
    return 0;
}

typedef struct { int k[3]; v3 cc; int used; } fcc_entry;

typedef struct {
    unsigned *tet_seen;   /* generation stamps, per tet: tested */
    unsigned *tet_cav;    /* generation stamps, per tet: in cavity */
    unsigned gen;
    int *slot_of;         /* [nv] vertex -> neighbour slot, -1 when absent */
    ivec stack, cavity, bface_t, bface_f, nbr;
    double *stolen;
    int stolen_cap;
    fcc_entry *fcc;
    int fcc_size;
    double *xs;           /* exact-predicate scratch, NIF_EXACT_SCRATCH doubles */
} orc_scratch;

static void scratch_free(orc_scratch *s) {
    free(s->tet_seen); free(s->tet_cav); free(s->slot_of);
    free(s->stack.a); free(s->cavity.a); free(s->bface_t.a); free(s->bface_f.a); free(s->nbr.a);
    free(s->stolen); free(s->fcc); free(s->xs);
}

static int scratch_init(orc_scratch *s, const orc_mesh *m) {
    memset(s, 0, sizeof(*s));
    s->tet_seen = calloc((size_t)m->nt, sizeof(unsigned));
    s->tet_cav = calloc((size_t)m->nt, sizeof(unsigned));
    s->slot_of = malloc(sizeof(int) * (size_t)m->nv);
    s->xs = malloc(sizeof(double) * NIF_EXACT_SCRATCH);
    if (!s->tet_seen || !s->tet_cav || !s->slot_of || !s->xs) return -1;
    for (int i = 0; i < m->nv; i++) s->slot_of[i] = -1;
    s->gen = 0;
    return 0;
}

/* face circumcentre cache keyed by the sorted vertex-id triple, computed with
 * the argument order of the first lookup (natural_insertionfree.c:233-253) */
static const v3 *fcc_lookup(orc_scratch *s, const orc_mesh *m, int a, int b, int c) {
    int k[3] = {a, b, c};
    if (k[0] > k[1]) { int t = k[0]; k[0] = k[1]; k[1] = t; }
    if (k[1] > k[2]) { int t = k[1]; k[1] = k[2]; k[2] = t; }
    if (k[0] > k[1]) { int t = k[0]; k[0] = k[1]; k[1] = t; }
    uint64_t h = (uint64_t)k[0] * 0x9e3779b97f4a7c15ULL ^ (uint64_t)k[1] * 0xc2b2ae3d27d4eb4fULL ^
                 (uint64_t)k[2] * 0x165667b19e3779f9ULL;
    int mask = s->fcc_size - 1;
    int i = (int)(h & (uint64_t)mask);
    for (;;) {
        fcc_entry *e = &s->fcc[i];
        if (!e->used) {
            e->used = 1;
            e->k[0] = k[0]; e->k[1] = k[1]; e->k[2] = k[2];
            e->cc = tri_cc(ld(V(m, a)), ld(V(m, b)), ld(V(m, c)));
            return &e->cc;
        }
        if (e->k[0] == k[0] && e->k[1] == k[1] && e->k[2] == k[2]) return &e->cc;
        i = (i + 1) & mask;
    }
}

typedef struct {
    long queries, walk_steps, insphere, cavity, boundary, neighbours;
    long old_terms, new_terms, face_cc, coincident, outside, empty, errors;
    long orient_unc, orient_flip, insphere_unc, insphere_flip;
} orc_stats;

/* Sign of orient3d(a, b, c, q) under the mesh's predicate mode.  Counts the
 * evaluation in st (when non-NULL) if the filter cannot certify it. */
static int pred_orient(const orc_mesh *m, orc_scratch *s, orc_stats *st, const double *a,
                       const double *b, const double *c, const double *q) {
    const double o = orc_orient(a, b, c, q);
    const int fs = o > 0 ? 1 : (o < 0 ? -1 : 0);
    if (m->pmode == ORC_PRED_FAST || !nif_orient_uncertain(o, nif_orient_permanent(a, b, c, q)))
        return fs;
    const int xs = nif_orient_exact_sign(a, b, c, q, s->xs);
    if (st) {
        st->orient_unc++;
        if ((xs < 0) != (fs < 0)) st->orient_flip++;
    }
    return m->pmode == ORC_PRED_EXACT ? xs : fs;
}

/* "inside the circumsphere" decision for tet t (inspherefast(...) > 0 with
 * the argument order fixed by the tet's orientation,
 * natural_insertionfree.c:511-515) under the mesh's predicate mode */
static int pred_in_cavity(const orc_mesh *m, orc_scratch *s, orc_stats *st, int t,
                          const double *q) {
    const int32_t *p = m->tv + 4 * (size_t)t;
    const int pos = m->pmode == ORC_PRED_EXACT ? m->pos_x[t] : m->pos[t];
    const double *a = V(m, pos ? p[0] : p[1]), *b = V(m, pos ? p[1] : p[0]);
    const double *c = V(m, p[2]), *d = V(m, p[3]);
    const double v = orc_insphere(a, b, c, d, q);
    if (m->pmode == ORC_PRED_FAST || !nif_insphere_uncertain(v, nif_insphere_permanent(a, b, c, d, q)))
        return v > 0;
    const int xs = nif_insphere_exact_sign(a, b, c, d, q, s->xs);
    if (st) {
        st->insphere_unc++;
        if ((xs > 0) != (v > 0)) st->insphere_flip++;
    }
    return m->pmode == ORC_PRED_EXACT ? xs > 0 : v > 0;
}

/* findContainingSimplex, delaunay.c:383-407 (walk with the first face whose
 * orient3d is negative, restarting from face 0 after every step).  Returns
 * the tet, -1 outside the super-simplex, -2 on step-limit; *on_face is set
 * when a face test of the final tet came out exactly zero. */
static int locate(const orc_mesh *m, const double *q, long *steps, orc_scratch *s,
                  orc_stats *st, int *on_face) {
    int t = m->seed_first ? 0 : nearest_centroid(m, q);
    long cap = 4L * m->nt + 1024;
    *on_face = 0;
    for (long it = 0; it < cap; it++) {
        const int32_t *p = m->tv + 4 * (size_t)t;
        int f = 0, zero = 0;
        for (; f < 4; f++) {
            const int sg = pred_orient(m, s, st, V(m, p[FACE3[f][0]]), V(m, p[FACE3[f][1]]),
                                       V(m, p[FACE3[f][2]]), q);
            if (sg < 0) break;
            if (sg == 0) zero = 1;
        }
        if (f == 4) { if (steps) *steps += it + 1; *on_face = zero; return t; }
        int nb = m->tn[4 * (size_t)t + f];
        if (nb < 0) { if (steps) *steps += it + 1; return -1; }
        t = nb;
    }
    return -2;
}

/* 1 if q lies in the closed tet t (every face test >= 0), exact-mode signs */
static int tet_contains(const orc_mesh *m, orc_scratch *s, int t, const double *q) {
    const int32_t *p = m->tv + 4 * (size_t)t;
    for (int f = 0; f < 4; f++)
        if (pred_orient(m, s, NULL, V(m, p[FACE3[f][0]]), V(m, p[FACE3[f][1]]),
                        V(m, p[FACE3[f][2]]), q) < 0)
            return 0;
    return 1;
}

static int slot_add(orc_scratch *s, int vid) {
    if (s->slot_of[vid] >= 0) return s->slot_of[vid];
    int slot = s->nbr.n;
    if (ipush(&s->nbr, vid)) return -1;
    if (slot >= s->stolen_cap) {
        int nc = s->stolen_cap ? 2 * s->stolen_cap : 64;
        while (nc <= slot) nc *= 2;
        double *ns = realloc(s->stolen, sizeof(double) * nc);
        if (!ns) return -1;
        s->stolen = ns; s->stolen_cap = nc;
    }
    s->stolen[slot] = 0.0;
    s->slot_of[vid] = slot;
    return slot;
}

/* getWeightsSingleQueryIF, natural_insertionfree.c:591-738.  Leaves the row
 * in s->nbr / s->stolen (neighbour count s->nbr.n).  Returns 0 or an error. */
/* findCavity (natural_insertionfree.c:486-551): LIFO flood from start; a tet
 * joins the cavity iff it passes the in-sphere decision; neighbours are
 * pushed in slot order 0..3.  Evaluations are counted in st when non-NULL. */
static int flood(const orc_mesh *m, const double *q, orc_scratch *s, orc_stats *st, int start) {
    if (++s->gen == 0) {
        memset(s->tet_seen, 0, sizeof(unsigned) * (size_t)m->nt);
        memset(s->tet_cav, 0, sizeof(unsigned) * (size_t)m->nt);
        s->gen = 1;
    }
    const unsigned g = s->gen;
    s->cavity.n = 0;
    s->stack.n = 0;
    if (ipush(&s->stack, start)) return ORC_ERR_NOMEM;
    while (s->stack.n > 0) {
        int t = s->stack.a[--s->stack.n];
        if (s->tet_seen[t] == g) continue;
        s->tet_seen[t] = g;
        if (st) st->insphere++;
        if (pred_in_cavity(m, s, st, t, q)) {
            if (ipush(&s->cavity, t)) return ORC_ERR_NOMEM;
            s->tet_cav[t] = g;
            for (int i = 0; i < 4; i++) {
                int nb = m->tn[4 * (size_t)t + i];
                if (nb >= 0 && s->tet_seen[nb] != g)
                    if (ipush(&s->stack, nb)) return ORC_ERR_NOMEM;
            }
        }
    }
    return ORC_OK;
}

/* getWeightsSingleQueryIF, natural_insertionfree.c:591-738.  Leaves the row
 * in s->nbr / s->stolen (neighbour count s->nbr.n).  Returns 0 or an error. */
static int query_one(const orc_mesh *m, const double *q, orc_scratch *s, orc_stats *st) {
    for (int i = 0; i < s->nbr.n; i++) s->slot_of[s->nbr.a[i]] = -1;
    s->nbr.n = 0;
    s->cavity.n = 0;
    s->bface_t.n = 0;
    s->bface_f.n = 0;

    long steps = 0;
    int on_face = 0;
    int start = locate(m, q, &steps, s, st, &on_face);
    st->walk_steps += steps;
    if (start == -2) { st->errors++; return ORC_ERR_WALK; }
    if (start == -1) { st->outside++; return ORC_OK; }

    int rc = flood(m, q, s, st, start);
    if (rc) return rc;
    if (m->pmode == ORC_PRED_EXACT && on_face && s->cavity.n > 0) {
        /* canonical start: the lowest-id cavity tet that contains q */
        int best = -1;
        for (int ci = 0; ci < s->cavity.n; ci++) {
            const int t = s->cavity.a[ci];
            if ((best < 0 || t < best) && tet_contains(m, s, t, q)) best = t;
        }
        if (best >= 0 && best != start) {
            start = best;
            rc = flood(m, q, s, NULL, start);
            if (rc) return rc;
        }
    }
    const unsigned g = s->gen;
    st->cavity += s->cavity.n;

    if (s->cavity.n == 0) {
        /* coincident-vertex path, natural_insertionfree.c:596-622 */
        const int32_t *p = m->tv + 4 * (size_t)start;
        int coin[4], nc = 0;
        for (int i = 0; i < 4; i++) {
            const double *pv = V(m, p[i]);
            if (p[i] < m->n && pv[0] == q[0] && pv[1] == q[1] && pv[2] == q[2]) coin[nc++] = p[i];
        }
        if (nc > 0) {
            double w = 1.0 / nc;
            for (int i = 0; i < nc; i++) {
                int slot = slot_add(s, coin[i]);
                if (slot < 0) return ORC_ERR_NOMEM;
                s->stolen[slot] = w;
            }
            st->coincident++;
        } else {
            st->empty++;
        }
        return ORC_OK;
    }

    /* extractBoundaryAndNeighbors, natural_insertionfree.c:559-584 */
    for (int ci = 0; ci < s->cavity.n; ci++) {
        int t = s->cavity.a[ci];
        const int32_t *p = m->tv + 4 * (size_t)t;
        for (int f = 0; f < 4; f++) {
            int nb = m->tn[4 * (size_t)t + f];
            if (nb < 0 || s->tet_cav[nb] != g) {
                if (ipush(&s->bface_t, t) || ipush(&s->bface_f, f)) return ORC_ERR_NOMEM;
                for (int j = 0; j < 3; j++) {
                    int vid = p[FACE3[f][j]];
                    if (vid < m->n && slot_add(s, vid) < 0) return ORC_ERR_NOMEM;
                }
            }
        }
    }
    st->boundary += s->bface_t.n;
    if (s->nbr.n == 0) { st->empty++; return ORC_OK; }
    st->neighbours += s->nbr.n;

    /* face circumcentre cache sized like natural_insertionfree.c:629-636 */
    int need = 4 * s->cavity.n, size = 16;
    while (need * 4 >= size * 3) size *= 2;
    if (size > s->fcc_size) {
        free(s->fcc);
        s->fcc = malloc(sizeof(fcc_entry) * size);
        if (!s->fcc) { s->fcc_size = 0; return ORC_ERR_NOMEM; }
        s->fcc_size = size;
    }
    for (int i = 0; i < s->fcc_size; i++) s->fcc[i].used = 0;

    /* old contributions: cavity tets, natural_insertionfree.c:642-676 */
    for (int ci = 0; ci < s->cavity.n; ci++) {
        int t = s->cavity.a[ci];
        const int32_t *p = m->tv + 4 * (size_t)t;
        v3 P[4] = {ld(V(m, p[0])), ld(V(m, p[1])), ld(V(m, p[2])), ld(V(m, p[3]))};
        v3 ct = tet_cc(P[0], P[1], P[2], P[3]);
        const v3 *fcc[4];
        fcc[0] = fcc_lookup(s, m, p[1], p[2], p[3]);
        fcc[1] = fcc_lookup(s, m, p[0], p[2], p[3]);
        fcc[2] = fcc_lookup(s, m, p[0], p[1], p[3]);
        fcc[3] = fcc_lookup(s, m, p[0], p[1], p[2]);
        for (int vi = 0; vi < 4; vi++) {
            if (p[vi] >= m->n) continue;
            int slot = s->slot_of[p[vi]];
            if (slot < 0) continue;
            int o[3], k = 0;
            for (int j = 0; j < 4; j++) if (j != vi) o[k++] = j; /* ascending */
            double vol = subcell(P[vi], P[o[0]], P[o[1]], P[o[2]], ct, *fcc[o[2]], *fcc[o[1]], *fcc[o[0]]);
            s->stolen[slot] += vol;
            st->old_terms++;
        }
    }

    /* new contributions: virtual tets (query + boundary face), :681-719 */
    v3 Q = ld(q);
    for (int bi = 0; bi < s->bface_t.n; bi++) {
        int t = s->bface_t.a[bi], f = s->bface_f.a[bi];
        const int32_t *p = m->tv + 4 * (size_t)t;
        int fv[3] = {p[FACE3[f][0]], p[FACE3[f][1]], p[FACE3[f][2]]};
        v3 F[3] = {ld(V(m, fv[0])), ld(V(m, fv[1])), ld(V(m, fv[2]))};
        v3 cv = tet_cc(Q, F[0], F[1], F[2]);
        const v3 *cf = fcc_lookup(s, m, fv[0], fv[1], fv[2]);
        for (int k = 0; k < 3; k++) {
            if (fv[k] >= m->n) continue;
            int slot = s->slot_of[fv[k]];
            if (slot < 0) continue;
            int a = (k + 1) % 3, b = (k + 2) % 3;
            v3 cqa = tri_cc(F[k], Q, F[a]);
            v3 cqb = tri_cc(F[k], Q, F[b]);
            double vol = subcell(F[k], Q, F[a], F[b], cv, cqa, cqb, *cf);
            s->stolen[slot] -= vol;
            st->new_terms++;
        }
    }
    for (int i = 0; i < s->fcc_size; i++) st->face_cc += s->fcc[i].used;

    /* normalisation, :721-737 */
    double total = 0.0;
    for (int i = 0; i < s->nbr.n; i++) total += s->stolen[i];
    if (total > 1e-30) {
        double inv = 1.0 / total;
        for (int i = 0; i < s->nbr.n; i++) s->stolen[i] *= inv;
    } else {
        for (int i = 0; i < s->nbr.n; i++) s->slot_of[s->nbr.a[i]] = -1;
        s->nbr.n = 0;
        st->empty++;
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* CSR driver (natural_insertionfree.c:761-831): rows in query order, columns */
/* in first-seen order, int32 row pointers, nnz > INT32_MAX -> error.         */
/* ------------------------------------------------------------------------- */

void orc_free(void *p) { free(p); }

/* queries: [M][3] centred float64.  rowptr: caller-provided int32[M+1].
 * *vals / *cols are malloc'd here (free with orc_free).  status (optional,
 * int8[M]) receives 0 or the per-row error.  stats (optional) gets counters
 * as 17 int64 values in orc_stats order. */
int orc_weights(const orc_mesh *m, const double *queries, int M, double **vals, int **cols,
                int *rowptr, signed char *status, long *stats) {
    if (!m || (!queries && M > 0) || M < 0 || !vals || !cols || !rowptr) return ORC_ERR_ARG;
    orc_scratch s;
    if (scratch_init(&s, m)) { scratch_free(&s); return ORC_ERR_NOMEM; }
    orc_stats st;
    memset(&st, 0, sizeof(st));
    size_t cap = 1024, used = 0;
    double *dv = malloc(sizeof(double) * cap);
    int *dc = malloc(sizeof(int) * cap);
    int rc = ORC_OK;
    if (!dv || !dc) rc = ORC_ERR_NOMEM;
    for (int i = 0; i < M && rc == ORC_OK; i++) {
        int e = query_one(m, queries + 3 * (size_t)i, &s, &st);
        st.queries++;
        if (status) status[i] = (signed char)e;
        if (e == ORC_ERR_NOMEM) { rc = e; break; }
        int nc = (e == ORC_OK) ? s.nbr.n : 0;
        if (used > (size_t)INT32_MAX) { rc = ORC_ERR_OVERFLOW; break; }
        rowptr[i] = (int)used;
        if (used + nc > cap) {
            while (used + nc > cap) cap *= 2;
            double *ndv = realloc(dv, sizeof(double) * cap);
            int *ndc = realloc(dc, sizeof(int) * cap);
            if (ndv) dv = ndv;
            if (ndc) dc = ndc;
            if (!ndv || !ndc) { rc = ORC_ERR_NOMEM; break; }
        }
        for (int k = 0; k < nc; k++) {
            dv[used + k] = s.stolen[k];
            dc[used + k] = s.nbr.a[k];
        }
        used += nc;
    }
    if (rc == ORC_OK && used > (size_t)INT32_MAX) rc = ORC_ERR_OVERFLOW;
    if (rc == ORC_OK) rowptr[M] = (int)used;
    scratch_free(&s);
    if (rc != ORC_OK) { free(dv); free(dc); *vals = NULL; *cols = NULL; return rc; }
    *vals = dv;
    *cols = dc;
    if (stats) {
        long *o = stats;
        o[0] = st.queries; o[1] = st.walk_steps; o[2] = st.insphere; o[3] = st.cavity;
        o[4] = st.boundary; o[5] = st.neighbours; o[6] = st.old_terms; o[7] = st.new_terms;
        o[8] = st.face_cc; o[9] = st.coincident; o[10] = st.outside; o[11] = st.empty;
        o[12] = st.errors; o[13] = st.orient_unc; o[14] = st.orient_flip;
        o[15] = st.insphere_unc; o[16] = st.insphere_flip;
    }
    return ORC_OK;
}

/* Row-by-row weights @ values as scipy's csr_matvec(s) accumulates it
 * (y = 0; y += w_k * x[col_k] in stored order), on doubles. */
void orc_spmm(int M, int D, const int *rowptr, const int *cols, const double *vals,
              const double *x, double *y) {
    for (int i = 0; i < M; i++) {
        for (int d = 0; d < D; d++) {
            double acc = 0.0;
            for (int k = rowptr[i]; k < rowptr[i + 1]; k++) acc += vals[k] * x[(size_t)cols[k] * D + d];
            y[(size_t)i * D + d] = acc;
        }
    }
}

/* Per-tet quantities the GPU precomputes once per mesh, for cross-checks:
 * orientation flag, tet circumcentre, and the four face circumcentres
 * (face opposite p[i], vertices in ascending slot order). */
void orc_tet_geometry(const orc_mesh *m, unsigned char *pos, double *tcc, double *fcc) {
    for (int t = 0; t < m->nt; t++) {
        const int32_t *p = m->tv + 4 * (size_t)t;
        v3 P[4] = {ld(V(m, p[0])), ld(V(m, p[1])), ld(V(m, p[2])), ld(V(m, p[3]))};
        if (pos) pos[t] = m->pos[t];
        if (tcc) {
            v3 c = tet_cc(P[0], P[1], P[2], P[3]);
            tcc[3 * (size_t)t] = c.x; tcc[3 * (size_t)t + 1] = c.y; tcc[3 * (size_t)t + 2] = c.z;
        }
        if (fcc) {
            for (int i = 0; i < 4; i++) {
                int o[3], k = 0;
                for (int j = 0; j < 4; j++) if (j != i) o[k++] = j;
                v3 c = tri_cc(P[o[0]], P[o[1]], P[o[2]]);
                double *out = fcc + 12 * (size_t)t + 3 * i;
                out[0] = c.x; out[1] = c.y; out[2] = c.z;
            }
        }
    }
}

/* predicate mode of later orc_weights calls: ORC_PRED_FAST/AUDIT/EXACT */
int orc_mesh_set_predicates(orc_mesh *m, int mode) {
    if (!m || mode < ORC_PRED_FAST || mode > ORC_PRED_EXACT) return ORC_ERR_ARG;
    m->pmode = mode;
    return ORC_OK;
}

/* walk seed of later orc_weights calls: 0 nearest tet centroid (natinterp3d's
 * k-d tree seed, the default), 1 tet 0 (natinterp3d without a k-d tree) */
int orc_mesh_set_seed(orc_mesh *m, int first_tet) {
    if (!m) return ORC_ERR_ARG;
    m->seed_first = first_tet != 0;
    return ORC_OK;
}

/* tets whose orientation sign the filter could not certify, and those whose
 * "orient3d > 0" flag the exact sign changes */
void orc_mesh_predicate_info(const orc_mesh *m, long out[2]) {
    out[0] = m->orient_unc;
    out[1] = m->orient_flip;
}

/* the exact arithmetic and filters on their own, for known-answer tests */
int orc_orient_exact_sign(const double *a, const double *b, const double *c, const double *d) {
    double s[NIF_ORIENT_SCRATCH];
    return nif_orient_exact_sign(a, b, c, d, s);
}

int orc_insphere_exact_sign(const double *a, const double *b, const double *c, const double *d,
                            const double *e) {
    double *s = malloc(sizeof(double) * NIF_EXACT_SCRATCH);
    if (!s) return -2;
    int r = nif_insphere_exact_sign(a, b, c, d, e, s);
    free(s);
    return r;
}

int orc_orient_uncertain(const double *a, const double *b, const double *c, const double *d) {
    return nif_orient_uncertain(orc_orient(a, b, c, d), nif_orient_permanent(a, b, c, d));
}

int orc_insphere_uncertain(const double *a, const double *b, const double *c, const double *d,
                           const double *e) {
    return nif_insphere_uncertain(orc_insphere(a, b, c, d, e),
                                  nif_insphere_permanent(a, b, c, d, e));
}

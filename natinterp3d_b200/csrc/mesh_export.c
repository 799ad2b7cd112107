/*
 * Host-side Delaunay construction and export for natinterp3d_b200.
 *
 * The tetrahedralization is still built by natinterp3d's own incremental
 * Bowyer-Watson constructor (buildNewMeshAndVertices, natural.c:114-118 of the
 * natinterp3d sources, which calls buildMesh in delaunay.c:108-161).  This
 * translation unit is compiled against those sources (the build recipe puts
 * the natinterp3d source directory on the include path); everything below the
 * includes is the exporter that flattens the pointer-linked mesh into the
 * packed index arrays that are uploaded to the GPU once per key set.
 *
 * Packed layout written by nif_mesh_export (all little-endian, C order):
 *   vxyz  [V][3] float64  V = N + 4.  Rows 0..N-1 are the mesh's data vertices
 *                         (index i of the caller's keys, possibly perturbed by
 *                         the constructor, delaunay.c:513-522); rows N..N+3 are
 *                         the super-simplex vertices whose reference index is
 *                         -1..-4 (delaunay.c:859).
 *   tet_v [T][4] int32    vertex ids of p[0..3] (delaunay.h:60).
 *   tet_n [T][4] int32    tet ids of s[0..3] (delaunay.h:64), -1 for NULL.
 * Tets are numbered in the order of the mesh's tet list, which is the order
 * natinterp3d packs them in (natural_insertionfree.c:413-425) and the order
 * its k-d tree of tet centroids is filled in (delaunay.c:151-159).
 */
#define UNITY_BUILD
#include "utils.c"
#include "kdtree.c"
#include "delaunay.c"
#include "natural.c"

#include <stdint.h>

#define NIF_API __attribute__((visibility("default")))

#define NIF_OK 0
#define NIF_ERR_ARG -1
#define NIF_ERR_DEGENERATE -2
#define NIF_ERR_NOMEM -3
#define NIF_ERR_INTERNAL -4

typedef struct nif_mesh {
    mesh *m;
    vertex *ps;
    int n;         /* data vertices */
    int n_tets;
} nif_mesh;

/* pointer -> tet index map (open addressing, power-of-two table) */
typedef struct {
    const void **keys;
    int *vals;
    size_t mask;
} ptr_map;

static size_t ptr_hash(const void *p) {
    uint64_t v = (uint64_t)(uintptr_t)p;
    v ^= v >> 33;
    v *= 0xff51afd7ed558ccdULL;
    v ^= v >> 29;
    return (size_t)v;
}

static int ptr_map_init(ptr_map *pm, size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 2) cap <<= 1;
    pm->keys = calloc(cap, sizeof(void *));
    pm->vals = malloc(cap * sizeof(int));
    pm->mask = cap - 1;
    return (pm->keys && pm->vals) ? 0 : -1;
}

static void ptr_map_put(ptr_map *pm, const void *k, int v) {
    size_t h = ptr_hash(k) & pm->mask;
    while (pm->keys[h] && pm->keys[h] != k) h = (h + 1) & pm->mask;
    pm->keys[h] = k;
    pm->vals[h] = v;
}

static int ptr_map_get(const ptr_map *pm, const void *k) {
    size_t h = ptr_hash(k) & pm->mask;
    while (pm->keys[h]) {
        if (pm->keys[h] == k) return pm->vals[h];
        h = (h + 1) & pm->mask;
    }
    return -1;
}

static void ptr_map_free(ptr_map *pm) {
    free(pm->keys);
    free(pm->vals);
}

/* The constructor divides by the data range and needs a non-flat
 * super-simplex (delaunay.c:832-863); a key set with zero extent along an
 * axis makes it call exit(1) from isDelaunay (delaunay.c:538-542).  Reject
 * such inputs up front so the host process survives. */
static int keys_are_buildable(const double *keys, int n) {
    if (n < 1) return 0;
    for (int d = 0; d < 3; d++) {
        double lo = keys[d], hi = keys[d];
        for (int i = 0; i < n; i++) {
            double x = keys[3 * i + d];
            if (!isfinite(x)) return 0;
            if (x < lo) lo = x;
            if (x > hi) hi = x;
        }
        if (!(hi - lo > 0.0) || !isfinite(hi - lo)) return 0;
    }
    return 1;
}

NIF_API int nif_mesh_build(const double *keys_centered, int n, nif_mesh **out) {
    if (!keys_centered || !out || n < 1) return NIF_ERR_ARG;
    *out = NULL;
    if (!keys_are_buildable(keys_centered, n)) return NIF_ERR_DEGENERATE;
    nif_mesh *h = calloc(1, sizeof(nif_mesh));
    if (!h) return NIF_ERR_NOMEM;
    buildNewMeshAndVertices((double *)keys_centered, n, &h->m, &h->ps);
    h->n = n;
    h->n_tets = getNumSimplicies(h->m);
    *out = h;
    return NIF_OK;
}

NIF_API void nif_mesh_free(nif_mesh *h) {
    if (!h) return;
    if (h->m) freeMeshAndVertices(h->m, h->ps);
    free(h);
}

NIF_API int nif_mesh_sizes(const nif_mesh *h, int *n_vertices, int *n_tets) {
    if (!h || !n_vertices || !n_tets) return NIF_ERR_ARG;
    *n_vertices = h->n + 4;
    *n_tets = h->n_tets;
    return NIF_OK;
}

static int vertex_id(const nif_mesh *h, const vertex *p) {
    return p->index >= 0 ? p->index : h->n + (-1 - p->index);
}

NIF_API int nif_mesh_export(const nif_mesh *h, double *vxyz, int32_t *tet_v, int32_t *tet_n) {
    if (!h || !vxyz || !tet_v || !tet_n) return NIF_ERR_ARG;
    const int n = h->n;
    for (int i = 0; i < n; i++) {
        vxyz[3 * i + 0] = h->ps[i].v[0];
        vxyz[3 * i + 1] = h->ps[i].v[1];
        vxyz[3 * i + 2] = h->ps[i].v[2];
    }
    for (int k = 0; k < 4; k++) {
        const vertex *sv = &h->m->superVerticies[k];
        if (sv->index != -1 - k) return NIF_ERR_INTERNAL;
        vxyz[3 * (n + k) + 0] = sv->v[0];
        vxyz[3 * (n + k) + 1] = sv->v[1];
        vxyz[3 * (n + k) + 2] = sv->v[2];
    }

    ptr_map pm;
    if (ptr_map_init(&pm, (size_t)h->n_tets) != 0) {
        ptr_map_free(&pm);
        return NIF_ERR_NOMEM;
    }
    listNode *iter = topOfLinkedList(h->m->tets);
    simplex *s;
    int t = 0;
    while ((s = nextElement(h->m->tets, &iter))) {
        ptr_map_put(&pm, s, t);
        t++;
    }
    if (t != h->n_tets) {
        ptr_map_free(&pm);
        return NIF_ERR_INTERNAL;
    }
    iter = topOfLinkedList(h->m->tets);
    t = 0;
    int rc = NIF_OK;
    while ((s = nextElement(h->m->tets, &iter))) {
        for (int j = 0; j < 4; j++) {
            tet_v[4 * t + j] = vertex_id(h, s->p[j]);
            if (s->s[j]) {
                int nb = ptr_map_get(&pm, s->s[j]);
                if (nb < 0) rc = NIF_ERR_INTERNAL;
                tet_n[4 * t + j] = nb;
            } else {
                tet_n[4 * t + j] = -1;
            }
        }
        t++;
    }
    ptr_map_free(&pm);
    return rc;
}

/* Degeneracy counters kept by the constructor (delaunay.c:106-107, 588, 649). */
NIF_API int nif_mesh_degeneracies(const nif_mesh *h, int *coplanar, int *cospherical) {
    if (!h || !coplanar || !cospherical) return NIF_ERR_ARG;
    *coplanar = h->m->coplanar_degenerecies;
    *cospherical = h->m->cospherical_degenerecies;
    return NIF_OK;
}

/* The natinterp3d mesh object itself; only the CPU checker uses it, to run
 * natinterp3d's own query code on exactly the mesh that was exported. */
NIF_API void *nif_mesh_native(const nif_mesh *h) {
    return h ? (void *)h->m : NULL;
}

/*
 * Test infrastructure only: a thin C shim around natinterp3d's own sources so
 * that the CPU checker and the timed CPU baseline can run natinterp3d's query
 * code unchanged.  The recipe in oracle/build_oracle.py compiles this file
 * with natinterp3d's unity translation unit (unity.c) on the include path and
 * natinterp3d's setup.py flags; the product never loads the result.
 *
 * Entry points mirror natinterp3d's C ABI:
 *   ref_build  -> buildNewMeshAndVertices        (natural.c:114-118)
 *   ref_free   -> freeMeshAndVertices            (natural.c:120-123)
 *   ref_query  -> getInsertionFreeWeights[Parallel]
 *                                                (natural_insertionfree.c:761-831, 836-940)
 *   ref_orient3d_robust / ref_insphere_robust -> Shewchuk's adaptive exact
 *                orient3d / insphere (predicates.c:2294, 4160), which
 *                natinterp3d ships but never calls; they pin the product's
 *                exact predicates
 * ref_query also accepts a mesh built by the product's constructor library
 * (same natinterp3d sources, same flags, hence the same struct layout), which
 * is how the checker runs natinterp3d's query on exactly the exported mesh.
 */
#include "unity.c"

#define REF_API __attribute__((visibility("default")))

REF_API int ref_build(const double *keys, int n, void **mesh_out, void **verts_out) {
    mesh *m = NULL;
    vertex *ps = NULL;
    buildNewMeshAndVertices((double *)keys, n, &m, &ps);
    *mesh_out = m;
    *verts_out = ps;
    return 0;
}

REF_API void ref_free(void *m, void *ps) {
    freeMeshAndVertices((mesh *)m, (vertex *)ps);
}

REF_API int ref_num_tets(void *m) {
    return getNumSimplicies((mesh *)m);
}

/* nthreads <= 0 selects the serial driver, as MeshAndVertices does. */
REF_API int ref_query(void *m, const double *queries, int num_queries, int nthreads,
              int num_keys, double **vals, int **cols, int *rowptr) {
    if (nthreads <= 0)
        return getInsertionFreeWeights((double *)queries, num_queries, (mesh *)m,
                                       num_keys, vals, cols, rowptr);
    return getInsertionFreeWeightsParallel((double *)queries, num_queries, (mesh *)m,
                                           nthreads, num_keys, vals, cols, rowptr);
}

REF_API void ref_free_buffer(void *p) {
    free(p);
}

static int ref_exact_ready = 0;

/* the adaptive predicates need exactinit() once (predicates.c:646) */
REF_API double ref_orient3d_robust(const double *a, const double *b, const double *c,
                                   const double *d) {
    if (!ref_exact_ready) {
        exactinit();
        ref_exact_ready = 1;
    }
    return orient3d((double *)a, (double *)b, (double *)c, (double *)d);
}

REF_API double ref_insphere_robust(const double *a, const double *b, const double *c,
                                   const double *d, const double *e) {
    if (!ref_exact_ready) {
        exactinit();
        ref_exact_ready = 1;
    }
    return insphere((double *)a, (double *)b, (double *)c, (double *)d, (double *)e);
}

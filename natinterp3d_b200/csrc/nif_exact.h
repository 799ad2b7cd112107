/*
 * Exact signs of the orient3d and insphere determinants for double inputs,
 * and the static error-bound filters that decide when the plain
 * floating-point value already has the right sign.  Compiles as C (the CPU
 * oracle) and as CUDA host/device code (the row kernels).
 *
 * Method: floating-point expansion arithmetic (J. R. Shewchuk, "Adaptive
 * Precision Floating-Point Arithmetic and Fast Robust Geometric Predicates",
 * Discrete & Computational Geometry 18:305-363, 1997).  A real number is held
 * as a sum of non-overlapping doubles sorted by increasing magnitude; sums
 * and products are formed without rounding error (Two-Sum; Two-Product via a
 * fused multiply-add), expansions are added with the paper's
 * Linear-Expansion-Sum, scaled with Scale-Expansion and shortened with
 * Compress, all with zero elimination.  The sign of an expansion is the sign
 * of its largest component.  The determinants are expanded in homogeneous
 * form, so no coordinate difference is ever rounded:
 *   orient3d(a,b,c,d) = det3(a,b,c) - det3(a,b,d) + det3(a,c,d) - det3(b,c,d)
 *   insphere(a,b,c,d,e) = sum_i (-1)^(i+1) |p_i|^2 orient3d(the other four)
 * with p = (a,b,c,d,e), i = 0..4; both are the exact values of what
 * orient3dfast and inspherefast evaluate in floating point.
 *
 * Filters: the paper's forward error bounds for exactly the evaluation
 * orders of orient3dfast and inspherefast,
 *   |fast - exact| <= (7 + 56 eps) eps * P_orient
 *   |fast - exact| <= (16 + 224 eps) eps * P_insphere,    eps = 2^-53,
 * P being the permanent: the same expression over absolute values.  When
 * |fast| exceeds the bound the fast sign is the exact sign.  Every operation
 * here must be a separately rounded IEEE double operation: compile with
 * -ffp-contract=off (C) or -fmad=false (CUDA).
 */
#ifndef NIF_EXACT_H
#define NIF_EXACT_H

#include <math.h>

#ifdef __CUDACC__
#define NIF_XI static __host__ __device__ __forceinline__
#define NIF_XF static __host__ __device__ __noinline__
#else
#define NIF_XI static inline
#define NIF_XF static __attribute__((unused))
#endif

#define NIF_EPS (1.0 / 9007199254740992.0) /* 2^-53, half an ulp of 1 */
#define NIF_O3D_BOUND ((7.0 + 56.0 * NIF_EPS) * NIF_EPS)
#define NIF_ISP_BOUND ((16.0 + 224.0 * NIF_EPS) * NIF_EPS)

/* Worst-case expansion lengths (no cancellation at all): 4 per two-product
 * difference, 24 per 3x3 determinant, 96 per orient3d, 6 per lift, 1152 per
 * lift * orient3d product, 5760 for the insphere sum.  Scratch in doubles: */
#define NIF_ORIENT_SCRATCH 288   /* nif_orient_exact_sign */
#define NIF_EXACT_SCRATCH 14112  /* nif_insphere_exact_sign */

/* ---- error-free transformations ----------------------------------------- */

/* a + b = *x + *y exactly, *x = fl(a + b) (Two-Sum; no magnitude precondition) */
NIF_XI void nif_two_sum(double a, double b, double *x, double *y) {
    const double s = a + b;
    const double bv = s - a;
    const double av = s - bv;
    *x = s;
    *y = (a - av) + (b - bv);
}

/* a * b = *x + *y exactly, *x = fl(a * b); the fused multiply-add yields the
 * rounding error of the product in one correctly rounded step */
NIF_XI void nif_two_prod(double a, double b, double *x, double *y) {
    const double p = a * b;
    *x = p;
    *y = fma(a, b, -p);
}

/* ---- expansion arithmetic (inputs non-overlapping, increasing magnitude) -- */

/* h = e + f (Linear-Expansion-Sum with zero elimination; Two-Sum in place of
 * the paper's Fast-Two-Sum, which gives the same outputs wherever the latter's
 * precondition holds).  Needs room for elen + flen components; returns the
 * length, >= 1 ([0] is zero). */
NIF_XF int nif_exp_sum(int elen, const double *e, int flen, const double *f, double *h) {
    int ei = 0, fi = 0, hi = 0;
    const int n = elen + flen;
    double g, g2, Q, q, R, hh;
    if (n == 0) {
        h[0] = 0.0;
        return 1;
    }
#define NIF_NEXT_G(out)                                                             \
    do {                                                                            \
        if (fi >= flen || (ei < elen && fabs(e[ei]) <= fabs(f[fi]))) out = e[ei++]; \
        else out = f[fi++];                                                         \
    } while (0)
    NIF_NEXT_G(g);
    if (n == 1) {
        h[0] = g;
        return 1;
    }
    NIF_NEXT_G(g2);
    nif_two_sum(g2, g, &Q, &q);
    for (int i = 2; i < n; i++) {
        NIF_NEXT_G(g);
        nif_two_sum(g, q, &R, &hh);
        if (hh != 0.0) h[hi++] = hh;
        nif_two_sum(Q, R, &Q, &q);
    }
#undef NIF_NEXT_G
    if (q != 0.0) h[hi++] = q;
    if (Q != 0.0 || hi == 0) h[hi++] = Q;
    return hi;
}

/* h = b * e (Scale-Expansion with zero elimination); room for 2 elen */
NIF_XF int nif_exp_scale(int elen, const double *e, double b, double *h) {
    double Q, hh, T, t, S;
    int hi = 0;
    nif_two_prod(e[0], b, &Q, &hh);
    if (hh != 0.0) h[hi++] = hh;
    for (int i = 1; i < elen; i++) {
        nif_two_prod(e[i], b, &T, &t);
        nif_two_sum(Q, t, &S, &hh);
        if (hh != 0.0) h[hi++] = hh;
        nif_two_sum(T, S, &Q, &hh);
        if (hh != 0.0) h[hi++] = hh;
    }
    if (Q != 0.0 || hi == 0) h[hi++] = Q;
    return hi;
}

/* Compress, in place: the same value, usually in far fewer components.  The
 * downward pass writes only above the index it reads, the upward pass only
 * below, so one array serves as input, intermediate and output. */
NIF_XF int nif_exp_compress(int m, double *e) {
    if (m <= 1) return m;
    double Q = e[m - 1], Qn, q;
    int bottom = m - 1;
    for (int i = m - 2; i >= 0; i--) {
        nif_two_sum(Q, e[i], &Qn, &q);
        if (q != 0.0) {
            e[bottom--] = Qn;
            Q = q;
        } else {
            Q = Qn;
        }
    }
    e[bottom] = Q;
    int top = 0;
    for (int i = bottom + 1; i < m; i++) {
        nif_two_sum(e[i], Q, &Qn, &q);
        if (q != 0.0) e[top++] = q;
        Q = Qn;
    }
    e[top++] = Q;
    return top;
}

NIF_XI int nif_exp_sign(int n, const double *e) {
    const double top = e[n - 1];
    return top > 0.0 ? 1 : (top < 0.0 ? -1 : 0);
}

NIF_XI void nif_exp_negate(int n, double *e) {
    for (int i = 0; i < n; i++) e[i] = -e[i];
}

/* a*b - c*d exactly (<= 4 components) */
NIF_XI int nif_two_two_diff(double a, double b, double c, double d, double *h) {
    double x[2], y[2], xh, xl, yh, yl;
    int xn = 0, yn = 0;
    nif_two_prod(a, b, &xh, &xl);
    nif_two_prod(c, d, &yh, &yl);
    if (xl != 0.0) x[xn++] = xl;
    x[xn++] = xh;
    if (yl != 0.0) y[yn++] = -yl;
    y[yn++] = -yh;
    return nif_exp_sum(xn, x, yn, y, h);
}

/* det of the 3x3 matrix with rows p, q, r, expanded along p (<= 24
 * components, compressed); s: 40 doubles of scratch */
NIF_XF int nif_det3(const double *p, const double *q, const double *r, double *h, double *s) {
    double m[4];
    double *s1 = s, *s2 = s + 8, *s3 = s + 16, *t = s + 24;
    int mn = nif_two_two_diff(q[1], r[2], q[2], r[1], m);
    const int n1 = nif_exp_scale(mn, m, p[0], s1);
    mn = nif_two_two_diff(q[0], r[2], q[2], r[0], m);
    const int n2 = nif_exp_scale(mn, m, -p[1], s2);
    mn = nif_two_two_diff(q[0], r[1], q[1], r[0], m);
    const int n3 = nif_exp_scale(mn, m, p[2], s3);
    const int nt = nif_exp_sum(n1, s1, n2, s2, t);
    const int n = nif_exp_sum(nt, t, n3, s3, h);
    return nif_exp_compress(n, h);
}

/* orient3d(a, b, c, d) exactly (<= 96 components, compressed) into h;
 * s: 192 doubles of scratch (the 3x3 scratch and the partial sums share
 * s[96..192): the partial sums are formed after the last 3x3 determinant) */
NIF_XF int nif_orient_exact(const double *a, const double *b, const double *c, const double *d,
                            double *h, double *s) {
    double *d1 = s, *d2 = s + 24, *d3 = s + 48, *d4 = s + 72, *t = s + 96;
    const int n1 = nif_det3(a, b, c, d1, t);
    const int n2 = nif_det3(a, b, d, d2, t);
    const int n3 = nif_det3(a, c, d, d3, t);
    const int n4 = nif_det3(b, c, d, d4, t);
    nif_exp_negate(n2, d2);
    nif_exp_negate(n4, d4);
    const int m1 = nif_exp_sum(n1, d1, n2, d2, t);
    const int m2 = nif_exp_sum(n3, d3, n4, d4, t + m1);
    const int n = nif_exp_sum(m1, t, m2, t + m1, h);
    return nif_exp_compress(n, h);
}

/* sign of orient3d(a, b, c, d): +1, 0 or -1; s: NIF_ORIENT_SCRATCH doubles */
NIF_XF int nif_orient_exact_sign(const double *a, const double *b, const double *c,
                                 const double *d, double *s) {
    const int n = nif_orient_exact(a, b, c, d, s, s + 96);
    return nif_exp_sign(n, s);
}

/* |p|^2 exactly (<= 6 components, compressed) */
NIF_XI int nif_lift(const double *p, double *h) {
    double x[2], y[2], z[2], t[4], hi, lo;
    int xn = 0, yn = 0, zn = 0;
    nif_two_prod(p[0], p[0], &hi, &lo);
    if (lo != 0.0) x[xn++] = lo;
    x[xn++] = hi;
    nif_two_prod(p[1], p[1], &hi, &lo);
    if (lo != 0.0) y[yn++] = lo;
    y[yn++] = hi;
    nif_two_prod(p[2], p[2], &hi, &lo);
    if (lo != 0.0) z[zn++] = lo;
    z[zn++] = hi;
    const int tn = nif_exp_sum(xn, x, yn, y, t);
    const int n = nif_exp_sum(tn, t, zn, z, h);
    return nif_exp_compress(n, h);
}

/* sign of insphere(a, b, c, d, e): +1, 0 or -1 with inspherefast's
 * convention (positive when e is inside the sphere through a, b, c, d and
 * orient3d(a, b, c, d) > 0); s: NIF_EXACT_SCRATCH doubles */
NIF_XF int nif_insphere_exact_sign(const double *a, const double *b, const double *c,
                                   const double *d, const double *e, double *s) {
    double *acc = s;            /* 5760 */
    double *acc2 = s + 5760;    /* 5760; also the orient3d scratch */
    double *prod = s + 11520;   /* 1152 */
    double *prod2 = s + 12672;  /* 1152 */
    double *orient = s + 13824; /* 96 */
    double *part = s + 13920;   /* 192 */
    double lift[6];
    const double *pts[5] = {a, b, c, d, e};
    int an = 1;
    acc[0] = 0.0;
    for (int i = 0; i < 5; i++) {
        const double *o[4];
        int k = 0;
        for (int j = 0; j < 5; j++)
            if (j != i) o[k++] = pts[j];
        const int on = nif_orient_exact(o[0], o[1], o[2], o[3], orient, acc2);
        if (on == 1 && orient[0] == 0.0) continue; /* zero minor: no contribution */
        const int ln = nif_lift(pts[i], lift);
        int pn = 0;
        for (int l = 0; l < ln; l++) {
            const int qn = nif_exp_scale(on, orient, lift[l], part);
            pn = nif_exp_sum(pn, prod, qn, part, prod2);
            for (int u = 0; u < pn; u++) prod[u] = prod2[u];
        }
        pn = nif_exp_compress(pn, prod);
        if ((i & 1) == 0) nif_exp_negate(pn, prod); /* rows a, c, e enter negated */
        an = nif_exp_sum(an, acc, pn, prod, acc2);
        an = nif_exp_compress(an, acc2);
        for (int u = 0; u < an; u++) acc[u] = acc2[u];
    }
    return nif_exp_sign(an, acc);
}

/* ---- static filters ------------------------------------------------------- */

/* permanent of orient3dfast's expression (same terms, absolute values) */
NIF_XI double nif_orient_permanent(const double *a, const double *b, const double *c,
                                   const double *d) {
    const double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
    const double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
    const double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
    return fabs(adx) * (fabs(bdy * cdz) + fabs(bdz * cdy)) +
           fabs(bdx) * (fabs(cdy * adz) + fabs(cdz * ady)) +
           fabs(cdx) * (fabs(ady * bdz) + fabs(adz * bdy));
}

/* permanent of inspherefast's expression */
NIF_XI double nif_insphere_permanent(const double *a, const double *b, const double *c,
                                     const double *d, const double *e) {
    const double aex = a[0] - e[0], bex = b[0] - e[0], cex = c[0] - e[0], dex = d[0] - e[0];
    const double aey = a[1] - e[1], bey = b[1] - e[1], cey = c[1] - e[1], dey = d[1] - e[1];
    const double aez = a[2] - e[2], bez = b[2] - e[2], cez = c[2] - e[2], dez = d[2] - e[2];
    const double ab = fabs(aex * bey) + fabs(bex * aey);
    const double bc = fabs(bex * cey) + fabs(cex * bey);
    const double cd = fabs(cex * dey) + fabs(dex * cey);
    const double da = fabs(dex * aey) + fabs(aex * dey);
    const double ac = fabs(aex * cey) + fabs(cex * aey);
    const double bd = fabs(bex * dey) + fabs(dex * bey);
    const double abc = fabs(aez) * bc + fabs(bez) * ac + fabs(cez) * ab;
    const double bcd = fabs(bez) * cd + fabs(cez) * bd + fabs(dez) * bc;
    const double cda = fabs(cez) * da + fabs(dez) * ac + fabs(aez) * cd;
    const double dab = fabs(dez) * ab + fabs(aez) * bd + fabs(bez) * da;
    const double al = aex * aex + aey * aey + aez * aez;
    const double bl = bex * bex + bey * bey + bez * bez;
    const double cl = cex * cex + cey * cey + cez * cez;
    const double dl = dex * dex + dey * dey + dez * dez;
    return (dl * abc + cl * dab) + (bl * cda + al * bcd);
}

/* 1 when the fast value's sign is not certified by the bound */
NIF_XI int nif_orient_uncertain(double fast, double permanent) {
    return !(fabs(fast) > NIF_O3D_BOUND * permanent);
}

NIF_XI int nif_insphere_uncertain(double fast, double permanent) {
    return !(fabs(fast) > NIF_ISP_BOUND * permanent);
}

#endif /* NIF_EXACT_H */

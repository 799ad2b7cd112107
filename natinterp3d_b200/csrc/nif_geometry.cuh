// FP64 geometry for the Sibson query kernels.
//
// Every operation is an explicitly rounded IEEE-754 double operation
// (__dadd_rn / __dsub_rn / __dmul_rn / __ddiv_rn), which the compiler never
// contracts into fused multiply-adds.  Each expression keeps the operand
// grouping of natinterp3d's C code (compiled there with -std=c11 and no
// -march, hence no FMA), so every determinant, circumcentre and volume below
// is bit-identical to natinterp3d's on the same inputs:
//   orient3dfast / inspherefast     predicates.c:1687-1710, 3301-3347
//   circumCenterTri3D               natural_insertionfree.c:24-49
//   circumCenterTet                 natural_insertionfree.c:54-84
//   voronoiSubcellVolume            natural_insertionfree.c:92-146
#pragma once
#include <cuda_runtime.h>

// The four large routines are inlined (measured faster on B200 than calls,
// which spill the FP64 state around each call); NIF_GEOM_OUTLINE compiles
// them out of line instead.
#ifdef NIF_GEOM_OUTLINE
#define NIF_GEOM_FN __device__ __noinline__
#else
#define NIF_GEOM_FN __device__ __forceinline__
#endif

namespace nif {

struct dv3 {
    double x, y, z;
};

__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ dv3 mk(double x, double y, double z) { return dv3{x, y, z}; }
__device__ __forceinline__ dv3 mk(const double4 &v) { return dv3{v.x, v.y, v.z}; }
__device__ __forceinline__ dv3 vsub(dv3 a, dv3 b) { return dv3{fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)}; }
__device__ __forceinline__ dv3 vadd(dv3 a, dv3 b) { return dv3{fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)}; }
__device__ __forceinline__ dv3 vscale(dv3 a, double s) { return dv3{fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)}; }
// b x c with natinterp3d's component formulas (delaunay.c:986-990)
__device__ __forceinline__ dv3 vcross(dv3 b, dv3 c) {
    return dv3{fsub(fmul(b.y, c.z), fmul(b.z, c.y)), fsub(fmul(b.z, c.x), fmul(b.x, c.z)),
               fsub(fmul(b.x, c.y), fmul(b.y, c.x))};
}
// (a0 b0 + a1 b1) + a2 b2  (delaunay.c:994-996)
__device__ __forceinline__ double vdot(dv3 a, dv3 b) {
    return fadd(fadd(fmul(a.x, b.x), fmul(a.y, b.y)), fmul(a.z, b.z));
}
__device__ __forceinline__ bool veq(dv3 a, dv3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// orient3dfast(a, b, c, d) = det[a-d; b-d; c-d]
__device__ __forceinline__ double orient_fast(dv3 a, dv3 b, dv3 c, dv3 d) {
    dv3 u = vsub(a, d), v = vsub(b, d), w = vsub(c, d);
    double t0 = fmul(u.x, fsub(fmul(v.y, w.z), fmul(v.z, w.y)));
    double t1 = fmul(v.x, fsub(fmul(w.y, u.z), fmul(w.z, u.y)));
    double t2 = fmul(w.x, fsub(fmul(u.y, v.z), fmul(u.z, v.y)));
    return fadd(fadd(t0, t1), t2);
}

// inspherefast(a, b, c, d, e): lifted 4x4 determinant relative to e
NIF_GEOM_FN double insphere_fast(dv3 a, dv3 b, dv3 c, dv3 d, dv3 e) {
    dv3 r0 = vsub(a, e), r1 = vsub(b, e), r2 = vsub(c, e), r3 = vsub(d, e);
    // 2x2 minors of the (x, y) columns: m(i,j) = x_i y_j - x_j y_i
    double m01 = fsub(fmul(r0.x, r1.y), fmul(r1.x, r0.y));
    double m12 = fsub(fmul(r1.x, r2.y), fmul(r2.x, r1.y));
    double m23 = fsub(fmul(r2.x, r3.y), fmul(r3.x, r2.y));
    double m30 = fsub(fmul(r3.x, r0.y), fmul(r0.x, r3.y));
    double m02 = fsub(fmul(r0.x, r2.y), fmul(r2.x, r0.y));
    double m13 = fsub(fmul(r1.x, r3.y), fmul(r3.x, r1.y));
    double abc = fadd(fsub(fmul(r0.z, m12), fmul(r1.z, m02)), fmul(r2.z, m01));
    double bcd = fadd(fsub(fmul(r1.z, m23), fmul(r2.z, m13)), fmul(r3.z, m12));
    double cda = fadd(fadd(fmul(r2.z, m30), fmul(r3.z, m02)), fmul(r0.z, m23));
    double dab = fadd(fadd(fmul(r3.z, m01), fmul(r0.z, m13)), fmul(r1.z, m30));
    double l0 = vdot(r0, r0), l1 = vdot(r1, r1), l2 = vdot(r2, r2), l3 = vdot(r3, r3);
    return fadd(fsub(fmul(l3, abc), fmul(l2, dab)), fsub(fmul(l1, cda), fmul(l0, bcd)));
}

// circumcentre of triangle (a, b, c); centroid when |ab x ac|^2 < 1e-30
NIF_GEOM_FN dv3 tri_cc(dv3 a, dv3 b, dv3 c) {
    dv3 ab = vsub(b, a), ac = vsub(c, a);
    dv3 n = vcross(ab, ac);
    double n2 = vdot(n, n);
    if (n2 < 1e-30) {
        return dv3{fdiv(fadd(fadd(a.x, b.x), c.x), 3.0), fdiv(fadd(fadd(a.y, b.y), c.y), 3.0),
                   fdiv(fadd(fadd(a.z, b.z), c.z), 3.0)};
    }
    double ab2 = vdot(ab, ab), ac2 = vdot(ac, ac);
    dv3 t = dv3{fsub(fmul(ab2, ac.x), fmul(ac2, ab.x)), fsub(fmul(ab2, ac.y), fmul(ac2, ab.y)),
                fsub(fmul(ab2, ac.z), fmul(ac2, ab.z))};
    dv3 cr = vcross(t, n);
    double inv = fdiv(1.0, fmul(2.0, n2));
    return vadd(a, vscale(cr, inv));
}

// circumcentre of tetrahedron (a, b, c, d); centroid when |denominator| < 1e-30
NIF_GEOM_FN dv3 tet_cc(dv3 a, dv3 b, dv3 c, dv3 d) {
    dv3 ba = vsub(b, a), ca = vsub(c, a), da = vsub(d, a);
    dv3 x1 = vcross(ba, ca), x2 = vcross(da, ba), x3 = vcross(ca, da);
    dv3 m1 = vscale(x1, vdot(da, da));
    dv3 m2 = vscale(x2, vdot(ca, ca));
    dv3 m3 = vscale(x3, vdot(ba, ba));
    dv3 s = vadd(m3, vadd(m1, m2));
    double den = fmul(2.0, vdot(ba, x3));
    if (fabs(den) < 1e-30) {
        return dv3{fmul(fadd(fadd(fadd(a.x, b.x), c.x), d.x), 0.25),
                   fmul(fadd(fadd(fadd(a.y, b.y), c.y), d.y), 0.25),
                   fmul(fadd(fadd(fadd(a.z, b.z), c.z), d.z), 0.25)};
    }
    return vadd(vscale(s, fdiv(1.0, den)), a);
}

// Signed volume of the part of tet (pk, pa, pb, pc) closer to pk than to the
// other vertices, from the tet circumcentre ct and the circumcentres of the
// three faces through pk (fab, fac, fbc); derivation in natinterp3d's
// docs/insertion-free.rst:88-165.
NIF_GEOM_FN double subcell_volume(dv3 pk, dv3 pa, dv3 pb, dv3 pc, dv3 ct, dv3 fab,
                                                dv3 fac, dv3 fbc) {
    dv3 ta = vsub(pa, pk), tb = vsub(pb, pk), tc = vsub(pc, pk);
    double sv = vdot(ta, vcross(tb, tc));
    dv3 a = pa, b = pb;
    if (sv < 0) {
        a = pb;
        b = pa;
        dv3 t = fac;
        fac = fbc;
        fbc = t;
    }
    dv3 df = vsub(fab, pk), dg = vsub(fac, pk), dh = vsub(fbc, pk), dt = vsub(ct, pk);
    dv3 c1 = vcross(df, dt), c2 = vcross(dt, dg), c3 = vcross(dh, dt);
    dv3 e1 = vsub(a, b), e2 = vsub(a, pc), e3 = vsub(b, pc);
    double vol = fmul(e1.x, c1.x);
    vol = fadd(vol, fmul(e1.y, c1.y));
    vol = fadd(vol, fmul(e1.z, c1.z));
    vol = fadd(vol, fmul(e2.x, c2.x));
    vol = fadd(vol, fmul(e2.y, c2.y));
    vol = fadd(vol, fmul(e2.z, c2.z));
    vol = fadd(vol, fmul(e3.x, c3.x));
    vol = fadd(vol, fmul(e3.y, c3.y));
    vol = fadd(vol, fmul(e3.z, c3.z));
    return fdiv(vol, 12.0);
}

}  // namespace nif

// Derivatives of the Sibson weights with respect to the query position.
//
// For a query q with natural neighbours k, stolen volumes s_k, total
// S = sum_k s_k and weights w_k = s_k / S (natural_insertionfree.c:721-737),
// only the virtual-tet terms depend on q: the cavity, its boundary and the
// cavity-tet terms are locally constant (:638-676), while each virtual-tet
// term is voronoiSubcellVolume(pk, q, pa, pb, cc(q,fa,fb,fc), cc(pk,q,pa),
// cc(pk,q,pb), cc(face)) (:681-719).  Hence
//   ds_k/dq = - sum over virtual terms of k of d(volume)/dq
//   dw_k/dq = (ds_k/dq - w_k sum_j ds_j/dq) / S
// and for a loss L with dL/dw_k = g_k,
//   dL/dq = sum_k g_k dw_k/dq = (1/S) sum_k (g_k - gbar) ds_k/dq,
//   gbar = sum_k g_k w_k.
// d(volume)/dq is evaluated exactly with forward-mode dual numbers over
// the same formulas: the value part of every dual operation is the same
// explicitly rounded operation as the weights kernel, so every branch (the
// degeneracy fallbacks and the orientation swap) takes the same side as in
// the forward pass and the derivative is that of the piece actually used.
#pragma once
#include "nif_geometry.cuh"

namespace nif {

// A value and its derivatives along ND directions (ND = 3: x, y and z at
// once; ND = 1: one direction per pass, a third of the live state).
template <int ND>
struct dualn {
    double v, d[ND];
};

template <int ND>
__device__ __forceinline__ dualn<ND> dconst(double c) {
    dualn<ND> r;
    r.v = c;
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = 0.0;
    return r;
}

template <int ND>
__device__ __forceinline__ dualn<ND> operator+(dualn<ND> a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fadd(a.v, b.v);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator-(dualn<ND> a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fsub(a.v, b.v);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
// The value parts are the forward's separately rounded operations (they
// decide the branches); the derivative parts only need to be accurate, so
// they use fused multiply-adds.
template <int ND>
__device__ __forceinline__ dualn<ND> operator*(dualn<ND> a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fmul(a.v, b.v);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = __fma_rn(a.v, b.d[i], a.d[i] * b.v);
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator/(dualn<ND> a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fdiv(a.v, b.v);
    const double inv = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = __fma_rn(-r.v, b.d[i], a.d[i]) * inv;
    return r;
}

// A dual and a constant of the differentiation (a plain double): the same
// value operation, and no derivative terms for the constant.
template <int ND>
__device__ __forceinline__ dualn<ND> operator*(dualn<ND> a, double b) {
    dualn<ND> r;
    r.v = fmul(a.v, b);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = a.d[i] * b;
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator*(double a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fmul(a, b.v);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = a * b.d[i];
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator+(dualn<ND> a, double b) {
    dualn<ND> r = a;
    r.v = fadd(a.v, b);
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator+(double a, dualn<ND> b) {
    dualn<ND> r = b;
    r.v = fadd(a, b.v);
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator-(dualn<ND> a, double b) {
    dualn<ND> r = a;
    r.v = fsub(a.v, b);
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator-(double a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fsub(a, b.v);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = -b.d[i];
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator/(dualn<ND> a, double b) {
    dualn<ND> r;
    r.v = fdiv(a.v, b);
    const double inv = 1.0 / b;
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = a.d[i] * inv;
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator/(double a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fdiv(a, b.v);
    const double inv = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = -(r.v * b.d[i]) * inv;
    return r;
}

template <int ND>
struct dvec {
    dualn<ND> x, y, z;
};

template <int ND>
__device__ __forceinline__ dvec<ND> dvconst(dv3 a) {
    return dvec<ND>{dconst<ND>(a.x), dconst<ND>(a.y), dconst<ND>(a.z)};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvsub(dvec<ND> a, dvec<ND> b) {
    return dvec<ND>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvadd(dvec<ND> a, dvec<ND> b) {
    return dvec<ND>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvscale(dvec<ND> a, dualn<ND> s) {
    return dvec<ND>{a.x * s, a.y * s, a.z * s};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvcross(dvec<ND> b, dvec<ND> c) {
    return dvec<ND>{b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
}
template <int ND>
__device__ __forceinline__ dualn<ND> dvdot(dvec<ND> a, dvec<ND> b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

template <int ND>
__device__ __forceinline__ dvec<ND> dvsub_c(dvec<ND> a, dv3 b) {
    return dvec<ND>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvsub_c(dv3 a, dvec<ND> b) {
    return dvec<ND>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvcross_c(dv3 b, dvec<ND> c) {
    return dvec<ND>{b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
}
template <int ND>
__device__ __forceinline__ dvec<ND> dvcross_c(dvec<ND> b, dv3 c) {
    return dvec<ND>{b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
}

// voronoiSubcellVolume(pk, q, pb, pc, ct, fab, fac, fbc) of a virtual-tet
// term: pk, pb, pc and the face circumcentre fbc are constants, q, the
// virtual-tet circumcentre ct and the triangle circumcentres fab, fac are
// duals.  Same formula, groupings and value operations as subcell_volume
// (including its orientation swap of a, b and of fac, fbc), without the
// constants' derivative terms.
template <int ND>
__device__ __forceinline__ dualn<ND> subcell_volume_q(dv3 pk, dvec<ND> q, dv3 pb, dv3 pc, dvec<ND> ct,
                                                      dvec<ND> fab, dvec<ND> fac, dv3 fbc) {
    const dvec<ND> ta = dvsub_c(q, pk);
    const dv3 tbc = vcross(vsub(pb, pk), vsub(pc, pk));
    const dualn<ND> sv = ta.x * tbc.x + ta.y * tbc.y + ta.z * tbc.z;
    const dvec<ND> df = dvsub_c(fab, pk), dt = dvsub_c(ct, pk);
    const dvec<ND> c1 = dvcross(df, dt);
    dualn<ND> vol = c1.x;
    if (!(sv.v < 0)) {
        // a = q, b = pb
        const dvec<ND> c2 = dvcross(dt, dvsub_c(fac, pk));
        const dvec<ND> c3 = dvcross_c(vsub(fbc, pk), dt);
        const dvec<ND> e1 = dvsub_c(q, pb), e2 = dvsub_c(q, pc);
        const dv3 e3 = vsub(pb, pc);
        vol = e1.x * c1.x;
        vol = vol + e1.y * c1.y;
        vol = vol + e1.z * c1.z;
        vol = vol + e2.x * c2.x;
        vol = vol + e2.y * c2.y;
        vol = vol + e2.z * c2.z;
        vol = vol + e3.x * c3.x;
        vol = vol + e3.y * c3.y;
        vol = vol + e3.z * c3.z;
    } else {
        // a = pb, b = q; fac and fbc swapped
        const dvec<ND> c2 = dvcross_c(dt, vsub(fbc, pk));
        const dvec<ND> c3 = dvcross(dvsub_c(fac, pk), dt);
        const dvec<ND> e1 = dvsub_c(pb, q), e3 = dvsub_c(q, pc);
        const dv3 e2 = vsub(pb, pc);
        vol = e1.x * c1.x;
        vol = vol + e1.y * c1.y;
        vol = vol + e1.z * c1.z;
        vol = vol + e2.x * c2.x;
        vol = vol + e2.y * c2.y;
        vol = vol + e2.z * c2.z;
        vol = vol + e3.x * c3.x;
        vol = vol + e3.y * c3.y;
        vol = vol + e3.z * c3.z;
    }
    return vol / 12.0;
}

// tri_cc(a, b, c) for constants a, c and a dual b: the same formula and
// groupings (and value operations) as tri_cc, without the constants'
// derivative terms
template <int ND>
__device__ __forceinline__ dvec<ND> tri_cc_cdc(dv3 a, dvec<ND> b, dv3 c) {
    const dvec<ND> ab{b.x - a.x, b.y - a.y, b.z - a.z};
    const dv3 ac = vsub(c, a);
    const dvec<ND> n{ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x};
    const dualn<ND> n2 = dvdot(n, n);
    if (n2.v < 1e-30) {
        return dvec<ND>{(a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0};
    }
    const dualn<ND> ab2 = dvdot(ab, ab);
    const double ac2 = vdot(ac, ac);
    const dvec<ND> t{ab2 * ac.x - ac2 * ab.x, ab2 * ac.y - ac2 * ab.y, ab2 * ac.z - ac2 * ab.z};
    const dvec<ND> cr = dvcross(t, n);
    const dualn<ND> inv = 1.0 / (2.0 * n2);
    return dvec<ND>{a.x + cr.x * inv, a.y + cr.y * inv, a.z + cr.z * inv};
}

// the same formulas and groupings as tri_cc / tet_cc / subcell_volume
template <int ND>
__device__ __forceinline__ dvec<ND> tri_cc_d(dvec<ND> a, dvec<ND> b, dvec<ND> c) {
    dvec<ND> ab = dvsub(b, a), ac = dvsub(c, a);
    dvec<ND> n = dvcross(ab, ac);
    dualn<ND> n2 = dvdot(n, n);
    if (n2.v < 1e-30) {
        const dualn<ND> three = dconst<ND>(3.0);
        return dvec<ND>{(a.x + b.x + c.x) / three, (a.y + b.y + c.y) / three,
                        (a.z + b.z + c.z) / three};
    }
    dualn<ND> ab2 = dvdot(ab, ab), ac2 = dvdot(ac, ac);
    dvec<ND> t = dvec<ND>{ab2 * ac.x - ac2 * ab.x, ab2 * ac.y - ac2 * ab.y, ab2 * ac.z - ac2 * ab.z};
    dvec<ND> cr = dvcross(t, n);
    dualn<ND> inv = dconst<ND>(1.0) / (dconst<ND>(2.0) * n2);
    return dvadd(a, dvscale(cr, inv));
}

// tet_cc(a, b, c, d) for a dual a and constants b, c, d (same value operations)
template <int ND>
__device__ __forceinline__ dvec<ND> tet_cc_q(dvec<ND> a, dv3 b, dv3 c, dv3 d) {
    const dvec<ND> ba = dvsub_c(b, a), ca = dvsub_c(c, a), da = dvsub_c(d, a);
    const dvec<ND> x1 = dvcross(ba, ca), x2 = dvcross(da, ba), x3 = dvcross(ca, da);
    const dvec<ND> m1 = dvscale(x1, dvdot(da, da));
    const dvec<ND> m2 = dvscale(x2, dvdot(ca, ca));
    const dvec<ND> m3 = dvscale(x3, dvdot(ba, ba));
    const dvec<ND> s = dvadd(m3, dvadd(m1, m2));
    const dualn<ND> den = 2.0 * dvdot(ba, x3);
    if (fabs(den.v) < 1e-30) {
        return dvec<ND>{(a.x + b.x + c.x + d.x) * 0.25, (a.y + b.y + c.y + d.y) * 0.25,
                        (a.z + b.z + c.z + d.z) * 0.25};
    }
    return dvadd(dvscale(s, 1.0 / den), a);
}

template <int ND>
__device__ __forceinline__ dvec<ND> tet_cc_d(dvec<ND> a, dvec<ND> b, dvec<ND> c, dvec<ND> d) {
    dvec<ND> ba = dvsub(b, a), ca = dvsub(c, a), da = dvsub(d, a);
    dvec<ND> x1 = dvcross(ba, ca), x2 = dvcross(da, ba), x3 = dvcross(ca, da);
    dvec<ND> m1 = dvscale(x1, dvdot(da, da));
    dvec<ND> m2 = dvscale(x2, dvdot(ca, ca));
    dvec<ND> m3 = dvscale(x3, dvdot(ba, ba));
    dvec<ND> s = dvadd(m3, dvadd(m1, m2));
    dualn<ND> den = dconst<ND>(2.0) * dvdot(ba, x3);
    if (fabs(den.v) < 1e-30) {
        const dualn<ND> q = dconst<ND>(0.25);
        return dvec<ND>{(a.x + b.x + c.x + d.x) * q, (a.y + b.y + c.y + d.y) * q,
                        (a.z + b.z + c.z + d.z) * q};
    }
    return dvadd(dvscale(s, dconst<ND>(1.0) / den), a);
}

template <int ND>
__device__ __forceinline__ dualn<ND> subcell_volume_d(dvec<ND> pk, dvec<ND> pa, dvec<ND> pb, dvec<ND> pc,
                                                      dvec<ND> ct, dvec<ND> fab, dvec<ND> fac,
                                                      dvec<ND> fbc) {
    dvec<ND> ta = dvsub(pa, pk), tb = dvsub(pb, pk), tc = dvsub(pc, pk);
    dualn<ND> sv = dvdot(ta, dvcross(tb, tc));
    dvec<ND> a = pa, b = pb;
    if (sv.v < 0) {
        a = pb;
        b = pa;
        dvec<ND> t = fac;
        fac = fbc;
        fbc = t;
    }
    dvec<ND> df = dvsub(fab, pk), dg = dvsub(fac, pk), dh = dvsub(fbc, pk), dt = dvsub(ct, pk);
    dvec<ND> c1 = dvcross(df, dt), c2 = dvcross(dt, dg), c3 = dvcross(dh, dt);
    dvec<ND> e1 = dvsub(a, b), e2 = dvsub(a, pc), e3 = dvsub(b, pc);
    dualn<ND> vol = e1.x * c1.x;
    vol = vol + e1.y * c1.y;
    vol = vol + e1.z * c1.z;
    vol = vol + e2.x * c2.x;
    vol = vol + e2.y * c2.y;
    vol = vol + e2.z * c2.z;
    vol = vol + e3.x * c3.x;
    vol = vol + e3.y * c3.y;
    vol = vol + e3.z * c3.z;
    return vol / dconst<ND>(12.0);
}

// the query as a dual vector with derivative seeds along x, y, z (ND = 3) or
// along the one axis given (ND = 1)
template <int ND>
__device__ __forceinline__ dvec<ND> query_dual(dv3 q, int axis) {
    dvec<ND> Q = dvconst<ND>(q);
    if (ND == 3) {
        Q.x.d[0] = 1.0;
        Q.y.d[ND > 1 ? 1 : 0] = 1.0;
        Q.z.d[ND > 2 ? 2 : 0] = 1.0;
    } else {
        (axis == 0 ? Q.x : (axis == 1 ? Q.y : Q.z)).d[0] = 1.0;
    }
    return Q;
}

// Gradient of sum_j c_j * (virtual-tet term of vertex j) over the three
// vertices of boundary face (fa, fb, fc); c_j = 0 skips a vertex.  The
// virtual-tet circumcentre is shared by the face's three terms; each term
// evaluates its two (vertex, query, vertex) triangle circumcentres in the
// forward pass's own argument order (natural_insertionfree.c:708-714), so
// its value part is bit-identical to the forward's.  One loop iteration per
// term keeps the live dual state small.  NIF_GRAD_ND = 1 differentiates one
// axis per pass (three passes, a third of the live derivative state).
#ifndef NIF_GRAD_ND
#define NIF_GRAD_ND 3
#endif
__device__ __forceinline__ dv3 virtual_face_grad(dv3 q, dv3 fa, dv3 fb, dv3 fc, dv3 cface, double c0,
                                                 double c1, double c2) {
    constexpr int ND = NIF_GRAD_ND;
    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll 1
    for (int axis = 0; axis < 3; axis += ND) {
        const dvec<ND> Q = query_dual<ND>(q, axis);
        const dvec<ND> ct = tet_cc_q<ND>(Q, fa, fb, fc);
#pragma unroll 1
        for (int j = 0; j < 3; j++) {
            const double cj = j == 0 ? c0 : (j == 1 ? c1 : c2);
            if (cj == 0.0) continue;
            const dv3 k = j == 0 ? fa : (j == 1 ? fb : fc);
            const dv3 n = j == 0 ? fb : (j == 1 ? fc : fa);  // face_verts[(j+1)%3]
            const dv3 p = j == 0 ? fc : (j == 1 ? fa : fb);  // face_verts[(j+2)%3]
            const dvec<ND> t1 = tri_cc_cdc<ND>(k, Q, n);
            const dvec<ND> t2 = tri_cc_cdc<ND>(k, Q, p);
            const dualn<ND> v = subcell_volume_q<ND>(k, Q, n, p, ct, t1, t2, cface);
            if (ND == 3) {
                gx += cj * v.d[0];
                gy += cj * v.d[ND > 1 ? 1 : 0];
                gz += cj * v.d[ND > 2 ? 2 : 0];
            } else {
                const double t = cj * v.d[0];
                gx += axis == 0 ? t : 0.0;
                gy += axis == 1 ? t : 0.0;
                gz += axis == 2 ? t : 0.0;
            }
        }
    }
    return dv3{gx, gy, gz};
}

}  // namespace nif

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
template <int ND>
__device__ __forceinline__ dualn<ND> operator*(dualn<ND> a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fmul(a.v, b.v);
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = a.v * b.d[i] + a.d[i] * b.v;
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator/(dualn<ND> a, dualn<ND> b) {
    dualn<ND> r;
    r.v = fdiv(a.v, b.v);
    const double inv = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < ND; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
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
        const dvec<ND> ct = tet_cc_d<ND>(Q, dvconst<ND>(fa), dvconst<ND>(fb), dvconst<ND>(fc));
#pragma unroll 1
        for (int j = 0; j < 3; j++) {
            const double cj = j == 0 ? c0 : (j == 1 ? c1 : c2);
            if (cj == 0.0) continue;
            const dv3 k = j == 0 ? fa : (j == 1 ? fb : fc);
            const dv3 n = j == 0 ? fb : (j == 1 ? fc : fa);  // face_verts[(j+1)%3]
            const dv3 p = j == 0 ? fc : (j == 1 ? fa : fb);  // face_verts[(j+2)%3]
            const dvec<ND> K = dvconst<ND>(k), N = dvconst<ND>(n), P = dvconst<ND>(p);
            const dvec<ND> t1 = tri_cc_d<ND>(K, Q, N);
            const dvec<ND> t2 = tri_cc_d<ND>(K, Q, P);
            const dualn<ND> v = subcell_volume_d<ND>(K, Q, N, P, ct, t1, t2, dvconst<ND>(cface));
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

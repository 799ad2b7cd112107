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

// value + derivative along x, y, z
struct dual3 {
    double v, dx, dy, dz;
};

__device__ __forceinline__ dual3 dconst(double c) { return dual3{c, 0.0, 0.0, 0.0}; }

__device__ __forceinline__ dual3 operator+(dual3 a, dual3 b) {
    return dual3{fadd(a.v, b.v), a.dx + b.dx, a.dy + b.dy, a.dz + b.dz};
}
__device__ __forceinline__ dual3 operator-(dual3 a, dual3 b) {
    return dual3{fsub(a.v, b.v), a.dx - b.dx, a.dy - b.dy, a.dz - b.dz};
}
__device__ __forceinline__ dual3 operator*(dual3 a, dual3 b) {
    return dual3{fmul(a.v, b.v), a.v * b.dx + a.dx * b.v, a.v * b.dy + a.dy * b.v,
                 a.v * b.dz + a.dz * b.v};
}
__device__ __forceinline__ dual3 operator/(dual3 a, dual3 b) {
    const double q = fdiv(a.v, b.v);
    const double r = 1.0 / b.v;
    return dual3{q, (a.dx - q * b.dx) * r, (a.dy - q * b.dy) * r, (a.dz - q * b.dz) * r};
}

struct dvec {
    dual3 x, y, z;
};

__device__ __forceinline__ dvec dvconst(dv3 a) { return dvec{dconst(a.x), dconst(a.y), dconst(a.z)}; }
__device__ __forceinline__ dvec dvsub(dvec a, dvec b) { return dvec{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ dvec dvadd(dvec a, dvec b) { return dvec{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ dvec dvscale(dvec a, dual3 s) { return dvec{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ dvec dvcross(dvec b, dvec c) {
    return dvec{b.y * c.z - b.z * c.y, b.z * c.x - b.x * c.z, b.x * c.y - b.y * c.x};
}
__device__ __forceinline__ dual3 dvdot(dvec a, dvec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// the same formulas and groupings as tri_cc / tet_cc / subcell_volume
__device__ __forceinline__ dvec tri_cc_d(dvec a, dvec b, dvec c) {
    dvec ab = dvsub(b, a), ac = dvsub(c, a);
    dvec n = dvcross(ab, ac);
    dual3 n2 = dvdot(n, n);
    if (n2.v < 1e-30) {
        const dual3 three = dconst(3.0);
        return dvec{(a.x + b.x + c.x) / three, (a.y + b.y + c.y) / three, (a.z + b.z + c.z) / three};
    }
    dual3 ab2 = dvdot(ab, ab), ac2 = dvdot(ac, ac);
    dvec t = dvec{ab2 * ac.x - ac2 * ab.x, ab2 * ac.y - ac2 * ab.y, ab2 * ac.z - ac2 * ab.z};
    dvec cr = dvcross(t, n);
    dual3 inv = dconst(1.0) / (dconst(2.0) * n2);
    return dvadd(a, dvscale(cr, inv));
}

__device__ __forceinline__ dvec tet_cc_d(dvec a, dvec b, dvec c, dvec d) {
    dvec ba = dvsub(b, a), ca = dvsub(c, a), da = dvsub(d, a);
    dvec x1 = dvcross(ba, ca), x2 = dvcross(da, ba), x3 = dvcross(ca, da);
    dvec m1 = dvscale(x1, dvdot(da, da));
    dvec m2 = dvscale(x2, dvdot(ca, ca));
    dvec m3 = dvscale(x3, dvdot(ba, ba));
    dvec s = dvadd(m3, dvadd(m1, m2));
    dual3 den = dconst(2.0) * dvdot(ba, x3);
    if (fabs(den.v) < 1e-30) {
        const dual3 q = dconst(0.25);
        return dvec{(a.x + b.x + c.x + d.x) * q, (a.y + b.y + c.y + d.y) * q,
                    (a.z + b.z + c.z + d.z) * q};
    }
    return dvadd(dvscale(s, dconst(1.0) / den), a);
}

__device__ __forceinline__ dual3 subcell_volume_d(dvec pk, dvec pa, dvec pb, dvec pc, dvec ct,
                                                  dvec fab, dvec fac, dvec fbc) {
    dvec ta = dvsub(pa, pk), tb = dvsub(pb, pk), tc = dvsub(pc, pk);
    dual3 sv = dvdot(ta, dvcross(tb, tc));
    dvec a = pa, b = pb;
    if (sv.v < 0) {
        a = pb;
        b = pa;
        dvec t = fac;
        fac = fbc;
        fbc = t;
    }
    dvec df = dvsub(fab, pk), dg = dvsub(fac, pk), dh = dvsub(fbc, pk), dt = dvsub(ct, pk);
    dvec c1 = dvcross(df, dt), c2 = dvcross(dt, dg), c3 = dvcross(dh, dt);
    dvec e1 = dvsub(a, b), e2 = dvsub(a, pc), e3 = dvsub(b, pc);
    dual3 vol = e1.x * c1.x;
    vol = vol + e1.y * c1.y;
    vol = vol + e1.z * c1.z;
    vol = vol + e2.x * c2.x;
    vol = vol + e2.y * c2.y;
    vol = vol + e2.z * c2.z;
    vol = vol + e3.x * c3.x;
    vol = vol + e3.y * c3.y;
    vol = vol + e3.z * c3.z;
    return vol / dconst(12.0);
}

// Gradient of sum_j c_j * (virtual-tet term of vertex j) over the three
// vertices of boundary face (fa, fb, fc); c_j = 0 skips a vertex.  The
// virtual-tet circumcentre is shared by the face's three terms; each term
// evaluates its two (vertex, query, vertex) triangle circumcentres in the
// forward pass's own argument order (natural_insertionfree.c:708-714), so
// its value part is bit-identical to the forward's.  One loop iteration per
// term keeps the live dual state small (it would otherwise spill).
__device__ __forceinline__ dv3 virtual_face_grad(dv3 q, dv3 fa, dv3 fb, dv3 fc, dv3 cface, double c0,
                                                 double c1, double c2) {
    const dvec Q = dvec{dual3{q.x, 1.0, 0.0, 0.0}, dual3{q.y, 0.0, 1.0, 0.0}, dual3{q.z, 0.0, 0.0, 1.0}};
    const dvec ct = tet_cc_d(Q, dvconst(fa), dvconst(fb), dvconst(fc));
    dv3 gsum = dv3{0.0, 0.0, 0.0};
#pragma unroll 1
    for (int j = 0; j < 3; j++) {
        const double cj = j == 0 ? c0 : (j == 1 ? c1 : c2);
        if (cj == 0.0) continue;
        const dv3 k = j == 0 ? fa : (j == 1 ? fb : fc);
        const dv3 n = j == 0 ? fb : (j == 1 ? fc : fa);  // face_verts[(j+1)%3]
        const dv3 p = j == 0 ? fc : (j == 1 ? fa : fb);  // face_verts[(j+2)%3]
        const dvec K = dvconst(k), N = dvconst(n), P = dvconst(p);
        const dvec t1 = tri_cc_d(K, Q, N);
        const dvec t2 = tri_cc_d(K, Q, P);
        const dual3 v = subcell_volume_d(K, Q, N, P, ct, t1, t2, dvconst(cface));
        gsum.x += cj * v.dx;
        gsum.y += cj * v.dy;
        gsum.z += cj * v.dz;
    }
    return gsum;
}

}  // namespace nif

// Box SAT shared by the batched call (sf_sat.cu) and the box world (sf_boxes.cu): the separating-axis test over the
// 3 + 3 face axes and 9 edge axes, reference/incident face clipping or the edge-edge closest points, and the reduction
// to 4 points (engine/src/phys.rs:502-628). The arithmetic keeps the reference's evaluation order (compiled with
// --fmad=false).
#pragma once
#include <cstdint>

namespace sf {

struct P3 { float x, y, z; };
__device__ __forceinline__ P3 p3(float a, float b, float c) { P3 r; r.x = a; r.y = b; r.z = c; return r; }
__device__ __forceinline__ P3 operator+(P3 a, P3 b) { return p3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ P3 operator-(P3 a, P3 b) { return p3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ P3 operator*(P3 a, float s) { return p3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ P3 operator-(P3 a) { return p3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float pdot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ P3 pcross(P3 a, P3 b) { return p3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
// engine/src/math.rs:87-90: sqrt of a non-positive value is 0
__device__ __forceinline__ float sqrt_e(float x) { return x <= 0.0f ? 0.0f : __fsqrt_rn(x); }

struct Box { P3 p; P3 c[3]; float h[3]; };

__device__ __forceinline__ Box load_box(const float *b) {
    Box r;
    r.p = p3(b[0], b[1], b[2]);
    float x = b[3], y = b[4], z = b[5], w = b[6];
    // Quat::to_m3 (engine/src/math.rs:60-66): the columns are the box axes
    r.c[0] = p3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w));
    r.c[1] = p3(2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w));
    r.c[2] = p3(2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y));
    r.h[0] = b[7]; r.h[1] = b[8]; r.h[2] = b[9];
    return r;
}

struct CPt { P3 p; float s; };

static __device__ int reduce4(CPt *pts, int cnt, P3 n) {
    if (cnt <= 4) return cnt;
    int i0 = 0;
    for (int k = 1; k < cnt; k++) if (pts[k].s < pts[i0].s) i0 = k;
    P3 q0 = pts[i0].p;
    int i1 = 0; float best = -1.0f;
    for (int k = 0; k < cnt; k++) { P3 d = pts[k].p - q0; float dd = pdot(d, d); if (dd > best) { best = dd; i1 = k; } }
    P3 e = pts[i1].p - q0;
    int i2 = 0; float b2 = -3.4028235e38f;
    for (int k = 0; k < cnt; k++) { float a = pdot(pcross(pts[k].p - q0, e), n); if (a > b2) { b2 = a; i2 = k; } }
    int i3 = 0; float b3 = -3.4028235e38f;
    for (int k = 0; k < cnt; k++) { float a = -pdot(pcross(pts[k].p - q0, e), n); if (a > b3) { b3 = a; i3 = k; } }
    int ids[4] = {i0, i1, i2, i3};
    CPt sel[4] = {pts[i0], pts[i1], pts[i2], pts[i3]};
    int out = 0;
    for (int k = 0; k < 4; k++) {
        bool dup = false;
        for (int t = 0; t < k; t++) if (ids[t] == ids[k]) dup = true;
        if (!dup) pts[out++] = sel[k];
    }
    return out;
}

static __device__ int collide_boxes(const Box &A, const Box &B, float margin, CPt *out, P3 *nout) {
    P3 t = B.p - A.p;
    float ac[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) ac[i][j] = fabsf(pdot(A.c[i], B.c[j])) + 1e-6f;
    float sa = -3.4028235e38f; int ia = 0;
    for (int i = 0; i < 3; i++) {
        float s = fabsf(pdot(t, A.c[i])) - (A.h[i] + B.h[0] * ac[i][0] + B.h[1] * ac[i][1] + B.h[2] * ac[i][2]);
        if (s > margin) return 0;
        if (s > sa) { sa = s; ia = i; }
    }
    float sbm = -3.4028235e38f; int jb = 0;
    for (int j = 0; j < 3; j++) {
        float s = fabsf(pdot(t, B.c[j])) - (B.h[j] + A.h[0] * ac[0][j] + A.h[1] * ac[1][j] + A.h[2] * ac[2][j]);
        if (s > margin) return 0;
        if (s > sbm) { sbm = s; jb = j; }
    }
    float se = -3.4028235e38f; int ei = 0, ej = 0; P3 el = p3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            P3 l = pcross(A.c[i], B.c[j]);
            float l2 = pdot(l, l);
            if (l2 < 1e-8f) continue;
            l = l * __fdiv_rn(1.0f, sqrt_e(l2));
            float r = A.h[0] * fabsf(pdot(A.c[0], l)) + A.h[1] * fabsf(pdot(A.c[1], l)) + A.h[2] * fabsf(pdot(A.c[2], l))
                    + B.h[0] * fabsf(pdot(B.c[0], l)) + B.h[1] * fabsf(pdot(B.c[1], l)) + B.h[2] * fabsf(pdot(B.c[2], l));
            float s = fabsf(pdot(t, l)) - r;
            if (s > margin) return 0;
            if (s > se) { se = s; ei = i; ej = j; el = l; }
        }
    const float face_tol = 0.005f;
    bool use_b = sbm > sa + face_tol;
    float face_best = use_b ? sbm : sa;
    if (se > face_best + 0.01f) {
        P3 n = pdot(t, el) < 0.0f ? -el : el;
        P3 ca = A.p, cb = B.p;
        for (int k = 0; k < 3; k++) {
            if (k != ei) { float s = pdot(A.c[k], n) > 0.0f ? 1.0f : -1.0f; ca = ca + A.c[k] * (s * A.h[k]); }
            if (k != ej) { float s = pdot(B.c[k], n) > 0.0f ? -1.0f : 1.0f; cb = cb + B.c[k] * (s * B.h[k]); }
        }
        P3 d1 = A.c[ei], d2 = B.c[ej];
        P3 r = ca - cb;
        float bb = pdot(d1, d2), c = pdot(d1, r), f = pdot(d2, r);
        float den = 1.0f - bb * bb;
        float s = den > 1e-6f ? __fdiv_rn(bb * f - c, den) : 0.0f;
        s = fminf(fmaxf(s, -A.h[ei]), A.h[ei]);
        float tt = bb * s + f;
        tt = fminf(fmaxf(tt, -B.h[ej]), B.h[ej]);
        s = fminf(fmaxf(bb * tt - c, -A.h[ei]), A.h[ei]);
        P3 q1 = ca + d1 * s, q2 = cb + d2 * tt;
        out[0].p = (q1 + q2) * 0.5f;
        out[0].s = pdot(q2 - q1, n);
        *nout = n;
        return 1;
    }
    const Box &R = use_b ? B : A;
    const Box &I = use_b ? A : B;
    const int k = use_b ? jb : ia;
    P3 n = R.c[k];
    if (pdot(I.p - R.p, n) < 0.0f) n = -n;
    int j = 0; float bd = -1.0f;
    for (int q = 0; q < 3; q++) { float d = fabsf(pdot(I.c[q], n)); if (d > bd) { bd = d; j = q; } }
    float sgn = pdot(I.c[j], n) > 0.0f ? -1.0f : 1.0f;
    P3 fc = I.p + I.c[j] * (sgn * I.h[j]);
    int u = (j + 1) % 3, v = (j + 2) % 3;
    P3 eu = I.c[u] * I.h[u], ev = I.c[v] * I.h[v];
    P3 poly[8], tmp[8];
    poly[0] = fc + eu + ev; poly[1] = fc - eu + ev; poly[2] = fc - eu - ev; poly[3] = fc + eu - ev;
    int pn = 4;
    const int u2 = (k + 1) % 3, v2 = (k + 2) % 3;
    for (int e = 0; e < 4; e++) {
        const int ax = e < 2 ? u2 : v2;
        const float sg = (e & 1) ? -1.0f : 1.0f;
        P3 dir = R.c[ax] * sg;
        float off = pdot(dir, R.p) + R.h[ax];
        int tn = 0;
        for (int q = 0; q < pn; q++) {
            P3 a0 = poly[q], a1 = poly[(q + 1) % pn];
            float d0 = pdot(a0, dir) - off, d1 = pdot(a1, dir) - off;
            if (d0 <= 0.0f && tn < 8) tmp[tn++] = a0;
            if ((d0 <= 0.0f) != (d1 <= 0.0f)) {
                float tq = __fdiv_rn(d0, d0 - d1);
                if (tn < 8) tmp[tn++] = a0 + (a1 - a0) * tq;
            }
        }
        pn = tn;
        for (int q = 0; q < pn; q++) poly[q] = tmp[q];
        if (pn == 0) return 0;
    }
    P3 rc = R.p + n * R.h[k];
    int cnt = 0;
    for (int q = 0; q < pn; q++) {
        P3 pp = poly[q];
        float sep = pdot(pp - rc, n);
        if (sep <= margin) { out[cnt].p = pp - n * (0.5f * sep); out[cnt].s = sep; cnt++; }
    }
    if (cnt == 0) return 0;
    *nout = use_b ? -n : n;
    return cnt;
}

}  // namespace sf

// Box SAT and convex-cell SAT shared by the batched calls (sf_sat.cu) and the box world (sf_boxes.cu). Box SAT: the
// separating-axis test over the 3 + 3 face axes and 9 edge axes, reference/incident face clipping or the edge-edge
// closest points, and the reduction to 4 points (engine/src/phys.rs:502-628). Convex cells: gpu/gpu_world.js:400-555. The arithmetic keeps the reference's evaluation order (compiled with
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

// ---------------------------------------------------------------- convex cells (gpu/gpu_world.js:400-555)
// A hull is 80 float4 (vertex, plane, face-index, edge, direction tables; see shatterforge_b200/hulls.py); a shape is
// a cell in its box: centre p, rotation R (columns), half extents h. The arithmetic order is fixed:
// R * v = c0 v.x + c1 v.y + c2 v.z, normalize(v) = v / |v|, inverseSqrt(x) = 1 / sqrt(x).
struct HShape { P3 p; P3 c[3]; P3 h; const float4 *H; };

__device__ __forceinline__ P3 f4xyz(float4 v) { return p3(v.x, v.y, v.z); }
__device__ __forceinline__ P3 rmul(const HShape &s, P3 v) { return s.c[0] * v.x + s.c[1] * v.y + s.c[2] * v.z; }
__device__ __forceinline__ P3 cmul(P3 a, P3 b) { return p3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ P3 cdiv(P3 a, P3 b) { return p3(__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y), __fdiv_rn(a.z, b.z)); }
__device__ __forceinline__ float plen(P3 a) { return __fsqrt_rn(pdot(a, a)); }
__device__ __forceinline__ P3 pnorm(P3 a) { const float l = plen(a); return p3(__fdiv_rn(a.x, l), __fdiv_rn(a.y, l), __fdiv_rn(a.z, l)); }
__device__ __forceinline__ P3 hw(const HShape &s, int k) { return s.p + rmul(s, cmul(s.h, f4xyz(s.H[1 + k]))); }
__device__ __forceinline__ int hfidx(const float4 *H, int f, int i) {
    const float4 v = H[29 + 2 * f + i / 4];
    const int r = i & 3;
    return (int)(r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w);
}
__device__ __forceinline__ int hfcnt(const float4 *H, int f) {
    const float4 v = H[77 + f / 4];
    const int r = f & 3;
    return (int)(r == 0 ? v.x : r == 1 ? v.y : r == 2 ? v.z : v.w);
}
__device__ __forceinline__ void hseg(const float4 *H, int k, int &a, int &b) {
    const float4 v = H[53 + k / 2];
    if (k & 1) { a = (int)v.z; b = (int)v.w; } else { a = (int)v.x; b = (int)v.y; }
}
__device__ __forceinline__ void hface(const HShape &s, int f, P3 &n, float &d) {
    const float4 pl = s.H[17 + f];
    const P3 nw = rmul(s, cdiv(p3(pl.x, pl.y, pl.z), s.h));
    const float l = plen(nw);
    n = p3(__fdiv_rn(nw.x, l), __fdiv_rn(nw.y, l), __fdiv_rn(nw.z, l));
    d = __fdiv_rn(pl.w, l) + pdot(n, s.p);
}
struct HContact { P3 n; int cnt; float4 pt[8]; };
__device__ __forceinline__ void hc_add(HContact &c, P3 x, float w) {
    if (c.cnt < 8) { c.pt[c.cnt] = make_float4(x.x, x.y, x.z, w); c.cnt++; return; }
    int hi = 0;
    for (int q = 1; q < 8; q++) if (c.pt[q].w > c.pt[hi].w) hi = q;
    if (w < c.pt[hi].w) c.pt[hi] = make_float4(x.x, x.y, x.z, w);
}
static __device__ void hull_ground(const HShape &s, float margin, HContact &c) {
    c.cnt = 0;
    c.n = p3(0.0f, -1.0f, 0.0f);
    const int nv = (int)s.H[0].x;
    for (int k = 0; k < nv; k++) {
        const P3 x = hw(s, k);
        if (x.y >= margin) continue;
        hc_add(c, p3(x.x, 0.5f * x.y, x.z), x.y);
    }
}
static __device__ void hull_hull(const HShape &A, const HShape &B, float margin, HContact &c) {
    c.cnt = 0;
    c.n = p3(0.0f, 0.0f, 0.0f);
    const float4 ha = A.H[0], hb = B.H[0];
    const int nfa = (int)ha.y, nfb = (int)hb.y, nva = (int)ha.x, nvb = (int)hb.x, nda = (int)ha.w, ndb = (int)hb.w;
    P3 VA[16], VB[16], DA[12], DB[12];
    for (int k = 0; k < nva; k++) VA[k] = hw(A, k);
    for (int k = 0; k < nvb; k++) VB[k] = hw(B, k);
    for (int k = 0; k < nda; k++) DA[k] = pnorm(rmul(A, cmul(A.h, f4xyz(A.H[65 + k]))));
    for (int k = 0; k < ndb; k++) DB[k] = pnorm(rmul(B, cmul(B.h, f4xyz(B.H[65 + k]))));
    float sa = -1e30f; int fa = 0;
    for (int f = 0; f < nfa; f++) {
        P3 n; float d; hface(A, f, n, d);
        float lo = 1e30f;
        for (int k = 0; k < nvb; k++) lo = fminf(lo, pdot(VB[k], n));
        const float s = lo - d;
        if (s > margin) return;
        if (s > sa) { sa = s; fa = f; }
    }
    float sb = -1e30f; int fb = 0;
    for (int f = 0; f < nfb; f++) {
        P3 n; float d; hface(B, f, n, d);
        float lo = 1e30f;
        for (int k = 0; k < nva; k++) lo = fminf(lo, pdot(VA[k], n));
        const float s = lo - d;
        if (s > margin) return;
        if (s > sb) { sb = s; fb = f; }
    }
    float se = -1e30f; P3 el = p3(0.0f, 0.0f, 0.0f); int ei = 0, ej = 0;
    for (int i = 0; i < nda; i++)
        for (int j = 0; j < ndb; j++) {
            const P3 l0 = pcross(DA[i], DB[j]);
            const float l2 = pdot(l0, l0);
            if (l2 < 1e-6f) continue;
            P3 l = l0 * __fdiv_rn(1.0f, __fsqrt_rn(l2));
            float alo = 1e30f, ahi = -1e30f, blo = 1e30f, bhi = -1e30f;
            for (int k = 0; k < nva; k++) { const float d = pdot(VA[k], l); alo = fminf(alo, d); ahi = fmaxf(ahi, d); }
            for (int k = 0; k < nvb; k++) { const float d = pdot(VB[k], l); blo = fminf(blo, d); bhi = fmaxf(bhi, d); }
            const float s1 = blo - ahi, s2 = alo - bhi;
            float s = s1;
            if (s2 > s1) { s = s2; l = -l; }
            if (s > margin) return;
            if (s > se) { se = s; el = l; ei = i; ej = j; }
        }
    const bool use_b = sb > sa + 0.005f;
    const float fbest = use_b ? sb : sa;
    if (se > fbest + 0.01f) {
        const P3 da = pnorm(rmul(A, cmul(A.h, f4xyz(A.H[65 + ei])))), db = pnorm(rmul(B, cmul(B.h, f4xyz(B.H[65 + ej]))));
        P3 a0 = A.p, a1 = A.p;
        float best = -1e30f;
        for (int k = 0; k < (int)ha.z; k++) {
            int x, y; hseg(A.H, k, x, y);
            const P3 q0 = hw(A, x), q1 = hw(A, y);
            if (fabsf(pdot(pnorm(q1 - q0), da)) < 0.999f) continue;
            const float m = pdot(q0 + q1, el);
            if (m > best) { best = m; a0 = q0; a1 = q1; }
        }
        P3 b0 = B.p, b1 = B.p;
        best = 1e30f;
        for (int k = 0; k < (int)hb.z; k++) {
            int x, y; hseg(B.H, k, x, y);
            const P3 q0 = hw(B, x), q1 = hw(B, y);
            if (fabsf(pdot(pnorm(q1 - q0), db)) < 0.999f) continue;
            const float m = pdot(q0 + q1, el);
            if (m < best) { best = m; b0 = q0; b1 = q1; }
        }
        const P3 d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
        const float aa = pdot(d1, d1), ee = pdot(d2, d2), ff = pdot(d2, r), cc = pdot(d1, r), bb = pdot(d1, d2);
        const float den = aa * ee - bb * bb;
        float s1 = 0.0f;
        if (den > 1e-9f) s1 = fminf(fmaxf(__fdiv_rn(bb * ff - cc * ee, den), 0.0f), 1.0f);
        float t1 = __fdiv_rn(bb * s1 + ff, fmaxf(ee, 1e-9f));
        if (t1 < 0.0f) { t1 = 0.0f; s1 = fminf(fmaxf(__fdiv_rn(-cc, fmaxf(aa, 1e-9f)), 0.0f), 1.0f); }
        else if (t1 > 1.0f) { t1 = 1.0f; s1 = fminf(fmaxf(__fdiv_rn(bb - cc, fmaxf(aa, 1e-9f)), 0.0f), 1.0f); }
        const P3 q1 = a0 + d1 * s1, q2 = b0 + d2 * t1;
        const P3 mid = (q1 + q2) * 0.5f;
        c.n = el;
        c.cnt = 1;
        c.pt[0] = make_float4(mid.x, mid.y, mid.z, pdot(q2 - q1, el));
        return;
    }
    const HShape &Rs = use_b ? B : A;
    const HShape &Is = use_b ? A : B;
    const int fr = use_b ? fb : fa;
    P3 n; float rw; hface(Rs, fr, n, rw);
    const int nfi = use_b ? nfa : nfb;
    int fi = 0; float bd = 1e30f;
    for (int f = 0; f < nfi; f++) { P3 m; float d; hface(Is, f, m, d); const float dd = pdot(m, n); if (dd < bd) { bd = dd; fi = f; } }
    P3 poly[16], tmp[16];
    int pn = hfcnt(Is.H, fi);
    for (int q = 0; q < pn; q++) poly[q] = hw(Is, hfidx(Is.H, fi, q));
    const int rn = hfcnt(Rs.H, fr);
    P3 rc = p3(0.0f, 0.0f, 0.0f);
    for (int q = 0; q < rn; q++) rc = rc + hw(Rs, hfidx(Rs.H, fr, q));
    const float frn = (float)rn;
    rc = p3(__fdiv_rn(rc.x, frn), __fdiv_rn(rc.y, frn), __fdiv_rn(rc.z, frn));
    for (int e = 0; e < rn; e++) {
        const P3 v0 = hw(Rs, hfidx(Rs.H, fr, e)), v1 = hw(Rs, hfidx(Rs.H, fr, (e + 1) % rn));
        P3 sn = pnorm(pcross(v1 - v0, n));
        if (pdot(sn, rc - v0) > 0.0f) sn = -sn;
        int tn = 0;
        for (int q = 0; q < pn; q++) {
            const P3 q0 = poly[q], q1 = poly[(q + 1) % pn];
            const float d0 = pdot(q0 - v0, sn), d1 = pdot(q1 - v0, sn);
            if (d0 <= 0.0f && tn < 16) tmp[tn++] = q0;
            if ((d0 <= 0.0f) != (d1 <= 0.0f) && tn < 16) tmp[tn++] = q0 + (q1 - q0) * __fdiv_rn(d0, d0 - d1);
        }
        pn = tn;
        for (int q = 0; q < pn; q++) poly[q] = tmp[q];
        if (pn == 0) return;
    }
    for (int q = 0; q < pn; q++) {
        const P3 pp = poly[q];
        const float sep = pdot(pp, n) - rw;
        if (sep > margin) continue;
        hc_add(c, pp - n * (0.5f * sep), sep);
    }
    c.n = use_b ? -n : n;
}
// gpu/gpu_world.js:532-554
static __device__ void hc_reduce4(HContact &c) {
    const int cnt = c.cnt;
    if (cnt <= 4) return;
    const P3 n = c.n;
    int i0 = 0;
    for (int k = 1; k < cnt; k++) if (c.pt[k].w < c.pt[i0].w) i0 = k;
    const P3 q0 = f4xyz(c.pt[i0]);
    int i1 = 0; float best = -1.0f;
    for (int k = 0; k < cnt; k++) { const P3 d = f4xyz(c.pt[k]) - q0; if (pdot(d, d) > best) { best = pdot(d, d); i1 = k; } }
    const P3 e = f4xyz(c.pt[i1]) - q0;
    int i2 = 0, i3 = 0; float b2 = -1e30f, b3 = -1e30f;
    for (int k = 0; k < cnt; k++) {
        const float a = pdot(pcross(f4xyz(c.pt[k]) - q0, e), n);
        if (a > b2) { b2 = a; i2 = k; }
        if (-a > b3) { b3 = -a; i3 = k; }
    }
    const int sel[4] = {i0, i1, i2, i3};
    float4 out[4]; int oc = 0;
    for (int k = 0; k < 4; k++) {
        bool dup = false;
        for (int q = 0; q < k; q++) if (sel[q] == sel[k]) dup = true;
        if (!dup) out[oc++] = c.pt[sel[k]];
    }
    for (int k = 0; k < oc; k++) c.pt[k] = out[k];
    c.cnt = oc;
}

}  // namespace sf

// Box-box narrow phase, batched: separating-axis test over the 3 + 3 face axes and 9 edge axes, reference/incident
// face clipping or the edge-edge closest points, then reduction to 4 points (engine/src/phys.rs:502-628).
// One thread per pair; the arithmetic keeps the reference's evaluation order (compiled with --fmad=false).
#include <vector>

#include "sf_internal.cuh"
#include "sf_boxsat.cuh"

namespace sf {

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
__device__ void hull_ground(const HShape &s, float margin, HContact &c) {
    c.cnt = 0;
    c.n = p3(0.0f, -1.0f, 0.0f);
    const int nv = (int)s.H[0].x;
    for (int k = 0; k < nv; k++) {
        const P3 x = hw(s, k);
        if (x.y >= margin) continue;
        hc_add(c, p3(x.x, 0.5f * x.y, x.z), x.y);
    }
}
__device__ void hull_hull(const HShape &A, const HShape &B, float margin, HContact &c) {
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
__device__ void hc_reduce4(HContact &c) {
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

__device__ __forceinline__ HShape load_hshape(const float *s, const float4 *hulls) {
    HShape r;
    r.p = p3(s[0], s[1], s[2]);
    const float x = s[3], y = s[4], z = s[5], w = s[6];
    r.c[0] = p3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w));
    r.c[1] = p3(2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w));
    r.c[2] = p3(2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y));
    r.h = p3(s[7], s[8], s[9]);
    r.H = hulls + (size_t)(int)s[10] * 80;
    return r;
}

__global__ void __launch_bounds__(128) k_collide_hulls(const float4 *hulls, uint32_t n_hulls, const float *sa, const float *sb,
                                                       uint32_t n, float margin, int do_reduce, float *out36, int32_t *count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *a = sa + (size_t)i * 11, *b = sb + (size_t)i * 11;
    HContact c;
    c.cnt = 0;
    c.n = p3(0.0f, 0.0f, 0.0f);
    const int ta = (int)a[10], tb = (int)b[10];
    if (ta < 0 || (uint32_t)ta >= n_hulls || (b[10] >= 0.0f && (uint32_t)tb >= n_hulls)) { count[i] = -1; return; }
    const HShape A = load_hshape(a, hulls);
    if (b[10] < 0.0f) hull_ground(A, margin, c);
    else hull_hull(A, load_hshape(b, hulls), margin, c);
    if (do_reduce) hc_reduce4(c);
    float *o = out36 + (size_t)i * 36;
    o[0] = c.n.x; o[1] = c.n.y; o[2] = c.n.z; o[3] = 0.0f;
    for (int k = 0; k < 8; k++) {
        const float4 v = k < c.cnt ? c.pt[k] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        o[4 + 4 * k] = v.x; o[5 + 4 * k] = v.y; o[6 + 4 * k] = v.z; o[7 + 4 * k] = v.w;
    }
    count[i] = c.cnt;
}

__global__ void k_collide_boxes(const float *ba, const float *bb, uint32_t n, float margin, float *out20, int32_t *count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Box A = load_box(ba + (size_t)i * 10), B = load_box(bb + (size_t)i * 10);
    CPt pts[8];
    P3 nrm = p3(0.0f, 0.0f, 0.0f);
    int c = collide_boxes(A, B, margin, pts, &nrm);
    if (c) c = reduce4(pts, c, nrm);
    float *o = out20 + (size_t)i * 20;
    o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
    for (int k = 0; k < 4; k++) {
        bool ok = k < c;
        o[4 + 4 * k] = ok ? pts[k].p.x : 0.0f;
        o[5 + 4 * k] = ok ? pts[k].p.y : 0.0f;
        o[6 + 4 * k] = ok ? pts[k].p.z : 0.0f;
        o[7 + 4 * k] = ok ? pts[k].s : 0.0f;
    }
    o[3] = 0.0f;
    count[i] = c;
}

}  // namespace sf

using namespace sf;

extern "C" sf_status sf_collide_boxes(const float *boxes_a, const float *boxes_b, uint32_t n_pairs, float margin, float *out20,
                                      int32_t *count) {
    if (n_pairs == 0) return SF_OK;
    if (!boxes_a || !boxes_b || !out20 || !count) { set_error("null argument"); return SF_ERR_ARG; }
    cudaStream_t s = nullptr;
    SF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DBuf<float> da, db, dout;
    DBuf<int32_t> dc;
    sf_status r = SF_OK;
    do {
        if (da.alloc((size_t)n_pairs * 10) || db.alloc((size_t)n_pairs * 10) || dout.alloc((size_t)n_pairs * 20) || dc.alloc(n_pairs)) {
            set_error("device allocation failed"); r = SF_ERR_CUDA; break;
        }
        cudaMemcpyAsync(da.p, boxes_a, (size_t)n_pairs * 40, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(db.p, boxes_b, (size_t)n_pairs * 40, cudaMemcpyHostToDevice, s);
        k_collide_boxes<<<grid_for(n_pairs, 128), 128, 0, s>>>(da.p, db.p, n_pairs, margin, dout.p, dc.p);
        cudaMemcpyAsync(out20, dout.p, (size_t)n_pairs * 80, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(count, dc.p, (size_t)n_pairs * 4, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error("box SAT: %s", cudaGetErrorString(e)); r = SF_ERR_CUDA; }
    } while (0);
    cudaStreamDestroy(s);
    return r;
}

extern "C" sf_status sf_collide_hulls(const float *hull_data, uint32_t n_hulls, const float *shapes_a, const float *shapes_b,
                                      uint32_t n_pairs, float margin, int32_t reduce, float *out36, int32_t *count) {
    if (n_pairs == 0) return SF_OK;
    if (!hull_data || !n_hulls || !shapes_a || !shapes_b || !out36 || !count) { set_error("null argument"); return SF_ERR_ARG; }
    for (uint32_t i = 0; i < n_pairs; i++) {
        const float ta = shapes_a[(size_t)i * 11 + 10], tb = shapes_b[(size_t)i * 11 + 10];
        if (!(ta >= 0.0f && ta < (float)n_hulls) || !(tb < (float)n_hulls)) { set_error("pair %u: hull id out of range", i); return SF_ERR_ARG; }
    }
    cudaStream_t s = nullptr;
    SF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DBuf<float4> dh;
    DBuf<float> da, db, dout;
    DBuf<int32_t> dc;
    sf_status r = SF_OK;
    do {
        if (dh.alloc((size_t)n_hulls * 80) || da.alloc((size_t)n_pairs * 11) || db.alloc((size_t)n_pairs * 11) ||
            dout.alloc((size_t)n_pairs * 36) || dc.alloc(n_pairs)) {
            set_error("device allocation failed"); r = SF_ERR_CUDA; break;
        }
        cudaMemcpyAsync(dh.p, hull_data, (size_t)n_hulls * 80 * 16, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(da.p, shapes_a, (size_t)n_pairs * 44, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(db.p, shapes_b, (size_t)n_pairs * 44, cudaMemcpyHostToDevice, s);
        k_collide_hulls<<<grid_for(n_pairs, 128), 128, 0, s>>>(dh.p, n_hulls, da.p, db.p, n_pairs, margin, reduce ? 1 : 0, dout.p, dc.p);
        cudaMemcpyAsync(out36, dout.p, (size_t)n_pairs * 36 * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(count, dc.p, (size_t)n_pairs * 4, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error("hull SAT: %s", cudaGetErrorString(e)); r = SF_ERR_CUDA; }
    } while (0);
    cudaStreamDestroy(s);
    return r;
}

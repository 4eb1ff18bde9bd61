// The engine crate's box world on the GPU (engine/src/phys.rs World::step, phys.rs:152-243): oriented boxes, the
// hashed-grid broadphase (phys.rs:356-408), ground and pair collisions with box SAT (phys.rs:410-445, 502-628),
// push_manifold with its warm start and friction anchors (phys.rs:447-497), the soft-step sub-steps (warm start,
// biased solve, integrate, relax; phys.rs:216-324) and island sleep (phys.rs:326-354).
//
// One thread block runs one scene's whole step; a launch steps every scene of the world. Inside a scene:
//   * the grid is a hash table of cell lists (linked entries, one per body and covered cell); the pair set is the
//     reference's (AABB overlap, reported in the cell of the larger minimum corner);
//   * every body lists its pairs with higher-numbered bodies, sorted, then its ground contact, so the manifold list
//     comes out in key order (a, b; ground as b = NONE) with no global sort, and the previous step's manifolds are
//     found by binary search in that order;
//   * manifolds are coloured greedily in a fixed priority order (Jones-Plassmann rounds reach the same colouring),
//     and each solve pass runs colour by colour with a block barrier between colours: inside a colour no two
//     manifolds share a moving body, so the result does not depend on the thread schedule;
//   * sleeping islands come from a lock-free union-find over the manifolds between two moving bodies.
// The f32 arithmetic keeps the reference's evaluation order (compiled with --fmad=false).
#include <algorithm>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "sf_internal.cuh"
#include "sf_boxsat.cuh"

namespace sf {
namespace {

constexpr uint32_t BX_NONE = 0xFFFFFFFFu;     // the ground
constexpr uint32_t BX_GROUND2 = 0xFFFFFFFEu;  // the second ground patch of a convex cell (corners 5-8)
__host__ __device__ __forceinline__ bool is_ground(uint32_t b) { return b >= BX_GROUND2; }
constexpr uint32_t BX_UNC = 0xFFFFFFFFu;
constexpr uint32_t BX_PPB = 48;      // pairs (with a higher-numbered body) a body may take, on average over its scene
constexpr uint32_t BX_SHORT = 32;    // pair lists up to this long are sorted by their own thread
constexpr uint32_t BX_EPB = 27;      // grid entries a body may take, on average over its scene
constexpr uint32_t BX_CPB = 8;       // manifolds a body may take, on average over its scene
constexpr int BX_MAXC = 128;         // colours
constexpr uint32_t BX_BIG = 4096;    // scenes above this many boxes step on a thread-block cluster
constexpr int BX_CL = 16, BX_CL_THREADS = 512;
enum { BXE_ENTRIES = 1, BXE_PAIRS = 2, BXE_MANIFOLDS = 4, BXE_COLOURS = 8, BXE_GUARD = 16 };

struct DM3 { P3 c[3]; };
struct BxBody { P3 p; float q[4]; P3 v, w, h; float inv_m; P3 inv_i; float sleep_t; P3 sleep_p; float sleep_q[4]; uint32_t awake, hull; };
struct DCp { P3 ra, rb, la, raxn, rbxn, iaxn, ibxn; float adj, nm, jn; };
struct DMan {
    uint32_t a, b, sa, sb; P3 n, t1, t2; float mu; uint32_t cnt, stick;
    DCp cp[4];
    P3 fa, fb, la_f, lb_f, e0; float tm1, tm2, twm, rad, jt1, jt2, jtw;
    P3 ca1, ca2, cb1, cb2, ia1, ia2, ib1, ib2, ian, ibn; float ima, imb;
};

struct BxArgs {
    BxBody *body;
    const float4 *hulls;     // the convex-cell library, 80 float4 a cell; a body's hull 0 is the whole box
    DM3 *rot; P3 *amin, *amax;
    uint32_t *ecnt, *sidx, *cand_n, *seglong, *uf, *mint;
    uint8_t *wake;
    uint32_t *ent_body, *ent_next, *head; int32_t *ent_cell;
    uint32_t *cand_a, *cand_b, *hit; float *geom;
    DMan *man[2]; uint64_t *mkey[2]; uint32_t *mcount[2];
    uint32_t *deg, *inc, *colour, *corder, *mwait;
    uint64_t *mrank;
    P3 *sv, *sw, *sdp, *sth, *sp0; float *sim; DM3 *sii; float4 *sq;
    const uint32_t *sc_b0, *sc_n, *sc_e0, *sc_t0, *sc_tcap, *sc_c0, *sc_m0;   // candidates at c0, manifolds at m0
    uint32_t *gs;        // BX_G words a scene: the team-wide words of a cluster team
    uint32_t *stats;     // 8 a scene: awake, pairs, manifolds, points, colours, status, JP rounds, 0
    unsigned long long *tns;   // 5 a scene: ns in broadphase, narrow phase, colouring, sub-steps, write-back and sleep
    sf_box_params P;
};

// ---------------------------------------------------------------- math (engine/src/math.rs)
__device__ __forceinline__ float plen2(P3 a) { return pdot(a, a); }
__device__ __forceinline__ float plen_e(P3 a) { return sqrt_e(plen2(a)); }
__device__ __forceinline__ float maxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float pget(P3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ P3 pnorm_e(P3 a) { float l = plen_e(a); return l > 1e-12f ? a * __fdiv_rn(1.0f, l) : p3(0.0f, 0.0f, 0.0f); }
__device__ __forceinline__ P3 m_mulv(const DM3 &r, P3 v) { return r.c[0] * v.x + r.c[1] * v.y + r.c[2] * v.z; }
__device__ __forceinline__ P3 m_tmulv(const DM3 &r, P3 v) { return p3(pdot(r.c[0], v), pdot(r.c[1], v), pdot(r.c[2], v)); }
__device__ __forceinline__ DM3 qm3(const float *q) {   // Quat::to_m3 (math.rs:54-60)
    float x = q[0], y = q[1], z = q[2], w = q[3];
    DM3 m;
    m.c[0] = p3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w));
    m.c[1] = p3(2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w));
    m.c[2] = p3(2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y));
    return m;
}
__device__ __forceinline__ DM3 m_sandwich(const DM3 &r, P3 d) {   // R diag(d) R^T (math.rs:71-75)
    P3 a = r.c[0] * d.x, b = r.c[1] * d.y, c = r.c[2] * d.z;
    DM3 o;
    for (int j = 0; j < 3; j++) o.c[j] = a * pget(r.c[0], j) + b * pget(r.c[1], j) + c * pget(r.c[2], j);
    return o;
}
__device__ __forceinline__ float4 qmul(float4 a, float4 o) {   // Quat::mul (math.rs:36-41), (x, y, z, w)
    return make_float4(a.w * o.x + a.x * o.w + a.y * o.z - a.z * o.y,
                       a.w * o.y - a.x * o.z + a.y * o.w + a.z * o.x,
                       a.w * o.z + a.x * o.y - a.y * o.x + a.z * o.w,
                       a.w * o.w - a.x * o.x - a.y * o.y - a.z * o.z);
}
__device__ __forceinline__ float4 qintegrate(float4 q, P3 w, float h) {   // Quat::integrate + normalized (math.rs:42-47)
    float4 dq = qmul(make_float4(w.x, w.y, w.z, 0.0f), q);
    float4 r = make_float4(q.x + 0.5f * h * dq.x, q.y + 0.5f * h * dq.y, q.z + 0.5f * h * dq.z, q.w + 0.5f * h * dq.w);
    float l = sqrt_e(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
    float k = l > 0.0f ? __fdiv_rn(1.0f, l) : 1.0f;
    return make_float4(r.x * k, r.y * k, r.z * k, r.w * k);
}
__device__ __forceinline__ void btangents(P3 n, P3 &t1, P3 &t2) {   // phys.rs:500-503
    P3 t = fabsf(n.x) > 0.57f ? p3(n.y, -n.x, 0.0f) : p3(0.0f, n.z, -n.y);
    t1 = pnorm_e(t);
    t2 = pcross(n, t1);
}
__device__ __forceinline__ float bfloor(float x) { float t = (float)(int32_t)x; return t > x ? t - 1.0f : t; }
__device__ __forceinline__ int32_t bcell(float x, float inv_cell) { return (int32_t)bfloor(x * inv_cell); }
__device__ __forceinline__ uint32_t bhash(int32_t x, int32_t y, int32_t z) {
    return (uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u;
}
// the colouring's manifold priority: a fixed mix of the body pair (b' = 0 for the ground, else b + 1)
__device__ __forceinline__ uint32_t pair_priority(uint32_t a, uint32_t bp) {
    uint32_t h = a * 0x9E3779B1u + bp * 0x85EBCA6Bu;
    h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
    return h;
}
__device__ __forceinline__ uint64_t man_rank(uint32_t a, uint32_t b, uint32_t m) {
    return ((uint64_t)pair_priority(a, is_ground(b) ? 0u : b + 1) << 32) | (uint64_t)(0xFFFFFFFFu - m);
}

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long x;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(x));
    return x;
}

__device__ __forceinline__ Box make_box(const BxBody &b, const DM3 &r) {
    Box x;
    x.p = b.p; x.c[0] = r.c[0]; x.c[1] = r.c[1]; x.c[2] = r.c[2]; x.h[0] = b.h.x; x.h[1] = b.h.y; x.h[2] = b.h.z;
    return x;
}

__device__ __forceinline__ HShape hshape(const BxBody &b, const DM3 &r, const float4 *hulls) {
    HShape s;
    s.p = b.p; s.c[0] = r.c[0]; s.c[1] = r.c[1]; s.c[2] = r.c[2]; s.h = b.h; s.H = hulls + (size_t)b.hull * 80;
    return s;
}
// a convex-cell contact reduced to 4 points (gpu/gpu_world.js:532-554, in emit) into the candidate's geometry words
__device__ int hull_out(HContact &c, float *g) {
    if (c.cnt) hc_reduce4(c);
    g[0] = c.n.x; g[1] = c.n.y; g[2] = c.n.z; g[3] = __int_as_float(c.cnt);
    for (int k = 0; k < 4; k++) {
        const bool ok = k < c.cnt;
        g[4 + 4 * k] = ok ? c.pt[k].x : 0.0f; g[5 + 4 * k] = ok ? c.pt[k].y : 0.0f;
        g[6 + 4 * k] = ok ? c.pt[k].z : 0.0f; g[7 + 4 * k] = ok ? c.pt[k].w : 0.0f;
    }
    return c.cnt;
}
// the ground candidates of a body: its ground contact, and a convex cell's second patch before it
__device__ __forceinline__ uint32_t ground_slots(const BxBody &b, P3 lo) { return b.awake && lo.y < 0.0f ? (b.hull ? 2u : 1u) : 0u; }

// collide_ground (phys.rs:419-432) or collide_pair (phys.rs:434-445) of candidate (a, b); the geometry goes to
// g[20] = normal 3, count, 4 x (point 3, depth). A wake is recorded (applied after every candidate has read the
// flags): the woken set is the same as waking at once, since a wake only turns a sleeping body awake.
__device__ int collide_candidate(const BxArgs &A, uint32_t b0, uint32_t a, uint32_t b, float *g) {
    const BxBody ba = A.body[b0 + a];
    const DM3 ra = A.rot[b0 + a];
    CPt pts[8]; P3 n = p3(0.0f, 0.0f, 0.0f);
    int cnt = 0;
    if (is_ground(b) && ba.hull) {
        // a convex cell on the ground (gpu/gpu_world.js:809-823): its corners under the margin, the first four as
        // one patch, the rest as a second
        const float margin = A.P.speculative + maxf(-ba.v.y, 0.0f) * (1.0f / 60.0f);
        HContact c;
        hull_ground(hshape(ba, ra, A.hulls), margin, c);
        const int lo = b == BX_GROUND2 ? 4 : 0, hi = b == BX_GROUND2 ? c.cnt : min(c.cnt, 4);
        HContact d;
        d.n = c.n; d.cnt = 0;
        for (int k = lo; k < hi; k++) d.pt[d.cnt++] = c.pt[k];
        return hull_out(d, g);
    }
    if (!is_ground(b) && (ba.hull || A.body[b0 + b].hull)) {
        // a pair with a convex cell (gpu/gpu_world.js:824-832); a plain box is the library's whole cube
        const BxBody bb = A.body[b0 + b];
        const DM3 rb = A.rot[b0 + b];
        const bool a_awake = ba.awake != 0, b_awake = bb.awake != 0, a_still = ba.sleep_t != 0.0f, b_still = bb.sleep_t != 0.0f;
        const float rel = plen_e(bb.v - ba.v) + plen_e(ba.w) * plen_e(ba.h) + plen_e(bb.w) * plen_e(bb.h);
        const float margin = A.P.speculative + rel * (1.0f / 60.0f);
        HContact c;
        hull_hull(hshape(ba, ra, A.hulls), hshape(bb, rb, A.hulls), margin, c);
        if (c.cnt) {
            if (a_awake && !b_awake && !a_still) A.wake[b0 + b] = 1;
            if (b_awake && !a_awake && !b_still) A.wake[b0 + a] = 1;
        }
        return hull_out(c, g);
    }
    if (is_ground(b)) {
        const float margin = A.P.speculative + maxf(-ba.v.y, 0.0f) * (1.0f / 60.0f);
        for (int k = 0; k < 8; k++) {
            P3 s = p3(k & 1 ? 1.0f : -1.0f, k & 2 ? 1.0f : -1.0f, k & 4 ? 1.0f : -1.0f);
            P3 c = ba.p + m_mulv(ra, p3(s.x * ba.h.x, s.y * ba.h.y, s.z * ba.h.z));
            if (c.y < margin) { pts[cnt].p = p3(c.x, 0.5f * c.y, c.z); pts[cnt].s = c.y; cnt++; }
        }
        n = p3(0.0f, -1.0f, 0.0f);
    } else {
        const BxBody bb = A.body[b0 + b];
        const DM3 rb = A.rot[b0 + b];
        const bool a_awake = ba.awake != 0, b_awake = bb.awake != 0, a_still = ba.sleep_t != 0.0f, b_still = bb.sleep_t != 0.0f;
        const float rel = plen_e(bb.v - ba.v) + plen_e(ba.w) * plen_e(ba.h) + plen_e(bb.w) * plen_e(bb.h);
        const float margin = A.P.speculative + rel * (1.0f / 60.0f);
        cnt = collide_boxes(make_box(ba, ra), make_box(bb, rb), margin, pts, &n);
        if (cnt) {
            if (a_awake && !b_awake && !a_still) A.wake[b0 + b] = 1;
            if (b_awake && !a_awake && !b_still) A.wake[b0 + a] = 1;
        }
    }
    if (cnt) cnt = reduce4(pts, cnt, n);
    g[0] = n.x; g[1] = n.y; g[2] = n.z; g[3] = __int_as_float(cnt);
    for (int k = 0; k < 4; k++) {
        const bool ok = k < cnt;
        g[4 + 4 * k] = ok ? pts[k].p.x : 0.0f; g[5 + 4 * k] = ok ? pts[k].p.y : 0.0f;
        g[6 + 4 * k] = ok ? pts[k].p.z : 0.0f; g[7 + 4 * k] = ok ? pts[k].s : 0.0f;
    }
    return cnt;
}

// push_manifold (phys.rs:447-497) and the manifold's masses (phys.rs:189-213)
__device__ void build_manifold(const BxArgs &A, int par, uint32_t b0, uint32_t s0, uint32_t m0, uint32_t nold,
                               uint32_t a, uint32_t b, const float *g, DMan &m) {
    const BxBody &ba = A.body[b0 + a];
    const P3 pa = ba.p;
    const DM3 ra = A.rot[b0 + a];
    const P3 pb = !is_ground(b) ? A.body[b0 + b].p : p3(0.0f, 0.0f, 0.0f);
    const uint32_t sa = A.sidx[b0 + a], sbi = !is_ground(b) ? A.sidx[b0 + b] : 0u;
    const P3 n = p3(g[0], g[1], g[2]);
    const int cnt = __float_as_int(g[3]);
    m.a = a; m.b = b; m.sa = sa; m.sb = sbi; m.n = n; btangents(n, m.t1, m.t2); m.mu = A.P.friction;
    m.cnt = (uint32_t)cnt; m.stick = A.P.anchor != 0;
    m.jt1 = m.jt2 = m.jtw = 0.0f;
    // the previous step's manifold of the pair: binary search of its key-ordered list
    const uint64_t key = ((uint64_t)a << 32) | b;
    const uint64_t *ok = A.mkey[par ^ 1] + m0;
    uint32_t lo = 0, hi = nold;
    while (lo < hi) { uint32_t mid = (lo + hi) >> 1; if (ok[mid] < key) lo = mid + 1; else hi = mid; }
    const DMan *o = (lo < nold && ok[lo] == key) ? A.man[par ^ 1] + m0 + lo : nullptr;
    DM3 rbm;
    rbm.c[0] = p3(1.0f, 0.0f, 0.0f); rbm.c[1] = p3(0.0f, 1.0f, 0.0f); rbm.c[2] = p3(0.0f, 0.0f, 1.0f);
    if (!is_ground(b)) rbm = A.rot[b0 + b];
    P3 pt[4]; float dep[4];
    for (int k = 0; k < 4; k++) { pt[k] = p3(g[4 + 4 * k], g[5 + 4 * k], g[6 + 4 * k]); dep[k] = g[7 + 4 * k]; }
    P3 cen = p3(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < cnt; k++) cen = cen + pt[k];
    cen = cen * __fdiv_rn(1.0f, (float)cnt);
    float rad = 0.0f;
    for (int k = 0; k < cnt; k++) rad += plen_e(pt[k] - cen);
    m.rad = __fdiv_rn(rad, (float)cnt);
    bool anchored = false;
    if (o) {
        if (o->stick) {
            P3 wa = pa + m_mulv(ra, o->la_f);
            P3 wb = !is_ground(b) ? pb + m_mulv(rbm, o->lb_f) : o->lb_f;
            float lim = maxf(0.05f, m.rad);
            if (plen2(wa - cen) < lim * lim && plen2(wb - wa) < 0.03f * 0.03f) {
                m.la_f = o->la_f; m.lb_f = o->lb_f; m.fa = wa - pa; m.fb = wb - pb; m.e0 = wb - wa; anchored = true;
            }
        }
        P3 f = o->t1 * o->jt1 + o->t2 * o->jt2;
        m.jt1 = pdot(f, m.t1); m.jt2 = pdot(f, m.t2); m.jtw = o->jtw * pdot(o->n, n);
    }
    if (!anchored) {
        m.fa = cen - pa; m.fb = cen - pb; m.la_f = m_tmulv(ra, m.fa);
        m.lb_f = !is_ground(b) ? m_tmulv(rbm, m.fb) : cen;
        m.e0 = p3(0.0f, 0.0f, 0.0f);
    }
    const float ima = A.sim[s0 + sa], imb = A.sim[s0 + sbi];
    const DM3 iia = A.sii[s0 + sa], iib = A.sii[s0 + sbi];
    m.ima = ima; m.imb = imb;
    for (int k = 0; k < 4; k++) {
        DCp c;
        if (k < cnt) {
            c.ra = pt[k] - pa;
            c.rb = !is_ground(b) ? pt[k] - pb : pt[k];
            c.adj = dep[k];
            c.la = m_tmulv(ra, c.ra);
            c.jn = 0.0f;
            if (o) {
                float best = 0.03f * 0.03f; int bi = -1;
                for (uint32_t q = 0; q < o->cnt; q++) { float d = plen2(o->cp[q].la - c.la); if (d < best) { best = d; bi = (int)q; } }
                if (bi >= 0) c.jn = o->cp[bi].jn;
            }
            c.raxn = pcross(c.ra, n); c.rbxn = pcross(c.rb, n);
            c.iaxn = m_mulv(iia, c.raxn); c.ibxn = m_mulv(iib, c.rbxn);
            float kk = ima + imb + pdot(c.raxn, c.iaxn) + pdot(c.rbxn, c.ibxn);
            c.nm = kk > 0.0f ? __fdiv_rn(1.0f, kk) : 0.0f;
        } else {
            c.ra = c.rb = c.la = c.raxn = c.rbxn = c.iaxn = c.ibxn = p3(0.0f, 0.0f, 0.0f);
            c.adj = c.nm = c.jn = 0.0f;
        }
        m.cp[k] = c;
    }
    m.ca1 = pcross(m.fa, m.t1); m.ca2 = pcross(m.fa, m.t2); m.cb1 = pcross(m.fb, m.t1); m.cb2 = pcross(m.fb, m.t2);
    m.ia1 = m_mulv(iia, m.ca1); m.ia2 = m_mulv(iia, m.ca2); m.ib1 = m_mulv(iib, m.cb1); m.ib2 = m_mulv(iib, m.cb2);
    float k1 = ima + imb + pdot(m.ca1, m.ia1) + pdot(m.cb1, m.ib1);
    float k2 = ima + imb + pdot(m.ca2, m.ia2) + pdot(m.cb2, m.ib2);
    m.tm1 = k1 > 0.0f ? __fdiv_rn(1.0f, k1) : 0.0f; m.tm2 = k2 > 0.0f ? __fdiv_rn(1.0f, k2) : 0.0f;
    m.ian = m_mulv(iia, n); m.ibn = m_mulv(iib, n);
    float kt = pdot(n, m.ian) + pdot(n, m.ibn);
    m.twm = kt > 0.0f ? __fdiv_rn(1.0f, kt) : 0.0f;
}

// World::warm_start for one manifold (phys.rs:245-263); the static side (slot 0) reads zeros and is not written
__device__ void warm_manifold(const BxArgs &A, uint32_t s0, const DMan &m) {
    const uint32_t sa = m.sa, sbi = m.sb;
    P3 va = A.sv[s0 + sa], wa = A.sw[s0 + sa], vb = A.sv[s0 + sbi], wb = A.sw[s0 + sbi];
    float pn = 0.0f;
    for (uint32_t k = 0; k < m.cnt; k++) {
        const float jn = m.cp[k].jn;
        pn += jn; wa = wa - m.cp[k].iaxn * jn; wb = wb + m.cp[k].ibxn * jn;
    }
    const P3 p = m.n * pn + m.t1 * m.jt1 + m.t2 * m.jt2;
    va = va - p * m.ima; vb = vb + p * m.imb;
    wa = wa - (m.ia1 * m.jt1 + m.ia2 * m.jt2 + m.ian * m.jtw);
    wb = wb + (m.ib1 * m.jt1 + m.ib2 * m.jt2 + m.ibn * m.jtw);
    if (sa) { A.sv[s0 + sa] = va; A.sw[s0 + sa] = wa; }
    if (sbi) { A.sv[s0 + sbi] = vb; A.sw[s0 + sbi] = wb; }
}

// World::solve for one manifold (phys.rs:265-324)
__device__ void solve_manifold(const BxArgs &A, uint32_t s0, DMan &m, bool use_bias, float inv_h, float bias_rate,
                               float mass_scale, float imp_scale) {
    const float max_push = A.P.max_push, ap = A.P.anchor_push, slop = A.P.anchor_slop;
    const uint32_t sa = m.sa, sbi = m.sb;
    P3 va = A.sv[s0 + sa], wa = A.sw[s0 + sa], vb = A.sv[s0 + sbi], wb = A.sw[s0 + sbi];
    const P3 tha = A.sth[s0 + sa], thb = A.sth[s0 + sbi];
    const P3 n = m.n, t1 = m.t1, t2 = m.t2;
    const P3 dpab = A.sdp[s0 + sbi] - A.sdp[s0 + sa];
    const float dn = pdot(dpab, n);
    const float ima = m.ima, imb = m.imb;
    float tot = 0.0f;
    for (uint32_t k = 0; k < m.cnt; k++) {
        DCp &c = m.cp[k];
        const float s = c.adj + dn + pdot(thb, c.rbxn) - pdot(tha, c.raxn);
        float bias, ms, is;
        if (s > 0.0f) { bias = s * inv_h; ms = 1.0f; is = 0.0f; }
        else if (use_bias) { bias = maxf(bias_rate * s, -max_push); ms = mass_scale; is = imp_scale; }
        else { bias = 0.0f; ms = 1.0f; is = 0.0f; }
        const float vn = pdot(vb - va, n) + pdot(wb, c.rbxn) - pdot(wa, c.raxn);
        const float jn = c.jn;
        float imp = -c.nm * ms * (vn + bias) - is * jn;
        const float nj = maxf(jn + imp, 0.0f);
        imp = nj - jn; c.jn = nj; tot += nj;
        va = va - n * (imp * ima); wa = wa - c.iaxn * imp;
        vb = vb + n * (imp * imb); wb = wb + c.ibxn * imp;
    }
    const float lim = m.mu * tot;
    const P3 dv = vb - va;
    const float v1 = pdot(dv, t1) + pdot(wb, m.cb1) - pdot(wa, m.ca1);
    const float v2 = pdot(dv, t2) + pdot(wb, m.cb2) - pdot(wa, m.ca2);
    const bool anchored = use_bias && m.stick;
    float b1 = 0.0f, b2 = 0.0f, ms = 1.0f, is = 0.0f;
    if (anchored) {
        const float e1 = pdot(m.e0, t1) + pdot(dpab, t1) + pdot(thb, m.cb1) - pdot(tha, m.ca1);
        const float e2 = pdot(m.e0, t2) + pdot(dpab, t2) + pdot(thb, m.cb2) - pdot(tha, m.ca2);
        const float s1 = e1 > slop ? e1 - slop : (e1 < -slop ? e1 + slop : 0.0f);
        const float s2 = e2 > slop ? e2 - slop : (e2 < -slop ? e2 + slop : 0.0f);
        b1 = minf(maxf(bias_rate * s1, -ap), ap);
        b2 = minf(maxf(bias_rate * s2, -ap), ap);
        ms = mass_scale; is = imp_scale;
    }
    const float o1 = m.jt1, o2 = m.jt2;
    float j1 = o1 - m.tm1 * ms * (v1 + b1) - is * o1;
    float j2 = o2 - m.tm2 * ms * (v2 + b2) - is * o2;
    const float l2 = j1 * j1 + j2 * j2;
    if (l2 > lim * lim) { const float kf = __fdiv_rn(lim, sqrt_e(l2)); j1 *= kf; j2 *= kf; m.stick = 0; }
    m.jt1 = j1; m.jt2 = j2;
    const float d1 = j1 - o1, d2 = j2 - o2;
    const P3 p = t1 * d1 + t2 * d2;
    va = va - p * ima; wa = wa - (m.ia1 * d1 + m.ia2 * d2);
    vb = vb + p * imb; wb = wb + (m.ib1 * d1 + m.ib2 * d2);
    const float wl = lim * m.rad;
    const float ot = m.jtw;
    const float jt = minf(maxf(ot - m.twm * pdot(wb - wa, n), -wl), wl);
    m.jtw = jt;
    const float dtw = jt - ot;
    wa = wa - m.ian * dtw; wb = wb + m.ibn * dtw;
    if (sa) { A.sv[s0 + sa] = va; A.sw[s0 + sa] = wa; }
    if (sbi) { A.sv[s0 + sbi] = vb; A.sw[s0 + sbi] = wb; }
}

__device__ __forceinline__ uint32_t uf_root(const uint32_t *uf, uint32_t x) {
    for (int g = 0; g < 1 << 20; g++) { uint32_t p = ((volatile const uint32_t *)uf)[x]; if (p == x) return x; x = p; }
    return x;
}

// the pairs of body a with the bodies above it (phys.rs:385-404): the entries of a's cells, in the same cell, with an
// awake side and a moving side, overlapping, and reported in the cell of the larger minimum corner. Writes them (in
// walk order) when ca/cb are given; returns the count.
__device__ uint32_t walk_pairs(const BxArgs &A, uint32_t b0, uint32_t e0, uint32_t t0, uint32_t mask, uint32_t ne_tot,
                               float inv_cell, uint32_t a, uint32_t *ca, uint32_t *cb) {
    const P3 lo = A.amin[b0 + a], hi = A.amax[b0 + a];
    const BxBody &ba = A.body[b0 + a];
    const bool a_awake = ba.awake != 0, a_static = ba.inv_m == 0.0f;
    uint32_t k = 0;
    const int32_t x0 = bcell(lo.x, inv_cell), y0 = bcell(lo.y, inv_cell), z0 = bcell(lo.z, inv_cell);
    const int32_t x1 = bcell(hi.x, inv_cell), y1 = bcell(hi.y, inv_cell), z1 = bcell(hi.z, inv_cell);
    for (int32_t x = x0; x <= x1; x++) for (int32_t y = y0; y <= y1; y++) for (int32_t z = z0; z <= z1; z++) {
        uint32_t guard = 0;
        for (uint32_t e = A.head[t0 + (bhash(x, y, z) & mask)]; e != BX_NONE && guard <= ne_tot; e = A.ent_next[e0 + e], guard++) {
            const uint32_t ib = A.ent_body[e0 + e];
            if (ib <= a) continue;
            const int32_t *cc = A.ent_cell + 3 * (size_t)(e0 + e);
            if (cc[0] != x || cc[1] != y || cc[2] != z) continue;
            const BxBody &bb = A.body[b0 + ib];
            if (!a_awake && !bb.awake) continue;
            if (a_static && bb.inv_m == 0.0f) continue;
            const P3 blo = A.amin[b0 + ib], bhi = A.amax[b0 + ib];
            if (lo.x > bhi.x || blo.x > hi.x || lo.y > bhi.y || blo.y > hi.y || lo.z > bhi.z || blo.z > hi.z) continue;
            if (bcell(maxf(lo.x, blo.x), inv_cell) != x || bcell(maxf(lo.y, blo.y), inv_cell) != y ||
                bcell(maxf(lo.z, blo.z), inv_cell) != z) continue;
            if (cb) { ca[k] = a; cb[k] = ib; }
            k++;
        }
    }
    return k;
}

namespace cg = cooperative_groups;
// team-wide words: errors, colours, grid entries (64-bit), counters, per-block scan totals, round flags, colour counts
// and colour starts
enum { G_ERR = 0, G_NCOL = 1, G_NE = 2, G_TOT = 8, G_CTA = 16, G_FLAG = 32, G_CCNT = 64, G_CBEG = 64 + BX_MAXC,
       BX_G = 64 + 2 * BX_MAXC + 64 };

template <int CL>
__device__ __forceinline__ void team_sync() {
    if constexpr (CL == 1) __syncthreads(); else cg::this_cluster().sync();
}
// the OR of p over the team; a cluster uses three flags in turn (the one it clears was last read two rounds back)
template <int CL>
__device__ __forceinline__ bool team_or(int p, uint32_t *G, uint32_t r, uint32_t t) {
    if constexpr (CL == 1) {
        return __syncthreads_or(p) != 0;
    } else {
        if (p) atomicOr(&G[G_FLAG + r % 3], 1u);
        if (t == 0) ((volatile uint32_t *)G)[G_FLAG + (r + 1) % 3] = 0;
        cg::this_cluster().sync();
        return ((volatile uint32_t *)G)[G_FLAG + r % 3] != 0;
    }
}
// exclusive scan of d[0, n) in place by the whole team; returns the total (to every thread)
template <int T, int CL>
__device__ uint32_t team_scan(uint32_t *d, uint32_t n, uint32_t *wsum, uint32_t *gcta, uint32_t tt, uint32_t rank) {
    constexpr uint32_t TT = T * CL;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = T >> 5;
    const uint32_t per = (n + TT - 1) / TT, lo = min(n, tt * per), hi = min(n, lo + per);
    uint32_t s = 0;
    for (uint32_t i = lo; i < hi; i++) s += d[i];
    uint32_t x = s;
    for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o); if (lane >= (uint32_t)o) x += y; }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? wsum[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) { uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o); if (lane >= (uint32_t)o) w += y; }
        wsum[lane] = w;
    }
    __syncthreads();
    uint32_t run = x - s + (warp ? wsum[warp - 1] : 0u);
    uint32_t total = wsum[nw - 1];
    if constexpr (CL > 1) {
        if (threadIdx.x == 0) ((volatile uint32_t *)gcta)[rank] = total;
        cg::this_cluster().sync();
        uint32_t base = 0, all = 0;
        for (uint32_t r = 0; r < CL; r++) { const uint32_t v = ((volatile uint32_t *)gcta)[r]; if (r < rank) base += v; all += v; }
        run += base; total = all;
    }
    for (uint32_t i = lo; i < hi; i++) { uint32_t v = d[i]; d[i] = run; run += v; }
    team_sync<CL>();
    return total;
}

// One step of every scene (World::step, phys.rs:152-243): one team a scene, a block (CL = 1) or a thread-block cluster
// of CL blocks whose barrier is the cluster's; team-wide counters live in shared memory for a block, in global memory
// for a cluster.
template <int T, int CL>
__global__ void __launch_bounds__(T, CL == 1 && T <= 256 ? 2 : 1) k_box_step(BxArgs A, float dt, int par, const uint32_t *slist) {
    __shared__ uint32_t wsum[32];
    __shared__ __align__(8) uint32_t gsh[CL == 1 ? BX_G : 2];
    constexpr uint32_t TT = T * CL;
    const uint32_t rank = CL > 1 ? (uint32_t)cg::this_cluster().block_rank() : 0u;
    const uint32_t sc = slist[blockIdx.x / CL], t = rank * T + threadIdx.x;
    uint32_t *Gp = CL == 1 ? gsh : A.gs + (size_t)sc * BX_G;
    volatile uint32_t *GV = Gp;
    const uint32_t b0 = A.sc_b0[sc], n = A.sc_n[sc], s0 = b0 + sc, e0 = A.sc_e0[sc], t0 = A.sc_t0[sc];
    const uint32_t c0 = A.sc_c0[sc], m0 = A.sc_m0[sc], ccap = (BX_PPB + 1) * n, mcap = BX_CPB * n + 64u;
    uint32_t *st = A.stats + (size_t)sc * 8;
    const sf_box_params &P = A.P;
    for (uint32_t k = t; k < G_CCNT; k += TT) GV[k] = 0;
    unsigned long long *tns = A.tns + (size_t)sc * 5;
    unsigned long long tm0 = t == 0 ? gtime() : 0ull, tm1 = 0;
    team_sync<CL>();
    const float spec = P.speculative, inv_cell = __fdiv_rn(1.0f, P.cell);
    // ---- bodies: rotation, AABB with the speculative margin, solver slots (phys.rs:157-171)
    for (uint32_t i = t; i < n; i += TT) {
        const BxBody b = A.body[b0 + i];
        const DM3 r = qm3(b.q);
        P3 e = p3(fabsf(r.c[0].x) * b.h.x + fabsf(r.c[1].x) * b.h.y + fabsf(r.c[2].x) * b.h.z,
                  fabsf(r.c[0].y) * b.h.x + fabsf(r.c[1].y) * b.h.y + fabsf(r.c[2].y) * b.h.z,
                  fabsf(r.c[0].z) * b.h.x + fabsf(r.c[1].z) * b.h.y + fabsf(r.c[2].z) * b.h.z);
        const float m = b.awake ? (plen_e(b.v) + plen_e(b.w) * plen_e(b.h)) * dt + 0.5f * spec : 0.5f * spec;
        e = e + p3(m, m, m);
        const P3 lo = b.p - e, hi = b.p + e;
        A.rot[b0 + i] = r; A.amin[b0 + i] = lo; A.amax[b0 + i] = hi;
        const uint64_t ne = (uint64_t)(bcell(hi.x, inv_cell) - bcell(lo.x, inv_cell) + 1) *
                            (uint64_t)(bcell(hi.y, inv_cell) - bcell(lo.y, inv_cell) + 1) *
                            (uint64_t)(bcell(hi.z, inv_cell) - bcell(lo.z, inv_cell) + 1);
        if (ne > (uint64_t)BX_EPB * n) atomicOr(&Gp[G_ERR], (uint32_t)BXE_ENTRIES);
        A.ecnt[b0 + i] = ne > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)ne;
        atomicAdd((unsigned long long *)(Gp + G_NE), (unsigned long long)ne);
        A.wake[b0 + i] = 0;
        A.uf[b0 + i] = i;
        uint32_t slot = 0;
        if (b.awake) {
            slot = i + 1;
            const uint32_t s = s0 + slot;
            A.sv[s] = b.v; A.sw[s] = b.w; A.sdp[s] = p3(0.0f, 0.0f, 0.0f); A.sth[s] = p3(0.0f, 0.0f, 0.0f);
            A.sim[s] = b.inv_m; A.sii[s] = m_sandwich(r, b.inv_i); A.sq[s] = make_float4(b.q[0], b.q[1], b.q[2], b.q[3]);
            A.sp0[s] = b.p;
            atomicAdd(&Gp[G_TOT + 1], 1u);
        }
        A.sidx[b0 + i] = slot;
    }
    if (t == 0) {
        const P3 z = p3(0.0f, 0.0f, 0.0f);
        DM3 zm; zm.c[0] = zm.c[1] = zm.c[2] = z;
        A.sv[s0] = z; A.sw[s0] = z; A.sdp[s0] = z; A.sth[s0] = z; A.sim[s0] = 0.0f; A.sii[s0] = zm;
        A.sq[s0] = make_float4(0.0f, 0.0f, 0.0f, 1.0f); A.sp0[s0] = z;
    }
    team_sync<CL>();
    if (GV[G_ERR] || (*(volatile unsigned long long *)(Gp + G_NE)) > (unsigned long long)BX_EPB * n) {
        if (t == 0) { st[0] = GV[G_TOT + 1]; st[1] = st[2] = st[3] = st[4] = 0; st[5] = BXE_ENTRIES; A.mcount[par][sc] = 0; }
        return;
    }
    const uint32_t ne_tot = (uint32_t)(*(volatile unsigned long long *)(Gp + G_NE));
    uint32_t tbl = 1;
    while (tbl < ne_tot * 2u) tbl <<= 1;
    if (tbl > A.sc_tcap[sc]) {
        if (t == 0) { st[0] = GV[G_TOT + 1]; st[1] = st[2] = st[3] = st[4] = 0; st[5] = BXE_ENTRIES; A.mcount[par][sc] = 0; }
        return;
    }
    const uint32_t mask = tbl - 1;
    for (uint32_t k = t; k < tbl; k += TT) A.head[t0 + k] = BX_NONE;
    team_sync<CL>();
    // ---- grid: one entry per body and covered cell, chained per hash slot
    for (uint32_t i = t; i < n; i += TT) {
        const P3 lo = A.amin[b0 + i], hi = A.amax[b0 + i];
        const int32_t x0 = bcell(lo.x, inv_cell), y0 = bcell(lo.y, inv_cell), z0 = bcell(lo.z, inv_cell);
        const int32_t x1 = bcell(hi.x, inv_cell), y1 = bcell(hi.y, inv_cell), z1 = bcell(hi.z, inv_cell);
        for (int32_t x = x0; x <= x1; x++) for (int32_t y = y0; y <= y1; y++) for (int32_t z = z0; z <= z1; z++) {
            const uint32_t e = atomicAdd(&Gp[G_TOT + 2], 1u);
            A.ent_body[e0 + e] = i;
            A.ent_cell[3 * (size_t)(e0 + e)] = x; A.ent_cell[3 * (size_t)(e0 + e) + 1] = y; A.ent_cell[3 * (size_t)(e0 + e) + 2] = z;
            A.ent_next[e0 + e] = atomicExch(&A.head[t0 + (bhash(x, y, z) & mask)], e);
        }
    }
    team_sync<CL>();
    // ---- pairs (phys.rs:385-404): each body lists, sorted, the overlapping bodies above it that the grid reports in
    // the cell holding the larger of the two minimum corners; then its ground contact (phys.rs:362-365). Counted,
    // scanned, then written; a list of more than BX_SHORT pairs (a static slab under a pile) is sorted by the block.
    for (uint32_t a = t; a < n; a += TT) {
        const uint32_t k = walk_pairs(A, b0, e0, t0, mask, ne_tot, inv_cell, a, nullptr, nullptr);
        atomicAdd(&Gp[G_TOT + 3], k);
        A.cand_n[b0 + a] = k + ground_slots(A.body[b0 + a], A.amin[b0 + a]);
    }
    team_sync<CL>();
    const uint32_t nc = team_scan<T, CL>(A.cand_n + b0, n, wsum, Gp + G_CTA, t, rank);
    if (nc > ccap) {
        if (t == 0) { st[0] = GV[G_TOT + 1]; st[1] = GV[G_TOT + 3]; st[2] = st[3] = st[4] = 0; st[5] = BXE_PAIRS; A.mcount[par][sc] = 0; }
        return;
    }
    if (t == 0) GV[G_TOT + 5] = 0;
    team_sync<CL>();
    for (uint32_t a = t; a < n; a += TT) {
        const uint32_t off = A.cand_n[b0 + a];
        uint32_t *cb = A.cand_b + c0 + off;
        const uint32_t k = walk_pairs(A, b0, e0, t0, mask, ne_tot, inv_cell, a, A.cand_a + c0 + off, cb);
        if (k <= BX_SHORT) {
            for (uint32_t x = 1; x < k; x++) {
                const uint32_t v = cb[x];
                uint32_t y = x;
                while (y > 0 && cb[y - 1] > v) { cb[y] = cb[y - 1]; y--; }
                cb[y] = v;
            }
        } else {
            A.seglong[b0 + atomicAdd(&Gp[G_TOT + 5], 1u)] = a;
        }
        const uint32_t ng = ground_slots(A.body[b0 + a], A.amin[b0 + a]);
        for (uint32_t q = 0; q < ng; q++) { A.cand_a[c0 + off + k + q] = a; A.cand_b[c0 + off + k + q] = ng == 2 && q == 0 ? BX_GROUND2 : BX_NONE; }
    }
    team_sync<CL>();
    // long lists: the pair partners are distinct bodies, so a bitmap over the scene's bodies and a scan of its
    // population counts put them in order
    const uint32_t nlong = GV[G_TOT + 5], nwords = (n + 31) / 32;
    for (uint32_t q = 0; q < nlong; q++) {
        const uint32_t a = A.seglong[b0 + q];
        const uint32_t off = A.cand_n[b0 + a], next = a + 1 < n ? A.cand_n[b0 + a + 1] : nc;
        const uint32_t k = next - off - ground_slots(A.body[b0 + a], A.amin[b0 + a]);
        uint32_t *bits = A.mint + b0, *pos = A.ecnt + b0, *cb = A.cand_b + c0 + off;
        for (uint32_t x = t; x < nwords; x += TT) bits[x] = 0;
        team_sync<CL>();
        for (uint32_t x = t; x < k; x += TT) atomicOr(&bits[cb[x] >> 5], 1u << (cb[x] & 31));
        team_sync<CL>();
        for (uint32_t x = t; x < nwords; x += TT) pos[x] = __popc(bits[x]);
        team_sync<CL>();
        team_scan<T, CL>(pos, nwords, wsum, Gp + G_CTA, t, rank);
        for (uint32_t x = t; x < nwords; x += TT) {
            uint32_t wv = bits[x], r = pos[x];
            while (wv) { const uint32_t bit = __ffs(wv) - 1; cb[r++] = x * 32 + bit; wv &= wv - 1; }
        }
        team_sync<CL>();
    }
    if (t == 0) { tm1 = gtime(); tns[0] += tm1 - tm0; tm0 = tm1; }
    // ---- narrow phase, then the manifolds in key order (phys.rs:406-497)
    for (uint32_t c = t; c < nc; c += TT)
        A.hit[c0 + c] = collide_candidate(A, b0, A.cand_a[c0 + c], A.cand_b[c0 + c], A.geom + (size_t)(c0 + c) * 20) ? 1u : 0u;
    team_sync<CL>();
    const uint32_t M = team_scan<T, CL>(A.hit + c0, nc, wsum, Gp + G_CTA, t, rank);
    if (M > mcap) {
        if (t == 0) { st[0] = GV[G_TOT + 1]; st[1] = GV[G_TOT + 3]; st[2] = M; st[3] = st[4] = 0; st[5] = BXE_MANIFOLDS; A.mcount[par][sc] = 0; }
        return;
    }
    const uint32_t nold = A.mcount[par ^ 1][sc];
    for (uint32_t c = t; c < nc; c += TT) {
        const float *g = A.geom + (size_t)(c0 + c) * 20;
        const int cnt = __float_as_int(g[3]);
        if (!cnt) continue;
        const uint32_t m = A.hit[c0 + c];
        const uint32_t a = A.cand_a[c0 + c], b = A.cand_b[c0 + c];
        build_manifold(A, par, b0, s0, m0, nold, a, b, g, A.man[par][m0 + m]);
        A.mkey[par][m0 + m] = ((uint64_t)a << 32) | b;
        atomicAdd(&Gp[G_TOT + 4], (uint32_t)cnt);
    }
    // the wakes (phys.rs:410-417): the body joins the solver from the next step
    for (uint32_t i = t; i < n; i += TT) {
        if (!A.wake[b0 + i]) continue;
        BxBody &b = A.body[b0 + i];
        if (b.awake || b.inv_m == 0.0f) continue;
        b.awake = 1; b.sleep_t = 0.0f; b.sleep_p = b.p;
        b.sleep_q[0] = b.q[0]; b.sleep_q[1] = b.q[1]; b.sleep_q[2] = b.q[2]; b.sleep_q[3] = b.q[3];
    }
    team_sync<CL>();
    if (t == 0) { tm1 = gtime(); tns[1] += tm1 - tm0; tm0 = tm1; }
    // ---- colouring: greedy in descending priority, by Jones-Plassmann rounds. A manifold takes the smallest colour
    // its higher-priority neighbours (manifolds sharing a moving body) left free once all of them have one.
    const uint32_t ns = n + 1;
    for (uint32_t k = t; k < ns; k += TT) A.deg[s0 + k] = 0;
    for (uint32_t m = t; m < M; m += TT) A.colour[m0 + m] = BX_UNC;
    team_sync<CL>();
    for (uint32_t m = t; m < M; m += TT) {
        const DMan &mm = A.man[par][m0 + m];
        if (mm.sa) atomicAdd(&A.deg[s0 + mm.sa], 1u);
        if (mm.sb) atomicAdd(&A.deg[s0 + mm.sb], 1u);
    }
    team_sync<CL>();
    team_scan<T, CL>(A.deg + s0, ns, wsum, Gp + G_CTA, t, rank);
    for (uint32_t m = t; m < M; m += TT) {
        const DMan &mm = A.man[par][m0 + m];
        if (mm.sa) A.inc[2 * (size_t)m0 + atomicAdd(&A.deg[s0 + mm.sa], 1u)] = m;
        if (mm.sb) A.inc[2 * (size_t)m0 + atomicAdd(&A.deg[s0 + mm.sb], 1u)] = m;
    }
    team_sync<CL>();
    // incident list of slot k: [k ? deg[k - 1] : 0, deg[k]). Each manifold counts its higher-priority neighbours;
    // a coloured manifold counts its lower-priority neighbours down, and one whose count reaches 0 takes its colour.
    volatile uint32_t *col = A.colour + m0;
    uint64_t *prio = A.mrank + m0;
    uint32_t *wait = A.mwait + m0;
    for (uint32_t m = t; m < M; m += TT) { const DMan &mm = A.man[par][m0 + m]; prio[m] = man_rank(mm.a, mm.b, m); }
    team_sync<CL>();
    for (uint32_t m = t; m < M; m += TT) {
        const DMan &mm = A.man[par][m0 + m];
        const uint64_t rk = prio[m];
        uint32_t hi_n = 0;
        for (int side = 0; side < 2; side++) {
            const uint32_t sl = side ? mm.sb : mm.sa;
            if (!sl) continue;
            for (uint32_t q = A.deg[s0 + sl - 1], e = A.deg[s0 + sl]; q < e; q++) {
                const uint32_t o = A.inc[2 * (size_t)m0 + q];
                if (o != m && prio[o] > rk) hi_n++;
            }
        }
        wait[m] = hi_n;
    }
    team_sync<CL>();
    uint32_t rounds = 0;
    for (;;) {
        int pend = 0;
        for (uint32_t m = t; m < M; m += TT) {
            if (col[m] != BX_UNC) continue;
            if (((volatile uint32_t *)wait)[m] != 0) { pend = 1; continue; }
            if constexpr (CL == 1) __threadfence_block(); else __threadfence();
            const DMan &mm = A.man[par][m0 + m];
            const uint64_t rk = prio[m];
            uint64_t used0 = 0, used1 = 0;
            for (int side = 0; side < 2; side++) {
                const uint32_t sl = side ? mm.sb : mm.sa;
                if (!sl) continue;
                for (uint32_t q = A.deg[s0 + sl - 1], e = A.deg[s0 + sl]; q < e; q++) {
                    const uint32_t o = A.inc[2 * (size_t)m0 + q];
                    if (o == m || prio[o] < rk) continue;
                    const uint32_t oc = col[o];
                    if (oc < 64) used0 |= 1ull << oc; else if (oc < 128) used1 |= 1ull << (oc - 64);
                }
            }
            uint32_t c = ~used0 ? (uint32_t)__ffsll((long long)~used0) - 1 : (~used1 ? 64u + (uint32_t)__ffsll((long long)~used1) - 1 : (uint32_t)BX_MAXC);
            if (c >= (uint32_t)BX_MAXC) { atomicOr(&Gp[G_ERR], (uint32_t)BXE_COLOURS); c = BX_MAXC - 1; }
            col[m] = c;
            if constexpr (CL == 1) __threadfence_block(); else __threadfence();
            for (int side = 0; side < 2; side++) {
                const uint32_t sl = side ? mm.sb : mm.sa;
                if (!sl) continue;
                for (uint32_t q = A.deg[s0 + sl - 1], e = A.deg[s0 + sl]; q < e; q++) {
                    const uint32_t o = A.inc[2 * (size_t)m0 + q];
                    if (o != m && prio[o] < rk) atomicSub(&wait[o], 1u);
                }
            }
        }
        rounds++;
        if (!team_or<CL>(pend, Gp, rounds, t)) break;
        if (rounds > M + 1) { if (t == 0) atomicOr(&Gp[G_ERR], (uint32_t)BXE_GUARD); break; }
    }
    team_sync<CL>();
    if (GV[G_ERR]) {
        if (t == 0) { st[0] = GV[G_TOT + 1]; st[1] = GV[G_TOT + 3]; st[2] = M; st[3] = GV[G_TOT + 4]; st[4] = 0; st[5] = GV[G_ERR]; A.mcount[par][sc] = 0; }
        return;
    }
    for (uint32_t k = t; k < BX_MAXC; k += TT) GV[G_CCNT + k] = 0;
    team_sync<CL>();
    for (uint32_t m = t; m < M; m += TT) atomicAdd(&Gp[G_CCNT + col[m]], 1u);
    team_sync<CL>();
    if (t == 0) {
        uint32_t run = 0, nc2 = 0;
        for (int k = 0; k < BX_MAXC; k++) { GV[G_CBEG + k] = run; run += GV[G_CCNT + k]; if (GV[G_CCNT + k]) nc2 = k + 1; GV[G_CCNT + k] = GV[G_CBEG + k]; }
        GV[G_CBEG + BX_MAXC] = run;
        GV[G_NCOL] = nc2;
    }
    team_sync<CL>();
    for (uint32_t m = t; m < M; m += TT) A.corder[m0 + atomicAdd(&Gp[G_CCNT + col[m]], 1u)] = m;
    team_sync<CL>();
    const uint32_t ncol = GV[G_NCOL];
    if (t == 0) { tm1 = gtime(); tns[2] += tm1 - tm0; tm0 = tm1; }
    // ---- sub-steps (phys.rs:182-231): gravity and the spin clamp, warm start, biased solve, integrate, relax
    const uint32_t sub = P.substeps > 0 ? P.substeps : 1u;
    const float h = dt / (float)sub;
    const float inv_h = __fdiv_rn(1.0f, h);
    const float hz = P.contact_hertz > 0.0f ? P.contact_hertz : inv_h / 6.0f;
    const float PI_F = 3.14159265358979323846f;
    const float omega = 2.0f * PI_F * hz;
    const float a1 = 2.0f * P.damping_ratio + h * omega;
    const float a2 = h * omega * a1;
    const float a3 = __fdiv_rn(1.0f, 1.0f + a2);
    const float bias_rate = __fdiv_rn(omega, a1), mass_scale = a2 * a3, imp_scale = a3 * P.leak;
    const P3 g = p3(P.gravity[0], P.gravity[1], P.gravity[2]);
    const float wmax = 0.25f * PI_F * inv_h;
    DMan *man = A.man[par] + m0;
    const uint32_t *ord = A.corder + m0;
    for (uint32_t s = 0; s < sub; s++) {
        for (uint32_t i = t; i < n; i += TT) {
            const uint32_t sl = A.sidx[b0 + i];
            if (!sl) continue;
            A.sv[s0 + sl] = A.sv[s0 + sl] + g * h;
            const P3 w = A.sw[s0 + sl];
            const float wl = plen2(w);
            if (wl > wmax * wmax) A.sw[s0 + sl] = w * __fdiv_rn(wmax, sqrt_e(wl));
        }
        team_sync<CL>();
        for (uint32_t c = 0; c < ncol; c++) {
            for (uint32_t k = GV[G_CBEG + c] + t; k < GV[G_CBEG + c + 1]; k += TT) warm_manifold(A, s0, man[ord[k]]);
            team_sync<CL>();
        }
        for (uint32_t c = 0; c < ncol; c++) {
            for (uint32_t k = GV[G_CBEG + c] + t; k < GV[G_CBEG + c + 1]; k += TT)
                solve_manifold(A, s0, man[ord[k]], true, inv_h, bias_rate, mass_scale, imp_scale);
            team_sync<CL>();
        }
        for (uint32_t i = t; i < n; i += TT) {
            const uint32_t sl = A.sidx[b0 + i];
            if (!sl) continue;
            const P3 v = A.sv[s0 + sl], w = A.sw[s0 + sl];
            A.sdp[s0 + sl] = A.sdp[s0 + sl] + v * h; A.sth[s0 + sl] = A.sth[s0 + sl] + w * h;
            A.sq[s0 + sl] = qintegrate(A.sq[s0 + sl], w, h);
        }
        team_sync<CL>();
        for (uint32_t c = 0; c < ncol; c++) {
            for (uint32_t k = GV[G_CBEG + c] + t; k < GV[G_CBEG + c + 1]; k += TT)
                solve_manifold(A, s0, man[ord[k]], false, inv_h, bias_rate, mass_scale, imp_scale);
            team_sync<CL>();
        }
    }
    if (t == 0) { tm1 = gtime(); tns[3] += tm1 - tm0; tm0 = tm1; }
    // ---- write back (phys.rs:233-236), then islands and sleep (phys.rs:326-354)
    for (uint32_t i = t; i < n; i += TT) {
        const uint32_t sl = A.sidx[b0 + i];
        if (!sl) continue;
        BxBody &b = A.body[b0 + i];
        b.v = A.sv[s0 + sl]; b.w = A.sw[s0 + sl]; b.p = A.sp0[s0 + sl] + A.sdp[s0 + sl];
        const float4 q = A.sq[s0 + sl];
        b.q[0] = q.x; b.q[1] = q.y; b.q[2] = q.z; b.q[3] = q.w;
    }
    uint32_t *uf = A.uf + b0;
    for (uint32_t i = t; i < n; i += TT) A.mint[b0 + i] = 0x7F7FFFFFu;
    for (uint32_t m = t; m < M; m += TT) {
        const DMan &mm = man[m];
        if (!mm.sa || !mm.sb) continue;
        uint32_t x = mm.a, y = mm.b;
        for (int gd = 0; gd < 1 << 20; gd++) {
            x = uf_root(uf, x); y = uf_root(uf, y);
            if (x == y) break;
            if (x < y) { uint32_t tt = x; x = y; y = tt; }
            if (atomicCAS(&uf[x], x, y) == x) break;
        }
    }
    team_sync<CL>();
    const float l2 = P.sleep_lin * P.sleep_lin, ang2 = P.sleep_ang * P.sleep_ang;
    for (uint32_t i = t; i < n; i += TT) {
        BxBody &b = A.body[b0 + i];
        if (!b.awake) continue;
        const float4 dq = qmul(make_float4(b.q[0], b.q[1], b.q[2], b.q[3]), make_float4(-b.sleep_q[0], -b.sleep_q[1], -b.sleep_q[2], b.sleep_q[3]));
        const float ang = 2.0f * sqrt_e(dq.x * dq.x + dq.y * dq.y + dq.z * dq.z);
        const bool nearb = plen2(b.p - b.sleep_p) < P.sleep_dist * P.sleep_dist && ang < P.sleep_rot;
        if (nearb && plen2(b.v) < 100.0f * l2 && plen2(b.w) < 100.0f * ang2) b.sleep_t += dt;
        else {
            b.sleep_t = 0.0f; b.sleep_p = b.p;
            b.sleep_q[0] = b.q[0]; b.sleep_q[1] = b.q[1]; b.sleep_q[2] = b.q[2]; b.sleep_q[3] = b.q[3];
        }
        if (P.allow_sleep) atomicMin(&A.mint[b0 + uf_root(uf, i)], __float_as_uint(b.sleep_t));
    }
    team_sync<CL>();
    if (P.allow_sleep) {
        for (uint32_t i = t; i < n; i += TT) {
            BxBody &b = A.body[b0 + i];
            if (!b.awake) continue;
            if (__uint_as_float(A.mint[b0 + uf_root(uf, i)]) >= P.sleep_time) {
                b.awake = 0; b.v = p3(0.0f, 0.0f, 0.0f); b.w = p3(0.0f, 0.0f, 0.0f);
            }
        }
    }
    if (t == 0) {
        st[0] = GV[G_TOT + 1]; st[1] = GV[G_TOT + 3]; st[2] = M; st[3] = GV[G_TOT + 4]; st[4] = ncol; st[5] = 0; st[6] = rounds; st[7] = 0;
        tns[4] += gtime() - tm0;
        A.mcount[par][sc] = M;
    }
}

__global__ void k_box_hull_ids(BxBody *body, const uint32_t *ids, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) body[i].hull = ids[i];
}

}  // namespace
}  // namespace sf

using namespace sf;

struct sf_box_world {
    sf_box_params P{};
    uint32_t n_scenes = 0, n_bodies = 0, max_n = 0;
    std::vector<uint32_t> b0, nn, c0, m0;
    DBuf<BxBody> body;
    DBuf<float4> hulls;
    uint32_t n_hulls = 0;
    DBuf<DM3> rot, sii;
    DBuf<P3> amin, amax, sv, sw, sdp, sth, sp0;
    DBuf<float> sim, geom;
    DBuf<float4> sq;
    DBuf<uint32_t> ecnt, sidx, cand_n, seglong, uf, mint, ent_body, ent_next, head, cand_a, cand_b, hit, deg, inc, colour,
        corder, mwait, stats, mcount0, mcount1, sc_b0, sc_n, sc_e0, sc_t0, sc_tcap, sc_c0, sc_m0;
    DBuf<int32_t> ent_cell;
    DBuf<uint8_t> wake;
    DBuf<DMan> man0, man1;
    DBuf<uint64_t> mkey0, mkey1, mrank;
    DBuf<unsigned long long> tns;
    DBuf<uint32_t> gs, slist;
    uint32_t n_small = 0, n_big = 0;
    bool cluster_ok = false;
    int par = 0;
    uint64_t steps = 0;
    float last_ms = 0.0f;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~sf_box_world() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

static uint32_t pow2_at_least(uint64_t x) { uint64_t t = 1; while (t < x) t <<= 1; return (uint32_t)t; }

static sf_status box_upload(sf_box_world *w, const float *boxes) {
    std::vector<BxBody> hb(w->n_bodies);
    for (uint32_t i = 0; i < w->n_bodies; i++) {   // World::add_box (engine/src/phys.rs:137-146)
        const float *r = boxes + (size_t)i * 11;
        BxBody b{};
        b.p = {r[0], r[1], r[2]};
        for (int k = 0; k < 4; k++) { b.q[k] = r[3 + k]; b.sleep_q[k] = r[3 + k]; }
        b.h = {r[7], r[8], r[9]};
        const float m = r[10] * 8.0f * b.h.x * b.h.y * b.h.z;
        if (m > 0.0f) {
            const float x2 = 4.0f * b.h.x * b.h.x, y2 = 4.0f * b.h.y * b.h.y, z2 = 4.0f * b.h.z * b.h.z;
            b.inv_m = 1.0f / m;
            b.inv_i = {12.0f / (m * (y2 + z2)), 12.0f / (m * (x2 + z2)), 12.0f / (m * (x2 + y2))};
        }
        b.awake = m > 0.0f ? 1u : 0u;
        b.sleep_p = b.p;
        hb[i] = b;
    }
    SF_CUDA(cudaMemcpyAsync(w->body.p, hb.data(), hb.size() * sizeof(BxBody), cudaMemcpyHostToDevice, w->stream));
    SF_CUDA(cudaMemsetAsync(w->mcount0.p, 0, w->n_scenes * 4, w->stream));
    SF_CUDA(cudaMemsetAsync(w->mcount1.p, 0, w->n_scenes * 4, w->stream));
    SF_CUDA(cudaMemsetAsync(w->stats.p, 0, (size_t)w->n_scenes * 32, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    w->par = 0;
    return SF_OK;
}

}  // namespace

extern "C" sf_status sf_box_world_create(const float *boxes, const uint32_t *scene_first, uint32_t n_scenes,
                                         const sf_box_params *params, sf_box_world **out) {
    if (!boxes || !scene_first || !params || !out || n_scenes == 0) { set_error("null argument"); return SF_ERR_ARG; }
    *out = nullptr;
    for (uint32_t s = 0; s < n_scenes; s++)
        if (scene_first[s + 1] < scene_first[s]) { set_error("scene_first must not decrease"); return SF_ERR_ARG; }
    if (scene_first[0] != 0) { set_error("scene_first[0] must be 0"); return SF_ERR_ARG; }
    if (params->cell <= 0.0f) { set_error("cell must be positive"); return SF_ERR_ARG; }
    sf_box_world *w = new sf_box_world();
    w->P = *params;
    w->n_scenes = n_scenes;
    w->n_bodies = scene_first[n_scenes];
    std::vector<uint32_t> e0(n_scenes), t0(n_scenes), tcap(n_scenes);
    uint64_t et = 0, tt = 0, ct = 0, mt = 0;
    w->b0.resize(n_scenes); w->nn.resize(n_scenes); w->c0.resize(n_scenes); w->m0.resize(n_scenes);
    for (uint32_t s = 0; s < n_scenes; s++) {
        const uint32_t n = scene_first[s + 1] - scene_first[s];
        w->b0[s] = scene_first[s]; w->nn[s] = n; w->max_n = std::max(w->max_n, n);
        e0[s] = (uint32_t)et; et += (uint64_t)BX_EPB * n;
        tcap[s] = pow2_at_least(2ull * BX_EPB * n); t0[s] = (uint32_t)tt; tt += tcap[s];
        w->c0[s] = (uint32_t)ct; ct += (uint64_t)(BX_PPB + 1) * n;
        w->m0[s] = (uint32_t)mt; mt += (uint64_t)BX_CPB * n + 64u;
    }
    if (et > 0xFFFFFFFFull || tt > 0xFFFFFFFFull || ct > 0xFFFFFFFFull || 2 * mt > 0xFFFFFFFFull) { delete w; set_error("box world too large"); return SF_ERR_CAPACITY; }
    const size_t nb = w->n_bodies, ns = nb + n_scenes;
    bool bad = false;
    auto A = [&](cudaError_t e) { if (e != cudaSuccess) bad = true; };
    A(w->body.alloc(nb)); A(w->rot.alloc(nb)); A(w->amin.alloc(nb)); A(w->amax.alloc(nb)); A(w->ecnt.alloc(nb));
    A(w->sidx.alloc(nb)); A(w->cand_n.alloc(nb)); A(w->seglong.alloc(nb)); A(w->uf.alloc(nb)); A(w->mint.alloc(nb));
    A(w->wake.alloc(nb));
    A(w->sii.alloc(ns)); A(w->sv.alloc(ns)); A(w->sw.alloc(ns)); A(w->sdp.alloc(ns)); A(w->sth.alloc(ns)); A(w->sp0.alloc(ns));
    A(w->sim.alloc(ns)); A(w->sq.alloc(ns)); A(w->deg.alloc(ns));
    A(w->ent_body.alloc(et)); A(w->ent_next.alloc(et)); A(w->ent_cell.alloc(3 * et)); A(w->head.alloc(tt));
    A(w->cand_a.alloc(ct)); A(w->cand_b.alloc(ct)); A(w->hit.alloc(ct)); A(w->geom.alloc(20 * ct));
    A(w->colour.alloc(mt)); A(w->corder.alloc(mt)); A(w->mwait.alloc(mt)); A(w->mrank.alloc(mt)); A(w->inc.alloc(2 * mt));
    A(w->man0.alloc(mt)); A(w->man1.alloc(mt)); A(w->mkey0.alloc(mt)); A(w->mkey1.alloc(mt));
    A(w->stats.alloc((size_t)n_scenes * 8)); A(w->tns.alloc((size_t)n_scenes * 5));
    A(w->gs.alloc((size_t)n_scenes * BX_G)); A(w->slist.alloc(n_scenes)); A(w->mcount0.alloc(n_scenes)); A(w->mcount1.alloc(n_scenes));
    A(w->sc_b0.alloc(n_scenes)); A(w->sc_n.alloc(n_scenes)); A(w->sc_e0.alloc(n_scenes)); A(w->sc_t0.alloc(n_scenes));
    A(w->sc_tcap.alloc(n_scenes)); A(w->sc_c0.alloc(n_scenes)); A(w->sc_m0.alloc(n_scenes));
    if (bad) { delete w; set_error("device allocation failed"); return SF_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&w->ev0) != cudaSuccess || cudaEventCreate(&w->ev1) != cudaSuccess) {
        delete w; set_error("stream or event creation failed"); return SF_ERR_CUDA;
    }
    cudaMemcpy(w->sc_b0.p, w->b0.data(), n_scenes * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(w->sc_n.p, w->nn.data(), n_scenes * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(w->sc_e0.p, e0.data(), n_scenes * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(w->sc_t0.p, t0.data(), n_scenes * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(w->sc_tcap.p, tcap.data(), n_scenes * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(w->sc_c0.p, w->c0.data(), n_scenes * 4, cudaMemcpyHostToDevice);
    if (cudaMemcpy(w->sc_m0.p, w->m0.data(), n_scenes * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        delete w; set_error("upload failed"); return SF_ERR_CUDA;
    }
    {
        std::vector<uint32_t> big, small;
        for (uint32_t s = 0; s < n_scenes; s++) (w->nn[s] > BX_BIG ? big : small).push_back(s);
        w->n_big = (uint32_t)big.size(); w->n_small = (uint32_t)small.size();
        big.insert(big.end(), small.begin(), small.end());
        cudaMemcpy(w->slist.p, big.data(), n_scenes * 4, cudaMemcpyHostToDevice);
        if (w->n_big) {
            cudaFuncSetAttribute(k_box_step<BX_CL_THREADS, BX_CL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            cudaLaunchConfig_t c = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = BX_CL; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
            c.gridDim = dim3(BX_CL);
            c.blockDim = dim3(BX_CL_THREADS);
            c.attrs = at;
            c.numAttrs = 1;
            int ncl = 0;
            if (cudaOccupancyMaxActiveClusters(&ncl, k_box_step<BX_CL_THREADS, BX_CL>, &c) != cudaSuccess) { ncl = 0; cudaGetLastError(); }
            w->cluster_ok = ncl > 0;
        }
    }
    sf_status r = box_upload(w, boxes);
    if (r != SF_OK) { delete w; return r; }
    *out = w;
    return SF_OK;
}

extern "C" void sf_box_world_destroy(sf_box_world *w) { delete w; }

extern "C" sf_status sf_box_world_step(sf_box_world *w, float dt, uint32_t nsteps) {
    if (!w) { set_error("null world"); return SF_ERR_ARG; }
    if (!(dt > 0.0f)) { set_error("dt must be positive"); return SF_ERR_ARG; }
    BxArgs a;
    a.body = w->body.p; a.hulls = w->hulls.p; a.rot = w->rot.p; a.amin = w->amin.p; a.amax = w->amax.p;
    a.ecnt = w->ecnt.p; a.sidx = w->sidx.p; a.cand_n = w->cand_n.p; a.seglong = w->seglong.p; a.uf = w->uf.p; a.mint = w->mint.p;
    a.wake = w->wake.p; a.ent_body = w->ent_body.p; a.ent_next = w->ent_next.p; a.head = w->head.p; a.ent_cell = w->ent_cell.p;
    a.cand_a = w->cand_a.p; a.cand_b = w->cand_b.p; a.hit = w->hit.p; a.geom = w->geom.p;
    a.man[0] = w->man0.p; a.man[1] = w->man1.p; a.mkey[0] = w->mkey0.p; a.mkey[1] = w->mkey1.p;
    a.mcount[0] = w->mcount0.p; a.mcount[1] = w->mcount1.p;
    a.deg = w->deg.p; a.inc = w->inc.p; a.colour = w->colour.p; a.corder = w->corder.p; a.mwait = w->mwait.p; a.mrank = w->mrank.p;
    a.sv = w->sv.p; a.sw = w->sw.p; a.sdp = w->sdp.p; a.sth = w->sth.p; a.sp0 = w->sp0.p; a.sim = w->sim.p; a.sii = w->sii.p;
    a.sq = w->sq.p;
    a.sc_b0 = w->sc_b0.p; a.sc_n = w->sc_n.p; a.sc_e0 = w->sc_e0.p; a.sc_t0 = w->sc_t0.p; a.sc_tcap = w->sc_tcap.p;
    a.sc_c0 = w->sc_c0.p; a.sc_m0 = w->sc_m0.p; a.stats = w->stats.p; a.tns = w->tns.p; a.gs = w->gs.p; a.P = w->P;
    SF_CUDA(cudaMemsetAsync(w->tns.p, 0, (size_t)w->n_scenes * 5 * sizeof(unsigned long long), w->stream));
    SF_CUDA(cudaEventRecord(w->ev0, w->stream));
    for (uint32_t k = 0; k < nsteps; k++) {
        // scenes of more than BX_BIG boxes: one 16-block cluster each; the rest: one block each
        if (w->n_big && w->cluster_ok) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = BX_CL; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(w->n_big * BX_CL);
            cfg.blockDim = dim3(BX_CL_THREADS);
            cfg.stream = w->stream;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            SF_CUDA(cudaLaunchKernelEx(&cfg, k_box_step<BX_CL_THREADS, BX_CL>, a, dt, w->par, (const uint32_t *)w->slist.p));
        } else if (w->n_big) {
            k_box_step<1024, 1><<<w->n_big, 1024, 0, w->stream>>>(a, dt, w->par, w->slist.p);
        }
        if (w->n_small) k_box_step<256, 1><<<w->n_small, 256, 0, w->stream>>>(a, dt, w->par, w->slist.p + w->n_big);
        w->par ^= 1;
    }
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaEventRecord(w->ev1, w->stream));
    SF_CUDA(cudaEventSynchronize(w->ev1));
    cudaEventElapsedTime(&w->last_ms, w->ev0, w->ev1);
    w->steps += nsteps;
    std::vector<uint32_t> st((size_t)w->n_scenes * 8);
    SF_CUDA(cudaMemcpy(st.data(), w->stats.p, st.size() * 4, cudaMemcpyDeviceToHost));
    for (uint32_t s = 0; s < w->n_scenes; s++)
        if (st[(size_t)s * 8 + 5]) {
            set_error("box world scene %u: capacity exceeded (flags 0x%x)", s, st[(size_t)s * 8 + 5]);
            return SF_ERR_CAPACITY;
        }
    return SF_OK;
}

// 22 floats a body: p3 q4 v3 w3 sleep_t sleep_p3 sleep_q4 awake
extern "C" sf_status sf_box_world_read(sf_box_world *w, float *out22) {
    if (!w || !out22) { set_error("null argument"); return SF_ERR_ARG; }
    std::vector<BxBody> hb(w->n_bodies);
    SF_CUDA(cudaMemcpyAsync(hb.data(), w->body.p, hb.size() * sizeof(BxBody), cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    for (uint32_t i = 0; i < w->n_bodies; i++) {
        const BxBody &b = hb[i];
        const float r[22] = {b.p.x, b.p.y, b.p.z, b.q[0], b.q[1], b.q[2], b.q[3], b.v.x, b.v.y, b.v.z, b.w.x, b.w.y, b.w.z,
                             b.sleep_t, b.sleep_p.x, b.sleep_p.y, b.sleep_p.z, b.sleep_q[0], b.sleep_q[1], b.sleep_q[2],
                             b.sleep_q[3], b.awake ? 1.0f : 0.0f};
        std::memcpy(out22 + (size_t)i * 22, r, sizeof(r));
    }
    return SF_OK;
}

extern "C" sf_status sf_box_world_stats(sf_box_world *w, uint32_t scene, sf_box_stats *out) {
    if (!w || !out || scene >= w->n_scenes) { set_error("bad argument"); return SF_ERR_ARG; }
    uint32_t st[8];
    SF_CUDA(cudaMemcpy(st, w->stats.p + (size_t)scene * 8, 32, cudaMemcpyDeviceToHost));
    out->awake = st[0]; out->pairs = st[1]; out->manifolds = st[2]; out->points = st[3]; out->colours = st[4];
    out->status = st[5]; out->rounds = st[6]; out->ms = w->last_ms; out->steps = w->steps;
    unsigned long long tn[5];
    SF_CUDA(cudaMemcpy(tn, w->tns.p + (size_t)scene * 5, sizeof(tn), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 5; k++) out->phase_ms[k] = (float)(tn[k] * 1e-6);
    return SF_OK;
}

// the last step's manifolds of one scene in key order, 16 words each: a, b, count, stick, normal 3, jn 4, jt1, jt2,
// jtw (f32 bits), colour
extern "C" sf_status sf_box_world_manifolds(sf_box_world *w, uint32_t scene, uint32_t *out16, uint32_t cap, uint32_t *count) {
    if (!w || !count || scene >= w->n_scenes) { set_error("bad argument"); return SF_ERR_ARG; }
    uint32_t m = 0;
    SF_CUDA(cudaMemcpy(&m, (w->par ? w->mcount0.p : w->mcount1.p) + scene, 4, cudaMemcpyDeviceToHost));
    *count = m;
    if (!out16 || cap == 0 || m == 0) return SF_OK;
    const uint32_t k = std::min(m, cap);
    std::vector<DMan> hm(k);
    std::vector<uint32_t> col(k);
    const DMan *src = (w->par ? w->man0.p : w->man1.p) + w->m0[scene];
    SF_CUDA(cudaMemcpy(hm.data(), src, k * sizeof(DMan), cudaMemcpyDeviceToHost));
    SF_CUDA(cudaMemcpy(col.data(), w->colour.p + w->m0[scene], k * 4, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < k; i++) {
        const DMan &x = hm[i];
        uint32_t *o = out16 + (size_t)i * 16;
        const float f[10] = {x.n.x, x.n.y, x.n.z, x.cp[0].jn, x.cp[1].jn, x.cp[2].jn, x.cp[3].jn, x.jt1, x.jt2, x.jtw};
        o[0] = x.a; o[1] = x.b; o[2] = x.cnt; o[3] = x.stick;
        std::memcpy(o + 4, f, sizeof(f));
        o[14] = col[i]; o[15] = 0;
    }
    return SF_OK;
}

// hull_data: n_hulls cells of 80 float4 (shatterforge_b200/hulls.py packed(); cell 0 the whole cube); hull_ids: a cell
// per box (0 = a plain box). Boxes keep their own mass and inertia (the record's density over the whole box).
extern "C" sf_status sf_box_world_set_hulls(sf_box_world *w, const float *hull_data, uint32_t n_hulls, const uint32_t *hull_ids) {
    if (!w || !hull_data || !hull_ids || n_hulls == 0) { set_error("null argument"); return SF_ERR_ARG; }
    for (uint32_t i = 0; i < w->n_bodies; i++)
        if (hull_ids[i] >= n_hulls) { set_error("box %u: hull %u of %u", i, hull_ids[i], n_hulls); return SF_ERR_ARG; }
    if (w->hulls.alloc((size_t)n_hulls * 80) != cudaSuccess) { set_error("device allocation failed"); return SF_ERR_CUDA; }
    w->n_hulls = n_hulls;
    DBuf<uint32_t> ids;
    if (ids.alloc(w->n_bodies) != cudaSuccess) { set_error("device allocation failed"); return SF_ERR_CUDA; }
    SF_CUDA(cudaMemcpyAsync(w->hulls.p, hull_data, (size_t)n_hulls * 80 * sizeof(float4), cudaMemcpyHostToDevice, w->stream));
    SF_CUDA(cudaMemcpyAsync(ids.p, hull_ids, (size_t)w->n_bodies * 4, cudaMemcpyHostToDevice, w->stream));
    if (w->n_bodies) k_box_hull_ids<<<grid_for(w->n_bodies, 256), 256, 0, w->stream>>>(w->body.p, ids.p, w->n_bodies);
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}

// ============================================================================================================
// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of Shatterforge's per-step physics hot path, used by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py as the checker. Nothing in the product library links, loads or calls this file.
//
// What it restates (file:line inside the reference project):
//   math helpers ........................ src/lib.rs:25-108   (minf/maxf are `if a < b {a} else {b}`, not fminf)
//   constants ........................... src/lib.rs:110-215
//   sparse chunk grid gget/gset ......... src/lib.rs:300-321
//   linked() ............................ src/lib.rs:378-383
//   bond_cap / finalize_brick ........... src/lib.rs:646-696
//   setup_body .......................... src/lib.rs:844-891
//   clamp_vel ........................... src/lib.rs:917-924
//   sor_brick / sor_struct .............. src/lib.rs:1005-1040
//   cond / axis_up / cond_w ............. src/lib.rs:1142-1151
//   stress_brick ........................ src/lib.rs:1153-1227  (decisions only; particles/shards/meshing left out)
//   update_cache / hkey / build_hash .... src/lib.rs:1367-1395
//   push_contact / gen_contacts ......... src/lib.rs:1396-1471
//   vel_at / eff_mass / apply_imp ....... src/lib.rs:1472-1492
//   prep_contacts / solve ............... src/lib.rs:1551-1601
//   integrate / pinch_check / substep ... src/lib.rs:1703-1783
//   step (rigid part) ................... src/lib.rs:3640-3651
//   union-find islands + island sleep ... engine/src/phys.rs:326-354, gpu/gpu_world.js:1634-1668
//   box SAT collide_boxes / reduce4 ..... engine/src/phys.rs:507-628
//   box world World::step ............. engine/src/phys.rs:152-354 (+ the WebGPU world's hull shapes, gpu/gpu_world.js:786-833)
//
// Floating point: every f32 expression keeps the reference's evaluation order, and the file is compiled with
// -ffp-contract=off (wasm32 f32 has no fused multiply-add), so the restatement is op-for-op IEEE-equivalent.
//
// Parity status: the reference is a wasm32-only Rust crate with no buildable toolchain here, and its own tests
// hold no numeric golden vectors for this path. Numeric parity of this oracle is therefore UNPINNED; it is pinned
// only by behavioural known answers (intact frames hold under self-weight, src/lib.rs stab test; sor fixed point
// against an FP64 solve; hull library volumes) that tests/test_oracle.py checks.
// The box world's list order is pinned by the reference's own published figures (the 20-box stack's 6.93 mm and
// 1.7 mm/s, the 2,000-box pile's 0.117-4.828 m range), which it reproduces to their printed digits
// (tests/test_oracle_boxes.py).
//
// Extensions beyond the reference, each behind a switch so the reference behaviour stays the default:
//   * capacities are dynamic (the reference drops contacts past MAXC = 30000; the count it would drop is reported);
//   * ORDER_COLOR solves contacts grouped by body-pair manifold in a greedy priority colouring order (the GPU's
//     order), ORDER_LIST keeps the reference's list order;
//   * SLEEP_ISLAND composes the per-body rest timer of src/lib.rs with the island rule of gpu/gpu_world.js:1660-1668;
//   * pinch_kill = 0 clamps small pinched bodies instead of removing them.
// ============================================================================================================
#include <cstdint>
#include <cstring>
#include <cmath>
#include <unordered_map>
#include <vector>
#include <algorithm>
#include <numeric>

namespace {

// ---------------------------------------------------------------- math (src/lib.rs:25-108)
struct V { float x[3]; float& operator[](int i) { return x[i]; } float operator[](int i) const { return x[i]; } };
typedef float M[9];
static inline float minf(float a, float b) { return a < b ? a : b; }
static inline float maxf(float a, float b) { return a > b ? a : b; }
static inline float clampf(float x, float a, float b) { return minf(maxf(x, a), b); }
static inline float fabs_(float x) { uint32_t u; std::memcpy(&u, &x, 4); u &= 0x7fffffffu; float r; std::memcpy(&r, &u, 4); return r; }
static inline V vv(float a, float b, float c) { V r; r.x[0] = a; r.x[1] = b; r.x[2] = c; return r; }
static inline V add(V a, V b) { return vv(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
static inline V sub(V a, V b) { return vv(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
static inline V mul(V a, float s) { return vv(a[0] * s, a[1] * s, a[2] * s); }
static inline V madd(V a, V b, float s) { return vv(a[0] + b[0] * s, a[1] + b[1] * s, a[2] + b[2] * s); }
static inline float dot(V a, V b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline V cross(V a, V b) { return vv(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]); }
static inline float len(V a) { return std::sqrt(dot(a, a)); }
static inline V mv(const float* m, V v) {
    return vv(m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2], m[6] * v[0] + m[7] * v[1] + m[8] * v[2]);
}
static inline void mmul(const float* a, const float* b, float* r) {
    float t[9];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) t[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
    std::memcpy(r, t, sizeof t);
}
static inline void mt(const float* a, float* r) { float t[9] = {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]}; std::memcpy(r, t, sizeof t); }
static void minv(const float* a, float* r) {
    float c0 = a[4] * a[8] - a[5] * a[7];
    float c1 = a[5] * a[6] - a[3] * a[8];
    float c2 = a[3] * a[7] - a[4] * a[6];
    float det = a[0] * c0 + a[1] * c1 + a[2] * c2;
    if (fabs_(det) < 1e-12f) { for (int k = 0; k < 9; k++) r[k] = 0.0f; return; }
    float id = 1.0f / det;
    float t[9] = {c0 * id, (a[2] * a[7] - a[1] * a[8]) * id, (a[1] * a[5] - a[2] * a[4]) * id,
                  c1 * id, (a[0] * a[8] - a[2] * a[6]) * id, (a[2] * a[3] - a[0] * a[5]) * id,
                  c2 * id, (a[1] * a[6] - a[0] * a[7]) * id, (a[0] * a[4] - a[1] * a[3]) * id};
    std::memcpy(r, t, sizeof t);
}
static void q_to_m(const float* q, float* r) {
    float x = q[0], y = q[1], z = q[2], w = q[3];
    float t[9] = {1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y - z * w), 2.0f * (x * z + y * w),
                  2.0f * (x * y + z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z - x * w),
                  2.0f * (x * z - y * w), 2.0f * (y * z + x * w), 1.0f - 2.0f * (x * x + y * y)};
    std::memcpy(r, t, sizeof t);
}
static void q_int(float* q, V w, float dt) {
    V qv = vv(q[0], q[1], q[2]);
    V d = add(mul(w, q[3]), cross(w, qv));
    float dw = -dot(w, qv);
    float r[4] = {q[0] + 0.5f * dt * d[0], q[1] + 0.5f * dt * d[1], q[2] + 0.5f * dt * d[2], q[3] + 0.5f * dt * dw};
    float l = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    if (l > 1e-9f) { for (int k = 0; k < 4; k++) r[k] /= l; } else { r[0] = 0; r[1] = 0; r[2] = 0; r[3] = 1; }
    for (int k = 0; k < 4; k++) q[k] = r[k];
}

// ---------------------------------------------------------------- constants (src/lib.rs:110-215)
const float S = 0.5f, H = 0.25f, RB = 0.27f, GR = 9.81f, MU = 0.65f, GROUNDK = 4.0f;
const int NX = 640, NY = 136, NZ = 640, CXN = NX / 8, CYN = NY / 8, CZN = NZ / 8, NCT = CXN * CYN * CZN;
const uint32_t HSIZE = 32768;
const uint32_t NONE = 0xFFFFFFFFu;
const uint32_t STATIC = 0xFFFFFFFFu;
const uint32_t MAXC_REF = 30000;
const uint8_t STEEL = 3, GLASS = 4, SLUG = 6;
const float MASS[9] = {0.0f, 300.0f, 230.0f, 250.0f, 60.0f, 70.0f, 2000.0f, 8.0f, 44.0f};
const float EB[9] = {0.0f, 15000.0f, 12000.0f, 1.5e6f, 300.0f, 6000.0f, 1e12f, 1e12f, 1e12f};   // src/lib.rs:178
const float PULV[9] = {0.0f, 0.7f, 0.55f, 0.0f, 1.0f, 0.5f, 0.0f, 0.0f, 0.0f};                 // src/lib.rs:180
const float CAPV[9] = {0.0f, 140000.0f, 50000.0f, 150000.0f, 1500.0f, 9000.0f, 1e12f, 1e12f, 1e12f};
const float CAPH[9] = {0.0f, 12000.0f, 12000.0f, 90000.0f, 400.0f, 5000.0f, 1e12f, 1e12f, 1e12f};
const float TENS[9] = {0.0f, 0.35f, 0.1f, 0.9f, 0.5f, 0.7f, 1.0f, 1.0f, 1.0f};
const float STIFF[9] = {0.0f, 1.0f, 0.8f, 2.0f, 0.02f, 0.4f, 1.0f, 1.0f, 1.0f};
const float DUCT[9] = {0.0f, 6.0f, 12.0f, 3.0f, 40.0f, 8.0f, 1.0f, 1.0f, 1.0f};
const int DIRS[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

static inline bool inb(int x, int y, int z) { return x >= 0 && y >= 0 && z >= 0 && x < NX && y < NY && z < NZ; }
static inline V lat_pos(int x, int y, int z) { return vv((float)(x - NX / 2) * S + H, (float)y * S + H, (float)(z - NZ / 2) * S + H); }
static inline uint32_t hkey(int x, int y, int z) {
    return ((uint32_t)(x * 73856093) ^ (uint32_t)(y * 19349663) ^ (uint32_t)(z * 83492791)) & (HSIZE - 1);
}
static inline int wrap_mul(int a, int b) { return (int)((uint32_t)a * (uint32_t)b); }
static inline uint32_t hkey_w(int x, int y, int z) {
    return ((uint32_t)wrap_mul(x, 73856093) ^ (uint32_t)wrap_mul(y, 19349663) ^ (uint32_t)wrap_mul(z, 83492791)) & (HSIZE - 1);
}

struct Contact {
    uint32_t a, b, bo, ba, bb;
    V n, p, ra, rb, t1, t2;
    float depth, mn, mt1, mt2, jn, jt1, jt2, bias, vn0;
    uint32_t off;   // 1: left out by the contact reduction (not coloured, not solved, no impulse)
};

enum { ORDER_LIST = 0, ORDER_COLOR = 1 };
enum { SLEEP_BODY = 0, SLEEP_ISLAND = 1 };

struct StepParams { uint32_t iterations, substeps, order, sleep_mode, pinch_kill, damage, reduce, warm; };

// manifold priority for the colouring: a fixed mix of the body pair (b' = 0 for the static side, else b + 1)
static inline uint32_t pair_priority(uint32_t a, uint32_t bp) {
    uint32_t h = a * 0x9E3779B1u + bp * 0x85EBCA6Bu;
    h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
    return h;
}

struct World {
    // grid
    std::vector<uint32_t> ctab, cpool;
    uint32_t ncpool = 0;
    // bricks: static [0, ns), body bricks [ns, ns + nd)
    uint32_t ns = 0, nd = 0;
    std::vector<uint8_t> mat, infill;
    std::vector<int32_t> bx, by, bz, sid;
    std::vector<uint32_t> body, next, sup;
    std::vector<V> local, wpos;
    std::vector<uint32_t> nb6;     // 6 per brick
    std::vector<float> bond, bmax; // 4 per brick
    std::vector<float> phi, ext, stress;
    std::vector<double> phi64;
    // bodies
    uint32_t nbody = 0;
    std::vector<uint8_t> alive, asleep, wake;
    std::vector<uint32_t> first, count, nc;
    std::vector<V> pos, v, w, vpre, wpre;
    std::vector<float> q;           // 4 per body
    std::vector<float> rot, iil, iiw; // 9 per body
    std::vector<float> m, im, sleep, rad, maxr;
    // per-step
    std::vector<uint32_t> hhead, hnext;
    std::vector<Contact> cs;
    std::vector<uint32_t> island;    // per body, last substep
    std::vector<uint32_t> man_a, man_b, man_color, man_start, man_count, man_contacts;
    uint32_t ncolors = 0;
    uint32_t chunk = 16;             // contacts per solve chunk of a body pair (0 = the whole pair)
    // contact reduction and warm start (off unless the step asks): the last substep's impulses per contact key
    struct WarmKey { uint64_t k1; uint32_t k2; bool operator==(const WarmKey& o) const { return k1 == o.k1 && k2 == o.k2; } };
    struct WarmHash { size_t operator()(const WarmKey& k) const { return std::hash<uint64_t>()(k.k1 * 0x9E3779B97F4A7C15ull ^ k.k2); } };
    struct WarmVal { float jn; V f; };
    std::unordered_map<WarmKey, WarmVal, WarmHash> warm_tab;
    bool warm_valid = false;
    uint32_t reduce = 0, warm = 0;
    uint32_t frame = 0;
    uint64_t would_drop = 0;         // contacts the reference would have dropped past MAXC
    // the per-frame load-path schedule, per structure (src/lib.rs:241: st_warm, st_solved, st_settle, st_resid)
    std::vector<int32_t> st_warm;
    std::vector<uint8_t> st_solved;
    std::vector<float> st_settle;
    std::vector<double> st_resid;
    std::vector<int64_t> st_size;    // bricks per structure at creation (the reference's st_hi - st_lo)
    std::vector<uint8_t> st_conn;    // per structure: a joint failed or a brick was crushed since the last walk
    uint32_t cap_bodies = 0, cap_bricks = 0;   // capacity for detached pieces (bodies, body bricks)
    std::vector<uint8_t> dirty;      // per body: a brick was removed since its last rebuild (bd_dirty)
    // the debris-body load field, per body (src/lib.rs:246-252: bd_vlast, bd_wlast, bd_resid, bd_nmax, bd_lt)
    std::vector<V> vlast, wlast;
    std::vector<double> bresid;
    std::vector<float> nmax, blt;
    std::vector<uint32_t> stamp;     // per brick: the crush that visited it last (src/lib.rs:1650)
    uint32_t stamp_id = 0, dmg_draws = 0;
    uint64_t dmg[7] = {0, 0, 0, 0, 0, 0, 0};  // candidates, crushed, removed, severed, cracked, ploughed loose, scraped
    std::vector<uint8_t> st_hit;     // per structure: woken by a hit since the last read (st_activate)
    uint32_t rebuilds = 0;           // bodies rebuilt so far (the lone-brick rule's draw key)
    uint32_t crush_n = 0;

    uint32_t gget(int x, int y, int z) const {
        if (!inb(x, y, z)) return 0;
        uint32_t t = ctab[((y >> 3) * CZN + (z >> 3)) * CXN + (x >> 3)];
        if (t == 0) return 0;
        return cpool[(size_t)(t - 1) * 512 + (((y & 7) * 8 + (z & 7)) * 8 + (x & 7))];
    }
    bool gset(int x, int y, int z, uint32_t val) {
        if (!inb(x, y, z)) return false;
        uint32_t ci = ((y >> 3) * CZN + (z >> 3)) * CXN + (x >> 3);
        uint32_t t = ctab[ci];
        if (t == 0) {
            if (val == 0) return true;
            ncpool++;
            t = ncpool;
            ctab[ci] = t;
            cpool.resize((size_t)ncpool * 512, 0);
        }
        cpool[(size_t)(t - 1) * 512 + (((y & 7) * 8 + (z & 7)) * 8 + (x & 7))] = val;
        return true;
    }
    uint32_t static_brick(int x, int y, int z) const {
        uint32_t g = gget(x, y, z);
        if (g == 0) return NONE;
        uint32_t j = g - 1;
        return (mat[j] != 0 && body[j] == STATIC) ? j : NONE;
    }
    // src/lib.rs:378-383
    bool linked(uint32_t i, int d, uint32_t& jo, float& hp) const {
        uint32_t j = nb6[(size_t)i * 6 + d];
        if (j == NONE || mat[j] == 0 || body[j] != body[i]) return false;
        float h = (d & 1) == 0 ? bond[(size_t)i * 4 + (d >> 1)] : bond[(size_t)j * 4 + (d >> 1)];
        if (h > 0.0f) { jo = j; hp = h; return true; }
        return false;
    }
    float axis_up(uint32_t i, int a) const { return body[i] == STATIC ? (a == 1 ? 1.0f : 0.0f) : rot[(size_t)body[i] * 9 + 3 + a]; }
    float cond_w(uint32_t i, uint32_t j, int a) const {
        float k = minf(STIFF[mat[i]], STIFF[mat[j]]);
        if (body[i] == STATIC) return k * (a == 1 ? 1.0f : 0.3f);
        float u = fabs_(axis_up(i, a));
        return k * (0.3f + 0.7f * u);
    }
    bool in_struct(uint32_t i, int s) const { return sid[i] == s && mat[i] != 0 && mat[i] < SLUG && body[i] == STATIC; }
};

static float bond_cap(uint8_t mi, uint8_t mj, int axis) {
    float a = axis == 1 ? CAPV[mi] : CAPH[mi];
    float b = axis == 1 ? CAPV[mj] : CAPH[mj];
    return minf(a, b);
}

// src/lib.rs:668-696 (corner jitter and face masks are rendering data and are left out)
static void finalize_brick(World& w, uint32_t i) {
    if (w.mat[i] == 0) return;
    for (int d = 0; d < 6; d++) {
        uint32_t g = w.gget(w.bx[i] + DIRS[d][0], w.by[i] + DIRS[d][1], w.bz[i] + DIRS[d][2]);
        w.nb6[(size_t)i * 6 + d] = g == 0 ? NONE : g - 1;
    }
    for (int a = 0; a < 3; a++) {
        uint32_t j = w.nb6[(size_t)i * 6 + a * 2];
        bool gap = j != NONE && w.infill[i] != w.infill[j] && (a != 1 || w.infill[i] == 1);
        if (j != NONE && !gap && w.mat[j] != 0 && w.body[j] == w.body[i] && w.sid[j] == w.sid[i]) {
            float c = bond_cap(w.mat[i], w.mat[j], a);
            w.bond[(size_t)i * 4 + a] = c; w.bmax[(size_t)i * 4 + a] = c;
        } else { w.bond[(size_t)i * 4 + a] = 0.0f; w.bmax[(size_t)i * 4 + a] = 0.0f; }
    }
    if (w.by[i] == 0 && w.body[i] == STATIC) {
        float c = CAPV[w.mat[i]] * 2.0f;
        w.bond[(size_t)i * 4 + 3] = c; w.bmax[(size_t)i * 4 + 3] = c;
    } else { w.bond[(size_t)i * 4 + 3] = 0.0f; w.bmax[(size_t)i * 4 + 3] = 0.0f; }
}

// src/lib.rs:844-891, for the body's bricks lst[0..n) with local[] already holding lattice positions
static void setup_body(World& w, uint32_t b, const uint32_t* lst, uint32_t n, V ppos, const float* prot, const float* pq, V pv, V pw) {
    float mass = 0.0f;
    V cl = vv(0, 0, 0);
    for (uint32_t t = 0; t < n; t++) { uint32_t i = lst[t]; float mm = MASS[w.mat[i]]; mass += mm; cl = madd(cl, w.local[i], mm); }
    cl = mul(cl, 1.0f / mass);
    float it[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float rad = 0.0f;
    const float cube = S * S / 6.0f;
    for (uint32_t t = 0; t < n; t++) {
        uint32_t i = lst[t];
        float mm = MASS[w.mat[i]];
        V r = sub(w.local[i], cl);
        w.local[i] = r;
        float rr = dot(r, r);
        rad = maxf(rad, rr);
        it[0] += mm * (rr - r[0] * r[0] + cube); it[4] += mm * (rr - r[1] * r[1] + cube); it[8] += mm * (rr - r[2] * r[2] + cube);
        it[1] -= mm * r[0] * r[1]; it[2] -= mm * r[0] * r[2]; it[5] -= mm * r[1] * r[2];
        w.body[i] = b;
        w.next[i] = t + 1 < n ? lst[t + 1] : NONE;
    }
    it[3] = it[1]; it[6] = it[2]; it[7] = it[5];
    float* iil = &w.iil[(size_t)b * 9];
    minv(it, iil);
    V off = mv(prot, cl);
    w.alive[b] = 1;
    w.first[b] = lst[0];
    w.count[b] = n;
    w.pos[b] = add(ppos, off);
    for (int k = 0; k < 4; k++) w.q[(size_t)b * 4 + k] = pq[k];
    std::memcpy(&w.rot[(size_t)b * 9], prot, 9 * sizeof(float));
    w.v[b] = add(pv, cross(pw, off));
    w.w[b] = pw;
    w.m[b] = mass; w.im[b] = 1.0f / mass;
    float t1[9], t2[9];
    mmul(prot, iil, t1); mt(prot, t2); mmul(t1, t2, &w.iiw[(size_t)b * 9]);
    w.sleep[b] = 0.0f; w.asleep[b] = 0; w.wake[b] = 0; w.maxr[b] = 0.0f;
    // a new field (src/lib.rs:845, 882): the load time, the residual and the peak factor start over
    w.blt[b] = 0.0f; w.bresid[b] = 1.0; w.nmax[b] = 1.0f; w.vlast[b] = w.v[b]; w.wlast[b] = pw;
    w.rad[b] = std::sqrt(rad) + H * 1.8f;
    for (uint32_t t = 0; t < n; t++) { uint32_t i = lst[t]; w.wpos[i] = add(w.pos[b], mv(prot, w.local[i])); }
}

static void clamp_vel(World& w, uint32_t b) {
    float vl = len(w.v[b]);
    if (vl > 60.0f) w.v[b] = mul(w.v[b], 60.0f / vl);
    float a = len(w.w[b]);
    float amax = minf(25.0f, 16.0f / maxf(w.rad[b], 0.3f));
    if (a > amax) w.w[b] = mul(w.w[b], amax / a);
}

static void kill_body(World& w, uint32_t b) {
    uint32_t k = w.first[b];
    while (k != NONE) { uint32_t nx = w.next[k]; if (w.body[k] == b) { w.mat[k] = 0; w.body[k] = STATIC; } k = nx; }
    w.alive[b] = 0; w.first[b] = NONE;
}

// ---------------------------------------------------------------- SOR (src/lib.rs:1005-1040)
template <class T> struct PhiRef;
static float sor_brick(World& w, uint32_t i, float omega) {
    uint8_t mi = w.mat[i];
    float sk = 0.0f, skp = 0.0f;
    for (int d = 0; d < 6; d++) {
        uint32_t j; float hp;
        if (!w.linked(i, d, j, hp)) continue;
        float k = w.cond_w(i, j, d >> 1);
        sk += k; skp += k * w.phi[j];
    }
    if (w.body[i] == STATIC) { if (w.by[i] == 0 && w.bond[(size_t)i * 4 + 3] > 0.0f) sk += GROUNDK * STIFF[mi]; }
    else if (w.frame - w.sup[i] < 10u) sk += GROUNDK * STIFF[mi];
    if (sk > 0.0f) {
        float target = (MASS[mi] + w.ext[i] + skp) / sk;
        float d = omega * (target - w.phi[i]);
        w.phi[i] += d;
        return fabs_(d);
    }
    return 0.0f;
}
// the same system in double precision (coefficients are the reference's f32 values, promoted)
static double sor_brick64(World& w, uint32_t i, double omega) {
    uint8_t mi = w.mat[i];
    double sk = 0.0, skp = 0.0;
    for (int d = 0; d < 6; d++) {
        uint32_t j; float hp;
        if (!w.linked(i, d, j, hp)) continue;
        double k = (double)w.cond_w(i, j, d >> 1);
        sk += k; skp += k * w.phi64[j];
    }
    if (w.body[i] == STATIC) { if (w.by[i] == 0 && w.bond[(size_t)i * 4 + 3] > 0.0f) sk += (double)(GROUNDK * STIFF[mi]); }
    // a body brick with a supporting contact in the last 10 frames rests on the ground (src/lib.rs:1016)
    else if ((uint32_t)(w.frame - w.sup[i]) < 10u) sk += (double)(GROUNDK * STIFF[mi]);
    if (sk > 0.0) {
        double target = ((double)(MASS[mi] + w.ext[i]) + skp) / sk;
        double d = omega * (target - w.phi64[i]);
        w.phi64[i] += d;
        return std::fabs(d);
    }
    return 0.0;
}

struct SorResult { uint32_t sweeps; double resid; };

// mode 0: reference lexicographic f32 sweeps; 1: the same in f64; 2: red-black f32 (red = even (x+y+z));
// 3: red-black f64
static SorResult sor_solve(World& w, int s, float omega, double tol, uint32_t max_sweeps, int mode) {
    std::vector<uint32_t> list;
    for (uint32_t i = 0; i < w.ns; i++) if (w.in_struct(i, s)) list.push_back(i);
    SorResult r{0, 1e30};
    if (list.empty()) { r.resid = 0.0; return r; }
    if (mode == 1 || mode == 3) {
        for (uint32_t i : list) w.phi64[i] = (double)w.phi[i];
    }
    while (r.sweeps < max_sweeps) {
        if (mode == 0) {
            float md = 0.0f, mp = 1.0f;
            for (uint32_t i : list) { float d = sor_brick(w, i, omega); if (d > md) md = d; if (w.phi[i] > mp) mp = w.phi[i]; }
            r.resid = (double)(md / mp);
        } else if (mode == 1) {
            double md = 0.0, mp = 1.0;
            for (uint32_t i : list) { double d = sor_brick64(w, i, (double)omega); if (d > md) md = d; if (w.phi64[i] > mp) mp = w.phi64[i]; }
            r.resid = md / mp;
        } else if (mode == 3) {
            double md = 0.0, mp = 1.0;
            for (int colour = 0; colour < 2; colour++)
                for (uint32_t i : list) {
                    if (((w.bx[i] + w.by[i] + w.bz[i]) & 1) != colour) continue;
                    double d = sor_brick64(w, i, (double)omega); if (d > md) md = d;
                }
            for (uint32_t i : list) if (w.phi64[i] > mp) mp = w.phi64[i];
            r.resid = md / mp;
        } else {
            float md = 0.0f, mp = 1.0f;
            for (int colour = 0; colour < 2; colour++)
                for (uint32_t i : list) {
                    if (((w.bx[i] + w.by[i] + w.bz[i]) & 1) != colour) continue;
                    float d = sor_brick(w, i, omega); if (d > md) md = d;
                }
            for (uint32_t i : list) if (w.phi[i] > mp) mp = w.phi[i];
            r.resid = (double)(md / mp);
        }
        r.sweeps++;
        if (r.resid < tol) break;
    }
    if (mode == 1 || mode == 3) for (uint32_t i : list) w.phi[i] = (float)w.phi64[i];
    return r;
}

// ---------------------------------------------------------------- joint checks (src/lib.rs:1153-1227)
enum { J_HOLD = 0, J_FATIGUE = 1, J_FAIL = 2, J_CRUSH = 3 };
struct Joint { uint32_t i, axis, j, decision, crushed; float ratio, bond_after; };
// a failed joint or a crushed brick leaves its structure pending a connectivity walk (src/lib.rs:714, 1202, 1223)
static void flag_conn(World& w, int32_t s) { if (s >= 0 && s < (int32_t)w.st_conn.size()) w.st_conn[s] = 1; }
static void remove_brick(World& w, uint32_t i);

static float stress_brick(World& w, uint32_t i, float dt, bool live, std::vector<Joint>& out) {
    uint8_t mi = w.mat[i];
    bool dynb = w.body[i] != STATIC;
    float maxr = 0.0f;
    for (int a = 0; a < 3; a++) {
        uint32_t j; float hp;
        if (!w.linked(i, a * 2, j, hp)) continue;
        float f = w.cond_w(i, j, a) * (w.phi[i] - w.phi[j]);
        float u = w.axis_up(i, a);
        float up = f > 0.0f ? maxf(u, 0.0f) : maxf(-u, 0.0f);
        float tens = minf(TENS[mi], TENS[w.mat[j]]);
        float capm = 1.0f - (1.0f - tens) * up;
        float hpw = hp;
        if (dynb) {
            float cv = minf(CAPV[mi], CAPV[w.mat[j]]), ch = minf(CAPH[mi], CAPH[w.mat[j]]);
            float lat = a == 1 ? cv : ch;
            float au = fabs_(u);
            hpw = hp * (cv * au + ch * (1.0f - au)) / maxf(lat, 1.0f);
        }
        float r = fabs_(f) / (hpw * capm);
        if (r > w.stress[i]) w.stress[i] = r;
        if (r > w.stress[j]) w.stress[j] = r;
        if (r > maxr) maxr = r;
        Joint jr{i, (uint32_t)a, j, J_HOLD, NONE, r, hp};
        if (live && r > 1.0f) {
            float nhp = dynb ? hp - hp * dt * DUCT[mi] * minf(r - 0.85f, 40.0f) : hp - hp * dt * 2.2f * minf(r - 0.85f, 2.5f);
            if (nhp < w.bmax[(size_t)i * 4 + a] * 0.08f) {
                if (up == 0.0f && fabs_(u) > 0.5f && w.crush_n < 300) {
                    w.crush_n++;
                    if (!dynb) flag_conn(w, w.sid[i]);
                    uint32_t k = CAPV[w.mat[j]] < CAPV[mi] ? j : i;
                    jr.decision = J_CRUSH; jr.crushed = k; jr.bond_after = hp;
                    out.push_back(jr);
                    remove_brick(w, k);   // a body brick's removal marks its body for rebuild (src/lib.rs:717)
                    return maxf(maxr, r);
                }
                w.bond[(size_t)i * 4 + a] = 0.0f;
                if (!dynb) flag_conn(w, w.sid[i]);
                else w.dirty[w.body[i]] = 1;   // src/lib.rs:1201
                jr.decision = J_FAIL; jr.bond_after = 0.0f;
            } else {
                w.bond[(size_t)i * 4 + a] = nhp;
                jr.decision = J_FATIGUE; jr.bond_after = nhp;
            }
        }
        out.push_back(jr);
    }
    if (!dynb && w.by[i] == 0 && w.bond[(size_t)i * 4 + 3] > 0.0f) {
        float f = GROUNDK * STIFF[mi] * w.phi[i];
        float r = f / w.bond[(size_t)i * 4 + 3];
        if (r > w.stress[i]) w.stress[i] = r;
        if (r > maxr) maxr = r;
        Joint jr{i, 3u, NONE, J_HOLD, NONE, r, w.bond[(size_t)i * 4 + 3]};
        if (live && r > 1.0f) {
            float& b3 = w.bond[(size_t)i * 4 + 3];
            b3 -= b3 * dt * 2.2f * (r - 0.85f);
            if (b3 < w.bmax[(size_t)i * 4 + 3] * 0.08f) { b3 = 0.0f; jr.decision = J_FAIL; flag_conn(w, w.sid[i]); }
            else jr.decision = J_FATIGUE;
            jr.bond_after = b3;
        }
        out.push_back(jr);
    }
    return maxr;
}

// ---------------------------------------------------------------- the per-frame schedule (src/lib.rs:1061-1079, 1268-1281)
// Restated with red-black FP64 sweeps that continue from the stored f64 potentials (the GPU path's arithmetic):
// the schedule (which structures sweep, how often, with which omega, from which budget) is the reference's.
static double rb64_sweep(World& w, const std::vector<uint32_t>& list, double omega) {
    double md = 0.0, mp = 1.0;
    for (int colour = 0; colour < 2; colour++)
        for (uint32_t i : list) {
            if (((w.bx[i] + w.by[i] + w.bz[i]) & 1) != colour) continue;
            double d = sor_brick64(w, i, omega);
            if (d > md) md = d;
        }
    for (uint32_t i : list) if (w.phi64[i] > mp) mp = w.phi64[i];
    return md / mp;
}
static void sched_size(World& w) {
    const int32_t n = (int32_t)w.st_size.size();
    if ((int32_t)w.st_warm.size() < n) {
        w.st_warm.resize(n, 0); w.st_solved.resize(n, 0); w.st_settle.resize(n, 0.0f); w.st_resid.resize(n, 0.0);
    }
}
static void warm_struct(World& w, int32_t s) {   // src/lib.rs:1061-1066
    sched_size(w);
    if (s < 0 || s >= (int32_t)w.st_warm.size() || w.st_solved[s]) return;
    w.st_solved[s] = 1;
    w.st_warm[s] = 560;
    w.st_settle[s] = 1e9f;
}
static void structure_frame(World& w, uint32_t frame, float dt, const int32_t* active, uint32_t n_active, uint32_t* counts) {
    sched_size(w);
    const int32_t nst = (int32_t)w.st_warm.size();
    std::vector<std::vector<uint32_t>> lists(nst);
    for (uint32_t i = 0; i < w.ns; i++) if (w.sid[i] >= 0 && w.in_struct(i, w.sid[i])) lists[w.sid[i]].push_back(i);
    uint32_t sweeps = 0, warm_sweeps = 0;
    std::vector<int32_t> act;
    for (uint32_t t = 0; t < n_active; t++) {
        int32_t s = active[t];
        if (s >= 0 && s < nst && w.st_solved[s] && w.st_size[s] > 0) act.push_back(s);
    }
    // the sweep loop of structural (src/lib.rs:1268-1281); a structure's size is its brick range at creation
    int64_t budget = 160000;
    for (int32_t s : act) {
        const int64_t size = w.st_size[s];
        const uint32_t nmin = w.st_resid[s] < 1e-4 ? (((frame + (uint32_t)s) % 3 == 0) ? 1u : 0u) : (size > 15000 ? 1u : 6u);
        if (nmin == 0) continue;
        uint32_t n = 0;
        for (;;) {
            w.st_resid[s] = rb64_sweep(w, lists[s], (double)1.85f);
            n++; budget -= size;
            if (n >= nmin && (w.st_resid[s] < (double)4e-4f || n >= 90 || budget <= 0)) break;
        }
        sweeps += n;
    }
    for (int32_t s : act) for (uint32_t i : lists[s]) w.phi[i] = (float)w.phi64[i];
    // the joint pass (src/lib.rs:1323-1339) of the live structures, in structure order, one crush budget a frame
    // (src/lib.rs:3645); structures that are not live only shade their stress display there and are left out
    std::vector<int32_t> live;
    for (int32_t s : act) if (w.st_settle[s] <= 0.0f && w.st_resid[s] < (double)1.5e-3f) live.push_back(s);
    std::sort(live.begin(), live.end());
    w.crush_n = 0;
    uint32_t joints = 0, over = 0, failed = 0, crushed = 0;
    float mr = 0.0f;
    for (int32_t s : live) {
        std::vector<Joint> out;
        for (uint32_t i : lists[s]) if (w.in_struct(i, s)) w.stress[i] = 0.0f;
        for (uint32_t i : lists[s]) if (w.in_struct(i, s)) { float r = stress_brick(w, i, dt, true, out); if (r > mr) mr = r; }
        for (const Joint& j : out) {
            joints++;
            if (j.ratio > 1.0f) over++;
            if (j.decision == J_FAIL) failed++;
            if (j.decision == J_CRUSH) crushed++;
        }
    }
    // the settle timers (src/lib.rs:1334)
    for (int32_t s : act) if (w.st_settle[s] > 0.0f && w.st_warm[s] == 0) w.st_settle[s] -= dt;
    // warm_step (src/lib.rs:1068-1079)
    int64_t wb = 120000;
    for (int32_t s = 0; s < nst; s++) {
        const int64_t size = w.st_size[s];
        if (size == 0) continue;
        while (w.st_warm[s] > 0 && wb > 0) {
            const float om = w.st_warm[s] > 60 ? 1.9f : 1.0f;
            w.st_resid[s] = rb64_sweep(w, lists[s], (double)om);
            w.st_warm[s] -= 1;
            wb -= size;
            warm_sweeps++;
            if (w.st_warm[s] == 0) w.st_settle[s] = 0.3f;
        }
    }
    for (int32_t s = 0; s < nst; s++) for (uint32_t i : lists[s]) w.phi[i] = (float)w.phi64[i];
    if (counts) {
        counts[0] = sweeps; counts[1] = warm_sweeps; counts[2] = (uint32_t)live.size(); counts[3] = joints;
        counts[4] = over; counts[5] = failed; counts[6] = crushed;
        std::memcpy(&counts[7], &mr, 4);
    }
}

// ---------------------------------------------------------------- connectivity (src/lib.rs:925-929, 1085-1141)
// wake_near (src/lib.rs:925-929)
static void wake_near(World& w, V p, float r) {
    for (uint32_t b = 0; b < w.nbody; b++)
        if (w.alive[b] && w.asleep[b] && len(sub(w.pos[b], p)) < r + w.rad[b]) { w.asleep[b] = 0; w.sleep[b] = 0.0f; }
}
// A new body for a detached piece: the next body id, its bricks appended to the body bricks in walk order (the
// reference keeps a brick's id when it changes owner; ids only order pair tests, and the library appends, so this
// restatement appends too). False when the capacity given at creation is spent.
// a new body of the listed static bricks in the next spare body and bricks (the bricks keep their bonds, their
// neighbours renumbered within the piece; the static bricks leave with potential and load 0), set up about the
// origin with velocity pv; returns the body
static uint32_t body_from_statics(World& w, const std::vector<uint32_t>& lst, V pv);
static bool detach_piece(World& w, const std::vector<uint32_t>& lst) {
    const uint32_t n = (uint32_t)lst.size();
    if (w.nbody + 1 > w.cap_bodies || w.nd + n > w.cap_bricks) return false;
    w.warm_valid = false;   // brick ids move: the warm-start table starts over
    const uint32_t b = body_from_statics(w, lst, vv(0, 0, 0));
    wake_near(w, w.pos[b], w.rad[b] + 1.5f);
    return true;
}
static uint32_t body_from_statics(World& w, const std::vector<uint32_t>& lst, V pv) {
    const uint32_t n = (uint32_t)lst.size();
    const uint32_t b = w.nbody++;
    w.alive.push_back(0); w.asleep.push_back(0); w.wake.push_back(0);
    w.first.push_back(NONE); w.count.push_back(0); w.nc.push_back(0);
    w.pos.push_back(vv(0, 0, 0)); w.v.push_back(vv(0, 0, 0)); w.w.push_back(vv(0, 0, 0));
    w.vpre.push_back(vv(0, 0, 0)); w.wpre.push_back(vv(0, 0, 0));
    for (int k = 0; k < 4; k++) w.q.push_back(0.0f);
    for (int k = 0; k < 9; k++) { w.rot.push_back(0.0f); w.iil.push_back(0.0f); w.iiw.push_back(0.0f); }
    w.m.push_back(0.0f); w.im.push_back(0.0f); w.sleep.push_back(0.0f); w.rad.push_back(0.0f); w.maxr.push_back(0.0f);
    w.island.push_back(NONE); w.dirty.push_back(0);
    w.vlast.push_back(vv(0, 0, 0)); w.wlast.push_back(vv(0, 0, 0)); w.bresid.push_back(1.0); w.nmax.push_back(1.0f); w.blt.push_back(0.0f);
    std::vector<uint32_t> nl;
    const uint32_t k0 = w.ns + w.nd;
    std::unordered_map<uint32_t, uint32_t> place;
    for (uint32_t t = 0; t < n; t++) place[lst[t]] = k0 + t;
    for (uint32_t i : lst) {
        const uint32_t k = w.ns + w.nd++;
        w.mat.push_back(w.mat[i]); w.infill.push_back(0);
        w.bx.push_back(w.bx[i]); w.by.push_back(w.by[i]); w.bz.push_back(w.bz[i]); w.sid.push_back(-1);
        w.body.push_back(STATIC); w.next.push_back(NONE); w.sup.push_back(0);
        w.local.push_back(lat_pos(w.bx[i], w.by[i], w.bz[i])); w.wpos.push_back(vv(0, 0, 0));
        // the brick keeps its bonds (src/lib.rs:1118); its neighbours are renumbered to the piece's new ids
        for (int d = 0; d < 6; d++) {
            const uint32_t j = w.nb6[(size_t)i * 6 + d];
            const auto it = j == NONE ? place.end() : place.find(j);
            w.nb6.push_back(it == place.end() ? NONE : it->second);
        }
        for (int a = 0; a < 4; a++) { w.bond.push_back(w.bond[(size_t)i * 4 + a]); w.bmax.push_back(w.bmax[(size_t)i * 4 + a]); }
        w.phi.push_back(0.0f); w.ext.push_back(0.0f); w.stress.push_back(0.0f); w.phi64.push_back(0.0);
        w.hnext.push_back(NONE);
        nl.push_back(k);
        // the static brick leaves the static set with potential and load 0 (src/lib.rs:1118)
        w.gset(w.bx[i], w.by[i], w.bz[i], 0);
        w.mat[i] = 0; w.phi[i] = 0.0f; w.phi64[i] = 0.0; w.ext[i] = 0.0f;
    }
    const float idm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const float q0[4] = {0, 0, 0, 1};
    setup_body(w, b, nl.data(), n, vv(0, 0, 0), idm, q0, pv, vv(0, 0, 0));
    return b;
}
// conn_struct (src/lib.rs:1085-1134): the grounded walk from the footings, then one body per remaining piece in brick
// order. counts: [0] pieces, [1] detached bricks, [2] 1 = a piece did not fit (the structure stays pending).
static void conn_struct(World& w, int32_t s, uint32_t* counts) {
    std::vector<uint8_t> stamp(w.ns, 0);
    std::vector<uint32_t> q;
    for (uint32_t i = 0; i < w.ns; i++)
        if (w.in_struct(i, s) && w.by[i] == 0 && w.bond[(size_t)i * 4 + 3] > 0.0f) { stamp[i] = 1; q.push_back(i); }
    for (size_t h = 0; h < q.size(); h++) {
        const uint32_t i = q[h];
        for (int d = 0; d < 6; d++) {
            uint32_t j; float hp;
            if (w.linked(i, d, j, hp) && !stamp[j]) { stamp[j] = 1; q.push_back(j); }
        }
    }
    bool retry = false;
    std::vector<uint32_t> lst;
    for (uint32_t st = 0; st < w.ns; st++) {
        if (!w.in_struct(st, s) || stamp[st]) continue;
        lst.clear();
        stamp[st] = 1;
        lst.push_back(st);
        for (size_t h = 0; h < lst.size(); h++) {
            const uint32_t i = lst[h];
            for (int d = 0; d < 6; d++) {
                uint32_t j; float hp;
                if (w.linked(i, d, j, hp) && !stamp[j]) { stamp[j] = 1; lst.push_back(j); }
            }
        }
        if (!detach_piece(w, lst)) { retry = true; continue; }
        counts[0]++;
        counts[1] += (uint32_t)lst.size();
    }
    if (retry) { w.st_conn[s] = 1; counts[2]++; }
}
// finalize_brick's bond rule (src/lib.rs:668-696) between face-adjacent bricks of one body (glass is infill; no
// foundation bond), for the bodies the scene describes
static void body_bonds(World& w) {
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!w.alive[b]) continue;
        std::vector<uint32_t> lst;
        for (uint32_t k = w.first[b]; k != NONE; k = w.next[k]) lst.push_back(k);
        for (uint32_t i : lst) {
            for (int d = 0; d < 6; d++) {
                uint32_t nj = NONE;
                for (uint32_t j : lst)
                    if (w.bx[j] == w.bx[i] + DIRS[d][0] && w.by[j] == w.by[i] + DIRS[d][1] && w.bz[j] == w.bz[i] + DIRS[d][2]) nj = j;
                w.nb6[(size_t)i * 6 + d] = nj;
            }
            const uint8_t ii = w.mat[i] == GLASS ? 1 : 0;
            for (int a = 0; a < 3; a++) {
                const uint32_t j = w.nb6[(size_t)i * 6 + a * 2];
                float c = 0.0f;
                if (j != NONE) {
                    const uint8_t ij = w.mat[j] == GLASS ? 1 : 0;
                    const bool gap = ii != ij && (a != 1 || ii == 1);
                    if (!gap && w.mat[j] != 0) c = bond_cap(w.mat[i], w.mat[j], a);
                }
                w.bond[(size_t)i * 4 + a] = c; w.bmax[(size_t)i * 4 + a] = c;
            }
            w.bond[(size_t)i * 4 + 3] = 0.0f; w.bmax[(size_t)i * 4 + 3] = 0.0f;
        }
    }
}
// remove_brick (src/lib.rs:705-718): a static brick leaves the grid and its structure is pending; a body brick's body
// is marked for rebuild
static void remove_brick(World& w, uint32_t i) {
    if (w.mat[i] == 0) return;
    if (w.body[i] == STATIC) {
        if (w.gget(w.bx[i], w.by[i], w.bz[i]) == i + 1) w.gset(w.bx[i], w.by[i], w.bz[i], 0);
        w.mat[i] = 0;
        flag_conn(w, w.sid[i]);
    } else {
        w.mat[i] = 0;
        w.dirty[w.body[i]] = 1;
    }
}
// h01 (src/lib.rs:341-345)
static float h01(uint32_t h, uint32_t k) {
    uint32_t x = h + k * 0x9E3779B9u;
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return (float)(x >> 8) / 16777216.0f;
}
// rebuild_body (src/lib.rs:930-1002) with the library's brick layout: a body's bricks are the ids [first, first +
// count); the first component moves to the front of that range in list order, every other takes the next body id and
// the next brick ids; ids left over are unowned. The lone-brick rule draws h01(bodies rebuilt so far, place in body)
// and counts the bodies awake now (the reference: its random stream and the last frame's awake count).
static void rebuild_body(World& w, uint32_t id, uint32_t* counts) {
    const uint32_t first = w.first[id], cnt = w.count[id];
    const uint32_t key = w.rebuilds++;
    w.dirty[id] = 0;
    counts[0]++;
    std::vector<uint32_t> lst;
    for (uint32_t t = 0; t < cnt; t++) {
        if (w.mat[first + t] != 0) lst.push_back(t);
        else { w.body[first + t] = STATIC; counts[2]++; }
    }
    if (lst.empty()) {   // the body dies; its ids are unowned, without neighbours, as the library frees them
        for (uint32_t t = 0; t < cnt; t++) for (int d = 0; d < 6; d++) w.nb6[(size_t)(first + t) * 6 + d] = NONE;
        w.alive[id] = 0; w.first[id] = NONE; w.count[id] = 0; counts[3]++;
        return;
    }
    std::vector<int32_t> comp(cnt, -1);
    uint32_t ncomp = 0;
    for (uint32_t t0 : lst) {
        if (comp[t0] >= 0) continue;
        comp[t0] = (int32_t)ncomp;
        std::vector<uint32_t> q{t0};
        for (size_t h = 0; h < q.size(); h++) {
            const uint32_t i = first + q[h];
            for (int d = 0; d < 6; d++) {
                uint32_t j; float hp;
                if (!w.linked(i, d, j, hp)) continue;
                const uint32_t tj = j - first;
                if (comp[tj] >= 0) continue;
                comp[tj] = (int32_t)ncomp;
                q.push_back(tj);
            }
        }
        ncomp++;
    }
    uint32_t nc = ncomp;
    if (nc > 1) {
        uint32_t extra = 0;
        for (uint32_t t : lst) if (comp[t] > 0) extra++;
        if (w.nbody + (nc - 1) > w.cap_bodies || w.nd + extra > w.cap_bricks) { for (uint32_t t : lst) comp[t] = 0; nc = 1; }
    }
    std::vector<std::vector<uint32_t>> groups(nc);
    for (uint32_t t : lst) groups[comp[t]].push_back(t);
    // the parent's pose and cached rotation (src/lib.rs:968)
    const V ppos = w.pos[id], pv = w.v[id], pw = w.w[id];
    float pq[4], prot[9];
    for (int k = 0; k < 4; k++) pq[k] = w.q[(size_t)id * 4 + k];
    for (int k = 0; k < 9; k++) prot[k] = w.rot[(size_t)id * 9 + k];
    uint32_t awake = 0;
    for (uint32_t b = 0; b < w.nbody; b++) if (w.alive[b] && !w.asleep[b]) awake++;
    // copies of the kept bricks (the first component's moves overwrite ids it reads)
    struct Rec { uint8_t mat, infill; int32_t x, y, z, sid; V local; uint32_t nb6[6]; float bond[4], bmax[4]; uint32_t sup; float phi, ext; double phi64; };
    std::vector<Rec> rec(cnt);
    for (uint32_t t = 0; t < cnt; t++) {
        const uint32_t i = first + t;
        Rec& r = rec[t];
        r.mat = w.mat[i]; r.infill = w.infill[i]; r.x = w.bx[i]; r.y = w.by[i]; r.z = w.bz[i]; r.sid = w.sid[i];
        r.local = w.local[i]; r.sup = w.sup[i]; r.phi = w.phi[i]; r.ext = w.ext[i]; r.phi64 = w.phi64[i];
        for (int d = 0; d < 6; d++) r.nb6[d] = w.nb6[(size_t)i * 6 + d];
        for (int a = 0; a < 4; a++) { r.bond[a] = w.bond[(size_t)i * 4 + a]; r.bmax[a] = w.bmax[(size_t)i * 4 + a]; }
    }
    for (uint32_t t = 0; t < cnt; t++) {   // the whole range is unowned until written again
        const uint32_t i = first + t;
        w.mat[i] = 0; w.body[i] = STATIC; w.next[i] = NONE;
        for (int d = 0; d < 6; d++) w.nb6[(size_t)i * 6 + d] = NONE;
    }
    std::vector<uint32_t> nid(cnt, NONE);
    std::vector<uint32_t> cbody(nc, NONE), cfirst(nc, 0);
    for (uint32_t c = 0; c < nc; c++) {
        const std::vector<uint32_t>& g = groups[c];
        if (c > 0 && g.size() == 1 && awake > 1500) {
            const float p = minf((float)(awake - 1500) / 2000.0f, 0.85f);
            if (rec[g[0]].mat != STEEL && h01(key, g[0]) < p) { counts[4]++; continue; }
        }
        if (c == 0) { cbody[c] = id; cfirst[c] = first; }
        else {
            const uint32_t b = w.nbody++;
            w.alive.push_back(0); w.asleep.push_back(0); w.wake.push_back(0);
            w.first.push_back(NONE); w.count.push_back(0); w.nc.push_back(0);
            w.pos.push_back(vv(0, 0, 0)); w.v.push_back(vv(0, 0, 0)); w.w.push_back(vv(0, 0, 0));
            w.vpre.push_back(vv(0, 0, 0)); w.wpre.push_back(vv(0, 0, 0));
            for (int k = 0; k < 4; k++) w.q.push_back(0.0f);
            for (int k = 0; k < 9; k++) { w.rot.push_back(0.0f); w.iil.push_back(0.0f); w.iiw.push_back(0.0f); }
            w.m.push_back(0.0f); w.im.push_back(0.0f); w.sleep.push_back(0.0f); w.rad.push_back(0.0f); w.maxr.push_back(0.0f);
            w.island.push_back(NONE); w.dirty.push_back(0);
    w.vlast.push_back(vv(0, 0, 0)); w.wlast.push_back(vv(0, 0, 0)); w.bresid.push_back(1.0); w.nmax.push_back(1.0f); w.blt.push_back(0.0f);
            cbody[c] = b;
            cfirst[c] = w.ns + w.nd;
            for (size_t t = 0; t < g.size(); t++) {
                w.nd++;
                w.mat.push_back(0); w.infill.push_back(0); w.bx.push_back(0); w.by.push_back(0); w.bz.push_back(0);
                w.sid.push_back(-1); w.body.push_back(STATIC); w.next.push_back(NONE); w.sup.push_back(0);
                w.local.push_back(vv(0, 0, 0)); w.wpos.push_back(vv(0, 0, 0));
                for (int d = 0; d < 6; d++) w.nb6.push_back(NONE);
                for (int a = 0; a < 4; a++) { w.bond.push_back(0.0f); w.bmax.push_back(0.0f); }
                w.phi.push_back(0.0f); w.ext.push_back(0.0f); w.stress.push_back(0.0f); w.phi64.push_back(0.0);
                w.hnext.push_back(NONE);
            }
            counts[1]++;
        }
        for (size_t t = 0; t < g.size(); t++) nid[g[t]] = cfirst[c] + (uint32_t)t;
    }
    for (uint32_t c = 0; c < nc; c++) {
        if (cbody[c] == NONE) continue;
        const std::vector<uint32_t>& g = groups[c];
        std::vector<uint32_t> ids;
        for (size_t t = 0; t < g.size(); t++) {
            const Rec& r = rec[g[t]];
            const uint32_t i = cfirst[c] + (uint32_t)t;
            w.mat[i] = r.mat; w.infill[i] = r.infill; w.bx[i] = r.x; w.by[i] = r.y; w.bz[i] = r.z; w.sid[i] = r.sid;
            w.local[i] = r.local; w.sup[i] = r.sup; w.phi[i] = r.phi; w.ext[i] = r.ext; w.phi64[i] = r.phi64;
            for (int d = 0; d < 6; d++) {
                const uint32_t j = r.nb6[d];
                uint32_t nj = NONE;
                if (j != NONE && j >= first && j < first + cnt && comp[j - first] == (int32_t)c) nj = nid[j - first];
                w.nb6[(size_t)i * 6 + d] = nj;
            }
            for (int a = 0; a < 4; a++) { w.bond[(size_t)i * 4 + a] = r.bond[a]; w.bmax[(size_t)i * 4 + a] = r.bmax[a]; }
            ids.push_back(i);
        }
        const float keep_lt = w.blt[cbody[c]];
        setup_body(w, cbody[c], ids.data(), (uint32_t)ids.size(), ppos, prot, pq, pv, pw);
        if (c == 0) w.blt[cbody[c]] = keep_lt;   // the body keeps its load time (src/lib.rs:998)
    }
}
// step's loop over marked bodies (src/lib.rs:3652). counts: bodies, pieces, removed bricks, dissolved, lone.
static void rebuild_bodies(World& w, uint32_t* counts) {
    for (int k = 0; k < 5; k++) counts[k] = 0;
    for (uint32_t b = 0; b < w.nbody; b++) if (w.alive[b] && w.dirty[b]) rebuild_body(w, b, counts);
    for (uint32_t b = 0; b < w.nbody; b++) w.dirty[b] = 0;
    if (counts[0]) w.warm_valid = false;   // brick ids move: the warm-start table starts over
}

// ---------------------------------------------------------------- the debris-body load field (src/lib.rs:1262-1365)
static void update_cache(World& w);
// body_loaded (src/lib.rs:1045-1047): awake, in contact, at least 8 bricks
static bool body_loaded(const World& w, uint32_t b) {
    return w.alive[b] && w.count[b] >= 8 && !w.asleep[b] && w.nc[b] > 0 && w.mat[w.first[b]] < SLUG;
}
static void body_list(const World& w, uint32_t b, std::vector<uint32_t>& out, bool only_present) {
    out.clear();
    for (uint32_t k = w.first[b]; k != NONE; k = w.next[k]) if (!only_present || w.mat[k] != 0) out.push_back(k);
}
// structural's body part after its loads: unsupported pieces start their field over, inertial loads g - a, the
// field's sweeps (red-black FP64 over the body's bricks, as the structures' sweeps here) from a budget of 160,000
// brick-updates in body order, then the pieces' joints (after the structures' joint pass, whose crush budget they
// continue). counts: [0] bodies swept, [1] sweeps, [2] brick updates, [3] joints, [4] over, [5] failed, [6] crushed,
// [7] the largest ratio's bits, [8] the frame's crushes after the pass. Brick updates count sweeps x bd_count, the
// budget's unit; crush_used is the structures' joint pass's crushes, which the budget of 300 counts on from.
static void body_frame(World& w, float dt, uint32_t crush_used, uint32_t* counts) {
    for (int k = 0; k < 9; k++) counts[k] = 0;
    w.crush_n = crush_used;
    update_cache(w);
    const uint32_t fr = w.frame;
    std::vector<uint32_t> lst;
    for (uint32_t b = 0; b < w.nbody; b++) {   // src/lib.rs:1262-1266
        if (!w.alive[b] || w.count[b] < 8) continue;
        body_list(w, b, lst, false);
        bool any = false;
        for (uint32_t k : lst) if ((uint32_t)(fr - w.sup[k]) < 10u) { any = true; break; }
        if (!any) for (uint32_t k : lst) { w.phi[k] = 0.0f; w.phi64[k] = 0.0; }
    }
    const float idt = 1.0f / maxf(dt, 1e-3f);   // src/lib.rs:1288-1304
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!w.alive[b]) continue;
        const V al = mul(sub(w.v[b], w.vlast[b]), idt), aa = mul(sub(w.w[b], w.wlast[b]), idt);
        w.vlast[b] = w.v[b]; w.wlast[b] = w.w[b];
        if (!body_loaded(w, b)) continue;
        const V pb = w.pos[b];
        float nm = 0.0f;
        body_list(w, b, lst, true);
        for (uint32_t k : lst) {
            const V a = add(al, cross(aa, sub(w.wpos[k], pb)));
            const V ge = vv(-a[0], -GR - a[1], -a[2]);
            const float n = minf(len(ge) / GR, 150.0f);
            if (n > nm) nm = n;
            w.ext[k] = MASS[w.mat[k]] * (n - 1.0f);
        }
        w.nmax[b] = nm;
    }
    int64_t budget = 160000;   // src/lib.rs:1305-1316
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!body_loaded(w, b) || w.count[b] > 60000) continue;
        if (w.bresid[b] < (double)2e-4f && w.nmax[b] < 1.5f && (fr + b) % 4 != 0) continue;
        const int64_t size = w.count[b];
        body_list(w, b, lst, true);
        uint32_t n = 0;
        for (;;) {
            const double r = rb64_sweep(w, lst, (double)1.8f);
            w.bresid[b] = r;
            n++; budget -= size;
            if (n >= 2 && (r < (double)4e-4f || n >= 60 || budget <= 0)) break;
        }
        for (uint32_t k : lst) w.phi[k] = (float)w.phi64[k];
        counts[0]++; counts[1] += n; counts[2] += n * (uint32_t)size;
    }
    float gm = 0.0f;   // src/lib.rs:1340-1360
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!body_loaded(w, b) || w.count[b] > 60000) continue;
        w.blt[b] += dt;
        const bool settled = w.bresid[b] < (double)2e-4f && w.nmax[b] < 1.5f;
        if (settled && (fr + b) % 4 != 0) continue;
        const float dtb = settled ? dt * 4.0f : dt;
        const bool live = (w.blt[b] > 0.3f && (w.bresid[b] < (double)1e-2f || w.blt[b] > 0.6f)) || w.nmax[b] > 2.5f;
        float bm = 0.0f;
        std::vector<Joint> out;
        body_list(w, b, lst, false);
        for (uint32_t k : lst) if (w.mat[k] != 0) { const float r = stress_brick(w, k, dtb, live, out); if (r > bm) bm = r; }
        w.maxr[b] = bm;
        if (bm > gm) gm = bm;
        for (const Joint& j : out) {
            counts[3]++;
            if (j.ratio > 1.0f) counts[4]++;
            if (j.decision == J_FAIL) counts[5]++;
            if (j.decision == J_CRUSH) counts[6]++;
        }
    }
    for (uint32_t b = 0; b < w.nbody; b++) if (w.alive[b] && !body_loaded(w, b)) w.blt[b] = maxf(w.blt[b] - 2.0f * dt, 0.0f);
    std::memcpy(&counts[7], &gm, 4);
    counts[8] = w.crush_n;
}

// st_now / st_top (src/lib.rs:1126-1128)
static void struct_tally(const World& w, int32_t s, uint32_t& now, int32_t& top) {
    now = 0; top = 0;
    for (uint32_t i = 0; i < w.ns; i++) if (w.in_struct(i, s)) { now++; top = std::max(top, w.by[i] + 1); }
}

// ---------------------------------------------------------------- rigid step (src/lib.rs:1367-1783)
static void update_cache(World& w) {
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!w.alive[b] || w.asleep[b]) continue;
        float* r = &w.rot[(size_t)b * 9];
        q_to_m(&w.q[(size_t)b * 4], r);
        float t1[9], t2[9];
        mmul(r, &w.iil[(size_t)b * 9], t1); mt(r, t2); mmul(t1, t2, &w.iiw[(size_t)b * 9]);
        V p = w.pos[b];
        uint32_t k = w.first[b];
        while (k != NONE) { w.wpos[k] = add(p, mv(r, w.local[k])); k = w.next[k]; }
    }
}
static void build_hash(World& w) {
    std::fill(w.hhead.begin(), w.hhead.end(), NONE);
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!w.alive[b]) continue;
        uint32_t k = w.first[b];
        while (k != NONE) {
            V p = w.wpos[k];
            uint32_t h = hkey_w((int)std::floor(p[0] / S), (int)std::floor(p[1] / S), (int)std::floor(p[2] / S));
            w.hnext[k] = w.hhead[h]; w.hhead[h] = k;
            k = w.next[k];
        }
    }
}
static void push_contact(World& w, uint32_t a, uint32_t b, uint32_t bo, uint32_t ba, uint32_t bb, V p, V n, float depth) {
    if (w.cs.size() >= MAXC_REF) w.would_drop++;
    Contact c;
    std::memset(&c, 0, sizeof c);
    c.a = a; c.b = b; c.bo = bo; c.ba = ba; c.bb = bb; c.p = p; c.n = n; c.depth = depth;
    w.cs.push_back(c);
    w.nc[a] += 1;
    if (b != STATIC) w.nc[b] += 1;
}
static void gen_contacts(World& w) {
    w.cs.clear();
    for (uint32_t b = 0; b < w.nbody; b++) w.nc[b] = 0;
    for (uint32_t a = 0; a < w.nbody; a++) {
        if (!w.alive[a] || w.asleep[a]) continue;
        const float* rot = &w.rot[(size_t)a * 9];
        float speed = len(w.v[a]) + len(w.w[a]) * w.rad[a] * 0.5f;
        uint32_t k = w.first[a];
        while (k != NONE) {
            uint32_t i = k;
            V p = w.wpos[i];
            if (p[1] < 0.5f) {
                for (int c = 0; c < 8; c++) {
                    V l = vv((c & 1) == 0 ? -H : H, (c & 2) == 0 ? -H : H, (c & 4) == 0 ? -H : H);
                    V cp = add(p, mv(rot, l));
                    if (cp[1] < 0.0f) { push_contact(w, a, STATIC, STATIC, i, NONE, cp, vv(0.0f, 1.0f, 0.0f), -cp[1]); w.sup[i] = w.frame; }
                }
            }
            int cx = (int)std::floor(p[0] / S) + NX / 2, cy = (int)std::floor(p[1] / S), cz = (int)std::floor(p[2] / S) + NZ / 2;
            for (int dz = -1; dz <= 1; dz++) for (int dy = -1; dy <= 1; dy++) for (int dx = -1; dx <= 1; dx++) {
                int x = cx + dx, y = cy + dy, z = cz + dz;
                uint32_t j = w.static_brick(x, y, z);
                if (j == NONE) continue;
                V c = lat_pos(x, y, z);
                V qq = vv(clampf(p[0], c[0] - H, c[0] + H), clampf(p[1], c[1] - H, c[1] + H), clampf(p[2], c[2] - H, c[2] + H));
                V d = sub(p, qq);
                float dist = len(d);
                if (dist >= RB) continue;
                if (dist > 1e-4f) {
                    if (d[1] > 0.3f * dist) w.sup[i] = w.frame;
                    push_contact(w, a, STATIC, STATIC, i, j, qq, mul(d, 1.0f / dist), RB - dist);
                } else {
                    V r = sub(p, c);
                    int ax = 0; for (int t = 1; t < 3; t++) if (fabs_(r[t]) > fabs_(r[ax])) ax = t;
                    V n = vv(0, 0, 0); n[ax] = r[ax] >= 0.0f ? 1.0f : -1.0f;
                    push_contact(w, a, STATIC, STATIC, i, j, p, n, H + RB - fabs_(r[ax]));
                }
            }
            int hx = (int)std::floor(p[0] / S), hy = (int)std::floor(p[1] / S), hz = (int)std::floor(p[2] / S);
            for (int dz = -1; dz <= 1; dz++) for (int dy = -1; dy <= 1; dy++) for (int dx = -1; dx <= 1; dx++) {
                uint32_t mm = w.hhead[hkey_w(hx + dx, hy + dy, hz + dz)];
                while (mm != NONE) {
                    uint32_t j = mm;
                    mm = w.hnext[j];
                    uint32_t bj = w.body[j];
                    if (bj == a || w.mat[j] == 0) continue;
                    bool other_awake = !w.asleep[bj];
                    if (other_awake && j < i) continue;
                    V d = sub(p, w.wpos[j]);
                    float dd = dot(d, d);
                    if (dd >= 4.0f * RB * RB || dd < 1e-10f) continue;
                    float dist = std::sqrt(dd);
                    V n = mul(d, 1.0f / dist);
                    V cp = madd(w.wpos[j], n, dist * 0.5f);
                    if (n[1] > 0.3f) w.sup[i] = w.frame; else if (n[1] < -0.3f) w.sup[j] = w.frame;
                    if (other_awake) push_contact(w, a, bj, bj, i, j, cp, n, 2.0f * RB - dist);
                    else {
                        if (speed > 0.7f) w.wake[bj] = 1;
                        push_contact(w, a, STATIC, bj, i, j, cp, n, 2.0f * RB - dist);
                    }
                }
            }
            k = w.next[i];
        }
    }
}
static inline V vel_at(const World& w, uint32_t b, V r) { if (b == STATIC) return vv(0, 0, 0); return add(w.v[b], cross(w.w[b], r)); }
static float eff_mass(const World& w, uint32_t a, uint32_t b, V ra, V rb, V n) {
    float k = w.im[a] + dot(n, cross(mv(&w.iiw[(size_t)a * 9], cross(ra, n)), ra));
    if (b != STATIC) k += w.im[b] + dot(n, cross(mv(&w.iiw[(size_t)b * 9], cross(rb, n)), rb));
    return k > 1e-12f ? 1.0f / k : 0.0f;
}
static void apply_imp(World& w, uint32_t a, uint32_t b, V ra, V rb, V p) {
    w.v[a] = madd(w.v[a], p, w.im[a]);
    V dw = mv(&w.iiw[(size_t)a * 9], cross(ra, p));
    w.w[a] = add(w.w[a], dw);
    if (b != STATIC) {
        w.v[b] = madd(w.v[b], p, -w.im[b]);
        V dw2 = mv(&w.iiw[(size_t)b * 9], cross(rb, p));
        w.w[b] = sub(w.w[b], dw2);
    }
}
// ---------------------------------------------------------------- contact reduction and warm start
// The GPU world's two devices for large contact sets (gpu/gpu_world.js:557-576, 834-920), restated for brick
// contacts and off by default. Warm start: a contact is known from the last substep by its key (its brick, the other
// side's kind and brick, and its place among the brick's contacts of that kind and brick); WARM_F of its normal
// impulse and of its friction impulse, projected on the new tangents and clamped to the cone, start the new solve and
// are applied once before the iterations. Reduction: a body pair with more than 32 contacts keeps, for each of the 26
// directions to a cube cell's neighbours, the contact whose point lies furthest along it, and the deepest (ties to
// the later contact); the others are neither coloured nor solved.
static World::WarmKey warm_key(const Contact& c, uint32_t ord) {
    const uint32_t kind = c.bb == NONE ? 0u : c.bo == STATIC ? 1u : c.b == STATIC ? 3u : 2u;
    return World::WarmKey{((uint64_t)c.ba << 32) | (uint64_t)c.bb, (kind << 16) | ord};
}
// keys of the list's contacts: a brick's contacts are contiguous, and ord counts the earlier ones with the same kind
// and other brick
static std::vector<World::WarmKey> warm_keys(const World& w) {
    std::vector<World::WarmKey> out(w.cs.size());
    for (size_t k = 0; k < w.cs.size(); k++) {
        const Contact& c = w.cs[k];
        const uint32_t kind = c.bb == NONE ? 0u : c.bo == STATIC ? 1u : c.b == STATIC ? 3u : 2u;
        uint32_t ord = 0;
        for (size_t q = k; q-- > 0 && w.cs[q].ba == c.ba;) {
            const Contact& e = w.cs[q];
            const uint32_t ek = e.bb == NONE ? 0u : e.bo == STATIC ? 1u : e.b == STATIC ? 3u : 2u;
            if (ek == kind && e.bb == c.bb) ord++;
        }
        out[k] = warm_key(c, ord);
    }
    return out;
}
static const uint32_t RED_K = 32, RED_D = 26;
// the share of the last substep's impulses a contact starts from: with the whole of them, the velocity bias that
// pushed a contact apart is carried too, and a stack of single bricks solved with 1 or 4 iterations toppled; at 0.8
// it stands, sinking less than from zero (0.022 m against 0.046 m at 1 iteration, 0.012 against 0.017 at 4)
static const float WARM_F = 0.8f;
static inline uint32_t f2o(float x) { uint32_t b; std::memcpy(&b, &x, 4); return (b & 0x80000000u) ? ~b : (b | 0x80000000u); }
// slot k < 26: the point's reach along the k-th direction to a cube cell's neighbours; slot 26: the depth
static inline float red_score(const Contact& c, uint32_t k) {
    if (k == RED_D) return c.depth;
    const uint32_t j = k >= 13 ? k + 1 : k;
    const float dx = (float)(j % 3) - 1.0f, dy = (float)((j / 3) % 3) - 1.0f, dz = (float)(j / 9) - 1.0f;
    return c.p[0] * dx + c.p[1] * dy + c.p[2] * dz;
}
static inline void warm_apply(World& w, const Contact& c) {
    apply_imp(w, c.a, c.b, c.ra, c.rb, add(mul(c.n, c.jn), add(mul(c.t1, c.jt1), mul(c.t2, c.jt2))));
}
static void warm_store(World& w) {
    const std::vector<World::WarmKey> keys = warm_keys(w);
    w.warm_tab.clear();
    for (size_t k = 0; k < w.cs.size(); k++) {
        const Contact& c = w.cs[k];
        if (c.off) continue;
        w.warm_tab[keys[k]] = World::WarmVal{c.jn, add(mul(c.t1, c.jt1), mul(c.t2, c.jt2))};
    }
    w.warm_valid = true;
}

static void prep_contacts(World& w, float h) {
    std::vector<World::WarmKey> keys;
    const bool look = w.warm && w.warm_valid;
    if (look) keys = warm_keys(w);
    size_t ci = 0;
    for (Contact& c : w.cs) {
        uint32_t a = c.a;
        c.ra = sub(c.p, w.pos[a]);
        c.rb = c.b != STATIC ? sub(c.p, w.pos[c.b]) : vv(0, 0, 0);
        c.mn = eff_mass(w, a, c.b, c.ra, c.rb, c.n);
        V dv = sub(vel_at(w, c.a, c.ra), vel_at(w, c.b, c.rb));
        float vn = dot(dv, c.n);
        c.vn0 = maxf(-vn, 0.0f);
        V vt = sub(dv, mul(c.n, vn));
        float lt = len(vt);
        if (lt > 1e-4f) c.t1 = mul(vt, 1.0f / lt);
        else {
            V t = fabs_(c.n[0]) < 0.9f ? vv(1, 0, 0) : vv(0, 1, 0);
            V x = cross(c.n, t); c.t1 = mul(x, 1.0f / len(x));
        }
        c.t2 = cross(c.n, c.t1);
        c.mt1 = eff_mass(w, a, c.b, c.ra, c.rb, c.t1);
        c.mt2 = eff_mass(w, a, c.b, c.ra, c.rb, c.t2);
        float bias = minf(0.2f / h * maxf(c.depth - 0.01f, 0.0f), 1.0f);
        if (vn < -2.0f) bias = maxf(bias, -0.12f * vn);
        c.bias = bias;
        if (look) {
            auto it = w.warm_tab.find(keys[ci]);
            if (it != w.warm_tab.end()) {
                const float jn = it->second.jn * WARM_F, lim = MU * jn;
                c.jn = jn;
                c.jt1 = clampf(dot(it->second.f, c.t1) * WARM_F, -lim, lim);
                c.jt2 = clampf(dot(it->second.f, c.t2) * WARM_F, -lim, lim);
            }
        }
        ci++;
    }
}
static inline void solve_contact(World& w, Contact& c) {
    uint32_t a = c.a;
    V dv = sub(vel_at(w, c.a, c.ra), vel_at(w, c.b, c.rb));
    float vn = dot(dv, c.n);
    float lam = c.mn * (-vn + c.bias);
    float old = c.jn;
    c.jn = maxf(old + lam, 0.0f);
    float d = c.jn - old;
    apply_imp(w, a, c.b, c.ra, c.rb, mul(c.n, d));
    float lim = MU * c.jn;
    dv = sub(vel_at(w, c.a, c.ra), vel_at(w, c.b, c.rb));
    float l1 = -c.mt1 * dot(dv, c.t1);
    float o1 = c.jt1; c.jt1 = clampf(o1 + l1, -lim, lim);
    float l2 = -c.mt2 * dot(dv, c.t2);
    float o2 = c.jt2; c.jt2 = clampf(o2 + l2, -lim, lim);
    V p = add(mul(c.t1, c.jt1 - o1), mul(c.t2, c.jt2 - o2));
    apply_imp(w, a, c.b, c.ra, c.rb, p);
}

// Manifolds: contacts grouped by (a, b) in list order, sorted by key (a, b') with b' = 0 for the static side.
// Colours: greedy in decreasing priority (ties: lower manifold index first), smallest colour free at both bodies;
// this is the colouring Jones-Plassmann rounds produce with the same priorities.
static void build_manifolds(World& w) {
    size_t n = w.cs.size();
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    auto key = [&](uint32_t k) -> uint64_t {
        const Contact& c = w.cs[k];
        uint64_t bp = c.b == STATIC ? 0 : (uint64_t)c.b + 1;
        return ((uint64_t)c.a << 32) | bp;
    };
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
    // contacts plough switched off take no part
    idx.erase(std::remove_if(idx.begin(), idx.end(), [&](uint32_t k) { return w.cs[k].off != 0; }), idx.end());
    n = idx.size();
    if (w.reduce) {
        std::vector<uint32_t> kept;
        kept.reserve(n);
        for (size_t s0 = 0; s0 < n;) {
            size_t e = s0 + 1;
            while (e < n && key(idx[e]) == key(idx[s0])) e++;
            if (e - s0 > RED_K) {
                uint32_t best[RED_D + 1], win[RED_D + 1];
                for (uint32_t k = 0; k <= RED_D; k++) { best[k] = 0; win[k] = 0; }
                for (size_t t = s0; t < e; t++)
                    for (uint32_t k = 0; k <= RED_D; k++) best[k] = std::max(best[k], f2o(red_score(w.cs[idx[t]], k)));
                for (size_t t = s0; t < e; t++)
                    for (uint32_t k = 0; k <= RED_D; k++)
                        if (f2o(red_score(w.cs[idx[t]], k)) == best[k]) win[k] = std::max(win[k], idx[t] + 1);
                for (size_t t = s0; t < e; t++) {
                    bool keep = false;
                    for (uint32_t k = 0; k <= RED_D; k++) keep = keep || win[k] == idx[t] + 1;
                    Contact& c = w.cs[idx[t]];
                    if (keep) kept.push_back(idx[t]);
                    else { c.off = 1; c.jn = 0.0f; c.jt1 = 0.0f; c.jt2 = 0.0f; }
                }
            } else {
                for (size_t t = s0; t < e; t++) kept.push_back(idx[t]);
            }
            s0 = e;
        }
        idx.swap(kept);
        n = idx.size();
    }
    w.man_a.clear(); w.man_b.clear(); w.man_start.clear(); w.man_count.clear(); w.man_contacts = idx;
    // a pair's contacts form chunks of at most K (K = 0: one chunk); the colouring and the solve see chunks
    std::vector<uint32_t> prio;
    size_t pair_start = 0;
    for (size_t t = 0; t < n; t++) {
        bool new_pair = t == 0 || key(idx[t]) != key(idx[t - 1]);
        if (new_pair) pair_start = t;
        uint32_t j = w.chunk ? (uint32_t)((t - pair_start) / w.chunk) : 0u;
        bool new_chunk = new_pair || (w.chunk && (t - pair_start) % w.chunk == 0);
        if (new_chunk) {
            const Contact& c = w.cs[idx[t]];
            w.man_a.push_back(c.a); w.man_b.push_back(c.b); w.man_start.push_back((uint32_t)t); w.man_count.push_back(0);
            uint32_t h = pair_priority(c.a, c.b == STATIC ? 0u : c.b + 1);
            prio.push_back(j ? pair_priority(h, j) : h);
        }
        w.man_count.back()++;
    }
    size_t nm = w.man_a.size();
    std::vector<uint32_t> order(nm);
    std::iota(order.begin(), order.end(), 0u);
    std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return prio[x] != prio[y] ? prio[x] > prio[y] : x < y; });
    // per body the colours its manifolds hold (grown as needed: a body resting on thousands of contacts holds many)
    std::vector<std::vector<uint64_t>> used(w.nbody, std::vector<uint64_t>(4, 0));
    auto held = [&](uint32_t x, uint32_t c) { return (c >> 6) < used[x].size() && ((used[x][c >> 6] >> (c & 63)) & 1); };
    auto hold = [&](uint32_t x, uint32_t c) {
        if ((c >> 6) >= used[x].size()) used[x].resize((c >> 6) + 1, 0);
        used[x][c >> 6] |= 1ull << (c & 63);
    };
    w.man_color.assign(nm, 0);
    w.ncolors = 0;
    for (uint32_t mi : order) {
        uint32_t a = w.man_a[mi], b = w.man_b[mi];
        uint32_t c = 0;
        for (;; c++) {
            bool busy = held(a, c);
            if (b != STATIC) busy = busy || held(b, c);
            if (!busy) break;
        }
        w.man_color[mi] = c;
        hold(a, c);
        if (b != STATIC) hold(b, c);
        if (c + 1 > w.ncolors) w.ncolors = c + 1;
    }
}
static void solve_list(World& w) { for (Contact& c : w.cs) if (!c.off) solve_contact(w, c); }
static void solve_colored(World& w) {
    // manifolds of one colour share no awake body, so their order inside a colour does not change the result
    std::vector<std::vector<uint32_t>> bycol(w.ncolors);
    for (size_t m = 0; m < w.man_a.size(); m++) bycol[w.man_color[m]].push_back((uint32_t)m);
    for (auto& lst : bycol)
        for (uint32_t m : lst)
            for (uint32_t t = 0; t < w.man_count[m]; t++) solve_contact(w, w.cs[w.man_contacts[w.man_start[m] + t]]);
}

// islands over manifolds between two awake bodies; label = smallest body id of the island (root = min id)
static void islands(World& w) {
    std::vector<uint32_t> par(w.nbody);
    std::iota(par.begin(), par.end(), 0u);
    auto find = [&](uint32_t x) { while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; } return x; };
    for (size_t m = 0; m < w.man_a.size(); m++) {
        uint32_t b = w.man_b[m];
        if (b == STATIC) continue;
        uint32_t x = find(w.man_a[m]), y = find(b);
        if (x == y) continue;
        if (x < y) std::swap(x, y);
        par[x] = y;
    }
    w.island.assign(w.nbody, NONE);
    for (uint32_t b = 0; b < w.nbody; b++) if (w.alive[b] && !w.asleep[b]) w.island[b] = find(b);
}

static void pinch_check(World& w, bool kill) {
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!w.alive[b] || w.asleep[b]) continue;
        V dw = sub(w.w[b], w.wpre[b]);
        float tip = len(dw) * w.rad[b];
        if (tip > 6.0f) w.w[b] = madd(w.wpre[b], dw, 6.0f / tip);
        V dv = sub(w.v[b], w.vpre[b]);
        float mm = len(dv);
        if (mm < 8.0f) continue;
        uint32_t f = w.first[b];
        if (f == NONE || w.mat[f] >= SLUG) continue;
        if (kill && w.count[b] <= 6) kill_body(w, b);
        else w.v[b] = madd(w.vpre[b], dv, 8.0f / mm);
    }
}
static void integrate(World& w, float h, int sleep_mode) {
    std::vector<uint8_t> rest(w.nbody, 0);
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (!w.alive[b] || w.asleep[b]) continue;
        clamp_vel(w, b);
        w.pos[b] = madd(w.pos[b], w.v[b], h);
        q_int(&w.q[(size_t)b * 4], w.w[b], h);
        w.v[b] = mul(w.v[b], 1.0f - 0.01f * h);
        w.w[b] = mul(w.w[b], 1.0f - 0.05f * h);
        bool small = w.count[b] <= 3;
        if (w.nc[b] > 0 && small) {
            w.w[b] = mul(w.w[b], 1.0f - minf(7.0f * h, 0.5f));
            w.v[b] = mul(w.v[b], 1.0f - minf(2.0f * h, 0.3f));
        }
        float v2 = dot(w.v[b], w.v[b]);
        float rr = w.rad[b];
        float w2 = dot(w.w[b], w.w[b]) * rr * rr;
        float vt = small ? 0.16f : 0.06f, wt = small ? 0.3f : 0.04f;
        if (v2 < vt && w2 < wt && w.nc[b] > 0 && w.maxr[b] < 0.95f) {
            w.sleep[b] += h;
            if (sleep_mode == SLEEP_BODY && w.sleep[b] > 0.45f) { w.asleep[b] = 1; w.v[b] = vv(0, 0, 0); w.w[b] = vv(0, 0, 0); }
        } else w.sleep[b] = 0.0f;
        V p = w.pos[b];
        if (p[1] < -15.0f || fabs_(p[0]) > 190.0f || fabs_(p[2]) > 190.0f || p[1] > 120.0f) kill_body(w, b);
    }
    if (sleep_mode == SLEEP_ISLAND) {
        // an island sleeps when its least-rested body has rested past the threshold, a body alone at twice it
        std::vector<float> mint(w.nbody, 3.4e38f);
        for (uint32_t b = 0; b < w.nbody; b++) {
            uint32_t r = w.island[b];
            if (r == NONE || !w.alive[b]) continue;
            if (w.sleep[b] < mint[r]) mint[r] = w.sleep[b];
        }
        for (uint32_t b = 0; b < w.nbody; b++) {
            uint32_t r = w.island[b];
            if (r == NONE || !w.alive[b] || w.asleep[b]) continue;
            if (mint[r] > 0.45f || w.sleep[b] > 0.9f) { w.asleep[b] = 1; w.v[b] = vv(0, 0, 0); w.w[b] = vv(0, 0, 0); }
        }
    }
    for (uint32_t b = 0; b < w.nbody; b++) {
        if (w.wake[b]) { w.wake[b] = 0; if (w.alive[b]) { w.asleep[b] = 0; w.sleep[b] = 0.0f; } }
    }
}
// ---------------------------------------------------------------- damage on contact (src/lib.rs:1602-1702)
static void st_hit(World& w, int32_t s) { if (s >= 0 && s < (int32_t)w.st_hit.size()) w.st_hit[s] = 1; }
static V bpos(const World& w, uint32_t i) { return w.body[i] == STATIC ? lat_pos(w.bx[i], w.by[i], w.bz[i]) : w.wpos[i]; }
// damage_brick (src/lib.rs:724-745)
static uint32_t damage_brick(World& w, uint32_t i, float frac, float absolute) {
    uint32_t broke = 0;
    for (int d = 0; d < 6; d++) {
        const uint32_t j = w.nb6[(size_t)i * 6 + d];
        if (j == NONE || w.mat[j] == 0) continue;
        const uint32_t o = (d & 1) == 0 ? i : j;
        const int a = d >> 1;
        float& b = w.bond[(size_t)o * 4 + a];
        if (b > 0.0f) {
            b -= w.bmax[(size_t)o * 4 + a] * frac + absolute;
            if (b <= w.bmax[(size_t)o * 4 + a] * 0.03f) { b = 0.0f; broke++; }
        }
    }
    float& b3 = w.bond[(size_t)i * 4 + 3];
    if (b3 > 0.0f) {
        b3 -= w.bmax[(size_t)i * 4 + 3] * frac * 0.5f + absolute * 0.5f;
        if (b3 <= 0.0f) { b3 = 0.0f; broke++; }
    }
    if (w.body[i] == STATIC) { st_hit(w, w.sid[i]); if (broke > 0) flag_conn(w, w.sid[i]); }
    else if (broke > 0) w.dirty[w.body[i]] = 1;
    return broke;
}
// sever_brick (src/lib.rs:746-752)
static void sever_brick(World& w, uint32_t i) {
    for (int a = 0; a < 4; a++) w.bond[(size_t)i * 4 + a] = 0.0f;
    for (int d = 1; d < 6; d += 2) {
        const uint32_t j = w.nb6[(size_t)i * 6 + d];
        if (j != NONE) w.bond[(size_t)j * 4 + (d >> 1)] = 0.0f;
    }
}
static float h01(uint32_t h, uint32_t k);
// rndv (src/lib.rs:330-336) on the draw sequence: three draws in (-1, 1) until their length is in (0.1, 1], then
// unit length
static V rndv_draw(World& w) {
    for (;;) {
        const float x = h01(0x243F6A88u, w.dmg_draws++) * 2.0f - 1.0f;
        const float y = h01(0x243F6A88u, w.dmg_draws++) * 2.0f - 1.0f;
        const float z = h01(0x243F6A88u, w.dmg_draws++) * 2.0f - 1.0f;
        const V v = vv(x, y, z);
        const float l = dot(v, v);
        if (l > 0.01f && l <= 1.0f) return mul(v, 1.0f / std::sqrt(l));
    }
}
// plough (src/lib.rs:1493-1550), after the contacts and before prep_contacts: a body driving into a static brick at
// 2 m/s or more with momentum of at least 0.35 of the brick's vertical capacity damages it (a body of more than 40
// bricks: damage_brick by mom / 1.5 CAPV, within 0.15..0.9) or knocks it loose as a one-brick body (severed, with
// 0.75 of the body's velocity plus 2 m/s and a spin of 6 rad/s in random directions; the body keeps m / (m + 1.5
// MASS) of its velocity); the contact and the later contacts with that brick are switched off. The random
// directions come from the damage draw sequence.
static void plough(World& w) {
    for (size_t k = 0; k < w.cs.size(); k++) {
        Contact& c = w.cs[k];
        if (c.b != STATIC || c.bb == NONE || c.bo != STATIC) continue;
        const uint32_t j = c.bb;
        if (w.mat[j] == 0 || w.body[j] != STATIC) { c.off = 1; continue; }
        const uint32_t a = c.a;
        const V ra = sub(c.p, w.pos[a]);
        const float vn = -dot(vel_at(w, a, ra), c.n);
        if (vn < 2.0f) continue;
        const float meff = w.m[a] * 3.0f / maxf((float)w.nc[a], 3.0f);
        const float mom = minf(meff, w.m[a]) * vn;
        const uint8_t mj = w.mat[j];
        if (mj >= SLUG || mom < CAPV[mj] * 0.35f) continue;
        if (w.count[a] > 40) {
            damage_brick(w, j, clampf(mom / (CAPV[mj] * 1.5f), 0.15f, 0.9f), 0.0f);
            w.dmg[6]++;
            continue;
        }
        if (w.nbody + 1 > w.cap_bodies || w.nd + 1 > w.cap_bricks) continue;   // ensure_bodies
        sever_brick(w, j);
        flag_conn(w, w.sid[j]);
        st_hit(w, w.sid[j]);
        const V rv = rndv_draw(w);
        const V pv = madd(mul(w.v[a], 0.75f), rv, 2.0f);
        const V ww = mul(rndv_draw(w), 6.0f);
        const uint32_t b = body_from_statics(w, std::vector<uint32_t>{j}, pv);
        w.w[b] = ww;
        const float m = w.m[a];
        w.v[a] = mul(w.v[a], m / (m + MASS[mj] * 1.5f));
        w.dmg[5]++;
        c.off = 1;
        for (size_t t = k + 1; t < w.cs.size(); t++) {
            Contact& e = w.cs[t];
            if (e.bb == j && e.bo == STATIC && e.b == STATIC) e.off = 1;
        }
    }
}
// crush_at (src/lib.rs:1641-1702); the pulverisation draw is h01 of a fixed seed and the world's draw count
static uint32_t crush_at(World& w, uint32_t start, float e, V p, uint32_t cap) {
    const uint8_t m0 = w.mat[start];
    if (m0 == 0 || m0 >= SLUG) return 0;
    if (e < EB[m0] * 0.15f) return 0;
    const uint32_t body = w.body[start];
    const int32_t sid = w.sid[start];
    if (w.stamp.size() < w.mat.size()) w.stamp.resize(w.mat.size(), 0);
    const uint32_t st = ++w.stamp_id;
    std::vector<uint32_t> q{start};
    w.stamp[start] = st;
    size_t head = 0;
    uint32_t crushed = 0;
    const uint32_t maxn = std::min(cap, 600u);
    std::vector<uint32_t> lst;
    while (head < q.size() && crushed < maxn) {
        size_t best = head;
        float bd = 1e18f;
        const size_t lim = std::min(head + 24, q.size());
        for (size_t t = head; t < lim; t++) { V d = sub(bpos(w, q[t]), p); float dd = dot(d, d); if (dd < bd) { bd = dd; best = t; } }
        std::swap(q[head], q[best]);
        const uint32_t i = q[head]; head++;
        const uint8_t m = w.mat[i];
        if (m == 0) continue;
        const float cost = EB[m];
        if (e < cost) { damage_brick(w, i, 0.6f * e / cost, 0.0f); w.dmg[4]++; break; }
        e -= cost;
        lst.push_back(i);
        crushed++;
        for (int d = 0; d < 6; d++) {
            uint32_t j; float hp;
            if (!w.linked(i, d, j, hp) || w.stamp[j] == st || w.body[j] != body || w.sid[j] != sid) continue;
            w.stamp[j] = st;
            q.push_back(j);
        }
    }
    for (uint32_t i : lst) {
        const uint8_t m = w.mat[i];
        if (m == 0) continue;
        if (h01(0x243F6A88u, w.dmg_draws++) < PULV[m]) {
            if (w.body[i] == STATIC) st_hit(w, w.sid[i]);   // remove_brick's st_static_change (src/lib.rs:713)
            remove_brick(w, i);
            w.dmg[2]++;
        }
        else {
            sever_brick(w, i);
            w.dmg[3]++;
            if (body == STATIC) { flag_conn(w, w.sid[i]); st_hit(w, w.sid[i]); }
            else w.dirty[body] = 1;
        }
    }
    w.dmg[1] += crushed;
    return crushed;
}
// impact_damage (src/lib.rs:1610-1640), one budget of 2,500 crushed bricks per substep
static void impact_damage(World& w) {
    uint32_t budget = 2500;
    for (const Contact& c : w.cs) {
        if (c.off) continue;   // switched off by plough or left out by the reduction
        const uint32_t ia = c.ba;
        const uint8_t ma = w.mat[ia];
        if (ma == 0 || ma >= SLUG) continue;
        const bool crush = c.vn0 >= 1.0f && 0.5f * c.jn * c.vn0 >= 150.0f;
        const bool heavy = c.bb != NONE && c.bo == STATIC && c.jn * c.vn0 > 4000.0f;
        if (crush || heavy) w.dmg[0]++;
        if (heavy) { const uint32_t j = c.bb; if (w.mat[j] != 0 && w.body[j] == STATIC) st_hit(w, w.sid[j]); }
        if (w.mat[ia] == 0) continue;
        if (c.vn0 < 1.0f) continue;
        const float e = 0.5f * c.jn * c.vn0;
        if (e < 150.0f) continue;
        const uint32_t jb = c.bb;
        const uint8_t mb = jb != NONE ? w.mat[jb] : 0;
        const float soft_a = 1.0f / EB[ma];
        const float soft_b = (jb == NONE || mb == 0 || mb >= SLUG) ? 0.0f : 1.0f / EB[mb];
        if (soft_a + soft_b <= 0.0f) continue;
        const float ea = e * soft_a / (soft_a + soft_b);
        if (ea > 0.0f && budget > 0) budget -= std::min(crush_at(w, ia, ea, c.p, budget), budget);
        if (soft_b > 0.0f && budget > 0) budget -= std::min(crush_at(w, jb, e - ea, c.p, budget), budget);
    }
}

static void substep(World& w, float h, const StepParams& P) {
    w.reduce = P.reduce; w.warm = P.warm;
    if (!P.warm) w.warm_valid = false;
    update_cache(w);
    for (uint32_t b = 0; b < w.nbody; b++) if (w.alive[b] && !w.asleep[b]) w.v[b][1] -= GR * h;
    build_hash(w);
    gen_contacts(w);
    if (P.damage) plough(w);
    prep_contacts(w, h);
    for (uint32_t b = 0; b < w.nbody; b++) if (w.alive[b]) { w.vpre[b] = w.v[b]; w.wpre[b] = w.w[b]; }
    build_manifolds(w);
    islands(w);
    if (P.warm && P.iterations) {   // the carried impulses, once, in the solve's order
        if (P.order == ORDER_COLOR) {
            std::vector<std::vector<uint32_t>> bycol(w.ncolors);
            for (size_t m = 0; m < w.man_a.size(); m++) bycol[w.man_color[m]].push_back((uint32_t)m);
            for (auto& lst : bycol)
                for (uint32_t m : lst)
                    for (uint32_t t = 0; t < w.man_count[m]; t++) warm_apply(w, w.cs[w.man_contacts[w.man_start[m] + t]]);
        } else {
            for (const Contact& c : w.cs) if (!c.off) warm_apply(w, c);
        }
    }
    for (uint32_t it = 0; it < P.iterations; it++) {
        if (P.order == ORDER_COLOR) solve_colored(w); else solve_list(w);
    }
    if (P.warm) warm_store(w);
    pinch_check(w, P.pinch_kill != 0);
    if (P.damage) impact_damage(w);
    integrate(w, h, (int)P.sleep_mode);
}
static void step(World& w, float dt, const StepParams& P) {
    dt = clampf(dt, 0.0f, 1.0f / 30.0f);
    w.frame += 1;
    uint32_t ns = P.substeps ? P.substeps : 2;
    float h = ns == 2 ? dt * 0.5f : dt / (float)ns;
    for (uint32_t s = 0; s < ns; s++) substep(w, h, P);
}

// ---------------------------------------------------------------- box SAT (engine/src/phys.rs:502-628)
struct P3 { float x, y, z; };
static inline P3 p3(float a, float b, float c) { return P3{a, b, c}; }
static inline P3 operator+(P3 a, P3 b) { return p3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline P3 operator-(P3 a, P3 b) { return p3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline P3 operator*(P3 a, float s) { return p3(a.x * s, a.y * s, a.z * s); }
static inline P3 operator-(P3 a) { return p3(-a.x, -a.y, -a.z); }
static inline float pdot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline P3 pcross(P3 a, P3 b) { return p3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float plen2(P3 a) { return pdot(a, a); }
static inline float pget(P3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline float sqrt_e(float x) { return x <= 0.0f ? 0.0f : std::sqrt(x); }  // engine/src/math.rs:87-90
struct M3 { P3 c[3]; };
static M3 quat_m3(const float* q) {  // engine/src/math.rs:60-66 (columns)
    float x = q[0], y = q[1], z = q[2], w = q[3];
    M3 m;
    m.c[0] = p3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w));
    m.c[1] = p3(2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w));
    m.c[2] = p3(2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y));
    return m;
}
struct CP { P3 p; float s; };

static int reduce4(CP* pts, int cnt, P3 n) {
    if (cnt <= 4) return cnt;
    int i0 = 0; for (int k = 1; k < cnt; k++) if (pts[k].s < pts[i0].s) i0 = k;
    P3 q0 = pts[i0].p;
    int i1 = 0; float best = -1.0f;
    for (int k = 0; k < cnt; k++) { float d = plen2(pts[k].p - q0); if (d > best) { best = d; i1 = k; } }
    P3 q1 = pts[i1].p;
    P3 e = q1 - q0;
    int i2 = 0; float b2 = -3.4028235e38f;
    for (int k = 0; k < cnt; k++) { float a = pdot(pcross(pts[k].p - q0, e), n); if (a > b2) { b2 = a; i2 = k; } }
    int i3 = 0; float b3 = -3.4028235e38f;
    for (int k = 0; k < cnt; k++) { float a = -pdot(pcross(pts[k].p - q0, e), n); if (a > b3) { b3 = a; i3 = k; } }
    int ids[4] = {i0, i1, i2, i3};
    CP sel[4] = {pts[i0], pts[i1], pts[i2], pts[i3]};
    int out = 0;
    for (int k = 0; k < 4; k++) {
        bool dup = false;
        for (int t = 0; t < k; t++) if (ids[t] == ids[k]) dup = true;
        if (dup) continue;
        pts[out++] = sel[k];
    }
    return out;
}

// returns the point count (0 = separated); normal from A to B
static int collide_boxes(P3 pa, const M3& ra, P3 ha, P3 pb, const M3& rb, P3 hb, float margin, CP* out, P3* nout) {
    P3 t = pb - pa;
    float ac[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) ac[i][j] = fabs_(pdot(ra.c[i], rb.c[j])) + 1e-6f;
    float hav[3] = {ha.x, ha.y, ha.z}, hbv[3] = {hb.x, hb.y, hb.z};
    float sa = -3.4028235e38f; int ia = 0;
    for (int i = 0; i < 3; i++) {
        float s = fabs_(pdot(t, ra.c[i])) - (hav[i] + hbv[0] * ac[i][0] + hbv[1] * ac[i][1] + hbv[2] * ac[i][2]);
        if (s > margin) return 0;
        if (s > sa) { sa = s; ia = i; }
    }
    float sbm = -3.4028235e38f; int jb = 0;
    for (int j = 0; j < 3; j++) {
        float s = fabs_(pdot(t, rb.c[j])) - (hbv[j] + hav[0] * ac[0][j] + hav[1] * ac[1][j] + hav[2] * ac[2][j]);
        if (s > margin) return 0;
        if (s > sbm) { sbm = s; jb = j; }
    }
    float se = -3.4028235e38f; int ei = 0, ej = 0; P3 el = p3(0, 0, 0);
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
        P3 l = pcross(ra.c[i], rb.c[j]);
        float l2 = plen2(l);
        if (l2 < 1e-8f) continue;
        l = l * (1.0f / sqrt_e(l2));
        float r = hav[0] * fabs_(pdot(ra.c[0], l)) + hav[1] * fabs_(pdot(ra.c[1], l)) + hav[2] * fabs_(pdot(ra.c[2], l))
                + hbv[0] * fabs_(pdot(rb.c[0], l)) + hbv[1] * fabs_(pdot(rb.c[1], l)) + hbv[2] * fabs_(pdot(rb.c[2], l));
        float s = fabs_(pdot(t, l)) - r;
        if (s > margin) return 0;
        if (s > se) { se = s; ei = i; ej = j; el = l; }
    }
    const float face_tol = 0.005f;
    bool use_b = sbm > sa + face_tol;
    float face_best = use_b ? sbm : sa;
    if (se > face_best + 0.01f) {
        P3 n = pdot(t, el) < 0.0f ? -el : el;
        P3 ca = pa, cb = pb;
        for (int k = 0; k < 3; k++) {
            if (k != ei) { float s = pdot(ra.c[k], n) > 0.0f ? 1.0f : -1.0f; ca = ca + ra.c[k] * (s * hav[k]); }
            if (k != ej) { float s = pdot(rb.c[k], n) > 0.0f ? -1.0f : 1.0f; cb = cb + rb.c[k] * (s * hbv[k]); }
        }
        P3 d1 = ra.c[ei], d2 = rb.c[ej];
        P3 r = ca - cb;
        float bb = pdot(d1, d2), c = pdot(d1, r), f = pdot(d2, r);
        float den = 1.0f - bb * bb;
        float s = den > 1e-6f ? (bb * f - c) / den : 0.0f;
        s = std::fmin(std::fmax(s, -hav[ei]), hav[ei]);
        float tt = bb * s + f;
        tt = std::fmin(std::fmax(tt, -hbv[ej]), hbv[ej]);
        s = std::fmin(std::fmax(bb * tt - c, -hav[ei]), hav[ei]);
        P3 q1 = ca + d1 * s, q2 = cb + d2 * tt;
        float sep = pdot(q2 - q1, n);
        out[0].p = (q1 + q2) * 0.5f; out[0].s = sep;
        *nout = n;
        return 1;
    }
    P3 pr, pi; const M3 *rr, *ri; const float *hr, *hi; int k; bool flip;
    if (use_b) { pr = pb; rr = &rb; hr = hbv; pi = pa; ri = &ra; hi = hav; k = jb; flip = true; }
    else { pr = pa; rr = &ra; hr = hav; pi = pb; ri = &rb; hi = hbv; k = ia; flip = false; }
    P3 n = rr->c[k];
    if (pdot(pi - pr, n) < 0.0f) n = -n;
    int j = 0; float bd = -1.0f;
    for (int qq = 0; qq < 3; qq++) { float d = fabs_(pdot(ri->c[qq], n)); if (d > bd) { bd = d; j = qq; } }
    float sgn = pdot(ri->c[j], n) > 0.0f ? -1.0f : 1.0f;
    P3 fc = pi + ri->c[j] * (sgn * hi[j]);
    int u = (j + 1) % 3, vq = (j + 2) % 3;
    P3 eu = ri->c[u] * hi[u], ev = ri->c[vq] * hi[vq];
    P3 poly[8], tmp[8];
    poly[0] = fc + eu + ev; poly[1] = fc - eu + ev; poly[2] = fc - eu - ev; poly[3] = fc + eu - ev;
    int pn = 4;
    int u2 = (k + 1) % 3, v2 = (k + 2) % 3;
    const int axs[4] = {u2, u2, v2, v2};
    const float sg[4] = {1.0f, -1.0f, 1.0f, -1.0f};
    for (int e = 0; e < 4; e++) {
        P3 dir = rr->c[axs[e]] * sg[e];
        float off = pdot(dir, pr) + hr[axs[e]];
        int tn = 0;
        for (int qq = 0; qq < pn; qq++) {
            P3 p0 = poly[qq], p1 = poly[(qq + 1) % pn];
            float d0 = pdot(p0, dir) - off, d1 = pdot(p1, dir) - off;
            if (d0 <= 0.0f) { if (tn < 8) { tmp[tn++] = p0; } }
            if ((d0 <= 0.0f) != (d1 <= 0.0f)) { float ttt = d0 / (d0 - d1); if (tn < 8) { tmp[tn++] = p0 + (p1 - p0) * ttt; } }
        }
        pn = tn;
        for (int qq = 0; qq < pn; qq++) poly[qq] = tmp[qq];
        if (pn == 0) return 0;
    }
    P3 rc = pr + n * hr[k];
    int cnt = 0;
    for (int qq = 0; qq < pn; qq++) {
        P3 p = poly[qq];
        float sep = pdot(p - rc, n);
        if (sep <= margin) { out[cnt].p = p - n * (0.5f * sep); out[cnt].s = sep; cnt++; }
    }
    if (cnt == 0) return 0;
    *nout = flip ? -n : n;
    return cnt;
}


// ---------------------------------------------------------------- convex-cell SAT (gpu/gpu_world.js:400-555)
// Hull data: 80 float4 per hull (see shatterforge_b200/hulls.py). A shape is a cell in its box: p, rotation, half
// extents h, hull id. Vector operations keep one fixed order (R*v = c0*v.x + c1*v.y + c2*v.z, normalize = v / |v|).
struct HullShape { P3 p; M3 R; P3 h; const float* H; };
static inline P3 hv4(const float* H, int k) { return p3(H[4 * k], H[4 * k + 1], H[4 * k + 2]); }
static inline P3 rmul(const M3& R, P3 v) { return R.c[0] * v.x + R.c[1] * v.y + R.c[2] * v.z; }
static inline P3 cmul(P3 a, P3 b) { return p3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline P3 cdiv(P3 a, P3 b) { return p3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline float plen(P3 a) { return std::sqrt(pdot(a, a)); }
static inline P3 pnorm(P3 a) { float l = plen(a); return p3(a.x / l, a.y / l, a.z / l); }
static inline int hnv(const float* H) { return (int)H[0]; }
static inline int hnf(const float* H) { return (int)H[1]; }
static inline int hns(const float* H) { return (int)H[2]; }
static inline int hnd(const float* H) { return (int)H[3]; }
static inline P3 hvert(const float* H, int k) { return hv4(H, 1 + k); }
static inline int hfidx(const float* H, int f, int i) { return (int)H[4 * (29 + 2 * f + i / 4) + (i % 4)]; }
static inline int hfcnt(const float* H, int f) { return (int)H[4 * (77 + f / 4) + (f % 4)]; }
static inline void hseg(const float* H, int k, int& a, int& b) { const float* v = H + 4 * (53 + k / 2); if (k & 1) { a = (int)v[2]; b = (int)v[3]; } else { a = (int)v[0]; b = (int)v[1]; } }
static inline P3 hdir(const float* H, int k) { return hv4(H, 65 + k); }
static inline P3 hw(const HullShape& s, int k) { return s.p + rmul(s.R, cmul(s.h, hvert(s.H, k))); }
static inline void hface(const HullShape& s, int f, P3& n, float& d) {
    const float* pl = s.H + 4 * (17 + f);
    P3 nw = rmul(s.R, cdiv(p3(pl[0], pl[1], pl[2]), s.h));
    float l = plen(nw);
    n = p3(nw.x / l, nw.y / l, nw.z / l);
    d = pl[3] / l + pdot(n, s.p);
}
struct HC { P3 n; int cnt; float pt[8][4]; };
static inline void hc_add(HC& c, P3 x, float w) {
    if (c.cnt < 8) { c.pt[c.cnt][0] = x.x; c.pt[c.cnt][1] = x.y; c.pt[c.cnt][2] = x.z; c.pt[c.cnt][3] = w; c.cnt++; return; }
    int hi = 0; for (int q = 1; q < 8; q++) if (c.pt[q][3] > c.pt[hi][3]) hi = q;
    if (w < c.pt[hi][3]) { c.pt[hi][0] = x.x; c.pt[hi][1] = x.y; c.pt[hi][2] = x.z; c.pt[hi][3] = w; }
}
static HC hull_ground(const HullShape& s, float margin) {
    HC c; c.cnt = 0; c.n = p3(0.0f, -1.0f, 0.0f);
    for (int k = 0; k < hnv(s.H); k++) {
        P3 x = hw(s, k);
        if (x.y >= margin) continue;
        hc_add(c, p3(x.x, 0.5f * x.y, x.z), x.y);
    }
    return c;
}
static HC hull_hull(const HullShape& A, const HullShape& B, float margin) {
    HC c; c.cnt = 0; c.n = p3(0, 0, 0);
    const int nfa = hnf(A.H), nfb = hnf(B.H), nva = hnv(A.H), nvb = hnv(B.H), nda = hnd(A.H), ndb = hnd(B.H);
    P3 VA[16], VB[16], DA[12], DB[12];
    for (int k = 0; k < nva; k++) VA[k] = hw(A, k);
    for (int k = 0; k < nvb; k++) VB[k] = hw(B, k);
    for (int k = 0; k < nda; k++) DA[k] = pnorm(rmul(A.R, cmul(A.h, hdir(A.H, k))));
    for (int k = 0; k < ndb; k++) DB[k] = pnorm(rmul(B.R, cmul(B.h, hdir(B.H, k))));
    float sa = -1e30f; int fa = 0;
    for (int f = 0; f < nfa; f++) {
        P3 n; float d; hface(A, f, n, d);
        float lo = 1e30f; for (int k = 0; k < nvb; k++) lo = std::fmin(lo, pdot(VB[k], n));
        float s = lo - d; if (s > margin) return c; if (s > sa) { sa = s; fa = f; }
    }
    float sb = -1e30f; int fb = 0;
    for (int f = 0; f < nfb; f++) {
        P3 n; float d; hface(B, f, n, d);
        float lo = 1e30f; for (int k = 0; k < nva; k++) lo = std::fmin(lo, pdot(VA[k], n));
        float s = lo - d; if (s > margin) return c; if (s > sb) { sb = s; fb = f; }
    }
    float se = -1e30f; P3 el = p3(0, 0, 0); int ei = 0, ej = 0;
    for (int i = 0; i < nda; i++) for (int j = 0; j < ndb; j++) {
        P3 l0 = pcross(DA[i], DB[j]); float l2 = pdot(l0, l0); if (l2 < 1e-6f) continue;
        P3 l = l0 * (1.0f / std::sqrt(l2));
        float alo = 1e30f, ahi = -1e30f, blo = 1e30f, bhi = -1e30f;
        for (int k = 0; k < nva; k++) { float d = pdot(VA[k], l); alo = std::fmin(alo, d); ahi = std::fmax(ahi, d); }
        for (int k = 0; k < nvb; k++) { float d = pdot(VB[k], l); blo = std::fmin(blo, d); bhi = std::fmax(bhi, d); }
        float s1 = blo - ahi, s2 = alo - bhi;
        float s = s1; if (s2 > s1) { s = s2; l = -l; }
        if (s > margin) return c;
        if (s > se) { se = s; el = l; ei = i; ej = j; }
    }
    bool use_b = sb > sa + 0.005f;
    float fbest = use_b ? sb : sa;
    if (se > fbest + 0.01f) {
        P3 da = pnorm(rmul(A.R, cmul(A.h, hdir(A.H, ei)))), db = pnorm(rmul(B.R, cmul(B.h, hdir(B.H, ej))));
        P3 a0 = A.p, a1 = A.p; float best = -1e30f;
        for (int k = 0; k < hns(A.H); k++) {
            int x, y; hseg(A.H, k, x, y); P3 q0 = hw(A, x), q1 = hw(A, y);
            if (fabs_(pdot(pnorm(q1 - q0), da)) < 0.999f) continue;
            float m = pdot(q0 + q1, el); if (m > best) { best = m; a0 = q0; a1 = q1; }
        }
        P3 b0 = B.p, b1 = B.p; best = 1e30f;
        for (int k = 0; k < hns(B.H); k++) {
            int x, y; hseg(B.H, k, x, y); P3 q0 = hw(B, x), q1 = hw(B, y);
            if (fabs_(pdot(pnorm(q1 - q0), db)) < 0.999f) continue;
            float m = pdot(q0 + q1, el); if (m < best) { best = m; b0 = q0; b1 = q1; }
        }
        P3 d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
        float aa = pdot(d1, d1), ee = pdot(d2, d2), ff = pdot(d2, r), cc = pdot(d1, r), bb = pdot(d1, d2);
        float den = aa * ee - bb * bb;
        float s1 = 0.0f; if (den > 1e-9f) s1 = std::fmin(std::fmax((bb * ff - cc * ee) / den, 0.0f), 1.0f);
        float t1 = (bb * s1 + ff) / std::fmax(ee, 1e-9f);
        if (t1 < 0.0f) { t1 = 0.0f; s1 = std::fmin(std::fmax(-cc / std::fmax(aa, 1e-9f), 0.0f), 1.0f); }
        else if (t1 > 1.0f) { t1 = 1.0f; s1 = std::fmin(std::fmax((bb - cc) / std::fmax(aa, 1e-9f), 0.0f), 1.0f); }
        P3 q1 = a0 + d1 * s1, q2 = b0 + d2 * t1;
        c.n = el; c.cnt = 1;
        P3 mid = (q1 + q2) * 0.5f;
        c.pt[0][0] = mid.x; c.pt[0][1] = mid.y; c.pt[0][2] = mid.z; c.pt[0][3] = pdot(q2 - q1, el);
        return c;
    }
    const HullShape& Rs = use_b ? B : A;
    const HullShape& Is = use_b ? A : B;
    const int fr = use_b ? fb : fa;
    P3 n; float rw; hface(Rs, fr, n, rw);
    const int nfi = use_b ? nfa : nfb;
    int fi = 0; float bd = 1e30f;
    for (int f = 0; f < nfi; f++) { P3 m; float d; hface(Is, f, m, d); float dd = pdot(m, n); if (dd < bd) { bd = dd; fi = f; } }
    P3 poly[16], tmp[16];
    int pn = hfcnt(Is.H, fi);
    for (int q = 0; q < pn; q++) poly[q] = hw(Is, hfidx(Is.H, fi, q));
    const int rn = hfcnt(Rs.H, fr);
    P3 rc = p3(0, 0, 0);
    for (int q = 0; q < rn; q++) rc = rc + hw(Rs, hfidx(Rs.H, fr, q));
    rc = p3(rc.x / (float)rn, rc.y / (float)rn, rc.z / (float)rn);
    for (int e = 0; e < rn; e++) {
        P3 v0 = hw(Rs, hfidx(Rs.H, fr, e)), v1 = hw(Rs, hfidx(Rs.H, fr, (e + 1) % rn));
        P3 sn = pnorm(pcross(v1 - v0, n)); if (pdot(sn, rc - v0) > 0.0f) sn = -sn;
        int tn = 0;
        for (int q = 0; q < pn; q++) {
            P3 q0 = poly[q], q1 = poly[(q + 1) % pn];
            float d0 = pdot(q0 - v0, sn), d1 = pdot(q1 - v0, sn);
            if (d0 <= 0.0f && tn < 16) tmp[tn++] = q0;
            if ((d0 <= 0.0f) != (d1 <= 0.0f) && tn < 16) tmp[tn++] = q0 + (q1 - q0) * (d0 / (d0 - d1));
        }
        pn = tn;
        for (int q = 0; q < pn; q++) poly[q] = tmp[q];
        if (pn == 0) return c;
    }
    for (int q = 0; q < pn; q++) {
        P3 pp = poly[q]; float sep = pdot(pp, n) - rw;
        if (sep > margin) continue;
        hc_add(c, pp - n * (0.5f * sep), sep);
    }
    c.n = use_b ? -n : n;
    return c;
}
// reduce4 as gpu/gpu_world.js:532-554
static void hc_reduce4(HC& c) {
    int cnt = c.cnt; if (cnt <= 4) return;
    P3 n = c.n;
    auto P = [&](int k) { return p3(c.pt[k][0], c.pt[k][1], c.pt[k][2]); };
    int i0 = 0; for (int k = 1; k < cnt; k++) if (c.pt[k][3] < c.pt[i0][3]) i0 = k;
    P3 q0 = P(i0);
    int i1 = 0; float best = -1.0f;
    for (int k = 0; k < cnt; k++) { P3 d = P(k) - q0; if (pdot(d, d) > best) { best = pdot(d, d); i1 = k; } }
    P3 e = P(i1) - q0;
    int i2 = 0, i3 = 0; float b2 = -1e30f, b3 = -1e30f;
    for (int k = 0; k < cnt; k++) { float a = pdot(pcross(P(k) - q0, e), n); if (a > b2) { b2 = a; i2 = k; } if (-a > b3) { b3 = -a; i3 = k; } }
    int sel[4] = {i0, i1, i2, i3};
    float out[4][4]; int oc = 0;
    for (int k = 0; k < 4; k++) {
        bool dup = false; for (int q = 0; q < k; q++) if (sel[q] == sel[k]) dup = true;
        if (!dup) { for (int t = 0; t < 4; t++) out[oc][t] = c.pt[sel[k]][t]; oc++; }
    }
    for (int k = 0; k < oc; k++) for (int t = 0; t < 4; t++) c.pt[k][t] = out[k][t];
    c.cnt = oc;
}

}  // namespace

// ============================================================================================================
// C interface for the tests (ctypes)
// ============================================================================================================
extern "C" {

struct ow_step_params { uint32_t iterations, substeps, order, sleep_mode, pinch_kill, chunk, damage, reduce, warm; };

void* ow_create(uint32_t n_static, const int32_t* static_xyz, const uint8_t* static_mat, const int32_t* static_sid,
                const uint8_t* static_infill, uint32_t n_bodies, const uint32_t* body_first, const int32_t* body_brick_xyz,
                const uint8_t* body_brick_mat, const float* body_pose) {
    World* w = new World();
    uint32_t nd = n_bodies ? body_first[n_bodies] : 0;
    w->ns = n_static; w->nd = nd;
    uint32_t nt = n_static + nd;
    w->ctab.assign(NCT, 0);
    w->mat.assign(nt, 0); w->infill.assign(nt, 0); w->bx.assign(nt, 0); w->by.assign(nt, 0); w->bz.assign(nt, 0);
    w->sid.assign(nt, -1); w->body.assign(nt, STATIC); w->next.assign(nt, NONE); w->sup.assign(nt, 0);
    w->local.assign(nt, vv(0, 0, 0)); w->wpos.assign(nt, vv(0, 0, 0));
    w->nb6.assign((size_t)nt * 6, NONE); w->bond.assign((size_t)nt * 4, 0.0f); w->bmax.assign((size_t)nt * 4, 0.0f);
    w->phi.assign(nt, 0.0f); w->ext.assign(nt, 0.0f); w->stress.assign(nt, 0.0f); w->phi64.assign(nt, 0.0);
    w->hhead.assign(HSIZE, NONE); w->hnext.assign(nt, NONE);
    for (uint32_t i = 0; i < n_static; i++) {
        int x = static_xyz[3 * i], y = static_xyz[3 * i + 1], z = static_xyz[3 * i + 2];
        uint8_t m = static_mat[i];
        if (!inb(x, y, z) || w->gget(x, y, z) != 0) { delete w; return nullptr; }
        w->mat[i] = m; w->bx[i] = x; w->by[i] = y; w->bz[i] = z; w->sid[i] = static_sid[i];
        w->infill[i] = (m == GLASS || static_infill[i]) ? 1 : 0;
        w->body[i] = STATIC;
        w->gset(x, y, z, i + 1);
        w->local[i] = lat_pos(x, y, z); w->wpos[i] = w->local[i];
    }
    for (uint32_t i = 0; i < n_static; i++) finalize_brick(*w, i);
    int32_t nst = 0;
    for (uint32_t i = 0; i < n_static; i++) nst = std::max(nst, w->sid[i] + 1);
    w->st_size.assign(nst, 0);
    w->st_conn.assign(nst, 0);
    w->st_hit.assign(nst, 0);
    for (uint32_t i = 0; i < n_static; i++) if (w->sid[i] >= 0) w->st_size[w->sid[i]]++;
    w->cap_bodies = n_bodies; w->cap_bricks = nd;
    w->nbody = n_bodies;
    uint32_t nb = n_bodies;
    w->alive.assign(nb, 0); w->asleep.assign(nb, 0); w->wake.assign(nb, 0);
    w->first.assign(nb, NONE); w->count.assign(nb, 0); w->nc.assign(nb, 0);
    w->pos.assign(nb, vv(0, 0, 0)); w->v = w->pos; w->w = w->pos; w->vpre = w->pos; w->wpre = w->pos;
    w->q.assign((size_t)nb * 4, 0.0f); w->rot.assign((size_t)nb * 9, 0.0f); w->iil = w->rot; w->iiw = w->rot;
    w->m.assign(nb, 0.0f); w->im = w->m; w->sleep = w->m; w->rad = w->m; w->maxr = w->m;
    w->vlast.assign(nb, vv(0, 0, 0)); w->wlast = w->vlast; w->bresid.assign(nb, 1.0); w->nmax.assign(nb, 1.0f);
    w->blt.assign(nb, 0.0f);
    w->island.assign(nb, NONE);
    std::vector<uint32_t> lst;
    for (uint32_t b = 0; b < nb; b++) {
        uint32_t s = body_first[b], e = body_first[b + 1];
        if (e <= s) { delete w; return nullptr; }
        lst.clear();
        for (uint32_t k = s; k < e; k++) {
            uint32_t i = n_static + k;
            int x = body_brick_xyz[3 * k], y = body_brick_xyz[3 * k + 1], z = body_brick_xyz[3 * k + 2];
            w->mat[i] = body_brick_mat[k]; w->bx[i] = x; w->by[i] = y; w->bz[i] = z; w->sid[i] = -1;
            w->local[i] = lat_pos(x, y, z);
            lst.push_back(i);
        }
        const float* ps = body_pose + (size_t)b * 13;
        float prot[9];
        q_to_m(ps + 3, prot);
        setup_body(*w, b, lst.data(), (uint32_t)lst.size(), vv(ps[0], ps[1], ps[2]), prot, ps + 3, vv(ps[7], ps[8], ps[9]), vv(ps[10], ps[11], ps[12]));
    }
    w->dirty.assign(nb, 0);
    body_bonds(*w);
    return w;
}
void ow_destroy(void* h) { delete (World*)h; }

void ow_counts(void* h, uint64_t* out) {
    World* w = (World*)h;
    out[0] = w->ns; out[1] = w->nd; out[2] = w->nbody; out[3] = w->cs.size(); out[4] = w->man_a.size();
    out[5] = w->ncolors; out[6] = w->would_drop; out[7] = w->frame; out[8] = w->ncpool;
}

// body state: pos3 q4 v3 w3 (13 floats), plus sleep timer; flags bit0 alive, bit1 asleep
void ow_get_bodies(void* h, float* state13, float* sleep, uint8_t* flags) {
    World* w = (World*)h;
    for (uint32_t b = 0; b < w->nbody; b++) {
        float* s = state13 + (size_t)b * 13;
        for (int k = 0; k < 3; k++) { s[k] = w->pos[b][k]; s[7 + k] = w->v[b][k]; s[10 + k] = w->w[b][k]; }
        for (int k = 0; k < 4; k++) s[3 + k] = w->q[(size_t)b * 4 + k];
        sleep[b] = w->sleep[b];
        flags[b] = (w->alive[b] ? 1 : 0) | (w->asleep[b] ? 2 : 0);
    }
}
void ow_set_bodies(void* h, const float* state13, const float* sleep, const uint8_t* flags) {
    World* w = (World*)h;
    for (uint32_t b = 0; b < w->nbody; b++) {
        const float* s = state13 + (size_t)b * 13;
        for (int k = 0; k < 3; k++) { w->pos[b][k] = s[k]; w->v[b][k] = s[7 + k]; w->w[b][k] = s[10 + k]; }
        for (int k = 0; k < 4; k++) w->q[(size_t)b * 4 + k] = s[3 + k];
        w->sleep[b] = sleep[b];
        bool was = w->alive[b];
        w->alive[b] = flags[b] & 1; w->asleep[b] = (flags[b] >> 1) & 1;
        if (was && !w->alive[b]) kill_body(*w, b);
    }
}
// per-body setup: m, im, rad, iil9 (12 floats); per body brick: local3
void ow_get_setup(void* h, float* body12, float* local3) {
    World* w = (World*)h;
    for (uint32_t b = 0; b < w->nbody; b++) {
        float* s = body12 + (size_t)b * 12;
        s[0] = w->m[b]; s[1] = w->im[b]; s[2] = w->rad[b];
        for (int k = 0; k < 9; k++) s[3 + k] = w->iil[(size_t)b * 9 + k];
    }
    for (uint32_t k = 0; k < w->nd; k++) for (int c = 0; c < 3; c++) local3[(size_t)k * 3 + c] = w->local[w->ns + k][c];
}
void ow_get_wpos(void* h, float* wpos3) {
    World* w = (World*)h;
    for (uint32_t k = 0; k < w->nd; k++) for (int c = 0; c < 3; c++) wpos3[(size_t)k * 3 + c] = w->wpos[w->ns + k][c];
}
// brick world positions are part of the state: a sleeping body keeps the positions of its last awake substep
void ow_set_wpos(void* h, const float* wpos3) {
    World* w = (World*)h;
    for (uint32_t k = 0; k < w->nd; k++) for (int c = 0; c < 3; c++) w->wpos[w->ns + k][c] = wpos3[(size_t)k * 3 + c];
}
void ow_get_bonds(void* h, float* bond4, uint32_t* nb6) {
    World* w = (World*)h;
    for (uint32_t i = 0; i < w->ns; i++) {
        for (int k = 0; k < 4; k++) bond4[(size_t)i * 4 + k] = w->bond[(size_t)i * 4 + k];
        for (int k = 0; k < 6; k++) nb6[(size_t)i * 6 + k] = w->nb6[(size_t)i * 6 + k];
    }
}

void ow_step(void* h, float dt, const ow_step_params* p) {
    StepParams P{p->iterations, p->substeps, p->order, p->sleep_mode, p->pinch_kill, p->damage, p->reduce, p->warm};
    ((World*)h)->chunk = p->chunk;
    step(*(World*)h, dt, P);
}
// substep pieces for per-phase parity: update_cache + gravity + hash + contacts (+ prep)
void ow_contacts_only(void* h, float hsub, int with_prep) {
    World* w = (World*)h;
    update_cache(*w);
    for (uint32_t b = 0; b < w->nbody; b++) if (w->alive[b] && !w->asleep[b]) w->v[b][1] -= GR * hsub;
    build_hash(*w);
    gen_contacts(*w);
    if (with_prep) prep_contacts(*w, hsub);
    build_manifolds(*w);
    islands(*w);
}

// contacts in list order. ids: a, b, bo, ba, bb (5 u32); f: p3 n3 depth (7 floats); s: jn jt1 jt2 mn mt1 mt2 bias vn0 (8),
// zeros for a contact the reduction left out
uint64_t ow_get_contacts(void* h, uint32_t* ids, float* f, float* s) {
    World* w = (World*)h;
    for (size_t k = 0; k < w->cs.size(); k++) {
        const Contact& c = w->cs[k];
        uint32_t* o = ids + k * 5; o[0] = c.a; o[1] = c.b; o[2] = c.bo; o[3] = c.ba; o[4] = c.bb;
        float* g = f + k * 7; for (int t = 0; t < 3; t++) { g[t] = c.p[t]; g[3 + t] = c.n[t]; } g[6] = c.depth;
        float* x = s + k * 8; x[0] = c.jn; x[1] = c.jt1; x[2] = c.jt2; x[3] = c.mn; x[4] = c.mt1; x[5] = c.mt2; x[6] = c.bias; x[7] = c.vn0;
        if (c.off) for (int t = 0; t < 8; t++) x[t] = 0.0f;
    }
    return w->cs.size();
}
void ow_get_islands(void* h, uint32_t* label) { World* w = (World*)h; for (uint32_t b = 0; b < w->nbody; b++) label[b] = w->island[b]; }
// manifolds: a, b, colour, count (4 u32 each), in manifold order
uint64_t ow_get_manifolds(void* h, uint32_t* out4) {
    World* w = (World*)h;
    for (size_t m = 0; m < w->man_a.size(); m++) {
        out4[m * 4] = w->man_a[m]; out4[m * 4 + 1] = w->man_b[m]; out4[m * 4 + 2] = w->man_color[m]; out4[m * 4 + 3] = w->man_count[m];
    }
    return w->man_a.size();
}

// ---- load path
double ow_sor(void* h, int32_t s, float omega, double tol, uint32_t max_sweeps, int32_t mode, uint32_t* sweeps) {
    SorResult r = sor_solve(*(World*)h, s, omega, tol, max_sweeps, mode);
    if (sweeps) *sweeps = r.sweeps;
    return r.resid;
}
void ow_structure_warm(void* h, int32_t s) { warm_struct(*(World*)h, s); }
void ow_structure_frame(void* h, uint32_t frame, float dt, const int32_t* active, uint32_t n, uint32_t* counts) {
    structure_frame(*(World*)h, frame, dt, active, n, counts);
}
void ow_structure_state(void* h, int32_t* warm, uint8_t* solved, float* settle, double* resid) {
    World* w = (World*)h;
    sched_size(*w);
    for (size_t s = 0; s < w->st_warm.size(); s++) {
        if (warm) warm[s] = w->st_warm[s];
        if (solved) solved[s] = w->st_solved[s];
        if (settle) settle[s] = w->st_settle[s];
        if (resid) resid[s] = w->st_resid[s];
    }
}
void ow_set_capacity(void* h, uint32_t spare_bodies, uint32_t spare_bricks) {
    World* w = (World*)h;
    w->cap_bodies = w->nbody + spare_bodies; w->cap_bricks = w->nd + spare_bricks;
}
// counts: pieces, detached bricks, structures left pending; now / top indexed by structure (NULL = not wanted)
void ow_connect(void* h, const int32_t* ids, uint32_t n, uint32_t* counts, uint32_t* now, int32_t* top) {
    World* w = (World*)h;
    counts[0] = counts[1] = counts[2] = 0;
    for (uint32_t k = 0; k < n; k++) {
        const int32_t s = ids[k];
        if (s < 0 || s >= (int32_t)w->st_conn.size()) continue;
        w->st_conn[s] = 0;
        conn_struct(*w, s, counts);
        uint32_t c; int32_t t;
        struct_tally(*w, s, c, t);
        if (now) now[s] = c;
        if (top) top[s] = t;
    }
}
// connectivity (src/lib.rs:1137-1141): every pending structure in structure order
void ow_connectivity(void* h, uint32_t* counts, uint32_t* now, int32_t* top) {
    World* w = (World*)h;
    std::vector<int32_t> ids;
    for (size_t s = 0; s < w->st_conn.size(); s++) if (w->st_conn[s]) ids.push_back((int32_t)s);
    ow_connect(h, ids.data(), (uint32_t)ids.size(), counts, now, top);
}
void ow_remove_bricks(void* h, const uint32_t* statics, uint32_t ns_, const uint32_t* body_bricks, uint32_t nb_) {
    World* w = (World*)h;
    for (uint32_t k = 0; k < ns_; k++) if (statics[k] < w->ns) remove_brick(*w, statics[k]);
    for (uint32_t k = 0; k < nb_; k++) if (body_bricks[k] < w->nd) remove_brick(*w, w->ns + body_bricks[k]);
}
void ow_rebuild_bodies(void* h, uint32_t* counts) { rebuild_bodies(*(World*)h, counts); }
void ow_body_frame(void* h, float dt, uint32_t crush_used, uint32_t* counts) { body_frame(*(World*)h, dt, crush_used, counts); }
// per body: last residual, peak load factor, load time, largest joint ratio
void ow_body_state(void* h, double* resid, float* nmax, float* lt, float* maxr) {
    World* w = (World*)h;
    for (uint32_t b = 0; b < w->nbody; b++) { resid[b] = w->bresid[b]; nmax[b] = w->nmax[b]; lt[b] = w->blt[b]; maxr[b] = w->maxr[b]; }
}
// per body brick: f64 potential and inertial load
void ow_body_phi(void* h, double* phi64, float* ext) {
    World* w = (World*)h;
    for (uint32_t k = 0; k < w->nd; k++) { phi64[k] = w->phi64[w->ns + k]; ext[k] = w->ext[w->ns + k]; }
}
// crush_at on one brick (a static id, or ns + a body-brick id) with energy e at point p; returns the bricks crushed
uint32_t ow_crush_at(void* h, uint32_t start, float e, float px, float py, float pz, uint32_t cap) {
    World* w = (World*)h;
    if (start >= w->mat.size()) return 0;
    return crush_at(*w, start, e, vv(px, py, pz), cap);
}
// damage counters since the last read (candidates, crushed, removed, severed, cracked) and per structure whether a hit
// woke it; both cleared by the read
// counts: candidates, crushed, removed, severed, cracked, ploughed loose, scraped (since the last read)
void ow_read_damage(void* h, uint64_t* counts, uint8_t* hit) {
    World* w = (World*)h;
    for (int k = 0; k < 7; k++) { counts[k] = w->dmg[k]; w->dmg[k] = 0; }
    for (size_t s = 0; s < w->st_hit.size(); s++) { if (hit) hit[s] = w->st_hit[s]; w->st_hit[s] = 0; }
}
void ow_body_bonds(void* h, float* bond4, uint32_t* nb6) {
    World* w = (World*)h;
    for (uint32_t k = 0; k < w->nd; k++) {
        const uint32_t i = w->ns + k;
        for (int a = 0; a < 4; a++) bond4[(size_t)k * 4 + a] = w->bond[(size_t)i * 4 + a];
        for (int d = 0; d < 6; d++) {
            const uint32_t j = w->nb6[(size_t)i * 6 + d];
            nb6[(size_t)k * 6 + d] = j == NONE ? NONE : j - w->ns;
        }
    }
}
void ow_conn_pending(void* h, uint8_t* flags) { World* w = (World*)h; for (size_t s = 0; s < w->st_conn.size(); s++) flags[s] = w->st_conn[s]; }
void ow_get_phi(void* h, float* phi) { World* w = (World*)h; for (uint32_t i = 0; i < w->ns; i++) phi[i] = w->phi[i]; }
void ow_get_phi64(void* h, double* phi) { World* w = (World*)h; for (uint32_t i = 0; i < w->ns; i++) phi[i] = w->phi64[i]; }
void ow_set_phi(void* h, const float* phi) { World* w = (World*)h; for (uint32_t i = 0; i < w->ns; i++) { w->phi[i] = phi[i]; w->phi64[i] = phi[i]; } }
void ow_set_ext(void* h, const float* ext) { World* w = (World*)h; for (uint32_t i = 0; i < w->ns; i++) w->ext[i] = ext[i]; }
// joints: i, axis, j, decision, crushed (5 u32) + ratio, bond_after (2 floats). Returns the count; maxr in *maxr.
uint64_t ow_stress(void* h, int32_t s, float dt, int32_t live, uint64_t cap, uint32_t* ids, float* vals, float* maxr) {
    World* w = (World*)h;
    std::vector<Joint> out;
    float mr = 0.0f;
    w->crush_n = 0;
    for (uint32_t i = 0; i < w->ns; i++) if (w->in_struct(i, s)) w->stress[i] = 0.0f;
    for (uint32_t i = 0; i < w->ns; i++) if (w->in_struct(i, s)) { float r = stress_brick(*w, i, dt, live != 0, out); if (r > mr) mr = r; }
    if (maxr) *maxr = mr;
    for (size_t k = 0; k < out.size() && k < cap; k++) {
        uint32_t* o = ids + k * 5; o[0] = out[k].i; o[1] = out[k].axis; o[2] = out[k].j; o[3] = out[k].decision; o[4] = out[k].crushed;
        vals[k * 2] = out[k].ratio; vals[k * 2 + 1] = out[k].bond_after;
    }
    return out.size();
}
// structural's resting-body loads (src/lib.rs:1233-1259) for the listed structures, after update_cache as step does
void ow_structure_loads(void* h, const int32_t* listed, uint32_t n) {
    World* w = (World*)h;
    std::vector<uint8_t> act(4096, 0);
    for (uint32_t k = 0; k < n; k++) if (listed[k] >= 0 && listed[k] < 4096) act[listed[k]] = 1;
    update_cache(*w);
    std::vector<float> extn(w->ns, 0.0f);
    auto target = [&](V p) -> uint32_t {
        int cx = (int)std::floor(p[0] / S) + NX / 2, cy = (int)std::floor((p[1] - RB - 0.02f) / S), cz = (int)std::floor(p[2] / S) + NZ / 2;
        uint32_t j = w->static_brick(cx, cy, cz);
        if (j == NONE || w->sid[j] < 0 || !act[w->sid[j]]) return NONE;
        return j;
    };
    for (uint32_t b = 0; b < w->nbody; b++) {
        if (!w->alive[b]) continue;
        uint32_t ns = 0, nground = 0;
        for (uint32_t k = w->first[b]; k != NONE; k = w->next[k]) {
            V p = w->wpos[k];
            if (p[1] < RB + 0.05f) nground++;
            if (target(p) != NONE) ns++;
        }
        if (ns == 0) continue;
        float share = w->m[b] / (float)(ns + nground);
        for (uint32_t k = w->first[b]; k != NONE; k = w->next[k]) {
            uint32_t j = target(w->wpos[k]);
            if (j != NONE) extn[j] += share;
        }
    }
    for (uint32_t i = 0; i < w->ns; i++) if (w->sid[i] >= 0 && act[w->sid[i]]) w->ext[i] = w->ext[i] * 0.8f + extn[i] * 0.2f;
}
void ow_get_ext(void* h, float* ext) { World* w = (World*)h; for (uint32_t i = 0; i < w->ns; i++) ext[i] = w->ext[i]; }

void ow_remove_static(void* h, uint32_t i) {
    World* w = (World*)h;
    if (i >= w->ns || w->mat[i] == 0) return;
    w->gset(w->bx[i], w->by[i], w->bz[i], 0);
    w->mat[i] = 0;
}


// ---- hull SAT: shapes are p3 q4 h3 hull (11 floats); b's hull < 0 = the ground. Output: normal 3, pad, 8 x (p3, sep).
int32_t ow_collide_hulls(const float* hulls, const float* A, const float* B, float margin, int32_t do_reduce, float* out36) {
    HullShape a{p3(A[0], A[1], A[2]), quat_m3(A + 3), p3(A[7], A[8], A[9]), hulls + (size_t)(int)A[10] * 320};
    HC c;
    if (B[10] < 0.0f) c = hull_ground(a, margin);
    else {
        HullShape b{p3(B[0], B[1], B[2]), quat_m3(B + 3), p3(B[7], B[8], B[9]), hulls + (size_t)(int)B[10] * 320};
        c = hull_hull(a, b, margin);
    }
    if (do_reduce) hc_reduce4(c);
    out36[0] = c.n.x; out36[1] = c.n.y; out36[2] = c.n.z; out36[3] = 0.0f;
    for (int k = 0; k < 8; k++) for (int t = 0; t < 4; t++) out36[4 + 4 * k + t] = k < c.cnt ? c.pt[k][t] : 0.0f;
    return c.cnt;
}

// ---- box SAT: boxes are p3 q4 h3 (10 floats). Output: normal3 + up to 8 points (p3, sep), reduced to 4.
int32_t ow_collide_boxes(const float* A, const float* B, float margin, int32_t do_reduce, float* out) {
    P3 pa = p3(A[0], A[1], A[2]), pb = p3(B[0], B[1], B[2]);
    M3 ra = quat_m3(A + 3), rb = quat_m3(B + 3);
    CP pts[8]; P3 n;
    int cnt = collide_boxes(pa, ra, p3(A[7], A[8], A[9]), pb, rb, p3(B[7], B[8], B[9]), margin, pts, &n);
    if (cnt == 0) return 0;
    if (do_reduce) cnt = reduce4(pts, cnt, n);
    out[0] = n.x; out[1] = n.y; out[2] = n.z;
    for (int k = 0; k < cnt; k++) { out[3 + 4 * k] = pts[k].p.x; out[4 + 4 * k] = pts[k].p.y; out[5 + 4 * k] = pts[k].p.z; out[6 + 4 * k] = pts[k].s; }
    return cnt;
}

// many pairs in one call (for timing the restatement without a call per pair): counts only
uint64_t ow_collide_boxes_batch(const float* A, const float* B, uint32_t n, float margin, int32_t do_reduce) {
    uint64_t hits = 0;
    float out[3 + 8 * 4];
    for (uint32_t i = 0; i < n; i++) hits += ow_collide_boxes(A + (size_t)i * 10, B + (size_t)i * 10, margin, do_reduce, out) > 0;
    return hits;
}
uint64_t ow_collide_hulls_batch(const float* hulls, const float* A, const float* B, uint32_t n, float margin, int32_t do_reduce) {
    uint64_t hits = 0;
    float out[36];
    for (uint32_t i = 0; i < n; i++) hits += ow_collide_hulls(hulls, A + (size_t)i * 11, B + (size_t)i * 11, margin, do_reduce, out) > 0;
    return hits;
}


// The reference's manifold colouring (gpu/gpu_world.js:922-1038, rounds scheduled at :2576-2577), restated on a
// manifold graph given as endpoint pairs: each round every uncoloured manifold picks one of the four lowest colours
// free at both its awake bodies (by its key and its own round), claims it at each with its priority (supports, i.e.
// manifolds with a static or sleeping side, first; then by key), breaks priority ties with a second hash, and keeps
// the colour where its claim is the strongest at both bodies. The first rounds_s rounds let only supports claim.
// What is uncoloured after rounds_s + rounds_a rounds, or finds no free colour, goes to the overflow pass
// (colour = color_limit). Shape ids for the keys are (a + 1 + salt * 2^20, b + 1) with b = 0 for the static side;
// the salt (the chunk's index within its body pair) keeps the keys of one pair's chunks distinct, as the reference's
// shape pairs are. Stats out: [0] colours used (highest colour + 1 among coloured), [1] overflow manifolds.
static uint32_t ref_mkey(uint32_t sa, uint32_t sb) {   // gpu/gpu_world.js:245-250
    uint32_t h = (sa * 0x9E3779B1u) ^ ((sb + 0x7F4A7C15u) * 0x85EBCA77u);
    h ^= h >> 15; h *= 0x2C1B3C6Du; h ^= h >> 12;
    return h | 1u;
}
static uint32_t ref_mkey2(uint32_t sa, uint32_t sb) {  // gpu/gpu_world.js:979-984
    uint32_t h = (sb * 0x2545F491u) ^ ((sa + 0x68E31DA4u) * 0xB5297A4Du);
    h ^= h >> 13; h *= 0x1B873593u; h ^= h >> 16;
    return h;
}

void ow_ref_colouring(uint32_t n, const uint32_t* a, const uint32_t* b, const uint32_t* salt, const uint8_t* a_awake,
                      const uint8_t* b_awake, uint32_t n_bodies, uint32_t color_limit, uint32_t rounds_s, uint32_t rounds_a, uint32_t* colour,
                      uint32_t* stats) {
    const uint32_t UNC = 0xfffffffeu, COL_ROUNDS = 12;
    if (color_limit > 31) color_limit = 31;
    std::vector<uint32_t> mask(n_bodies, 0), claim((size_t)n_bodies * 32, 0), claim2((size_t)n_bodies * 32, 0);
    std::vector<uint32_t> mtry(n, 0), key(n), key2(n), pri(n);
    for (uint32_t m = 0; m < n; m++) {
        colour[m] = UNC;
        const uint32_t sa = a[m] + 1 + (salt ? salt[m] << 20 : 0u), sb = b[m] == 0xFFFFFFFFu ? 0u : b[m] + 1;
        key[m] = ref_mkey(sa, sb);
        key2[m] = ref_mkey2(sa, sb);
        const bool support = !a_awake[m] || !b_awake[m];
        pri[m] = (support ? 0u : 0x2000000u) | (key[m] >> 7);
    }
    const uint32_t all = color_limit >= 32 ? 0xffffffffu : ((1u << color_limit) - 1u);
    uint32_t gr = 0;
    for (uint32_t r = 0; r < rounds_s + rounds_a; r++) {
        const bool support_only = r < rounds_s;
        // claim
        for (uint32_t m = 0; m < n; m++) {
            if (colour[m] != UNC) continue;
            const bool da = a_awake[m], db = b_awake[m];
            if (support_only && da && db) continue;
            const uint32_t round = mtry[m] & 0xffffu;
            uint32_t used = 0;
            if (da) used |= mask[a[m]];
            if (db) used |= mask[b[m]];
            uint32_t free = all & ~used;
            if (free == 0 || round >= COL_ROUNDS) { colour[m] = color_limit; continue; }
            const uint32_t nf = (uint32_t)__builtin_popcount(free);
            const uint32_t pick = ((key[m] >> 3) + round * 0x9E37u) % (nf < 4 ? nf : 4);
            for (uint32_t k = 0; k < pick; k++) free &= free - 1;
            const uint32_t c = (uint32_t)__builtin_ctz(free);
            const uint32_t v = ((gr + 1) << 27) | (0x3ffffffu - pri[m]);
            if (da) claim[(size_t)a[m] * 32 + c] = std::max(claim[(size_t)a[m] * 32 + c], v);
            if (db) claim[(size_t)b[m] * 32 + c] = std::max(claim[(size_t)b[m] * 32 + c], v);
            mtry[m] = (round + 1) | (c << 16) | 0x80000000u;
        }
        const uint32_t tag = (gr + 1) << 27;
        auto claimed = [&](uint32_t m, bool stage2) {
            const uint32_t c = (mtry[m] >> 16) & 0x7fffu;
            const bool da = a_awake[m], db = b_awake[m];
            const uint32_t v = tag | (0x3ffffffu - pri[m]);
            if (da && claim[(size_t)a[m] * 32 + c] != v) return false;
            if (db && claim[(size_t)b[m] * 32 + c] != v) return false;
            const uint32_t v2 = tag | (key2[m] >> 5);
            if (!stage2) {
                if (da) claim2[(size_t)a[m] * 32 + c] = std::max(claim2[(size_t)a[m] * 32 + c], v2);
                if (db) claim2[(size_t)b[m] * 32 + c] = std::max(claim2[(size_t)b[m] * 32 + c], v2);
                return true;
            }
            if (da && claim2[(size_t)a[m] * 32 + c] != v2) return false;
            if (db && claim2[(size_t)b[m] * 32 + c] != v2) return false;
            return true;
        };
        // tie
        for (uint32_t m = 0; m < n; m++)
            if (colour[m] == UNC && (mtry[m] & 0x80000000u)) claimed(m, false);
        // resolve
        for (uint32_t m = 0; m < n; m++) {
            if (colour[m] != UNC || !(mtry[m] & 0x80000000u)) continue;
            const bool won = claimed(m, true);
            mtry[m] &= 0x7fffffffu;
            if (!won) continue;
            const uint32_t c = (mtry[m] >> 16) & 0x7fffu;
            colour[m] = c;
            if (a_awake[m]) mask[a[m]] |= 1u << c;
            if (b_awake[m]) mask[b[m]] |= 1u << c;
        }
        gr++;
    }
    uint32_t used = 0, ovf = 0;
    for (uint32_t m = 0; m < n; m++) {
        if (colour[m] == UNC) colour[m] = color_limit;
        if (colour[m] >= color_limit) ovf++;
        else used = std::max(used, colour[m] + 1);
    }
    stats[0] = used;
    stats[1] = ovf;
}

}  // extern "C"

// ============================================================================================================
// The engine crate's box world (engine/src/phys.rs): World::step (phys.rs:152-243) with the hashed-grid broadphase
// (phys.rs:356-408), ground and pair collisions (phys.rs:410-445), push_manifold with its warm start and friction
// anchors (phys.rs:447-497), the soft-step warm start and solve (phys.rs:245-324) and island sleep
// (phys.rs:326-354). BOX_LIST keeps the reference's manifold list order: ground manifolds in body order, then the
// pairs in hash-slot order, solved one after another. BOX_COLOR takes the same manifolds in key order (a, b; the
// ground as b = NONE after b's pairs), colours them greedily in a fixed priority order and solves colour by colour
// (the GPU's order: inside a colour no two manifolds share a moving body, so the order inside it does not matter).
// ============================================================================================================
namespace {

enum { BOX_LIST = 0, BOX_COLOR = 1 };
static const uint32_t BNONE = 0xFFFFFFFFu;      // the ground
static const uint32_t BGROUND2 = 0xFFFFFFFEu;   // a convex cell's second ground patch
static inline bool bground(uint32_t b) { return b >= BGROUND2; }

struct BoxParams {      // the layout of sf_box_params
    float gravity[3]; uint32_t substeps;
    float contact_hertz, damping_ratio, max_push, friction, speculative;
    float sleep_lin, sleep_ang, sleep_time, sleep_dist, sleep_rot;
    int32_t allow_sleep; float cell, leak; int32_t anchor; float anchor_push, anchor_slop;
    uint32_t reserved[4];
};
struct Q4 { float x, y, z, w; };
static inline Q4 q4(float x, float y, float z, float w) { return Q4{x, y, z, w}; }
// Quat::mul, integrate, normalized, conj (engine/src/math.rs:36-48)
static inline Q4 qmul(Q4 a, Q4 o) {
    return q4(a.w * o.x + a.x * o.w + a.y * o.z - a.z * o.y,
              a.w * o.y - a.x * o.z + a.y * o.w + a.z * o.x,
              a.w * o.z + a.x * o.y - a.y * o.x + a.z * o.w,
              a.w * o.w - a.x * o.x - a.y * o.y - a.z * o.z);
}
static inline Q4 qnormalized(Q4 q) {
    float l = sqrt_e(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    float k = l > 0.0f ? 1.0f / l : 1.0f;
    return q4(q.x * k, q.y * k, q.z * k, q.w * k);
}
static inline Q4 qintegrate(Q4 q, P3 w, float h) {
    Q4 dq = qmul(q4(w.x, w.y, w.z, 0.0f), q);
    return qnormalized(q4(q.x + 0.5f * h * dq.x, q.y + 0.5f * h * dq.y, q.z + 0.5f * h * dq.z, q.w + 0.5f * h * dq.w));
}
static inline M3 q_m3(Q4 q) { float f[4] = {q.x, q.y, q.z, q.w}; return quat_m3(f); }
static inline P3 m_mulv(const M3& r, P3 v) { return r.c[0] * v.x + r.c[1] * v.y + r.c[2] * v.z; }
static inline P3 m_tmulv(const M3& r, P3 v) { return p3(pdot(r.c[0], v), pdot(r.c[1], v), pdot(r.c[2], v)); }
static inline M3 m_sandwich(const M3& r, P3 d) {   // R diag(d) R^T (engine/src/math.rs:71-75)
    P3 a = r.c[0] * d.x, b = r.c[1] * d.y, c = r.c[2] * d.z;
    M3 o;
    for (int j = 0; j < 3; j++) o.c[j] = a * pget(r.c[0], j) + b * pget(r.c[1], j) + c * pget(r.c[2], j);
    return o;
}
static inline float plen_e(P3 a) { return sqrt_e(plen2(a)); }
static inline P3 pnorm_e(P3 a) { float l = plen_e(a); return l > 1e-12f ? a * (1.0f / l) : p3(0, 0, 0); }
static inline P3 pmax(P3 a, P3 b) { return p3(maxf(a.x, b.x), maxf(a.y, b.y), maxf(a.z, b.z)); }
// tangents (phys.rs:500-503)
static inline void btangents(P3 n, P3& t1, P3& t2) {
    P3 t = fabs_(n.x) > 0.57f ? p3(n.y, -n.x, 0.0f) : p3(0.0f, n.z, -n.y);
    t1 = pnorm_e(t);
    t2 = pcross(n, t1);
}
// floor as engine/src/math.rs:94 (truncate, then step down)
static inline float bfloor(float x) { float t = (float)(int32_t)x; return t > x ? t - 1.0f : t; }
static inline int32_t bcell(float x, float inv_cell) { return (int32_t)bfloor(x * inv_cell); }
static inline uint32_t bhash(int32_t x, int32_t y, int32_t z) {
    return (uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u;
}

struct BBody {
    P3 p; Q4 q; P3 v, w, h; float inv_m; P3 inv_i; bool awake; float sleep_t; P3 sleep_p; Q4 sleep_q;
    M3 rot; P3 amin, amax;
    uint32_t hull;    // a convex cell of the library (0: a plain box)
};
struct BCp { P3 ra, rb, la, raxn, rbxn, iaxn, ibxn; float adj, nm, jn; };
struct BMan {
    uint32_t a, b, sa, sb; P3 n, t1, t2; float mu; uint32_t cnt; BCp cp[4];
    P3 fa, fb, la_f, lb_f, e0; float tm1, tm2, twm, rad, jt1, jt2, jtw; bool stick;
    P3 ca1, ca2, cb1, cb2, ia1, ia2, ib1, ib2, ian, ibn; float ima, imb;
    uint32_t colour;
};
static inline uint64_t bkey(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

struct BoxWorld {
    std::vector<BBody> bodies;
    std::vector<float> hulls;    // the convex-cell library, 320 floats a cell
    BoxParams prm{};
    int order = BOX_LIST;
    std::vector<BMan> man, old;
    std::unordered_map<uint64_t, uint32_t> old_map;
    std::vector<P3> sv, sw, sdp, sth, sp0; std::vector<float> sim; std::vector<M3> sii; std::vector<Q4> sq;
    std::vector<uint32_t> sbody, sidx, corder;
    uint32_t ncolours = 0, st_awake = 0, st_pairs = 0, st_manifolds = 0, st_points = 0;

    // World::add_box (phys.rs:137-146)
    void add_box(P3 p, Q4 q, P3 h, float density) {
        float m = density * 8.0f * h.x * h.y * h.z;
        BBody b{};
        if (m > 0.0f) {
            float x2 = 4.0f * h.x * h.x, y2 = 4.0f * h.y * h.y, z2 = 4.0f * h.z * h.z;
            b.inv_m = 1.0f / m;
            b.inv_i = p3(12.0f / (m * (y2 + z2)), 12.0f / (m * (x2 + z2)), 12.0f / (m * (x2 + y2)));
        }
        b.p = p; b.q = q; b.h = h; b.awake = m > 0.0f; b.sleep_p = p; b.sleep_q = q;
        b.rot = q_m3(q); b.amin = p; b.amax = p;
        bodies.push_back(b);
    }
    uint32_t spush(P3 v, P3 w, float im, const M3& ii, Q4 q, P3 p0, uint32_t body) {
        sv.push_back(v); sw.push_back(w); sdp.push_back(p3(0, 0, 0)); sth.push_back(p3(0, 0, 0)); sim.push_back(im);
        sii.push_back(ii); sq.push_back(q); sp0.push_back(p0); sbody.push_back(body);
        return (uint32_t)sv.size() - 1;
    }
    void sclear() {
        sv.clear(); sw.clear(); sdp.clear(); sth.clear(); sim.clear(); sii.clear(); sq.clear(); sp0.clear(); sbody.clear();
        M3 z; z.c[0] = z.c[1] = z.c[2] = p3(0, 0, 0);
        spush(p3(0, 0, 0), p3(0, 0, 0), 0.0f, z, q4(0, 0, 0, 1), p3(0, 0, 0), BNONE);
    }

    void step(float dt) {
        const uint32_t n = (uint32_t)bodies.size();
        sidx.assign(n, 0);
        sclear();
        const float spec = prm.speculative;
        for (uint32_t i = 0; i < n; i++) {           // phys.rs:157-171
            BBody& b = bodies[i];
            b.rot = q_m3(b.q);
            P3 e = p3(fabs_(b.rot.c[0].x) * b.h.x + fabs_(b.rot.c[1].x) * b.h.y + fabs_(b.rot.c[2].x) * b.h.z,
                      fabs_(b.rot.c[0].y) * b.h.x + fabs_(b.rot.c[1].y) * b.h.y + fabs_(b.rot.c[2].y) * b.h.z,
                      fabs_(b.rot.c[0].z) * b.h.x + fabs_(b.rot.c[1].z) * b.h.y + fabs_(b.rot.c[2].z) * b.h.z);
            float m = b.awake ? (plen_e(b.v) + plen_e(b.w) * plen_e(b.h)) * dt + 0.5f * spec : 0.5f * spec;
            e = e + p3(m, m, m);
            b.amin = b.p - e; b.amax = b.p + e;
            if (b.awake) sidx[i] = spush(b.v, b.w, b.inv_m, m_sandwich(b.rot, b.inv_i), b.q, b.p, i);
        }
        std::swap(man, old);
        man.clear();
        st_pairs = 0;
        collide_all(dt);
        // masses (phys.rs:184-214)
        const uint32_t sub = prm.substeps > 0 ? prm.substeps : 1;
        const float h = dt / (float)sub;
        const float inv_h = 1.0f / h;
        const float hz = prm.contact_hertz > 0.0f ? prm.contact_hertz : inv_h / 6.0f;
        const float PI_F = 3.14159265358979323846f;
        const float omega = 2.0f * PI_F * hz;
        const float a1 = 2.0f * prm.damping_ratio + h * omega;
        const float a2 = h * omega * a1;
        const float a3 = 1.0f / (1.0f + a2);
        const float bias_rate = omega / a1, mass_scale = a2 * a3, imp_scale = a3 * prm.leak;
        uint32_t pts = 0;
        for (BMan& m : man) {
            const float ima = sim[m.sa], imb = sim[m.sb];
            const M3 iia = sii[m.sa], iib = sii[m.sb];
            m.ima = ima; m.imb = imb;
            const P3 nn = m.n;
            for (uint32_t k = 0; k < m.cnt; k++) {
                BCp& c = m.cp[k];
                c.raxn = pcross(c.ra, nn); c.rbxn = pcross(c.rb, nn);
                c.iaxn = m_mulv(iia, c.raxn); c.ibxn = m_mulv(iib, c.rbxn);
                float kk = ima + imb + pdot(c.raxn, c.iaxn) + pdot(c.rbxn, c.ibxn);
                c.nm = kk > 0.0f ? 1.0f / kk : 0.0f;
            }
            m.ca1 = pcross(m.fa, m.t1); m.ca2 = pcross(m.fa, m.t2); m.cb1 = pcross(m.fb, m.t1); m.cb2 = pcross(m.fb, m.t2);
            m.ia1 = m_mulv(iia, m.ca1); m.ia2 = m_mulv(iia, m.ca2); m.ib1 = m_mulv(iib, m.cb1); m.ib2 = m_mulv(iib, m.cb2);
            float k1 = ima + imb + pdot(m.ca1, m.ia1) + pdot(m.cb1, m.ib1);
            float k2 = ima + imb + pdot(m.ca2, m.ia2) + pdot(m.cb2, m.ib2);
            m.tm1 = k1 > 0.0f ? 1.0f / k1 : 0.0f; m.tm2 = k2 > 0.0f ? 1.0f / k2 : 0.0f;
            m.ian = m_mulv(iia, nn); m.ibn = m_mulv(iib, nn);
            float kt = pdot(nn, m.ian) + pdot(nn, m.ibn);
            m.twm = kt > 0.0f ? 1.0f / kt : 0.0f;
            pts += m.cnt;
        }
        st_manifolds = (uint32_t)man.size(); st_points = pts;
        corder.resize(man.size());
        for (uint32_t k = 0; k < man.size(); k++) corder[k] = k;
        ncolours = 0;
        if (order == BOX_COLOR) colour_manifolds();
        // sub-steps (phys.rs:216-231)
        const P3 g = p3(prm.gravity[0], prm.gravity[1], prm.gravity[2]);
        const float wmax = 0.25f * PI_F * inv_h;
        const uint32_t nb = (uint32_t)sv.size();
        for (uint32_t s = 0; s < sub; s++) {
            for (uint32_t i = 1; i < nb; i++) {
                sv[i] = sv[i] + g * h;
                P3 w = sw[i]; float wl = plen2(w);
                if (wl > wmax * wmax) sw[i] = w * (wmax / sqrt_e(wl));
            }
            warm_start();
            solve(true, inv_h, bias_rate, mass_scale, imp_scale);
            for (uint32_t i = 1; i < nb; i++) {
                P3 v = sv[i], w = sw[i];
                sdp[i] = sdp[i] + v * h; sth[i] = sth[i] + w * h;
                sq[i] = qintegrate(sq[i], w, h);
            }
            solve(false, inv_h, bias_rate, mass_scale, imp_scale);
        }
        for (uint32_t i = 1; i < nb; i++) {          // write back (phys.rs:233-236)
            BBody& b = bodies[sbody[i]];
            b.v = sv[i]; b.w = sw[i]; b.p = sp0[i] + sdp[i]; b.q = sq[i];
        }
        sleep_islands(dt);
        old_map.clear();
        for (uint32_t k = 0; k < man.size(); k++) old_map[bkey(man[k].a, man[k].b)] = k;
        st_awake = nb - 1;
    }

    // phys.rs:245-263
    void warm_start() {
        for (uint32_t o = 0; o < man.size(); o++) {
            const BMan& m = man[corder[o]];
            const uint32_t sa = m.sa, sbi = m.sb;
            P3 va = sv[sa], wa = sw[sa], vb = sv[sbi], wb = sw[sbi];
            float pn = 0.0f;
            for (uint32_t k = 0; k < m.cnt; k++) {
                const BCp& c = m.cp[k];
                pn += c.jn; wa = wa - c.iaxn * c.jn; wb = wb + c.ibxn * c.jn;
            }
            P3 p = m.n * pn + m.t1 * m.jt1 + m.t2 * m.jt2;
            va = va - p * m.ima; vb = vb + p * m.imb;
            wa = wa - (m.ia1 * m.jt1 + m.ia2 * m.jt2 + m.ian * m.jtw);
            wb = wb + (m.ib1 * m.jt1 + m.ib2 * m.jt2 + m.ibn * m.jtw);
            sv[sa] = va; sw[sa] = wa; sv[sbi] = vb; sw[sbi] = wb;
            sv[0] = p3(0, 0, 0); sw[0] = p3(0, 0, 0);
        }
    }

    // phys.rs:265-324
    void solve(bool use_bias, float inv_h, float bias_rate, float mass_scale, float imp_scale) {
        const float max_push = prm.max_push, ap = prm.anchor_push, slop = prm.anchor_slop;
        for (uint32_t o = 0; o < man.size(); o++) {
            BMan& m = man[corder[o]];
            const uint32_t sa = m.sa, sbi = m.sb;
            P3 va = sv[sa], wa = sw[sa], vb = sv[sbi], wb = sw[sbi];
            const P3 tha = sth[sa], thb = sth[sbi];
            const P3 n = m.n, t1 = m.t1, t2 = m.t2;
            const P3 dpab = sdp[sbi] - sdp[sa];
            const float dn = pdot(dpab, n);
            const float ima = m.ima, imb = m.imb;
            float tot = 0.0f;
            for (uint32_t k = 0; k < m.cnt; k++) {
                BCp& c = m.cp[k];
                float s = c.adj + dn + pdot(thb, c.rbxn) - pdot(tha, c.raxn);
                float bias, ms, is;
                if (s > 0.0f) { bias = s * inv_h; ms = 1.0f; is = 0.0f; }
                else if (use_bias) { bias = maxf(bias_rate * s, -max_push); ms = mass_scale; is = imp_scale; }
                else { bias = 0.0f; ms = 1.0f; is = 0.0f; }
                float vn = pdot(vb - va, n) + pdot(wb, c.rbxn) - pdot(wa, c.raxn);
                float imp = -c.nm * ms * (vn + bias) - is * c.jn;
                float nj = maxf(c.jn + imp, 0.0f);
                imp = nj - c.jn; c.jn = nj; tot += nj;
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
                float e1 = pdot(m.e0, t1) + pdot(dpab, t1) + pdot(thb, m.cb1) - pdot(tha, m.ca1);
                float e2 = pdot(m.e0, t2) + pdot(dpab, t2) + pdot(thb, m.cb2) - pdot(tha, m.ca2);
                auto sl = [&](float e) { return e > slop ? e - slop : (e < -slop ? e + slop : 0.0f); };
                b1 = minf(maxf(bias_rate * sl(e1), -ap), ap);
                b2 = minf(maxf(bias_rate * sl(e2), -ap), ap);
                ms = mass_scale; is = imp_scale;
            }
            const float o1 = m.jt1, o2 = m.jt2;
            float j1 = o1 - m.tm1 * ms * (v1 + b1) - is * o1;
            float j2 = o2 - m.tm2 * ms * (v2 + b2) - is * o2;
            const float l2 = j1 * j1 + j2 * j2;
            if (l2 > lim * lim) { float kf = lim / sqrt_e(l2); j1 *= kf; j2 *= kf; m.stick = false; }
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
            sv[sa] = va; sw[sa] = wa; sv[sbi] = vb; sw[sbi] = wb;
            sv[0] = p3(0, 0, 0); sw[0] = p3(0, 0, 0);
        }
    }

    // phys.rs:326-354
    void sleep_islands(float dt) {
        const uint32_t n = (uint32_t)bodies.size();
        std::vector<uint32_t> uf(n);
        for (uint32_t i = 0; i < n; i++) uf[i] = i;
        auto find = [&](uint32_t x) { while (uf[x] != x) { uint32_t p = uf[uf[x]]; uf[x] = p; x = p; } return x; };
        for (const BMan& m : man) {
            if (m.sa == 0 || m.sb == 0) continue;
            uint32_t ra = find(m.a), rb = find(m.b);
            if (ra != rb) uf[ra] = rb;
        }
        const float l2 = prm.sleep_lin * prm.sleep_lin, a2 = prm.sleep_ang * prm.sleep_ang;
        for (BBody& b : bodies) {
            if (!b.awake) continue;
            Q4 dq = qmul(b.q, q4(-b.sleep_q.x, -b.sleep_q.y, -b.sleep_q.z, b.sleep_q.w));
            float ang = 2.0f * sqrt_e(dq.x * dq.x + dq.y * dq.y + dq.z * dq.z);
            bool near = plen2(b.p - b.sleep_p) < prm.sleep_dist * prm.sleep_dist && ang < prm.sleep_rot;
            if (near && plen2(b.v) < 100.0f * l2 && plen2(b.w) < 100.0f * a2) b.sleep_t += dt;
            else { b.sleep_t = 0.0f; b.sleep_p = b.p; b.sleep_q = b.q; }
        }
        if (!prm.allow_sleep) return;
        std::vector<float> min_t(n, 3.4028235e38f);
        for (uint32_t i = 0; i < n; i++) if (bodies[i].awake) { uint32_t r = find(i); min_t[r] = minf(min_t[r], bodies[i].sleep_t); }
        for (uint32_t i = 0; i < n; i++) {
            if (!bodies[i].awake) continue;
            uint32_t r = find(i);
            if (min_t[r] >= prm.sleep_time) { BBody& b = bodies[i]; b.awake = false; b.v = p3(0, 0, 0); b.w = p3(0, 0, 0); }
        }
    }

    // the AABB-overlap pairs of the hashed grid (phys.rs:356-408), in hash-slot order, a < b
    void broadphase(std::vector<std::pair<uint32_t, uint32_t>>& pairs) {
        const uint32_t n = (uint32_t)bodies.size();
        const float inv_cell = 1.0f / prm.cell;
        struct Ent { uint32_t h, i; int32_t c[3]; };
        std::vector<Ent> tmp;
        for (uint32_t i = 0; i < n; i++) {
            const BBody& b = bodies[i];
            int32_t c0[3] = {bcell(b.amin.x, inv_cell), bcell(b.amin.y, inv_cell), bcell(b.amin.z, inv_cell)};
            int32_t c1[3] = {bcell(b.amax.x, inv_cell), bcell(b.amax.y, inv_cell), bcell(b.amax.z, inv_cell)};
            for (int32_t x = c0[0]; x <= c1[0]; x++) for (int32_t y = c0[1]; y <= c1[1]; y++) for (int32_t z = c0[2]; z <= c1[2]; z++)
                tmp.push_back(Ent{bhash(x, y, z), i, {x, y, z}});
        }
        const size_t ne = tmp.size();
        size_t tbl = 1; while (tbl < ne * 2) tbl <<= 1;
        const uint32_t mask = (uint32_t)(tbl - 1);
        std::vector<uint32_t> cnt(tbl + 1, 0);
        for (const Ent& e : tmp) cnt[(e.h & mask) + 1]++;
        for (size_t k = 0; k < tbl; k++) cnt[k + 1] += cnt[k];
        std::vector<Ent> ent(ne);
        std::vector<uint32_t> fill(cnt.begin(), cnt.begin() + tbl);
        for (const Ent& e : tmp) ent[fill[e.h & mask]++] = e;
        for (size_t s = 0; s < tbl; s++) {
            const uint32_t lo = cnt[s], hi = cnt[s + 1];
            if (hi - lo < 2) continue;
            for (uint32_t x = lo; x < hi; x++) for (uint32_t y = x + 1; y < hi; y++) {
                const Ent &ea = ent[x], &eb = ent[y];
                if (ea.c[0] != eb.c[0] || ea.c[1] != eb.c[1] || ea.c[2] != eb.c[2] || ea.i == eb.i) continue;
                const BBody &a = bodies[ea.i], &b = bodies[eb.i];
                if (!a.awake && !b.awake) continue;
                if (a.inv_m == 0.0f && b.inv_m == 0.0f) continue;
                if (a.amin.x > b.amax.x || b.amin.x > a.amax.x || a.amin.y > b.amax.y || b.amin.y > a.amax.y ||
                    a.amin.z > b.amax.z || b.amin.z > a.amax.z) continue;
                P3 m = pmax(a.amin, b.amin);
                if (bcell(m.x, inv_cell) != ea.c[0] || bcell(m.y, inv_cell) != ea.c[1] || bcell(m.z, inv_cell) != ea.c[2]) continue;
                pairs.push_back(ea.i < eb.i ? std::make_pair(ea.i, eb.i) : std::make_pair(eb.i, ea.i));
            }
        }
    }

    // phys.rs:410-417
    void wake(uint32_t i) {
        BBody& b = bodies[i];
        if (b.awake || b.inv_m == 0.0f) return;
        b.awake = true; b.sleep_t = 0.0f; b.sleep_p = b.p; b.sleep_q = b.q;
    }
    // phys.rs:419-432: the corners below the margin, at half their height, depth = their height
    HullShape hshape(const BBody& b) const { return HullShape{b.p, b.rot, b.h, hulls.data() + (size_t)b.hull * 320}; }
    // a contact of the convex-cell SAT, reduced to 4 points (gpu/gpu_world.js:532-554, in emit), pushed as a manifold
    void push_hc(uint32_t a, uint32_t b, HC c) {
        hc_reduce4(c);
        CP pts[8];
        for (int k = 0; k < c.cnt; k++) { pts[k].p = p3(c.pt[k][0], c.pt[k][1], c.pt[k][2]); pts[k].s = c.pt[k][3]; }
        push_manifold(a, b, c.n, pts, c.cnt);
    }
    // a convex cell on the ground (gpu/gpu_world.js:809-823): the corners under the margin; past four, the rest are a
    // second patch, emitted first; `which` = 1 the second patch only, 2 the first only, 3 both
    void collide_ground_cell(uint32_t i, int which) {
        const BBody& b = bodies[i];
        const float margin = prm.speculative + maxf(-b.v.y, 0.0f) * (1.0f / 60.0f);
        HC c = hull_ground(hshape(b), margin);
        if (c.cnt > 4) {
            HC c2; c2.n = c.n; c2.cnt = c.cnt - 4;
            for (int q = 0; q < c2.cnt; q++) for (int t = 0; t < 4; t++) c2.pt[q][t] = c.pt[4 + q][t];
            c.cnt = 4;
            if (which & 1) push_hc(i, BGROUND2, c2);
        }
        if (c.cnt > 0 && (which & 2)) push_hc(i, BNONE, c);
    }
    void collide_ground(uint32_t i) {
        const BBody& b = bodies[i];
        if (b.hull) { collide_ground_cell(i, 3); return; }
        CP pts[8]; int cnt = 0;
        const float margin = prm.speculative + maxf(-b.v.y, 0.0f) * (1.0f / 60.0f);
        for (int k = 0; k < 8; k++) {
            P3 s = p3(k & 1 ? 1.0f : -1.0f, k & 2 ? 1.0f : -1.0f, k & 4 ? 1.0f : -1.0f);
            P3 c = b.p + m_mulv(b.rot, p3(s.x * b.h.x, s.y * b.h.y, s.z * b.h.z));
            if (c.y < margin) { pts[cnt].p = p3(c.x, 0.5f * c.y, c.z); pts[cnt].s = c.y; cnt++; }
        }
        if (cnt == 0) return;
        const P3 n = p3(0.0f, -1.0f, 0.0f);
        cnt = reduce4(pts, cnt, n);
        push_manifold(i, BNONE, n, pts, cnt);
    }
    // phys.rs:434-445; `defer` collects the wakes (applied after all pairs) instead of waking at once: the woken set
    // and every manifold are the same either way, since a wake only ever turns a sleeping body awake.
    void collide_pair(uint32_t ia, uint32_t ib, std::vector<uint8_t>* defer) {
        const BBody &a = bodies[ia], &b = bodies[ib];
        const bool a_awake = a.awake, b_awake = b.awake, a_still = a.sleep_t != 0.0f, b_still = b.sleep_t != 0.0f;
        const float rel = plen_e(b.v - a.v) + plen_e(a.w) * plen_e(a.h) + plen_e(b.w) * plen_e(b.h);
        const float margin = prm.speculative + rel * (1.0f / 60.0f);
        if (a.hull || b.hull) {       // a pair with a convex cell (gpu/gpu_world.js:824-832); a box is the whole cube
            HC c = hull_hull(hshape(a), hshape(b), margin);
            if (c.cnt == 0) return;
            if (a_awake && !b_awake && !a_still) { if (defer) (*defer)[ib] = 1; else wake(ib); }
            if (b_awake && !a_awake && !b_still) { if (defer) (*defer)[ia] = 1; else wake(ia); }
            push_hc(ia, ib, c);
            return;
        }
        CP pts[8]; P3 n;
        int cnt = collide_boxes(a.p, a.rot, a.h, b.p, b.rot, b.h, margin, pts, &n);
        if (cnt == 0) return;
        if (a_awake && !b_awake && !a_still) { if (defer) (*defer)[ib] = 1; else wake(ib); }
        if (b_awake && !a_awake && !b_still) { if (defer) (*defer)[ia] = 1; else wake(ia); }
        cnt = reduce4(pts, cnt, n);
        push_manifold(ia, ib, n, pts, cnt);
    }
    // phys.rs:447-497
    void push_manifold(uint32_t a, uint32_t b, P3 n, const CP* pts, int cnt) {
        const BBody& ba = bodies[a];
        const P3 pa = ba.p; const M3 ra = ba.rot;
        const P3 pb = !bground(b) ? bodies[b].p : p3(0, 0, 0);
        const uint32_t sa = sidx[a], sbi = !bground(b) ? sidx[b] : 0;
        if (sa == 0 && sbi == 0) return;
        BMan m{};
        m.a = a; m.b = b; m.sa = sa; m.sb = sbi; m.n = n; btangents(n, m.t1, m.t2); m.mu = prm.friction;
        m.cnt = (uint32_t)cnt; m.stick = prm.anchor != 0;
        auto it = old_map.find(bkey(a, b));
        const BMan* o = it == old_map.end() ? nullptr : &old[it->second];
        M3 rbm; rbm.c[0] = p3(1, 0, 0); rbm.c[1] = p3(0, 1, 0); rbm.c[2] = p3(0, 0, 1);
        if (!bground(b)) rbm = bodies[b].rot;
        P3 cen = p3(0, 0, 0);
        for (int k = 0; k < cnt; k++) cen = cen + pts[k].p;
        cen = cen * (1.0f / (float)cnt);
        float rad = 0.0f;
        for (int k = 0; k < cnt; k++) rad += plen_e(pts[k].p - cen);
        m.rad = rad / (float)cnt;
        bool anchored = false;
        if (o) {
            if (o->stick) {
                P3 wa = pa + m_mulv(ra, o->la_f);
                P3 wb = !bground(b) ? pb + m_mulv(rbm, o->lb_f) : o->lb_f;
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
            m.lb_f = !bground(b) ? m_tmulv(rbm, m.fb) : cen;
            m.e0 = p3(0, 0, 0);
        }
        for (int k = 0; k < cnt; k++) {
            BCp& c = m.cp[k];
            c.ra = pts[k].p - pa;
            c.rb = !bground(b) ? pts[k].p - pb : pts[k].p;
            c.adj = pts[k].s;
            c.la = m_tmulv(ra, c.ra);
            if (o) {
                float best = 0.03f * 0.03f; int bi = -1;
                for (uint32_t q = 0; q < o->cnt; q++) { float d = plen2(o->cp[q].la - c.la); if (d < best) { best = d; bi = (int)q; } }
                if (bi >= 0) c.jn = o->cp[bi].jn;
            }
        }
        man.push_back(m);
    }

    void collide_all(float) {
        const uint32_t n = (uint32_t)bodies.size();
        std::vector<std::pair<uint32_t, uint32_t>> pairs;
        if (order == BOX_LIST) {                     // phys.rs:361-407
            for (uint32_t i = 0; i < n; i++) if (bodies[i].awake && bodies[i].amin.y < 0.0f) collide_ground(i);
            broadphase(pairs);
            st_pairs = (uint32_t)pairs.size();
            for (auto& pr : pairs) collide_pair(pr.first, pr.second, nullptr);
            return;
        }
        // key order: for each a its pairs (a, b) by b, then its ground manifold (a, NONE)
        std::vector<uint8_t> ground(n, 0), defer(n, 0);
        for (uint32_t i = 0; i < n; i++) ground[i] = bodies[i].awake && bodies[i].amin.y < 0.0f;
        broadphase(pairs);
        st_pairs = (uint32_t)pairs.size();
        std::sort(pairs.begin(), pairs.end());
        size_t q = 0;
        for (uint32_t a = 0; a < n; a++) {
            for (; q < pairs.size() && pairs[q].first == a; q++) collide_pair(a, pairs[q].second, &defer);
            if (ground[a]) collide_ground(a);
        }
        for (uint32_t i = 0; i < n; i++) if (defer[i]) wake(i);
    }

    // greedy colouring in descending priority (pair_priority of the key, then the earlier manifold first); a colour
    // is shared only by manifolds with no moving body in common
    void colour_manifolds() {
        const uint32_t M = (uint32_t)man.size();
        std::vector<uint64_t> rank(M);
        for (uint32_t k = 0; k < M; k++) {
            const BMan& m = man[k];
            rank[k] = ((uint64_t)pair_priority(m.a, bground(m.b) ? 0u : m.b + 1) << 32) | (uint64_t)(0xFFFFFFFFu - k);
        }
        std::vector<uint32_t> by(M);
        for (uint32_t k = 0; k < M; k++) by[k] = k;
        std::sort(by.begin(), by.end(), [&](uint32_t x, uint32_t y) { return rank[x] > rank[y]; });
        std::vector<std::vector<uint64_t>> used(sv.size());
        auto has = [&](uint32_t s, uint32_t c) { return s != 0 && c / 64 < used[s].size() && (used[s][c / 64] >> (c % 64)) & 1; };
        auto put = [&](uint32_t s, uint32_t c) {
            if (s == 0) return;
            if (used[s].size() <= c / 64) used[s].resize(c / 64 + 1, 0);
            used[s][c / 64] |= 1ull << (c % 64);
        };
        for (uint32_t k : by) {
            BMan& m = man[k];
            uint32_t c = 0;
            while (has(m.sa, c) || has(m.sb, c)) c++;
            m.colour = c;
            put(m.sa, c); put(m.sb, c);
            ncolours = std::max(ncolours, c + 1);
        }
        std::stable_sort(corder.begin(), corder.end(), [&](uint32_t x, uint32_t y) { return man[x].colour < man[y].colour; });
    }
};

}  // namespace

extern "C" {

// boxes: n records of p3 q4 h3 density (World::add_box)
void* obx_create(const float* boxes, uint32_t n, const void* params, int32_t order) {
    BoxWorld* w = new BoxWorld();
    std::memcpy(&w->prm, params, sizeof(BoxParams));
    w->order = order;
    for (uint32_t i = 0; i < n; i++) {
        const float* b = boxes + (size_t)i * 11;
        w->add_box(p3(b[0], b[1], b[2]), q4(b[3], b[4], b[5], b[6]), p3(b[7], b[8], b[9]), b[10]);
    }
    return w;
}
void obx_destroy(void* w) { delete (BoxWorld*)w; }
// the convex-cell library (n cells of 320 floats) and a cell per box (0 = a plain box)
void obx_set_hulls(void* wp, const float* data, uint32_t n, const uint32_t* ids) {
    BoxWorld* w = (BoxWorld*)wp;
    w->hulls.assign(data, data + (size_t)n * 320);
    for (size_t i = 0; i < w->bodies.size(); i++) w->bodies[i].hull = ids[i];
}
void obx_step(void* w, float dt, uint32_t nsteps) { for (uint32_t k = 0; k < nsteps; k++) ((BoxWorld*)w)->step(dt); }
// 22 floats a body: p3 q4 v3 w3 sleep_t sleep_p3 sleep_q4 awake
void obx_read(void* wp, float* out) {
    BoxWorld* w = (BoxWorld*)wp;
    for (size_t i = 0; i < w->bodies.size(); i++) {
        const BBody& b = w->bodies[i];
        float r[22] = {b.p.x, b.p.y, b.p.z, b.q.x, b.q.y, b.q.z, b.q.w, b.v.x, b.v.y, b.v.z, b.w.x, b.w.y, b.w.z,
                       b.sleep_t, b.sleep_p.x, b.sleep_p.y, b.sleep_p.z, b.sleep_q.x, b.sleep_q.y, b.sleep_q.z, b.sleep_q.w,
                       b.awake ? 1.0f : 0.0f};
        std::memcpy(out + i * 22, r, sizeof(r));
    }
}
// awake, pairs, manifolds, points, colours
void obx_stats(void* wp, uint32_t* out) {
    BoxWorld* w = (BoxWorld*)wp;
    out[0] = w->st_awake; out[1] = w->st_pairs; out[2] = w->st_manifolds; out[3] = w->st_points; out[4] = w->ncolours;
}
// 16 words a manifold in list order: a, b, cnt, stick, n3, jn4, jt1, jt2, jtw, colour (floats as bits)
uint32_t obx_manifolds(void* wp, uint32_t* out, uint32_t cap) {
    BoxWorld* w = (BoxWorld*)wp;
    uint32_t k = 0;
    for (; k < w->man.size() && k < cap; k++) {
        const BMan& m = w->man[k];
        float f[12] = {m.n.x, m.n.y, m.n.z, m.cp[0].jn, m.cp[1].jn, m.cp[2].jn, m.cp[3].jn, m.jt1, m.jt2, m.jtw, 0, 0};
        uint32_t* o = out + (size_t)k * 16;
        o[0] = m.a; o[1] = m.b; o[2] = m.cnt; o[3] = m.stick;
        std::memcpy(o + 4, f, 10 * sizeof(float));
        o[14] = m.colour; o[15] = 0;
    }
    return (uint32_t)w->man.size();
}

}  // extern "C"

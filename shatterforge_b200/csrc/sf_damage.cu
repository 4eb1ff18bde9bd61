// Damage on contact: impact_damage and crush_at (src/lib.rs:1602-1702) with damage_brick, sever_brick and
// remove_brick (src/lib.rs:705-752), once per substep between the pinch clamps and integration, as the reference's
// substep orders them (src/lib.rs:1780-1782).
//
// The energy a contact absorbed in the substep, E = 1/2 jn vn0, is split between its two bricks in proportion to how
// easily each crushes (1 / EB), and each side spends its share crushing its body's (or its structure's) bricks
// nearest the contact point, growing outward through intact bonds; the brick it cannot afford is cracked instead.
// A crushed brick is ground away (removed) with probability PULV of its material, else it is severed from its
// neighbours. Removed and severed static bricks leave their structure pending a connectivity walk; a body that loses
// or severs a brick is marked for rebuild_body. The walk is sequential in the reference (a crush changes what later
// contacts find, and one budget of 2,500 bricks a substep is shared in list order), so it runs in one thread over the
// contacts a parallel pass has already filtered and compacted in list order.
//
// Random numbers: the reference draws the pulverisation test from its world stream (src/lib.rs:1687), whose position
// also depends on dust and shard effects outside this path; here each draw is h01 (src/lib.rs:341-345) of a fixed
// seed and the scene's draw count. Dust, shards, impact events and the per-body impulse tally are effects outside
// the path and are left out.
#include <algorithm>
#include <cstring>
#include <vector>

#include "sf_internal.cuh"

namespace sf {

constexpr uint32_t BODY_REF = 0x80000000u;      // a brick reference: static id, or BODY_REF | body-brick id
constexpr uint32_t CRUSH_QUEUE = 4096;          // >= 1 + 6 x 600: the ring growth's queue for one crush
constexpr uint32_t CRUSH_MAX = 600;
constexpr uint32_t DRAW_SEED = 0x243F6A88u;

struct DamageState {
    DBuf<uint32_t> flag, pos, cand, ncand, stamp_s, stamp_k, scratch, scene_draws, counters;
    DBuf<uint8_t> hit;
    // plough: per static brick the contact that knocked it loose (NONE), per substep's new body its static brick, id,
    // pose and spin (at most the spare bodies), the per-scene ranges and use, the substep's counts
    DBuf<uint32_t> p_at, p_loose, p_newb, p_sc, p_count;
    DBuf<float> p_pose;
    DBuf<float4> p_spin;
    uint64_t ploughed = 0, scraped = 0;   // since the last read
    bool ready = false;
};

struct DamageArgs {
    const uint32_t *cand, *ncand;
    const uint32_t *L_a, *L_b, *L_bo, *L_ba, *L_bb, *invperm;
    const float4 *L_p, *S_j, *S_rb;
    const uint32_t *b_scene;
    const uint8_t *alive;
    uint8_t *s_mat;
    const uint32_t *s_cell, *s_scene, *s_nb6, *ctab;
    uint32_t *cpool;
    const int32_t *s_sid;
    float *s_bond;
    const float *s_bmax;
    uint8_t *k_mat;
    const uint32_t *k_body, *k_nb6;
    const float4 *k_wpos;
    float *k_bond;
    const float *k_bmax;
    uint8_t *b_dirty, *st_conn, *st_hit;
    uint32_t nst;
    uint32_t *stamp_s, *stamp_k, *scratch, *scene_draws, *counters;
};

__device__ __forceinline__ float h01_d(uint32_t h, uint32_t k) {
    uint32_t x = h + k * 0x9E3779B9u;
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return __uint2float_rn(x >> 8) / 16777216.0f;
}

// the brick-level operations on a reference; a body brick of a body that is no longer alive (removed by the pinch
// clamp this substep) reads as removed, as kill_body leaves it
struct Bricks {
    const DamageArgs &A;
    __device__ bool is_body(uint32_t r) const { return (r & BODY_REF) != 0; }
    __device__ uint32_t idx(uint32_t r) const { return r & ~BODY_REF; }
    __device__ uint8_t mat(uint32_t r) const {
        if (!is_body(r)) return A.s_mat[r];
        const uint32_t k = idx(r);
        return A.alive[A.k_body[k]] ? A.k_mat[k] : 0;
    }
    __device__ uint32_t body(uint32_t r) const { return is_body(r) ? A.k_body[idx(r)] : STATIC; }
    __device__ int32_t sid(uint32_t r) const { return is_body(r) ? -1 : A.s_sid[r]; }
    __device__ V3 pos(uint32_t r) const {
        if (is_body(r)) { const float4 p = A.k_wpos[idx(r)]; return v3(p.x, p.y, p.z); }
        int x, y, z;
        unpack_cell(A.s_cell[r], x, y, z);
        return lat_pos(x, y, z);
    }
    __device__ uint32_t nbr(uint32_t r, int d) const {
        if (is_body(r)) { const uint32_t j = A.k_nb6[(size_t)idx(r) * 6 + d]; return j == NONE ? NONE : (BODY_REF | j); }
        return A.s_nb6[(size_t)r * 6 + d];
    }
    __device__ float &bond(uint32_t r, int a) const {
        return is_body(r) ? A.k_bond[(size_t)idx(r) * 4 + a] : A.s_bond[(size_t)r * 4 + a];
    }
    __device__ float bmax(uint32_t r, int a) const {
        return is_body(r) ? A.k_bmax[(size_t)idx(r) * 4 + a] : A.s_bmax[(size_t)r * 4 + a];
    }
    // linked (src/lib.rs:378-383)
    __device__ uint32_t linked(uint32_t r, int d) const {
        const uint32_t j = nbr(r, d);
        if (j == NONE || mat(j) == 0 || body(j) != body(r)) return NONE;
        const float hp = (d & 1) == 0 ? bond(r, d >> 1) : bond(j, d >> 1);
        return hp > 0.0f ? j : NONE;
    }
    __device__ void pending(int32_t s) const { if (s >= 0 && (uint32_t)s < A.nst) A.st_conn[s] = 1; }
    __device__ void activate(int32_t s) const { if (s >= 0 && (uint32_t)s < A.nst) A.st_hit[s] = 1; }
    // remove_brick (src/lib.rs:705-718)
    __device__ void remove(uint32_t r) const {
        if (mat(r) == 0) return;
        if (is_body(r)) {
            A.k_mat[idx(r)] = 0;
            A.b_dirty[body(r)] = 1;
            return;
        }
        int x, y, z;
        unpack_cell(A.s_cell[r], x, y, z);
        const uint32_t t = A.ctab[(size_t)A.s_scene[r] * NCT + chunk_slot(x, y, z)];
        if (t) {
            uint32_t &g = A.cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
            if (g == r + 1) g = 0;
        }
        A.s_mat[r] = 0;
        pending(A.s_sid[r]);
        activate(A.s_sid[r]);
    }
    // sever_brick (src/lib.rs:746-752)
    __device__ void sever(uint32_t r) const {
        for (int a = 0; a < 4; a++) bond(r, a) = 0.0f;
        for (int d = 1; d < 6; d += 2) {
            const uint32_t j = nbr(r, d);
            if (j != NONE) bond(j, d >> 1) = 0.0f;
        }
    }
    // damage_brick (src/lib.rs:724-745): returns the bonds it broke
    __device__ uint32_t damage(uint32_t r, float frac, float absolute) const {
        uint32_t broke = 0;
        for (int d = 0; d < 6; d++) {
            const uint32_t j = nbr(r, d);
            if (j == NONE || mat(j) == 0) continue;
            const uint32_t o = (d & 1) == 0 ? r : j;
            const int a = d >> 1;
            float &b = bond(o, a);
            if (b > 0.0f) {
                const float bm = bmax(o, a);
                b -= bm * frac + absolute;
                if (b <= bm * 0.03f) { b = 0.0f; broke++; }
            }
        }
        float &b3 = bond(r, 3);
        if (b3 > 0.0f) {
            b3 -= bmax(r, 3) * frac * 0.5f + absolute * 0.5f;
            if (b3 <= 0.0f) { b3 = 0.0f; broke++; }
        }
        if (!is_body(r)) {
            activate(A.s_sid[r]);
            if (broke > 0) pending(A.s_sid[r]);
        } else if (broke > 0) A.b_dirty[body(r)] = 1;
        return broke;
    }
};

// crush_at (src/lib.rs:1641-1702): e spent on the bricks of start's body (or structure) nearest p, ring by ring
__device__ uint32_t crush_at(const Bricks &K, uint32_t start, float e, V3 p, uint32_t cap, uint32_t *stamp_ctr,
                             uint32_t *queue, uint32_t *lst, uint32_t *draws) {
    const DamageArgs &A = K.A;
    const uint8_t m0 = K.mat(start);
    if (m0 == 0 || m0 >= SLUG) return 0;
    if (e < c_mat.eb[m0] * 0.15f) return 0;
    const uint32_t body = K.body(start);
    const int32_t sid = K.sid(start);
    const uint32_t st = ++(*stamp_ctr);
    auto stamp = [&](uint32_t r) -> uint32_t & { return K.is_body(r) ? A.stamp_k[K.idx(r)] : A.stamp_s[r]; };
    queue[0] = start;
    uint32_t qn = 1, head = 0, crushed = 0, ncr = 0;
    stamp(start) = st;
    const uint32_t maxn = min(cap, CRUSH_MAX);
    while (head < qn && crushed < maxn) {
        uint32_t best = head;
        float bd = 1e18f;
        const uint32_t lim = min(head + 24, qn);
        for (uint32_t t = head; t < lim; t++) {
            const V3 d = sub(K.pos(queue[t]), p);
            const float dd = dot(d, d);
            if (dd < bd) { bd = dd; best = t; }
        }
        const uint32_t sw = queue[head]; queue[head] = queue[best]; queue[best] = sw;
        const uint32_t i = queue[head];
        head++;
        const uint8_t m = K.mat(i);
        if (m == 0) continue;
        const float cost = c_mat.eb[m];
        if (e < cost) {
            K.damage(i, div_rn(0.6f * e, cost), 0.0f);
            atomicAdd(&A.counters[4], 1u);
            break;
        }
        e -= cost;
        lst[ncr++] = i;
        crushed++;
        for (int d = 0; d < 6; d++) {
            const uint32_t j = K.linked(i, d);
            if (j == NONE || stamp(j) == st || K.body(j) != body || K.sid(j) != sid) continue;
            if (qn >= CRUSH_QUEUE) break;
            stamp(j) = st;
            queue[qn++] = j;
        }
    }
    for (uint32_t t = 0; t < ncr; t++) {
        const uint32_t i = lst[t];
        const uint8_t m = K.mat(i);
        if (m == 0) continue;
        if (h01_d(DRAW_SEED, (*draws)++) < c_mat.pulv[m]) {
            K.remove(i);
            atomicAdd(&A.counters[2], 1u);
        } else {
            K.sever(i);
            atomicAdd(&A.counters[3], 1u);
            if (body == STATIC) { K.pending(A.s_sid[i]); K.activate(A.s_sid[i]); }
            else A.b_dirty[body] = 1;
        }
    }
    atomicAdd(&A.counters[1], crushed);
    return crushed;
}

// candidates: a body brick of a crushable material, and either enough energy to crush (vn0 >= 1, E >= 150 J) or a
// heavy hit on a static brick (jn vn0 > 4,000, which wakes the structure's load solver)
__global__ void k_dmg_flags(uint32_t nc, DamageArgs A, uint32_t *flag) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    const uint32_t t = A.invperm[k];
    if (t == NONE) { flag[k] = 0; return; }   // left out by the contact reduction: no impulse
    const float jn = A.S_j[t].x, vn0 = A.S_rb[t].w;
    const uint32_t ia = A.L_ba[k];
    const uint8_t ma = A.alive[A.k_body[ia]] ? A.k_mat[ia] : 0;
    bool on = ma != 0 && ma < SLUG;
    if (on) {
        const bool crush = vn0 >= 1.0f && 0.5f * jn * vn0 >= 150.0f;
        const bool heavy = A.L_bb[k] != NONE && A.L_bo[k] == STATIC && jn * vn0 > 4000.0f;
        on = crush || heavy;
    }
    flag[k] = on ? 1u : 0u;
}
__global__ void k_dmg_compact(uint32_t nc, const uint32_t *flag, const uint32_t *pos, uint32_t *cand) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nc && flag[k]) cand[pos[k]] = k;
}

// impact_damage (src/lib.rs:1610-1640) over the candidates in list order; one budget of 2,500 crushed bricks per
// scene and substep
__global__ void k_dmg_apply(DamageArgs A) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const Bricks K{A};
    const uint32_t n = *A.ncand;
    uint32_t *queue = A.scratch, *lst = A.scratch + CRUSH_QUEUE, *stamp_ctr = A.scratch + CRUSH_QUEUE + CRUSH_MAX;
    uint32_t scene = NONE, budget = 0;
    for (uint32_t c = 0; c < n; c++) {
        const uint32_t k = A.cand[c];
        const uint32_t a = A.L_a[k];
        const uint32_t q = A.b_scene[a];
        if (q != scene) { scene = q; budget = 2500; }
        const uint32_t t = A.invperm[k];
        const float jn = A.S_j[t].x, vn0 = A.S_rb[t].w;
        const uint32_t ia = BODY_REF | A.L_ba[k];
        const uint8_t ma = K.mat(ia);
        if (ma == 0 || ma >= SLUG) continue;
        atomicAdd(&A.counters[0], 1u);
        const uint32_t bbk = A.L_bb[k];
        if (bbk != NONE && A.L_bo[k] == STATIC && jn * vn0 > 4000.0f) {
            if (A.s_mat[bbk] != 0) K.activate(A.s_sid[bbk]);
        }
        if (vn0 < 1.0f) continue;
        const float e = 0.5f * jn * vn0;
        if (e < 150.0f) continue;
        const uint32_t jb = bbk == NONE ? NONE : (A.L_bo[k] == STATIC ? bbk : (BODY_REF | bbk));
        const uint8_t mb = jb != NONE ? K.mat(jb) : 0;
        const float soft_a = div_rn(1.0f, c_mat.eb[ma]);
        const float soft_b = (jb == NONE || mb == 0 || mb >= SLUG) ? 0.0f : div_rn(1.0f, c_mat.eb[mb]);
        if (soft_a + soft_b <= 0.0f) continue;
        const float ea = div_rn(e * soft_a, soft_a + soft_b);
        const float4 p4 = A.L_p[k];
        const V3 p = v3(p4.x, p4.y, p4.z);
        uint32_t *draws = &A.scene_draws[q];
        if (ea > 0.0f && budget > 0) budget -= min(crush_at(K, ia, ea, p, budget, stamp_ctr, queue, lst, draws), budget);
        if (soft_b > 0.0f && budget > 0) budget -= min(crush_at(K, jb, e - ea, p, budget, stamp_ctr, queue, lst, draws), budget);
    }
}

// ---------------------------------------------------------------- plough (src/lib.rs:1493-1550)
// After the contacts and before prep_contacts, in list order: a body driving into a static brick at 2 m/s or more with
// momentum min(3 m / max(contacts, 3), m) vn of at least 0.35 of the brick's vertical capacity damages it (a body of
// more than 40 bricks: damage_brick by mom / 1.5 CAPV within 0.15..0.9) or, while the scene has a spare body and
// brick, knocks it loose: severed, taken out of the static set (potential and load 0) and set up as a one-brick body
// with 0.75 of the body's velocity plus 2 m/s and a spin of 6 rad/s in random directions (rndv on the scene's damage
// draws); the body keeps m / (m + 1.5 MASS) of its velocity, and that contact and the later ones with the brick are
// switched off. A parallel pass keeps the contacts that could qualify (2 m/s reached with or without the body's
// velocity, which only shrinks; enough momentum at that speed); one thread walks them in order.
struct PloughArgs {
    uint32_t nc;
    const uint32_t *L_a, *L_b, *L_bo, *L_bb;
    const float4 *L_p, *L_n;
    const uint32_t *cand, *ncand;
    uint8_t *off;
    uint32_t *at;          // per static brick: the contact at which it was knocked loose, else NONE
    uint32_t *loose;       // the static bricks knocked loose this substep
    uint32_t *counters;    // [0] knocked loose, [1] scraped (damage_brick by a large body)
    const float4 *pos, *w;
    float4 *v;
    const float *m;
    const uint32_t *nc_b, *count;
    uint32_t *sc;          // per scene: body_off, bodies, brick_off, bricks, bodies used, bricks used
    int32_t *k_xyz;
    uint32_t *k_nb6, *b_first, *b_count;
    float *k_bmax;
    float *pose;           // per new body: pose 13 (origin, identity, velocity, no spin)
    float4 *spin;
    uint32_t *newb;
    float *s_phi, *s_ext;
    double *s_phi64;
};
__device__ __forceinline__ bool plough_kind(uint32_t b, uint32_t bo, uint32_t bb) {
    return b == STATIC && bo == STATIC && bb != NONE;
}
__global__ void k_plough_flags(PloughArgs P, DamageArgs A, uint32_t *flag) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.nc) return;
    uint32_t on = 0;
    if (plough_kind(P.L_b[k], P.L_bo[k], P.L_bb[k])) {
        const uint32_t j = P.L_bb[k], a = P.L_a[k];
        const uint8_t mj = A.s_mat[j];
        if (mj != 0 && mj < SLUG) {
            const float4 p4 = P.L_p[k], n4 = P.L_n[k], pa = P.pos[a], v4 = P.v[a], w4 = P.w[a];
            const V3 n = v3(n4.x, n4.y, n4.z);
            const V3 ra = sub(v3(p4.x, p4.y, p4.z), v3(pa.x, pa.y, pa.z));
            const float spin = -dot(cross(v3(w4.x, w4.y, w4.z), ra), n);
            const float full = -dot(add(v3(v4.x, v4.y, v4.z), cross(v3(w4.x, w4.y, w4.z), ra)), n);
            const float vmax = maxf(full, spin);
            const float mm = P.m[a];
            const float meff = mm * 3.0f / maxf((float)P.nc_b[a], 3.0f);
            on = vmax >= 1.99f && minf(meff, mm) * vmax >= c_mat.capv[mj] * 0.35f * 0.999f ? 1u : 0u;
        }
    }
    flag[k] = on;
}
// rndv (src/lib.rs:330-336) on the scene's draw sequence (a rejection loop; 64 tries fail with probability 1e-20)
__device__ V3 rndv_draw(uint32_t *ctr) {
    for (int t = 0; t < 64; t++) {
        const float x = h01_d(DRAW_SEED, (*ctr)++) * 2.0f - 1.0f;
        const float y = h01_d(DRAW_SEED, (*ctr)++) * 2.0f - 1.0f;
        const float z = h01_d(DRAW_SEED, (*ctr)++) * 2.0f - 1.0f;
        const V3 v = v3(x, y, z);
        const float l = dot(v, v);
        if (l > 0.01f && l <= 1.0f) return mul(v, div_rn(1.0f, sqrt_rn(l)));
    }
    return v3(0.0f, 1.0f, 0.0f);
}
__global__ void k_plough_apply(PloughArgs P, DamageArgs A) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const Bricks K{A};
    const uint32_t n = *P.ncand;
    for (uint32_t c = 0; c < n; c++) {
        const uint32_t k = P.cand[c];
        const uint32_t j = P.L_bb[k], a = P.L_a[k];
        if (A.s_mat[j] == 0) { P.off[k] = 1; continue; }   // knocked loose by an earlier contact of this pass
        const float4 p4 = P.L_p[k], n4 = P.L_n[k], pa = P.pos[a], v4 = P.v[a], w4 = P.w[a];
        const V3 ra = sub(v3(p4.x, p4.y, p4.z), v3(pa.x, pa.y, pa.z));
        const V3 va = v3(v4.x, v4.y, v4.z);
        const float vn = -dot(add(va, cross(v3(w4.x, w4.y, w4.z), ra)), v3(n4.x, n4.y, n4.z));
        if (vn < 2.0f) continue;
        const float mm = P.m[a];
        const float meff = mm * 3.0f / maxf((float)P.nc_b[a], 3.0f);
        const float mom = minf(meff, mm) * vn;
        const uint8_t mj = A.s_mat[j];
        if (mj >= SLUG || mom < c_mat.capv[mj] * 0.35f) continue;
        if (P.count[a] > 40) {
            K.damage(j, clampf(mom / (c_mat.capv[mj] * 1.5f), 0.15f, 0.9f), 0.0f);
            P.counters[1]++;
            continue;
        }
        const uint32_t q = A.b_scene[a];
        uint32_t *S = P.sc + (size_t)q * 6;
        if (S[4] + 1 > S[1] || S[5] + 1 > S[3]) continue;   // ensure_bodies
        K.sever(j);
        K.pending(A.s_sid[j]);
        K.activate(A.s_sid[j]);
        const V3 rv = rndv_draw(&A.scene_draws[q]);
        const V3 pv = madd(mul(va, 0.75f), rv, 2.0f);
        const V3 ww = mul(rndv_draw(&A.scene_draws[q]), 6.0f);
        const uint32_t b = S[0] + S[4]++, kk = S[2] + S[5]++;
        int x, y, z;
        unpack_cell(A.s_cell[j], x, y, z);
        P.k_xyz[3 * kk] = x; P.k_xyz[3 * kk + 1] = y; P.k_xyz[3 * kk + 2] = z;
        A.k_mat[kk] = mj;
        for (int d = 0; d < 6; d++) P.k_nb6[(size_t)kk * 6 + d] = NONE;
        for (int t = 0; t < 4; t++) {
            A.k_bond[(size_t)kk * 4 + t] = A.s_bond[(size_t)j * 4 + t];
            P.k_bmax[(size_t)kk * 4 + t] = A.s_bmax[(size_t)j * 4 + t];
        }
        P.b_first[b] = kk;
        P.b_count[b] = 1;
        K.remove(j);
        P.s_phi[j] = 0.0f; P.s_phi64[j] = 0.0; P.s_ext[j] = 0.0f;
        const uint32_t e = P.counters[0]++;
        float *po = P.pose + (size_t)e * 13;
        const float f13[13] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, pv.x, pv.y, pv.z, 0.0f, 0.0f, 0.0f};
        for (int t = 0; t < 13; t++) po[t] = f13[t];
        P.spin[e] = make_float4(ww.x, ww.y, ww.z, 0.0f);
        P.newb[e] = b;
        P.loose[e] = j;
        const V3 vs = mul(va, mm / (mm + c_mat.mass[mj] * 1.5f));
        P.v[a] = make_float4(vs.x, vs.y, vs.z, 0.0f);
        P.off[k] = 1;
        P.at[j] = k;
    }
}
// the contacts after the one that knocked their static brick loose are off
__global__ void k_plough_off(PloughArgs P) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.nc || !plough_kind(P.L_b[t], P.L_bo[t], P.L_bb[t])) return;
    const uint32_t k0 = P.at[P.L_bb[t]];
    if (k0 != NONE && k0 < t) P.off[t] = 1;
}
__global__ void k_plough_reset(uint32_t n, const uint32_t *loose, uint32_t *at) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) at[loose[e]] = NONE;
}
__global__ void k_plough_spin(uint32_t n, const uint32_t *newb, const float4 *spin, float4 *w) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) w[newb[e]] = spin[e];
}

void damage_destroy(sf_world *w) {
    delete w->damage;
    w->damage = nullptr;
}

static cudaError_t damage_ready(sf_world *w, cudaStream_t s) {
    if (!w->damage) w->damage = new DamageState();
    DamageState &D = *w->damage;
    cudaError_t e;
    if (!D.ready) {
        if ((e = upload_mat_tables(s)) != cudaSuccess) return e;
        if ((e = D.stamp_s.alloc(std::max<uint32_t>(w->ns, 1))) != cudaSuccess) return e;
        if ((e = D.stamp_k.alloc(std::max<uint32_t>(w->nd, 1))) != cudaSuccess) return e;
        if ((e = D.scratch.alloc(CRUSH_QUEUE + CRUSH_MAX + 1)) != cudaSuccess) return e;
        if ((e = D.scene_draws.alloc(std::max<uint32_t>(w->n_scenes, 1))) != cudaSuccess) return e;
        if ((e = D.counters.alloc(8)) != cudaSuccess) return e;
        if ((e = D.hit.alloc(std::max<uint32_t>(w->n_struct, 1))) != cudaSuccess) return e;
        if ((e = D.ncand.alloc(1)) != cudaSuccess) return e;
        cudaMemsetAsync(D.stamp_s.p, 0, D.stamp_s.bytes(), s);
        cudaMemsetAsync(D.stamp_k.p, 0, D.stamp_k.bytes(), s);
        cudaMemsetAsync(D.scratch.p, 0, D.scratch.bytes(), s);
        cudaMemsetAsync(D.scene_draws.p, 0, D.scene_draws.bytes(), s);
        cudaMemsetAsync(D.counters.p, 0, D.counters.bytes(), s);
        cudaMemsetAsync(D.hit.p, 0, D.hit.bytes(), s);
        uint32_t spare = 0;
        for (uint32_t q = 0; q < w->n_scenes; q++) spare += w->scenes[q].n_bodies;
        spare = std::max<uint32_t>(spare, 1);
        if ((e = D.p_at.alloc(std::max<uint32_t>(w->ns, 1))) != cudaSuccess) return e;
        if ((e = D.p_loose.alloc(spare)) != cudaSuccess) return e;
        if ((e = D.p_newb.alloc(spare)) != cudaSuccess) return e;
        if ((e = D.p_pose.alloc((size_t)spare * 13)) != cudaSuccess) return e;
        if ((e = D.p_spin.alloc(spare)) != cudaSuccess) return e;
        if ((e = D.p_sc.alloc((size_t)std::max<uint32_t>(w->n_scenes, 1) * 6)) != cudaSuccess) return e;
        if ((e = D.p_count.alloc(2)) != cudaSuccess) return e;
        cudaMemsetAsync(D.p_at.p, 0xFF, D.p_at.bytes(), s);
        D.ready = true;
    }
    return cudaGetLastError();
}
static void fill_damage_args(sf_world *w, DamageState &D, DamageArgs &A) {
    A.cand = D.cand.p; A.ncand = D.ncand.p;
    A.b_scene = w->b_scene.p; A.alive = w->b_alive.p;
    A.s_mat = w->s_mat.p; A.s_cell = w->s_cell.p; A.s_scene = w->s_scene.p; A.s_nb6 = w->s_nb6.p; A.ctab = w->ctab.p;
    A.cpool = w->cpool.p; A.s_sid = w->s_sid.p; A.s_bond = w->s_bond.p; A.s_bmax = w->s_bmax.p;
    A.k_mat = w->k_mat.p; A.k_body = w->k_body.p; A.k_nb6 = w->k_nb6.p; A.k_wpos = w->k_wpos.p; A.k_bond = w->k_bond.p;
    A.k_bmax = w->k_bmax.p; A.b_dirty = w->b_dirty.p; A.st_conn = w->st_conn.p; A.st_hit = D.hit.p;
    A.nst = w->n_struct;
    A.stamp_s = D.stamp_s.p; A.stamp_k = D.stamp_k.p; A.scratch = D.scratch.p; A.scene_draws = D.scene_draws.p;
    A.counters = D.counters.p;
}

cudaError_t plough_substep(sf_world *w, const PloughIn &in, cudaStream_t s, uint32_t *n_loose) {
    *n_loose = 0;
    cudaError_t e;
    if ((e = damage_ready(w, s)) != cudaSuccess) return e;
    if (in.nc == 0) return cudaSuccess;
    DamageState &D = *w->damage;
    if ((e = D.flag.grow(in.nc)) != cudaSuccess) return e;
    if ((e = D.pos.grow(in.nc)) != cudaSuccess) return e;
    if ((e = D.cand.grow(in.nc)) != cudaSuccess) return e;
    std::vector<uint32_t> sc((size_t)w->n_scenes * 6);
    for (uint32_t q = 0; q < w->n_scenes; q++) {
        const Scene &c = w->scenes[q];
        const uint32_t v[6] = {c.body_off, c.n_bodies, c.brick_off, c.n_bricks, c.bodies_used, c.bricks_used};
        for (int t = 0; t < 6; t++) sc[(size_t)q * 6 + t] = v[t];
    }
    if ((e = cudaMemcpyAsync(D.p_sc.p, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(in.off, 0, in.nc, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(D.p_count.p, 0, 8, s)) != cudaSuccess) return e;
    DamageArgs A;
    fill_damage_args(w, D, A);
    PloughArgs P;
    P.nc = in.nc; P.L_a = in.L_a; P.L_b = in.L_b; P.L_bo = in.L_bo; P.L_bb = in.L_bb; P.L_p = in.L_p; P.L_n = in.L_n;
    P.cand = D.cand.p; P.ncand = D.ncand.p; P.off = in.off; P.at = D.p_at.p; P.loose = D.p_loose.p;
    P.counters = D.p_count.p; P.pos = w->b_pos.p; P.w = w->b_w.p; P.v = w->b_v.p; P.m = w->b_m.p; P.nc_b = w->b_nc.p;
    P.count = w->b_count.p; P.sc = D.p_sc.p; P.k_xyz = w->k_xyz.p; P.k_nb6 = w->k_nb6.p; P.b_first = w->b_first.p;
    P.b_count = w->b_count.p; P.k_bmax = w->k_bmax.p; P.pose = D.p_pose.p; P.spin = D.p_spin.p; P.newb = D.p_newb.p;
    P.s_phi = w->s_phi.p; P.s_ext = w->s_ext.p; P.s_phi64 = w->s_phi64.p;
    const unsigned g = grid_for(in.nc, 256);
    k_plough_flags<<<g, 256, 0, s>>>(P, A, D.flag.p);
    if ((e = exclusive_scan_u32(D.flag.p, D.pos.p, in.nc, D.ncand.p, *in.wk, s)) != cudaSuccess) return e;
    k_dmg_compact<<<g, 256, 0, s>>>(in.nc, D.flag.p, D.pos.p, D.cand.p);
    k_plough_apply<<<1, 32, 0, s>>>(P, A);
    w->launches += 3;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    uint32_t cnt[2];
    if ((e = cudaMemcpyAsync(cnt, D.p_count.p, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    D.ploughed += cnt[0];
    D.scraped += cnt[1];
    if (cnt[0] == 0) return cudaSuccess;
    // the later contacts with those bricks are off; the new bodies are set up scene by scene (ids and poses run in
    // list order, so each scene's new bodies are consecutive), then given their spin
    k_plough_off<<<g, 256, 0, s>>>(P);
    k_plough_reset<<<grid_for(cnt[0], 256), 256, 0, s>>>(cnt[0], D.p_loose.p, D.p_at.p);
    w->launches += 2;
    std::vector<uint32_t> used(sc.size());
    if ((e = cudaMemcpyAsync(used.data(), D.p_sc.p, sc.size() * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    size_t at = 0;
    for (uint32_t q = 0; q < w->n_scenes; q++) {
        Scene &c = w->scenes[q];
        const uint32_t nq = used[(size_t)q * 6 + 4] - c.bodies_used;
        if (!nq) continue;
        const uint32_t b0 = c.body_off + c.bodies_used;
        if ((e = setup_bodies(w, b0, nq, D.p_pose.p + at * 13)) != cudaSuccess) return e;
        if ((e = step_reset_labels(w, b0, nq)) != cudaSuccess) return e;
        c.bodies_used = used[(size_t)q * 6 + 4];
        c.bricks_used = used[(size_t)q * 6 + 5];
        at += nq;
    }
    k_plough_spin<<<grid_for(cnt[0], 256), 256, 0, s>>>(cnt[0], D.p_newb.p, D.p_spin.p, w->b_w.p);
    w->launches++;
    *n_loose = cnt[0];
    return cudaGetLastError();
}

cudaError_t damage_substep(sf_world *w, const DamageIn &in, cudaStream_t s) {
    cudaError_t e;
    if ((e = damage_ready(w, s)) != cudaSuccess) return e;
    DamageState &D = *w->damage;
    if (in.nc == 0) return cudaSuccess;
    if ((e = D.flag.grow(in.nc)) != cudaSuccess) return e;
    if ((e = D.pos.grow(in.nc)) != cudaSuccess) return e;
    if ((e = D.cand.grow(in.nc)) != cudaSuccess) return e;
    DamageArgs A;
    fill_damage_args(w, D, A);
    A.L_a = in.L_a; A.L_b = in.L_b; A.L_bo = in.L_bo; A.L_ba = in.L_ba; A.L_bb = in.L_bb; A.invperm = in.invperm;
    A.L_p = in.L_p; A.S_j = in.S_j; A.S_rb = in.S_rb;
    k_dmg_flags<<<grid_for(in.nc, 256), 256, 0, s>>>(in.nc, A, D.flag.p);
    if ((e = exclusive_scan_u32(D.flag.p, D.pos.p, in.nc, D.ncand.p, *in.wk, s)) != cudaSuccess) return e;
    k_dmg_compact<<<grid_for(in.nc, 256), 256, 0, s>>>(in.nc, D.flag.p, D.pos.p, D.cand.p);
    k_dmg_apply<<<1, 32, 0, s>>>(A);
    w->launches += 3;
    return cudaGetLastError();
}

}  // namespace sf

using namespace sf;

extern "C" {

sf_status sf_read_damage(sf_world *w, sf_damage_report *report, uint8_t *activated) {
    if (!w) { set_error("null argument"); return SF_ERR_ARG; }
    sf_damage_report r{};
    if (w->damage && w->damage->ready) {
        DamageState &D = *w->damage;
        uint32_t c[8];
        SF_CUDA(cudaMemcpyAsync(c, D.counters.p, sizeof c, cudaMemcpyDeviceToHost, w->stream));
        if (activated && w->n_struct) SF_CUDA(cudaMemcpyAsync(activated, D.hit.p, w->n_struct, cudaMemcpyDeviceToHost, w->stream));
        SF_CUDA(cudaMemsetAsync(D.counters.p, 0, D.counters.bytes(), w->stream));
        SF_CUDA(cudaMemsetAsync(D.hit.p, 0, D.hit.bytes(), w->stream));
        SF_CUDA(cudaStreamSynchronize(w->stream));
        r.contacts = c[0]; r.crushed = c[1]; r.removed = c[2]; r.severed = c[3]; r.cracked = c[4];
        r.ploughed = D.ploughed; r.scraped = D.scraped;
        D.ploughed = D.scraped = 0;
    } else if (activated && w->n_struct) {
        std::memset(activated, 0, w->n_struct);
    }
    if (report) *report = r;
    return SF_OK;
}

}  // extern "C"

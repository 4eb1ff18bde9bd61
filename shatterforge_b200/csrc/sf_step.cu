// Rigid-body step over brick spheres (src/lib.rs:1367-1783), all scenes of a world per launch.
//
// One substep:
//   k_update_cache   rotation and world inverse inertia of awake bodies, then gravity       src/lib.rs:1368-1378, 1772
//   k_brick_pos      world position of each awake body's bricks                                src/lib.rs:1375
//   k_cell_keys      64-bit cell key (scene, hashed cell) of every live brick; radix-sorted, stable, so each
//                    bucket holds its bricks in ascending index order; k_bucket_ranges marks each bucket's range
//                    — the same 32768 buckets as build_hash (src/lib.rs:1379-1395), hash collisions included
//   k_contacts       count, scan, fill: every brick of an awake body finds its ground corners, static cells and
//                    hashed neighbours exactly as gen_contacts (src/lib.rs:1405-1471); walking each bucket from its
//                    highest index down reproduces the reference's chain order, so the filled list IS the
//                    reference's contact list order
//   manifolds        contacts grouped by body pair (a, b; b = static side for ground, static cells and sleeping
//                    partners) with a stable radix sort, so each manifold keeps its contacts in list order
//   k_prep           prep_contacts (src/lib.rs:1551-1577) per contact, written in manifold order
//   colouring        Jones-Plassmann rounds on the manifold conflict graph (two manifolds conflict when they share
//                    an awake body); priority = hash of the pair, ties to the lower manifold index; the smallest
//                    colour free at both bodies — the same colouring as a greedy pass in priority order
//   k_solve          persistent kernel: for each iteration, for each colour, each manifold's contacts solved in list
//                    order with solve()'s sequential-impulse math (src/lib.rs:1579-1601); a bounded grid barrier
//                    separates colours. Manifolds of one colour share no awake body, so the result does not
//                    depend on their order inside a colour.
//   islands          union-find over manifolds between two awake bodies, larger root linked under the smaller by
//                    CAS with path halving (gpu/gpu_world.js:1634-1655, engine/src/phys.rs:326-354)
//   k_integrate      pinch clamps (src/lib.rs:1746-1768) and integrate (src/lib.rs:1703-1742)
#include <algorithm>
#include <cstring>

#include "sf_internal.cuh"

namespace sf {

struct StepState {
    Work wk;
    // hashed cell sort
    DBuf<uint32_t> ckey, ckey_alt;   // per active brick: its hash key (active scene index x HSIZE + bucket) and rank
    DBuf<uint32_t> cval;             // the hash table's entries: brick ids, bucket by bucket
    DBuf<uint32_t> aw_flag, awk_pos, awk_list, bucket_bits, scene_awake, scene_bricks;
    uint32_t n_awk = 0;
    bool use_sparse = false, last_sparse = false;
    DBuf<uint32_t> bstart;          // the hash table: per (active scene, bucket) count, then start (+1 for the end)
    DBuf<float4> srec;
    DBuf<uint2> sent;
    DBuf<uint4> slot_id;
    DBuf<float4> slot_p, slot_n;
    // contacts, list order
    DBuf<uint32_t> ccount, coff;
    DBuf<uint32_t> L_a, L_b, L_bo, L_ba, L_bb;
    DBuf<float4> L_p, L_n;
    // manifold order
    DBuf<uint64_t> mkey, mkey_alt;
    DBuf<uint32_t> perm, perm_alt, invperm;
    DBuf<uint32_t> mflag, mpos, pair_start, cflag, cpos;
    DBuf<uint32_t> man_a, man_b, man_start, man_count, man_prio, man_color, man_round;
    DBuf<float4> S_n, S_t1, S_t2, S_ra, S_rb, S_j;
    // contact reduction: per pair a big flag and its place among the big pairs, per big pair 27 best scores and 27
    // winners, per sorted contact a keep flag and its place among the kept
    DBuf<uint32_t> red_big, red_pos, red_keep, red_kpos, red_slots;
    DBuf<uint8_t> c_off;            // per contact: switched off by plough this substep
    // warm start: two open-addressing tables (the last substep's, the one being written), keyed by contact key
    struct WarmTable { DBuf<uint32_t> claim; DBuf<unsigned long long> k1; DBuf<uint32_t> k2; DBuf<float4> val; uint32_t mask = 0; };
    WarmTable warm[2];
    int warm_cur = 0;                // the table the next substep reads
    bool warm_valid = false;
    std::vector<uint8_t> warm_scene; // per scene: its entries in the table still apply (no brick ids moved since)
    DBuf<uint8_t> warm_scene_dev;
    bool warm_scene_dirty = true;
    // colouring
    DBuf<uint32_t> bm_count, bm_start, bm_fill, bm_list;
    DBuf<uint32_t> masks, vmasks;
    DBuf<uint32_t> wl0, wl1;
    DBuf<uint32_t> col_count, col_hstart, col_start, col_fill, col_list, jds_off, seg_tot, seg_base;
    // sync domains: contiguous runs of active scenes, each coloured and solved by its own blocks with its own barrier
    // (scenes never share a body, so no colour or round of one domain waits for another's)
    DBuf<uint32_t> dom_of_act, man_dom, dom_m0, dom_m1, dom_ncol, dom_cnt;
    DBuf<uint4> blk_dom;           // per block of the colouring / solve launch: domain, rank in it, its block count
    DBuf<GridBarrier> dom_gb;
    struct Partition { unsigned R = 0; uint32_t D = 0; std::vector<uint4> blk; std::vector<uint32_t> dom_of_act; };
    std::vector<Partition> parts;  // by launch size, for the current active set
    uint32_t part_D = 1;           // domains of the partition in use this substep
    int part_in_use = -1;          // which of `parts` the device tables hold
    // islands
    DBuf<uint32_t> parent, label, mint;
    // per-scene body offsets (for scene-local priorities)
    DBuf<uint32_t> body_off_of_body;
    // the active set of the current step
    DBuf<uint32_t> act_body, act_brick, cidx, scene_act, man_ca, man_cb;
    DBuf<uint4> seg;
    DBuf<uint8_t> live_dev;
    uint8_t *h_live_pin = nullptr;          // pinned mirror of live_dev
    std::vector<uint8_t> live;              // per scene: an awake body at the end of the last step
    std::vector<uint32_t> act;              // active scenes, ascending
    std::vector<uint32_t> act_brick_base;   // per scene: first active-list brick of the last substep, NONE if idle
    uint32_t nb_act = 0, nd_act = 0;
    bool act_valid = false;
    // device scalars: [0] contacts, [1] manifolds, [2] colours, [3] rounds, [4..6] jp counts, [7] alive, [8] awake,
    // [9] islands
    DBuf<uint32_t> dev;
    uint32_t *h_dev = nullptr;   // pinned mirror
    uint64_t capacity = 0;
    uint64_t last_contacts = 0;
    int solve_occ = 1, jp_occ = 1;
    uint32_t max_scene_bodies = 0;
    // launch-shape tuning: pending timings of this step's tuned launches
    Tuner solve_t;
    struct Pending { Tuner *t; int bucket, ci; cudaEvent_t e0, e1; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> tev;
    size_t tev_used = 0;
    bool have_contacts = false;
    // profiling: PH_N + 1 events per substep, elapsed times folded in after each sf_world_step
    bool profile = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<uint32_t> sub_nc;
    double ph_ms[SF_PHASES] = {};
    uint64_t ph_substeps = 0, solve_contact_iters = 0, solve_launches = 0;
    // contact generation alone: an event pair per launch, folded in with the phases
    std::vector<cudaEvent_t> gen_ev;
    size_t gen_used = 0;
    double gen_ms = 0.0;
    uint64_t gen_bricks = 0;
};

static void prof_mark(sf_world *w) {
    StepState *S = w->step;
    if (!S->profile) return;
    if (S->ev_used == S->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) { S->profile = false; return; }
        S->ev_pool.push_back(e);
    }
    cudaEventRecord(S->ev_pool[S->ev_used++], w->stream);
}

enum { DV_CONTACTS = 0, DV_MANIFOLDS = 1, DV_COLORS = 2, DV_ROUNDS = 3, DV_WL0 = 4, DV_WL1 = 5, DV_WL2 = 6,
       DV_ALIVE = 7, DV_AWAKE = 8, DV_ISLANDS = 9, DV_PAIRS = 10, DV_AWK = 11, DV_INC = 12, DV_NBIG = 13, DV_KEPT = 14, DV_MAXDEG = 15, DV_N = 16 };
constexpr int JDS_K = 32;   // the largest manifold chunk: the depth of the solve's contact layout

// ---------------------------------------------------------------- pose cache
// Kernels over bodies or bricks take the substep's active list (global ids of the bodies / bricks of the scenes
// that step); a null list means every body / brick of the world.
__device__ __forceinline__ uint32_t pick(const uint32_t *list, uint32_t t) { return list ? list[t] : t; }

__global__ void k_update_cache(uint32_t nb, const uint32_t *list, float h, const uint8_t *alive, const uint8_t *asleep,
                               const float4 *q, const float *iil, float *rot, float *iiw, float4 *v, uint32_t *bnc) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    if (bnc) bnc[b] = 0;
    if (!alive[b] || asleep[b]) return;
    float4 qq = q[b];
    float r[9], il[9], t1[9], t2[9], t3[9];
    q_to_m(qq.x, qq.y, qq.z, qq.w, r);
#pragma unroll
    for (int k = 0; k < 9; k++) il[k] = iil[(size_t)b * 9 + k];
    mmul(r, il, t1);
    mtr(r, t2);
    mmul(t1, t2, t3);
#pragma unroll
    for (int k = 0; k < 9; k++) { rot[(size_t)b * 9 + k] = r[k]; iiw[(size_t)b * 9 + k] = t3[k]; }
    float4 vv = v[b];
    vv.y -= GR * h;
    v[b] = vv;
}

__global__ void k_brick_pos(uint32_t nd, const uint32_t *list, const uint32_t *kbody, const uint8_t *alive,
                            const uint8_t *asleep, const float4 *pos, const float *rot, const float4 *local, float4 *wpos) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nd) return;
    const uint32_t i = pick(list, t);
    uint32_t b = kbody[i];
    if (!alive[b] || asleep[b]) return;
    float r[9];
#pragma unroll
    for (int k = 0; k < 9; k++) r[k] = rot[(size_t)b * 9 + k];
    float4 l = local[i], p = pos[b];
    V3 wp = add(v3(p.x, p.y, p.z), mv(r, v3(l.x, l.y, l.z)));
    wpos[i] = make_float4(wp.x, wp.y, wp.z, 0.0f);
}

__device__ __forceinline__ int floor_cell(float x) { return __float2int_rz(floorf(x / S)); }

// The hash holds the bricks a bucket walk can meet: every awake brick, and each other live brick whose bucket is one
// of the 27 around an awake brick (gen_contacts walks only those buckets, so a brick outside them is never read; the
// walk's order inside a bucket, by brick index, is unchanged by leaving it out). A scene with more than 1/8 of its
// bricks awake simply puts every live brick in (marking would cost more than it saves).
__global__ void k_awake_flags(uint32_t nd, const uint32_t *list, const uint32_t *kbody, const uint32_t *bscene,
                              const uint32_t *scene_act, const uint8_t *alive, const uint8_t *asleep, uint32_t *flag,
                              uint32_t *scene_awake) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t aw = 0, sk = NONE;
    if (t < nd) {
        const uint32_t b = kbody[pick(list, t)];
        aw = (alive[b] && !asleep[b]) ? 1u : 0u;
        flag[t] = aw;
        if (aw) sk = scene_act[bscene[b]];
    }
    // one atomic per (warp, scene) group
    const unsigned peers = __match_any_sync(0xffffffffu, sk);
    if (sk != NONE && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&scene_awake[sk], __popc(peers));
}
__device__ __forceinline__ bool scene_full(const uint32_t *scene_awake, const uint32_t *scene_bricks, uint32_t sk) {
    return (uint64_t)scene_awake[sk] * 8 > scene_bricks[sk];
}
__global__ void k_compact_list(uint32_t nd, const uint32_t *list, const uint32_t *flag, const uint32_t *pos, uint32_t *out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nd && flag[t]) out[pos[t]] = pick(list, t);
}
// each awake brick marks the 27 buckets around it in its scene's bitmap (32768 bits per active scene)
__global__ void k_mark_buckets(const uint32_t *n_p, const uint32_t *awk, const uint32_t *kbody, const uint32_t *bscene,
                               const uint32_t *scene_act, const uint32_t *scene_awake, const uint32_t *scene_bricks,
                               const float4 *wpos, uint32_t *bits) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= *n_p) return;
    const uint32_t i = awk[u];
    const uint32_t sk = scene_act[bscene[kbody[i]]];
    if (scene_full(scene_awake, scene_bricks, sk)) return;
    const float4 p = wpos[i];
    const int hx = floor_cell(p.x), hy = floor_cell(p.y), hz = floor_cell(p.z);
    uint32_t *sb = bits + (size_t)sk * (HSIZE / 32);
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const uint32_t h = hkey(hx + dx, hy + dy, hz + dz);
                const uint32_t m = 1u << (h & 31);
                if (!(__ldcg(&sb[h >> 5]) & m)) atomicOr(&sb[h >> 5], m);
            }
}
// The spatial hash as a counting sort into the reference's 32768 buckets per active scene (build_hash,
// src/lib.rs:1379-1395): each hashed brick takes an arrival rank in its bucket (k_hash_count), an exclusive scan of
// the counts gives every bucket's start (the table is then CSR: bucket k holds [start[k], start[k + 1])), the bricks
// are placed by start + rank (k_hash_place), and each bucket's few entries are put in ascending brick-id order
// (k_hash_order), which is the order a walk from the highest id down needs (the reference's chain order).
// A brick goes in when it is alive; in the sparse form (most bricks asleep) only when it is awake, its scene has more
// than 1/8 of its bricks awake, or its bucket is one a walk can reach (gen_contacts walks only the 27 buckets around
// an awake brick, so leaving other bricks out changes no walk).
__global__ void k_hash_count(uint32_t nd, const uint32_t *list, const uint32_t *kbody, const uint32_t *bscene,
                             const uint32_t *scene_act, const uint32_t *scene_awake, const uint32_t *scene_bricks,
                             const uint8_t *alive, const uint8_t *asleep, const float4 *wpos, const uint32_t *bits,
                             uint32_t *cnt, uint32_t *tkey, uint32_t *trank) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nd) return;
    const uint32_t i = pick(list, t);
    const uint32_t b = kbody[i];
    uint32_t key = NONE, rank = 0;
    if (alive[b]) {
        const float4 p = wpos[i];
        const uint32_t sk = scene_act[bscene[b]];
        const uint32_t h = hkey(floor_cell(p.x), floor_cell(p.y), floor_cell(p.z));
        const bool in = !bits || !asleep[b] || scene_full(scene_awake, scene_bricks, sk) ||
                        ((bits[(size_t)sk * (HSIZE / 32) + (h >> 5)] >> (h & 31)) & 1u);
        if (in) {
            key = sk * HSIZE + h;
            rank = atomicAdd(&cnt[key], 1u);
        }
    }
    tkey[t] = key;
    trank[t] = rank;
}
__global__ void k_hash_place(uint32_t nd, const uint32_t *list, const uint32_t *tkey, const uint32_t *trank,
                             const uint32_t *start, uint32_t *cval) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nd) return;
    const uint32_t key = tkey[t];
    if (key != NONE) cval[start[key] + trank[t]] = pick(list, t);
}
// a bucket holds a few bricks (the table has 32768 buckets a scene): insertion sort by brick id
__global__ void k_hash_order(uint32_t nbk, const uint32_t *start, uint32_t *cval) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nbk) return;
    const uint32_t lo = start[k], hi = start[k + 1];
    for (uint32_t a = lo + 1; a < hi; a++) {
        const uint32_t v = cval[a];
        uint32_t b = a;
        while (b > lo && cval[b - 1] > v) { cval[b] = cval[b - 1]; b--; }
        cval[b] = v;
    }
}

// A brick's world cell packed in 32 bits (x 11, y 10, z 11 bits about offsets 1024, 512, 1024), each coordinate
// clamped to its field. Clamping never separates two cells: cells within 2 of each other per axis stay within 2.
__device__ __forceinline__ uint32_t pack_wcell(int x, int y, int z) {
    x = min(max(x + 1024, 0), 2047); y = min(max(y + 512, 0), 1023); z = min(max(z + 1024, 0), 2047);
    return (uint32_t)x | ((uint32_t)y << 11) | ((uint32_t)z << 21);
}
// true when the packed cells differ by at most 2 in every coordinate: two brick centres closer than 2 RB = 0.54 m
// (1.08 cells) always are, so a bucket entry that fails this cannot touch the brick and is skipped unread
__device__ __forceinline__ bool wcell_near(uint32_t a, uint32_t b) {
    const int dx = (int)(a & 2047u) - (int)(b & 2047u);
    const int dy = (int)((a >> 11) & 1023u) - (int)((b >> 11) & 1023u);
    const int dz = (int)(a >> 21) - (int)(b >> 21);
    return (uint32_t)(dx + 2) <= 4u && (uint32_t)(dy + 2) <= 4u && (uint32_t)(dz + 2) <= 4u;
}

// Packed bucket entries in sorted order: world position and brick id (srec), and the packed world cell with the body
// id, its asleep bit (31) and the removed-brick bit (30) (sent), so a bucket walk reads contiguous arrays: the 8-byte
// words first, the position only for entries near enough to touch (a full bucket holds mostly other cells that
// share its hash).
__global__ void k_bucket_records(const uint32_t *n_p, const uint32_t *cval, const uint32_t *kbody, const uint8_t *kmat,
                                 const uint8_t *asleep, const float4 *wpos, float4 *srec, uint2 *sent) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= *n_p) return;
    uint32_t j = cval[q];
    uint32_t bj = kbody[j];
    float4 p = wpos[j];
    srec[q] = make_float4(p.x, p.y, p.z, __uint_as_float(j));
    sent[q] = make_uint2(pack_wcell(floor_cell(p.x), floor_cell(p.y), floor_cell(p.z)),
                         bj | (asleep[bj] ? 0x80000000u : 0u) | (kmat[j] == 0 ? 0x40000000u : 0u));
}

// ---------------------------------------------------------------- contacts
struct ContactArgs {
    uint32_t nd;                       // active bricks
    const uint32_t *list, *scene_act;  // active brick -> global brick; scene -> index in the active set
    const uint32_t *kbody, *bscene, *ctab, *cpool;
    const int4 *sbox;
    const uint8_t *alive, *asleep, *smat;
    const float4 *wpos, *v, *w;
    const float *rot, *rad;
    const uint32_t *bstart;            // per (active scene, bucket): first entry; the next bucket's start ends it
    const float4 *srec;
    const uint2 *sent;
    uint32_t *ccount;
    const uint32_t *coff;
    uint8_t *wake;
    uint32_t *sup;                     // per body brick: the frame a contact last supported it (nullptr: not kept)
    uint32_t frame;
    // slot scratch, slot-major: slot k of active brick t at k * nd + t
    uint4 *slot_id;
    float4 *slot_p, *slot_n;
    uint32_t *L_a, *L_b, *L_bo, *L_ba, *L_bb;
    float4 *L_p, *L_n;
};
constexpr int CSLOTS = 12;
constexpr int WALK = 8;        // bucket entries whose packed words one brick loads together

// gen_contacts for one brick of an awake body (src/lib.rs:1410-1468), contacts emitted in the reference's order.
template <bool WAKE, class Emit>
__device__ __forceinline__ void gen_brick(const ContactArgs &A, uint32_t i, uint32_t a, Emit &&emit) {
    const uint32_t sc = A.bscene[a];
    const float4 p4 = A.wpos[i];
    const V3 p = v3(p4.x, p4.y, p4.z);
    // ground: the brick's 8 cube corners below y = 0 (src/lib.rs:1415-1421)
    if (p.y < 0.5f) {
        float r[9];
#pragma unroll
        for (int k = 0; k < 9; k++) r[k] = A.rot[(size_t)a * 9 + k];
        for (int c = 0; c < 8; c++) {
            V3 l = v3((c & 1) == 0 ? -H : H, (c & 2) == 0 ? -H : H, (c & 4) == 0 ? -H : H);
            V3 cp = add(p, mv(r, l));
            if (cp.y < 0.0f) {
                if (WAKE && A.sup) A.sup[i] = A.frame;
                emit(STATIC, STATIC, NONE, cp, v3(0.0f, 1.0f, 0.0f), -cp.y);
            }
        }
    }
    // static cells of the 3^3 block (src/lib.rs:1422-1440): the block spans at most 2 x 2 x 2 chunks, read once
    const int cx = floor_cell(p.x) + NX / 2, cy = floor_cell(p.y), cz = floor_cell(p.z) + NZ / 2;
    const int4 blo = A.sbox[2 * sc], bhi = A.sbox[2 * sc + 1];
    if (cx + 1 >= blo.x && cx - 1 <= bhi.x && cy + 1 >= blo.y && cy - 1 <= bhi.y && cz + 1 >= blo.z && cz - 1 <= bhi.z) {
        const int ox = (cx - 1) >> 3, oy = (cy - 1) >> 3, oz = (cz - 1) >> 3;
        uint32_t ch[8];
        bool any = false;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int qx = ((ox + (k & 1)) << 3), qy = ((oy + ((k >> 1) & 1)) << 3), qz = ((oz + (k >> 2)) << 3);
            uint32_t t = 0;
            if (inb(qx, qy, qz)) t = A.ctab[(size_t)sc * NCT + chunk_slot(qx, qy, qz)];
            ch[k] = t;
            any |= t != 0;
        }
        if (any) {
            for (int dz = -1; dz <= 1; dz++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        const int x = cx + dx, y = cy + dy, z = cz + dz;
                        if (!inb(x, y, z)) continue;
                        const int k = ((x >> 3) - ox) | (((y >> 3) - oy) << 1) | (((z >> 3) - oz) << 2);
                        const uint32_t t = ch[k];
                        if (t == 0) continue;
                        const uint32_t g = A.cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
                        if (g == 0) continue;
                        const uint32_t j = g - 1;
                        if (A.smat[j] == 0) continue;
                        const V3 c = lat_pos(x, y, z);
                        const V3 qq = v3(clampf(p.x, c.x - H, c.x + H), clampf(p.y, c.y - H, c.y + H), clampf(p.z, c.z - H, c.z + H));
                        const V3 d = sub(p, qq);
                        const float dist = len(d);
                        if (dist >= RB) continue;
                        if (dist > 1e-4f) {
                            if (WAKE && A.sup && d.y > 0.3f * dist) A.sup[i] = A.frame;
                            emit(STATIC, STATIC, j, qq, mul(d, div_rn(1.0f, dist)), RB - dist);
                        } else {
                            const V3 r = sub(p, c);
                            const float ar[3] = {r.x, r.y, r.z};
                            int ax = 0;
                            for (int q = 1; q < 3; q++) if (fabsf(ar[q]) > fabsf(ar[ax])) ax = q;
                            float nv[3] = {0.0f, 0.0f, 0.0f};
                            nv[ax] = ar[ax] >= 0.0f ? 1.0f : -1.0f;
                            emit(STATIC, STATIC, j, p, v3(nv[0], nv[1], nv[2]), H + RB - fabsf(ar[ax]));
                        }
                    }
        }
    }
    // hashed neighbours in the 27 buckets around the brick (src/lib.rs:1441-1466); a bucket walked from its highest
    // brick id down is the reference's chain order
    {
        const int hx = floor_cell(p.x), hy = floor_cell(p.y), hz = floor_cell(p.z);
        const uint32_t sk = A.scene_act[sc];
        float speed = 0.0f;
        if (WAKE) {
            const float4 vv = A.v[a], ww = A.w[a];
            speed = len(v3(vv.x, vv.y, vv.z)) + len(v3(ww.x, ww.y, ww.z)) * A.rad[a] * 0.5f;
        }
        const float lim2 = 4.0f * RB * RB;
        const uint32_t mycell = pack_wcell(hx, hy, hz);
        const uint32_t *bst = A.bstart + (size_t)sk * HSIZE;
        for (int dz = -1; dz <= 1; dz++) {
            // The layer's nine buckets are walked as one sequence: bucket c (the reference's dy, dx order) from its
            // highest brick id down; entry t of the sequence lies in bucket c with pre[c] <= t < pre[c + 1]. The
            // nine buckets' bounds are fetched together, then the packed (cell, body) words of WALK entries at a time, so a
            // brick waits on a few rounds of loads per layer instead of one per entry; only entries near enough to
            // touch (a full bucket holds mostly other cells that share its hash) go on to the position record.
            uint32_t hi[9], pre[10];
            pre[0] = 0;
#pragma unroll
            for (int c = 0; c < 9; c++) {
                const uint32_t h = hkey(hx + (c % 3) - 1, hy + (c / 3) - 1, hz + dz);
                const uint32_t lo = bst[h];
                hi[c] = bst[h + 1];
                pre[c + 1] = pre[c] + (hi[c] - lo);
            }
            const uint32_t n = pre[9];
            for (uint32_t b0 = 0; b0 < n; b0 += WALK) {
                uint2 e[WALK];
                uint32_t qq[WALK];
#pragma unroll
                for (int u = 0; u < WALK; u++) {
                    const uint32_t t = b0 + u;
                    uint32_t h = hi[0], p0 = pre[0];
#pragma unroll
                    for (int k = 1; k < 9; k++) if (t >= pre[k]) { h = hi[k]; p0 = pre[k]; }
                    qq[u] = h - 1u - (t - p0);
                    e[u] = t < n ? A.sent[qq[u]] : make_uint2(0u, 0u);
                }
#pragma unroll
                for (int u = 0; u < WALK; u++) {
                    if (b0 + u >= n) break;
                    if (!wcell_near(mycell, e[u].x)) continue;
                    const uint32_t info = e[u].y;
                    const uint32_t bj = info & 0x3FFFFFFFu;
                    if (bj == a || (info & 0x40000000u)) continue;
                    const float4 rec = A.srec[qq[u]];
                    const uint32_t j = __float_as_uint(rec.w);
                    const bool other_awake = !(info & 0x80000000u);
                    if (other_awake && j < i) continue;
                    const V3 pj = v3(rec.x, rec.y, rec.z);
                    const V3 d = sub(p, pj);
                    const float dd = dot(d, d);
                    if (dd >= lim2 || dd < 1e-10f) continue;
                    const float dist = sqrt_rn(dd);
                    const V3 nn = mul(d, div_rn(1.0f, dist));
                    const V3 cp = madd(pj, nn, dist * 0.5f);
                    if (WAKE && A.sup) {
                        if (nn.y > 0.3f) A.sup[i] = A.frame;
                        else if (nn.y < -0.3f) A.sup[j] = A.frame;
                    }
                    if (other_awake) emit(bj, bj, j, cp, nn, 2.0f * RB - dist);
                    else {
                        if (WAKE && speed > 0.7f) A.wake[bj] = 1;
                        emit(STATIC, bj, j, cp, nn, 2.0f * RB - dist);
                    }
                }
            }
        }
    }
}

// pass 1: every contact of every awake brick counted; the first CSLOTS kept in the brick's slots
#ifndef SF_GEN_BLOCKS_PER_SM
#define SF_GEN_BLOCKS_PER_SM 6   // 80 registers (a few spilled): measured faster than 4 or 5 blocks an SM
#endif
__global__ void __launch_bounds__(128, SF_GEN_BLOCKS_PER_SM) k_contacts_gen(ContactArgs A) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.nd) return;
    const uint32_t i = pick(A.list, t);
    const uint32_t a = A.kbody[i];
    if (!A.alive[a] || A.asleep[a]) { A.ccount[t] = 0; return; }
    uint32_t n = 0;
    const size_t nd = A.nd;
    auto emit = [&](uint32_t b, uint32_t bo, uint32_t bb, V3 cp, V3 nn, float depth) {
        if (n < CSLOTS) {
            const size_t o = (size_t)n * nd + t;
            A.slot_id[o] = make_uint4(b, bo, bb, 0u);
            A.slot_p[o] = make_float4(cp.x, cp.y, cp.z, depth);
            A.slot_n[o] = make_float4(nn.x, nn.y, nn.z, 0.0f);
        }
        n++;
    };
    gen_brick<true>(A, i, a, emit);
    A.ccount[t] = n;
}

// pass 2: each brick's contacts to their place in the list; a brick with more than CSLOTS regenerates them
__global__ void __launch_bounds__(128) k_contacts_place(ContactArgs A) {
    const uint32_t ta = blockIdx.x * blockDim.x + threadIdx.x;
    if (ta >= A.nd) return;
    const uint32_t n = A.ccount[ta];
    if (n == 0) return;
    const uint32_t i = pick(A.list, ta);
    const uint32_t a = A.kbody[i];
    const uint32_t base = A.coff[ta];
    const size_t nd = A.nd;
    if (n <= CSLOTS) {
        for (uint32_t k = 0; k < n; k++) {
            const size_t o = (size_t)k * nd + ta;
            const uint4 id = A.slot_id[o];
            const float4 pp = A.slot_p[o], nn = A.slot_n[o];
            const uint32_t t = base + k;
            A.L_a[t] = a; A.L_b[t] = id.x; A.L_bo[t] = id.y; A.L_ba[t] = i; A.L_bb[t] = id.z;
            A.L_p[t] = make_float4(pp.x, pp.y, pp.z, 0.0f);
            A.L_n[t] = make_float4(nn.x, nn.y, nn.z, pp.w);
        }
        return;
    }
    uint32_t k = 0;
    auto emit = [&](uint32_t b, uint32_t bo, uint32_t bb, V3 cp, V3 nn, float depth) {
        const uint32_t t = base + k;
        A.L_a[t] = a; A.L_b[t] = b; A.L_bo[t] = bo; A.L_ba[t] = i; A.L_bb[t] = bb;
        A.L_p[t] = make_float4(cp.x, cp.y, cp.z, 0.0f);
        A.L_n[t] = make_float4(nn.x, nn.y, nn.z, depth);
        k++;
    };
    gen_brick<false>(A, i, a, emit);
}

__global__ void k_body_nc(uint32_t nc, const uint32_t *L_a, const uint32_t *L_b, uint32_t *bnc) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    atomicAdd(&bnc[L_a[k]], 1u);
    uint32_t b = L_b[k];
    if (b != STATIC) atomicAdd(&bnc[b], 1u);
}

// ---------------------------------------------------------------- manifolds
// key = (a, b') with b' = 0 for the static side, else b's index in its scene + 1 (both bodies are in one scene, so
// the pair order is the same as with global ids, in fewer key bits)
__global__ void k_man_keys(uint32_t nc, uint64_t span, const uint32_t *L_a, const uint32_t *L_b, const uint32_t *body_off,
                           uint64_t *key, uint32_t *val) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    uint32_t b = L_b[k];
    uint64_t bp = b == STATIC ? 0 : (uint64_t)(b - body_off[b]) + 1;
    key[k] = (uint64_t)L_a[k] * span + bp;
    val[k] = k;
}
__global__ void k_man_flags(uint32_t nc, const uint64_t *key, uint32_t *flag) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc) return;
    flag[t] = (t == 0 || key[t] != key[t - 1]) ? 1u : 0u;
}
__global__ void k_pair_start(uint32_t nc, const uint32_t *flag, const uint32_t *pos, uint32_t *pair_start) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nc && flag[t]) pair_start[pos[t]] = t;
}
// A body pair's contacts are solved in chunks of at most K (K = 0: the whole pair at once). Chunks of one pair share
// its bodies, so they conflict and take different colours; a chunk is the unit the colouring and the solve see.
__global__ void k_chunk_flags(uint32_t nc, uint32_t K, const uint32_t *flag, const uint32_t *pos, const uint32_t *pair_start,
                              uint32_t *cflag) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc) return;
    const uint32_t mid = pos[t] + flag[t] - 1;
    cflag[t] = K ? ((t - pair_start[mid]) % K == 0 ? 1u : 0u) : flag[t];
}
__global__ void k_man_write(uint32_t nc, uint32_t K, const uint32_t *cflag, const uint32_t *cpos, const uint32_t *flag,
                            const uint32_t *pos, const uint32_t *pair_start, const uint32_t *perm, const uint32_t *L_a,
                            const uint32_t *L_b, const uint32_t *body_off_of_body, const uint32_t *cidx,
                            const uint32_t *bscene, const uint32_t *scene_act, const uint32_t *dom_of_act,
                            uint32_t *man_a, uint32_t *man_b, uint32_t *man_ca, uint32_t *man_cb, uint32_t *man_start,
                            uint32_t *man_prio, uint32_t *man_dom) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc || !cflag[t]) return;
    uint32_t m = cpos[t];
    uint32_t k = perm[t];
    uint32_t a = L_a[k], b = L_b[k];
    man_a[m] = a; man_b[m] = b; man_start[m] = t;
    man_dom[m] = dom_of_act[scene_act[bscene[a]]];
    man_ca[m] = cidx[a]; man_cb[m] = b == STATIC ? STATIC : cidx[b];
    uint32_t off = body_off_of_body[a];
    uint32_t h = pair_priority(a - off, b == STATIC ? 0u : b - off + 1u);
    const uint32_t j = K ? (t - pair_start[pos[t] + flag[t] - 1]) / K : 0u;
    man_prio[m] = j ? pair_priority(h, j) : h;
}
__global__ void k_man_count(const uint32_t *nm_p, uint32_t nc, const uint32_t *man_start, uint32_t *man_count) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t nm = *nm_p;
    if (m >= nm) return;
    uint32_t e = m + 1 < nm ? man_start[m + 1] : nc;
    man_count[m] = e - man_start[m];
}

// ---------------------------------------------------------------- contact reduction (gpu/gpu_world.js:834-920)
// A body pair with more than RED_K contacts keeps, for each of the 26 directions to a cube cell's neighbours, the
// contact whose point reaches furthest along it, and the deepest; ties go to the later contact in list order. The
// pair's other contacts leave the sorted list before the manifolds are cut, so they are neither coloured nor solved.
constexpr uint32_t RED_K = 32, RED_D = 26, RED_S = RED_D + 1;
__device__ __forceinline__ uint32_t f2o(float x) {
    const uint32_t b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float red_score(float4 p, float depth, uint32_t k) {
    if (k == RED_D) return depth;
    const uint32_t j = k >= 13 ? k + 1 : k;
    const float dx = (float)(j % 3) - 1.0f, dy = (float)((j / 3) % 3) - 1.0f, dz = (float)(j / 9) - 1.0f;
    return p.x * dx + p.y * dy + p.z * dz;
}
// per pair: more than RED_K contacts (pairs past the count are 0 for the scan)
__global__ void k_red_big(uint32_t nc, const uint32_t *np_p, const uint32_t *pair_start, uint32_t *big) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nc) return;
    const uint32_t np = *np_p;
    uint32_t b = 0;
    if (p < np) b = ((p + 1 < np ? pair_start[p + 1] : nc) - pair_start[p]) > RED_K ? 1u : 0u;
    big[p] = b;
}
__device__ __forceinline__ uint32_t pair_of(uint32_t t, const uint32_t *flag, const uint32_t *pos) {
    return pos[t] + flag[t] - 1;
}
__global__ void k_red_score(uint32_t nc, const uint32_t *flag, const uint32_t *pos, const uint32_t *big,
                            const uint32_t *bigpos, const uint32_t *perm, const float4 *L_p, const float4 *L_n,
                            uint32_t *best) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc) return;
    const uint32_t p = pair_of(t, flag, pos);
    if (!big[p]) return;
    const uint32_t k = perm[t];
    const float4 pt = L_p[k];
    const float depth = L_n[k].w;
    uint32_t *b = best + (size_t)bigpos[p] * RED_S;
    for (uint32_t d = 0; d < RED_S; d++) atomicMax(&b[d], f2o(red_score(pt, depth, d)));
}
__global__ void k_red_pick(uint32_t nc, const uint32_t *flag, const uint32_t *pos, const uint32_t *big,
                           const uint32_t *bigpos, const uint32_t *perm, const float4 *L_p, const float4 *L_n,
                           const uint32_t *best, uint32_t *win) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc) return;
    const uint32_t p = pair_of(t, flag, pos);
    if (!big[p]) return;
    const uint32_t k = perm[t];
    const float4 pt = L_p[k];
    const float depth = L_n[k].w;
    const size_t o = (size_t)bigpos[p] * RED_S;
    for (uint32_t d = 0; d < RED_S; d++)
        if (f2o(red_score(pt, depth, d)) == best[o + d]) atomicMax(&win[o + d], k + 1);
}
__global__ void k_red_keep(uint32_t nc, const uint32_t *flag, const uint32_t *pos, const uint32_t *big,
                           const uint32_t *bigpos, const uint32_t *perm, const uint32_t *win, uint32_t *keep) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc) return;
    const uint32_t p = pair_of(t, flag, pos);
    uint32_t on = 1;
    if (big[p]) {
        on = 0;
        const uint32_t k = perm[t];
        const size_t o = (size_t)bigpos[p] * RED_S;
        for (uint32_t d = 0; d < RED_S; d++) on |= win[o + d] == k + 1 ? 1u : 0u;
    }
    keep[t] = on;
}
// the sorted contacts plough left on
__global__ void k_off_keep(uint32_t nc, const uint32_t *perm, const uint8_t *off, uint32_t *keep) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nc) keep[t] = off[perm[t]] ? 0u : 1u;
}
__global__ void k_red_compact(uint32_t nc, const uint32_t *keep, const uint32_t *kpos, const uint32_t *perm,
                              const uint64_t *key, uint32_t *perm2, uint64_t *key2) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nc && keep[t]) { perm2[kpos[t]] = perm[t]; key2[kpos[t]] = key[t]; }
}

// ---------------------------------------------------------------- warm start (gpu/gpu_world.js:557-576, 615-683)
// A contact's key: its brick, the other side's kind (0 ground, 1 static brick, 2 awake body's brick, 3 sleeping
// body's brick) and brick, and its place among its brick's earlier contacts of that kind and brick (a brick's
// contacts are contiguous in the list).
__device__ __forceinline__ uint32_t contact_kind(uint32_t b, uint32_t bo, uint32_t bb) {
    return bb == NONE ? 0u : bo == STATIC ? 1u : b == STATIC ? 3u : 2u;
}
__device__ __forceinline__ void warm_key(uint32_t k, const uint32_t *L_b, const uint32_t *L_bo, const uint32_t *L_ba,
                                         const uint32_t *L_bb, unsigned long long &k1, uint32_t &k2) {
    const uint32_t ba = L_ba[k], bb = L_bb[k];
    const uint32_t kind = contact_kind(L_b[k], L_bo[k], bb);
    uint32_t ord = 0;
    for (uint32_t q = k; q-- > 0 && L_ba[q] == ba;)
        if (L_bb[q] == bb && contact_kind(L_b[q], L_bo[q], L_bb[q]) == kind) ord++;
    k1 = ((unsigned long long)ba << 32) | bb;
    k2 = (kind << 16) | ord;
}
__device__ __forceinline__ uint32_t warm_hash(unsigned long long k1, uint32_t k2) {
    unsigned long long h = k1 * 0x9E3779B97F4A7C15ull ^ ((unsigned long long)k2 * 0xC2B2AE3D27D4EB4Full);
    h ^= h >> 29; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 32;
    return (uint32_t)h;
}
// the share of the last substep's impulses a contact starts from (the whole carried the velocity bias too, and
// stacks of single bricks solved with few iterations toppled)
constexpr float WARM_F = 0.8f;
struct WarmRef {
    const uint32_t *claim;
    const unsigned long long *k1;
    const uint32_t *k2;
    const float4 *val;
    uint32_t mask;
};
// the slot holding the key, or NONE (an empty slot ends the probe; keys are unique)
__device__ __forceinline__ uint32_t warm_find(const WarmRef &T, unsigned long long k1, uint32_t k2) {
    uint32_t s = warm_hash(k1, k2) & T.mask;
    for (uint32_t probe = 0; probe < 64; probe++) {
        if (T.claim[s] == 0) return NONE;
        if (T.k1[s] == k1 && T.k2[s] == k2) return s;
        s = (s + 1) & T.mask;
    }
    return NONE;
}
// after the solve: every solved contact's normal impulse and friction vector under its key
__global__ void k_warm_store(uint32_t nc, const uint32_t *invperm, const uint32_t *L_b, const uint32_t *L_bo,
                             const uint32_t *L_ba, const uint32_t *L_bb, const float4 *S_t1, const float4 *S_t2,
                             const float4 *S_j, uint32_t *claim, unsigned long long *tk1, uint32_t *tk2, float4 *val,
                             uint32_t mask, uint32_t *err) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    const uint32_t d = invperm[k];
    if (d == NONE) return;
    unsigned long long k1;
    uint32_t k2;
    warm_key(k, L_b, L_bo, L_ba, L_bb, k1, k2);
    const float4 j = S_j[d], a = S_t1[d], b = S_t2[d];
    const V3 f = add(mul(v3(a.x, a.y, a.z), j.y), mul(v3(b.x, b.y, b.z), j.z));
    uint32_t s = warm_hash(k1, k2) & mask;
    for (uint32_t probe = 0; probe < 64; probe++) {
        if (atomicCAS(&claim[s], 0u, 1u) == 0u) {
            tk1[s] = k1; tk2[s] = k2; val[s] = make_float4(j.x, f.x, f.y, f.z);
            return;
        }
        s = (s + 1) & mask;
    }
    atomicOr(err, (unsigned)ERR_CAPACITY_CONTACTS);   // the table is sized so this cannot happen
}

// each domain's manifolds form one run (manifolds are ordered by body, bodies by scene, domains are runs of scenes)
__global__ void k_dom_ranges(const uint32_t *nm_p, const uint32_t *man_dom, uint32_t *m0, uint32_t *m1) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nm = *nm_p;
    if (m >= nm) return;
    const uint32_t d = man_dom[m];
    if (m == 0 || man_dom[m - 1] != d) m0[d] = m;
    if (m + 1 == nm || man_dom[m + 1] != d) m1[d] = m + 1;
}

__device__ __forceinline__ float eff_mass(float ima, const float *iia, bool hasb, float imb, const float *iib, V3 ra, V3 rb, V3 n) {
    float k = ima + dot(n, cross(mv(iia, cross(ra, n)), ra));
    if (hasb) k += imb + dot(n, cross(mv(iib, cross(rb, n)), rb));
    return k > 1e-12f ? div_rn(1.0f, k) : 0.0f;
}

struct PrepArgs {
    uint32_t nc;
    float h;
    uint32_t nseg;                           // (domain, colour) segments of the colour lists
    const uint32_t *nm_p;                    // manifolds of the substep (device count)
    const uint32_t *perm, *man_a, *man_b, *man_count;
    const uint32_t *man_start, *col_start, *col_list, *jds_off;
    const float4 *L_p, *L_n, *pos, *v, *w;
    const float *im, *iiw;
    float4 *S_n, *S_t1, *S_t2, *S_ra, *S_rb, *S_j;
    uint32_t *invperm;
    // warm start: the last substep's table, read when `warm` is set
    int warm;
    WarmRef wt;
    const uint32_t *L_b, *L_bo, *L_ba, *L_bb;
    const uint8_t *wscene;                   // per scene: its table entries apply
    const uint32_t *bscene;
};

// One thread per manifold, in colour-list order (position p of segment c, a (domain, colour) pair): the two bodies
// are read once, then each of the manifold's contacts is prepared into its slot of the contact layout,
// jds_off[c][kk] + p (consecutive threads write consecutive slots). The per-contact arithmetic is prep_contacts'
// (src/lib.rs:1553-1580).
__global__ void k_prep(PrepArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *A.nm_p) return;
    uint32_t lo = 0, hi = A.nseg;   // the last segment c with col_start[c] <= i (empty segments start where it does)
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A.col_start[mid] <= i) lo = mid; else hi = mid;
    }
    const uint32_t c = lo, p = i - A.col_start[c];
    const uint32_t m = A.col_list[i];
    const uint32_t a = A.man_a[m], b = A.man_b[m], cnt = A.man_count[m], t0 = A.man_start[m];
    const bool hasb = b != STATIC;
    const float4 pa = A.pos[a], va = A.v[a], wa = A.w[a];
    float iia[9], iib[9];
#pragma unroll
    for (int q = 0; q < 9; q++) iia[q] = A.iiw[(size_t)a * 9 + q];
    const float ima = A.im[a];
    float imb = 0.0f;
    float4 pb = make_float4(0, 0, 0, 0), vb = pb, wb = pb;
    if (hasb) {
        pb = A.pos[b]; vb = A.v[b]; wb = A.w[b];
#pragma unroll
        for (int q = 0; q < 9; q++) iib[q] = A.iiw[(size_t)b * 9 + q];
        imb = A.im[b];
    }
    const uint32_t *off = A.jds_off + c * JDS_K;
    for (uint32_t kk = 0; kk < cnt; kk++) {
        const uint32_t d = off[kk] + p;
        const uint32_t k = A.perm[t0 + kk];
        const float4 p4 = A.L_p[k], n4 = A.L_n[k];
        const V3 pt = v3(p4.x, p4.y, p4.z), n = v3(n4.x, n4.y, n4.z);
        const float depth = n4.w;
        const V3 ra = sub(pt, v3(pa.x, pa.y, pa.z));
        V3 rb = v3(0.0f, 0.0f, 0.0f);
        const V3 vela = add(v3(va.x, va.y, va.z), cross(v3(wa.x, wa.y, wa.z), ra));
        V3 velb = v3(0.0f, 0.0f, 0.0f);
        if (hasb) {
            rb = sub(pt, v3(pb.x, pb.y, pb.z));
            velb = add(v3(vb.x, vb.y, vb.z), cross(v3(wb.x, wb.y, wb.z), rb));
        }
        const float mn = eff_mass(ima, iia, hasb, imb, iib, ra, rb, n);
        const V3 dv = sub(vela, velb);
        const float vn = dot(dv, n);
        const float vn0 = maxf(-vn, 0.0f);
        const V3 vt = sub(dv, mul(n, vn));
        const float lt = len(vt);
        V3 t1;
        if (lt > 1e-4f) t1 = mul(vt, div_rn(1.0f, lt));
        else {
            V3 tt = fabsf(n.x) < 0.9f ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
            V3 x = cross(n, tt);
            t1 = mul(x, div_rn(1.0f, len(x)));
        }
        const V3 t2 = cross(n, t1);
        const float mt1 = eff_mass(ima, iia, hasb, imb, iib, ra, rb, t1);
        const float mt2 = eff_mass(ima, iia, hasb, imb, iib, ra, rb, t2);
        float bias = minf(div_rn(0.2f, A.h) * maxf(depth - 0.01f, 0.0f), 1.0f);
        if (vn < -2.0f) bias = maxf(bias, -0.12f * vn);
        A.S_n[d] = make_float4(n.x, n.y, n.z, mn);
        A.S_t1[d] = make_float4(t1.x, t1.y, t1.z, mt1);
        A.S_t2[d] = make_float4(t2.x, t2.y, t2.z, mt2);
        A.S_ra[d] = make_float4(ra.x, ra.y, ra.z, bias);
        A.S_rb[d] = make_float4(rb.x, rb.y, rb.z, vn0);
        float4 j0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (A.warm && A.wscene[A.bscene[a]]) {
            unsigned long long k1;
            uint32_t k2;
            warm_key(k, A.L_b, A.L_bo, A.L_ba, A.L_bb, k1, k2);
            const uint32_t sl = warm_find(A.wt, k1, k2);
            if (sl != NONE) {
                const float4 o = A.wt.val[sl];
                const float jn = o.x * WARM_F, lim = MU * jn;
                const V3 f = v3(o.y, o.z, o.w);
                j0 = make_float4(jn, clampf(dot(f, t1) * WARM_F, -lim, lim), clampf(dot(f, t2) * WARM_F, -lim, lim), 0.0f);
            }
        }
        A.S_j[d] = j0;
        A.invperm[k] = d;
    }
}

// ---------------------------------------------------------------- colouring
// The body-to-manifold lists and the colour masks are indexed by the body's place in the substep's active list
// (man_ca / man_cb), so their size and clearing follow the active bodies only.
// (and the largest count of manifolds at one body, which picks the colouring's form)
__global__ void k_bm_count(const uint32_t *nm_p, const uint32_t *man_a, const uint32_t *man_b, uint32_t *bm_count,
                           uint32_t *maxdeg) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= *nm_p) return;
    uint32_t d = atomicAdd(&bm_count[man_a[m]], 1u) + 1;
    uint32_t b = man_b[m];
    if (b != STATIC) d = max(d, atomicAdd(&bm_count[b], 1u) + 1);
    atomicMax(maxdeg, d);
}
__global__ void k_bm_fill(const uint32_t *nm_p, const uint32_t *man_a, const uint32_t *man_b, const uint32_t *bm_start,
                          uint32_t *bm_fill, uint32_t *bm_list) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= *nm_p) return;
    uint32_t a = man_a[m];
    bm_list[bm_start[a] + atomicAdd(&bm_fill[a], 1u)] = m;
    uint32_t b = man_b[m];
    if (b != STATIC) bm_list[bm_start[b] + atomicAdd(&bm_fill[b], 1u)] = m;
}

struct JpArgs {
    const uint32_t *man_a, *man_b, *prio, *bm_start, *bm_list;   // man_a / man_b: active-list body ids
    uint32_t *man_round, *man_color, *masks;
    uint32_t *wl0, *wl1, *dev;
    const uint4 *blk_dom;             // per block: domain, rank in the domain, blocks of the domain
    const uint32_t *dom_m0, *dom_m1;  // per domain: its manifolds [m0, m1)
    uint32_t *dom_cnt;                // per domain: three rotating worklist counters
    uint32_t max_colors, max_rounds;
    uint32_t mw;                      // colour-mask words per body: max_colors / 32 rounded up
    GridBarrier *gb;                  // per domain
    uint32_t *err;
    uint32_t seq_launched;            // k_colour_seq ran before (it colours the substeps it takes)
};

__device__ __forceinline__ bool jp_blocked(const JpArgs &A, uint32_t body, uint32_t m, uint32_t pm, uint32_t r) {
    const uint32_t s0 = A.bm_start[body], s1 = A.bm_start[body + 1];
    for (uint32_t q = s0; q < s1; q++) {
        const uint32_t nbr = A.bm_list[q];
        if (nbr == m) continue;
        if (__ldcg(&A.man_round[nbr]) < r) continue;   // coloured in an earlier round
        const uint32_t pn = A.prio[nbr];
        if (pn > pm || (pn == pm && nbr < m)) return true;
    }
    return false;
}

// The barrier of one sync domain: a block alone needs only __syncthreads; several blocks meet at the domain's own
// bounded grid barrier (false once a wait timed out).
__device__ __forceinline__ bool dom_sync(GridBarrier *gb, uint32_t nblk, uint32_t *err) {
    if (nblk == 1) { __syncthreads(); return true; }
    return grid_sync(gb, nblk, err);
}

// the substeps the one-pass colouring (k_colour_seq) takes: few manifolds, or a hub among them
constexpr uint32_t SEQ_COLOUR_MAX = 1024, SEQ_COLOUR_SMALL = 256, SEQ_HUB = 64, SEQ_T = 1024;
constexpr uint32_t SEQ_COLOUR_LAUNCH = 16384;   // contacts up to which the one-pass form is launched to decide
__device__ __forceinline__ bool colour_seq_form(const uint32_t *dev) {
    const uint32_t nm = dev[DV_MANIFOLDS];
    return nm <= SEQ_COLOUR_MAX && (nm <= SEQ_COLOUR_SMALL || dev[DV_MAXDEG] > SEQ_HUB);
}

// Jones-Plassmann rounds, each domain on its own blocks: a round colours every manifold of the domain's worklist whose
// higher-priority neighbours are all coloured (the smallest colour free at both bodies) and passes the others on.
// Neighbouring manifolds share a body, hence a scene, hence a domain, so each domain's result is the greedy
// colouring in priority order whatever the other domains do.
__global__ void __launch_bounds__(128) k_jp(JpArgs A) {
    if (A.seq_launched && colour_seq_form(A.dev)) return;   // k_colour_seq coloured them
    const uint4 bd = A.blk_dom[blockIdx.x];
    const uint32_t d = bd.x, rank = bd.y, nblk = bd.z;
    const uint32_t m0 = A.dom_m0[d], nm = A.dom_m1[d] - m0;
    uint32_t *cnt = A.dom_cnt + 3 * d;
    const uint32_t stride = nblk * blockDim.x;
    uint32_t r = 0;
    for (; r < A.max_rounds; r++) {
        const uint32_t n_in = r == 0 ? nm : __ldcg(&cnt[r % 3]);
        if (n_in == 0) break;
        const uint32_t *wl_in = ((r & 1) ? A.wl1 : A.wl0) + m0;
        uint32_t *wl_out = ((r & 1) ? A.wl0 : A.wl1) + m0;
        uint32_t *cnt_out = &cnt[(r + 1) % 3];
        if (rank == 0 && threadIdx.x == 0) cnt[(r + 2) % 3] = 0;
        // a warp walks 32 consecutive entries at a time, so that it can append its blocked manifolds to the next
        // worklist with one atomic
        const uint32_t lane = threadIdx.x & 31u;
        for (uint32_t t0 = rank * blockDim.x + (threadIdx.x & ~31u); t0 < n_in; t0 += stride) {
            const uint32_t t = t0 + lane;
            const bool valid = t < n_in;
            uint32_t m = 0, a = 0, b = STATIC, pm = 0;
            bool blocked = false;
            if (valid) {
                m = r == 0 ? m0 + t : __ldcg(&wl_in[t]);
                a = A.man_a[m]; b = A.man_b[m]; pm = A.prio[m];
                blocked = jp_blocked(A, a, m, pm, r);
                if (!blocked && b != STATIC) blocked = jp_blocked(A, b, m, pm, r);
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, valid && blocked);
            if (bal) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(cnt_out, (uint32_t)__popc(bal));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (valid && blocked) wl_out[base + __popc(bal & ((1u << lane) - 1u))] = m;
            }
            if (!valid || blocked) continue;
            // the lowest colour free at both bodies
            uint32_t c = 0xFFFFFFFFu;
            for (uint32_t k = 0; k < A.mw && c == 0xFFFFFFFFu; k++) {
                const uint32_t used = __ldcg(&A.masks[(size_t)a * A.mw + k]) |
                                      (b != STATIC ? __ldcg(&A.masks[(size_t)b * A.mw + k]) : 0u);
                if (~used) c = 32 * k + (__ffs(~used) - 1);
            }
            if (c >= A.max_colors) { atomicOr(A.err, (unsigned)ERR_CAPACITY_COLORS); c = A.max_colors - 1; }
            A.man_color[m] = c;
            atomicExch(&A.man_round[m], r);
            atomicOr(&A.masks[(size_t)a * A.mw + (c >> 5)], 1u << (c & 31));
            if (b != STATIC) atomicOr(&A.masks[(size_t)b * A.mw + (c >> 5)], 1u << (c & 31));
        }
        if (!dom_sync(A.gb + d, nblk, A.err)) return;
    }
    if (rank == 0 && threadIdx.x == 0) {
        atomicMax(&A.dev[DV_ROUNDS], r);
        if (r >= A.max_rounds) atomicOr(A.err, (unsigned)ERR_JP_ROUNDS);
    }
}

// The colouring in one pass, for a substep of at most SEQ_COLOUR_MAX manifolds that are few (at most 256) or meet
// at a hub (a body holding more than SEQ_HUB of them, a large piece resting on many chunks): the manifolds sorted by
// priority (highest first, ties to the lower index) and coloured one after another with the smallest colour free at
// both bodies, which is the colouring the Jones-Plassmann rounds reach (domains do not share bodies, so one order over
// all of them gives each domain its own result). At a hub the rounds are as many as its colours and each scans all
// its manifolds again; this pass costs well under a microsecond a manifold. One block; k_jp returns at once when it
// runs.
__global__ void __launch_bounds__(SEQ_T) k_colour_seq(JpArgs A) {
    __shared__ unsigned long long key[SEQ_COLOUR_MAX];
    __shared__ uint32_t s_m[SEQ_COLOUR_MAX], s_a[SEQ_COLOUR_MAX], s_b[SEQ_COLOUR_MAX];
    if (!colour_seq_form(A.dev)) return;
    const uint32_t nm = A.dev[DV_MANIFOLDS];
    uint32_t n2 = 1;
    while (n2 < nm) n2 <<= 1;
    for (uint32_t t = threadIdx.x; t < n2; t += SEQ_T)
        key[t] = t < nm ? (((unsigned long long)A.prio[t] << 32) | (0xFFFFFFFFu - t)) : 0ull;
    __syncthreads();
    // bitonic sort, descending
    for (uint32_t k = 2; k <= n2; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < n2; t += SEQ_T) {
                const uint32_t ix = t ^ j;
                if (ix > t) {
                    const unsigned long long x = key[t], y = key[ix];
                    const bool desc = (t & k) == 0;
                    if (desc ? (x < y) : (x > y)) { key[t] = y; key[ix] = x; }
                }
            }
            __syncthreads();
        }
    }
    // the manifolds' bodies in sorted order, fetched in parallel for the one thread that colours
    for (uint32_t q = threadIdx.x; q < nm; q += SEQ_T) {
        const uint32_t m = 0xFFFFFFFFu - (uint32_t)(key[q] & 0xFFFFFFFFull);
        s_m[q] = m; s_a[q] = A.man_a[m]; s_b[q] = A.man_b[m];
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (uint32_t q = 0; q < nm; q++) {
        const uint32_t m = s_m[q], a = s_a[q], b = s_b[q];
        uint32_t c = 0xFFFFFFFFu;
        for (uint32_t k = 0; k < A.mw && c == 0xFFFFFFFFu; k++) {
            const uint32_t used = A.masks[(size_t)a * A.mw + k] | (b != STATIC ? A.masks[(size_t)b * A.mw + k] : 0u);
            if (~used) c = 32 * k + (__ffs(~used) - 1);
        }
        if (c >= A.max_colors) { atomicOr(A.err, (unsigned)ERR_CAPACITY_COLORS); c = A.max_colors - 1; }
        A.man_color[m] = c;
        A.man_round[m] = q;
        A.masks[(size_t)a * A.mw + (c >> 5)] |= 1u << (c & 31);
        if (b != STATIC) A.masks[(size_t)b * A.mw + (c >> 5)] |= 1u << (c & 31);
    }
    atomicMax(&A.dev[DV_ROUNDS], nm);   // one manifold a round
}

// Warp-aggregated counter increment: the lanes that share a key take one atomicAdd on ctr[key] between them; each
// gets old value + its rank among those lanes. Every lane of the warp must call it; invalid lanes take nothing.
__device__ __forceinline__ uint32_t warp_add1(uint32_t *ctr, uint32_t key, bool valid) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t peers = __match_any_sync(0xffffffffu, valid ? key : 0xFFFFFFFFu);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (valid && lane == leader) base = atomicAdd(&ctr[key], (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// manifolds counted by (segment, contact count), count descending, where segment = domain * cstride + colour:
// bucket segment * (JDS_K + 1) + (JDS_K - count)
constexpr int JDS_ROW = JDS_K + 1;
// Most manifolds fall in a few buckets: the lanes of a warp that share a bucket take one atomic between them
// (warp_add1), and the colour counts (per domain and overall) are reduced over the warp first. (The order of a
// bucket's manifolds is arbitrary either way; a colour's manifolds are independent.)
__global__ void k_col_count(const uint32_t *nm_p, const uint32_t *man_color, const uint32_t *man_count,
                            const uint32_t *man_dom, uint32_t cstride, uint32_t *hist, uint32_t *dom_ncol, uint32_t *dev) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = m < *nm_p;
    const uint32_t c = valid ? man_color[m] : 0u;
    const uint32_t d = valid ? man_dom[m] : 0u;
    warp_add1(hist, valid ? (d * cstride + c) * JDS_ROW + (JDS_K - man_count[m]) : 0u, valid);
    const uint32_t peers = __match_any_sync(0xffffffffu, valid ? d : 0xFFFFFFFFu);
    const uint32_t dm = __reduce_max_sync(peers, valid ? c + 1 : 0u);
    if (valid && (threadIdx.x & 31u) == (uint32_t)(__ffs(peers) - 1)) atomicMax(&dom_ncol[d], dm);
    const uint32_t cm = __reduce_max_sync(0xffffffffu, valid ? c + 1 : 0u);
    if ((threadIdx.x & 31u) == 0 && cm) atomicMax(&dev[DV_COLORS], cm);
}
__global__ void k_col_fill(const uint32_t *nm_p, const uint32_t *man_color, const uint32_t *man_count,
                           const uint32_t *man_dom, uint32_t cstride, const uint32_t *hstart, uint32_t *hfill,
                           uint32_t *col_list) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = m < *nm_p;
    const uint32_t bkt = valid ? (man_dom[m] * cstride + man_color[m]) * JDS_ROW + (JDS_K - man_count[m]) : 0u;
    const uint32_t slot = warp_add1(hfill, bkt, valid);
    if (valid) col_list[hstart[bkt] + slot] = m;
}
// per segment: the contacts it holds (its contact-layout size)
__global__ void k_seg_totals(uint32_t nseg, const uint32_t *hist, uint32_t *tot) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nseg) return;
    // n[k] = manifolds with more than k contacts = those in buckets j <= JDS_K - 1 - k; contacts = sum of n[k]
    uint32_t run = 0, total = 0;
    for (int j = 0; j < JDS_K; j++) { run += hist[(size_t)c * JDS_ROW + j]; total += run; }
    tot[c] = total;
}
// per segment: its start in col_list and the JDS offsets of its contact layout (segments' contacts in segment order)
__global__ void k_seg_table(uint32_t nseg, const uint32_t *hist, const uint32_t *hstart, const uint32_t *base,
                            const uint32_t *nm_p, uint32_t *col_start, uint32_t *jds_off) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nseg) return;
    uint32_t n[JDS_K];
    uint32_t run = 0;
#pragma unroll
    for (int j = 0; j < JDS_K; j++) { run += hist[(size_t)c * JDS_ROW + j]; n[JDS_K - 1 - j] = run; }
    uint32_t b = base[c];
    col_start[c] = hstart[(size_t)c * JDS_ROW];
    if (c == nseg - 1) col_start[nseg] = *nm_p;
#pragma unroll
    for (int k = 0; k < JDS_K; k++) { jds_off[(size_t)c * JDS_K + k] = b; b += n[k]; }
}

// proper-colouring check: no two manifolds of one colour at one awake body
__global__ void k_col_verify(const uint32_t *nm_p, const uint32_t *man_a, const uint32_t *man_b, const uint32_t *man_color,
                             uint32_t mw, uint32_t *vmasks, uint32_t *err) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= *nm_p) return;
    uint32_t c = man_color[m];
    uint32_t bit = 1u << (c & 31);
    if (atomicOr(&vmasks[(size_t)man_a[m] * mw + (c >> 5)], bit) & bit) atomicOr(err, (unsigned)ERR_VERIFY_COLOR);
    uint32_t b = man_b[m];
    if (b != STATIC && (atomicOr(&vmasks[(size_t)b * mw + (c >> 5)], bit) & bit)) atomicOr(err, (unsigned)ERR_VERIFY_COLOR);
}

// ---------------------------------------------------------------- the coloured sequential-impulse solve
// Contact layout (jagged diagonal, per colour): a colour's manifolds are listed by contact count, most first, and
// contact k of the colour's p-th manifold sits at jds_off[colour * JDS_K + k] + p. The k-th contacts of a colour's
// manifolds are therefore contiguous, so the threads of a warp (consecutive p) read them coalesced.
struct SolveArgs {
    uint32_t iterations;
    const uint32_t *dev;           // DV_COLORS
    const uint4 *blk_dom;          // per block: domain, rank in the domain, blocks of the domain
    const uint32_t *dom_ncol;      // per domain: colours used
    uint32_t cstride;              // segment of (domain d, colour c) = d * cstride + c
    const uint32_t *col_start, *col_list, *jds_off;
    const uint32_t *man_a, *man_b, *man_count;
    const float4 *S_n, *S_t1, *S_t2, *S_ra, *S_rb;
    float4 *S_j;
    float4 *v, *w;
    const float *im, *iiw;
    GridBarrier *gb;
    uint32_t *err;
    uint32_t warm;                 // 1: a first pass applies the warm-started impulses
};

// Body velocities and impulses written by other blocks are read through L2 (__ldcg) in the grid-wide solve; in the
// one-block solve every write is the block's own, ordered by __syncthreads, so plain (L1-cached) loads are exact.
template <bool ONE_BLOCK> __device__ __forceinline__ float4 ld_rw(const float4 *p) {
    if (ONE_BLOCK) return *p;
    return __ldcg(p);
}

template <bool ONE_BLOCK>
__device__ __forceinline__ void solve_manifold(const SolveArgs &A, uint32_t m, uint32_t p, const uint32_t *off) {
    const uint32_t a = A.man_a[m], b = A.man_b[m];
    const bool hasb = b != STATIC;
    const uint32_t cnt = A.man_count[m];
    float4 t4 = ld_rw<ONE_BLOCK>(&A.v[a]);
    V3 va = v3(t4.x, t4.y, t4.z);
    t4 = ld_rw<ONE_BLOCK>(&A.w[a]);
    V3 wa = v3(t4.x, t4.y, t4.z);
    const float ima = A.im[a];
    float ia[9], ib[9];
#pragma unroll
    for (int q = 0; q < 9; q++) ia[q] = A.iiw[(size_t)a * 9 + q];
    V3 vb = v3(0.0f, 0.0f, 0.0f), wb = v3(0.0f, 0.0f, 0.0f);
    float imb = 0.0f;
    if (hasb) {
        t4 = ld_rw<ONE_BLOCK>(&A.v[b]); vb = v3(t4.x, t4.y, t4.z);
        t4 = ld_rw<ONE_BLOCK>(&A.w[b]); wb = v3(t4.x, t4.y, t4.z);
        imb = A.im[b];
#pragma unroll
        for (int q = 0; q < 9; q++) ib[q] = A.iiw[(size_t)b * 9 + q];
    }
    // the next contact's data is loaded while the current one is solved (the chain through the bodies is serial)
    float4 nx_n = make_float4(0, 0, 0, 0), nx_t1 = nx_n, nx_t2 = nx_n, nx_ra = nx_n, nx_rb = nx_n, nx_j = nx_n;
    uint32_t at = off[0] + p;
    if (cnt) {
        nx_n = __ldg(&A.S_n[at]); nx_t1 = __ldg(&A.S_t1[at]); nx_t2 = __ldg(&A.S_t2[at]);
        nx_ra = __ldg(&A.S_ra[at]); nx_rb = __ldg(&A.S_rb[at]); nx_j = ld_rw<ONE_BLOCK>(&A.S_j[at]);
    }
    for (uint32_t k = 0; k < cnt; k++) {
        const float4 n4 = nx_n, t14 = nx_t1, t24 = nx_t2, ra4 = nx_ra, rb4 = nx_rb;
        float4 j4 = nx_j;
        const uint32_t cur = at;
        if (k + 1 < cnt) {
            at = off[k + 1] + p;
            nx_n = __ldg(&A.S_n[at]); nx_t1 = __ldg(&A.S_t1[at]); nx_t2 = __ldg(&A.S_t2[at]);
            nx_ra = __ldg(&A.S_ra[at]); nx_rb = __ldg(&A.S_rb[at]); nx_j = ld_rw<ONE_BLOCK>(&A.S_j[at]);
        }
        const V3 n = v3(n4.x, n4.y, n4.z), t1 = v3(t14.x, t14.y, t14.z), t2 = v3(t24.x, t24.y, t24.z);
        const V3 ra = v3(ra4.x, ra4.y, ra4.z), rb = v3(rb4.x, rb4.y, rb4.z);
        const float mn = n4.w, mt1 = t14.w, mt2 = t24.w, bias = ra4.w;
        // normal
        V3 dv = sub(add(va, cross(wa, ra)), hasb ? add(vb, cross(wb, rb)) : v3(0.0f, 0.0f, 0.0f));
        float vn = dot(dv, n);
        float lam = mn * (-vn + bias);
        float old = j4.x;
        j4.x = maxf(old + lam, 0.0f);
        float d = j4.x - old;
        {
            V3 P = mul(n, d);
            va = madd(va, P, ima);
            wa = add(wa, mv(ia, cross(ra, P)));
            if (hasb) { vb = madd(vb, P, -imb); wb = sub(wb, mv(ib, cross(rb, P))); }
        }
        // friction, two independent clamps
        float lim = MU * j4.x;
        dv = sub(add(va, cross(wa, ra)), hasb ? add(vb, cross(wb, rb)) : v3(0.0f, 0.0f, 0.0f));
        float l1 = -mt1 * dot(dv, t1);
        float o1 = j4.y;
        j4.y = clampf(o1 + l1, -lim, lim);
        float l2 = -mt2 * dot(dv, t2);
        float o2 = j4.z;
        j4.z = clampf(o2 + l2, -lim, lim);
        {
            V3 P = add(mul(t1, j4.y - o1), mul(t2, j4.z - o2));
            va = madd(va, P, ima);
            wa = add(wa, mv(ia, cross(ra, P)));
            if (hasb) { vb = madd(vb, P, -imb); wb = sub(wb, mv(ib, cross(rb, P))); }
        }
        A.S_j[cur] = j4;
    }
    A.v[a] = make_float4(va.x, va.y, va.z, 0.0f);
    A.w[a] = make_float4(wa.x, wa.y, wa.z, 0.0f);
    if (hasb) {
        A.v[b] = make_float4(vb.x, vb.y, vb.z, 0.0f);
        A.w[b] = make_float4(wb.x, wb.y, wb.z, 0.0f);
    }
}

// the warm-started impulses of a manifold's contacts, applied once in its order (apply_imp with the whole impulse)
template <bool ONE_BLOCK>
__device__ __forceinline__ void warm_manifold(const SolveArgs &A, uint32_t m, uint32_t p, const uint32_t *off) {
    const uint32_t a = A.man_a[m], b = A.man_b[m];
    const bool hasb = b != STATIC;
    const uint32_t cnt = A.man_count[m];
    float4 t4 = ld_rw<ONE_BLOCK>(&A.v[a]);
    V3 va = v3(t4.x, t4.y, t4.z);
    t4 = ld_rw<ONE_BLOCK>(&A.w[a]);
    V3 wa = v3(t4.x, t4.y, t4.z);
    const float ima = A.im[a];
    float ia[9], ib[9];
#pragma unroll
    for (int q = 0; q < 9; q++) ia[q] = A.iiw[(size_t)a * 9 + q];
    V3 vb = v3(0.0f, 0.0f, 0.0f), wb = v3(0.0f, 0.0f, 0.0f);
    float imb = 0.0f;
    if (hasb) {
        t4 = ld_rw<ONE_BLOCK>(&A.v[b]); vb = v3(t4.x, t4.y, t4.z);
        t4 = ld_rw<ONE_BLOCK>(&A.w[b]); wb = v3(t4.x, t4.y, t4.z);
        imb = A.im[b];
#pragma unroll
        for (int q = 0; q < 9; q++) ib[q] = A.iiw[(size_t)b * 9 + q];
    }
    for (uint32_t k = 0; k < cnt; k++) {
        const uint32_t at = off[k] + p;
        const float4 n4 = __ldg(&A.S_n[at]), t14 = __ldg(&A.S_t1[at]), t24 = __ldg(&A.S_t2[at]);
        const float4 ra4 = __ldg(&A.S_ra[at]), rb4 = __ldg(&A.S_rb[at]), j4 = ld_rw<ONE_BLOCK>(&A.S_j[at]);
        const V3 ra = v3(ra4.x, ra4.y, ra4.z), rb = v3(rb4.x, rb4.y, rb4.z);
        const V3 P = add(mul(v3(n4.x, n4.y, n4.z), j4.x),
                         add(mul(v3(t14.x, t14.y, t14.z), j4.y), mul(v3(t24.x, t24.y, t24.z), j4.z)));
        va = madd(va, P, ima);
        wa = add(wa, mv(ia, cross(ra, P)));
        if (hasb) { vb = madd(vb, P, -imb); wb = sub(wb, mv(ib, cross(rb, P))); }
    }
    A.v[a] = make_float4(va.x, va.y, va.z, 0.0f);
    A.w[a] = make_float4(wa.x, wa.y, wa.z, 0.0f);
    if (hasb) {
        A.v[b] = make_float4(vb.x, vb.y, vb.z, 0.0f);
        A.w[b] = make_float4(wb.x, wb.y, wb.z, 0.0f);
    }
}

constexpr int SOLVE_BLOCK = 128;

// A colour's manifolds are listed by contact count, most first. Thread g takes position g of even rounds and the
// mirrored position of odd rounds (2 stride - 1 - g, ...), so the threads that get a round's largest manifolds get
// the next round's smallest; consecutive threads still take consecutive positions (coalesced contact loads).
__device__ __forceinline__ uint32_t snake_pos(uint32_t r, uint32_t g, uint32_t stride) {
    return (r & 1u) ? (r + 1) * stride - 1 - g : r * stride + g;
}

// Each sync domain runs its own iterations and colours on its own blocks, meeting at its own barrier after each
// colour: scenes never share a body, so no domain waits for another's colours.
__global__ void __launch_bounds__(SOLVE_BLOCK) k_solve(SolveArgs A) {
    __shared__ uint32_t off[JDS_K];
    const uint4 bd = A.blk_dom[blockIdx.x];
    const uint32_t d = bd.x, nblk = bd.z;
    const uint32_t ncol = A.dom_ncol[d];
    const uint32_t stride = nblk * blockDim.x;
    const uint32_t g = bd.y * blockDim.x + threadIdx.x;
    for (uint32_t it = 0; it < A.iterations + A.warm; it++) {
        const bool wp = A.warm && it == 0;
        for (uint32_t c = 0; c < ncol; c++) {
            const uint32_t seg = d * A.cstride + c;
            if (threadIdx.x < JDS_K) off[threadIdx.x] = A.jds_off[(size_t)seg * JDS_K + threadIdx.x];
            __syncthreads();
            const uint32_t s0 = A.col_start[seg], n = A.col_start[seg + 1] - s0;
            for (uint32_t r = 0; r * stride < n; r++) {
                const uint32_t p = snake_pos(r, g, stride);
                if (p < n) {
                    if (wp) warm_manifold<false>(A, A.col_list[s0 + p], p, off);
                    else solve_manifold<false>(A, A.col_list[s0 + p], p, off);
                }
            }
            if (!dom_sync(A.gb + d, nblk, A.err)) return;
        }
    }
}

// small substeps: one block, colours separated by __syncthreads instead of a grid barrier
constexpr int SOLVE_ONE_BLOCK = 512;
constexpr uint32_t SOLVE_ONE_BLOCK_MAX_CONTACTS = 8192;
constexpr uint32_t SMALL_SUBSTEP_CONTACTS = 1024;
__global__ void __launch_bounds__(SOLVE_ONE_BLOCK) k_solve_one_block(SolveArgs A) {
    __shared__ uint32_t off[JDS_K];
    const uint32_t ncol = A.dev[DV_COLORS];
    for (uint32_t it = 0; it < A.iterations + A.warm; it++) {
        const bool wp = A.warm && it == 0;
        for (uint32_t c = 0; c < ncol; c++) {
            if (threadIdx.x < JDS_K) off[threadIdx.x] = A.jds_off[c * JDS_K + threadIdx.x];
            __syncthreads();
            const uint32_t s0 = A.col_start[c], n = A.col_start[c + 1] - s0;
            for (uint32_t r = 0; r * blockDim.x < n; r++) {
                const uint32_t p = snake_pos(r, threadIdx.x, blockDim.x);
                if (p < n) {
                    if (wp) warm_manifold<true>(A, A.col_list[s0 + p], p, off);
                    else solve_manifold<true>(A, A.col_list[s0 + p], p, off);
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------- islands
__global__ void k_uf_init(uint32_t nb, const uint32_t *list, uint32_t *parent, uint32_t *mint) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    parent[b] = b;
    mint[b] = 0x7f7fffffu;
}
__global__ void k_uf_union(const uint32_t *nm_p, const uint32_t *man_a, const uint32_t *man_b, uint32_t *parent,
                           uint32_t *err) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= *nm_p) return;
    uint32_t b = man_b[m];
    if (b == STATIC) return;
    uf_union(parent, man_a[m], b, err);
}
__global__ void k_uf_label(uint32_t nb, const uint32_t *list, const uint8_t *alive, const uint8_t *asleep, uint32_t *parent,
                           uint32_t *label, uint32_t *dev, uint32_t *err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    bool root = false;
    if (t < nb) {
        const uint32_t b = pick(list, t);
        if (!alive[b] || asleep[b]) label[b] = NONE;
        else {
            const uint32_t r = uf_find(parent, b, err);
            label[b] = r;
            root = r == b;
        }
    }
    const uint32_t n = __popc(__ballot_sync(0xffffffffu, root));   // one atomic per warp
    if ((threadIdx.x & 31u) == 0 && n) atomicAdd(&dev[DV_ISLANDS], n);
}

// ---------------------------------------------------------------- pinch clamps + integrate
struct IntArgs {
    uint32_t nb;
    const uint32_t *list;
    float h;
    int pinch_kill, island_mode;
    int phase;   // 0: pinch clamps then integration; 1: the pinch clamps only; 2: integration only
    uint8_t *alive, *asleep;
    float4 *pos, *q, *v, *w;
    const float4 *vpre, *wpre;
    const float *rad;
    float *sleep;
    const float *maxr;
    const uint32_t *nc, *count, *first;
    const uint8_t *kmat;
};

__device__ __forceinline__ void kill_mark(const IntArgs &A, uint32_t b) { A.alive[b] = 0; }

__global__ void k_integrate(IntArgs A) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.nb) return;
    const uint32_t b = pick(A.list, t);
    if (!A.alive[b] || A.asleep[b]) return;
    float4 t4 = A.v[b];
    V3 v = v3(t4.x, t4.y, t4.z);
    t4 = A.w[b];
    V3 w = v3(t4.x, t4.y, t4.z);
    const float rad = A.rad[b];
    // pinch_check (src/lib.rs:1746-1768)
    if (A.phase != 2) {
        float4 p4 = A.wpre[b];
        V3 wpre = v3(p4.x, p4.y, p4.z);
        p4 = A.vpre[b];
        V3 vpre = v3(p4.x, p4.y, p4.z);
        V3 dw = sub(w, wpre);
        float tip = len(dw) * rad;
        if (tip > 6.0f) w = madd(wpre, dw, div_rn(6.0f, tip));
        V3 dv = sub(v, vpre);
        float m = len(dv);
        if (m >= 8.0f && A.kmat[A.first[b]] < SLUG) {
            if (A.pinch_kill && A.count[b] <= 6) {
                A.alive[b] = 0;
                A.w[b] = make_float4(w.x, w.y, w.z, 0.0f);
                return;
            }
            v = madd(vpre, dv, div_rn(8.0f, m));
        }
        if (A.phase == 1) {
            A.v[b] = make_float4(v.x, v.y, v.z, 0.0f);
            A.w[b] = make_float4(w.x, w.y, w.z, 0.0f);
            return;
        }
    }
    // clamp_vel (src/lib.rs:917-924)
    {
        float vl = len(v);
        if (vl > 60.0f) v = mul(v, div_rn(60.0f, vl));
        float al = len(w);
        float amax = minf(25.0f, div_rn(16.0f, maxf(rad, 0.3f)));
        if (al > amax) w = mul(w, div_rn(amax, al));
    }
    const float h = A.h;
    t4 = A.pos[b];
    V3 p = madd(v3(t4.x, t4.y, t4.z), v, h);
    // q_int (src/lib.rs:100-108)
    float4 q4 = A.q[b];
    {
        V3 qv = v3(q4.x, q4.y, q4.z);
        V3 d = add(mul(w, q4.w), cross(w, qv));
        float dw = -dot(w, qv);
        float r0 = q4.x + 0.5f * h * d.x, r1 = q4.y + 0.5f * h * d.y, r2 = q4.z + 0.5f * h * d.z, r3 = q4.w + 0.5f * h * dw;
        float l = sqrt_rn(r0 * r0 + r1 * r1 + r2 * r2 + r3 * r3);
        if (l > 1e-9f) q4 = make_float4(div_rn(r0, l), div_rn(r1, l), div_rn(r2, l), div_rn(r3, l));
        else q4 = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    }
    v = mul(v, 1.0f - 0.01f * h);
    w = mul(w, 1.0f - 0.05f * h);
    const bool small = A.count[b] <= 3;
    const uint32_t nc = A.nc[b];
    if (nc > 0 && small) {
        w = mul(w, 1.0f - minf(7.0f * h, 0.5f));
        v = mul(v, 1.0f - minf(2.0f * h, 0.3f));
    }
    float v2 = dot(v, v);
    float w2 = dot(w, w) * rad * rad;
    float vt = small ? 0.16f : 0.06f, wt = small ? 0.3f : 0.04f;
    float sl = A.sleep[b];
    uint8_t asl = 0;
    if (v2 < vt && w2 < wt && nc > 0 && A.maxr[b] < 0.95f) {
        sl += h;
        if (!A.island_mode && sl > 0.45f) { asl = 1; v = v3(0.0f, 0.0f, 0.0f); w = v3(0.0f, 0.0f, 0.0f); }
    } else sl = 0.0f;
    A.sleep[b] = sl;
    if (asl) A.asleep[b] = 1;
    A.pos[b] = make_float4(p.x, p.y, p.z, 0.0f);
    A.q[b] = q4;
    A.v[b] = make_float4(v.x, v.y, v.z, 0.0f);
    A.w[b] = make_float4(w.x, w.y, w.z, 0.0f);
    if (p.y < -15.0f || fabsf(p.x) > 190.0f || fabsf(p.z) > 190.0f || p.y > 120.0f) A.alive[b] = 0;
}

__global__ void k_island_min(uint32_t nb, const uint32_t *list, const uint8_t *alive, const uint32_t *label,
                             const float *sleep, uint32_t *mint) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    uint32_t r = label[b];
    if (r == NONE || !alive[b]) return;
    atomicMin(&mint[r], __float_as_uint(sleep[b]));
}
__global__ void k_island_sleep(uint32_t nb, const uint32_t *list, const uint8_t *alive, uint8_t *asleep,
                               const uint32_t *label, const float *sleep, const uint32_t *mint, float4 *v, float4 *w) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    uint32_t r = label[b];
    if (r == NONE || !alive[b] || asleep[b]) return;
    if (__uint_as_float(mint[r]) > 0.45f || sleep[b] > 0.9f) {
        asleep[b] = 1;
        v[b] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w[b] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}
__global__ void k_wake(uint32_t nb, const uint32_t *list, uint8_t *wake, const uint8_t *alive, uint8_t *asleep,
                       float *sleep) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    if (!wake[b]) return;
    wake[b] = 0;
    if (alive[b]) { asleep[b] = 0; sleep[b] = 0.0f; }
}
__global__ void k_save_pre(uint32_t nb, const uint32_t *list, const uint8_t *alive, const float4 *v, const float4 *w,
                           float4 *vpre, float4 *wpre) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    if (!alive[b]) return;
    vpre[b] = v[b];
    wpre[b] = w[b];
}
__global__ void k_count_bodies(uint32_t nb, const uint8_t *alive, const uint8_t *asleep, uint32_t *dev) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t al = 0, aw = 0;
    if (b < nb && alive[b]) { al = 1; aw = asleep[b] ? 0 : 1; }
    al = __reduce_add_sync(0xffffffffu, al);
    aw = __reduce_add_sync(0xffffffffu, aw);
    if ((threadIdx.x & 31) == 0) {
        if (al) atomicAdd(&dev[DV_ALIVE], al);
        if (aw) atomicAdd(&dev[DV_AWAKE], aw);
    }
}
// the kill of a body also removes its bricks (kill_body, src/lib.rs:826-843)
__global__ void k_kill_bricks(uint32_t nd, const uint32_t *list, const uint32_t *kbody, const uint8_t *alive, uint8_t *kmat) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nd) return;
    const uint32_t i = pick(list, t);
    if (!alive[kbody[i]]) kmat[i] = 0;
}

// ---------------------------------------------------------------- the active set
// Scenes step only while one of their bodies is awake: a scene whose bodies all sleep (or are dead) is left
// unchanged by a substep (gen_contacts, integrate and the islands all skip sleeping bodies), so leaving it out is
// exact. A caller may also hold scenes out (a served pool steps only the scenes with work). The active scenes'
// bodies and bricks are listed in scene order; seg[k] = (body_off, body_base, brick_off, brick_base) of the k-th.
__device__ __forceinline__ uint32_t seg_of(const uint4 *seg, uint32_t K, uint32_t t, bool bricks) {
    uint32_t lo = 0, hi = K;   // last k with base <= t
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t base = bricks ? seg[mid].w : seg[mid].y;
        if (base <= t) lo = mid; else hi = mid;
    }
    return lo;
}
__global__ void k_build_lists(uint32_t K, const uint4 *seg, uint32_t nb_act, uint32_t nd_act, uint32_t *act_body,
                              uint32_t *cidx, uint32_t *act_brick) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nb_act) {
        const uint4 g = seg[seg_of(seg, K, t, false)];
        const uint32_t b = g.x + (t - g.y);
        act_body[t] = b;
        cidx[b] = t;
    }
    if (t < nd_act) {
        const uint4 g = seg[seg_of(seg, K, t, true)];
        act_brick[t] = g.z + (t - g.w);
    }
}
__global__ void k_scene_live(uint32_t nb, const uint32_t *list, const uint8_t *alive, const uint8_t *asleep,
                             const uint32_t *bscene, uint8_t *live) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    const uint32_t b = pick(list, t);
    if (alive[b] && !asleep[b]) live[bscene[b]] = 1;
}

// ---------------------------------------------------------------- host side
static int bits_for(uint64_t v) { int b = 0; while (b < 64 && (v >> b) != 0) b++; return b; }

// Sync domains for the colouring and the solve: the active scenes are cut into contiguous runs and every run gets
// blocks in proportion to its bricks (a stand-in for its contacts). A scene with at least 1 / DOM_MAX of the
// active bricks is a domain of its own; smaller ones are gathered until a run reaches that share. A run of one block
// needs only __syncthreads between colours; larger runs meet at their own grid barrier.
constexpr uint32_t DOM_MAX = 256;

static void make_partition(const sf_world *w, const StepState *S, unsigned R, bool single, StepState::Partition &P) {
    const size_t K = S->act.size();
    P.R = R;
    P.dom_of_act.assign(std::max<size_t>(K, 1), 0);
    P.blk.assign(R, make_uint4(0, 0, R, 0));
    P.D = 1;
    for (unsigned b = 0; b < R; b++) P.blk[b] = make_uint4(0, b, R, 0);
    if (single || K <= 1 || R <= 1) return;
    std::vector<double> load(K);
    double total = 0.0;
    for (size_t k = 0; k < K; k++) { load[k] = std::max(1.0, (double)w->scenes[S->act[k]].n_bricks); total += load[k]; }
    const uint32_t dmax = std::min<uint32_t>(R, DOM_MAX);
    const double target = total / dmax;
    std::vector<std::pair<size_t, size_t>> runs;
    std::vector<double> rl;
    size_t a = 0;
    double acc = 0.0;
    for (size_t k = 0; k < K; k++) {
        if (load[k] >= target) {
            if (k > a) { runs.push_back({a, k}); rl.push_back(acc); }
            runs.push_back({k, k + 1}); rl.push_back(load[k]);
            a = k + 1; acc = 0.0;
            continue;
        }
        acc += load[k];
        if (acc >= target) { runs.push_back({a, k + 1}); rl.push_back(acc); a = k + 1; acc = 0.0; }
    }
    if (a < K) { runs.push_back({a, K}); rl.push_back(acc); }
    // a large scene can split a gathering run in two: merge the lightest neighbouring pair until dmax runs remain
    while (runs.size() > dmax) {
        size_t best = 0;
        for (size_t i = 1; i + 1 < runs.size(); i++) if (rl[i] + rl[i + 1] < rl[best] + rl[best + 1]) best = i;
        runs[best].second = runs[best + 1].second;
        rl[best] += rl[best + 1];
        runs.erase(runs.begin() + best + 1);
        rl.erase(rl.begin() + best + 1);
    }
    const size_t D = runs.size();
    std::vector<unsigned> nb(D);
    unsigned sum = 0;
    for (size_t d = 0; d < D; d++) { nb[d] = std::max(1u, (unsigned)(rl[d] * R / total)); sum += nb[d]; }
    while (sum > R) {   // take a block from the run that has the most blocks per load
        size_t best = D;
        for (size_t d = 0; d < D; d++)
            if (nb[d] > 1 && (best == D || nb[d] / rl[d] > nb[best] / rl[best])) best = d;
        nb[best]--; sum--;
    }
    while (sum < R) {   // give a block to the run with the most load per block
        size_t best = 0;
        for (size_t d = 1; d < D; d++) if (rl[d] / nb[d] > rl[best] / nb[best]) best = d;
        nb[best]++; sum++;
    }
    P.D = (uint32_t)D;
    unsigned b = 0;
    for (size_t d = 0; d < D; d++) {
        for (size_t k = runs[d].first; k < runs[d].second; k++) P.dom_of_act[k] = (uint32_t)d;
        for (unsigned r = 0; r < nb[d]; r++) P.blk[b++] = make_uint4((uint32_t)d, r, nb[d], 0);
    }
}

// the partition for a launch of R blocks over the current active set (built once per active set and launch size)
static sf_status use_partition(sf_world *w, unsigned R, bool single) {
    StepState *S = w->step;
    const unsigned key = single ? 0x80000000u | R : R;
    size_t at = S->parts.size();
    for (size_t k = 0; k < S->parts.size(); k++) if (S->parts[k].R == key) at = k;
    if (at == S->parts.size()) {
        S->parts.emplace_back();
        make_partition(w, S, R, single, S->parts.back());
        S->parts.back().R = key;
    }
    StepState::Partition &P = S->parts[at];
    // the blocks' table and the scenes' domains, uploaded when the partition in use changes
    if (S->part_in_use != (int)at) {
        cudaStream_t s = w->stream;
        SF_CUDA(S->blk_dom.grow(P.blk.size()));
        SF_CUDA(S->dom_of_act.grow(P.dom_of_act.size()));
        SF_CUDA(cudaMemcpyAsync(S->blk_dom.p, P.blk.data(), P.blk.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
        SF_CUDA(cudaMemcpyAsync(S->dom_of_act.p, P.dom_of_act.data(), P.dom_of_act.size() * 4, cudaMemcpyHostToDevice, s));
        S->part_in_use = (int)at;
    }
    S->part_D = P.D;
    return SF_OK;
}

static cudaError_t grow_contacts(StepState *S, uint64_t need) {
    if (need <= S->capacity) return cudaSuccess;
    uint64_t cap = std::max<uint64_t>(need + need / 2, 4096);
    cudaError_t e;
#define G(buf) if ((e = S->buf.alloc(cap)) != cudaSuccess) return e
    G(L_a); G(L_b); G(L_bo); G(L_ba); G(L_bb); G(L_p); G(L_n);
    G(mkey); G(mkey_alt); G(perm); G(perm_alt); G(invperm); G(mflag); G(mpos); G(pair_start); G(cflag); G(cpos);
    G(man_a); G(man_b); G(man_ca); G(man_cb); G(man_start); G(man_count); G(man_prio); G(man_color); G(man_round); G(man_dom);
    G(S_n); G(S_t1); G(S_t2); G(S_ra); G(S_rb); G(S_j);
    G(wl0); G(wl1); G(col_list);
    G(red_big); G(red_pos); G(red_keep); G(red_kpos);
#undef G
    if ((e = S->red_slots.alloc(2 * 27 * (cap / 33 + 1))) != cudaSuccess) return e;
    if ((e = S->bm_list.alloc(2 * cap)) != cudaSuccess) return e;
    S->capacity = cap;
    return cudaSuccess;
}

void step_warm_invalidate(sf_world *w, uint32_t scene) {
    StepState *S = w->step;
    if (!S || scene >= S->warm_scene.size()) return;
    S->warm_scene[scene] = 0;
    S->warm_scene_dirty = true;
}

sf_status step_create(sf_world *w) {
    StepState *S = new StepState();
    w->step = S;
    uint32_t nb = w->nb, nd = w->nd;
    const uint32_t nsc = std::max<uint32_t>(w->n_scenes, 1);
    S->warm_scene.assign(nsc, 0);
    cudaStream_t s = w->stream;
    SF_CUDA(S->ckey.alloc(nd)); SF_CUDA(S->ckey_alt.alloc(nd)); SF_CUDA(S->cval.alloc(nd));
    SF_CUDA(S->aw_flag.alloc(nd)); SF_CUDA(S->awk_pos.alloc(nd)); SF_CUDA(S->awk_list.alloc(nd));
    SF_CUDA(S->bucket_bits.alloc((size_t)nsc * (HSIZE / 32)));
    SF_CUDA(S->scene_awake.alloc(nsc)); SF_CUDA(S->scene_bricks.alloc(nsc));
    SF_CUDA(S->bstart.alloc((size_t)nsc * HSIZE + 1));
    SF_CUDA(S->srec.alloc(nd)); SF_CUDA(S->sent.alloc(nd));
    SF_CUDA(S->slot_id.alloc((size_t)nd * CSLOTS)); SF_CUDA(S->slot_p.alloc((size_t)nd * CSLOTS)); SF_CUDA(S->slot_n.alloc((size_t)nd * CSLOTS));
    SF_CUDA(S->ccount.alloc((size_t)nd + 1)); SF_CUDA(S->coff.alloc((size_t)nd + 1));
    SF_CUDA(S->bm_count.alloc((size_t)nb + 1)); SF_CUDA(S->bm_start.alloc((size_t)nb + 1)); SF_CUDA(S->bm_fill.alloc((size_t)nb + 1));
    const uint32_t mw = (w->P.max_colors + 31) / 32;
    SF_CUDA(S->masks.alloc((size_t)nb * mw + mw)); SF_CUDA(S->vmasks.alloc((size_t)nb * mw + mw));
    {
        const size_t nseg = (size_t)DOM_MAX * w->P.max_colors;
        SF_CUDA(S->col_count.alloc(nseg * JDS_ROW + 1)); SF_CUDA(S->col_start.alloc(nseg + 2));
        SF_CUDA(S->col_fill.alloc(nseg * JDS_ROW + 1)); SF_CUDA(S->jds_off.alloc(nseg * JDS_K));
        SF_CUDA(S->col_hstart.alloc(nseg * JDS_ROW + 1)); SF_CUDA(S->seg_tot.alloc(nseg)); SF_CUDA(S->seg_base.alloc(nseg));
        SF_CUDA(S->dom_m0.alloc(DOM_MAX)); SF_CUDA(S->dom_m1.alloc(DOM_MAX)); SF_CUDA(S->dom_ncol.alloc(DOM_MAX));
        SF_CUDA(S->dom_cnt.alloc(3 * DOM_MAX)); SF_CUDA(S->dom_gb.alloc(DOM_MAX));
    }
    if (w->P.manifold_chunk == 0 || w->P.manifold_chunk > (uint32_t)JDS_K) w->P.manifold_chunk = JDS_K;
    SF_CUDA(S->parent.alloc(nb)); SF_CUDA(S->label.alloc(nb)); SF_CUDA(S->mint.alloc(nb));
    SF_CUDA(cudaMemsetAsync(S->label.p, 0xFF, S->label.bytes(), s));
    SF_CUDA(S->act_body.alloc(nb)); SF_CUDA(S->cidx.alloc(nb)); SF_CUDA(S->act_brick.alloc(nd));
    SF_CUDA(S->scene_act.alloc(nsc)); SF_CUDA(S->seg.alloc(nsc)); SF_CUDA(S->live_dev.alloc(nsc));
    SF_CUDA(cudaMallocHost((void **)&S->h_live_pin, nsc));
    S->live.assign(w->n_scenes, 1);   // every scene steps until a step shows it asleep
    S->act_brick_base.assign(w->n_scenes, NONE);
    SF_CUDA(S->dev.alloc(DV_N));
    SF_CUDA(cudaMemsetAsync(S->dev.p, 0, S->dev.bytes(), s));
    SF_CUDA(cudaMallocHost((void **)&S->h_dev, DV_N * sizeof(uint32_t)));
    std::vector<uint32_t> off(nb);
    for (const Scene &sc : w->scenes) {
        for (uint32_t b = 0; b < sc.n_bodies; b++) off[sc.body_off + b] = sc.body_off;
        S->max_scene_bodies = std::max(S->max_scene_bodies, sc.n_bodies);
    }
    SF_CUDA(S->body_off_of_body.alloc(nb));
    if (nb) SF_CUDA(cudaMemcpyAsync(S->body_off_of_body.p, off.data(), nb * 4, cudaMemcpyHostToDevice, s));
    uint64_t initial = w->P.contact_capacity ? w->P.contact_capacity : (uint64_t)std::max<uint32_t>(nd, 1) * 4;
    SF_CUDA(grow_contacts(S, initial));
    int occ = 0;
    SF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_solve, SOLVE_BLOCK, 0));
    S->solve_occ = std::max(1, occ);
    SF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_jp, SOLVE_BLOCK, 0));
    S->jp_occ = std::max(1, occ);
    {
        // the colouring and the solve run on the same blocks (one partition into sync domains serves both)
        const int top = std::min(S->solve_occ, S->jp_occ);
        int c[4], n = 0;
        for (int v = 1; v <= 4; v++) if (v <= top) c[n++] = v;
        S->solve_t.init(c, n);
    }
    SF_CUDA(cudaStreamSynchronize(s));   // the host vector `off` is the copy's source
    return SF_OK;
}

cudaError_t refresh_poses(sf_world *w) {
    const uint32_t nb = w->nb, nd = w->nd;
    if (nb == 0 || nd == 0) return cudaSuccess;
    cudaStream_t s = w->stream;
    // h = 0: v.y - 0 leaves every velocity bit unchanged
    k_update_cache<<<grid_for(nb, 128), 128, 0, s>>>(nb, nullptr, 0.0f, w->b_alive.p, w->b_asleep.p, w->b_q.p, w->b_iil.p,
                                                     w->b_rot.p, w->b_iiw.p, w->b_v.p, nullptr);
    k_brick_pos<<<grid_for(nd, 256), 256, 0, s>>>(nd, nullptr, w->k_body.p, w->b_alive.p, w->b_asleep.p, w->b_pos.p,
                                                  w->b_rot.p, w->k_local.p, w->k_wpos.p);
    w->launches += 2;
    return cudaGetLastError();
}

static cudaEvent_t tune_event(StepState *S) {
    if (S->tev_used == S->tev.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        S->tev.push_back(e);
    }
    return S->tev[S->tev_used++];
}
// time a tuned launch: events around it, resolved after the step
static void tune_begin(StepState *S, Tuner *t, int bucket, int ci, cudaStream_t s) {
    if (ci < 0) return;
    cudaEvent_t e0 = tune_event(S), e1 = tune_event(S);
    if (!e0 || !e1) return;
    cudaEventRecord(e0, s);
    S->pending.push_back({t, bucket, ci, e0, e1});
}
static void tune_end(StepState *S, int ci, cudaStream_t s) {
    if (ci < 0 || S->pending.empty()) return;
    cudaEventRecord(S->pending.back().e1, s);
}
static void tune_resolve(StepState *S) {
    for (const StepState::Pending &p : S->pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.e0, p.e1) == cudaSuccess) p.t->record(p.bucket, p.ci, ms);
    }
    S->pending.clear();
    S->tev_used = 0;
}

void step_destroy(sf_world *w) {
    if (w->step) for (cudaEvent_t e : w->step->tev) cudaEventDestroy(e);
    if (w->step) for (cudaEvent_t e : w->step->gen_ev) cudaEventDestroy(e);
    if (w->step) for (cudaEvent_t e : w->step->ev_pool) cudaEventDestroy(e);
    if (w->step && w->step->h_dev) cudaFreeHost(w->step->h_dev);
    if (w->step && w->step->h_live_pin) cudaFreeHost(w->step->h_live_pin);
    delete w->step;
    w->step = nullptr;
}

void step_mark_live(sf_world *w, uint32_t scene) {
    if (w->step && scene < w->step->live.size()) w->step->live[scene] = 1;
}
void step_mark_all_live(sf_world *w) {
    if (w->step) std::fill(w->step->live.begin(), w->step->live.end(), (uint8_t)1);
}
void step_set_live(sf_world *w, uint32_t scene, bool live) {
    if (w->step && scene < w->step->live.size()) w->step->live[scene] = live ? 1 : 0;
}
cudaError_t step_reset_labels(sf_world *w, uint32_t first_body, uint32_t n) {
    if (!w->step || n == 0) return cudaSuccess;
    return cudaMemsetAsync(w->step->label.p + first_body, 0xFF, (size_t)n * 4, w->stream);
}

// The active set of the next step: live scenes the caller lets step. Lists are rebuilt only when the set changes.
static sf_status set_active(sf_world *w, const uint8_t *mask) {
    StepState *S = w->step;
    cudaStream_t s = w->stream;
    std::vector<uint32_t> act;
    for (uint32_t q = 0; q < w->n_scenes; q++)
        if (S->live[q] && (!mask || mask[q]) && w->scenes[q].n_bodies) act.push_back(q);
    if (S->act_valid && act == S->act) return SF_OK;
    // scenes that fell asleep leave the set: their bodies' island labels are those of sleeping bodies
    for (uint32_t q : S->act)
        if (!S->live[q] && !std::binary_search(act.begin(), act.end(), q)) {
            const Scene &sc = w->scenes[q];
            SF_CUDA(cudaMemsetAsync(S->label.p + sc.body_off, 0xFF, (size_t)sc.n_bodies * 4, s));
        }
    std::vector<uint32_t> scene_act(std::max<uint32_t>(w->n_scenes, 1), NONE);
    std::vector<uint4> seg(std::max<size_t>(act.size(), 1));
    std::vector<uint32_t> nbr(std::max<size_t>(act.size(), 1), 0);
    uint32_t nb_act = 0, nd_act = 0;
    for (size_t k = 0; k < act.size(); k++) {
        const Scene &sc = w->scenes[act[k]];
        scene_act[act[k]] = (uint32_t)k;
        seg[k] = make_uint4(sc.body_off, nb_act, sc.brick_off, nd_act);
        nbr[k] = sc.n_bricks;
        nb_act += sc.n_bodies;
        nd_act += sc.n_bricks;
    }
    SF_CUDA(cudaMemcpyAsync(S->scene_bricks.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(S->scene_act.p, scene_act.data(), scene_act.size() * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(S->seg.p, seg.data(), seg.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    const uint32_t n = std::max(nb_act, nd_act);
    if (n) {
        k_build_lists<<<grid_for(n, 256), 256, 0, s>>>((uint32_t)act.size(), S->seg.p, nb_act, nd_act, S->act_body.p,
                                                       S->cidx.p, S->act_brick.p);
        w->launches++;
    }
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaStreamSynchronize(s));   // the host vectors above are the copies' sources
    S->act = std::move(act);
    S->nb_act = nb_act;
    S->nd_act = nd_act;
    S->act_valid = true;
    S->parts.clear();
    S->part_in_use = -1;
    return SF_OK;
}

static sf_status substep(sf_world *w, float h) {
    StepState *S = w->step;
    cudaStream_t s = w->stream;
    const uint32_t nb = S->nb_act, nd = S->nd_act;
    const uint32_t *blist = S->act_body.p, *klist = S->act_brick.p;
    if ((uint64_t)S->act.size() * HSIZE >= 0xFFFFFFFFull) {
        set_error("%zu active scenes exceed the hash key range", S->act.size());
        return SF_ERR_CAPACITY;
    }
    std::fill(S->act_brick_base.begin(), S->act_brick_base.end(), NONE);
    if (!w->P.warm_start) S->warm_valid = false;
    if (nb == 0 || nd == 0) {
        S->warm_valid = false;   // no contacts this substep: the next one finds none
        SF_CUDA(cudaMemsetAsync(S->dev.p, 0, DV_ALIVE * sizeof(uint32_t), s));
        SF_CUDA(cudaMemsetAsync(S->dev.p + DV_ISLANDS, 0, (DV_N - DV_ISLANDS) * sizeof(uint32_t), s));
        for (int p = 0; p <= SF_PHASES; p++) prof_mark(w);
        if (S->profile) S->sub_nc.push_back(0);
        S->have_contacts = true;
        return SF_OK;
    }
    {
        uint32_t base = 0;
        for (uint32_t q : S->act) { S->act_brick_base[q] = base; base += w->scenes[q].n_bricks; }
    }
    uint64_t &L = w->launches;
    // pose cache + gravity, brick positions
    prof_mark(w);
    k_update_cache<<<grid_for(nb, 128), 128, 0, s>>>(nb, blist, h, w->b_alive.p, w->b_asleep.p, w->b_q.p, w->b_iil.p,
                                                     w->b_rot.p, w->b_iiw.p, w->b_v.p, w->b_nc.p);
    k_brick_pos<<<grid_for(nd, 256), 256, 0, s>>>(nd, klist, w->k_body.p, w->b_alive.p, w->b_asleep.p, w->b_pos.p,
                                                  w->b_rot.p, w->k_local.p, w->k_wpos.p);
    L += 2;
    prof_mark(w);
    // Sparse form (most bricks asleep): the awake bricks, in active-list order, and the hashed cells they can reach.
    // Dense form: every live brick hashed, every active brick a contact thread. Both give the same contacts.
    const bool sparse = S->use_sparse;
    S->last_sparse = sparse;
    uint32_t n_awk = nd;
    const uint32_t *clist = klist;
    const size_t nbk = S->act.size() * (size_t)HSIZE;
    if (sparse) {
        clist = S->awk_list.p;
        SF_CUDA(cudaMemsetAsync(S->scene_awake.p, 0, S->act.size() * 4, s));
        k_awake_flags<<<grid_for(nd, 256), 256, 0, s>>>(nd, klist, w->k_body.p, w->b_scene.p, S->scene_act.p, w->b_alive.p,
                                                        w->b_asleep.p, S->aw_flag.p, S->scene_awake.p);
        SF_CUDA(exclusive_scan_u32(S->aw_flag.p, S->awk_pos.p, nd, S->dev.p + DV_AWK, S->wk, s));
        k_compact_list<<<grid_for(nd, 256), 256, 0, s>>>(nd, klist, S->aw_flag.p, S->awk_pos.p, S->awk_list.p);
        SF_CUDA(cudaMemsetAsync(S->bucket_bits.p, 0, (size_t)S->act.size() * (HSIZE / 32) * 4, s));
        k_mark_buckets<<<grid_for(nd, 128), 128, 0, s>>>(S->dev.p + DV_AWK, S->awk_list.p, w->k_body.p, w->b_scene.p,
                                                         S->scene_act.p, S->scene_awake.p, S->scene_bricks.p, w->k_wpos.p,
                                                         S->bucket_bits.p);
        L += 3;
    }
    // the hash table (counting sort into the buckets; see k_hash_count)
    SF_CUDA(cudaMemsetAsync(S->bstart.p, 0, nbk * 4, s));
    k_hash_count<<<grid_for(nd, 256), 256, 0, s>>>(nd, klist, w->k_body.p, w->b_scene.p, S->scene_act.p,
                                                   sparse ? S->scene_awake.p : nullptr, S->scene_bricks.p, w->b_alive.p,
                                                   w->b_asleep.p, w->k_wpos.p, sparse ? S->bucket_bits.p : nullptr,
                                                   S->bstart.p, S->ckey.p, S->ckey_alt.p);
    SF_CUDA(exclusive_scan_u32(S->bstart.p, S->bstart.p, nbk, S->bstart.p + nbk, S->wk, s));
    k_hash_place<<<grid_for(nd, 256), 256, 0, s>>>(nd, klist, S->ckey.p, S->ckey_alt.p, S->bstart.p, S->cval.p);
    k_hash_order<<<grid_for(nbk, 256), 256, 0, s>>>((uint32_t)nbk, S->bstart.p, S->cval.p);
    k_bucket_records<<<grid_for(nd, 256), 256, 0, s>>>(S->bstart.p + nbk, S->cval.p, w->k_body.p, w->k_mat.p, w->b_asleep.p,
                                                       w->k_wpos.p, S->srec.p, S->sent.p);
    L += 4;
    if (sparse) {
        SF_CUDA(cudaMemcpyAsync(S->h_dev + DV_AWK, S->dev.p + DV_AWK, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
        n_awk = S->h_dev[DV_AWK];
    }
    S->n_awk = n_awk;
    prof_mark(w);
    // contacts: generate into slots and count, scan, place in list order
    ContactArgs C;
    C.nd = n_awk; C.list = clist; C.scene_act = S->scene_act.p;
    C.sbox = w->sbox.p; C.kbody = w->k_body.p; C.bscene = w->b_scene.p; C.ctab = w->ctab.p; C.cpool = w->cpool.p;
    C.alive = w->b_alive.p; C.asleep = w->b_asleep.p; C.smat = w->s_mat.p; C.wpos = w->k_wpos.p;
    C.v = w->b_v.p; C.w = w->b_w.p; C.rot = w->b_rot.p; C.rad = w->b_rad.p; C.bstart = S->bstart.p; C.srec = S->srec.p;
    C.sent = S->sent.p; C.ccount = S->ccount.p; C.coff = S->coff.p; C.wake = w->b_wake.p;
    C.sup = w->k_sup.p; C.frame = w->frame;
    C.slot_id = S->slot_id.p; C.slot_p = S->slot_p.p; C.slot_n = S->slot_n.p;
    C.L_a = S->L_a.p; C.L_b = S->L_b.p; C.L_bo = S->L_bo.p; C.L_ba = S->L_ba.p; C.L_bb = S->L_bb.p; C.L_p = S->L_p.p; C.L_n = S->L_n.p;
    cudaEvent_t g0 = nullptr, g1 = nullptr;
    if (S->profile && n_awk) {
        while (S->gen_ev.size() < S->gen_used + 2) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) break;
            S->gen_ev.push_back(e);
        }
        if (S->gen_ev.size() >= S->gen_used + 2) {
            g0 = S->gen_ev[S->gen_used]; g1 = S->gen_ev[S->gen_used + 1];
            S->gen_used += 2;
            S->gen_bricks += n_awk;
        }
    }
    if (g0) cudaEventRecord(g0, s);
    if (n_awk) k_contacts_gen<<<grid_for(n_awk, 128), 128, 0, s>>>(C);
    if (g1) cudaEventRecord(g1, s);
    SF_CUDA(exclusive_scan_u32(S->ccount.p, S->coff.p, n_awk, S->dev.p + DV_CONTACTS, S->wk, s));
    SF_CUDA(cudaMemcpyAsync(S->h_dev, S->dev.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    const uint32_t nc = S->h_dev[DV_CONTACTS];
    S->last_contacts = nc;
    if (nc > S->capacity) {
        if (w->P.contact_capacity) { set_error("%u contacts exceed the fixed capacity %llu", nc, (unsigned long long)S->capacity); return SF_ERR_CAPACITY; }
        SF_CUDA(grow_contacts(S, nc));
        C.L_a = S->L_a.p; C.L_b = S->L_b.p; C.L_bo = S->L_bo.p; C.L_ba = S->L_ba.p; C.L_bb = S->L_bb.p; C.L_p = S->L_p.p; C.L_n = S->L_n.p;
    }
    if (n_awk) k_contacts_place<<<grid_for(n_awk, 128), 128, 0, s>>>(C);
    SF_CUDA(cudaMemsetAsync(S->dev.p + DV_MANIFOLDS, 0, (DV_N - DV_MANIFOLDS) * sizeof(uint32_t), s));
    const uint32_t g_nc = grid_for(std::max<uint32_t>(nc, 1), 256);
    if (nc) { k_body_nc<<<g_nc, 256, 0, s>>>(nc, S->L_a.p, S->L_b.p, w->b_nc.p); L++; }
    L += 1;
    // plough (src/lib.rs:1776), with damage on: may knock static bricks loose as new bodies and switch contacts off
    uint32_t n_loose = 0;
    if (w->P.damage && nc) {
        SF_CUDA(S->c_off.grow(nc));
        PloughIn PI;
        PI.nc = nc; PI.L_a = S->L_a.p; PI.L_b = S->L_b.p; PI.L_bo = S->L_bo.p; PI.L_bb = S->L_bb.p; PI.L_p = S->L_p.p;
        PI.L_n = S->L_n.p; PI.off = S->c_off.p; PI.wk = &S->wk;
        SF_CUDA(plough_substep(w, PI, s, &n_loose));
    }
    if (S->profile) S->sub_nc.push_back(nc);
    prof_mark(w);
    // The launch size of the colouring and the solve, and its partition into sync domains. A substep with few contacts
    // is solved by one block (k_solve_one_block); its colouring then runs as a single domain.
    const bool one_block = nc <= SOLVE_ONE_BLOCK_MAX_CONTACTS;
    int sci = -1;
    const int sb = Tuner::bucket(nc);
    const unsigned top_occ = (unsigned)std::min(S->solve_occ, S->jp_occ);
    unsigned per_sm = w->P.solve_blocks ? std::min<unsigned>(w->P.solve_blocks, top_occ)
                                        : (unsigned)S->solve_t.choose(sb, sci);
    if (one_block) sci = -1;
    // A small substep (at most SMALL_SUBSTEP_CONTACTS contacts) colours on one block, whose rounds end at
    // __syncthreads instead of a grid barrier: a body with many chunks (a large piece on the ground) needs a round per
    // colour, and the rounds, not the work, set the time.
    const unsigned R = (one_block && nc <= SMALL_SUBSTEP_CONTACTS)
                           ? 1u
                           : (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)w->sms * per_sm,
                                                                                (nc + SOLVE_BLOCK - 1) / SOLVE_BLOCK + 1));
    const uint32_t cstride = w->P.max_colors;
    uint32_t ncm = nc;   // the contacts that enter the manifolds (fewer after a contact reduction)
    // manifolds
    if (nc) {
        sf_status pst = use_partition(w, R, one_block);
        if (pst != SF_OK) return pst;
        const uint32_t D = S->part_D;
        const uint64_t span = (uint64_t)S->max_scene_bodies + 1;
        k_man_keys<<<g_nc, 256, 0, s>>>(nc, span, S->L_a.p, S->L_b.p, S->body_off_of_body.p, S->mkey.p, S->perm.p);
        bool alt = false;
        SF_CUDA(radix_sort_u64(S->mkey.p, S->perm.p, S->mkey_alt.p, S->perm_alt.p, nc, bits_for((uint64_t)w->nb * span + span), S->wk, s, &alt));
        if (alt) { S->mkey.swap(S->mkey_alt); S->perm.swap(S->perm_alt); }
        const uint32_t K = w->P.manifold_chunk;
        uint32_t ncs = nc;   // the sorted contacts still on (plough switches some off)
        if (n_loose) {
            k_off_keep<<<g_nc, 256, 0, s>>>(nc, S->perm.p, S->c_off.p, S->red_keep.p);
            SF_CUDA(exclusive_scan_u32(S->red_keep.p, S->red_kpos.p, nc, S->dev.p + DV_KEPT, S->wk, s));
            k_red_compact<<<g_nc, 256, 0, s>>>(nc, S->red_keep.p, S->red_kpos.p, S->perm.p, S->mkey.p, S->perm_alt.p,
                                               S->mkey_alt.p);
            S->perm.swap(S->perm_alt);
            S->mkey.swap(S->mkey_alt);
            SF_CUDA(cudaMemcpyAsync(S->h_dev + DV_KEPT, S->dev.p + DV_KEPT, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            SF_CUDA(cudaStreamSynchronize(s));
            ncs = S->h_dev[DV_KEPT];
            L += 2;
        }
        ncm = ncs;
        if (ncs) {
        k_man_flags<<<g_nc, 256, 0, s>>>(ncs, S->mkey.p, S->mflag.p);
        SF_CUDA(exclusive_scan_u32(S->mflag.p, S->mpos.p, ncs, S->dev.p + DV_PAIRS, S->wk, s));
        k_pair_start<<<g_nc, 256, 0, s>>>(ncs, S->mflag.p, S->mpos.p, S->pair_start.p);
        }
        if (w->P.reduce && ncs) {
            k_red_big<<<g_nc, 256, 0, s>>>(ncs, S->dev.p + DV_PAIRS, S->pair_start.p, S->red_big.p);
            SF_CUDA(exclusive_scan_u32(S->red_big.p, S->red_pos.p, ncs, S->dev.p + DV_NBIG, S->wk, s));
            SF_CUDA(cudaMemsetAsync(S->red_slots.p, 0, S->red_slots.bytes(), s));
            uint32_t *best = S->red_slots.p, *win = S->red_slots.p + S->red_slots.n / 2;
            k_red_score<<<g_nc, 256, 0, s>>>(ncs, S->mflag.p, S->mpos.p, S->red_big.p, S->red_pos.p, S->perm.p, S->L_p.p,
                                             S->L_n.p, best);
            k_red_pick<<<g_nc, 256, 0, s>>>(ncs, S->mflag.p, S->mpos.p, S->red_big.p, S->red_pos.p, S->perm.p, S->L_p.p,
                                            S->L_n.p, best, win);
            k_red_keep<<<g_nc, 256, 0, s>>>(ncs, S->mflag.p, S->mpos.p, S->red_big.p, S->red_pos.p, S->perm.p, win,
                                            S->red_keep.p);
            SF_CUDA(exclusive_scan_u32(S->red_keep.p, S->red_kpos.p, ncs, S->dev.p + DV_KEPT, S->wk, s));
            k_red_compact<<<g_nc, 256, 0, s>>>(ncs, S->red_keep.p, S->red_kpos.p, S->perm.p, S->mkey.p, S->perm_alt.p,
                                               S->mkey_alt.p);
            S->perm.swap(S->perm_alt);
            S->mkey.swap(S->mkey_alt);
            SF_CUDA(cudaMemcpyAsync(S->h_dev + DV_KEPT, S->dev.p + DV_KEPT, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            SF_CUDA(cudaStreamSynchronize(s));
            ncm = S->h_dev[DV_KEPT];
            // the pairs again, over the kept contacts (every pair keeps at least one)
            k_man_flags<<<g_nc, 256, 0, s>>>(ncm, S->mkey.p, S->mflag.p);
            SF_CUDA(exclusive_scan_u32(S->mflag.p, S->mpos.p, ncm, S->dev.p + DV_PAIRS, S->wk, s));
            k_pair_start<<<g_nc, 256, 0, s>>>(ncm, S->mflag.p, S->mpos.p, S->pair_start.p);
            L += 8;
        }
        k_chunk_flags<<<g_nc, 256, 0, s>>>(ncm, K, S->mflag.p, S->mpos.p, S->pair_start.p, S->cflag.p);
        SF_CUDA(exclusive_scan_u32(S->cflag.p, S->cpos.p, ncm, S->dev.p + DV_MANIFOLDS, S->wk, s));
        k_man_write<<<g_nc, 256, 0, s>>>(ncm, K, S->cflag.p, S->cpos.p, S->mflag.p, S->mpos.p, S->pair_start.p, S->perm.p,
                                         S->L_a.p, S->L_b.p, S->body_off_of_body.p, S->cidx.p, w->b_scene.p, S->scene_act.p,
                                         S->dom_of_act.p, S->man_a.p, S->man_b.p, S->man_ca.p, S->man_cb.p, S->man_start.p,
                                         S->man_prio.p, S->man_dom.p);
        k_man_count<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, ncm, S->man_start.p, S->man_count.p);
        SF_CUDA(cudaMemsetAsync(S->dom_m0.p, 0, (size_t)D * 4, s));
        SF_CUDA(cudaMemsetAsync(S->dom_m1.p, 0, (size_t)D * 4, s));
        k_dom_ranges<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_dom.p, S->dom_m0.p, S->dom_m1.p);
        L += 7;
        prof_mark(w);
        // colouring, on the active list's body ids, each domain on its own blocks
        SF_CUDA(cudaMemsetAsync(S->bm_count.p, 0, ((size_t)nb + 1) * 4, s));
        SF_CUDA(cudaMemsetAsync(S->bm_fill.p, 0, ((size_t)nb + 1) * 4, s));
        const uint32_t mw = (w->P.max_colors + 31) / 32;
        SF_CUDA(cudaMemsetAsync(S->masks.p, 0, (size_t)nb * mw * 4, s));
        SF_CUDA(cudaMemsetAsync(S->man_round.p, 0xFF, (size_t)nc * 4, s));
        k_bm_count<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_ca.p, S->man_cb.p, S->bm_count.p,
                                        S->dev.p + DV_MAXDEG);
        SF_CUDA(exclusive_scan_u32(S->bm_count.p, S->bm_start.p, (size_t)nb + 1, nullptr, S->wk, s));
        k_bm_fill<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_ca.p, S->man_cb.p, S->bm_start.p, S->bm_fill.p, S->bm_list.p);
        SF_CUDA(cudaMemsetAsync(S->dom_gb.p, 0, (size_t)D * sizeof(GridBarrier), s));
        SF_CUDA(cudaMemsetAsync(S->dom_cnt.p, 0, (size_t)D * 3 * 4, s));
        JpArgs J;
        J.man_a = S->man_ca.p; J.man_b = S->man_cb.p; J.prio = S->man_prio.p;
        J.bm_start = S->bm_start.p; J.bm_list = S->bm_list.p; J.man_round = S->man_round.p; J.man_color = S->man_color.p;
        J.masks = S->masks.p; J.wl0 = S->wl0.p; J.wl1 = S->wl1.p; J.dev = S->dev.p; J.blk_dom = S->blk_dom.p;
        J.dom_m0 = S->dom_m0.p; J.dom_m1 = S->dom_m1.p; J.dom_cnt = S->dom_cnt.p; J.max_colors = w->P.max_colors; J.mw = mw;
        J.max_rounds = 1u << 16; J.gb = S->dom_gb.p; J.err = w->err.p;
        void *jargs[] = {&J};
        J.seq_launched = nc <= SEQ_COLOUR_LAUNCH ? 1u : 0u;
        if (J.seq_launched) k_colour_seq<<<1, SEQ_T, 0, s>>>(J);
        SF_CUDA(cudaLaunchCooperativeKernel((void *)k_jp, dim3(R), dim3(SOLVE_BLOCK), jargs, 0, s));
        // colour lists: each (domain, colour) segment's manifolds by contact count (most first), and the contact layout
        const uint32_t nseg = D * cstride;
        SF_CUDA(cudaMemsetAsync(S->col_count.p, 0, (size_t)nseg * JDS_ROW * 4, s));
        SF_CUDA(cudaMemsetAsync(S->col_fill.p, 0, (size_t)nseg * JDS_ROW * 4, s));
        SF_CUDA(cudaMemsetAsync(S->dom_ncol.p, 0, (size_t)D * 4, s));
        k_col_count<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_color.p, S->man_count.p, S->man_dom.p, cstride,
                                         S->col_count.p, S->dom_ncol.p, S->dev.p);
        SF_CUDA(exclusive_scan_u32(S->col_count.p, S->col_hstart.p, (size_t)nseg * JDS_ROW, nullptr, S->wk, s));
        k_col_fill<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_color.p, S->man_count.p, S->man_dom.p, cstride,
                                        S->col_hstart.p, S->col_fill.p, S->col_list.p);
        k_seg_totals<<<grid_for(nseg, 128), 128, 0, s>>>(nseg, S->col_count.p, S->seg_tot.p);
        SF_CUDA(exclusive_scan_u32(S->seg_tot.p, S->seg_base.p, nseg, nullptr, S->wk, s));
        k_seg_table<<<grid_for(nseg, 128), 128, 0, s>>>(nseg, S->col_count.p, S->col_hstart.p, S->seg_base.p,
                                                        S->dev.p + DV_MANIFOLDS, S->col_start.p, S->jds_off.p);
        L += 6;
        if (w->P.verify) {
            SF_CUDA(cudaMemsetAsync(S->vmasks.p, 0, (size_t)nb * mw * 4, s));
            k_col_verify<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_ca.p, S->man_cb.p, S->man_color.p, mw,
                                              S->vmasks.p, w->err.p);
            L++;
        }
        prof_mark(w);
        PrepArgs PA;
        PA.nc = nc; PA.h = h; PA.nseg = nseg; PA.nm_p = S->dev.p + DV_MANIFOLDS; PA.perm = S->perm.p;
        PA.man_a = S->man_a.p; PA.man_b = S->man_b.p; PA.man_count = S->man_count.p; PA.L_p = S->L_p.p; PA.L_n = S->L_n.p;
        PA.man_start = S->man_start.p; PA.col_start = S->col_start.p; PA.col_list = S->col_list.p;
        PA.jds_off = S->jds_off.p;
        PA.pos = w->b_pos.p; PA.v = w->b_v.p; PA.w = w->b_w.p; PA.im = w->b_im.p; PA.iiw = w->b_iiw.p;
        PA.S_n = S->S_n.p; PA.S_t1 = S->S_t1.p; PA.S_t2 = S->S_t2.p; PA.S_ra = S->S_ra.p; PA.S_rb = S->S_rb.p; PA.S_j = S->S_j.p;
        PA.invperm = S->invperm.p;
        const bool warm_read = w->P.warm_start && S->warm_valid;
        const StepState::WarmTable &WT = S->warm[S->warm_cur];
        PA.warm = warm_read ? 1 : 0;
        PA.wt = WarmRef{WT.claim.p, WT.k1.p, WT.k2.p, WT.val.p, WT.mask};
        PA.L_b = S->L_b.p; PA.L_bo = S->L_bo.p; PA.L_ba = S->L_ba.p; PA.L_bb = S->L_bb.p;
        if (warm_read && S->warm_scene_dirty) {
            SF_CUDA(S->warm_scene_dev.grow(w->n_scenes));
            SF_CUDA(cudaMemcpyAsync(S->warm_scene_dev.p, S->warm_scene.data(), w->n_scenes, cudaMemcpyHostToDevice, s));
            SF_CUDA(cudaStreamSynchronize(s));   // the host vector is the copy's source
            S->warm_scene_dirty = false;
        }
        PA.wscene = S->warm_scene_dev.p; PA.bscene = w->b_scene.p;
        if (w->P.reduce || n_loose) SF_CUDA(cudaMemsetAsync(S->invperm.p, 0xFF, (size_t)nc * 4, s));   // left out: no slot
        k_prep<<<g_nc, 256, 0, s>>>(PA);
        L++;
    } else {
        prof_mark(w);
        prof_mark(w);
    }
    k_save_pre<<<grid_for(nb, 256), 256, 0, s>>>(nb, blist, w->b_alive.p, w->b_v.p, w->b_w.p, w->b_vpre.p, w->b_wpre.p);
    L++;
    prof_mark(w);
    if (nc && w->P.iterations) {
        SolveArgs A;
        A.iterations = w->P.iterations; A.dev = S->dev.p; A.col_start = S->col_start.p; A.col_list = S->col_list.p;
        A.blk_dom = S->blk_dom.p; A.dom_ncol = S->dom_ncol.p; A.cstride = cstride;
        A.jds_off = S->jds_off.p; A.man_a = S->man_a.p; A.man_b = S->man_b.p; A.man_count = S->man_count.p;
        A.S_n = S->S_n.p; A.S_t1 = S->S_t1.p; A.S_t2 = S->S_t2.p; A.S_ra = S->S_ra.p; A.S_rb = S->S_rb.p; A.S_j = S->S_j.p;
        A.v = w->b_v.p; A.w = w->b_w.p; A.im = w->b_im.p; A.iiw = w->b_iiw.p; A.gb = S->dom_gb.p; A.err = w->err.p;
        A.warm = w->P.warm_start ? 1u : 0u;
        if (one_block) {
            // a small substep's colours are short: one warp's barrier is cheaper than 16 warps'
            k_solve_one_block<<<1, nc <= SMALL_SUBSTEP_CONTACTS / 2 ? 32 : SOLVE_ONE_BLOCK, 0, s>>>(A);
        } else {
            SF_CUDA(cudaMemsetAsync(S->dom_gb.p, 0, (size_t)S->part_D * sizeof(GridBarrier), s));
            void *sargs[] = {&A};
            tune_begin(S, &S->solve_t, sb, sci, s);
            SF_CUDA(cudaLaunchCooperativeKernel((void *)k_solve, dim3(R), dim3(SOLVE_BLOCK), sargs, 0, s));
            tune_end(S, sci, s);
        }
        L++;
        S->solve_launches++;
        S->solve_contact_iters += (uint64_t)ncm * w->P.iterations;
    }
    if (w->P.warm_start) {
        // the table the next substep reads: every solved contact's impulses under its key
        if (nc) {
            StepState::WarmTable &T = S->warm[S->warm_cur ^ 1];
            uint64_t want = 1024;
            while (want < 4ull * nc) want <<= 1;
            if ((uint64_t)T.mask + 1 < want) {
                SF_CUDA(T.claim.alloc(want)); SF_CUDA(T.k1.alloc(want)); SF_CUDA(T.k2.alloc(want)); SF_CUDA(T.val.alloc(want));
                T.mask = (uint32_t)(want - 1);
            }
            SF_CUDA(cudaMemsetAsync(T.claim.p, 0, ((size_t)T.mask + 1) * 4, s));
            k_warm_store<<<g_nc, 256, 0, s>>>(nc, S->invperm.p, S->L_b.p, S->L_bo.p, S->L_ba.p, S->L_bb.p, S->S_t1.p,
                                              S->S_t2.p, S->S_j.p, T.claim.p, T.k1.p, T.k2.p, T.val.p, T.mask, w->err.p);
            L++;
            S->warm_cur ^= 1;
            S->warm_valid = true;
            std::fill(S->warm_scene.begin(), S->warm_scene.end(), 1);
            S->warm_scene_dirty = true;
        } else {
            S->warm_valid = false;
        }
    }
    prof_mark(w);
    // islands over the manifolds of this substep
    k_uf_init<<<grid_for(nb, 256), 256, 0, s>>>(nb, blist, S->parent.p, S->mint.p);
    if (nc) { k_uf_union<<<g_nc, 256, 0, s>>>(S->dev.p + DV_MANIFOLDS, S->man_a.p, S->man_b.p, S->parent.p, w->err.p); L++; }
    k_uf_label<<<grid_for(nb, 256), 256, 0, s>>>(nb, blist, w->b_alive.p, w->b_asleep.p, S->parent.p, S->label.p, S->dev.p,
                                                 w->err.p);
    L += 2;
    prof_mark(w);
    IntArgs I;
    I.nb = nb; I.list = blist; I.h = h; I.pinch_kill = w->P.pinch_kill ? 1 : 0; I.island_mode = w->P.sleep_mode == SF_SLEEP_ISLAND;
    I.alive = w->b_alive.p; I.asleep = w->b_asleep.p; I.pos = w->b_pos.p; I.q = w->b_q.p; I.v = w->b_v.p; I.w = w->b_w.p;
    I.vpre = w->b_vpre.p; I.wpre = w->b_wpre.p; I.rad = w->b_rad.p; I.sleep = w->b_sleep.p; I.maxr = w->b_maxr.p;
    I.nc = w->b_nc.p; I.count = w->b_count.p; I.first = w->b_first.p; I.kmat = w->k_mat.p;
    I.phase = 0;
    if (w->P.damage && nc) {
        // impact_damage runs between the pinch clamps and integration (src/lib.rs:1780-1782)
        I.phase = 1;
        k_integrate<<<grid_for(nb, 128), 128, 0, s>>>(I);
        DamageIn D;
        D.nc = nc; D.L_a = S->L_a.p; D.L_b = S->L_b.p; D.L_bo = S->L_bo.p; D.L_ba = S->L_ba.p; D.L_bb = S->L_bb.p;
        D.invperm = S->invperm.p; D.L_p = S->L_p.p; D.S_j = S->S_j.p; D.S_rb = S->S_rb.p; D.wk = &S->wk;
        SF_CUDA(damage_substep(w, D, s));
        I.phase = 2;
        L++;
    }
    k_integrate<<<grid_for(nb, 128), 128, 0, s>>>(I);
    if (I.island_mode) {
        k_island_min<<<grid_for(nb, 256), 256, 0, s>>>(nb, blist, w->b_alive.p, S->label.p, w->b_sleep.p, S->mint.p);
        k_island_sleep<<<grid_for(nb, 256), 256, 0, s>>>(nb, blist, w->b_alive.p, w->b_asleep.p, S->label.p, w->b_sleep.p,
                                                         S->mint.p, w->b_v.p, w->b_w.p);
    }
    k_wake<<<grid_for(nb, 256), 256, 0, s>>>(nb, blist, w->b_wake.p, w->b_alive.p, w->b_asleep.p, w->b_sleep.p);
    k_kill_bricks<<<grid_for(nd, 256), 256, 0, s>>>(nd, klist, w->k_body.p, w->b_alive.p, w->k_mat.p);
    L += I.island_mode ? 5 : 3;
    prof_mark(w);
    SF_CUDA(cudaGetLastError());
    S->have_contacts = true;
    return SF_OK;
}

// after a step: which active scenes still have an awake body (read back with the step's counters)
static sf_status queue_live_readback(sf_world *w) {
    StepState *S = w->step;
    cudaStream_t s = w->stream;
    if (S->act.empty()) return SF_OK;
    SF_CUDA(cudaMemsetAsync(S->live_dev.p, 0, w->n_scenes, s));
    if (S->nb_act) {
        k_scene_live<<<grid_for(S->nb_act, 256), 256, 0, s>>>(S->nb_act, S->act_body.p, w->b_alive.p, w->b_asleep.p,
                                                             w->b_scene.p, S->live_dev.p);
        w->launches++;
    }
    SF_CUDA(cudaMemcpyAsync(S->h_live_pin, S->live_dev.p, w->n_scenes, cudaMemcpyDeviceToHost, s));
    return SF_OK;
}
static void apply_live_readback(sf_world *w) {
    StepState *S = w->step;
    for (uint32_t q : S->act) S->live[q] = S->h_live_pin[q];
}

static sf_status step_impl(sf_world *w, float dt, uint32_t nsteps, const uint8_t *mask) {
    if (!w) return SF_ERR_ARG;
    if (!(dt == dt)) { set_error("dt is NaN"); return SF_ERR_ARG; }
    StepState *S = w->step;
    cudaStream_t s = w->stream;
    dt = clampf(dt, 0.0f, 1.0f / 30.0f);
    const uint32_t ns = w->P.substeps;
    const float h = ns == 2 ? dt * 0.5f : dt / (float)ns;
    SF_CUDA(cudaMemsetAsync(w->err.p, 0, sizeof(uint32_t), s));
    SF_CUDA(cudaEventRecord(w->ev0, s));
    for (uint32_t k = 0; k < nsteps; k++) {
        w->frame++;
        sf_status r = set_active(w, mask);
        if (r != SF_OK) return r;
        for (uint32_t q = 0; q < ns; q++) {
            r = substep(w, h);
            if (r != SF_OK) return r;
        }
        r = queue_live_readback(w);
        if (r != SF_OK) return r;
        if (k + 1 < nsteps) {
            SF_CUDA(cudaStreamSynchronize(s));
            apply_live_readback(w);
            tune_resolve(S);
        }
    }
    SF_CUDA(cudaMemsetAsync(S->dev.p + DV_ALIVE, 0, 2 * sizeof(uint32_t), s));
    if (w->nb) k_count_bodies<<<grid_for(w->nb, 256), 256, 0, s>>>(w->nb, w->b_alive.p, w->b_asleep.p, S->dev.p);
    SF_CUDA(cudaEventRecord(w->ev1, s));
    SF_CUDA(cudaMemcpyAsync(S->h_dev, S->dev.p, DV_N * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    sf_status r = read_error_word(w);   // synchronises the stream
    if (nsteps) apply_live_readback(w);
    tune_resolve(S);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, w->ev0, w->ev1);
    sf_stats &st = w->stats;
    // the next step hashes sparsely once at most half the active scenes' bodies are awake (below that the smaller
    // sort and the contact pass over awake bricks only pay for the extra passes and the count read-back; measured on
    // the 256-scene mix)
    S->use_sparse = nsteps && (uint64_t)S->h_dev[DV_AWAKE] * 2 <= (uint64_t)S->nb_act;
    st.contacts = S->h_dev[DV_CONTACTS];
    st.manifolds = S->h_dev[DV_MANIFOLDS];
    st.colors = S->h_dev[DV_COLORS];
    st.color_rounds = S->h_dev[DV_ROUNDS];
    st.islands = S->h_dev[DV_ISLANDS];
    st.alive = S->h_dev[DV_ALIVE];
    st.awake = S->h_dev[DV_AWAKE];
    st.contact_capacity = S->capacity;
    st.ms_last_step = ms;
    st.launches = w->launches + S->wk.launches + sor_launches(w->sor);
    st.graph_launches = sor_graph_launches(w->sor);
    if (S->profile) {
        // each substep recorded SF_PHASES + 1 events
        const size_t per = SF_PHASES + 1;
        for (size_t base = 0; base + per <= S->ev_used; base += per) {
            for (int p = 0; p < SF_PHASES; p++) {
                float e = 0.0f;
                if (cudaEventElapsedTime(&e, S->ev_pool[base + p], S->ev_pool[base + p + 1]) == cudaSuccess) S->ph_ms[p] += e;
            }
            S->ph_substeps++;
        }
        S->ev_used = 0;
        for (size_t k = 0; k + 1 < S->gen_used; k += 2) {
            float e = 0.0f;
            if (cudaEventElapsedTime(&e, S->gen_ev[k], S->gen_ev[k + 1]) == cudaSuccess) S->gen_ms += e;
        }
        S->gen_used = 0;
    }
    return r;
}

}  // namespace sf

using namespace sf;

extern "C" {

sf_status sf_world_step(sf_world *w, float dt, uint32_t nsteps) { return step_impl(w, dt, nsteps, nullptr); }

sf_status sf_read_tuning(sf_world *w, uint32_t which, int32_t *blocks_per_sm, uint32_t n) {
    if (!w || !blocks_per_sm) { set_error("null argument"); return SF_ERR_ARG; }
    // the colouring runs on the solve's blocks, so both read the solve's tuner
    const Tuner *t = (which == SF_TUNE_SOLVE || which == SF_TUNE_COLOR) ? &w->step->solve_t : sor_tuner(w->sor);
    if (!t) { set_error("no such tuner"); return SF_ERR_ARG; }
    for (uint32_t b = 0; b < n; b++) blocks_per_sm[b] = b < (uint32_t)Tuner::NB ? t->settled((int)b) : -1;
    return SF_OK;
}

sf_status sf_world_step_scenes(sf_world *w, float dt, uint32_t nsteps, const uint8_t *scene_mask) {
    if (!w || !scene_mask) { set_error("null argument"); return SF_ERR_ARG; }
    return step_impl(w, dt, nsteps, scene_mask);
}

sf_status sf_set_profiling(sf_world *w, int32_t on) {
    if (!w) return SF_ERR_ARG;
    w->step->profile = on != 0;
    w->step->ev_used = 0;
    return SF_OK;
}

sf_status sf_read_profile(sf_world *w, sf_profile *out) {
    if (!w || !out) return SF_ERR_ARG;
    StepState *S = w->step;
    std::memset(out, 0, sizeof *out);
    for (int p = 0; p < SF_PHASES; p++) out->ms[p] = S->ph_ms[p];
    out->substeps = S->ph_substeps;
    out->solve_launches = S->solve_launches;
    out->solve_contact_iters = S->solve_contact_iters;
    uint64_t sum = 0;
    for (uint32_t n : S->sub_nc) sum += n;
    out->contacts_sum = sum;
    out->launches = w->launches + S->wk.launches + sor_launches(w->sor);
    out->gen_ms = S->gen_ms;
    out->gen_bricks = S->gen_bricks;
    return SF_OK;
}

sf_status sf_reset_profile(sf_world *w) {
    if (!w) return SF_ERR_ARG;
    StepState *S = w->step;
    for (int p = 0; p < SF_PHASES; p++) S->ph_ms[p] = 0.0;
    S->ph_substeps = 0; S->solve_launches = 0; S->solve_contact_iters = 0; S->sub_nc.clear(); S->ev_used = 0;
    S->gen_ms = 0.0; S->gen_bricks = 0; S->gen_used = 0;
    w->launches = 0; S->wk.launches = 0; sor_reset_launches(w->sor);
    return SF_OK;
}

sf_status sf_world_set_stream(sf_world *w, void *stream) {
    if (!w) return SF_ERR_ARG;
    SF_CUDA(cudaStreamSynchronize(w->stream));
    w->stream = stream ? (cudaStream_t)stream : w->own_stream;
    return SF_OK;
}

sf_status sf_read_contacts(sf_world *w, uint32_t scene, uint32_t *ids5, float *f7, float *s8, uint64_t cap, uint64_t *n) {
    if (!w || scene >= w->n_scenes) return SF_ERR_ARG;
    StepState *S = w->step;
    if (!S->have_contacts) { set_error("no step has run yet"); return SF_ERR_STATE; }
    const Scene &sc = w->scenes[scene];
    uint32_t nc = (uint32_t)S->last_contacts;
    cudaStream_t s = w->stream;
    // the scene's contacts are the list range of its awake bricks in the last substep (none if it was idle): the
    // awake list is the active list's awake bricks in order, so the scene's bricks map to one run of it
    uint32_t lo = 0, hi = 0;
    const uint32_t kb = S->act_brick_base[scene];
    if (sc.n_bricks && kb != NONE && S->n_awk) {
        uint32_t a0 = kb, a1 = std::min(kb + sc.n_bricks, S->n_awk);
        if (S->last_sparse) {
            a1 = S->n_awk;
            SF_CUDA(cudaMemcpyAsync(&a0, S->awk_pos.p + kb, 4, cudaMemcpyDeviceToHost, s));
            if (kb + sc.n_bricks < S->nd_act) SF_CUDA(cudaMemcpyAsync(&a1, S->awk_pos.p + kb + sc.n_bricks, 4, cudaMemcpyDeviceToHost, s));
            SF_CUDA(cudaStreamSynchronize(s));
        }
        lo = nc; hi = nc;
        if (a0 < S->n_awk) SF_CUDA(cudaMemcpyAsync(&lo, S->coff.p + a0, 4, cudaMemcpyDeviceToHost, s));
        if (a1 < S->n_awk) SF_CUDA(cudaMemcpyAsync(&hi, S->coff.p + a1, 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
    }
    uint64_t cnt = hi - lo;
    if (n) *n = cnt;
    if (!ids5 && !f7 && !s8) return SF_OK;
    if (cap < cnt) { set_error("contact buffer holds %llu, need %llu", (unsigned long long)cap, (unsigned long long)cnt); return SF_ERR_CAPACITY; }
    std::vector<uint32_t> a(cnt), b(cnt), bo(cnt), ba(cnt), bb(cnt), inv(cnt);
    std::vector<float4> p(cnt), nn(cnt);
    if (cnt) {
        SF_CUDA(cudaMemcpyAsync(a.data(), S->L_a.p + lo, cnt * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(b.data(), S->L_b.p + lo, cnt * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(bo.data(), S->L_bo.p + lo, cnt * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(ba.data(), S->L_ba.p + lo, cnt * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(bb.data(), S->L_bb.p + lo, cnt * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(p.data(), S->L_p.p + lo, cnt * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(nn.data(), S->L_n.p + lo, cnt * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(inv.data(), S->invperm.p + lo, cnt * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<float4> sn, st1, st2, sra, srb, sj;
    // contacts the reduction left out have no slot (NONE) and read as zeros
    bool any_slot = false;
    uint32_t mlo = NONE, mhi = 0;
    for (uint32_t x : inv) if (x != NONE) { any_slot = true; mlo = std::min(mlo, x); mhi = std::max(mhi, x + 1); }
    if (s8 && cnt && any_slot) {
        size_t m = mhi - mlo;
        sn.resize(m); st1.resize(m); st2.resize(m); sra.resize(m); srb.resize(m); sj.resize(m);
        SF_CUDA(cudaMemcpyAsync(sn.data(), S->S_n.p + mlo, m * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(st1.data(), S->S_t1.p + mlo, m * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(st2.data(), S->S_t2.p + mlo, m * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(sra.data(), S->S_ra.p + mlo, m * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(srb.data(), S->S_rb.p + mlo, m * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(sj.data(), S->S_j.p + mlo, m * 16, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
        for (auto &x : inv) if (x != NONE) x -= mlo;
    }
    auto loc_body = [&](uint32_t g) { return g == STATIC ? STATIC : g - sc.body_off; };
    auto loc_dyn = [&](uint32_t g) { return sc.n_static + (g - sc.brick_off); };
    for (uint64_t k = 0; k < cnt; k++) {
        if (ids5) {
            uint32_t *o = ids5 + k * 5;
            o[0] = loc_body(a[k]); o[1] = loc_body(b[k]); o[2] = loc_body(bo[k]); o[3] = loc_dyn(ba[k]);
            if (bb[k] == NONE) o[4] = NONE;
            else if (bo[k] == STATIC) o[4] = bb[k] - sc.static_off;
            else o[4] = loc_dyn(bb[k]);
        }
        if (f7) {
            float *g = f7 + k * 7;
            g[0] = p[k].x; g[1] = p[k].y; g[2] = p[k].z; g[3] = nn[k].x; g[4] = nn[k].y; g[5] = nn[k].z; g[6] = nn[k].w;
        }
        if (s8) {
            uint32_t t = inv[k];
            float *x = s8 + k * 8;
            if (t == NONE || !any_slot) { for (int q = 0; q < 8; q++) x[q] = 0.0f; continue; }
            x[0] = sj[t].x; x[1] = sj[t].y; x[2] = sj[t].z; x[3] = sn[t].w; x[4] = st1[t].w; x[5] = st2[t].w; x[6] = sra[t].w; x[7] = srb[t].w;
        }
    }
    return SF_OK;
}

sf_status sf_read_manifolds(sf_world *w, uint32_t scene, uint32_t *out4, uint64_t cap, uint64_t *n) {
    if (!w || scene >= w->n_scenes) return SF_ERR_ARG;
    StepState *S = w->step;
    if (!S->have_contacts) { set_error("no step has run yet"); return SF_ERR_STATE; }
    const Scene &sc = w->scenes[scene];
    cudaStream_t s = w->stream;
    uint32_t nm = 0;
    SF_CUDA(cudaMemcpyAsync(&nm, S->dev.p + DV_MANIFOLDS, 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> a(nm), b(nm), c(nm), k(nm);
    if (nm) {
        SF_CUDA(cudaMemcpyAsync(a.data(), S->man_a.p, nm * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(b.data(), S->man_b.p, nm * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(c.data(), S->man_color.p, nm * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaMemcpyAsync(k.data(), S->man_count.p, nm * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
    }
    uint64_t cnt = 0;
    for (uint32_t m = 0; m < nm; m++) {
        if (a[m] < sc.body_off || a[m] >= sc.body_off + sc.n_bodies) continue;
        if (out4 && cnt < cap) {
            uint32_t *o = out4 + cnt * 4;
            o[0] = a[m] - sc.body_off; o[1] = b[m] == STATIC ? STATIC : b[m] - sc.body_off; o[2] = c[m]; o[3] = k[m];
        }
        cnt++;
    }
    if (n) *n = cnt;
    if (out4 && cap < cnt) return SF_ERR_CAPACITY;
    return SF_OK;
}

sf_status sf_read_islands(sf_world *w, uint32_t *label) {
    if (!w || !label) return SF_ERR_ARG;
    SF_CUDA(cudaMemcpyAsync(label, w->step->label.p, (size_t)w->nb * 4, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}

}  // extern "C"

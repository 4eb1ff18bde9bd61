// Connectivity of the load-path structures, and detachment of unsupported pieces into rigid bodies.
//
//   conn_struct   src/lib.rs:1085-1134   one structure: the bricks reached from its grounded footings through intact
//                                        bonds stay static; every other bonded piece becomes one compound body
//   connectivity  src/lib.rs:1137-1141   the structures flagged since the last call, in structure order
//
// Work split. Labelling is data-parallel over every static brick of the requested structures: one pass links the
// bricks of each intact +x / +y / +z bond in a union-find forest, a second marks the roots of components that hold a
// grounded footing, a third collects the bricks of the other components. Only those bricks (the pieces about to
// fall, a small fraction of a standing structure) are read back. The host walks them in the reference's order —
// seeds in brick order, neighbours in direction order, breadth first — because a body's brick order is the order
// its mass, centre and inertia sums round in (setup_body sums in list order), and gives each piece the scene's next
// spare body and bricks. The GPU then removes the static bricks, sets the bodies up (k_setup_bodies, the same kernel
// as world creation) and wakes the sleeping bodies near each new one (wake_near).
//
// Left out, as in the rest of this path: the salvage tally, impact events, crowd panic, render-cache marks and zone
// touches of conn_struct, and the blast impulse (apply_blast_to_body is a no-op without an active blast).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "sf_internal.cuh"

namespace sf {

// per read-back brick: 6 neighbours, 4 bonds and 4 capacities (as bits), material
constexpr int STAGE_WORDS = 15;

struct ConnState {
    DBuf<uint32_t> parent;       // per static brick: union-find parent, NONE = not in a requested structure
    DBuf<uint8_t> ground;        // per static brick, meaningful at component roots: the component is grounded
    DBuf<uint32_t> list;         // static bricks of ungrounded components (unordered)
    DBuf<uint32_t> count;        // [0] list length, [1] the error word at labelling
    DBuf<uint32_t> stage;        // STAGE_WORDS per listed brick
    DBuf<uint8_t> sel;           // per structure: requested in this call
    DBuf<uint32_t> removed;      // static bricks this call turned into body bricks
    DBuf<float> pose;            // 13 per new body: at the origin, identity rotation, at rest
    DBuf<uint32_t> newb;         // per scene: first and end of the bodies this call created
    DBuf<uint32_t> tally;        // per structure: bricks left, top cell + 1
    DBuf<uint32_t> bslot, brec;  // new body bricks and their neighbours, bonds and capacities (14 words each)
    std::vector<int32_t> where;  // per static brick: its index in the host copy of the list, -1 = not listed
};

// ---------------------------------------------------------------- labelling
__global__ void k_cc_init(uint32_t ns, const int32_t *sid, const uint8_t *mat, const uint8_t *sel, uint32_t *parent,
                          uint8_t *ground) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const int32_t s = sid[i];
    parent[i] = (mat[i] != 0 && s >= 0 && sel[s]) ? i : NONE;
    ground[i] = 0;
}

// the walked structures are no longer pending (connectivity clears st_conn before conn_struct, src/lib.rs:1140)
__global__ void k_cc_unflag(uint32_t nst, const uint8_t *sel, uint8_t *conn) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nst && sel[s]) conn[s] = 0;
}

// linked (src/lib.rs:378-383) between two static bricks: neighbours, both present, the bond between them > 0. A bond
// lives on the brick on the negative side, so walking each brick's +x, +y and +z links visits every link once. Bonds
// form only between bricks of one structure (finalize_brick), so a requested brick links only requested bricks.
__global__ void k_cc_link(uint32_t ns, const uint32_t *nb6, const float *bond, uint32_t *parent, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns || __ldcg(&parent[i]) == NONE) return;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const uint32_t j = nb6[(size_t)i * 6 + 2 * a];
        if (j == NONE || __ldcg(&parent[j]) == NONE) continue;
        if (bond[(size_t)i * 4 + a] > 0.0f) uf_union(parent, i, j, err);
    }
}

// the seeds of the grounded walk (src/lib.rs:1089-1091): bricks of the structure proper (in_struct, src/lib.rs:1027:
// material below SLUG) on the bottom row whose foundation bond is intact
__global__ void k_cc_ground(uint32_t ns, const uint8_t *mat, const uint32_t *cell, const float *bond, uint32_t *parent,
                            uint8_t *ground, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns || __ldcg(&parent[i]) == NONE || mat[i] >= SLUG) return;
    int x, y, z;
    unpack_cell(cell[i], x, y, z);
    if (y == 0 && bond[(size_t)i * 4 + 3] > 0.0f) ground[uf_find(parent, i, err)] = 1;
}

// every labelled brick whose component holds no grounded footing; one atomic per warp
__global__ void k_cc_collect(uint32_t ns, uint32_t *parent, const uint8_t *ground, uint32_t *list, uint32_t *count,
                             uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool out = false;
    if (i < ns && __ldcg(&parent[i]) != NONE) out = !ground[uf_find(parent, i, err)];
    const unsigned m = __ballot_sync(0xffffffffu, out);
    if (!m) return;
    const unsigned lane = threadIdx.x & 31u, lead = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == lead) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, lead);
    if (out) list[base + __popc(m & ((1u << lane) - 1u))] = i;
}

__global__ void k_cc_gather(uint32_t n, const uint32_t *list, const uint32_t *nb6, const float *bond, const float *bmax,
                            const uint8_t *mat, uint32_t *stage) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = list[k];
    uint32_t *o = stage + (size_t)k * STAGE_WORDS;
#pragma unroll
    for (int d = 0; d < 6; d++) o[d] = nb6[(size_t)i * 6 + d];
#pragma unroll
    for (int a = 0; a < 4; a++) {
        o[6 + a] = __float_as_uint(bond[(size_t)i * 4 + a]);
        o[10 + a] = __float_as_uint(bmax[(size_t)i * 4 + a]);
    }
    o[14] = mat[i];
}

// a detached piece's bricks keep their bonds (src/lib.rs:1118 leaves them): the new body bricks get the static
// bricks' bonds and capacities, and their neighbours renumbered to the piece's new body bricks
__global__ void k_cc_bonds(uint32_t n, const uint32_t *slot, const uint32_t *rec, uint32_t *k_nb6, float *k_bond,
                           float *k_bmax) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t k = slot[t];
    const uint32_t *r = rec + (size_t)t * 14;
#pragma unroll
    for (int d = 0; d < 6; d++) k_nb6[(size_t)k * 6 + d] = r[d];
#pragma unroll
    for (int a = 0; a < 4; a++) {
        k_bond[(size_t)k * 4 + a] = __uint_as_float(r[6 + a]);
        k_bmax[(size_t)k * 4 + a] = __uint_as_float(r[10 + a]);
    }
}

// ---------------------------------------------------------------- detachment
// the static side of conn_struct's per-brick reset (src/lib.rs:1118): the brick leaves the static set (material 0,
// its grid cell empty) with potential and load 0; its bonds stay with it
__global__ void k_cc_remove(uint32_t n, const uint32_t *removed, const uint32_t *scene, const uint32_t *cell,
                            const uint32_t *ctab, uint32_t *cpool, uint8_t *mat, float *phi, double *phi64, float *ext) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = removed[k];
    int x, y, z;
    unpack_cell(cell[i], x, y, z);
    const uint32_t t = ctab[(size_t)scene[i] * NCT + chunk_slot(x, y, z)];
    if (t) {
        uint32_t &g = cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
        if (g == i + 1) g = 0;
    }
    mat[i] = 0;
    phi[i] = 0.0f;
    phi64[i] = 0.0;
    ext[i] = 0.0f;
}

// wake_near (src/lib.rs:925-929) of every body this call created, in one pass: a sleeping body wakes when its centre
// is closer to a new body's centre than (the new body's radius + 1.5) + its own radius. The new bodies are awake and
// the sleeping ones do not move, so the order of the reference's calls cannot change the outcome.
__global__ void k_cc_wake(uint32_t nb, const uint32_t *b_scene, const uint32_t *newb, const uint8_t *alive,
                          uint8_t *asleep, float *sleep, const float4 *pos, const float *rad) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !alive[b] || !asleep[b]) return;
    const uint32_t s = b_scene[b];
    const uint32_t lo = newb[2 * s], hi = newb[2 * s + 1];
    const float4 pb = pos[b];
    const float rb = rad[b];
    for (uint32_t k = lo; k < hi; k++) {
        const float4 pk = pos[k];
        const float l = len(sub(v3(pb.x, pb.y, pb.z), v3(pk.x, pk.y, pk.z)));
        if (l < (rad[k] + 1.5f) + rb) {
            asleep[b] = 0;
            sleep[b] = 0.0f;
            return;
        }
    }
}

// st_now / st_top (src/lib.rs:1126-1128): per requested structure, the bricks it still has and its top row + 1
__global__ void k_cc_tally(uint32_t ns, const int32_t *sid, const uint8_t *mat, const uint32_t *cell, const uint8_t *sel,
                           uint32_t *tally) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const int32_t s = sid[i];
    const uint8_t m = mat[i];
    if (m == 0 || m >= SLUG || s < 0 || !sel[s]) return;
    int x, y, z;
    unpack_cell(cell[i], x, y, z);
    atomicAdd(&tally[2 * s], 1u);
    atomicMax(&tally[2 * s + 1], (uint32_t)(y + 1));
}

void conn_destroy(sf_world *w) {
    delete w->conn;
    w->conn = nullptr;
}

static uint32_t scene_of_static(const sf_world *w, uint32_t i) {
    uint32_t lo = 0, hi = w->n_scenes;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (w->scenes[mid].static_off <= i) lo = mid; else hi = mid;
    }
    return lo;
}

static sf_status conn_impl(sf_world *w, const std::vector<int32_t> &ids, uint32_t *now, int32_t *top,
                           sf_connect_report *report) {
    const auto t0 = std::chrono::steady_clock::now();
    sf_connect_report rep{};
    const uint32_t ns = w->ns, nst = w->n_struct;
    cudaStream_t st = w->stream;
    if (ids.empty() || ns == 0) {
        if (report) *report = rep;
        return SF_OK;
    }
    if (!w->conn) w->conn = new ConnState();
    ConnState &C = *w->conn;
    SF_CUDA(C.parent.alloc(ns));
    SF_CUDA(C.ground.alloc(ns));
    SF_CUDA(C.list.alloc(ns));
    SF_CUDA(C.count.alloc(4));
    SF_CUDA(C.sel.alloc(nst));
    SF_CUDA(C.tally.alloc((size_t)nst * 2));
    SF_CUDA(C.newb.alloc((size_t)w->n_scenes * 2));
    if (C.where.size() != ns) C.where.assign(ns, -1);

    std::vector<uint8_t> sel(nst, 0);
    for (int32_t q : ids) sel[q] = 1;
    SF_CUDA(cudaMemcpyAsync(C.sel.p, sel.data(), nst, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemsetAsync(C.count.p, 0, 4 * sizeof(uint32_t), st));
    const unsigned g = grid_for(ns, 256);
    k_cc_unflag<<<grid_for(nst, 256), 256, 0, st>>>(nst, C.sel.p, w->st_conn.p);
    k_cc_init<<<g, 256, 0, st>>>(ns, w->s_sid.p, w->s_mat.p, C.sel.p, C.parent.p, C.ground.p);
    k_cc_link<<<g, 256, 0, st>>>(ns, w->s_nb6.p, w->s_bond.p, C.parent.p, w->err.p);
    k_cc_ground<<<g, 256, 0, st>>>(ns, w->s_mat.p, w->s_cell.p, w->s_bond.p, C.parent.p, C.ground.p, w->err.p);
    k_cc_collect<<<g, 256, 0, st>>>(ns, C.parent.p, C.ground.p, C.list.p, C.count.p, w->err.p);
    SF_CUDA(cudaMemcpyAsync(C.count.p + 1, w->err.p, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    w->launches += 5;
    SF_CUDA(cudaGetLastError());
    uint32_t hc[2] = {0, 0};
    SF_CUDA(cudaMemcpyAsync(hc, C.count.p, sizeof hc, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    if (hc[1] & ERR_ISLANDS) return read_error_word(w);
    const uint32_t n = hc[0];
    rep.structures = (uint32_t)ids.size();
    rep.listed = n;

    // ---- the listed bricks on the host, in brick order
    std::vector<uint32_t> list(n), stage((size_t)n * STAGE_WORDS);
    if (n) {
        SF_CUDA(C.stage.grow((size_t)n * STAGE_WORDS));
        k_cc_gather<<<grid_for(n, 256), 256, 0, st>>>(n, C.list.p, w->s_nb6.p, w->s_bond.p, w->s_bmax.p, w->s_mat.p,
                                                      C.stage.p);
        w->launches++;
        SF_CUDA(cudaGetLastError());
        SF_CUDA(cudaMemcpyAsync(list.data(), C.list.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaMemcpyAsync(stage.data(), C.stage.p, (size_t)n * STAGE_WORDS * 4, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<uint32_t> order(n);
    for (uint32_t k = 0; k < n; k++) order[k] = k;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return list[a] < list[b]; });
    for (uint32_t k = 0; k < n; k++) C.where[list[k]] = (int32_t)k;
    auto rec = [&](uint32_t i) { return &stage[(size_t)C.where[i] * STAGE_WORDS]; };
    auto bond_of = [&](const uint32_t *r, int a) { float f; std::memcpy(&f, &r[6 + a], 4); return f; };

    // ---- conn_struct's walk of the pieces (src/lib.rs:1099-1117), structure by structure in the requested order
    struct Piece { uint32_t scene, body, first, count; };
    std::vector<Piece> pieces;
    std::vector<uint32_t> removed;
    std::vector<std::vector<uint32_t>> sc_first(w->n_scenes), sc_count(w->n_scenes);
    std::vector<std::vector<int32_t>> sc_xyz(w->n_scenes);
    std::vector<std::vector<uint8_t>> sc_mat(w->n_scenes);
    std::vector<uint32_t> used_b0(w->n_scenes), used_k0(w->n_scenes);
    for (uint32_t q = 0; q < w->n_scenes; q++) { used_b0[q] = w->scenes[q].bodies_used; used_k0[q] = w->scenes[q].bricks_used; }
    std::vector<uint8_t> stamp(n, 0);
    std::vector<uint32_t> piece;
    std::vector<uint32_t> newslot(n, NONE), bslot, brec;   // body-brick slot of each listed brick; bond records
    for (int32_t s : ids) {
        bool retry = false;
        for (uint32_t k = 0; k < n; k++) {
            const uint32_t seed = list[order[k]];
            const uint32_t *rs = rec(seed);
            if (stamp[C.where[seed]] || w->h_sid[seed] != s || rs[14] >= SLUG) continue;
            piece.clear();
            stamp[C.where[seed]] = 1;
            piece.push_back(seed);
            for (size_t h = 0; h < piece.size(); h++) {
                const uint32_t i = piece[h];
                const uint32_t *ri = rec(i);
                for (int d = 0; d < 6; d++) {
                    const uint32_t j = ri[d];
                    // a neighbour outside the list is grounded or not requested: never linked to a listed brick
                    if (j == NONE || C.where[j] < 0 || stamp[C.where[j]]) continue;
                    const float hp = (d & 1) == 0 ? bond_of(ri, d >> 1) : bond_of(rec(j), d >> 1);
                    if (!(hp > 0.0f)) continue;
                    stamp[C.where[j]] = 1;
                    piece.push_back(j);
                }
            }
            // alloc_body (src/lib.rs:755-766): here the scene's next spare body and bricks; without room the piece
            // stays static and the structure pending, as conn_struct's retry when ensure_bodies fails
            const uint32_t q = scene_of_static(w, seed);
            Scene &sc = w->scenes[q];
            const uint32_t cnt = (uint32_t)piece.size();
            if (sc.bodies_used + 1 > sc.n_bodies || sc.bricks_used + cnt > sc.n_bricks) { retry = true; continue; }
            const uint32_t body = sc.body_off + sc.bodies_used, first = sc.brick_off + sc.bricks_used;
            sc.bodies_used += 1;
            sc.bricks_used += cnt;
            pieces.push_back(Piece{q, body, first, cnt});
            sc_first[q].push_back(first);
            sc_count[q].push_back(cnt);
            for (uint32_t t = 0; t < cnt; t++) newslot[C.where[piece[t]]] = first + t;
            for (uint32_t t = 0; t < cnt; t++) {
                const uint32_t *ri = rec(piece[t]);
                bslot.push_back(first + t);
                for (int d = 0; d < 6; d++) {
                    const uint32_t j = ri[d];
                    const bool same = j != NONE && C.where[j] >= 0 && newslot[C.where[j]] != NONE &&
                                      newslot[C.where[j]] >= first && newslot[C.where[j]] < first + cnt;
                    brec.push_back(same ? newslot[C.where[j]] : NONE);
                }
                for (int a = 0; a < 8; a++) brec.push_back(ri[6 + a]);
            }
            for (uint32_t i : piece) {
                int x, y, z;
                unpack_cell(w->h_s_cell[i], x, y, z);
                sc_xyz[q].push_back(x); sc_xyz[q].push_back(y); sc_xyz[q].push_back(z);
                sc_mat[q].push_back((uint8_t)rec(i)[14]);
                removed.push_back(i);
            }
            rep.detached += cnt;
        }
        if (retry) { w->h_conn_retry[s] = 1; rep.retry++; }
        else w->h_conn_retry[s] = 0;
    }
    for (uint32_t k = 0; k < n; k++) C.where[list[k]] = -1;
    rep.pieces = (uint32_t)pieces.size();

    // ---- the GPU side of the new bodies
    std::vector<float> pose((size_t)pieces.size() * 13, 0.0f);
    for (size_t p = 0; p < pieces.size(); p++) pose[p * 13 + 6] = 1.0f;
    std::vector<uint32_t> newb((size_t)w->n_scenes * 2, 0);
    if (!pieces.empty()) {
        SF_CUDA(C.removed.grow(removed.size()));
        SF_CUDA(C.pose.grow(pose.size()));
        SF_CUDA(cudaMemcpyAsync(C.removed.p, removed.data(), removed.size() * 4, cudaMemcpyHostToDevice, st));
        SF_CUDA(cudaMemcpyAsync(C.pose.p, pose.data(), pose.size() * 4, cudaMemcpyHostToDevice, st));
        k_cc_remove<<<grid_for(removed.size(), 256), 256, 0, st>>>((uint32_t)removed.size(), C.removed.p, w->s_scene.p,
                                                                   w->s_cell.p, w->ctab.p, w->cpool.p, w->s_mat.p,
                                                                   w->s_phi.p, w->s_phi64.p, w->s_ext.p);
        w->launches++;
        SF_CUDA(cudaGetLastError());
        size_t pose_at = 0;
        for (uint32_t q = 0; q < w->n_scenes; q++) {
            const Scene &sc = w->scenes[q];
            const uint32_t nbq = sc.bodies_used - used_b0[q], nkq = sc.bricks_used - used_k0[q];
            newb[2 * q] = sc.body_off + used_b0[q];
            newb[2 * q + 1] = sc.body_off + sc.bodies_used;
            if (!nbq) continue;
            const uint32_t b0 = sc.body_off + used_b0[q], k0 = sc.brick_off + used_k0[q];
            SF_CUDA(cudaMemcpyAsync(w->b_first.p + b0, sc_first[q].data(), (size_t)nbq * 4, cudaMemcpyHostToDevice, st));
            SF_CUDA(cudaMemcpyAsync(w->b_count.p + b0, sc_count[q].data(), (size_t)nbq * 4, cudaMemcpyHostToDevice, st));
            SF_CUDA(cudaMemcpyAsync(w->k_xyz.p + (size_t)k0 * 3, sc_xyz[q].data(), (size_t)nkq * 12, cudaMemcpyHostToDevice, st));
            SF_CUDA(cudaMemcpyAsync(w->k_mat.p + k0, sc_mat[q].data(), nkq, cudaMemcpyHostToDevice, st));
            SF_CUDA(setup_bodies(w, b0, nbq, C.pose.p + pose_at * 13));
            step_warm_invalidate(w, q);   // new body bricks take ids
            SF_CUDA(step_reset_labels(w, b0, nbq));
            pose_at += nbq;
        }
        if (w->k_nb6.p) {
            SF_CUDA(C.bslot.grow(bslot.size()));
            SF_CUDA(C.brec.grow(brec.size()));
            SF_CUDA(cudaMemcpyAsync(C.bslot.p, bslot.data(), bslot.size() * 4, cudaMemcpyHostToDevice, st));
            SF_CUDA(cudaMemcpyAsync(C.brec.p, brec.data(), brec.size() * 4, cudaMemcpyHostToDevice, st));
            k_cc_bonds<<<grid_for(bslot.size(), 256), 256, 0, st>>>((uint32_t)bslot.size(), C.bslot.p, C.brec.p,
                                                                   w->k_nb6.p, w->k_bond.p, w->k_bmax.p);
            w->launches++;
            SF_CUDA(cudaGetLastError());
        }
        SF_CUDA(cudaMemcpyAsync(C.newb.p, newb.data(), newb.size() * 4, cudaMemcpyHostToDevice, st));
        k_cc_wake<<<grid_for(w->nb, 256), 256, 0, st>>>(w->nb, w->b_scene.p, C.newb.p, w->b_alive.p, w->b_asleep.p,
                                                        w->b_sleep.p, w->b_pos.p, w->b_rad.p);
        w->launches++;
        SF_CUDA(cudaGetLastError());
        for (uint32_t q = 0; q < w->n_scenes; q++)
            if (newb[2 * q + 1] > newb[2 * q]) step_set_live(w, q, true);
    }
    // ---- st_now / st_top
    if (now || top) {
        std::vector<uint32_t> tl((size_t)nst * 2);
        SF_CUDA(cudaMemsetAsync(C.tally.p, 0, (size_t)nst * 8, st));
        k_cc_tally<<<g, 256, 0, st>>>(ns, w->s_sid.p, w->s_mat.p, w->s_cell.p, C.sel.p, C.tally.p);
        w->launches++;
        SF_CUDA(cudaGetLastError());
        SF_CUDA(cudaMemcpyAsync(tl.data(), C.tally.p, (size_t)nst * 8, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaStreamSynchronize(st));
        for (int32_t s : ids) {
            if (now) now[s] = tl[2 * s];
            if (top) top[s] = (int32_t)tl[2 * s + 1];
        }
    }
    SF_CUDA(cudaStreamSynchronize(st));   // the host vectors above are the copies' sources
    sf_status r = read_error_word(w);
    rep.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (report) *report = rep;
    return r;
}

}  // namespace sf

using namespace sf;

extern "C" {

sf_status sf_structure_connect(sf_world *w, const int32_t *structures, uint32_t n, uint32_t *now, int32_t *top,
                               sf_connect_report *report) {
    if (!w || (n && !structures)) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    std::vector<int32_t> ids(structures, structures + n);
    for (int32_t q : ids)
        if (q < 0 || (uint32_t)q >= w->n_struct) { set_error("structure %d out of range", q); return SF_ERR_ARG; }
    std::vector<uint8_t> seen(w->n_struct, 0);
    for (int32_t q : ids) {
        if (seen[q]) { set_error("structure %d listed twice", q); return SF_ERR_ARG; }
        seen[q] = 1;
    }
    return conn_impl(w, ids, now, top, report);
}

sf_status sf_world_connectivity(sf_world *w, uint32_t *now, int32_t *top, sf_connect_report *report) {
    if (!w) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    const uint32_t nst = w->n_struct;
    std::vector<uint8_t> flag(nst, 0);
    if (nst) {
        SF_CUDA(cudaMemcpyAsync(flag.data(), w->st_conn.p, nst, cudaMemcpyDeviceToHost, w->stream));
        SF_CUDA(cudaMemsetAsync(w->st_conn.p, 0, nst, w->stream));
        SF_CUDA(cudaStreamSynchronize(w->stream));
    }
    std::vector<int32_t> ids;
    for (uint32_t q = 0; q < nst; q++)
        if (flag[q] || w->h_conn_retry[q]) ids.push_back((int32_t)q);
    return conn_impl(w, ids, now, top, report);
}

}  // extern "C"

// Brick removal and the splitting of bodies.
//
//   remove_brick   src/lib.rs:705-718   a brick leaves the world: a static one marks its structure pending a
//                                       connectivity walk, a body brick marks its body for rebuild
//   rebuild_body   src/lib.rs:930-1002  a marked body drops its removed bricks and splits into bonded components:
//                                       the first stays in the body, each other becomes a new body; all are set up
//                                       about the parent's pose (setup_body, src/lib.rs:844-891)
//
// A body's bricks are one contiguous range of body-brick slots. On a rebuild the first component's bricks move to the
// front of the body's range (in list order) and every other component's bricks to the scene's next spare slots; the
// slots left over belong to the sentinel body. Only the marked bodies' bricks are read back: the host walks them in
// the reference's order (components seeded in list order, breadth first, neighbours in direction order), because a
// body's brick order is the order its set-up sums round in, then writes the new ranges and sets the bodies up on the
// GPU with the same kernel as world creation, from the bricks' current local offsets and the parent's cached rotation.
//
// The lone-brick rule (src/lib.rs:980-990: with more than 1,500 bodies awake, a one-brick piece other than steel turns
// to debris with probability min((awake - 1500) / 2000, 0.85)) draws from a hash of (scene, its rebuild count,
// brick) with the reference's h01 mixing (src/lib.rs:341-345) in place of the world's random stream, whose position
// depends on particle effects outside this path; its awake count is the scene's at the rebuild.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "sf_internal.cuh"

namespace sf {

constexpr int SPLIT_WORDS = 26;
constexpr int LITE = 11, L_MAT = 0, L_NB6 = 1, L_BOND = 7;   // the words the host walk reads: 3 .. 13 of a record   // per read-back brick: xyz 3, mat, 6 neighbours, 4 bonds, 4 capacities, local 3,
                                  // the load field's support stamp, f32 potential, load and f64 potential (2)

struct SplitState {
    DBuf<uint32_t> list, count, bsel, brec, slots, words, freed, awake, moves, lite;
    DBuf<uint8_t> keep;                 // per set-up body: the rebuilt body itself, which keeps its load time
    DBuf<float> pose;
    std::vector<uint32_t> scene_rebuilds;
};

// ---------------------------------------------------------------- removal
__global__ void k_remove_static(uint32_t n, const uint32_t *ids, const uint32_t *scene, const uint32_t *cell,
                                const int32_t *sid, const uint32_t *ctab, uint32_t *cpool, uint8_t *mat, uint8_t *conn,
                                uint32_t nst) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = ids[k];
    if (mat[i] == 0) return;
    int x, y, z;
    unpack_cell(cell[i], x, y, z);
    const uint32_t t = ctab[(size_t)scene[i] * NCT + chunk_slot(x, y, z)];
    if (t) {
        uint32_t &g = cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
        if (g == i + 1) g = 0;
    }
    mat[i] = 0;
    const int32_t s = sid[i];
    if (s >= 0 && (uint32_t)s < nst) conn[s] = 1;
}
__global__ void k_remove_body_bricks(uint32_t n, const uint32_t *ids, const uint32_t *kbody, const uint8_t *alive,
                                     uint8_t *kmat, uint8_t *dirty) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = ids[k];
    const uint32_t b = kbody[i];
    if (kmat[i] == 0 || !alive[b]) return;
    kmat[i] = 0;
    dirty[b] = 1;
}

// ---------------------------------------------------------------- rebuild
__global__ void k_dirty_collect(uint32_t nb, const uint8_t *dirty, const uint8_t *alive, uint32_t *list, uint32_t *count) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = b < nb && dirty[b] && alive[b];
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (!m) return;
    const unsigned lane = threadIdx.x & 31u, lead = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == lead) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, lead);
    if (on) list[base + __popc(m & ((1u << lane) - 1u))] = b;
}

// per listed body: first, count, scene, then its pose (position, quaternion, velocity, spin) and cached rotation
__global__ void k_body_snapshot(uint32_t n, const uint32_t *list, const uint32_t *first, const uint32_t *count,
                                const uint32_t *scene, const float4 *pos, const float4 *q, const float4 *v,
                                const float4 *w, const float *rot, uint32_t *out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t b = list[k];
    uint32_t *o = out + (size_t)k * 25;
    o[0] = first[b]; o[1] = count[b]; o[2] = scene[b];
    const float4 p = pos[b], qq = q[b], vv = v[b], ww = w[b];
    const float f[13] = {p.x, p.y, p.z, qq.x, qq.y, qq.z, qq.w, vv.x, vv.y, vv.z, ww.x, ww.y, ww.z};
    for (int j = 0; j < 13; j++) o[3 + j] = __float_as_uint(f[j]);
    for (int j = 0; j < 9; j++) o[16 + j] = __float_as_uint(rot[(size_t)b * 9 + j]);
}

// the bricks of the listed slots, SPLIT_WORDS each
__global__ void k_brick_snapshot(uint32_t n, const uint32_t *slots, const int32_t *xyz, const uint8_t *kmat,
                                 const uint32_t *nb6, const float *bond, const float *bmax, const float4 *local,
                                 const uint32_t *sup, const float *phi, const float *ext, const double *phi64,
                                 uint32_t *out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = slots[k];
    uint32_t *o = out + (size_t)k * SPLIT_WORDS;
    o[0] = (uint32_t)xyz[3 * i]; o[1] = (uint32_t)xyz[3 * i + 1]; o[2] = (uint32_t)xyz[3 * i + 2];
    o[3] = kmat[i];
    for (int d = 0; d < 6; d++) o[4 + d] = nb6[(size_t)i * 6 + d];
    for (int a = 0; a < 4; a++) {
        o[10 + a] = __float_as_uint(bond[(size_t)i * 4 + a]);
        o[14 + a] = __float_as_uint(bmax[(size_t)i * 4 + a]);
    }
    const float4 l = local[i];
    o[18] = __float_as_uint(l.x); o[19] = __float_as_uint(l.y); o[20] = __float_as_uint(l.z);
    o[21] = sup[i]; o[22] = __float_as_uint(phi[i]); o[23] = __float_as_uint(ext[i]);
    const unsigned long long p = (unsigned long long)__double_as_longlong(phi64[i]);
    o[24] = (uint32_t)p; o[25] = (uint32_t)(p >> 32);
}

// the walk's words of each snapshot record, packed
__global__ void k_brick_lite(uint32_t n, const uint32_t *rec, uint32_t *lite) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * LITE) return;
    const uint32_t e = t / LITE, w = t - e * LITE;
    lite[t] = rec[(size_t)e * SPLIT_WORDS + 3 + w];
}

// the kept bricks of the rebuilt bodies to their new slots, from the snapshot: fields as they were, neighbours
// renumbered (a neighbour in the same piece to its new slot, any other to none)
struct BrickMove {
    const uint32_t *dst, *src, *body;   // per moved brick
    const uint32_t *nmap, *ncomp;       // per snapshot entry
    const uint32_t *brange;             // per rebuilt body: first slot, bricks, snapshot offset
    const uint32_t *rec;                // the snapshot, SPLIT_WORDS per entry
};
__global__ void k_brick_move(uint32_t n, BrickMove M, int32_t *xyz, uint8_t *kmat, uint32_t *nb6, float *bond,
                             float *bmax, float4 *local, uint32_t *sup, float *phi, float *ext, double *phi64) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = M.dst[k], e = M.src[k], bk = M.body[k];
    const uint32_t first = M.brange[3 * bk], cnt = M.brange[3 * bk + 1], at = M.brange[3 * bk + 2];
    const uint32_t *r = M.rec + (size_t)e * SPLIT_WORDS;
    const uint32_t c = M.ncomp[e];
    xyz[3 * i] = (int32_t)r[0]; xyz[3 * i + 1] = (int32_t)r[1]; xyz[3 * i + 2] = (int32_t)r[2];
    kmat[i] = (uint8_t)r[3];
    for (int d = 0; d < 6; d++) {
        const uint32_t js = r[4 + d];
        uint32_t ns = NONE;
        if (js != NONE && js >= first && js < first + cnt) {
            const uint32_t e2 = at + (js - first);
            if (M.ncomp[e2] == c && M.nmap[e2] != NONE) ns = M.nmap[e2];
        }
        nb6[(size_t)i * 6 + d] = ns;
    }
    for (int a = 0; a < 4; a++) {
        bond[(size_t)i * 4 + a] = __uint_as_float(r[10 + a]);
        bmax[(size_t)i * 4 + a] = __uint_as_float(r[14 + a]);
    }
    local[i] = make_float4(__uint_as_float(r[18]), __uint_as_float(r[19]), __uint_as_float(r[20]), 0.0f);
    sup[i] = r[21]; phi[i] = __uint_as_float(r[22]); ext[i] = __uint_as_float(r[23]);
    phi64[i] = __longlong_as_double((long long)(((unsigned long long)r[25] << 32) | r[24]));
}

// slots no body owns any more: material 0, owned by the sentinel, no neighbours
__global__ void k_brick_free(uint32_t n, const uint32_t *slots, uint32_t sentinel, uint8_t *kmat, uint32_t *kbody,
                             uint32_t *nb6) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = slots[k];
    kmat[i] = 0;
    kbody[i] = sentinel;
    for (int d = 0; d < 6; d++) nb6[(size_t)i * 6 + d] = NONE;
}

// per body word: first, count (new ranges of the rebuilt and new bodies), or a dying body (count 0: dead)
__global__ void k_body_ranges(uint32_t n, const uint32_t *words, uint32_t *first, uint32_t *count, uint8_t *alive,
                              uint8_t *dirty) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t b = words[3 * k], f = words[3 * k + 1], c = words[3 * k + 2];
    first[b] = f;
    count[b] = c;
    dirty[b] = 0;
    if (c == 0) alive[b] = 0;
}

__global__ void k_scene_awake(uint32_t nb, const uint32_t *scene, const uint8_t *alive, const uint8_t *asleep,
                              uint32_t *awake) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || !alive[b] || asleep[b]) return;
    atomicAdd(&awake[scene[b]], 1u);
}

// h01 (src/lib.rs:341-345): a 32-bit mix of h + k * 0x9E3779B9 to a float in [0, 1)
static float h01(uint32_t h, uint32_t k) {
    uint32_t x = h + k * 0x9E3779B9u;
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return (float)(x >> 8) / 16777216.0f;
}

static SplitState *split_state(sf_world *w) {
    if (!w->split) {
        w->split = new SplitState();
        w->split->scene_rebuilds.assign(w->n_scenes, 0);
    }
    return w->split;
}

void split_destroy(sf_world *w) {
    delete w->split;
    w->split = nullptr;
}

static sf_status rebuild_impl(sf_world *w, sf_rebuild_report *report) {
    const auto t0 = std::chrono::steady_clock::now();
    sf_rebuild_report rep{};
    cudaStream_t st = w->stream;
    SplitState &X = *split_state(w);
    const uint32_t nb = w->nb;
    SF_CUDA(X.list.alloc(nb));
    SF_CUDA(X.count.alloc(2));
    SF_CUDA(cudaMemsetAsync(X.count.p, 0, 8, st));
    k_dirty_collect<<<grid_for(nb, 256), 256, 0, st>>>(nb, w->b_dirty.p, w->b_alive.p, X.list.p, X.count.p);
    w->launches++;
    SF_CUDA(cudaGetLastError());
    uint32_t nd_ = 0;
    SF_CUDA(cudaMemcpyAsync(&nd_, X.count.p, 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    if (nd_ == 0) {
        SF_CUDA(cudaMemsetAsync(w->b_dirty.p, 0, w->b_dirty.bytes(), st));   // dead bodies' marks
        rep.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (report) *report = rep;
        return SF_OK;
    }
    // the marked bodies in body order, their ranges and poses
    std::vector<uint32_t> bodies(nd_);
    SF_CUDA(cudaMemcpyAsync(bodies.data(), X.list.p, (size_t)nd_ * 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    std::sort(bodies.begin(), bodies.end());
    SF_CUDA(cudaMemcpyAsync(X.list.p, bodies.data(), (size_t)nd_ * 4, cudaMemcpyHostToDevice, st));
    SF_CUDA(X.bsel.grow((size_t)nd_ * 25));
    k_body_snapshot<<<grid_for(nd_, 128), 128, 0, st>>>(nd_, X.list.p, w->b_first.p, w->b_count.p, w->b_scene.p,
                                                        w->b_pos.p, w->b_q.p, w->b_v.p, w->b_w.p, w->b_rot.p,
                                                        X.bsel.p);
    SF_CUDA(X.awake.alloc(w->n_scenes));
    SF_CUDA(cudaMemsetAsync(X.awake.p, 0, (size_t)w->n_scenes * 4, st));
    k_scene_awake<<<grid_for(nb, 256), 256, 0, st>>>(nb, w->b_scene.p, w->b_alive.p, w->b_asleep.p, X.awake.p);
    w->launches += 2;
    SF_CUDA(cudaGetLastError());
    std::vector<uint32_t> bs((size_t)nd_ * 25), awake(w->n_scenes);
    SF_CUDA(cudaMemcpyAsync(bs.data(), X.bsel.p, bs.size() * 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaMemcpyAsync(awake.data(), X.awake.p, awake.size() * 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    // their bricks
    std::vector<uint32_t> slots;
    std::vector<size_t> at(nd_ + 1, 0);
    for (uint32_t k = 0; k < nd_; k++) {
        const uint32_t f = bs[(size_t)k * 25], c = bs[(size_t)k * 25 + 1];
        at[k] = slots.size();
        for (uint32_t t = 0; t < c; t++) slots.push_back(f + t);
    }
    at[nd_] = slots.size();
    // the walk reads, per brick, material, neighbours and bonds (LITE words); the records stay on the device
    std::vector<uint32_t> rec(slots.size() * LITE);
    if (!slots.empty()) {
        SF_CUDA(X.slots.grow(slots.size()));
        SF_CUDA(X.brec.grow(slots.size() * SPLIT_WORDS));
        SF_CUDA(cudaMemcpyAsync(X.slots.p, slots.data(), slots.size() * 4, cudaMemcpyHostToDevice, st));
        k_brick_snapshot<<<grid_for(slots.size(), 256), 256, 0, st>>>((uint32_t)slots.size(), X.slots.p, w->k_xyz.p,
                                                                      w->k_mat.p, w->k_nb6.p, w->k_bond.p,
                                                                      w->k_bmax.p, w->k_local.p, w->k_sup.p,
                                                                      w->k_phi.p, w->k_ext.p, w->k_phi64.p, X.brec.p);
        w->launches++;
        SF_CUDA(cudaGetLastError());
        SF_CUDA(X.lite.grow(rec.size()));
        k_brick_lite<<<grid_for(rec.size(), 256), 256, 0, st>>>((uint32_t)slots.size(), X.brec.p, X.lite.p);
        w->launches++;
        SF_CUDA(cudaMemcpyAsync(rec.data(), X.lite.p, rec.size() * 4, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaStreamSynchronize(st));
    }
    auto bondf = [](uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; };

    // ---- rebuild_body's walk, body by body
    std::vector<uint32_t> wslots, wsrc, wbody, freed, ranges, setup_ids;
    std::vector<uint32_t> nmap(slots.size(), NONE), pcomp(slots.size(), NONE);
    std::vector<uint8_t> setup_keep;
    std::vector<float> poses;
    std::vector<uint8_t> live_scene(w->n_scenes, 0);
    for (uint32_t k = 0; k < nd_; k++) {
        const uint32_t *B = &bs[(size_t)k * 25];
        const uint32_t id = bodies[k], first = B[0], cnt = B[1], q = B[2];
        Scene &sc = w->scenes[q];
        const uint32_t *R = &rec[at[k] * LITE];
        const uint32_t draw_key = X.scene_rebuilds[q]++;
        rep.bodies++;
        live_scene[q] = 1;
        step_warm_invalidate(w, q);   // brick ids move
        // bricks still there, in list order (a removed brick leaves the body)
        std::vector<uint32_t> lst;
        for (uint32_t t = 0; t < cnt; t++) {
            if (R[(size_t)t * LITE + L_MAT] != 0) lst.push_back(t);
            else rep.removed++;
        }
        if (lst.empty()) {
            for (uint32_t t = 0; t < cnt; t++) freed.push_back(first + t);
            ranges.insert(ranges.end(), {id, 0u, 0u});
            rep.dissolved++;
            continue;
        }
        // components: breadth first from each unvisited brick in list order, over intact bonds (linked)
        std::vector<int32_t> comp(cnt, -1);
        uint32_t ncomp = 0;
        std::vector<uint32_t> qu;
        for (uint32_t t0 : lst) {
            if (comp[t0] >= 0) continue;
            comp[t0] = (int32_t)ncomp;
            qu.assign(1, t0);
            for (size_t h = 0; h < qu.size(); h++) {
                const uint32_t i = qu[h];
                const uint32_t *ri = &R[(size_t)i * LITE];
                for (int d = 0; d < 6; d++) {
                    const uint32_t js = ri[L_NB6 + d];
                    if (js == NONE || js < first || js >= first + cnt) continue;
                    const uint32_t j = js - first;
                    if (comp[j] >= 0 || R[(size_t)j * LITE + L_MAT] == 0) continue;
                    const float hp = (d & 1) == 0 ? bondf(ri[L_BOND + (d >> 1)]) : bondf(R[(size_t)j * LITE + L_BOND + (d >> 1)]);
                    if (!(hp > 0.0f)) continue;
                    comp[j] = (int32_t)ncomp;
                    qu.push_back(j);
                }
            }
            ncomp++;
        }
        // no room for the new pieces: keep the body whole (src/lib.rs:970-971)
        uint32_t nc = ncomp;
        if (nc > 1) {
            uint32_t extra = 0;
            for (uint32_t t : lst) if (comp[t] > 0) extra++;
            if (sc.bodies_used + (nc - 1) > sc.n_bodies || sc.bricks_used + extra > sc.n_bricks) {
                for (uint32_t t : lst) comp[t] = 0;
                nc = 1;
            }
        }
        // stable grouping by component
        std::vector<std::vector<uint32_t>> groups(nc);
        for (uint32_t t : lst) groups[comp[t]].push_back(t);
        // the first piece stays at the front of the range; the rest of the range is free (new pieces take new slots)
        for (uint32_t t = (uint32_t)groups[0].size(); t < cnt; t++) freed.push_back(first + t);
        // the new slot of each kept brick
        std::vector<uint32_t> nslot(cnt, NONE);
        std::vector<uint32_t> cbody(nc, NONE), cfirst(nc, 0);
        for (uint32_t c = 0; c < nc; c++) {
            const std::vector<uint32_t> &g = groups[c];
            if (c > 0 && g.size() == 1 && awake[q] > 1500) {
                const uint32_t m = R[(size_t)g[0] * LITE + L_MAT];
                const float p = std::min((float)(awake[q] - 1500) / 2000.0f, 0.85f);
                if (m != STEEL && h01(draw_key, g[0]) < p) { rep.lone++; continue; }
            }
            if (c == 0) { cbody[c] = id; cfirst[c] = first; }
            else {
                cbody[c] = sc.body_off + sc.bodies_used++;
                cfirst[c] = sc.brick_off + sc.bricks_used;
                sc.bricks_used += (uint32_t)g.size();
                rep.pieces++;
            }
            for (uint32_t t = 0; t < g.size(); t++) nslot[g[t]] = cfirst[c] + t;
        }
        // the per-brick map the GPU renumbers neighbours by: new slot and piece (a neighbour in another piece, or
        // gone, is none)
        for (uint32_t t = 0; t < cnt; t++) {
            nmap[at[k] + t] = nslot[t];
            pcomp[at[k] + t] = comp[t] < 0 ? NONE : (uint32_t)comp[t];
        }
        for (uint32_t c = 0; c < nc; c++) {
            if (cbody[c] == NONE) continue;
            const std::vector<uint32_t> &g = groups[c];
            for (uint32_t t = 0; t < g.size(); t++) {
                wslots.push_back(cfirst[c] + t);
                wsrc.push_back((uint32_t)(at[k] + g[t]));
                wbody.push_back(k);
            }
            ranges.insert(ranges.end(), {cbody[c], cfirst[c], (uint32_t)g.size()});
            setup_ids.push_back(cbody[c]);
            setup_keep.push_back(c == 0 ? 1 : 0);
            for (int j = 0; j < 22; j++) { float f; std::memcpy(&f, &B[3 + j], 4); poses.push_back(f); }
        }
    }
    // ---- the GPU side
    if (!freed.empty()) {
        SF_CUDA(X.freed.grow(freed.size()));
        SF_CUDA(cudaMemcpyAsync(X.freed.p, freed.data(), freed.size() * 4, cudaMemcpyHostToDevice, st));
        k_brick_free<<<grid_for(freed.size(), 256), 256, 0, st>>>((uint32_t)freed.size(), X.freed.p, w->sentinel,
                                                                  w->k_mat.p, w->k_body.p, w->k_nb6.p);
        w->launches++;
    }
    if (!wslots.empty()) {
        // per moved brick: destination, snapshot entry, body; per snapshot entry: new slot and piece; per body: its
        // old range and snapshot offset
        const size_t nw = wslots.size();
        std::vector<uint32_t> up;
        up.reserve(nw * 3 + slots.size() * 2 + (size_t)nd_ * 3);
        up.insert(up.end(), wslots.begin(), wslots.end());
        up.insert(up.end(), wsrc.begin(), wsrc.end());
        up.insert(up.end(), wbody.begin(), wbody.end());
        up.insert(up.end(), nmap.begin(), nmap.end());
        up.insert(up.end(), pcomp.begin(), pcomp.end());
        for (uint32_t k = 0; k < nd_; k++) { up.push_back(bs[(size_t)k * 25]); up.push_back(bs[(size_t)k * 25 + 1]); up.push_back((uint32_t)at[k]); }
        SF_CUDA(X.moves.grow(up.size()));
        SF_CUDA(cudaMemcpyAsync(X.moves.p, up.data(), up.size() * 4, cudaMemcpyHostToDevice, st));
        BrickMove M;
        M.dst = X.moves.p; M.src = M.dst + nw; M.body = M.src + nw; M.nmap = M.body + nw; M.ncomp = M.nmap + slots.size();
        M.brange = M.ncomp + slots.size();
        M.rec = X.brec.p;
        k_brick_move<<<grid_for(nw, 256), 256, 0, st>>>((uint32_t)nw, M, w->k_xyz.p, w->k_mat.p, w->k_nb6.p,
                                                        w->k_bond.p, w->k_bmax.p, w->k_local.p, w->k_sup.p, w->k_phi.p,
                                                        w->k_ext.p, w->k_phi64.p);
        w->launches++;
    }
    const uint32_t nr = (uint32_t)(ranges.size() / 3);
    SF_CUDA(X.words.grow(ranges.size()));
    SF_CUDA(cudaMemcpyAsync(X.words.p, ranges.data(), ranges.size() * 4, cudaMemcpyHostToDevice, st));
    k_body_ranges<<<grid_for(nr, 128), 128, 0, st>>>(nr, X.words.p, w->b_first.p, w->b_count.p, w->b_alive.p,
                                                     w->b_dirty.p);
    w->launches++;
    SF_CUDA(cudaGetLastError());
    if (!setup_ids.empty()) {
        SF_CUDA(X.list.grow(setup_ids.size()));
        SF_CUDA(X.pose.grow(poses.size()));
        SF_CUDA(cudaMemcpyAsync(X.list.p, setup_ids.data(), setup_ids.size() * 4, cudaMemcpyHostToDevice, st));
        SF_CUDA(cudaMemcpyAsync(X.pose.p, poses.data(), poses.size() * 4, cudaMemcpyHostToDevice, st));
        SF_CUDA(setup_bodies_from_local(w, X.list.p, (uint32_t)setup_ids.size(), X.pose.p));
        SF_CUDA(X.keep.grow(setup_keep.size()));
        SF_CUDA(cudaMemcpyAsync(X.keep.p, setup_keep.data(), setup_keep.size(), cudaMemcpyHostToDevice, st));
        SF_CUDA(body_load_setup(w, X.list.p, 0u, (uint32_t)setup_ids.size(), X.keep.p));
    }
    SF_CUDA(cudaMemsetAsync(w->b_dirty.p, 0, w->b_dirty.bytes(), st));
    for (uint32_t q = 0; q < w->n_scenes; q++) if (live_scene[q]) step_set_live(w, q, true);
    SF_CUDA(cudaStreamSynchronize(st));   // host vectors are the copies' sources
    rep.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (report) *report = rep;
    return read_error_word(w);
}

}  // namespace sf

using namespace sf;

extern "C" {

sf_status sf_world_remove_bricks(sf_world *w, const uint32_t *statics, uint32_t n_statics, const uint32_t *body_bricks,
                                 uint32_t n_body_bricks) {
    if (!w || (n_statics && !statics) || (n_body_bricks && !body_bricks)) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->pool.empty()) { set_error("a scene pool's bricks are removed by unloading the scene"); return SF_ERR_STATE; }
    if (n_body_bricks && !w->b_dirty.p) { set_error("bodies split only in a world created with spare capacity"); return SF_ERR_STATE; }
    for (uint32_t k = 0; k < n_statics; k++)
        if (statics[k] >= w->ns) { set_error("static brick %u does not exist", statics[k]); return SF_ERR_ARG; }
    for (uint32_t k = 0; k < n_body_bricks; k++)
        if (body_bricks[k] >= w->nd) { set_error("body brick %u does not exist", body_bricks[k]); return SF_ERR_ARG; }
    cudaStream_t st = w->stream;
    DBuf<uint32_t> a, b;
    if (n_statics) {
        SF_CUDA(a.alloc(n_statics));
        SF_CUDA(cudaMemcpyAsync(a.p, statics, (size_t)n_statics * 4, cudaMemcpyHostToDevice, st));
        k_remove_static<<<grid_for(n_statics, 256), 256, 0, st>>>(n_statics, a.p, w->s_scene.p, w->s_cell.p, w->s_sid.p,
                                                                  w->ctab.p, w->cpool.p, w->s_mat.p, w->st_conn.p,
                                                                  w->n_struct);
        w->launches++;
    }
    if (n_body_bricks) {
        SF_CUDA(b.alloc(n_body_bricks));
        SF_CUDA(cudaMemcpyAsync(b.p, body_bricks, (size_t)n_body_bricks * 4, cudaMemcpyHostToDevice, st));
        k_remove_body_bricks<<<grid_for(n_body_bricks, 256), 256, 0, st>>>(n_body_bricks, b.p, w->k_body.p,
                                                                          w->b_alive.p, w->k_mat.p, w->b_dirty.p);
        w->launches++;
    }
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaStreamSynchronize(st));
    return SF_OK;
}

sf_status sf_read_body_bonds(sf_world *w, float *bond4, uint32_t *nb6) {
    if (!w) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->k_nb6.p) { set_error("body bricks have bonds only in a world created with spare capacity"); return SF_ERR_STATE; }
    if (bond4) SF_CUDA(cudaMemcpyAsync(bond4, w->k_bond.p, (size_t)w->nd * 16, cudaMemcpyDeviceToHost, w->stream));
    if (nb6) SF_CUDA(cudaMemcpyAsync(nb6, w->k_nb6.p, (size_t)w->nd * 24, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}

sf_status sf_world_rebuild_bodies(sf_world *w, sf_rebuild_report *report) {
    if (!w) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->b_dirty.p) {
        if (report) *report = sf_rebuild_report{};
        return SF_OK;   // no spare capacity: bodies cannot split and nothing marks them
    }
    return rebuild_impl(w, report);
}

}  // extern "C"

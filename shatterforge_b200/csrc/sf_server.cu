// Serving: a request loop over resident worlds with continuous batching (host code).
//
// Two workers run side by side, each on its own CUDA stream, so their device work overlaps:
//   rigid      scene-step requests. Scenes live in the slots of one scene pool; each tick steps every resident
//              scene that has a pending request by one step, in one set of launches (sf_world_step_scenes). A
//              request that arrives while others run joins at the next tick; a request finishes after its
//              nsteps ticks. A scene without a slot is admitted when a slot that fits is free, or by evicting the
//              least recently used idle scene to pinned host memory (sf_pool_save) and restoring it later
//              (sf_pool_restore, bit for bit).
//   structure  structure-solve requests on the resident structures world. Each tick solves every structure with
//              a pending request for up to sweeps_per_tick sweeps in one persistent launch
//              (sf_structure_solve_set); a structure leaves when its residual is below the request's tolerance
//              or its sweeps reach the request's limit. Solves restart from the stored potentials, so a solve
//              split over ticks takes exactly the sweeps of one uninterrupted solve.
// With batching off, one worker takes the requests one at a time in arrival order and runs each to completion
// with its own launches: the plain per-request path the batched one is compared against.
//
// Requests carry an arrival time on the server clock (seconds since sf_server_start); a worker sees a request
// only from then on, so a whole arrival process can be submitted up front and replayed in real time.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "sf_internal.cuh"

namespace sf {

struct SceneCopy {
    std::vector<int32_t> static_xyz, static_sid, body_brick_xyz;
    std::vector<uint8_t> static_mat, static_infill, body_brick_mat;
    std::vector<uint32_t> body_first;
    std::vector<float> body_pose;
    uint32_t n_static = 0, n_bodies = 0, n_bricks = 0, n_chunks = 0;
    sf_scene_desc desc() const {
        sf_scene_desc d{};
        d.n_static = n_static;
        d.static_xyz = static_xyz.data(); d.static_mat = static_mat.data();
        d.static_sid = static_sid.data(); d.static_infill = static_infill.data();
        d.n_bodies = n_bodies;
        d.body_first = body_first.data(); d.body_brick_xyz = body_brick_xyz.data();
        d.body_brick_mat = body_brick_mat.data(); d.body_pose = body_pose.data();
        return d;
    }
};

struct Req {
    sf_request r{};
    uint64_t ticket = 0;
    std::vector<uint32_t> load_brick;
    std::vector<float> load_value;
    uint32_t steps = 0, sweeps = 0;
    double residual = 0.0, t_start = -1.0;
};

struct SceneRec {
    SceneCopy sc;
    int slot = -1;
    uint64_t last_used = 0;
    std::deque<Req *> q;
    uint8_t *snap = nullptr;     // pinned snapshot of an evicted scene
    uint64_t snap_bytes = 0;
    bool has_snap = false;
    std::vector<float> init13, init_sleep;   // optional body state at the first load
    std::vector<uint8_t> init_flags;
};

}  // namespace sf

using namespace sf;
using Clock = std::chrono::steady_clock;

struct sf_server {
    sf_server_desc D{};
    std::vector<sf_pool_slot> slots;
    sf_world *pool = nullptr;
    sf_world *structs = nullptr;
    int device = 0;
    std::vector<std::unique_ptr<SceneRec>> scenes;
    std::vector<int> slot_owner;
    std::vector<std::deque<Req *>> squeue;     // per structure
    std::vector<std::unique_ptr<Req>> all;     // owns every request
    std::mutex mu;
    std::condition_variable cv_in, cv_out;
    std::multimap<double, Req *> incoming;     // by arrival time
    std::deque<sf_result> results;
    std::vector<std::thread> threads;
    std::atomic<bool> stop{false};
    bool started = false;
    Clock::time_point t0;
    uint64_t next_ticket = 1;
    uint64_t submitted = 0, completed = 0;
    sf_server_stats st{};
    uint64_t pool_bytes = 0;
    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// counters shared by the workers and sf_server_get_stats
template <class F> void bump(sf_server *S, F &&f) {
    std::lock_guard<std::mutex> lk(S->mu);
    f(S->st);
}

void complete(sf_server *S, Req *q, sf_status status, double t) {
    sf_result r{};
    r.ticket = q->ticket; r.kind = q->r.kind; r.world = q->r.world; r.status = (uint32_t)status;
    r.steps = q->steps; r.sweeps = q->sweeps; r.residual = q->residual;
    r.t_arrival = q->r.t_arrival; r.t_start = q->t_start < 0 ? t : q->t_start; r.t_done = t;
    std::lock_guard<std::mutex> lk(S->mu);
    S->results.push_back(r);
    S->completed++;
    S->st.completed++;
    S->cv_out.notify_all();
}

// move the requests of `kind` (0 = any) that have arrived into their queues; returns the next later arrival
double take_arrivals(sf_server *S, uint32_t kind, std::vector<Req *> *plain) {
    std::lock_guard<std::mutex> lk(S->mu);
    const double t = S->now();
    double next = 1e300;
    for (auto it = S->incoming.begin(); it != S->incoming.end();) {
        Req *q = it->second;
        if (kind && q->r.kind != kind) { ++it; continue; }
        if (it->first > t) { next = std::min(next, it->first); break; }
        if (plain) plain->push_back(q);
        else if (q->r.kind == SF_REQ_STEP) S->scenes[q->r.world]->q.push_back(q);
        else S->squeue[q->r.world].push_back(q);
        it = S->incoming.erase(it);
    }
    return next;
}

void wait_for_work(sf_server *S, double next_arrival) {
    std::unique_lock<std::mutex> lk(S->mu);
    const double dt = next_arrival - S->now();
    if (S->stop) return;
    if (dt > 0) S->cv_in.wait_for(lk, std::chrono::duration<double>(std::min(dt, 0.05)));
}

bool fits(const sf_pool_slot &c, const SceneCopy &sc) {
    return sc.n_bodies <= c.bodies && sc.n_bricks <= c.bricks && sc.n_static <= c.statics && sc.n_chunks <= c.chunks;
}

// a slot for scene `id`: the smallest free slot that fits, else the least recently used idle resident scene's
sf_status admit(sf_server *S, uint32_t id, bool &ok) {
    ok = false;
    SceneRec &R = *S->scenes[id];
    int best = -1;
    for (size_t s = 0; s < S->slots.size(); s++)
        if (S->slot_owner[s] < 0 && fits(S->slots[s], R.sc) && (best < 0 || S->slots[s].bodies < S->slots[best].bodies)) best = (int)s;
    if (best < 0) {
        uint64_t oldest = UINT64_MAX;
        for (size_t s = 0; s < S->slots.size(); s++) {
            const int o = S->slot_owner[s];
            if (o < 0 || !fits(S->slots[s], R.sc)) continue;
            const SceneRec &V = *S->scenes[o];
            if (!V.q.empty()) continue;
            if (V.last_used < oldest) { oldest = V.last_used; best = (int)s; }
        }
        if (best < 0) return SF_OK;   // wait for a slot
        SceneRec &V = *S->scenes[S->slot_owner[best]];
        uint64_t need = sf_pool_snapshot_bytes(V.sc.n_bodies, V.sc.n_bricks);
        if (!V.snap) {
            if (cudaMallocHost((void **)&V.snap, std::max<uint64_t>(need, 1)) != cudaSuccess) { set_error("pinned snapshot allocation failed"); return SF_ERR_CUDA; }
            V.snap_bytes = need;
        }
        sf_status r = sf_pool_save(S->pool, (uint32_t)best, V.snap, V.snap_bytes, nullptr);
        if (r != SF_OK) return r;
        V.has_snap = true;
        V.slot = -1;
        S->slot_owner[best] = -1;
        bump(S, [](sf_server_stats &t) { t.evictions++; });
    }
    const sf_scene_desc d = R.sc.desc();
    sf_status r = R.has_snap ? sf_pool_restore(S->pool, (uint32_t)best, &d, R.snap, R.snap_bytes)
                             : sf_pool_load(S->pool, (uint32_t)best, &d);
    if (r == SF_OK && !R.has_snap && !R.init13.empty())
        r = sf_pool_write_bodies(S->pool, (uint32_t)best, R.init13.data(), R.init_sleep.data(), R.init_flags.data());
    if (r != SF_OK) return r;
    const bool restored = R.has_snap;
    bump(S, [&](sf_server_stats &t) { if (restored) t.restores++; else t.loads++; });
    R.slot = best;
    S->slot_owner[best] = (int)id;
    ok = true;
    return SF_OK;
}

void rigid_worker(sf_server *S) {
    cudaSetDevice(S->device);
    std::vector<uint8_t> mask(S->slots.size());
    uint64_t tick = 0;
    while (!S->stop) {
        const double next = take_arrivals(S, SF_REQ_STEP, nullptr);
        // admission, oldest head first
        std::vector<std::pair<double, uint32_t>> want;
        for (uint32_t id = 0; id < S->scenes.size(); id++) {
            SceneRec &R = *S->scenes[id];
            if (!R.q.empty() && R.slot < 0) want.push_back({R.q.front()->r.t_arrival, id});
        }
        std::sort(want.begin(), want.end());
        for (auto &wq : want) {
            bool ok = false;
            sf_status r = admit(S, wq.second, ok);
            if (r != SF_OK) {
                SceneRec &R = *S->scenes[wq.second];
                while (!R.q.empty()) { complete(S, R.q.front(), r, S->now()); R.q.pop_front(); }
            }
        }
        std::fill(mask.begin(), mask.end(), 0);
        std::vector<uint32_t> act;
        const double t = S->now();
        for (uint32_t id = 0; id < S->scenes.size(); id++) {
            SceneRec &R = *S->scenes[id];
            if (R.slot < 0 || R.q.empty()) continue;
            Req *q = R.q.front();
            if (q->t_start < 0) q->t_start = t;
            mask[R.slot] = 1;
            act.push_back(id);
        }
        if (act.empty()) { wait_for_work(S, next); continue; }
        const auto b0 = Clock::now();
        sf_status r = sf_world_step_scenes(S->pool, S->D.dt, 1, mask.data());
        tick++;
        for (uint32_t id : act) {
            SceneRec &R = *S->scenes[id];
            R.last_used = tick;
            Req *q = R.q.front();
            q->steps++;
            sf_status rr = r;
            if (rr == SF_OK && q->steps < q->r.nsteps) continue;
            if (rr == SF_OK && q->r.out_state13) rr = sf_pool_read_bodies(S->pool, (uint32_t)R.slot, q->r.out_state13, nullptr, nullptr);
            complete(S, q, rr, S->now());
            R.q.pop_front();
        }
        const double busy = std::chrono::duration<double>(Clock::now() - b0).count();
        bump(S, [&](sf_server_stats &t) { t.step_ticks++; t.busy_s += busy; });
    }
}

void structure_worker(sf_server *S) {
    cudaSetDevice(S->device);
    const uint32_t nst = S->structs->n_struct;
    std::vector<uint32_t> sweeps(std::max<uint32_t>(nst, 1));
    std::vector<double> resid(std::max<uint32_t>(nst, 1));
    const uint32_t per_tick = S->D.sweeps_per_tick ? S->D.sweeps_per_tick : 128;
    while (!S->stop) {
        const double next = take_arrivals(S, SF_REQ_SOLVE, nullptr);
        std::vector<Req *> heads;
        for (uint32_t q = 0; q < nst; q++) if (!S->squeue[q].empty()) heads.push_back(S->squeue[q].front());
        if (heads.empty()) { wait_for_work(S, next); continue; }
        const auto b0 = Clock::now();
        // loads of the requests that start now, in ticket order
        std::vector<uint32_t> lb;
        std::vector<float> lv;
        const double t = S->now();
        std::sort(heads.begin(), heads.end(), [](const Req *a, const Req *b) { return a->ticket < b->ticket; });
        for (Req *q : heads)
            if (q->t_start < 0) {
                q->t_start = t;
                lb.insert(lb.end(), q->load_brick.begin(), q->load_brick.end());
                lv.insert(lv.end(), q->load_value.begin(), q->load_value.end());
            }
        sf_status r = sf_structure_add_loads(S->structs, (uint32_t)lb.size(), lb.data(), lv.data());
        // one launch per distinct (omega, tol)
        std::vector<bool> done(heads.size(), false);
        for (size_t g = 0; g < heads.size() && r == SF_OK; g++) {
            if (done[g]) continue;
            std::vector<int32_t> ids;
            std::vector<size_t> members;
            uint32_t cap = per_tick;
            for (size_t k = g; k < heads.size(); k++)
                if (!done[k] && heads[k]->r.omega == heads[g]->r.omega && heads[k]->r.tol == heads[g]->r.tol) {
                    ids.push_back((int32_t)heads[k]->r.world);
                    members.push_back(k);
                    done[k] = true;
                    cap = std::min(cap, heads[k]->r.max_sweeps - heads[k]->sweeps);
                }
            sf_solve_report rep{};
            r = sf_structure_solve_set(S->structs, ids.data(), (uint32_t)ids.size(), heads[g]->r.omega, heads[g]->r.tol,
                                       std::max<uint32_t>(cap, 1), &rep);
            if (r == SF_OK) r = sf_read_solve_detail(S->structs, sweeps.data(), resid.data());
            bump(S, [](sf_server_stats &t) { t.solve_ticks++; });
            for (size_t k : members) {
                Req *q = heads[k];
                const uint32_t s = q->r.world;
                if (r != SF_OK) { complete(S, q, r, S->now()); S->squeue[s].pop_front(); continue; }
                q->sweeps += sweeps[s];
                q->residual = resid[s];
                if (resid[s] < (double)q->r.tol || q->sweeps >= q->r.max_sweeps || sweeps[s] == 0) {
                    complete(S, q, SF_OK, S->now());
                    S->squeue[s].pop_front();
                }
            }
        }
        if (r != SF_OK)
            for (Req *q : heads) {
                auto &dq = S->squeue[q->r.world];
                if (!dq.empty() && dq.front() == q) { complete(S, q, r, S->now()); dq.pop_front(); }
            }
        const double busy = std::chrono::duration<double>(Clock::now() - b0).count();
        bump(S, [&](sf_server_stats &t) { t.busy_s += busy; });
    }
}

// batching off: one request at a time, in arrival order, each run to completion
void plain_worker(sf_server *S) {
    cudaSetDevice(S->device);
    std::vector<uint8_t> mask(S->slots.size());
    std::deque<Req *> fifo;
    uint64_t tick = 0;
    while (!S->stop) {
        std::vector<Req *> got;
        const double next = take_arrivals(S, 0, &got);
        fifo.insert(fifo.end(), got.begin(), got.end());
        if (fifo.empty()) { wait_for_work(S, next); continue; }
        Req *q = fifo.front();
        fifo.pop_front();
        const auto b0 = Clock::now();
        q->t_start = S->now();
        sf_status r = SF_OK;
        if (q->r.kind == SF_REQ_STEP) {
            SceneRec &R = *S->scenes[q->r.world];
            if (R.slot < 0) {
                bool ok = false;
                r = admit(S, q->r.world, ok);
                if (r == SF_OK && !ok) { set_error("no slot fits scene %u", q->r.world); r = SF_ERR_BUDGET; }
            }
            if (r == SF_OK) {
                std::fill(mask.begin(), mask.end(), 0);
                mask[R.slot] = 1;
                r = sf_world_step_scenes(S->pool, S->D.dt, q->r.nsteps, mask.data());
                R.last_used = ++tick;
                const uint32_t ns = q->r.nsteps;
                bump(S, [&](sf_server_stats &t) { t.step_ticks += ns; });
                if (r == SF_OK) q->steps = q->r.nsteps;
                if (r == SF_OK && q->r.out_state13) r = sf_pool_read_bodies(S->pool, (uint32_t)R.slot, q->r.out_state13, nullptr, nullptr);
            }
        } else {
            r = sf_structure_add_loads(S->structs, (uint32_t)q->load_brick.size(), q->load_brick.data(), q->load_value.data());
            const int32_t id = (int32_t)q->r.world;
            sf_solve_report rep{};
            if (r == SF_OK) r = sf_structure_solve_set(S->structs, &id, 1, q->r.omega, q->r.tol, q->r.max_sweeps, &rep);
            if (r == SF_OK) {
                uint32_t sw = 0;
                double rs = 0.0;
                std::vector<uint32_t> sweeps(S->structs->n_struct);
                std::vector<double> resid(S->structs->n_struct);
                r = sf_read_solve_detail(S->structs, sweeps.data(), resid.data());
                sw = sweeps[id]; rs = resid[id];
                q->sweeps = sw; q->residual = rs;
            }
            bump(S, [](sf_server_stats &t) { t.solve_ticks++; });
        }
        complete(S, q, r, S->now());
        const double busy = std::chrono::duration<double>(Clock::now() - b0).count();
        bump(S, [&](sf_server_stats &t) { t.busy_s += busy; });
    }
}

uint32_t count_chunks(const sf_scene_desc &d) {
    std::vector<uint32_t> keys(d.n_static);
    for (uint32_t k = 0; k < d.n_static; k++)
        keys[k] = chunk_slot(d.static_xyz[3 * k], d.static_xyz[3 * k + 1], d.static_xyz[3 * k + 2]);
    std::sort(keys.begin(), keys.end());
    return (uint32_t)(std::unique(keys.begin(), keys.end()) - keys.begin());
}

}  // namespace

extern "C" {

sf_status sf_server_create(const sf_server_desc *desc, sf_server **out) {
    if (!desc || !out || (desc->n_slots && !desc->slots)) { set_error("null argument"); return SF_ERR_ARG; }
    *out = nullptr;
    if (!(desc->dt > 0.0f)) { set_error("dt must be positive"); return SF_ERR_ARG; }
    std::unique_ptr<sf_server, void (*)(sf_server *)> S(new sf_server(), sf_server_destroy);
    S->D = *desc;
    S->slots.assign(desc->slots, desc->slots + desc->n_slots);
    S->D.slots = nullptr;
    SF_CUDA(cudaGetDevice(&S->device));
    uint64_t est = 0;
    if (desc->n_slots) {
        sf_status r = sf_pool_bytes(desc->n_slots, desc->slots, &est);
        if (r != SF_OK) return r;
    }
    if (desc->budget_bytes && est > desc->budget_bytes) {
        set_error("the pool's slots take %llu bytes, over the budget of %llu", (unsigned long long)est, (unsigned long long)desc->budget_bytes);
        return SF_ERR_BUDGET;
    }
    size_t free0 = 0, total = 0;
    SF_CUDA(cudaMemGetInfo(&free0, &total));
    if (desc->n_slots) {
        sf_status r = sf_pool_create(desc->n_slots, S->slots.data(), &desc->params, &S->pool);
        if (r != SF_OK) return r;
    }
    if (desc->structures) {
        sf_status r = sf_world_create(desc->structures, &desc->params, &S->structs);
        if (r != SF_OK) return r;
        S->squeue.resize(S->structs->n_struct);
    }
    size_t free1 = 0;
    SF_CUDA(cudaMemGetInfo(&free1, &total));
    S->pool_bytes = free0 > free1 ? free0 - free1 : 0;
    S->st.pool_bytes = S->pool_bytes;
    if (desc->budget_bytes && S->pool_bytes > desc->budget_bytes) {
        set_error("resident state takes %llu bytes, over the budget of %llu", (unsigned long long)S->pool_bytes, (unsigned long long)desc->budget_bytes);
        return SF_ERR_BUDGET;
    }
    S->slot_owner.assign(S->slots.size(), -1);
    *out = S.release();
    return SF_OK;
}

sf_status sf_server_add_scene(sf_server *S, const sf_scene_desc *d, uint32_t *id) {
    if (!S || !d || !id) { set_error("null argument"); return SF_ERR_ARG; }
    if (S->started) { set_error("scenes are registered before sf_server_start"); return SF_ERR_STATE; }
    if (!S->pool) { set_error("the server has no scene pool"); return SF_ERR_STATE; }
    auto R = std::make_unique<SceneRec>();
    SceneCopy &c = R->sc;
    c.n_static = d->n_static;
    c.n_bodies = d->n_bodies;
    if (d->n_bodies && !d->body_first) { set_error("null body_first"); return SF_ERR_ARG; }
    c.n_bricks = d->n_bodies ? d->body_first[d->n_bodies] : 0;
    if (c.n_static) {
        if (!d->static_xyz || !d->static_mat || !d->static_sid || !d->static_infill) { set_error("null static array"); return SF_ERR_ARG; }
        c.static_xyz.assign(d->static_xyz, d->static_xyz + (size_t)c.n_static * 3);
        c.static_mat.assign(d->static_mat, d->static_mat + c.n_static);
        c.static_sid.assign(d->static_sid, d->static_sid + c.n_static);
        c.static_infill.assign(d->static_infill, d->static_infill + c.n_static);
        for (uint32_t k = 0; k < c.n_static; k++)
            if (!inb(c.static_xyz[3 * k], c.static_xyz[3 * k + 1], c.static_xyz[3 * k + 2])) { set_error("static %u outside the lattice", k); return SF_ERR_ARG; }
    }
    if (c.n_bodies) {
        if (!d->body_brick_xyz || !d->body_brick_mat || !d->body_pose) { set_error("null body array"); return SF_ERR_ARG; }
        c.body_first.assign(d->body_first, d->body_first + c.n_bodies + 1);
        c.body_brick_xyz.assign(d->body_brick_xyz, d->body_brick_xyz + (size_t)c.n_bricks * 3);
        c.body_brick_mat.assign(d->body_brick_mat, d->body_brick_mat + c.n_bricks);
        c.body_pose.assign(d->body_pose, d->body_pose + (size_t)c.n_bodies * 13);
    }
    c.n_chunks = count_chunks(c.desc());
    bool any = false;
    for (const sf_pool_slot &s : S->slots) any |= fits(s, c);
    if (!any) { set_error("no slot of the pool fits a scene of %u bodies, %u bricks", c.n_bodies, c.n_bricks); return SF_ERR_BUDGET; }
    *id = (uint32_t)S->scenes.size();
    S->scenes.push_back(std::move(R));
    return SF_OK;
}

sf_status sf_server_set_scene_state(sf_server *S, uint32_t id, const float *state13, const float *sleep,
                                    const uint8_t *flags) {
    if (!S || !state13 || !sleep || !flags) { set_error("null argument"); return SF_ERR_ARG; }
    if (S->started) { set_error("scene states are set before sf_server_start"); return SF_ERR_STATE; }
    if (id >= S->scenes.size()) { set_error("scene %u is not registered", id); return SF_ERR_ARG; }
    SceneRec &R = *S->scenes[id];
    const uint32_t n = R.sc.n_bodies;
    R.init13.assign(state13, state13 + (size_t)n * 13);
    R.init_sleep.assign(sleep, sleep + n);
    R.init_flags.assign(flags, flags + n);
    return SF_OK;
}

sf_status sf_server_start(sf_server *S) {
    if (!S) return SF_ERR_ARG;
    if (S->started) { set_error("already started"); return SF_ERR_STATE; }
    S->t0 = Clock::now();
    S->started = true;
    if (!S->D.batching) S->threads.emplace_back(plain_worker, S);
    else {
        if (S->pool) S->threads.emplace_back(rigid_worker, S);
        if (S->structs) S->threads.emplace_back(structure_worker, S);
    }
    return SF_OK;
}

sf_status sf_server_submit(sf_server *S, const sf_request *r, uint64_t *ticket) {
    if (!S || !r) { set_error("null argument"); return SF_ERR_ARG; }
    if (r->kind == SF_REQ_STEP) {
        if (!S->pool || r->world >= S->scenes.size()) { set_error("scene %u is not registered", r->world); return SF_ERR_ARG; }
        if (r->nsteps == 0) { set_error("a step request needs nsteps > 0"); return SF_ERR_ARG; }
    } else if (r->kind == SF_REQ_SOLVE) {
        if (!S->structs || r->world >= S->structs->n_struct) { set_error("structure %u does not exist", r->world); return SF_ERR_ARG; }
        if (!(r->omega > 0.0f && r->omega < 2.0f) || !(r->tol > 0.0f) || r->max_sweeps == 0) { set_error("bad solve parameters"); return SF_ERR_ARG; }
        if (r->n_loads && (!r->load_brick || !r->load_value)) { set_error("null load arrays"); return SF_ERR_ARG; }
        for (uint32_t k = 0; k < r->n_loads; k++)
            if (r->load_brick[k] >= S->structs->ns) { set_error("load on static brick %u, which does not exist", r->load_brick[k]); return SF_ERR_ARG; }
    } else { set_error("unknown request kind %u", r->kind); return SF_ERR_ARG; }
    auto q = std::make_unique<Req>();
    q->r = *r;
    if (r->kind == SF_REQ_SOLVE && r->n_loads) {
        q->load_brick.assign(r->load_brick, r->load_brick + r->n_loads);
        q->load_value.assign(r->load_value, r->load_value + r->n_loads);
    }
    q->r.load_brick = nullptr; q->r.load_value = nullptr;
    std::lock_guard<std::mutex> lk(S->mu);
    if (q->r.t_arrival < 0.0) q->r.t_arrival = 0.0;
    q->ticket = S->next_ticket++;
    if (ticket) *ticket = q->ticket;
    S->incoming.emplace(q->r.t_arrival, q.get());
    S->all.push_back(std::move(q));
    S->submitted++;
    S->cv_in.notify_all();
    return SF_OK;
}

sf_status sf_server_poll(sf_server *S, sf_result *out, uint32_t cap, uint32_t *n, uint32_t wait_ms) {
    if (!S || !n || (cap && !out)) { set_error("null argument"); return SF_ERR_ARG; }
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->results.empty() && wait_ms)
        S->cv_out.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !S->results.empty(); });
    uint32_t k = 0;
    while (k < cap && !S->results.empty()) { out[k++] = S->results.front(); S->results.pop_front(); }
    *n = k;
    return SF_OK;
}

sf_status sf_server_drain(sf_server *S, uint32_t timeout_ms) {
    if (!S) return SF_ERR_ARG;
    if (!S->started) { set_error("not started"); return SF_ERR_STATE; }
    std::unique_lock<std::mutex> lk(S->mu);
    const bool ok = S->cv_out.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return S->completed == S->submitted; });
    if (!ok) { set_error("%llu of %llu requests still open", (unsigned long long)(S->submitted - S->completed), (unsigned long long)S->submitted); return SF_ERR_TIMEOUT; }
    return SF_OK;
}

sf_status sf_server_get_stats(sf_server *S, sf_server_stats *out) {
    if (!S || !out) return SF_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->pending = S->submitted - S->completed;
    out->now_s = S->started ? S->now() : 0.0;
    return SF_OK;
}

sf_status sf_server_read_phi64(sf_server *S, double *phi) {
    if (!S || !phi) { set_error("null argument"); return SF_ERR_ARG; }
    if (!S->structs) { set_error("the server has no structures"); return SF_ERR_STATE; }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->started && S->completed != S->submitted) { set_error("requests are still open"); return SF_ERR_STATE; }
    }
    return sf_read_phi64(S->structs, phi);
}

void sf_server_destroy(sf_server *S) {
    if (!S) return;
    S->stop = true;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->cv_in.notify_all();
    }
    for (auto &t : S->threads) if (t.joinable()) t.join();
    for (auto &R : S->scenes) if (R->snap) cudaFreeHost(R->snap);
    if (S->pool) sf_world_destroy(S->pool);
    if (S->structs) sf_world_destroy(S->structs);
    delete S;
}

}  // extern "C"

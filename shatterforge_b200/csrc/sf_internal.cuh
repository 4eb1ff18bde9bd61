// Internal declarations of the B200 physics library: constants, f32 helpers in the reference's evaluation order,
// device buffers and the world object. Every physics kernel is compiled with --fmad=false so each multiply and
// add rounds separately, as the reference's wasm32 f32 code does; together with the evaluation order below this
// makes the device arithmetic op-for-op equal to the reference's.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/sf.h"

namespace sf {

// ---------------------------------------------------------------- constants (src/lib.rs:110-215)
constexpr float S = 0.5f, H = 0.25f, RB = 0.27f, GR = 9.81f, MU = 0.65f, GROUNDK = 4.0f;
constexpr int NX = 640, NY = 136, NZ = 640, CXN = NX / 8, CYN = NY / 8, CZN = NZ / 8, NCT = CXN * CYN * CZN;
constexpr uint32_t HSIZE = 32768;
constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr uint32_t STATIC = 0xFFFFFFFFu;
constexpr uint8_t STEEL = 3, GLASS = 4, SLUG = 6;
constexpr int MAXCOL = 1024;   // sf_params.max_colors at most (default 128)

struct MatTables {
    float mass[9], capv[9], caph[9], tens[9], stiff[9], duct[9];
    float gk[9];       // GROUNDK * STIFF[m], rounded once as the reference computes it
    float eb[9];       // energy that crushes one brick (J), src/lib.rs:178
    float pulv[9];     // share of crushed bricks ground to dust rather than broken loose, src/lib.rs:180
};
void host_mat_tables(MatTables &t);
// each translation unit that reads the tables holds its own copy and uploads it at world creation
static __constant__ MatTables c_mat;
static inline cudaError_t upload_mat_tables(cudaStream_t s) {
    MatTables t;
    host_mat_tables(t);
    return cudaMemcpyToSymbolAsync(c_mat, &t, sizeof t, 0, cudaMemcpyHostToDevice, s);
}

// error bits of the device error word
enum : uint32_t {
    ERR_TIMEOUT = 1u << 0,
    ERR_CAPACITY_CONTACTS = 1u << 1,
    ERR_CAPACITY_COLORS = 1u << 2,
    ERR_VERIFY_COLOR = 1u << 3,
    ERR_JP_ROUNDS = 1u << 4,
    ERR_SOR_NONFINITE = 1u << 5,
    ERR_ISLANDS = 1u << 6,         // a union-find walk or link ran past its bound (corrupt or cyclic parents)
};

// ---------------------------------------------------------------- f32 helpers (src/lib.rs:25-108 order)
struct V3 { float x, y, z; };
__host__ __device__ __forceinline__ V3 v3(float a, float b, float c) { V3 r; r.x = a; r.y = b; r.z = c; return r; }
__host__ __device__ __forceinline__ float minf(float a, float b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ float maxf(float a, float b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ float clampf(float x, float a, float b) { return minf(maxf(x, a), b); }
__host__ __device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ V3 madd(V3 a, V3 b, float s) { return v3(a.x + b.x * s, a.y + b.y * s, a.z + b.z * s); }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float sqrt_rn(float x) { return __fsqrt_rn(x); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float len(V3 a) { return __fsqrt_rn(dot(a, a)); }
__host__ __device__ __forceinline__ float fabs_bits(float x) { return fabsf(x); }
__host__ __device__ __forceinline__ V3 mv(const float *m, V3 v) {
    return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z, m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
__host__ __device__ __forceinline__ void mmul(const float *a, const float *b, float *r) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}
__host__ __device__ __forceinline__ void mtr(const float *a, float *r) {
    r[0] = a[0]; r[1] = a[3]; r[2] = a[6]; r[3] = a[1]; r[4] = a[4]; r[5] = a[7]; r[6] = a[2]; r[7] = a[5]; r[8] = a[8];
}
__host__ __device__ __forceinline__ void q_to_m(float x, float y, float z, float w, float *r) {
    r[0] = 1.0f - 2.0f * (y * y + z * z); r[1] = 2.0f * (x * y - z * w); r[2] = 2.0f * (x * z + y * w);
    r[3] = 2.0f * (x * y + z * w); r[4] = 1.0f - 2.0f * (x * x + z * z); r[5] = 2.0f * (y * z - x * w);
    r[6] = 2.0f * (x * z - y * w); r[7] = 2.0f * (y * z + x * w); r[8] = 1.0f - 2.0f * (x * x + y * y);
}
__host__ __device__ __forceinline__ V3 lat_pos(int x, int y, int z) {
    return v3((float)(x - NX / 2) * S + H, (float)y * S + H, (float)(z - NZ / 2) * S + H);
}
__host__ __device__ __forceinline__ uint32_t hkey(int x, int y, int z) {
    return ((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u) & (HSIZE - 1);
}
__host__ __device__ __forceinline__ uint32_t pair_priority(uint32_t a, uint32_t bp) {
    uint32_t h = a * 0x9E3779B1u + bp * 0x85EBCA6Bu;
    h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
    return h;
}
__host__ __device__ __forceinline__ uint32_t pack_cell(int x, int y, int z) {
    return (uint32_t)x | ((uint32_t)y << 10) | ((uint32_t)z << 18);
}
__host__ __device__ __forceinline__ void unpack_cell(uint32_t c, int &x, int &y, int &z) {
    x = (int)(c & 1023u); y = (int)((c >> 10) & 255u); z = (int)(c >> 18);
}
__host__ __device__ __forceinline__ uint32_t chunk_slot(int x, int y, int z) { return (uint32_t)(((y >> 3) * CZN + (z >> 3)) * CXN + (x >> 3)); }
__host__ __device__ __forceinline__ uint32_t cell_in_chunk(int x, int y, int z) { return (uint32_t)(((y & 7) * 8 + (z & 7)) * 8 + (x & 7)); }
__host__ __device__ __forceinline__ bool inb(int x, int y, int z) { return x >= 0 && y >= 0 && z >= 0 && x < NX && y < NY && z < NZ; }

// ---------------------------------------------------------------- device buffers
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DBuf() { release(); }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    cudaError_t alloc(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        size_t c = count ? count : 1;
        cudaError_t e = cudaMalloc((void **)&p, c * sizeof(T));
        if (e == cudaSuccess) n = c; else p = nullptr;
        return e;
    }
    cudaError_t grow(size_t count) { return count <= n && p ? cudaSuccess : alloc(count + count / 4 + 1024); }
    size_t bytes() const { return n * sizeof(T); }
    // exchange the buffers of two DBufs (ping-pong pairs whose roles a pass swaps)
    void swap(DBuf &o) { T *tp = p; p = o.p; o.p = tp; size_t tn = n; n = o.n; o.n = tn; }
};

// Online autotuner for launch shapes that do not change results (blocks per SM of the persistent kernels: the
// order of work inside a colour or a red-black half-sweep does not change any value). Keyed on a size bucket
// (log2 of the launch's work items); the first launches of a bucket try each candidate twice, timed with CUDA
// events, and the bucket then keeps the fastest.
struct Tuner {
    static constexpr int NB = 40, NC = 4, TRIES = 2;
    int cand[NC] = {1, 2, 3, 4};
    int ncand = 0;
    struct Entry { int best = -1; float sum[NC] = {}; int n[NC] = {}; } e[NB];
    void init(const int *c, int n) { ncand = 0; for (int k = 0; k < n && ncand < NC; k++) if (c[k] > 0) cand[ncand++] = c[k]; }
    static int bucket(uint64_t work) { int b = 0; while (b < NB - 1 && (work >> (b + 1))) b++; return b; }
    // the value to launch with, and the candidate index to record (-1 once the bucket is settled)
    int choose(int b, int &ci) const {
        const Entry &x = e[b];
        ci = -1;
        if (x.best >= 0 || ncand == 0) return ncand ? cand[x.best] : 1;
        for (int k = 0; k < ncand; k++) if (x.n[k] < TRIES) { ci = k; return cand[k]; }
        return cand[0];
    }
    void record(int b, int ci, float ms) {
        Entry &x = e[b];
        if (ci < 0 || x.best >= 0) return;
        x.sum[ci] += ms;
        x.n[ci]++;
        for (int k = 0; k < ncand; k++) if (x.n[k] < TRIES) return;
        int best = 0;
        for (int k = 1; k < ncand; k++) if (x.sum[k] < x.sum[best]) best = k;
        x.best = best;
    }
    int settled(int b) const { return e[b].best >= 0 ? cand[e[b].best] : -1; }
};

// persistent-kernel grid barrier state (bounded spin, see grid_sync)
struct GridBarrier { unsigned count; unsigned gen; };

struct StepState;    // sf_step.cu
struct SorState;     // sf_sor.cu
struct ConnState;    // sf_connect.cu
struct SplitState;   // sf_split.cu
struct DamageState;  // sf_damage.cu
struct BodyLoadState;  // sf_bodyload.cu
uint64_t sor_launches(const SorState *st);
const Tuner *sor_tuner(const SorState *st);
uint64_t sor_graph_launches(const SorState *st);
void sor_reset_launches(SorState *st);

// Device buffers of one structure's load-path solve when the caller supplies every buffer (no allocation inside).
struct SorBuffers {
    const uint32_t *cell, *scene, *ctab;
    const uint8_t *mat;
    const int32_t *sid;
    const uint32_t *nb6;
    const float *bond, *ext;
    double *phi64;
    float *phi;
    double *cphi;
    float *crhs;
    uint32_t *ccode;
    int32_t *csid;
    const int32_t *chunk_nbr, *chunk_sid;
    const uint32_t *work, *active0;
    unsigned long long *resid_buf;
    uint32_t *sweeps;
    double *resid;
    GridBarrier *gb;
    uint32_t *err;
};
cudaError_t sor_solve_on_buffers(const SorBuffers &B, uint32_t n_bricks, uint32_t n_chunks, float omega, float tol,
                                 uint32_t max_sweeps, int sms, cudaStream_t s);
// finalize_brick's links and bonds for bricks of one scene on caller-provided buffers (no allocation inside)
cudaError_t finalize_on_buffers(uint32_t ns, const uint32_t *cell, const uint32_t *scene, const uint8_t *mat,
                                const uint8_t *infill, const int32_t *sid, const uint32_t *ctab, const uint32_t *cpool,
                                uint32_t *nb6, float *bond, float *bmax, cudaStream_t s);

// n_bodies and n_bricks are the scene's capacities; a world created with spare capacity for detached pieces holds
// its bodies in [body_off, body_off + bodies_used) and their bricks in [brick_off, brick_off + bricks_used), the
// rest dead (bodies) or owned by the sentinel body (bricks) until sf_structure_connect takes them.
struct Scene {
    uint32_t static_off, n_static;
    uint32_t body_off, n_bodies;
    uint32_t brick_off, n_bricks;
    uint32_t chunk_off, n_chunks;
    uint32_t bodies_used = 0, bricks_used = 0;
};

// A scene pool keeps fixed-capacity scene slots (the Scene ranges above are the capacities); a slot holds one
// loaded scene or nothing. Bodies past the loaded count are dead, bricks past it belong to the sentinel body.
struct PoolSlot {
    uint32_t bodies = 0, bricks = 0, statics = 0, chunks = 0;   // loaded counts
    bool loaded = false;
};

}  // namespace sf

struct sf_world {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;      // where all device work goes (the caller's, or own_stream)
    cudaStream_t own_stream = nullptr;
    uint64_t launches = 0;              // kernels this world launched (scans and sorts counted in their Work)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    sf_params P{};
    uint32_t n_scenes = 0, ns = 0, nd = 0, nb = 0, n_struct = 0, n_chunks = 0;
    uint32_t frame = 0;
    std::vector<sf::Scene> scenes;
    std::vector<int4> h_sbox;            // per scene: static bricks' lattice bounding box (lo, hi)
    sf::DBuf<int4> sbox;

    // static grid: per scene chunk table (NCT entries, global chunk index + 1) and chunk pool (static id + 1)
    sf::DBuf<uint32_t> ctab, cpool;
    std::vector<uint32_t> h_chunk_cell;  // per chunk: packed lattice origin
    std::vector<uint32_t> h_chunk_scene;
    // static bricks
    sf::DBuf<uint32_t> s_cell, s_scene, s_nb6;
    sf::DBuf<uint8_t> s_mat, s_infill;
    sf::DBuf<int32_t> s_sid;
    sf::DBuf<float> s_bond, s_bmax, s_phi, s_ext, s_stress;
    sf::DBuf<double> s_phi64;        // the solver's potential; s_phi is its f32 copy (the reference's type)
    std::vector<int32_t> h_sid;
    std::vector<uint32_t> h_s_cell;
    // bodies
    sf::DBuf<float4> b_pos, b_q, b_v, b_w, b_vpre, b_wpre;
    sf::DBuf<float> b_rot, b_iil, b_iiw, b_m, b_im, b_rad, b_sleep, b_maxr;
    sf::DBuf<uint8_t> b_alive, b_asleep, b_wake;
    sf::DBuf<uint32_t> b_first, b_count, b_nc, b_scene;
    // body bricks
    sf::DBuf<float4> k_local, k_wpos;
    sf::DBuf<uint32_t> k_body;
    sf::DBuf<uint8_t> k_mat;
    sf::DBuf<int32_t> k_xyz;

    sf::DBuf<float> stage13;     // packed body state for the read/write calls
    sf::DBuf<uint8_t> stage_flags, stage_dirty;
    sf::DBuf<uint32_t> err;      // [0] error bits, [1..] counters
    sf::DBuf<sf::GridBarrier> barrier;

    // body bricks' bonds, in worlds with spare capacity (the ones whose bodies can split): per body brick its six face
    // neighbours in the same body (body-brick ids, NONE = none), four bonds and their capacities as static bricks have;
    // per body: a brick was removed or a bond broke since its last rebuild
    sf::DBuf<uint32_t> k_nb6;
    sf::DBuf<float> k_bond, k_bmax;
    sf::DBuf<uint8_t> b_dirty;
    uint64_t rebuilds = 0;               // rebuild_body calls so far (a draw counter of the lone-brick rule)
    // the debris-body load field (structural's body part, src/lib.rs:1262-1365), in the same worlds: per body brick
    // the frame a contact last supported it, its potential (f64, with the f32 copy the joints read) and its inertial
    // load; per body the velocities of the last frame, the last sweep's residual, the peak load factor and the time
    // its field has been loaded
    sf::DBuf<uint32_t> k_sup;
    sf::DBuf<double> k_phi64;
    sf::DBuf<float> k_phi, k_ext;
    sf::DBuf<float4> b_vlast, b_wlast;
    sf::DBuf<double> b_resid;
    sf::DBuf<float> b_nmax, b_lt;
    sf::BodyLoadState *bodyload = nullptr;
    // connectivity: per structure, set on the GPU when a joint pass fails a joint or crushes a brick (pending walk);
    // structures a full scene could not take are pending on the host
    sf::DBuf<uint8_t> st_conn;
    std::vector<uint8_t> h_conn_retry;
    sf::ConnState *conn = nullptr;
    sf::SplitState *split = nullptr;
    sf::DamageState *damage = nullptr;

    sf::SorState *sor = nullptr;
    sf::StepState *step = nullptr;
    std::vector<sf::PoolSlot> pool;      // non-empty for a scene pool
    uint32_t sentinel = 0xFFFFFFFFu;     // a scene pool's always-dead body
    sf_stats stats{};
};

namespace sf {
// error helpers
void set_error(const char *fmt, ...);
#define SF_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            ::sf::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return SF_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

inline unsigned grid_for(size_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

// scratch for scans and sorts (grows on demand, never shrinks)
struct Work {
    DBuf<uint32_t> scan_a, scan_b, hist;
    uint64_t launches = 0;   // kernels launched by the scans and sorts
};
// exclusive scan of n uint32 values (in place allowed); the total is written to *d_total if non-null
cudaError_t exclusive_scan_u32(const uint32_t *in, uint32_t *out, size_t n, uint32_t *d_total, Work &wk, cudaStream_t s);
// stable LSD radix sort of (key, value) pairs on key bits [0, bits). With in_alt null the result ends in keys/vals
// (the alt buffers, n entries each, are scratch); otherwise it stays where the last pass left it and *in_alt says
// whether that is the alt pair (the caller then swaps the buffers' roles instead of copying back)
cudaError_t radix_sort_u64(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt, uint32_t *vals_alt, size_t n, int bits,
                           Work &wk, cudaStream_t s, bool *in_alt = nullptr);
cudaError_t radix_sort_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt, uint32_t *vals_alt, size_t n, int bits,
                           Work &wk, cudaStream_t s, bool *in_alt = nullptr);

// ---------------------------------------------------------------- bounded grid barrier for persistent kernels
// Every block of a cooperative launch calls it; a wait that outlasts the limit sets ERR_TIMEOUT and returns false
// (the caller then leaves the kernel and the host reports SF_ERR_TIMEOUT). The barrier state must be zeroed before
// each launch that uses it.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr unsigned long long BARRIER_LIMIT_NS = 4000000000ull;   // 4 s
// Every device-side wait in this library goes through bounded_wait: spin until done() holds, for at most limit_ns of
// wall time (and at most 2^30 polls, a backstop should the clock misbehave); on running out, set ERR_TIMEOUT in *err
// and return false. A wait also gives up (returns false) once another wait has set ERR_TIMEOUT, so that waits on work
// that will now never finish end promptly instead of each running out its own limit.
template <class Done>
__device__ __forceinline__ bool bounded_wait(Done done, unsigned long long limit_ns, unsigned *err) {
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    while (!done()) {
        ++spins;
        if ((spins & 255u) == 0) {
            if (globaltimer_ns() - t0 > limit_ns || spins >= (1u << 30)) {
                atomicOr(err, (unsigned)ERR_TIMEOUT);
                return false;
            }
            if (ld_acquire_u32(err) & ERR_TIMEOUT) return false;
        }
        __nanosleep(20);
    }
    return true;
}
// spin while *p == v
__device__ __forceinline__ bool bounded_wait_while_equal(const unsigned *p, unsigned v, unsigned long long limit_ns,
                                                         unsigned *err) {
    return bounded_wait([&] { return ld_acquire_u32(p) != v; }, limit_ns, err);
}
__device__ __forceinline__ bool grid_sync(GridBarrier *gb, unsigned nblocks, unsigned *err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned gen = ld_acquire_u32(&gb->gen);
        __threadfence();
        unsigned arrived = atomicAdd(&gb->count, 1u);
        int ok = 1;
        if (arrived == nblocks - 1) {
            atomicExch(&gb->count, 0u);
            __threadfence();
            atomicAdd(&gb->gen, 1u);
        } else {
            ok = bounded_wait_while_equal(&gb->gen, gen, BARRIER_LIMIT_NS, err) ? 1 : 0;
        }
        __threadfence();
        if (ld_acquire_u32(err) & ERR_TIMEOUT) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

sf_status sor_create(sf_world *w);
void sor_destroy(sf_world *w);
sf_status step_create(sf_world *w);
void step_destroy(sf_world *w);
// update_cache without gravity: rotation, world inverse inertia and brick positions of awake bodies
cudaError_t refresh_poses(sf_world *w);
// the step's active set: a scene marked live steps at the next step even if its bodies were asleep
void step_mark_live(sf_world *w, uint32_t scene);
void step_mark_all_live(sf_world *w);
// brick ids of a scene moved (a rebuild or a detachment): its entries in the last substep's warm-start table no
// longer apply
void step_warm_invalidate(sf_world *w, uint32_t scene);
void step_set_live(sf_world *w, uint32_t scene, bool live);
cudaError_t step_reset_labels(sf_world *w, uint32_t first_body, uint32_t n);
sf_status read_error_word(sf_world *w);
void conn_destroy(sf_world *w);
void split_destroy(sf_world *w);
void damage_destroy(sf_world *w);
void bodyload_destroy(sf_world *w);
// the load-field state of bodies just set up (setup_body, src/lib.rs:845, 882): listed ids (d_list) or base..base+n;
// d_keep (optional, per entry) keeps the body's load time
cudaError_t body_load_setup(sf_world *w, const uint32_t *d_list, uint32_t base, uint32_t n, const uint8_t *d_keep);
// the substep's contacts in list order, for impact damage (sf_damage.cu)
struct DamageIn {
    uint32_t nc;
    const uint32_t *L_a, *L_b, *L_bo, *L_ba, *L_bb, *invperm;
    const float4 *L_p, *S_j, *S_rb;
    Work *wk;
};
cudaError_t damage_substep(sf_world *w, const DamageIn &in, cudaStream_t s);
// plough (src/lib.rs:1493-1550) over the substep's contacts before prep: marks the contacts it switches off in `off`
// (one byte per contact) and sets up the one-brick bodies it knocks loose; *n_loose = how many
struct PloughIn {
    uint32_t nc;
    const uint32_t *L_a, *L_b, *L_bo, *L_bb;
    const float4 *L_p, *L_n;
    uint8_t *off;
    Work *wk;
};
cudaError_t plough_substep(sf_world *w, const PloughIn &in, cudaStream_t s, uint32_t *n_loose);
// setup_body (src/lib.rs:844-891) of bodies base .. base + nb - 1 from their bricks' lattice cells and poses
// (sf_world.cu)
cudaError_t setup_bodies(sf_world *w, uint32_t base, uint32_t nb, const float *d_pose13);
// setup_body of the listed bodies from their bricks' current local offsets, about a parent pose given with its
// cached rotation: pose22 = position 3, quaternion 4, velocity 3, spin 3, rotation 9 (rebuild_body, src/lib.rs:995)
cudaError_t setup_bodies_from_local(sf_world *w, const uint32_t *d_list, uint32_t n, const float *d_pose22);
// finalize_brick's bond rule (src/lib.rs:668-696) between face-adjacent bricks of each body (sf_world.cu)
cudaError_t body_bonds(sf_world *w);

// Union-find over a parent array whose entries only ever point to smaller indices: a walk ends within n hops and a
// link attempt fails only when another thread linked the same root first. The bounds are far beyond both; only a
// corrupt parent array reaches them, which sets ERR_ISLANDS instead of looping.
__device__ __forceinline__ uint32_t uf_find(uint32_t *parent, uint32_t x, uint32_t *err) {
    for (int guard = 0; guard < (1 << 20); guard++) {
        uint32_t p = __ldcg(&parent[x]);
        if (p == x) return x;
        uint32_t gp = __ldcg(&parent[p]);
        if (gp != p) atomicCAS(&parent[x], p, gp);
        x = p;
    }
    atomicOr(err, (unsigned)ERR_ISLANDS);
    return x;
}
__device__ __forceinline__ void uf_union(uint32_t *parent, uint32_t x, uint32_t y, uint32_t *err) {
    for (int it = 0; it < (1 << 16); it++) {
        x = uf_find(parent, x, err);
        y = uf_find(parent, y, err);
        if (x == y) return;
        if (x < y) { uint32_t t = x; x = y; y = t; }
        if (atomicCAS(&parent[x], x, y) == x) return;
    }
    atomicOr(err, (unsigned)ERR_ISLANDS);
}
}  // namespace sf

// The debris-body load field: the body part of `structural` (src/lib.rs:1262-1266, 1282-1365).
//
//   unsupported reset  src/lib.rs:1262-1266  a piece of 8 or more bricks with no supporting contact in the last 10
//                                            frames starts its potentials over
//   inertial loading   src/lib.rs:1288-1304  each brick of a loaded piece carries MASS (n - 1) on top of its weight,
//                                            n = |g - a| / g (capped at 150), a from the piece's change of velocity
//                                            and spin over the frame
//   body sweeps        src/lib.rs:1305-1316  the piece's potential field (conductances scaled by how upright each
//                                            link is, a supporting contact acting as ground) relaxed with omega 1.8:
//                                            at least 2 sweeps, until the residual is below 4e-4, 60 sweeps or the
//                                            frame's budget of 160,000 brick-updates (shared in body order) is spent
//   body joints        src/lib.rs:1340-1360  stress_brick's body branch (ratios against direction-weighted
//                                            capacities, fatigue at the material's DUCT pace, crushes and failures
//                                            that mark the piece for rebuild_body), judged on a settled field or
//                                            during a hard impact
//
// As for the structures, the sweeps are red-black in FP64 (every body-lattice link joins opposite parities); one
// block relaxes one body. The budget is applied exactly: every eligible body first runs to its own stopping point
// from a saved copy of the potentials; the host then walks the bodies in order, and if the budget cut any of them the
// solve reruns from the copy with those caps. The joints of all judged bodies are evaluated in parallel on the
// potentials, and the decisions that change something are applied by one thread in body and brick order, where a
// crush (one budget of 300 a frame, shared with the structures' joint pass before it) removes a brick and so the
// joints after it that touch that brick.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "sf_internal.cuh"

namespace sf {

constexpr int BL_SOR_THREADS = 256, BL_SOR_BIG_THREADS = 1024;
constexpr uint32_t BL_BIG = 2048;   // bricks from which a body's sweeps take the larger block
constexpr uint32_t BL_HUGE = 16384;  // bricks from which a body's sweeps take a cluster of BL_CL blocks
constexpr int BL_CL = 16;
constexpr int64_t BL_BUDGET = 160000;   // brick updates a frame, per scene (src/lib.rs:1305)
constexpr uint8_t BJ_HOLD = 0, BJ_FATIGUE = 1, BJ_FAIL = 2, BJ_CRUSH = 3, BJ_ABSENT = 255;

struct BodyLoadState {
    DBuf<uint32_t> flag;          // per body: a supporting contact in the last 10 frames
    DBuf<uint8_t> loaded;         // per body: body_loaded this frame
    DBuf<float4> acc;             // per body: linear, angular acceleration
    DBuf<uint32_t> nm_bits;       // per body: the largest load factor's bits
    DBuf<uint32_t> elig, nelig;   // bodies whose field is swept this frame, ascending
    DBuf<uint32_t> caps, sweeps, sizes, cut;   // sizes: count and scene per listed body; cut: bodies the budget cut
    DBuf<double> resid_out;
    DBuf<double> phi_save;
    DBuf<uint32_t> scene_body_off;
    DBuf<uint8_t> judged;         // per body: its joints are judged this frame
    DBuf<uint8_t> jlive;
    DBuf<float> jdt;
    DBuf<float> j_ratio, j_bond;  // 3 per body brick (+x, +y, +z)
    DBuf<uint8_t> j_dec;
    DBuf<uint32_t> j_crushed;
    DBuf<uint32_t> cand;          // per body brick: a joint decision changes something
    DBuf<uint32_t> cpos, clist;   // their places, and the list of them ascending
    Work wk;
    DBuf<uint32_t> jl, njl;       // judged bodies, ascending
    DBuf<uint32_t> counters;      // joints, over, failed, crushed, crushes after the pass, largest ratio's bits
    DBuf<uint32_t> maxr_bits;
    bool ready = false;
    bool cluster_ok = false;      // the device can hold a cluster of BL_CL 1,024-thread blocks
};

__device__ __forceinline__ bool body_loaded_d(uint32_t b, const uint8_t *alive, const uint32_t *count,
                                              const uint8_t *asleep, const uint32_t *nc, const uint32_t *first,
                                              const uint8_t *kmat) {
    return alive[b] && count[b] >= 8 && !asleep[b] && nc[b] > 0 && kmat[first[b]] < SLUG;
}

// a brick of a live piece of 8 or more with a supporting contact in the last 10 frames marks its piece supported
__global__ void k_bl_support(uint32_t nd, const uint32_t *kbody, const uint8_t *alive, const uint32_t *count,
                             const uint32_t *sup, uint32_t frame, uint32_t *flag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = kbody[i];
    if (alive[b] && count[b] >= 8 && (uint32_t)(frame - sup[i]) < 10u) flag[b] = 1;
}
// src/lib.rs:1262-1266: an unsupported piece's potentials start over
__global__ void k_bl_reset(uint32_t nd, const uint32_t *kbody, const uint8_t *alive, const uint32_t *count,
                           const uint32_t *flag, double *phi64, float *phi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = kbody[i];
    if (alive[b] && count[b] >= 8 && !flag[b]) { phi64[i] = 0.0; phi[i] = 0.0f; }
}
// src/lib.rs:1289-1295: the frame's acceleration of every live piece, and which pieces are loaded
__global__ void k_bl_accel(uint32_t nb, float idt, const uint8_t *alive, const uint32_t *count, const uint8_t *asleep,
                           const uint32_t *nc, const uint32_t *first, const uint8_t *kmat, const float4 *v,
                           const float4 *w, float4 *vlast, float4 *wlast, float4 *acc, uint8_t *loaded,
                           uint32_t *nm_bits) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    loaded[b] = 0;
    nm_bits[b] = 0;
    if (!alive[b]) return;
    const float4 v4 = v[b], w4 = w[b], vl = vlast[b], wl = wlast[b];
    const V3 al = mul(sub(v3(v4.x, v4.y, v4.z), v3(vl.x, vl.y, vl.z)), idt);
    const V3 aa = mul(sub(v3(w4.x, w4.y, w4.z), v3(wl.x, wl.y, wl.z)), idt);
    vlast[b] = make_float4(v4.x, v4.y, v4.z, 0.0f);
    wlast[b] = make_float4(w4.x, w4.y, w4.z, 0.0f);
    acc[2 * b] = make_float4(al.x, al.y, al.z, 0.0f);
    acc[2 * b + 1] = make_float4(aa.x, aa.y, aa.z, 0.0f);
    loaded[b] = body_loaded_d(b, alive, count, asleep, nc, first, kmat) ? 1 : 0;
}
// src/lib.rs:1296-1303: the effective gravity g - a a brick feels, as a load factor n on its weight
__global__ void k_bl_inertial(uint32_t nd, const uint32_t *kbody, const uint8_t *loaded, const uint8_t *kmat,
                              const float4 *wpos, const float4 *pos, const float4 *acc, float *ext, uint32_t *nm_bits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = kbody[i];
    const uint8_t m = kmat[i];
    if (!loaded[b] || m == 0) return;
    const float4 a4 = acc[2 * b], w4 = acc[2 * b + 1], p4 = wpos[i], pb = pos[b];
    const V3 a = add(v3(a4.x, a4.y, a4.z), cross(v3(w4.x, w4.y, w4.z), sub(v3(p4.x, p4.y, p4.z), v3(pb.x, pb.y, pb.z))));
    const V3 ge = v3(-a.x, -GR - a.y, -a.z);
    const float n = minf(div_rn(len(ge), GR), 150.0f);
    ext[i] = c_mat.mass[m] * (n - 1.0f);
    atomicMax(&nm_bits[b], __float_as_uint(n));
}
__global__ void k_bl_nmax(uint32_t nb, const uint8_t *loaded, const uint32_t *nm_bits, float *nmax) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb && loaded[b]) nmax[b] = __uint_as_float(nm_bits[b]);
}

// src/lib.rs:1306-1309: a loaded piece of at most 60,000 bricks is swept unless its field has settled (residual below
// 2e-4, peak load factor below 1.5), which is swept every fourth frame only (by its id in its scene)
__global__ void k_bl_eligible(uint32_t nb, uint32_t frame, const uint8_t *loaded, const uint32_t *count,
                              const double *resid, const float *nmax, const uint32_t *bscene, const uint32_t *sbo,
                              uint32_t *list, uint32_t *n) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    bool on = false;
    if (b < nb && loaded[b] && count[b] <= 60000u) {
        const uint32_t lb = b - sbo[bscene[b]];
        on = !(resid[b] < (double)2e-4f && nmax[b] < 1.5f && (frame + lb) % 4u != 0u);
    }
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (!m) return;
    const unsigned lane = threadIdx.x & 31u, lead = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == lead) base = atomicAdd(n, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, lead);
    if (on) list[base + __popc(m & ((1u << lane) - 1u))] = b;
}

struct BodySorArgs {
    const uint32_t *first, *count, *kbody, *knb6, *sup;
    const uint8_t *kmat;
    const int32_t *kxyz;
    const float *kbond, *rot, *kext;
    double *phi64;
    uint32_t frame;
};

// sor_brick (src/lib.rs:1005-1026) for a body brick, in FP64 on the f32 coefficients: links to bricks of the same
// body with an intact bond, each conducting min(STIFF) (0.3 + 0.7 |up component of the link's axis|) (cond_w,
// src/lib.rs:1146-1151); a supporting contact in the last 10 frames adds the ground term
__device__ __forceinline__ double body_update(const BodySorArgs &A, uint32_t b, uint32_t i, uint8_t mi, double omega) {
    double sk = 0.0, skp = 0.0;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        const uint32_t j = A.knb6[(size_t)i * 6 + d];
        if (j == NONE) continue;
        const uint8_t mj = A.kmat[j];
        if (mj == 0 || A.kbody[j] != b) continue;
        const int a = d >> 1;
        const float hp = (d & 1) == 0 ? A.kbond[(size_t)i * 4 + a] : A.kbond[(size_t)j * 4 + a];
        if (!(hp > 0.0f)) continue;
        const float kk = minf(c_mat.stiff[mi], c_mat.stiff[mj]);
        const float u = fabsf(A.rot[(size_t)b * 9 + 3 + a]);
        const double k = (double)(kk * (0.3f + 0.7f * u));
        sk += k;
        skp += k * A.phi64[j];
    }
    if ((uint32_t)(A.frame - A.sup[i]) < 10u) sk += (double)c_mat.gk[mi];
    if (sk > 0.0) {
        const double target = ((double)(c_mat.mass[mi] + A.kext[i]) + skp) / sk;
        const double dd = omega * (target - A.phi64[i]);
        A.phi64[i] += dd;
        return fabs(dd);
    }
    return 0.0;
}

// One block per listed body: red-black sweeps of its bricks (parity of the body lattice cell) until, after at least
// 2, the residual max |dphi| / max(phi, 1) is below 4e-4, or 60 sweeps, or its cap. Bodies of BL_BIG bricks or more
// take blocks of 1,024 threads, the rest 256 (the order inside a half-sweep does not change the result).
template <int T>
__global__ void __launch_bounds__(T, 1) k_bl_sor(const uint32_t *list, const uint32_t *caps, BodySorArgs A,
                                              uint32_t *sweeps_out, double *resid_out) {
    __shared__ unsigned long long s_d[T / 32], s_p[T / 32];
    __shared__ int s_stop;
    __shared__ double s_r;
    const uint32_t b = list[blockIdx.x];
    const uint32_t f = A.first[b], c = A.count[b];
    const uint32_t cap = caps ? caps[blockIdx.x] : 60u;
    const double omega = (double)1.8f;
    const unsigned long long one = (unsigned long long)__double_as_longlong(1.0);
    uint32_t done = 0;
    for (uint32_t sweep = 0; sweep < cap; sweep++) {
        unsigned long long md = 0ull;
        for (int colour = 0; colour < 2; colour++) {
            for (uint32_t t = threadIdx.x; t < c; t += blockDim.x) {
                const uint32_t i = f + t;
                const uint8_t mi = A.kmat[i];
                if (mi == 0) continue;
                if (((A.kxyz[3 * i] + A.kxyz[3 * i + 1] + A.kxyz[3 * i + 2]) & 1) != colour) continue;
                md = max(md, (unsigned long long)__double_as_longlong(body_update(A, b, i, mi, omega)));
            }
            __syncthreads();
        }
        unsigned long long mp = one;
        for (uint32_t t = threadIdx.x; t < c; t += blockDim.x) {
            const uint32_t i = f + t;
            if (A.kmat[i] == 0) continue;
            const double p = A.phi64[i];
            if (p > 1.0) mp = max(mp, (unsigned long long)__double_as_longlong(p));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            md = max(md, __shfl_xor_sync(0xffffffffu, md, o));
            mp = max(mp, __shfl_xor_sync(0xffffffffu, mp, o));
        }
        if ((threadIdx.x & 31u) == 0) { s_d[threadIdx.x >> 5] = md; s_p[threadIdx.x >> 5] = mp; }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long dm = 0ull, pm = one;
            for (uint32_t k = 0; k < blockDim.x / 32; k++) { dm = max(dm, s_d[k]); pm = max(pm, s_p[k]); }
            const double r = __longlong_as_double((long long)dm) / __longlong_as_double((long long)pm);
            s_r = r;
            s_stop = (sweep + 1 >= 2 && r < (double)4e-4f) ? 1 : 0;
        }
        __syncthreads();
        done = sweep + 1;
        if (s_stop) break;
    }
    if (threadIdx.x == 0) {
        sweeps_out[blockIdx.x] = done;
        resid_out[blockIdx.x] = done ? s_r : 0.0;
    }
}
// The same sweeps for a body of BL_HUGE bricks or more on a cluster of BL_CL blocks: the blocks share the body's
// bricks (brick t to block t / 1,024 mod BL_CL), a cluster barrier ends each half-sweep's writes, and each block's
// maxima go to its shared memory, from where every block's thread 0 reads all of the cluster's before the next
// sweep (two barriers a sweep; the stop decision is the same everywhere).
__global__ void __launch_bounds__(BL_SOR_BIG_THREADS, 1) k_bl_sor_cluster(const uint32_t *list, const uint32_t *caps,
                                                                       BodySorArgs A, uint32_t *sweeps_out,
                                                                       double *resid_out) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ unsigned long long s_d[BL_SOR_BIG_THREADS / 32], s_p[BL_SOR_BIG_THREADS / 32];
    __shared__ unsigned long long s_red[2][2];
    __shared__ int s_stop;
    __shared__ double s_r;
    const uint32_t rank = cl.block_rank(), slot = blockIdx.x / BL_CL;
    const uint32_t b = list[slot];
    const uint32_t f = A.first[b], c = A.count[b];
    const uint32_t cap = caps ? caps[slot] : 60u;
    const double omega = (double)1.8f;
    const unsigned long long one = (unsigned long long)__double_as_longlong(1.0);
    const uint32_t t0 = rank * BL_SOR_BIG_THREADS + threadIdx.x, stride = BL_CL * BL_SOR_BIG_THREADS;
    uint32_t done = 0;
    for (uint32_t sweep = 0; sweep < cap; sweep++) {
        unsigned long long md = 0ull;
        for (int colour = 0; colour < 2; colour++) {
            for (uint32_t t = t0; t < c; t += stride) {
                const uint32_t i = f + t;
                const uint8_t mi = A.kmat[i];
                if (mi == 0) continue;
                if (((A.kxyz[3 * i] + A.kxyz[3 * i + 1] + A.kxyz[3 * i + 2]) & 1) != colour) continue;
                md = max(md, (unsigned long long)__double_as_longlong(body_update(A, b, i, mi, omega)));
            }
            if (colour == 0) cl.sync();
        }
        unsigned long long mp = one;
        for (uint32_t t = t0; t < c; t += stride) {
            const uint32_t i = f + t;
            if (A.kmat[i] == 0) continue;
            const double p = A.phi64[i];
            if (p > 1.0) mp = max(mp, (unsigned long long)__double_as_longlong(p));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            md = max(md, __shfl_xor_sync(0xffffffffu, md, o));
            mp = max(mp, __shfl_xor_sync(0xffffffffu, mp, o));
        }
        if ((threadIdx.x & 31u) == 0) { s_d[threadIdx.x >> 5] = md; s_p[threadIdx.x >> 5] = mp; }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long dm = 0ull, pm = one;
            for (uint32_t k = 0; k < BL_SOR_BIG_THREADS / 32; k++) { dm = max(dm, s_d[k]); pm = max(pm, s_p[k]); }
            s_red[sweep & 1][0] = dm;
            s_red[sweep & 1][1] = pm;
        }
        cl.sync();   // ends the sweep's writes and publishes the blocks' maxima
        if (threadIdx.x == 0) {
            unsigned long long dm = 0ull, pm = one;
            for (uint32_t r = 0; r < BL_CL; r++) {
                const unsigned long long *q = cl.map_shared_rank(&s_red[sweep & 1][0], r);
                dm = max(dm, q[0]);
                pm = max(pm, q[1]);
            }
            const double rr = __longlong_as_double((long long)dm) / __longlong_as_double((long long)pm);
            s_r = rr;
            s_stop = (sweep + 1 >= 2 && rr < (double)4e-4f) ? 1 : 0;
        }
        __syncthreads();
        done = sweep + 1;
        if (s_stop) break;
    }
    if (rank == 0 && threadIdx.x == 0) {
        sweeps_out[slot] = done;
        resid_out[slot] = done ? s_r : 0.0;
    }
    cl.sync();   // no block leaves while another may still read its shared memory
}
__global__ void k_bl_store(uint32_t n, const uint32_t *list, const double *resid_out, double *resid) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) resid[list[k]] = resid_out[k];
}
// the f32 copy the joints read, for the bricks of the swept bodies
__global__ void k_bl_phi32(uint32_t nd, const uint32_t *kbody, const uint8_t *kmat, const uint8_t *swept,
                           const double *phi64, float *phi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nd && kmat[i] != 0 && swept[kbody[i]]) phi[i] = (float)phi64[i];
}
__global__ void k_bl_sizes(uint32_t n, const uint32_t *list, const uint32_t *count, const uint32_t *bscene,
                           uint32_t *out2) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) { out2[2 * k] = count[list[k]]; out2[2 * k + 1] = bscene[list[k]]; }
}
// the marked bodies' potentials back to the copy taken before the sweeps
__global__ void k_bl_restore(uint32_t nd, const uint32_t *kbody, const uint8_t *mark, const double *saved, double *phi64) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nd && mark[kbody[i]]) phi64[i] = saved[i];
}
__global__ void k_bl_mark(uint32_t n, const uint32_t *list, uint8_t *mark) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) mark[list[k]] = 1;
}

// src/lib.rs:1340-1351, 1363: per loaded piece of at most 60,000 bricks its load time grows; it is judged unless its
// field has settled and it is not its fourth frame; a settled piece is judged with 4 dt; its joints are live once
// loaded for 0.3 s with a residual below 1e-2 (or for 0.6 s), or at once under a peak factor above 2.5. A live piece
// that is not loaded lets its load time run down.
__global__ void k_bl_judge(uint32_t nb, uint32_t frame, float dt, const uint8_t *alive, const uint8_t *loaded,
                           const uint32_t *count, const double *resid, const float *nmax, const uint32_t *bscene,
                           const uint32_t *sbo, float *lt, uint8_t *judged, uint8_t *jlive, float *jdt) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    judged[b] = 0;
    if (!alive[b]) return;
    if (!loaded[b]) { lt[b] = maxf(lt[b] - 2.0f * dt, 0.0f); return; }
    if (count[b] > 60000u) return;
    const float l = lt[b] + dt;
    lt[b] = l;
    const bool settled = resid[b] < (double)2e-4f && nmax[b] < 1.5f;
    const uint32_t lb = b - sbo[bscene[b]];
    if (settled && (frame + lb) % 4u != 0u) return;
    judged[b] = 1;
    jdt[b] = settled ? dt * 4.0f : dt;
    jlive[b] = ((l > 0.3f && (resid[b] < (double)1e-2f || l > 0.6f)) || nmax[b] > 2.5f) ? 1 : 0;
}

struct BodyJointArgs {
    const uint32_t *kbody, *knb6;
    const uint8_t *kmat, *judged, *jlive;
    const float *kbond, *kbmax, *kphi, *rot, *jdt;
    float *ratio, *bond_after;
    uint8_t *dec;
    uint32_t *crushed, *cand;
};

// stress_brick's body branch (src/lib.rs:1153-1211) for every joint of a judged body's brick, evaluated as if
// nothing before it failed; the sequential pass below applies them in the reference's order
__global__ void k_bl_joint_eval(uint32_t nd, BodyJointArgs A) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = A.kbody[i];
    const uint8_t mi = A.kmat[i];
    const bool on = A.judged[b] && mi != 0;
    uint32_t flag = 0;
    for (int a = 0; a < 3; a++) {
        const size_t o = (size_t)i * 3 + a;
        uint8_t dec = BJ_ABSENT;
        float r = 0.0f, after = 0.0f;
        uint32_t kc = NONE;
        const uint32_t j = on ? A.knb6[(size_t)i * 6 + 2 * a] : NONE;
        if (j != NONE && A.kmat[j] != 0 && A.kbody[j] == b) {
            const float hp = A.kbond[(size_t)i * 4 + a];
            if (hp > 0.0f) {
                const uint8_t mj = A.kmat[j];
                const float u = A.rot[(size_t)b * 9 + 3 + a];
                const float au = fabsf(u);
                const float cw = minf(c_mat.stiff[mi], c_mat.stiff[mj]) * (0.3f + 0.7f * au);
                const float f = cw * (A.kphi[i] - A.kphi[j]);
                const float up = f > 0.0f ? maxf(u, 0.0f) : maxf(-u, 0.0f);
                const float tens = minf(c_mat.tens[mi], c_mat.tens[mj]);
                const float capm = 1.0f - (1.0f - tens) * up;
                const float cv = minf(c_mat.capv[mi], c_mat.capv[mj]), ch = minf(c_mat.caph[mi], c_mat.caph[mj]);
                const float lat = a == 1 ? cv : ch;
                const float hpw = div_rn(hp * (cv * au + ch * (1.0f - au)), maxf(lat, 1.0f));
                r = div_rn(fabsf(f), hpw * capm);
                dec = BJ_HOLD;
                after = hp;
                if (A.jlive[b] && r > 1.0f) {
                    const float nhp = hp - hp * A.jdt[b] * c_mat.duct[mi] * minf(r - 0.85f, 40.0f);
                    if (nhp < A.kbmax[(size_t)i * 4 + a] * 0.08f) {
                        if (up == 0.0f && au > 0.5f) { dec = BJ_CRUSH; kc = c_mat.capv[mj] < c_mat.capv[mi] ? j : i; }
                        else { dec = BJ_FAIL; after = 0.0f; }
                    } else { dec = BJ_FATIGUE; after = nhp; }
                    flag = 1;
                }
            }
        }
        A.ratio[o] = r; A.bond_after[o] = after; A.dec[o] = dec; A.crushed[o] = kc;
    }
    A.cand[i] = flag;
}

__device__ __forceinline__ bool bjoint_later(uint32_t i2, int a2, uint32_t i, int a) { return i2 > i || (i2 == i && a2 > a); }

// The decisions in the reference's order: bodies ascending, each body's bricks in list order (its slots), each
// brick's +x, +y, +z joint. A crush (while the frame's budget of 300 lasts, else a failure) removes the weaker brick
// and ends that brick's pass; later joints touching the removed brick disappear.
__global__ void k_bl_joint_apply(const uint32_t *clist, const uint32_t *ncand_p, const uint32_t *kbody,
                                 uint32_t crush_used, const uint32_t *knb6, uint8_t *kmat, float *kbond, uint8_t *dec,
                                 const float *bond_after, const uint32_t *crushed, uint8_t *dirty, uint32_t *counters) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t crush_n = crush_used;
    const uint32_t n = *ncand_p;
    // the bricks with a joint decision that changes something, ascending: bodies' brick ranges ascend with their ids,
    // so this is body order and, in each body, list order
    for (uint32_t q = 0; q < n; q++) {
        const uint32_t i = clist[q], b = kbody[i];
        for (int a = 0; a < 3; a++) {
            const size_t o = (size_t)i * 3 + a;
            uint8_t d = dec[o];
            if (d == BJ_ABSENT || d == BJ_HOLD) continue;
            if (kmat[i] == 0) { dec[o] = BJ_ABSENT; continue; }
            if (d == BJ_CRUSH) {
                if (crush_n >= 300) { d = BJ_FAIL; dec[o] = BJ_FAIL; }
                else {
                    crush_n++;
                    const uint32_t k = crushed[o];
                    kmat[k] = 0;
                    dirty[b] = 1;
                    for (int a2 = a + 1; a2 < 3; a2++) dec[(size_t)i * 3 + a2] = BJ_ABSENT;
                    if (k > i) for (int a2 = 0; a2 < 3; a2++) dec[(size_t)k * 3 + a2] = BJ_ABSENT;
                    for (int a2 = 0; a2 < 3; a2++) {
                        const uint32_t i2 = knb6[(size_t)k * 6 + a2 * 2 + 1];
                        if (i2 != NONE && bjoint_later(i2, a2, i, a)) dec[(size_t)i2 * 3 + a2] = BJ_ABSENT;
                    }
                    break;
                }
            }
            if (d == BJ_FAIL) { kbond[(size_t)i * 4 + a] = 0.0f; dirty[b] = 1; }
            else kbond[(size_t)i * 4 + a] = bond_after[o];
        }
    }
    counters[4] = crush_n;
}
__global__ void k_bl_cand_list(uint32_t nd, const uint32_t *cand, const uint32_t *cpos, uint32_t *clist) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nd && cand[i]) clist[cpos[i]] = i;
}

// per judged body brick: its joints that were evaluated (not absent) counted, and the body's largest ratio
__global__ void k_bl_joint_tally(uint32_t nd, const uint32_t *kbody, const uint8_t *judged, const uint8_t *dec,
                                 const float *ratio, uint32_t *maxr_bits, uint32_t *counters) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = kbody[i];
    if (!judged[b]) return;
    uint32_t nj = 0, over = 0, fail = 0, crush = 0;
    float mr = 0.0f;
    for (int a = 0; a < 3; a++) {
        const size_t o = (size_t)i * 3 + a;
        const uint8_t d = dec[o];
        if (d == BJ_ABSENT) continue;
        const float r = ratio[o];
        nj++;
        if (r > 1.0f) over++;
        if (d == BJ_FAIL) fail++;
        if (d == BJ_CRUSH) crush++;
        mr = maxf(mr, r);
    }
    if (nj) {
        atomicAdd(&counters[0], nj);
        if (over) atomicAdd(&counters[1], over);
        if (fail) atomicAdd(&counters[2], fail);
        if (crush) atomicAdd(&counters[3], crush);
        atomicMax(&maxr_bits[b], __float_as_uint(mr));
        atomicMax(&counters[5], __float_as_uint(mr));
    }
}
__global__ void k_bl_maxr(uint32_t nb, const uint8_t *judged, const uint32_t *maxr_bits, float *maxr) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb && judged[b]) maxr[b] = __uint_as_float(maxr_bits[b]);
}

__global__ void k_bl_collect(uint32_t nb, const uint8_t *judged, uint32_t *list, uint32_t *n) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = b < nb && judged[b];
    const unsigned m = __ballot_sync(0xffffffffu, on);
    if (!m) return;
    const unsigned lane = threadIdx.x & 31u, lead = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == lead) base = atomicAdd(n, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, lead);
    if (on) list[base + __popc(m & ((1u << lane) - 1u))] = b;
}

// after setup_body (src/lib.rs:845, 882): a new field's residual and peak factor start over, its load time too unless
// kept (rebuild_body's first piece keeps it, src/lib.rs:998), and the last frame's velocities are the new ones
__global__ void k_bl_setup(uint32_t n, uint32_t base, const uint32_t *list, const uint8_t *keep, const float4 *v,
                           const float4 *w, float4 *vlast, float4 *wlast, double *resid, float *nmax, float *lt) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t b = list ? list[k] : base + k;
    vlast[b] = v[b]; wlast[b] = w[b];
    resid[b] = 1.0; nmax[b] = 1.0f;
    if (!(keep && keep[k])) lt[b] = 0.0f;
}
cudaError_t body_load_setup(sf_world *w, const uint32_t *d_list, uint32_t base, uint32_t n, const uint8_t *d_keep) {
    if (!w->b_vlast.p || n == 0) return cudaSuccess;
    k_bl_setup<<<grid_for(n, 256), 256, 0, w->stream>>>(n, base, d_list, d_keep, w->b_v.p, w->b_w.p, w->b_vlast.p,
                                                       w->b_wlast.p, w->b_resid.p, w->b_nmax.p, w->b_lt.p);
    w->launches++;
    return cudaGetLastError();
}

void bodyload_destroy(sf_world *w) {
    delete w->bodyload;
    w->bodyload = nullptr;
}

static sf_status bodies_frame_impl(sf_world *w, float dt, uint32_t crush_used, sf_bodies_report *report) {
    const auto t0 = std::chrono::steady_clock::now();
    sf_bodies_report rep{};
    cudaStream_t st = w->stream;
    if (!w->bodyload) w->bodyload = new BodyLoadState();
    BodyLoadState &B = *w->bodyload;
    const uint32_t nb = w->nb, nd = w->nd, frame = w->frame;
    if (nb == 0 || nd == 0) { if (report) *report = rep; return SF_OK; }
    if (!B.ready) {
        SF_CUDA(upload_mat_tables(st));
        std::vector<uint32_t> sbo(w->n_scenes);
        for (uint32_t q = 0; q < w->n_scenes; q++) sbo[q] = w->scenes[q].body_off;
        SF_CUDA(B.scene_body_off.alloc(std::max<uint32_t>(w->n_scenes, 1)));
        SF_CUDA(cudaMemcpyAsync(B.scene_body_off.p, sbo.data(), sbo.size() * 4, cudaMemcpyHostToDevice, st));
        SF_CUDA(B.flag.alloc(nb)); SF_CUDA(B.loaded.alloc(nb)); SF_CUDA(B.acc.alloc((size_t)nb * 2));
        SF_CUDA(B.nm_bits.alloc(nb)); SF_CUDA(B.elig.alloc(nb)); SF_CUDA(B.nelig.alloc(2));
        SF_CUDA(B.caps.alloc(nb)); SF_CUDA(B.sweeps.alloc(nb)); SF_CUDA(B.sizes.alloc((size_t)nb * 2)); SF_CUDA(B.cut.alloc(nb)); SF_CUDA(B.resid_out.alloc(nb));
        SF_CUDA(B.phi_save.alloc(nd)); SF_CUDA(B.judged.alloc(nb)); SF_CUDA(B.jlive.alloc(nb)); SF_CUDA(B.jdt.alloc(nb));
        SF_CUDA(B.j_ratio.alloc((size_t)nd * 3)); SF_CUDA(B.j_bond.alloc((size_t)nd * 3)); SF_CUDA(B.j_dec.alloc((size_t)nd * 3));
        SF_CUDA(B.j_crushed.alloc((size_t)nd * 3)); SF_CUDA(B.cand.alloc(nd)); SF_CUDA(B.cpos.alloc(nd)); SF_CUDA(B.clist.alloc(nd)); SF_CUDA(B.jl.alloc(nb)); SF_CUDA(B.njl.alloc(2));
        SF_CUDA(B.counters.alloc(8)); SF_CUDA(B.maxr_bits.alloc(nb));
        {
            SF_CUDA(cudaFuncSetAttribute(k_bl_sor_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cudaLaunchConfig_t c = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = BL_CL; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
            c.gridDim = dim3(BL_CL);
            c.blockDim = dim3(BL_SOR_BIG_THREADS);
            c.attrs = at;
            c.numAttrs = 1;
            int ncl = 0;
            if (cudaOccupancyMaxActiveClusters(&ncl, k_bl_sor_cluster, &c) != cudaSuccess) { ncl = 0; cudaGetLastError(); }
            B.cluster_ok = ncl > 0;
        }
        B.ready = true;
    }
    // the poses after the last integrate (update_cache before structural, src/lib.rs:3654)
    SF_CUDA(refresh_poses(w));
    const unsigned gd = grid_for(nd, 256), gb = grid_for(nb, 256);
    SF_CUDA(cudaMemsetAsync(B.flag.p, 0, (size_t)nb * 4, st));
    k_bl_support<<<gd, 256, 0, st>>>(nd, w->k_body.p, w->b_alive.p, w->b_count.p, w->k_sup.p, frame, B.flag.p);
    k_bl_reset<<<gd, 256, 0, st>>>(nd, w->k_body.p, w->b_alive.p, w->b_count.p, B.flag.p, w->k_phi64.p, w->k_phi.p);
    const float idt = 1.0f / std::max(dt, 1e-3f);
    k_bl_accel<<<gb, 256, 0, st>>>(nb, idt, w->b_alive.p, w->b_count.p, w->b_asleep.p, w->b_nc.p, w->b_first.p,
                                   w->k_mat.p, w->b_v.p, w->b_w.p, w->b_vlast.p, w->b_wlast.p, B.acc.p, B.loaded.p,
                                   B.nm_bits.p);
    k_bl_inertial<<<gd, 256, 0, st>>>(nd, w->k_body.p, B.loaded.p, w->k_mat.p, w->k_wpos.p, w->b_pos.p, B.acc.p,
                                      w->k_ext.p, B.nm_bits.p);
    k_bl_nmax<<<gb, 256, 0, st>>>(nb, B.loaded.p, B.nm_bits.p, w->b_nmax.p);
    SF_CUDA(cudaMemsetAsync(B.nelig.p, 0, 8, st));
    k_bl_eligible<<<gb, 256, 0, st>>>(nb, frame, B.loaded.p, w->b_count.p, w->b_resid.p, w->b_nmax.p, w->b_scene.p,
                                      B.scene_body_off.p, B.elig.p, B.nelig.p);
    w->launches += 6;
    SF_CUDA(cudaGetLastError());
    uint32_t ne = 0;
    SF_CUDA(cudaMemcpyAsync(&ne, B.nelig.p, 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    // ---- the swept bodies: their stopping points, then the budget in body order, scene by scene
    SF_CUDA(cudaMemsetAsync(B.judged.p, 0, nb, st));   // the swept mark here; the judged mark below
    if (ne) {
        std::vector<uint32_t> list(ne);
        SF_CUDA(cudaMemcpyAsync(list.data(), B.elig.p, (size_t)ne * 4, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaStreamSynchronize(st));
        std::sort(list.begin(), list.end());
        SF_CUDA(cudaMemcpyAsync(B.elig.p, list.data(), (size_t)ne * 4, cudaMemcpyHostToDevice, st));
        // sizes (bd_count, the budget's unit) and scenes of the listed bodies
        k_bl_sizes<<<grid_for(ne, 256), 256, 0, st>>>(ne, B.elig.p, w->b_count.p, w->b_scene.p, B.sizes.p);
        std::vector<uint32_t> sz((size_t)ne * 2);
        SF_CUDA(cudaMemcpyAsync(sz.data(), B.sizes.p, (size_t)ne * 8, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaStreamSynchronize(st));
        BodySorArgs A;
        A.first = w->b_first.p; A.count = w->b_count.p; A.kbody = w->k_body.p; A.knb6 = w->k_nb6.p; A.sup = w->k_sup.p;
        A.kmat = w->k_mat.p; A.kxyz = w->k_xyz.p; A.kbond = w->k_bond.p; A.rot = w->b_rot.p; A.kext = w->k_ext.p;
        A.phi64 = w->k_phi64.p; A.frame = frame;
        // the sweeps of listed bodies (ids, caps, sizes in body order): the small bodies' blocks first, then the big
        // ones'; the residuals stored; returns the sweeps each ran, in body order
        std::vector<uint32_t> dl, dc, pos_of;
        auto run_sor = [&](const std::vector<uint32_t> &ids, const std::vector<uint32_t> &cp,
                           const std::vector<uint32_t> &size, std::vector<uint32_t> &done) -> cudaError_t {
            const uint32_t n = (uint32_t)ids.size();
            // three classes in the device list: small bodies, big ones (one 1,024-thread block), huge ones (a cluster)
            auto cls = [&](uint32_t x) { return x < BL_BIG ? 0 : (x < BL_HUGE || !B.cluster_ok) ? 1 : 2; };
            dl.clear(); dc.clear(); pos_of.assign(n, 0);
            uint32_t nk[3] = {0, 0, 0};
            for (int k3 = 0; k3 < 3; k3++)
                for (uint32_t k = 0; k < n; k++)
                    if (cls(size[k]) == k3) { pos_of[k] = (uint32_t)dl.size(); dl.push_back(ids[k]); dc.push_back(cp[k]); nk[k3]++; }
            cudaError_t e;
            if ((e = cudaMemcpyAsync(B.cut.p, dl.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
            if ((e = cudaMemcpyAsync(B.caps.p, dc.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
            if (nk[0])
                k_bl_sor<BL_SOR_THREADS><<<nk[0], BL_SOR_THREADS, 0, st>>>(B.cut.p, B.caps.p, A, B.sweeps.p, B.resid_out.p);
            const uint32_t o1 = nk[0], o2 = nk[0] + nk[1];
            if (nk[1])
                k_bl_sor<BL_SOR_BIG_THREADS><<<nk[1], BL_SOR_BIG_THREADS, 0, st>>>(B.cut.p + o1, B.caps.p + o1, A,
                                                                                 B.sweeps.p + o1, B.resid_out.p + o1);
            if (nk[2]) {
                cudaLaunchConfig_t cfg = {};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = BL_CL; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
                cfg.gridDim = dim3(nk[2] * BL_CL);
                cfg.blockDim = dim3(BL_SOR_BIG_THREADS);
                cfg.stream = st;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                if ((e = cudaLaunchKernelEx(&cfg, k_bl_sor_cluster, (const uint32_t *)(B.cut.p + o2),
                                            (const uint32_t *)(B.caps.p + o2), A, B.sweeps.p + o2,
                                            B.resid_out.p + o2)) != cudaSuccess) return e;
            }
            k_bl_store<<<grid_for(n, 256), 256, 0, st>>>(n, B.cut.p, B.resid_out.p, w->b_resid.p);
            w->launches += 1 + (nk[0] ? 1 : 0) + (nk[1] ? 1 : 0) + (nk[2] ? 1 : 0);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            std::vector<uint32_t> sw(n);
            if ((e = cudaMemcpyAsync(sw.data(), B.sweeps.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
            done.assign(n, 0);
            for (uint32_t k = 0; k < n; k++) done[k] = sw[pos_of[k]];
            return cudaSuccess;
        };
        // no body can sweep more than the scene's whole budget allows it: the first pass stops there
        std::vector<uint32_t> cap_a(ne), caps(ne), nat, size_of(ne), cut_list, cut_caps, cut_size, cut_done;
        for (uint32_t k = 0; k < ne; k++) {
            const int64_t size = sz[2 * k];
            size_of[k] = sz[2 * k];
            cap_a[k] = (uint32_t)std::min<int64_t>(60, std::max<int64_t>(2, (BL_BUDGET + size - 1) / size));
        }
        SF_CUDA(cudaMemcpyAsync(B.phi_save.p, w->k_phi64.p, (size_t)nd * 8, cudaMemcpyDeviceToDevice, st));
        SF_CUDA(run_sor(list, cap_a, size_of, nat));
        // the budget in body order: a body stops at the first n >= 2 after which the budget is spent
        int64_t budget = BL_BUDGET;
        uint32_t scene = NONE;
        for (uint32_t k = 0; k < ne; k++) {
            if (sz[2 * k + 1] != scene) { scene = sz[2 * k + 1]; budget = BL_BUDGET; }
            const int64_t size = sz[2 * k];
            const int64_t need = budget <= 0 ? 2 : std::max<int64_t>(2, (budget + size - 1) / size);
            caps[k] = (uint32_t)std::min<int64_t>(nat[k], need);
            if (caps[k] < nat[k]) { cut_list.push_back(list[k]); cut_caps.push_back(caps[k]); cut_size.push_back(sz[2 * k]); }
            budget -= (int64_t)caps[k] * size;
            rep.sweeps += caps[k];
            rep.brick_updates += (uint64_t)caps[k] * (uint64_t)size;
        }
        // the bodies the budget cut start again from the saved potentials with their caps
        const uint32_t nc = (uint32_t)cut_list.size();
        if (nc) {
            SF_CUDA(cudaMemcpyAsync(B.cut.p, cut_list.data(), (size_t)nc * 4, cudaMemcpyHostToDevice, st));
            k_bl_mark<<<grid_for(nc, 256), 256, 0, st>>>(nc, B.cut.p, B.judged.p);
            k_bl_restore<<<gd, 256, 0, st>>>(nd, w->k_body.p, B.judged.p, B.phi_save.p, w->k_phi64.p);
            w->launches += 2;
            SF_CUDA(run_sor(cut_list, cut_caps, cut_size, cut_done));
        }
        k_bl_mark<<<grid_for(ne, 256), 256, 0, st>>>(ne, B.elig.p, B.judged.p);
        k_bl_phi32<<<gd, 256, 0, st>>>(nd, w->k_body.p, w->k_mat.p, B.judged.p, w->k_phi64.p, w->k_phi.p);
        w->launches += 2;
        SF_CUDA(cudaGetLastError());
        rep.bodies = ne;
        SF_CUDA(cudaStreamSynchronize(st));   // the host vectors are copy sources
    }
    // ---- the joints of the judged bodies
    k_bl_judge<<<gb, 256, 0, st>>>(nb, frame, dt, w->b_alive.p, B.loaded.p, w->b_count.p, w->b_resid.p, w->b_nmax.p,
                                   w->b_scene.p, B.scene_body_off.p, w->b_lt.p, B.judged.p, B.jlive.p, B.jdt.p);
    BodyJointArgs J;
    J.kbody = w->k_body.p; J.knb6 = w->k_nb6.p; J.kmat = w->k_mat.p; J.judged = B.judged.p; J.jlive = B.jlive.p;
    J.kbond = w->k_bond.p; J.kbmax = w->k_bmax.p; J.kphi = w->k_phi.p; J.rot = w->b_rot.p; J.jdt = B.jdt.p;
    J.ratio = B.j_ratio.p; J.bond_after = B.j_bond.p; J.dec = B.j_dec.p; J.crushed = B.j_crushed.p; J.cand = B.cand.p;
    k_bl_joint_eval<<<gd, 256, 0, st>>>(nd, J);
    SF_CUDA(cudaMemsetAsync(B.njl.p, 0, 8, st));
    w->launches += 2;
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaMemsetAsync(B.counters.p, 0, B.counters.bytes(), st));
    SF_CUDA(cudaMemsetAsync(B.maxr_bits.p, 0, (size_t)nb * 4, st));
    k_bl_collect<<<gb, 256, 0, st>>>(nb, B.judged.p, B.jl.p, B.njl.p);
    uint32_t nj = 0;
    SF_CUDA(cudaMemcpyAsync(&nj, B.njl.p, 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    if (nj) {
        // the bricks whose decisions change something, ascending, for the ordered pass
        SF_CUDA(exclusive_scan_u32(B.cand.p, B.cpos.p, nd, B.njl.p + 1, B.wk, st));
        k_bl_cand_list<<<gd, 256, 0, st>>>(nd, B.cand.p, B.cpos.p, B.clist.p);
        k_bl_joint_apply<<<1, 32, 0, st>>>(B.clist.p, B.njl.p + 1, w->k_body.p, crush_used, w->k_nb6.p, w->k_mat.p,
                                           w->k_bond.p, B.j_dec.p, B.j_bond.p, B.j_crushed.p, w->b_dirty.p,
                                           B.counters.p);
        k_bl_joint_tally<<<gd, 256, 0, st>>>(nd, w->k_body.p, B.judged.p, B.j_dec.p, B.j_ratio.p, B.maxr_bits.p,
                                             B.counters.p);
        k_bl_maxr<<<gb, 256, 0, st>>>(nb, B.judged.p, B.maxr_bits.p, w->b_maxr.p);
        w->launches += 4;
        SF_CUDA(cudaGetLastError());
        uint32_t c[8];
        SF_CUDA(cudaMemcpyAsync(c, B.counters.p, sizeof c, cudaMemcpyDeviceToHost, st));
        SF_CUDA(cudaStreamSynchronize(st));
        rep.joints = c[0]; rep.over = c[1]; rep.failed = c[2]; rep.crushed = c[3]; rep.judged = nj;
        rep.crushes_used = c[4];
        std::memcpy(&rep.max_ratio, &c[5], 4);
    } else {
        rep.crushes_used = crush_used;
    }
    step_mark_all_live(w);
    rep.ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (report) *report = rep;
    return read_error_word(w);
}

}  // namespace sf

using namespace sf;

extern "C" {

sf_status sf_bodies_frame(sf_world *w, float dt, uint32_t crushes_used, sf_bodies_report *report) {
    if (!w) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->k_phi64.p) { set_error("bodies carry load fields only in a world created with spare capacity"); return SF_ERR_STATE; }
    if (!(dt >= 0.0f)) { set_error("dt %g", (double)dt); return SF_ERR_ARG; }
    return bodies_frame_impl(w, dt, crushes_used, report);
}

sf_status sf_read_body_fields(sf_world *w, double *phi64, float *ext, double *resid, float *nmax, float *lt, float *maxr) {
    if (!w) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->k_phi64.p) { set_error("bodies carry load fields only in a world created with spare capacity"); return SF_ERR_STATE; }
    cudaStream_t st = w->stream;
    if (phi64) SF_CUDA(cudaMemcpyAsync(phi64, w->k_phi64.p, (size_t)w->nd * 8, cudaMemcpyDeviceToHost, st));
    if (ext) SF_CUDA(cudaMemcpyAsync(ext, w->k_ext.p, (size_t)w->nd * 4, cudaMemcpyDeviceToHost, st));
    if (resid) SF_CUDA(cudaMemcpyAsync(resid, w->b_resid.p, (size_t)w->nb * 8, cudaMemcpyDeviceToHost, st));
    if (nmax) SF_CUDA(cudaMemcpyAsync(nmax, w->b_nmax.p, (size_t)w->nb * 4, cudaMemcpyDeviceToHost, st));
    if (lt) SF_CUDA(cudaMemcpyAsync(lt, w->b_lt.p, (size_t)w->nb * 4, cudaMemcpyDeviceToHost, st));
    if (maxr) SF_CUDA(cudaMemcpyAsync(maxr, w->b_maxr.p, (size_t)w->nb * 4, cudaMemcpyDeviceToHost, st));
    SF_CUDA(cudaStreamSynchronize(st));
    return SF_OK;
}

}  // extern "C"

// World lifecycle: validation, the sparse chunk grid, brick and body set-up on the device, and the read-outs.
//
// Set-up kernels follow the reference op for op:
//   k_finalize_bricks  finalize_brick's neighbour links and bond capacities (src/lib.rs:646-690)
//   k_setup_bodies     setup_body's mass, centre, inertia, radius and local offsets (src/lib.rs:844-891)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "sf_internal.cuh"

using namespace sf;

namespace sf {

__device__ __forceinline__ uint32_t grid_get(const uint32_t *ctab, const uint32_t *cpool, uint32_t scene, int x, int y, int z) {
    if (!inb(x, y, z)) return 0;
    uint32_t t = ctab[(size_t)scene * NCT + chunk_slot(x, y, z)];
    if (t == 0) return 0;
    return cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
}

// static bricks base .. base + ns - 1
__global__ void k_finalize_bricks(uint32_t ns, uint32_t base, const uint32_t *cell, const uint32_t *scene, const uint8_t *mat,
                                  const uint8_t *infill, const int32_t *sid, const uint32_t *ctab, const uint32_t *cpool,
                                  uint32_t *nb6, float *bond, float *bmax) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ns) return;
    const uint32_t i = base + t;
    int x, y, z;
    unpack_cell(cell[i], x, y, z);
    uint32_t sc = scene[i];
    const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    uint32_t nb[6];
#pragma unroll
    for (int d = 0; d < 6; d++) {
        uint32_t g = grid_get(ctab, cpool, sc, x + D[d][0], y + D[d][1], z + D[d][2]);
        nb[d] = g == 0 ? NONE : g - 1;
        nb6[(size_t)i * 6 + d] = nb[d];
    }
    uint8_t mi = mat[i];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        uint32_t j = nb[a * 2];
        float c = 0.0f;
        if (j != NONE) {
            bool gap = infill[i] != infill[j] && (a != 1 || infill[i] == 1);
            if (!gap && mat[j] != 0 && sid[j] == sid[i] && mi != 0) {
                uint8_t mj = mat[j];
                float ca = a == 1 ? c_mat.capv[mi] : c_mat.caph[mi];
                float cb = a == 1 ? c_mat.capv[mj] : c_mat.caph[mj];
                c = minf(ca, cb);
            }
        }
        bond[(size_t)i * 4 + a] = c;
        bmax[(size_t)i * 4 + a] = c;
    }
    float f = (y == 0 && mi != 0) ? c_mat.capv[mi] * 2.0f : 0.0f;
    bond[(size_t)i * 4 + 3] = f;
    bmax[(size_t)i * 4 + 3] = f;
}

// setup_body (src/lib.rs:844-891) for bodies base .. base + nb - 1 (or list[0 .. nb - 1]), their parent poses at
// pose[0 ..], `stride` floats each. Stride 13: the bricks' positions are their lattice cells' centres and the rotation
// follows from the quaternion (a body set up from a description or a detached piece). Stride 22: the positions are
// the bricks' current local offsets and the rotation is given after the 13 (rebuild_body passes the parent's cached
// rotation, src/lib.rs:968, 995). The mass, centre and inertia sums must round in the reference's order (its bricks
// in list order): a body of fewer than SETUP_BIG bricks is summed by one thread; a larger one by a block whose
// threads form each brick's terms in parallel, tile by tile, while one thread adds them up in order.
constexpr uint32_t SETUP_BIG = 512;
constexpr int SETUP_T = 256;
struct SetupArgs {
    uint32_t nb, base;
    const uint32_t *list, *first, *count;
    const int32_t *xyz;
    const uint8_t *kmat;
    const float *pose;
    uint32_t stride;
    float4 *local, *wpos;
    uint32_t *kbody;
    float4 *pos, *q, *v, *w;
    float *rot, *iil, *iiw, *m, *im, *rad, *sleep, *maxr;
    uint8_t *alive, *asleep, *wake;
};
__device__ __forceinline__ V3 setup_brick_pos(const SetupArgs &A, uint32_t i) {
    if (A.stride == 22) { const float4 l = A.local[i]; return v3(l.x, l.y, l.z); }
    return lat_pos(A.xyz[3 * i], A.xyz[3 * i + 1], A.xyz[3 * i + 2]);
}
// a spare body (capacity for detached pieces) or the sentinel: dead, at rest, finite
__device__ void setup_dead(const SetupArgs &A, uint32_t b) {
    A.pos[b] = make_float4(0.0f, 0.0f, 0.0f, 0.0f); A.q[b] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    A.v[b] = make_float4(0.0f, 0.0f, 0.0f, 0.0f); A.w[b] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int k = 0; k < 9; k++) {
        A.rot[(size_t)b * 9 + k] = (k % 4 == 0) ? 1.0f : 0.0f;
        A.iil[(size_t)b * 9 + k] = 0.0f; A.iiw[(size_t)b * 9 + k] = 0.0f;
    }
    A.m[b] = 0.0f; A.im[b] = 0.0f; A.rad[b] = 0.0f; A.sleep[b] = 0.0f; A.maxr[b] = 0.0f;
    A.alive[b] = 0; A.asleep[b] = 0; A.wake[b] = 0;
}
// the body's own fields from its sums: inverse inertia (minv, src/lib.rs:79-91), pose, velocity, radius; returns the
// position and rotation its bricks' world positions follow from
__device__ void setup_tail(const SetupArgs &A, uint32_t lb, uint32_t b, float mass, V3 cl, float *it, float rr_max,
                           V3 &p, float *prot) {
    it[3] = it[1]; it[6] = it[2]; it[7] = it[5];
    float inv[9];
    {
        const float *a = it;
        float c0 = a[4] * a[8] - a[5] * a[7];
        float c1 = a[5] * a[6] - a[3] * a[8];
        float c2 = a[3] * a[7] - a[4] * a[6];
        float det = a[0] * c0 + a[1] * c1 + a[2] * c2;
        if (fabsf(det) < 1e-12f) {
            for (int k = 0; k < 9; k++) inv[k] = 0.0f;
        } else {
            float id = div_rn(1.0f, det);
            inv[0] = c0 * id; inv[1] = (a[2] * a[7] - a[1] * a[8]) * id; inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
            inv[3] = c1 * id; inv[4] = (a[0] * a[8] - a[2] * a[6]) * id; inv[5] = (a[2] * a[3] - a[0] * a[5]) * id;
            inv[6] = c2 * id; inv[7] = (a[1] * a[6] - a[0] * a[7]) * id; inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
        }
    }
    const float *ps = A.pose + (size_t)lb * A.stride;
    if (A.stride == 22) for (int k = 0; k < 9; k++) prot[k] = ps[13 + k];
    else q_to_m(ps[3], ps[4], ps[5], ps[6], prot);
    V3 off = mv(prot, cl);
    p = add(v3(ps[0], ps[1], ps[2]), off);
    V3 pv = v3(ps[7], ps[8], ps[9]), pw = v3(ps[10], ps[11], ps[12]);
    V3 vel = add(pv, cross(pw, off));
    A.pos[b] = make_float4(p.x, p.y, p.z, 0.0f);
    A.q[b] = make_float4(ps[3], ps[4], ps[5], ps[6]);
    A.v[b] = make_float4(vel.x, vel.y, vel.z, 0.0f);
    A.w[b] = make_float4(pw.x, pw.y, pw.z, 0.0f);
    for (int k = 0; k < 9; k++) { A.rot[(size_t)b * 9 + k] = prot[k]; A.iil[(size_t)b * 9 + k] = inv[k]; }
    float t1[9], t2[9], t3[9];
    mmul(prot, inv, t1); mtr(prot, t2); mmul(t1, t2, t3);
    for (int k = 0; k < 9; k++) A.iiw[(size_t)b * 9 + k] = t3[k];
    A.m[b] = mass; A.im[b] = div_rn(1.0f, mass);
    A.rad[b] = sqrt_rn(rr_max) + H * 1.8f;
    A.sleep[b] = 0.0f; A.maxr[b] = 0.0f;
    A.alive[b] = 1; A.asleep[b] = 0; A.wake[b] = 0;
}
// one thread per body of fewer than SETUP_BIG bricks
__global__ void k_setup_bodies(SetupArgs A) {
    const uint32_t lb = blockIdx.x * blockDim.x + threadIdx.x;
    if (lb >= A.nb) return;
    const uint32_t b = A.list ? A.list[lb] : A.base + lb;
    uint32_t s = A.first[b], n = A.count[b];
    if (n >= SETUP_BIG) return;
    if (n == 0) { setup_dead(A, b); return; }
    float mass = 0.0f;
    V3 cl = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t t = 0; t < n; t++) {
        uint32_t i = s + t;
        V3 l = setup_brick_pos(A, i);
        float mm = c_mat.mass[A.kmat[i]];
        mass += mm;
        cl = madd(cl, l, mm);
    }
    cl = mul(cl, div_rn(1.0f, mass));
    float it[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float rr_max = 0.0f;
    const float cube = S * S / 6.0f;
    for (uint32_t t = 0; t < n; t++) {
        uint32_t i = s + t;
        V3 l = setup_brick_pos(A, i);
        float mm = c_mat.mass[A.kmat[i]];
        V3 r = sub(l, cl);
        A.local[i] = make_float4(r.x, r.y, r.z, 0.0f);
        float rr = dot(r, r);
        rr_max = maxf(rr_max, rr);
        it[0] += mm * (rr - r.x * r.x + cube); it[4] += mm * (rr - r.y * r.y + cube); it[8] += mm * (rr - r.z * r.z + cube);
        it[1] -= mm * r.x * r.y; it[2] -= mm * r.x * r.z; it[5] -= mm * r.y * r.z;
        A.kbody[i] = b;
    }
    V3 p;
    float prot[9];
    setup_tail(A, lb, b, mass, cl, it, rr_max, p, prot);
    for (uint32_t t = 0; t < n; t++) {
        uint32_t i = s + t;
        float4 l = A.local[i];
        V3 wp = add(p, mv(prot, v3(l.x, l.y, l.z)));
        A.wpos[i] = make_float4(wp.x, wp.y, wp.z, 0.0f);
    }
}
// one block per body of SETUP_BIG bricks or more: each thread forms one brick's products of a tile, thread 0 adds
// the tile's terms in list order (the same roundings as one thread), then the bricks' offsets and world positions are
// written in parallel
__global__ void __launch_bounds__(SETUP_T) k_setup_big(SetupArgs A) {
    __shared__ float s_t[7][SETUP_T];
    __shared__ float s_cl[3], s_p[3], s_rot[9];
    const uint32_t lb = blockIdx.x;
    const uint32_t b = A.list ? A.list[lb] : A.base + lb;
    const uint32_t s = A.first[b], n = A.count[b];
    if (n < SETUP_BIG) return;
    const uint32_t k = threadIdx.x;
    float mass = 0.0f;
    V3 cl = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t t0 = 0; t0 < n; t0 += SETUP_T) {
        if (t0 + k < n) {
            const uint32_t i = s + t0 + k;
            const V3 l = setup_brick_pos(A, i);
            const float mm = c_mat.mass[A.kmat[i]];
            s_t[0][k] = mm; s_t[1][k] = l.x * mm; s_t[2][k] = l.y * mm; s_t[3][k] = l.z * mm;
        }
        __syncthreads();
        if (k == 0) {
            const uint32_t e = min((uint32_t)SETUP_T, n - t0);
            for (uint32_t q = 0; q < e; q++) {
                mass += s_t[0][q];
                cl = v3(cl.x + s_t[1][q], cl.y + s_t[2][q], cl.z + s_t[3][q]);
            }
        }
        __syncthreads();
    }
    if (k == 0) {
        cl = mul(cl, div_rn(1.0f, mass));
        s_cl[0] = cl.x; s_cl[1] = cl.y; s_cl[2] = cl.z;
    }
    __syncthreads();
    cl = v3(s_cl[0], s_cl[1], s_cl[2]);
    float it[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float rr_max = 0.0f;
    const float cube = S * S / 6.0f;
    for (uint32_t t0 = 0; t0 < n; t0 += SETUP_T) {
        if (t0 + k < n) {
            const uint32_t i = s + t0 + k;
            const V3 l = setup_brick_pos(A, i);
            const float mm = c_mat.mass[A.kmat[i]];
            const V3 r = sub(l, cl);
            const float rr = dot(r, r);
            s_t[0][k] = mm * (rr - r.x * r.x + cube); s_t[1][k] = mm * (rr - r.y * r.y + cube);
            s_t[2][k] = mm * (rr - r.z * r.z + cube);
            s_t[3][k] = mm * r.x * r.y; s_t[4][k] = mm * r.x * r.z; s_t[5][k] = mm * r.y * r.z;
            s_t[6][k] = rr;
            A.local[i] = make_float4(r.x, r.y, r.z, 0.0f);
            A.kbody[i] = b;
        }
        __syncthreads();
        if (k == 0) {
            const uint32_t e = min((uint32_t)SETUP_T, n - t0);
            for (uint32_t q = 0; q < e; q++) {
                it[0] += s_t[0][q]; it[4] += s_t[1][q]; it[8] += s_t[2][q];
                it[1] -= s_t[3][q]; it[2] -= s_t[4][q]; it[5] -= s_t[5][q];
                rr_max = maxf(rr_max, s_t[6][q]);
            }
        }
        __syncthreads();
    }
    if (k == 0) {
        V3 p;
        float prot[9];
        setup_tail(A, lb, b, mass, cl, it, rr_max, p, prot);
        s_p[0] = p.x; s_p[1] = p.y; s_p[2] = p.z;
        for (int q = 0; q < 9; q++) s_rot[q] = prot[q];
    }
    __syncthreads();
    const V3 p = v3(s_p[0], s_p[1], s_p[2]);
    for (uint32_t t = k; t < n; t += SETUP_T) {
        const uint32_t i = s + t;
        const float4 l = A.local[i];
        const V3 wp = add(p, mv(s_rot, v3(l.x, l.y, l.z)));
        A.wpos[i] = make_float4(wp.x, wp.y, wp.z, 0.0f);
    }
}
static cudaError_t launch_setup(sf_world *w, cudaStream_t st, uint32_t nb, uint32_t base, const uint32_t *list,
                                const float *pose, uint32_t stride) {
    if (nb == 0) return cudaSuccess;
    SetupArgs A;
    A.nb = nb; A.base = base; A.list = list; A.first = w->b_first.p; A.count = w->b_count.p; A.xyz = w->k_xyz.p;
    A.kmat = w->k_mat.p; A.pose = pose; A.stride = stride; A.local = w->k_local.p; A.wpos = w->k_wpos.p;
    A.kbody = w->k_body.p; A.pos = w->b_pos.p; A.q = w->b_q.p; A.v = w->b_v.p; A.w = w->b_w.p; A.rot = w->b_rot.p;
    A.iil = w->b_iil.p; A.iiw = w->b_iiw.p; A.m = w->b_m.p; A.im = w->b_im.p; A.rad = w->b_rad.p;
    A.sleep = w->b_sleep.p; A.maxr = w->b_maxr.p; A.alive = w->b_alive.p; A.asleep = w->b_asleep.p;
    A.wake = w->b_wake.p;
    k_setup_bodies<<<grid_for(nb, 128), 128, 0, st>>>(A);
    k_setup_big<<<nb, SETUP_T, 0, st>>>(A);
    w->launches += 2;
    return cudaGetLastError();
}

__global__ void k_pack_bodies(uint32_t nb, const float4 *pos, const float4 *q, const float4 *v, const float4 *w,
                              const uint8_t *alive, const uint8_t *asleep, float *out13, uint8_t *flags) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    float4 p = pos[b], qq = q[b], vv = v[b], ww = w[b];
    float *o = out13 + (size_t)b * 13;
    o[0] = p.x; o[1] = p.y; o[2] = p.z; o[3] = qq.x; o[4] = qq.y; o[5] = qq.z; o[6] = qq.w;
    o[7] = vv.x; o[8] = vv.y; o[9] = vv.z; o[10] = ww.x; o[11] = ww.y; o[12] = ww.z;
    flags[b] = (alive[b] ? 1 : 0) | (asleep[b] ? 2 : 0);
}
// dirty[b] = the body's pose changed (or it came back to life): its rotation cache and brick positions are refreshed
__global__ void k_unpack_bodies(uint32_t nb, const float *in13, const uint8_t *flags, float4 *pos, float4 *q, float4 *v,
                                float4 *w, uint8_t *alive, uint8_t *asleep, uint8_t *dirty) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const float *o = in13 + (size_t)b * 13;
    const float4 np = make_float4(o[0], o[1], o[2], 0.0f), nq = make_float4(o[3], o[4], o[5], o[6]);
    const float4 op = pos[b], oq = q[b];
    auto same = [](float x, float y) { return __float_as_uint(x) == __float_as_uint(y); };
    const bool moved = !(same(np.x, op.x) && same(np.y, op.y) && same(np.z, op.z) && same(nq.x, oq.x) &&
                         same(nq.y, oq.y) && same(nq.z, oq.z) && same(nq.w, oq.w));
    dirty[b] = (moved || ((flags[b] & 1) && !alive[b])) ? 1 : 0;
    pos[b] = np;
    q[b] = nq;
    v[b] = make_float4(o[7], o[8], o[9], 0.0f);
    w[b] = make_float4(o[10], o[11], o[12], 0.0f);
    alive[b] = flags[b] & 1;
    asleep[b] = (flags[b] >> 1) & 1;
}

// rotation, world inverse inertia and brick positions of the dirty bodies base .. base + nb - 1 (sleeping ones too:
// the step refreshes only awake bodies)
__global__ void k_refresh_bodies(uint32_t nb, uint32_t base, const uint8_t *dirty, const uint8_t *alive, const float4 *q,
                                 const float *iil, float *rot, float *iiw, const float4 *pos, const uint32_t *first,
                                 const uint32_t *count, const float4 *local, float4 *wpos) {
    const uint32_t lb = blockIdx.x * blockDim.x + threadIdx.x;
    if (lb >= nb || !dirty[lb]) return;
    const uint32_t b = base + lb;
    if (!alive[b]) return;
    const float4 qq = q[b];
    float r[9], il[9], t1[9], t2[9], t3[9];
    q_to_m(qq.x, qq.y, qq.z, qq.w, r);
    for (int k = 0; k < 9; k++) il[k] = iil[(size_t)b * 9 + k];
    mmul(r, il, t1);
    mtr(r, t2);
    mmul(t1, t2, t3);
    for (int k = 0; k < 9; k++) { rot[(size_t)b * 9 + k] = r[k]; iiw[(size_t)b * 9 + k] = t3[k]; }
    const float4 p = pos[b];
    for (uint32_t t = 0; t < count[b]; t++) {
        const uint32_t i = first[b] + t;
        const float4 l = local[i];
        const V3 wp = add(v3(p.x, p.y, p.z), mv(r, v3(l.x, l.y, l.z)));
        wpos[i] = make_float4(wp.x, wp.y, wp.z, 0.0f);
    }
}

__global__ void k_kill_marked(uint32_t nb, const uint8_t *alive, const uint32_t *first, const uint32_t *count, uint8_t *kmat) {
    uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb || alive[b]) return;
    for (uint32_t t = 0; t < count[b]; t++) kmat[first[b] + t] = 0;
}

cudaError_t finalize_on_buffers(uint32_t ns, const uint32_t *cell, const uint32_t *scene, const uint8_t *mat,
                                const uint8_t *infill, const int32_t *sid, const uint32_t *ctab, const uint32_t *cpool,
                                uint32_t *nb6, float *bond, float *bmax, cudaStream_t s) {
    cudaError_t e = upload_mat_tables(s);
    if (e != cudaSuccess || ns == 0) return e;
    k_finalize_bricks<<<grid_for(ns, 256), 256, 0, s>>>(ns, 0u, cell, scene, mat, infill, sid, ctab, cpool, nb6, bond, bmax);
    return cudaGetLastError();
}

// host-written body state for bodies base .. base + nb - 1
sf_status write_bodies_range(sf_world *w, uint32_t base, uint32_t nb, const float *state13, const float *sleep,
                             const uint8_t *flags) {
    if (nb == 0) return SF_OK;
    cudaStream_t s = w->stream;
    SF_CUDA(w->stage13.grow((size_t)nb * 13));
    SF_CUDA(w->stage_flags.grow(nb));
    SF_CUDA(w->stage_dirty.grow(nb));
    SF_CUDA(cudaMemcpyAsync(w->stage13.p, state13, (size_t)nb * 13 * sizeof(float), cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(w->b_sleep.p + base, sleep, nb * sizeof(float), cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(w->stage_flags.p, flags, nb, cudaMemcpyHostToDevice, s));
    k_unpack_bodies<<<grid_for(nb, 256), 256, 0, s>>>(nb, w->stage13.p, w->stage_flags.p, w->b_pos.p + base,
                                                      w->b_q.p + base, w->b_v.p + base, w->b_w.p + base,
                                                      w->b_alive.p + base, w->b_asleep.p + base, w->stage_dirty.p);
    k_refresh_bodies<<<grid_for(nb, 128), 128, 0, s>>>(nb, base, w->stage_dirty.p, w->b_alive.p, w->b_q.p, w->b_iil.p,
                                                       w->b_rot.p, w->b_iiw.p, w->b_pos.p, w->b_first.p, w->b_count.p,
                                                       w->k_local.p, w->k_wpos.p);
    k_kill_marked<<<grid_for(nb, 256), 256, 0, s>>>(nb, w->b_alive.p + base, w->b_first.p + base, w->b_count.p + base,
                                                    w->k_mat.p);
    w->launches += 3;
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

sf_status read_error_word(sf_world *w) {
    uint32_t e = 0;
    SF_CUDA(cudaMemcpyAsync(&e, w->err.p, sizeof e, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    w->stats.error_word = e;
    if (e & ERR_TIMEOUT) { set_error("a device barrier wait timed out"); return SF_ERR_TIMEOUT; }
    if (e & (ERR_CAPACITY_CONTACTS | ERR_CAPACITY_COLORS)) { set_error("device capacity exceeded (error bits 0x%x)", e); return SF_ERR_CAPACITY; }
    if (e & (ERR_VERIFY_COLOR | ERR_JP_ROUNDS | ERR_ISLANDS)) { set_error("device self-check failed (error bits 0x%x)", e); return SF_ERR_VERIFY; }
    return SF_OK;
}

}  // namespace sf

template <class T>
static cudaError_t upload(sf::DBuf<T> &d, const std::vector<T> &h, cudaStream_t s) {
    cudaError_t e = d.alloc(h.size());
    if (e != cudaSuccess) return e;
    if (h.empty()) return cudaSuccess;
    return cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

namespace sf {
static cudaError_t setup_launch(sf_world *w, uint32_t base, const uint32_t *list, uint32_t nb, const float *pose,
                                uint32_t stride) {
    if (nb == 0) return cudaSuccess;
    return launch_setup(w, w->stream, nb, base, list, pose, stride);
}
cudaError_t setup_bodies(sf_world *w, uint32_t base, uint32_t nb, const float *d_pose13) {
    const cudaError_t e = setup_launch(w, base, nullptr, nb, d_pose13, 13u);
    if (e != cudaSuccess) return e;
    return body_load_setup(w, nullptr, base, nb, nullptr);
}
cudaError_t setup_bodies_from_local(sf_world *w, const uint32_t *d_list, uint32_t n, const float *d_pose22) {
    return setup_launch(w, 0u, d_list, n, d_pose22, 22u);
}

// finalize_brick (src/lib.rs:668-696) between the bricks of one body: a face neighbour is a brick of the same body one
// lattice cell away; the bond of each +x / +y / +z pair is the weaker brick's capacity on that axis unless an infill
// gap separates them (glass is infill); bodies have no foundation bond. One thread per brick, scanning its body.
__global__ void k_body_bonds(uint32_t nd, const uint32_t *kbody, const uint8_t *alive, const uint32_t *first,
                             const uint32_t *count, const int32_t *xyz, const uint8_t *kmat, uint32_t *nb6, float *bond,
                             float *bmax) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    uint32_t nb[6] = {NONE, NONE, NONE, NONE, NONE, NONE};
    const uint32_t b = kbody[i];
    const uint8_t mi = kmat[i];
    if (alive[b] && mi) {
        const int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        const uint32_t f = first[b], n = count[b];
        for (uint32_t t = 0; t < n; t++) {
            const uint32_t j = f + t;
            const int dx = xyz[3 * j] - x, dy = xyz[3 * j + 1] - y, dz = xyz[3 * j + 2] - z;
            const int ad = abs(dx) + abs(dy) + abs(dz);
            if (ad != 1) continue;
            const int d = dx ? (dx > 0 ? 0 : 1) : dy ? (dy > 0 ? 2 : 3) : (dz > 0 ? 4 : 5);
            nb[d] = j;
        }
    }
#pragma unroll
    for (int d = 0; d < 6; d++) nb6[(size_t)i * 6 + d] = nb[d];
    const uint8_t inf_i = mi == GLASS ? 1 : 0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const uint32_t j = nb[2 * a];
        float c = 0.0f;
        if (j != NONE && mi) {
            const uint8_t mj = kmat[j];
            const uint8_t inf_j = mj == GLASS ? 1 : 0;
            const bool gap = inf_i != inf_j && (a != 1 || inf_i == 1);
            if (!gap && mj != 0) {
                const float ca = a == 1 ? c_mat.capv[mi] : c_mat.caph[mi];
                const float cb = a == 1 ? c_mat.capv[mj] : c_mat.caph[mj];
                c = minf(ca, cb);
            }
        }
        bond[(size_t)i * 4 + a] = c;
        bmax[(size_t)i * 4 + a] = c;
    }
    bond[(size_t)i * 4 + 3] = 0.0f;
    bmax[(size_t)i * 4 + 3] = 0.0f;
}
cudaError_t body_bonds(sf_world *w) {
    if (w->nd == 0) return cudaSuccess;
    k_body_bonds<<<grid_for(w->nd, 256), 256, 0, w->stream>>>(w->nd, w->k_body.p, w->b_alive.p, w->b_first.p,
                                                             w->b_count.p, w->k_xyz.p, w->k_mat.p, w->k_nb6.p,
                                                             w->k_bond.p, w->k_bmax.p);
    w->launches++;
    return cudaGetLastError();
}
}  // namespace sf

extern "C" {

void sf_params_default(sf_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->substeps = 2;
    p->iterations = 10;
    p->sleep_mode = SF_SLEEP_BODY;
    p->pinch_kill = 1;
    p->max_colors = 128;
    p->contact_capacity = 0;
    p->verify = 1;
    p->solve_blocks = 0;
    p->manifold_chunk = 16;
    p->sor_cluster = 1;
}

sf_status sf_world_create(const sf_world_desc *desc, const sf_params *params, sf_world **out) {
    if (!desc || !out || (desc->n_scenes && !desc->scenes)) { set_error("null argument"); return SF_ERR_ARG; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return SF_ERR_CUDA; }
    std::unique_ptr<sf_world, void (*)(sf_world *)> w(new sf_world(), sf_world_destroy);
    if (params) w->P = *params; else sf_params_default(&w->P);
    if (w->P.substeps == 0) w->P.substeps = 2;
    if (w->P.max_colors == 0 || w->P.max_colors > (uint32_t)MAXCOL) w->P.max_colors = MAXCOL;
    SF_CUDA(cudaGetDevice(&w->device));
    SF_CUDA(cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, w->device));
    SF_CUDA(cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking));
    w->stream = w->own_stream;
    SF_CUDA(cudaEventCreate(&w->ev0));
    SF_CUDA(cudaEventCreate(&w->ev1));
    SF_CUDA(upload_mat_tables(w->stream));

    // ---- validate and lay out scenes
    uint32_t n_scenes = desc->n_scenes;
    w->n_scenes = n_scenes;
    w->scenes.resize(n_scenes);
    uint64_t ns = 0, nd = 0, nb = 0;
    int32_t max_sid = -1;
    for (uint32_t s = 0; s < n_scenes; s++) {
        const sf_scene_desc &d = desc->scenes[s];
        if (d.n_static && (!d.static_xyz || !d.static_mat || !d.static_sid || !d.static_infill)) { set_error("scene %u: null static array", s); return SF_ERR_ARG; }
        if (d.n_bodies && (!d.body_first || !d.body_brick_xyz || !d.body_brick_mat || !d.body_pose)) { set_error("scene %u: null body array", s); return SF_ERR_ARG; }
        Scene &sc = w->scenes[s];
        sc.static_off = (uint32_t)ns; sc.n_static = d.n_static;
        sc.body_off = (uint32_t)nb; sc.n_bodies = d.n_bodies;
        uint32_t nbr = d.n_bodies ? d.body_first[d.n_bodies] : 0;
        if (d.n_bodies && d.body_first[0] != 0) { set_error("scene %u: body_first[0] must be 0", s); return SF_ERR_ARG; }
        for (uint32_t b = 0; b < d.n_bodies; b++)
            if (d.body_first[b + 1] <= d.body_first[b]) { set_error("scene %u body %u: no bricks", s, b); return SF_ERR_ARG; }
        sc.brick_off = (uint32_t)nd; sc.n_bricks = nbr;
        for (uint32_t k = 0; k < nbr; k++) {
            uint8_t m = d.body_brick_mat[k];
            if (m == 0 || m > 8) { set_error("scene %u body brick %u: material %u", s, k, m); return SF_ERR_ARG; }
        }
        for (uint32_t b = 0; b < d.n_bodies; b++)
            for (int k = 0; k < 13; k++)
                if (!std::isfinite(d.body_pose[(size_t)b * 13 + k])) { set_error("scene %u body %u: non-finite pose", s, b); return SF_ERR_ARG; }
        for (uint32_t i = 0; i < d.n_static; i++) max_sid = std::max(max_sid, d.static_sid[i]);
        sc.bodies_used = d.n_bodies; sc.bricks_used = nbr;
        sc.n_bodies += w->P.detach_bodies; sc.n_bricks += w->P.detach_bricks;
        ns += d.n_static; nd += sc.n_bricks; nb += sc.n_bodies;
    }
    // spare capacity for detached pieces: unused bricks belong to an always-dead sentinel body after the scenes'
    const bool spare = w->P.detach_bodies || w->P.detach_bricks;
    if (w->P.damage && !spare) { set_error("damage needs spare capacity (detach_bodies, detach_bricks)"); return SF_ERR_ARG; }
    if (spare) nb += 1;
    if (ns >= 0x7fffffffu || nd >= 0x7fffffffu || nb >= 0x7fffffffu) { set_error("world too large"); return SF_ERR_CAPACITY; }
    w->ns = (uint32_t)ns; w->nd = (uint32_t)nd; w->nb = (uint32_t)nb;
    if (spare) w->sentinel = (uint32_t)nb - 1;
    w->n_struct = (uint32_t)(max_sid + 1);

    // ---- static bricks and the chunk grid (host-side table build, uploaded once)
    std::vector<uint32_t> h_ctab((size_t)n_scenes * NCT, 0), h_cpool;
    std::vector<uint32_t> s_cell(ns), s_scene(ns);
    std::vector<uint8_t> s_mat(ns), s_inf(ns);
    std::vector<int32_t> s_sid(ns);
    uint32_t nchunks = 0;
    for (uint32_t s = 0; s < n_scenes; s++) {
        const sf_scene_desc &d = desc->scenes[s];
        Scene &sc = w->scenes[s];
        sc.chunk_off = nchunks;
        for (uint32_t k = 0; k < d.n_static; k++) {
            int x = d.static_xyz[3 * k], y = d.static_xyz[3 * k + 1], z = d.static_xyz[3 * k + 2];
            uint8_t m = d.static_mat[k];
            if (!inb(x, y, z)) { set_error("scene %u static %u: cell (%d,%d,%d) outside the lattice", s, k, x, y, z); return SF_ERR_ARG; }
            if (m == 0 || m > 8) { set_error("scene %u static %u: material %u", s, k, m); return SF_ERR_ARG; }
            if (d.static_sid[k] < -1) { set_error("scene %u static %u: structure id %d", s, k, d.static_sid[k]); return SF_ERR_ARG; }
            uint32_t gi = sc.static_off + k;
            uint32_t &t = h_ctab[(size_t)s * NCT + chunk_slot(x, y, z)];
            if (t == 0) {
                nchunks++;
                t = nchunks;
                h_cpool.resize((size_t)nchunks * 512, 0);
                w->h_chunk_cell.push_back(pack_cell(x & ~7, y & ~7, z & ~7));
                w->h_chunk_scene.push_back(s);
            }
            uint32_t &slot = h_cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
            if (slot != 0) { set_error("scene %u static %u: cell (%d,%d,%d) already holds a brick", s, k, x, y, z); return SF_ERR_ARG; }
            slot = gi + 1;
            s_cell[gi] = pack_cell(x, y, z); s_scene[gi] = s; s_mat[gi] = m;
            s_inf[gi] = (m == GLASS || d.static_infill[k]) ? 1 : 0;
            s_sid[gi] = d.static_sid[k];
        }
        sc.n_chunks = nchunks - sc.chunk_off;
        // the scene's static bricks' bounding box (empty: lo > hi), which lets a brick far from all of them skip
        // the static-cell search
        int4 lo = make_int4(1 << 20, 1 << 20, 1 << 20, 0), hi = make_int4(-(1 << 20), -(1 << 20), -(1 << 20), 0);
        for (uint32_t k = 0; k < d.n_static; k++) {
            int x = d.static_xyz[3 * k], y = d.static_xyz[3 * k + 1], z = d.static_xyz[3 * k + 2];
            lo.x = std::min(lo.x, x); lo.y = std::min(lo.y, y); lo.z = std::min(lo.z, z);
            hi.x = std::max(hi.x, x); hi.y = std::max(hi.y, y); hi.z = std::max(hi.z, z);
        }
        w->h_sbox.push_back(lo);
        w->h_sbox.push_back(hi);
    }
    w->n_chunks = nchunks;
    w->h_sid = s_sid;
    w->h_s_cell = s_cell;
    cudaStream_t st = w->stream;
    SF_CUDA(upload(w->ctab, h_ctab, st));
    SF_CUDA(upload(w->sbox, w->h_sbox, st));
    SF_CUDA(upload(w->cpool, h_cpool, st));
    SF_CUDA(upload(w->s_cell, s_cell, st));
    SF_CUDA(upload(w->s_scene, s_scene, st));
    SF_CUDA(upload(w->s_mat, s_mat, st));
    SF_CUDA(upload(w->s_infill, s_inf, st));
    SF_CUDA(upload(w->s_sid, s_sid, st));
    SF_CUDA(w->s_nb6.alloc((size_t)ns * 6));
    SF_CUDA(w->s_bond.alloc((size_t)ns * 4));
    SF_CUDA(w->s_bmax.alloc((size_t)ns * 4));
    SF_CUDA(w->s_phi.alloc(ns));
    SF_CUDA(w->s_phi64.alloc(ns));
    SF_CUDA(cudaMemsetAsync(w->s_phi64.p, 0, w->s_phi64.bytes(), st));
    SF_CUDA(w->s_ext.alloc(ns));
    SF_CUDA(w->s_stress.alloc(ns));
    SF_CUDA(cudaMemsetAsync(w->s_phi.p, 0, w->s_phi.bytes(), st));
    SF_CUDA(cudaMemsetAsync(w->s_ext.p, 0, w->s_ext.bytes(), st));
    SF_CUDA(cudaMemsetAsync(w->s_stress.p, 0, w->s_stress.bytes(), st));
    if (ns) {
        k_finalize_bricks<<<grid_for(ns, 256), 256, 0, st>>>((uint32_t)ns, 0u, w->s_cell.p, w->s_scene.p, w->s_mat.p,
                                                           w->s_infill.p, w->s_sid.p, w->ctab.p, w->cpool.p, w->s_nb6.p,
                                                           w->s_bond.p, w->s_bmax.p);
        SF_CUDA(cudaGetLastError());
    }

    // ---- bodies and body bricks
    std::vector<uint32_t> b_first(nb), b_count(nb), b_scene(nb);
    std::vector<int32_t> k_xyz((size_t)nd * 3);
    std::vector<uint8_t> k_mat(nd);
    std::vector<float> pose((size_t)nb * 13);
    for (uint32_t s = 0; s < n_scenes; s++) {
        const sf_scene_desc &d = desc->scenes[s];
        const Scene &sc = w->scenes[s];
        for (uint32_t b = 0; b < d.n_bodies; b++) {
            uint32_t gb = sc.body_off + b;
            b_first[gb] = sc.brick_off + d.body_first[b];
            b_count[gb] = d.body_first[b + 1] - d.body_first[b];
            std::memcpy(&pose[(size_t)gb * 13], d.body_pose + (size_t)b * 13, 13 * sizeof(float));
        }
        for (uint32_t b = 0; b < sc.n_bodies; b++) b_scene[sc.body_off + b] = s;
        if (sc.bricks_used) {
            std::memcpy(&k_xyz[(size_t)sc.brick_off * 3], d.body_brick_xyz, (size_t)sc.bricks_used * 3 * sizeof(int32_t));
            std::memcpy(&k_mat[sc.brick_off], d.body_brick_mat, sc.bricks_used);
        }
    }
    SF_CUDA(upload(w->b_first, b_first, st));
    SF_CUDA(upload(w->b_count, b_count, st));
    SF_CUDA(upload(w->b_scene, b_scene, st));
    SF_CUDA(upload(w->k_xyz, k_xyz, st));
    SF_CUDA(upload(w->k_mat, k_mat, st));
    sf::DBuf<float> d_pose;
    SF_CUDA(upload(d_pose, pose, st));
    SF_CUDA(w->b_pos.alloc(nb)); SF_CUDA(w->b_q.alloc(nb)); SF_CUDA(w->b_v.alloc(nb)); SF_CUDA(w->b_w.alloc(nb));
    SF_CUDA(w->b_vpre.alloc(nb)); SF_CUDA(w->b_wpre.alloc(nb));
    SF_CUDA(w->b_rot.alloc((size_t)nb * 9)); SF_CUDA(w->b_iil.alloc((size_t)nb * 9)); SF_CUDA(w->b_iiw.alloc((size_t)nb * 9));
    SF_CUDA(w->b_m.alloc(nb)); SF_CUDA(w->b_im.alloc(nb)); SF_CUDA(w->b_rad.alloc(nb)); SF_CUDA(w->b_sleep.alloc(nb));
    SF_CUDA(w->b_maxr.alloc(nb));
    SF_CUDA(w->b_alive.alloc(nb)); SF_CUDA(w->b_asleep.alloc(nb)); SF_CUDA(w->b_wake.alloc(nb));
    SF_CUDA(w->b_nc.alloc(nb));
    SF_CUDA(cudaMemsetAsync(w->b_nc.p, 0, w->b_nc.bytes(), st));
    SF_CUDA(w->k_local.alloc(nd)); SF_CUDA(w->k_wpos.alloc(nd));
    SF_CUDA(upload(w->k_body, std::vector<uint32_t>(nd, spare ? w->sentinel : 0u), st));
    if (spare) {
        SF_CUDA(cudaMemsetAsync(w->k_local.p, 0, w->k_local.bytes(), st));
        SF_CUDA(cudaMemsetAsync(w->k_wpos.p, 0, w->k_wpos.bytes(), st));
    }
    if (nb) {
        SF_CUDA(launch_setup(w.get(), st, (uint32_t)nb, 0u, nullptr, d_pose.p, 13u));
        SF_CUDA(cudaGetLastError());
    }
    SF_CUDA(w->err.alloc(64));
    SF_CUDA(cudaMemsetAsync(w->err.p, 0, w->err.bytes(), st));
    SF_CUDA(w->barrier.alloc(4));
    SF_CUDA(cudaMemsetAsync(w->barrier.p, 0, w->barrier.bytes(), st));
    if (spare) {
        SF_CUDA(w->k_nb6.alloc((size_t)std::max<uint64_t>(nd, 1) * 6));
        SF_CUDA(w->k_bond.alloc((size_t)std::max<uint64_t>(nd, 1) * 4));
        SF_CUDA(w->k_bmax.alloc((size_t)std::max<uint64_t>(nd, 1) * 4));
        SF_CUDA(w->b_dirty.alloc(nb));
        SF_CUDA(cudaMemsetAsync(w->b_dirty.p, 0, w->b_dirty.bytes(), st));
        SF_CUDA(body_bonds(w.get()));
        // the debris-body load field: potentials and loads start at 0, no contact has supported a brick yet
        const size_t ndd = std::max<uint64_t>(nd, 1);
        SF_CUDA(w->k_sup.alloc(ndd)); SF_CUDA(w->k_phi64.alloc(ndd)); SF_CUDA(w->k_phi.alloc(ndd)); SF_CUDA(w->k_ext.alloc(ndd));
        SF_CUDA(w->b_vlast.alloc(nb)); SF_CUDA(w->b_wlast.alloc(nb)); SF_CUDA(w->b_resid.alloc(nb));
        SF_CUDA(w->b_nmax.alloc(nb)); SF_CUDA(w->b_lt.alloc(nb));
        SF_CUDA(cudaMemsetAsync(w->k_sup.p, 0, w->k_sup.bytes(), st));
        SF_CUDA(cudaMemsetAsync(w->k_phi64.p, 0, w->k_phi64.bytes(), st));
        SF_CUDA(cudaMemsetAsync(w->k_phi.p, 0, w->k_phi.bytes(), st));
        SF_CUDA(cudaMemsetAsync(w->k_ext.p, 0, w->k_ext.bytes(), st));
        SF_CUDA(cudaMemsetAsync(w->b_lt.p, 0, w->b_lt.bytes(), st));
        SF_CUDA(body_load_setup(w.get(), nullptr, 0u, (uint32_t)nb, nullptr));
    }
    SF_CUDA(w->st_conn.alloc(std::max<uint32_t>(w->n_struct, 1)));
    SF_CUDA(cudaMemsetAsync(w->st_conn.p, 0, w->st_conn.bytes(), st));
    w->h_conn_retry.assign(w->n_struct, 0);
    sf_status r = sor_create(w.get());
    if (r != SF_OK) return r;
    r = step_create(w.get());
    if (r != SF_OK) return r;
    SF_CUDA(cudaStreamSynchronize(st));
    *out = w.release();
    return SF_OK;
}

void sf_world_destroy(sf_world *w) {
    if (!w) return;
    if (w->stream) cudaStreamSynchronize(w->stream);
    sor_destroy(w);
    step_destroy(w);
    conn_destroy(w);
    split_destroy(w);
    damage_destroy(w);
    bodyload_destroy(w);
    if (w->ev0) cudaEventDestroy(w->ev0);
    if (w->ev1) cudaEventDestroy(w->ev1);
    cudaStream_t s = w->own_stream;
    delete w;
    if (s) cudaStreamDestroy(s);
}

sf_status sf_world_get_info(const sf_world *w, sf_world_info *info) {
    if (!w || !info) return SF_ERR_ARG;
    info->n_scenes = w->n_scenes; info->n_static = w->ns; info->n_bodies = w->nb; info->n_body_bricks = w->nd;
    info->n_structures = w->n_struct; info->n_chunks = w->n_chunks;
    return SF_OK;
}

sf_status sf_world_scene_ranges(const sf_world *w, uint32_t scene, uint32_t out8[8]) {
    if (!w || !out8 || scene >= w->n_scenes) { set_error("no such scene"); return SF_ERR_ARG; }
    const Scene &sc = w->scenes[scene];
    const bool pool = !w->pool.empty();
    out8[0] = sc.static_off; out8[1] = sc.n_static; out8[2] = sc.body_off; out8[3] = sc.n_bodies;
    out8[4] = sc.brick_off; out8[5] = sc.n_bricks;
    out8[6] = pool ? w->pool[scene].bodies : sc.bodies_used;
    out8[7] = pool ? w->pool[scene].bricks : sc.bricks_used;
    return SF_OK;
}

sf_status sf_get_stats(const sf_world *w, sf_stats *st) {
    if (!w || !st) return SF_ERR_ARG;
    *st = w->stats;
    return SF_OK;
}

// Body state crosses the boundary as 13 floats per body (the layout a host engine keeps); the device keeps float4
// columns. One copy of the packed block each way, packed and unpacked on the device.
sf_status sf_read_bodies(sf_world *w, float *state13, float *sleep, uint8_t *flags) {
    if (!w) return SF_ERR_ARG;
    uint32_t nb = w->nb;
    if (nb == 0) return SF_OK;
    cudaStream_t s = w->stream;
    SF_CUDA(w->stage13.grow((size_t)nb * 13));
    SF_CUDA(w->stage_flags.grow(nb));
    k_pack_bodies<<<grid_for(nb, 256), 256, 0, s>>>(nb, w->b_pos.p, w->b_q.p, w->b_v.p, w->b_w.p, w->b_alive.p,
                                                    w->b_asleep.p, w->stage13.p, w->stage_flags.p);
    w->launches++;
    if (state13) SF_CUDA(cudaMemcpyAsync(state13, w->stage13.p, (size_t)nb * 13 * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (sleep) SF_CUDA(cudaMemcpyAsync(sleep, w->b_sleep.p, nb * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (flags) SF_CUDA(cudaMemcpyAsync(flags, w->stage_flags.p, nb, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

sf_status sf_write_bodies(sf_world *w, const float *state13, const float *sleep, const uint8_t *flags) {
    if (!w || !state13 || !sleep || !flags) return SF_ERR_ARG;
    sf_status r = write_bodies_range(w, 0, w->nb, state13, sleep, flags);
    step_mark_all_live(w);
    return r;
}

sf_status sf_read_body_setup(sf_world *w, float *body12, float *local3) {
    if (!w) return SF_ERR_ARG;
    uint32_t nb = w->nb, nd = w->nd;
    std::vector<float> m(nb), im(nb), rad(nb), iil((size_t)nb * 9);
    std::vector<float4> loc(nd);
    cudaStream_t s = w->stream;
    SF_CUDA(cudaMemcpyAsync(m.data(), w->b_m.p, nb * 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(im.data(), w->b_im.p, nb * 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(rad.data(), w->b_rad.p, nb * 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(iil.data(), w->b_iil.p, (size_t)nb * 36, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(loc.data(), w->k_local.p, nd * sizeof(float4), cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    for (uint32_t b = 0; b < nb && body12; b++) {
        float *o = body12 + (size_t)b * 12;
        o[0] = m[b]; o[1] = im[b]; o[2] = rad[b];
        for (int k = 0; k < 9; k++) o[3 + k] = iil[(size_t)b * 9 + k];
    }
    for (uint32_t k = 0; k < nd && local3; k++) { local3[3 * k] = loc[k].x; local3[3 * k + 1] = loc[k].y; local3[3 * k + 2] = loc[k].z; }
    return SF_OK;
}

sf_status sf_read_brick_positions(sf_world *w, float *wpos3) {
    if (!w || !wpos3) return SF_ERR_ARG;
    std::vector<float4> p(w->nd);
    SF_CUDA(cudaMemcpyAsync(p.data(), w->k_wpos.p, w->nd * sizeof(float4), cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    for (uint32_t k = 0; k < w->nd; k++) { wpos3[3 * k] = p[k].x; wpos3[3 * k + 1] = p[k].y; wpos3[3 * k + 2] = p[k].z; }
    return SF_OK;
}

sf_status sf_read_phi(sf_world *w, float *phi) {
    if (!w || !phi) return SF_ERR_ARG;
    SF_CUDA(cudaMemcpyAsync(phi, w->s_phi.p, (size_t)w->ns * 4, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}
sf_status sf_write_phi(sf_world *w, const float *phi) {
    if (!w || !phi) return SF_ERR_ARG;
    std::vector<double> p64(phi, phi + w->ns);
    SF_CUDA(cudaMemcpyAsync(w->s_phi.p, phi, (size_t)w->ns * 4, cudaMemcpyHostToDevice, w->stream));
    SF_CUDA(cudaMemcpyAsync(w->s_phi64.p, p64.data(), (size_t)w->ns * 8, cudaMemcpyHostToDevice, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}
sf_status sf_read_phi64(sf_world *w, double *phi) {
    if (!w || !phi) return SF_ERR_ARG;
    SF_CUDA(cudaMemcpyAsync(phi, w->s_phi64.p, (size_t)w->ns * 8, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}
sf_status sf_write_ext(sf_world *w, const float *ext) {
    if (!w || !ext) return SF_ERR_ARG;
    SF_CUDA(cudaMemcpyAsync(w->s_ext.p, ext, (size_t)w->ns * 4, cudaMemcpyHostToDevice, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}
sf_status sf_read_ext(sf_world *w, float *ext) {
    if (!w || !ext) return SF_ERR_ARG;
    SF_CUDA(cudaMemcpyAsync(ext, w->s_ext.p, (size_t)w->ns * 4, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}
sf_status sf_read_bonds(sf_world *w, float *bond4, uint32_t *nb6, uint8_t *mat) {
    if (!w) return SF_ERR_ARG;
    cudaStream_t s = w->stream;
    if (bond4) SF_CUDA(cudaMemcpyAsync(bond4, w->s_bond.p, (size_t)w->ns * 16, cudaMemcpyDeviceToHost, s));
    if (nb6) SF_CUDA(cudaMemcpyAsync(nb6, w->s_nb6.p, (size_t)w->ns * 24, cudaMemcpyDeviceToHost, s));
    if (mat) SF_CUDA(cudaMemcpyAsync(mat, w->s_mat.p, (size_t)w->ns, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- scene pools
// A pool is a world laid out by capacity: slot s owns fixed ranges of bodies, bricks, static bricks and chunks,
// and a scene is loaded into a slot, saved out of it and restored into it without touching the other slots. The
// step's active set never includes an empty slot, so the pool's cost follows the loaded, awake scenes.
namespace sf {

// device bytes per unit of capacity (the arrays of sf_world, StepState and an initial 4 contacts per brick)
constexpr uint64_t POOL_BYTES_BODY = 320, POOL_BYTES_BRICK = 1560, POOL_BYTES_STATIC = 96, POOL_BYTES_CHUNK = 2048;
constexpr uint64_t POOL_BYTES_SLOT = (uint64_t)NCT * 4 + (uint64_t)HSIZE * 8 + 64;

static uint64_t slot_bytes(const sf_pool_slot &c) {
    return POOL_BYTES_SLOT + c.bodies * POOL_BYTES_BODY + c.bricks * POOL_BYTES_BRICK + c.statics * POOL_BYTES_STATIC +
           c.chunks * POOL_BYTES_CHUNK;
}

// mutable state of a loaded scene, in this order: per body pos, q, v, w (float4), rot, iiw (9 floats), sleep
// (float), alive, asleep (bytes); per brick world position (float4) and material (byte; 0 = removed)
static uint64_t snapshot_bytes(uint64_t nb, uint64_t nd) { return nb * (64 + 72 + 4 + 2) + nd * (16 + 1); }

struct SnapPart { void *dev; size_t elem; };

static void snapshot_parts(sf_world *w, const Scene &sc, SnapPart parts[11]) {
    const uint32_t b = sc.body_off, k = sc.brick_off;
    parts[0] = {w->b_pos.p + b, 16}; parts[1] = {w->b_q.p + b, 16}; parts[2] = {w->b_v.p + b, 16};
    parts[3] = {w->b_w.p + b, 16}; parts[4] = {w->b_rot.p + (size_t)b * 9, 36}; parts[5] = {w->b_iiw.p + (size_t)b * 9, 36};
    parts[6] = {w->b_sleep.p + b, 4}; parts[7] = {w->b_alive.p + b, 1}; parts[8] = {w->b_asleep.p + b, 1};
    parts[9] = {w->k_wpos.p + k, 16}; parts[10] = {w->k_mat.p + k, 1};
}

// validates a scene against a slot's capacity; a pool serves rigid scenes, so static bricks must not belong to a
// structure
static sf_status check_slot_scene(const sf_world *w, uint32_t slot, const sf_scene_desc *d) {
    if (w->pool.empty()) { set_error("not a scene pool"); return SF_ERR_ARG; }
    if (!d || slot >= w->pool.size()) { set_error("bad slot %u or null scene", slot); return SF_ERR_ARG; }
    const Scene &sc = w->scenes[slot];
    if (d->n_static && (!d->static_xyz || !d->static_mat || !d->static_sid || !d->static_infill)) { set_error("null static array"); return SF_ERR_ARG; }
    if (d->n_bodies && (!d->body_first || !d->body_brick_xyz || !d->body_brick_mat || !d->body_pose)) { set_error("null body array"); return SF_ERR_ARG; }
    const uint32_t nbr = d->n_bodies ? d->body_first[d->n_bodies] : 0;
    if (d->n_bodies > sc.n_bodies || nbr > sc.n_bricks || d->n_static > sc.n_static) {
        set_error("scene (%u bodies, %u bricks, %u static) exceeds slot %u (%u, %u, %u)", d->n_bodies, nbr, d->n_static,
                  slot, sc.n_bodies, sc.n_bricks, sc.n_static);
        return SF_ERR_CAPACITY;
    }
    if (d->n_bodies && d->body_first[0] != 0) { set_error("body_first[0] must be 0"); return SF_ERR_ARG; }
    for (uint32_t b = 0; b < d->n_bodies; b++) {
        if (d->body_first[b + 1] <= d->body_first[b]) { set_error("body %u: no bricks", b); return SF_ERR_ARG; }
        for (int k = 0; k < 13; k++)
            if (!std::isfinite(d->body_pose[(size_t)b * 13 + k])) { set_error("body %u: non-finite pose", b); return SF_ERR_ARG; }
    }
    for (uint32_t k = 0; k < nbr; k++)
        if (d->body_brick_mat[k] == 0 || d->body_brick_mat[k] > 8) { set_error("body brick %u: material %u", k, d->body_brick_mat[k]); return SF_ERR_ARG; }
    for (uint32_t k = 0; k < d->n_static; k++) {
        const int x = d->static_xyz[3 * k], y = d->static_xyz[3 * k + 1], z = d->static_xyz[3 * k + 2];
        if (!inb(x, y, z)) { set_error("static %u: cell (%d,%d,%d) outside the lattice", k, x, y, z); return SF_ERR_ARG; }
        if (d->static_mat[k] == 0 || d->static_mat[k] > 8) { set_error("static %u: material %u", k, d->static_mat[k]); return SF_ERR_ARG; }
        if (d->static_sid[k] != -1) { set_error("static %u: structure %d; a scene pool holds no load-path structures", k, d->static_sid[k]); return SF_ERR_ARG; }
    }
    return SF_OK;
}

}  // namespace sf

extern "C" {

sf_status sf_pool_bytes(uint32_t n_slots, const sf_pool_slot *slots, uint64_t *bytes) {
    if (!bytes || (n_slots && !slots)) { set_error("null argument"); return SF_ERR_ARG; }
    uint64_t t = 0;
    for (uint32_t s = 0; s < n_slots; s++) t += slot_bytes(slots[s]);
    *bytes = t;
    return SF_OK;
}

uint64_t sf_pool_snapshot_bytes(uint32_t n_bodies, uint32_t n_bricks) { return snapshot_bytes(n_bodies, n_bricks); }

sf_status sf_pool_create(uint32_t n_slots, const sf_pool_slot *slots, const sf_params *params, sf_world **out) {
    if (!out || !n_slots || !slots) { set_error("null argument or no slots"); return SF_ERR_ARG; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return SF_ERR_CUDA; }
    std::unique_ptr<sf_world, void (*)(sf_world *)> w(new sf_world(), sf_world_destroy);
    if (params) w->P = *params; else sf_params_default(&w->P);
    if (w->P.substeps == 0) w->P.substeps = 2;
    if (w->P.max_colors == 0 || w->P.max_colors > (uint32_t)MAXCOL) w->P.max_colors = MAXCOL;
    if (w->P.damage || w->P.detach_bodies || w->P.detach_bricks) {
        set_error("a scene pool has no spare capacity for detached pieces: damage and detach_* are for sf_world_create");
        return SF_ERR_ARG;
    }
    SF_CUDA(cudaGetDevice(&w->device));
    SF_CUDA(cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, w->device));
    SF_CUDA(cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking));
    w->stream = w->own_stream;
    SF_CUDA(cudaEventCreate(&w->ev0));
    SF_CUDA(cudaEventCreate(&w->ev1));
    SF_CUDA(upload_mat_tables(w->stream));
    cudaStream_t st = w->stream;
    w->n_scenes = n_slots;
    w->scenes.resize(n_slots);
    w->pool.assign(n_slots, PoolSlot{});
    uint64_t ns = 0, nd = 0, nb = 0, nch = 0;
    for (uint32_t s = 0; s < n_slots; s++) {
        const sf_pool_slot &c = slots[s];
        if (c.bodies == 0 || c.bricks < c.bodies) { set_error("slot %u: %u bodies, %u bricks", s, c.bodies, c.bricks); return SF_ERR_ARG; }
        Scene &sc = w->scenes[s];
        sc.static_off = (uint32_t)ns; sc.n_static = c.statics;
        sc.body_off = (uint32_t)nb; sc.n_bodies = c.bodies;
        sc.brick_off = (uint32_t)nd; sc.n_bricks = c.bricks;
        sc.chunk_off = (uint32_t)nch; sc.n_chunks = c.chunks;
        ns += c.statics; nd += c.bricks; nb += c.bodies; nch += c.chunks;
    }
    nb += 1;   // the sentinel body: never alive, owner of every unused brick
    if (ns >= 0x7fffffffu || nd >= 0x7fffffffu || nb >= 0x7fffffffu || nch >= (1u << 24)) { set_error("pool too large"); return SF_ERR_CAPACITY; }
    w->ns = (uint32_t)ns; w->nd = (uint32_t)nd; w->nb = (uint32_t)nb; w->n_chunks = (uint32_t)nch; w->n_struct = 0;
    w->sentinel = (uint32_t)nb - 1;
    // static grid: empty tables, static bricks absent (material 0, no structure)
    SF_CUDA(w->ctab.alloc((size_t)n_slots * NCT)); SF_CUDA(cudaMemsetAsync(w->ctab.p, 0, w->ctab.bytes(), st));
    SF_CUDA(w->cpool.alloc(std::max<uint64_t>(nch, 1) * 512)); SF_CUDA(cudaMemsetAsync(w->cpool.p, 0, w->cpool.bytes(), st));
    w->h_sbox.assign((size_t)n_slots * 2, make_int4(0, 0, 0, 0));
    for (uint32_t s = 0; s < n_slots; s++) {
        w->h_sbox[2 * s] = make_int4(1 << 20, 1 << 20, 1 << 20, 0);
        w->h_sbox[2 * s + 1] = make_int4(-(1 << 20), -(1 << 20), -(1 << 20), 0);
    }
    SF_CUDA(upload(w->sbox, w->h_sbox, st));
    std::vector<uint32_t> s_scene(ns);
    for (uint32_t s = 0; s < n_slots; s++)
        std::fill(s_scene.begin() + w->scenes[s].static_off, s_scene.begin() + w->scenes[s].static_off + w->scenes[s].n_static, s);
    SF_CUDA(upload(w->s_scene, s_scene, st));
    std::vector<int32_t> s_sid(ns, -1);
    SF_CUDA(upload(w->s_sid, s_sid, st));
    SF_CUDA(w->s_cell.alloc(ns)); SF_CUDA(w->s_mat.alloc(ns)); SF_CUDA(w->s_infill.alloc(ns));
    SF_CUDA(cudaMemsetAsync(w->s_mat.p, 0, w->s_mat.bytes(), st));
    SF_CUDA(w->s_nb6.alloc((size_t)ns * 6)); SF_CUDA(w->s_bond.alloc((size_t)ns * 4)); SF_CUDA(w->s_bmax.alloc((size_t)ns * 4));
    SF_CUDA(w->s_phi.alloc(ns)); SF_CUDA(w->s_phi64.alloc(ns)); SF_CUDA(w->s_ext.alloc(ns)); SF_CUDA(w->s_stress.alloc(ns));
    // bodies: all dead; every brick belongs to the sentinel
    std::vector<uint32_t> b_scene(nb, 0);
    for (uint32_t s = 0; s < n_slots; s++)
        std::fill(b_scene.begin() + w->scenes[s].body_off, b_scene.begin() + w->scenes[s].body_off + w->scenes[s].n_bodies, s);
    SF_CUDA(upload(w->b_scene, b_scene, st));
    SF_CUDA(w->b_first.alloc(nb)); SF_CUDA(w->b_count.alloc(nb));
    SF_CUDA(cudaMemsetAsync(w->b_first.p, 0, w->b_first.bytes(), st));
    SF_CUDA(cudaMemsetAsync(w->b_count.p, 0, w->b_count.bytes(), st));
    SF_CUDA(w->k_xyz.alloc((size_t)nd * 3)); SF_CUDA(w->k_mat.alloc(nd));
    SF_CUDA(cudaMemsetAsync(w->k_mat.p, 0, w->k_mat.bytes(), st));
    std::vector<uint32_t> k_body(nd, w->sentinel);
    SF_CUDA(upload(w->k_body, k_body, st));
    SF_CUDA(w->b_pos.alloc(nb)); SF_CUDA(w->b_q.alloc(nb)); SF_CUDA(w->b_v.alloc(nb)); SF_CUDA(w->b_w.alloc(nb));
    SF_CUDA(w->b_vpre.alloc(nb)); SF_CUDA(w->b_wpre.alloc(nb));
    SF_CUDA(w->b_rot.alloc((size_t)nb * 9)); SF_CUDA(w->b_iil.alloc((size_t)nb * 9)); SF_CUDA(w->b_iiw.alloc((size_t)nb * 9));
    SF_CUDA(w->b_m.alloc(nb)); SF_CUDA(w->b_im.alloc(nb)); SF_CUDA(w->b_rad.alloc(nb)); SF_CUDA(w->b_sleep.alloc(nb));
    SF_CUDA(w->b_maxr.alloc(nb));
    SF_CUDA(w->b_alive.alloc(nb)); SF_CUDA(w->b_asleep.alloc(nb)); SF_CUDA(w->b_wake.alloc(nb)); SF_CUDA(w->b_nc.alloc(nb));
    SF_CUDA(cudaMemsetAsync(w->b_alive.p, 0, w->b_alive.bytes(), st));
    SF_CUDA(cudaMemsetAsync(w->b_asleep.p, 0, w->b_asleep.bytes(), st));
    SF_CUDA(cudaMemsetAsync(w->b_wake.p, 0, w->b_wake.bytes(), st));
    SF_CUDA(cudaMemsetAsync(w->b_nc.p, 0, w->b_nc.bytes(), st));
    SF_CUDA(w->k_local.alloc(nd)); SF_CUDA(w->k_wpos.alloc(nd));
    SF_CUDA(w->err.alloc(64));
    SF_CUDA(cudaMemsetAsync(w->err.p, 0, w->err.bytes(), st));
    SF_CUDA(w->barrier.alloc(4));
    SF_CUDA(cudaMemsetAsync(w->barrier.p, 0, w->barrier.bytes(), st));
    sf_status r = step_create(w.get());   // no load-path state: a pool holds rigid scenes only
    if (r != SF_OK) return r;
    for (uint32_t s = 0; s < n_slots; s++) step_set_live(w.get(), s, false);
    SF_CUDA(cudaStreamSynchronize(st));
    *out = w.release();
    return SF_OK;
}

sf_status sf_pool_load(sf_world *w, uint32_t slot, const sf_scene_desc *d) {
    if (!w) { set_error("null world"); return SF_ERR_ARG; }
    sf_status r = check_slot_scene(w, slot, d);
    if (r != SF_OK) return r;
    const Scene &sc = w->scenes[slot];
    cudaStream_t st = w->stream;
    const uint32_t nbr = d->n_bodies ? d->body_first[d->n_bodies] : 0;
    // static part: the slot's chunk table, its chunks and its static bricks
    std::vector<uint32_t> ctab(NCT, 0), cpool((size_t)sc.n_chunks * 512, 0);
    std::vector<uint32_t> s_cell(sc.n_static, 0);
    std::vector<uint8_t> s_mat(sc.n_static, 0), s_inf(sc.n_static, 0);
    uint32_t used = 0;
    int4 lo = make_int4(1 << 20, 1 << 20, 1 << 20, 0), hi = make_int4(-(1 << 20), -(1 << 20), -(1 << 20), 0);
    for (uint32_t k = 0; k < d->n_static; k++) {
        const int x = d->static_xyz[3 * k], y = d->static_xyz[3 * k + 1], z = d->static_xyz[3 * k + 2];
        uint32_t &t = ctab[chunk_slot(x, y, z)];
        if (t == 0) {
            if (used == sc.n_chunks) { set_error("scene needs more than the slot's %u chunks", sc.n_chunks); return SF_ERR_CAPACITY; }
            t = sc.chunk_off + (++used);
        }
        uint32_t &cell = cpool[(size_t)(t - 1 - sc.chunk_off) * 512 + cell_in_chunk(x, y, z)];
        if (cell) { set_error("static %u: cell (%d,%d,%d) already holds a brick", k, x, y, z); return SF_ERR_ARG; }
        cell = sc.static_off + k + 1;
        s_cell[k] = pack_cell(x, y, z);
        s_mat[k] = d->static_mat[k];
        s_inf[k] = (d->static_mat[k] == GLASS || d->static_infill[k]) ? 1 : 0;
        lo.x = std::min(lo.x, x); lo.y = std::min(lo.y, y); lo.z = std::min(lo.z, z);
        hi.x = std::max(hi.x, x); hi.y = std::max(hi.y, y); hi.z = std::max(hi.z, z);
    }
    w->h_sbox[2 * slot] = lo;
    w->h_sbox[2 * slot + 1] = hi;
    // bodies and bricks; unused bodies dead, unused bricks owned by the sentinel
    std::vector<uint32_t> b_first(sc.n_bodies, 0), b_count(sc.n_bodies, 0), k_body(sc.n_bricks, w->sentinel);
    std::vector<int32_t> k_xyz((size_t)sc.n_bricks * 3, 0);
    std::vector<uint8_t> k_mat(sc.n_bricks, 0);
    for (uint32_t b = 0; b < d->n_bodies; b++) {
        b_first[b] = sc.brick_off + d->body_first[b];
        b_count[b] = d->body_first[b + 1] - d->body_first[b];
    }
    if (nbr) {
        std::memcpy(k_xyz.data(), d->body_brick_xyz, (size_t)nbr * 12);
        std::memcpy(k_mat.data(), d->body_brick_mat, nbr);
    }
    DBuf<float> d_pose;
    SF_CUDA(d_pose.alloc(std::max<size_t>((size_t)d->n_bodies * 13, 1)));
    SF_CUDA(cudaMemcpyAsync(w->ctab.p + (size_t)slot * NCT, ctab.data(), ctab.size() * 4, cudaMemcpyHostToDevice, st));
    if (!cpool.empty()) SF_CUDA(cudaMemcpyAsync(w->cpool.p + (size_t)sc.chunk_off * 512, cpool.data(), cpool.size() * 4, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemcpyAsync(w->sbox.p + 2 * slot, &w->h_sbox[2 * slot], 2 * sizeof(int4), cudaMemcpyHostToDevice, st));
    if (sc.n_static) {
        SF_CUDA(cudaMemcpyAsync(w->s_cell.p + sc.static_off, s_cell.data(), s_cell.size() * 4, cudaMemcpyHostToDevice, st));
        SF_CUDA(cudaMemcpyAsync(w->s_mat.p + sc.static_off, s_mat.data(), s_mat.size(), cudaMemcpyHostToDevice, st));
        SF_CUDA(cudaMemcpyAsync(w->s_infill.p + sc.static_off, s_inf.data(), s_inf.size(), cudaMemcpyHostToDevice, st));
    }
    SF_CUDA(cudaMemcpyAsync(w->b_first.p + sc.body_off, b_first.data(), b_first.size() * 4, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemcpyAsync(w->b_count.p + sc.body_off, b_count.data(), b_count.size() * 4, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemcpyAsync(w->k_body.p + sc.brick_off, k_body.data(), k_body.size() * 4, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemcpyAsync(w->k_xyz.p + (size_t)sc.brick_off * 3, k_xyz.data(), k_xyz.size() * 4, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemcpyAsync(w->k_mat.p + sc.brick_off, k_mat.data(), k_mat.size(), cudaMemcpyHostToDevice, st));
    if (d->n_bodies) SF_CUDA(cudaMemcpyAsync(d_pose.p, d->body_pose, (size_t)d->n_bodies * 52, cudaMemcpyHostToDevice, st));
    SF_CUDA(cudaMemsetAsync(w->b_alive.p + sc.body_off, 0, sc.n_bodies, st));
    SF_CUDA(cudaMemsetAsync(w->b_asleep.p + sc.body_off, 0, sc.n_bodies, st));
    SF_CUDA(cudaMemsetAsync(w->b_wake.p + sc.body_off, 0, sc.n_bodies, st));
    if (d->n_static)
        k_finalize_bricks<<<grid_for(d->n_static, 256), 256, 0, st>>>(d->n_static, sc.static_off, w->s_cell.p,
                                                                      w->s_scene.p, w->s_mat.p, w->s_infill.p,
                                                                      w->s_sid.p, w->ctab.p, w->cpool.p, w->s_nb6.p,
                                                                      w->s_bond.p, w->s_bmax.p);
    if (d->n_bodies)
        SF_CUDA(launch_setup(w, st, d->n_bodies, sc.body_off, nullptr, d_pose.p, 13u));
    w->launches += 2;
    SF_CUDA(cudaGetLastError());
    SF_CUDA(step_reset_labels(w, sc.body_off, sc.n_bodies));
    SF_CUDA(cudaStreamSynchronize(st));   // host vectors and the pose buffer are the copies' sources
    PoolSlot &ps = w->pool[slot];
    ps.bodies = d->n_bodies; ps.bricks = nbr; ps.statics = d->n_static; ps.chunks = used; ps.loaded = true;
    step_set_live(w, slot, d->n_bodies > 0);
    step_warm_invalidate(w, slot);   // another scene's bricks in this slot's ids
    return SF_OK;
}

sf_status sf_pool_clear(sf_world *w, uint32_t slot) {
    if (!w || w->pool.empty() || slot >= w->pool.size()) { set_error("not a pool slot"); return SF_ERR_ARG; }
    const Scene &sc = w->scenes[slot];
    cudaStream_t st = w->stream;
    SF_CUDA(cudaMemsetAsync(w->b_alive.p + sc.body_off, 0, sc.n_bodies, st));
    SF_CUDA(cudaMemsetAsync(w->k_mat.p + sc.brick_off, 0, sc.n_bricks, st));
    SF_CUDA(cudaMemsetAsync(w->ctab.p + (size_t)slot * NCT, 0, (size_t)NCT * 4, st));
    if (sc.n_static) SF_CUDA(cudaMemsetAsync(w->s_mat.p + sc.static_off, 0, sc.n_static, st));
    SF_CUDA(step_reset_labels(w, sc.body_off, sc.n_bodies));
    SF_CUDA(cudaStreamSynchronize(st));
    w->pool[slot] = PoolSlot{};
    step_set_live(w, slot, false);
    step_warm_invalidate(w, slot);
    return SF_OK;
}

sf_status sf_pool_save(sf_world *w, uint32_t slot, void *host, uint64_t cap, uint64_t *bytes) {
    if (!w || w->pool.empty() || slot >= w->pool.size() || !w->pool[slot].loaded) { set_error("no scene in that slot"); return SF_ERR_ARG; }
    const PoolSlot &ps = w->pool[slot];
    const uint64_t need = snapshot_bytes(ps.bodies, ps.bricks);
    if (bytes) *bytes = need;
    if (!host) return SF_OK;
    if (cap < need) { set_error("snapshot needs %llu bytes, buffer holds %llu", (unsigned long long)need, (unsigned long long)cap); return SF_ERR_CAPACITY; }
    SnapPart parts[11];
    snapshot_parts(w, w->scenes[slot], parts);
    uint8_t *o = (uint8_t *)host;
    for (int k = 0; k < 11; k++) {
        const size_t n = (k < 9 ? ps.bodies : ps.bricks) * parts[k].elem;
        if (n) SF_CUDA(cudaMemcpyAsync(o, parts[k].dev, n, cudaMemcpyDeviceToHost, w->stream));
        o += n;
    }
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}

sf_status sf_pool_restore(sf_world *w, uint32_t slot, const sf_scene_desc *d, const void *host, uint64_t bytes) {
    if (!w || !host) { set_error("null argument"); return SF_ERR_ARG; }
    const uint32_t nbr = d && d->n_bodies ? d->body_first[d->n_bodies] : 0;
    if (!d || bytes != snapshot_bytes(d->n_bodies, nbr)) { set_error("snapshot size does not match the scene"); return SF_ERR_ARG; }
    sf_status r = sf_pool_load(w, slot, d);   // the scene's fixed parts (mass, inertia, offsets, static grid)
    if (r != SF_OK) return r;
    SnapPart parts[11];
    snapshot_parts(w, w->scenes[slot], parts);
    const uint8_t *o = (const uint8_t *)host;
    for (int k = 0; k < 11; k++) {
        const size_t n = (k < 9 ? d->n_bodies : nbr) * parts[k].elem;
        if (n) SF_CUDA(cudaMemcpyAsync(parts[k].dev, o, n, cudaMemcpyHostToDevice, w->stream));
        o += n;
    }
    SF_CUDA(cudaStreamSynchronize(w->stream));
    step_set_live(w, slot, true);
    return SF_OK;
}

sf_status sf_pool_write_bodies(sf_world *w, uint32_t slot, const float *state13, const float *sleep, const uint8_t *flags) {
    if (!w || w->pool.empty() || slot >= w->pool.size() || !w->pool[slot].loaded) { set_error("no scene in that slot"); return SF_ERR_ARG; }
    if (!state13 || !sleep || !flags) { set_error("null argument"); return SF_ERR_ARG; }
    sf_status r = write_bodies_range(w, w->scenes[slot].body_off, w->pool[slot].bodies, state13, sleep, flags);
    step_set_live(w, slot, true);
    return r;
}

sf_status sf_pool_read_bodies(sf_world *w, uint32_t slot, float *state13, float *sleep, uint8_t *flags) {
    if (!w || w->pool.empty() || slot >= w->pool.size()) { set_error("not a pool slot"); return SF_ERR_ARG; }
    const PoolSlot &ps = w->pool[slot];
    const Scene &sc = w->scenes[slot];
    const uint32_t nb = ps.bodies;
    if (nb == 0) return SF_OK;
    cudaStream_t s = w->stream;
    SF_CUDA(w->stage13.grow((size_t)nb * 13));
    SF_CUDA(w->stage_flags.grow(nb));
    const uint32_t b = sc.body_off;
    k_pack_bodies<<<grid_for(nb, 256), 256, 0, s>>>(nb, w->b_pos.p + b, w->b_q.p + b, w->b_v.p + b, w->b_w.p + b,
                                                    w->b_alive.p + b, w->b_asleep.p + b, w->stage13.p, w->stage_flags.p);
    w->launches++;
    if (state13) SF_CUDA(cudaMemcpyAsync(state13, w->stage13.p, (size_t)nb * 52, cudaMemcpyDeviceToHost, s));
    if (sleep) SF_CUDA(cudaMemcpyAsync(sleep, w->b_sleep.p + b, (size_t)nb * 4, cudaMemcpyDeviceToHost, s));
    if (flags) SF_CUDA(cudaMemcpyAsync(flags, w->stage_flags.p, nb, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

}  // extern "C"

// Box-box narrow phase, batched: separating-axis test over the 3 + 3 face axes and 9 edge axes, reference/incident
// face clipping or the edge-edge closest points, then reduction to 4 points (engine/src/phys.rs:502-628).
// One thread per pair; the arithmetic keeps the reference's evaluation order (compiled with --fmad=false).
#include <vector>

#include "sf_internal.cuh"
#include "sf_boxsat.cuh"

namespace sf {

__device__ __forceinline__ HShape load_hshape(const float *s, const float4 *hulls) {
    HShape r;
    r.p = p3(s[0], s[1], s[2]);
    const float x = s[3], y = s[4], z = s[5], w = s[6];
    r.c[0] = p3(1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w));
    r.c[1] = p3(2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w));
    r.c[2] = p3(2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y));
    r.h = p3(s[7], s[8], s[9]);
    r.H = hulls + (size_t)(int)s[10] * 80;
    return r;
}

__global__ void __launch_bounds__(128) k_collide_hulls(const float4 *hulls, uint32_t n_hulls, const float *sa, const float *sb,
                                                       uint32_t n, float margin, int do_reduce, float *out36, int32_t *count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *a = sa + (size_t)i * 11, *b = sb + (size_t)i * 11;
    HContact c;
    c.cnt = 0;
    c.n = p3(0.0f, 0.0f, 0.0f);
    const int ta = (int)a[10], tb = (int)b[10];
    if (ta < 0 || (uint32_t)ta >= n_hulls || (b[10] >= 0.0f && (uint32_t)tb >= n_hulls)) { count[i] = -1; return; }
    const HShape A = load_hshape(a, hulls);
    if (b[10] < 0.0f) hull_ground(A, margin, c);
    else hull_hull(A, load_hshape(b, hulls), margin, c);
    if (do_reduce) hc_reduce4(c);
    float *o = out36 + (size_t)i * 36;
    o[0] = c.n.x; o[1] = c.n.y; o[2] = c.n.z; o[3] = 0.0f;
    for (int k = 0; k < 8; k++) {
        const float4 v = k < c.cnt ? c.pt[k] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        o[4 + 4 * k] = v.x; o[5 + 4 * k] = v.y; o[6 + 4 * k] = v.z; o[7 + 4 * k] = v.w;
    }
    count[i] = c.cnt;
}

__global__ void k_collide_boxes(const float *ba, const float *bb, uint32_t n, float margin, float *out20, int32_t *count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Box A = load_box(ba + (size_t)i * 10), B = load_box(bb + (size_t)i * 10);
    CPt pts[8];
    P3 nrm = p3(0.0f, 0.0f, 0.0f);
    int c = collide_boxes(A, B, margin, pts, &nrm);
    if (c) c = reduce4(pts, c, nrm);
    float *o = out20 + (size_t)i * 20;
    o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
    for (int k = 0; k < 4; k++) {
        bool ok = k < c;
        o[4 + 4 * k] = ok ? pts[k].p.x : 0.0f;
        o[5 + 4 * k] = ok ? pts[k].p.y : 0.0f;
        o[6 + 4 * k] = ok ? pts[k].p.z : 0.0f;
        o[7 + 4 * k] = ok ? pts[k].s : 0.0f;
    }
    o[3] = 0.0f;
    count[i] = c;
}

}  // namespace sf

using namespace sf;

extern "C" sf_status sf_collide_boxes(const float *boxes_a, const float *boxes_b, uint32_t n_pairs, float margin, float *out20,
                                      int32_t *count) {
    if (n_pairs == 0) return SF_OK;
    if (!boxes_a || !boxes_b || !out20 || !count) { set_error("null argument"); return SF_ERR_ARG; }
    cudaStream_t s = nullptr;
    SF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DBuf<float> da, db, dout;
    DBuf<int32_t> dc;
    sf_status r = SF_OK;
    do {
        if (da.alloc((size_t)n_pairs * 10) || db.alloc((size_t)n_pairs * 10) || dout.alloc((size_t)n_pairs * 20) || dc.alloc(n_pairs)) {
            set_error("device allocation failed"); r = SF_ERR_CUDA; break;
        }
        cudaMemcpyAsync(da.p, boxes_a, (size_t)n_pairs * 40, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(db.p, boxes_b, (size_t)n_pairs * 40, cudaMemcpyHostToDevice, s);
        k_collide_boxes<<<grid_for(n_pairs, 128), 128, 0, s>>>(da.p, db.p, n_pairs, margin, dout.p, dc.p);
        cudaMemcpyAsync(out20, dout.p, (size_t)n_pairs * 80, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(count, dc.p, (size_t)n_pairs * 4, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error("box SAT: %s", cudaGetErrorString(e)); r = SF_ERR_CUDA; }
    } while (0);
    cudaStreamDestroy(s);
    return r;
}

extern "C" sf_status sf_collide_hulls(const float *hull_data, uint32_t n_hulls, const float *shapes_a, const float *shapes_b,
                                      uint32_t n_pairs, float margin, int32_t reduce, float *out36, int32_t *count) {
    if (n_pairs == 0) return SF_OK;
    if (!hull_data || !n_hulls || !shapes_a || !shapes_b || !out36 || !count) { set_error("null argument"); return SF_ERR_ARG; }
    for (uint32_t i = 0; i < n_pairs; i++) {
        const float ta = shapes_a[(size_t)i * 11 + 10], tb = shapes_b[(size_t)i * 11 + 10];
        if (!(ta >= 0.0f && ta < (float)n_hulls) || !(tb < (float)n_hulls)) { set_error("pair %u: hull id out of range", i); return SF_ERR_ARG; }
    }
    cudaStream_t s = nullptr;
    SF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DBuf<float4> dh;
    DBuf<float> da, db, dout;
    DBuf<int32_t> dc;
    sf_status r = SF_OK;
    do {
        if (dh.alloc((size_t)n_hulls * 80) || da.alloc((size_t)n_pairs * 11) || db.alloc((size_t)n_pairs * 11) ||
            dout.alloc((size_t)n_pairs * 36) || dc.alloc(n_pairs)) {
            set_error("device allocation failed"); r = SF_ERR_CUDA; break;
        }
        cudaMemcpyAsync(dh.p, hull_data, (size_t)n_hulls * 80 * 16, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(da.p, shapes_a, (size_t)n_pairs * 44, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(db.p, shapes_b, (size_t)n_pairs * 44, cudaMemcpyHostToDevice, s);
        k_collide_hulls<<<grid_for(n_pairs, 128), 128, 0, s>>>(dh.p, n_hulls, da.p, db.p, n_pairs, margin, reduce ? 1 : 0, dout.p, dc.p);
        cudaMemcpyAsync(out36, dout.p, (size_t)n_pairs * 36 * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(count, dc.p, (size_t)n_pairs * 4, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { set_error("hull SAT: %s", cudaGetErrorString(e)); r = SF_ERR_CUDA; }
    } while (0);
    cudaStreamDestroy(s);
    return r;
}

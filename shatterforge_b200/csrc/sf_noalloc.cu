// sf_structure_solve_static: the load-path solve of one structure for callers that cannot allocate GPU memory —
// a host engine that gives this library no allocator of its own, or a frame loop that must not allocate once it
// runs. Every device buffer the solve needs lives in one file-scope array below, sized for at most
// SF_STATIC_MAX_BRICKS bricks in SF_STATIC_MAX_CHUNKS chunks of the lattice; the call makes no cudaMalloc or
// cudaFree and no allocating library call. The array is reused by every call and keeps the previous call's contents,
// so each call clears what must start at zero. Two calls whose work overlaps on the GPU race on it.
#include <mutex>

#include "sf_internal.cuh"

namespace sf {
namespace {

constexpr size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t MAXB = SF_STATIC_MAX_BRICKS, MAXC = SF_STATIC_MAX_CHUNKS;
constexpr size_t O_CTAB = 0;
constexpr size_t O_CPOOL = O_CTAB + al256((size_t)NCT * 4);
constexpr size_t O_CHCELL = O_CPOOL + al256(MAXC * 512 * 4);
constexpr size_t O_CHNBR = O_CHCELL + al256(MAXC * 4);
constexpr size_t O_CHSID = O_CHNBR + al256(MAXC * 24);
constexpr size_t O_WORK = O_CHSID + al256(MAXC * 4);
constexpr size_t O_XYZ = O_WORK + al256(MAXC * 4);
constexpr size_t O_CELL = O_XYZ + al256(MAXB * 12);
constexpr size_t O_SCENE = O_CELL + al256(MAXB * 4);
constexpr size_t O_MAT = O_SCENE + al256(MAXB * 4);
constexpr size_t O_INF = O_MAT + al256(MAXB);
constexpr size_t O_SID = O_INF + al256(MAXB);
constexpr size_t O_NB6 = O_SID + al256(MAXB * 4);
constexpr size_t O_BOND = O_NB6 + al256(MAXB * 24);
constexpr size_t O_BMAX = O_BOND + al256(MAXB * 16);
constexpr size_t O_PHI64 = O_BMAX + al256(MAXB * 16);
constexpr size_t O_PHI = O_PHI64 + al256(MAXB * 8);
constexpr size_t O_EXT = O_PHI + al256(MAXB * 4);
constexpr size_t O_CPHI = O_EXT + al256(MAXB * 4);
constexpr size_t O_CRHS = O_CPHI + al256(MAXC * 512 * 8);
constexpr size_t O_CCODE = O_CRHS + al256(MAXC * 512 * 4);
constexpr size_t O_CSID = O_CCODE + al256(MAXC * 512 * 4);
constexpr size_t O_MISC = O_CSID + al256(MAXC * 512 * 4);
// inside the misc block
constexpr size_t M_RESID_BUF = 0, M_SWEEPS = 48, M_RESID = 56, M_ACTIVE = 64, M_BARRIER = 72, M_ERR = 80, M_NCH = 84;
constexpr size_t SCRATCH_BYTES = O_MISC + 256;
static_assert(SCRATCH_BYTES == SF_STATIC_SCRATCH_BYTES, "sf.h states the scratch size");

enum : uint32_t { NA_ERR_CELL = 1u << 8, NA_ERR_DUP = 1u << 9, NA_ERR_CHUNKS = 1u << 10, NA_ERR_MAT = 1u << 11 };

}  // namespace

static __device__ __align__(256) unsigned char g_static_scratch[SCRATCH_BYTES];

__global__ void k_na_mark(uint32_t n, const int32_t *xyz, uint32_t *ctab, uint32_t *err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!inb(x, y, z)) { atomicOr(err, (unsigned)NA_ERR_CELL); return; }
    ctab[chunk_slot(x, y, z)] = 1;
}

// chunk ids in lattice-slot order (one block scans the whole chunk table)
__global__ void __launch_bounds__(1024) k_na_ids(uint32_t *ctab, uint32_t *chunk_cell, uint32_t *nch, uint32_t *err) {
    __shared__ uint32_t part[1024];
    const uint32_t per = (NCT + 1023) / 1024;
    const uint32_t s0 = threadIdx.x * per, s1 = min((uint32_t)NCT, s0 + per);
    uint32_t c = 0;
    for (uint32_t k = s0; k < s1; k++) c += ctab[k] != 0;
    part[threadIdx.x] = c;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
        uint32_t v = threadIdx.x >= o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t id = part[threadIdx.x] - c;
    for (uint32_t k = s0; k < s1; k++) {
        if (!ctab[k]) continue;
        if (id < MAXC) {
            ctab[k] = id + 1;
            const int cx = (int)(k % CXN), cz = (int)((k / CXN) % CZN), cy = (int)(k / (CXN * CZN));
            chunk_cell[id] = pack_cell(cx * 8, cy * 8, cz * 8);
        } else {
            ctab[k] = 0;
            atomicOr(err, (unsigned)NA_ERR_CHUNKS);
        }
        id++;
    }
    if (threadIdx.x == 1023) *nch = part[1023];
}

__global__ void k_na_fill(uint32_t n, const int32_t *xyz, const uint32_t *ctab, uint32_t *cpool, uint32_t *cell,
                          uint32_t *scene, int32_t *sid, const uint8_t *mat, uint8_t *infill, uint32_t *err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!inb(x, y, z)) return;
    if (mat[i] == 0 || mat[i] > 8) atomicOr(err, (unsigned)NA_ERR_MAT);
    uint32_t t = ctab[chunk_slot(x, y, z)];
    if (t == 0) return;
    if (atomicCAS(&cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)], 0u, i + 1) != 0u) atomicOr(err, (unsigned)NA_ERR_DUP);
    cell[i] = pack_cell(x, y, z);
    scene[i] = 0;
    sid[i] = 0;
    infill[i] = (mat[i] == GLASS || infill[i]) ? 1 : 0;
}

__global__ void k_na_meta(const uint32_t *nch_p, const uint32_t *chunk_cell, const uint32_t *ctab, int32_t *chunk_nbr,
                          int32_t *chunk_sid, uint32_t *work, uint32_t *active) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) *active = 1;
    if (c >= *nch_p) return;
    const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    int x, y, z;
    unpack_cell(chunk_cell[c], x, y, z);
    for (int d = 0; d < 6; d++) {
        int nx = x + 8 * D[d][0], ny = y + 8 * D[d][1], nz = z + 8 * D[d][2];
        uint32_t t = inb(nx, ny, nz) ? ctab[chunk_slot(nx, ny, nz)] : 0u;
        chunk_nbr[(size_t)c * 6 + d] = t ? (int32_t)(t - 1) : -1;
    }
    chunk_sid[c] = 0;
    work[c] = c;
}

// the array's device address, looked up once per device with that device current (host code may not use the
// symbol itself as a pointer)
static std::mutex g_na_mu;
static unsigned char *g_na_base[64] = {};

static sf_status na_base(unsigned char **out) {
    int dev = 0;
    SF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { set_error("device ordinal %d out of range", dev); return SF_ERR_ARG; }
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_base[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p) { set_error("cudaGetSymbolAddress failed: %s", cudaGetErrorString(e)); return SF_ERR_CUDA; }
        g_na_base[dev] = (unsigned char *)p;
    }
    *out = g_na_base[dev];
    return SF_OK;
}

}  // namespace sf

using namespace sf;

extern "C" sf_status sf_structure_solve_static(uint32_t n_bricks, const int32_t *xyz, const uint8_t *mat, const uint8_t *infill,
                                               const float *ext, float omega, float tol, uint32_t max_sweeps, double *phi_out,
                                               uint32_t *sweeps_out, double *resid_out, void *stream) {
    if (sweeps_out) *sweeps_out = 0;
    if (resid_out) *resid_out = 0.0;
    if (n_bricks == 0) return SF_OK;
    if (!xyz || !mat || !infill || !phi_out) { set_error("null argument"); return SF_ERR_ARG; }
    if (n_bricks > SF_STATIC_MAX_BRICKS) {
        set_error("%u bricks exceed the scratch-free solve's maximum of %d", n_bricks, SF_STATIC_MAX_BRICKS);
        return SF_ERR_CAPACITY;
    }
    if (!(omega > 0.0f && omega < 2.0f)) { set_error("omega %g outside (0, 2)", (double)omega); return SF_ERR_ARG; }
    unsigned char *base = nullptr;
    sf_status st = na_base(&base);
    if (st != SF_OK) return st;
    int dev = 0, sms = 0;
    SF_CUDA(cudaGetDevice(&dev));
    SF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t *ctab = (uint32_t *)(base + O_CTAB), *cpool = (uint32_t *)(base + O_CPOOL);
    uint32_t *chunk_cell = (uint32_t *)(base + O_CHCELL), *work = (uint32_t *)(base + O_WORK);
    int32_t *chunk_nbr = (int32_t *)(base + O_CHNBR), *chunk_sid = (int32_t *)(base + O_CHSID);
    int32_t *d_xyz = (int32_t *)(base + O_XYZ);
    uint32_t *cell = (uint32_t *)(base + O_CELL), *scene = (uint32_t *)(base + O_SCENE);
    uint8_t *d_mat = base + O_MAT, *d_inf = base + O_INF;
    int32_t *sid = (int32_t *)(base + O_SID);
    uint32_t *nb6 = (uint32_t *)(base + O_NB6);
    float *bond = (float *)(base + O_BOND), *bmax = (float *)(base + O_BMAX), *phi = (float *)(base + O_PHI);
    float *d_ext = (float *)(base + O_EXT);
    double *phi64 = (double *)(base + O_PHI64), *cphi = (double *)(base + O_CPHI);
    float *crhs = (float *)(base + O_CRHS);
    uint32_t *ccode = (uint32_t *)(base + O_CCODE);
    int32_t *csid = (int32_t *)(base + O_CSID);
    unsigned char *misc = base + O_MISC;
    uint32_t *err = (uint32_t *)(misc + M_ERR), *nch_d = (uint32_t *)(misc + M_NCH);
    // what must start at zero: the chunk table, the chunk pool, the potentials, the counters and the barrier
    SF_CUDA(cudaMemsetAsync(ctab, 0, (size_t)NCT * 4, s));
    SF_CUDA(cudaMemsetAsync(cpool, 0, MAXC * 512 * 4, s));
    SF_CUDA(cudaMemsetAsync(phi64, 0, (size_t)n_bricks * 8, s));
    SF_CUDA(cudaMemsetAsync(phi, 0, (size_t)n_bricks * 4, s));
    SF_CUDA(cudaMemsetAsync(misc, 0, 256, s));
    SF_CUDA(cudaMemcpyAsync(d_xyz, xyz, (size_t)n_bricks * 12, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(d_mat, mat, n_bricks, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(d_inf, infill, n_bricks, cudaMemcpyHostToDevice, s));
    if (ext) SF_CUDA(cudaMemcpyAsync(d_ext, ext, (size_t)n_bricks * 4, cudaMemcpyHostToDevice, s));
    else SF_CUDA(cudaMemsetAsync(d_ext, 0, (size_t)n_bricks * 4, s));
    k_na_mark<<<grid_for(n_bricks, 256), 256, 0, s>>>(n_bricks, d_xyz, ctab, err);
    k_na_ids<<<1, 1024, 0, s>>>(ctab, chunk_cell, nch_d, err);
    k_na_fill<<<grid_for(n_bricks, 256), 256, 0, s>>>(n_bricks, d_xyz, ctab, cpool, cell, scene, sid, d_mat, d_inf, err);
    SF_CUDA(cudaGetLastError());
    uint32_t h[2] = {0, 0};   // error bits, chunk count
    SF_CUDA(cudaMemcpyAsync(h, misc + M_ERR, 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    if (h[0] & NA_ERR_CELL) { set_error("a brick lies outside the 640 x 136 x 640 lattice"); return SF_ERR_ARG; }
    if (h[0] & NA_ERR_MAT) { set_error("a brick has a material outside 1..8"); return SF_ERR_ARG; }
    if (h[0] & NA_ERR_DUP) { set_error("two bricks share a lattice cell"); return SF_ERR_ARG; }
    if ((h[0] & NA_ERR_CHUNKS) || h[1] > SF_STATIC_MAX_CHUNKS) {
        set_error("the bricks occupy %u chunks of 8^3 cells; the scratch-free solve holds at most %d", h[1], SF_STATIC_MAX_CHUNKS);
        return SF_ERR_CAPACITY;
    }
    const uint32_t nch = h[1];
    SF_CUDA(finalize_on_buffers(n_bricks, cell, scene, d_mat, d_inf, sid, ctab, cpool, nb6, bond, bmax, s));
    k_na_meta<<<grid_for(nch, 128), 128, 0, s>>>(nch_d, chunk_cell, ctab, chunk_nbr, chunk_sid, work, (uint32_t *)(misc + M_ACTIVE));
    SF_CUDA(cudaGetLastError());
    SorBuffers B;
    B.cell = cell; B.scene = scene; B.ctab = ctab; B.mat = d_mat; B.sid = sid; B.nb6 = nb6; B.bond = bond; B.ext = d_ext;
    B.phi64 = phi64; B.phi = phi; B.cphi = cphi; B.crhs = crhs; B.ccode = ccode; B.csid = csid; B.chunk_nbr = chunk_nbr;
    B.chunk_sid = chunk_sid; B.work = work; B.active0 = (const uint32_t *)(misc + M_ACTIVE);
    B.resid_buf = (unsigned long long *)(misc + M_RESID_BUF); B.sweeps = (uint32_t *)(misc + M_SWEEPS);
    B.resid = (double *)(misc + M_RESID); B.gb = (GridBarrier *)(misc + M_BARRIER); B.err = err;
    SF_CUDA(sor_solve_on_buffers(B, n_bricks, nch, omega, tol, max_sweeps, sms, s));
    uint32_t sw = 0, e2 = 0;
    double rs = 0.0;
    SF_CUDA(cudaMemcpyAsync(phi_out, phi64, (size_t)n_bricks * 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(&sw, misc + M_SWEEPS, 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(&rs, misc + M_RESID, 8, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(&e2, misc + M_ERR, 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    if (sweeps_out) *sweeps_out = sw;
    if (resid_out) *resid_out = rs;
    if (e2 & ERR_TIMEOUT) { set_error("a device barrier wait timed out"); return SF_ERR_TIMEOUT; }
    if (e2 & ERR_SOR_NONFINITE) { set_error("non-finite potential (ungrounded piece?)"); return SF_ERR_VERIFY; }
    return SF_OK;
}

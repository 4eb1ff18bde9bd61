// Load path: scalar potential-flow SOR and the joint checks (src/lib.rs:1005-1040, 1142-1227).
//
// Layout. The solve runs on the sparse chunk grid itself (src/lib.rs:302-321): every occupied 8^3 chunk owns 512
// cells of four arrays —
//   cphi  f64   the potential (the reference keeps f32; f32 stalls above a 1e-5 relative error on tall frames,
//               so the device iterates in f64 on the reference's f32 coefficients)
//   crhs  f32   MASS[mat] + ext (the constant part of sor_brick's numerator)
//   ccode u32   six 4-bit link codes (the material whose STIFF is the smaller of the pair; 0 = no link), the
//               cell's own material in bits 24-27 and the foundation bit 28
//   csid  i32   structure id of the cell (-1 = not a structure brick)
// — 16 B of reads per brick and 8 B of writes per sweep; links never need an index array because a link always
// goes to the face-adjacent cell, in this chunk or in the neighbour chunk recorded in chunk_nbr.
//
// Order. The reference sweeps Gauss-Seidel in brick-index order. Here the sweep is red-black: every lattice link
// joins cells of opposite parity (x + y + z), so all red cells are independent given the black ones and vice
// versa. Each cell's update keeps sor_brick's arithmetic (links in the direction order +x, -x, +y, -y, +z, -z,
// then the foundation term; target = ((MASS + ext) + sum k phi) / sum k). The iteration converges to the same
// fixed point as the reference's; tests compare against an FP64 solve of the same system.
//
// Residual. As sor_struct: max |dphi| over the sweep divided by max(phi, 1) over the structure, per structure.
#include <algorithm>
#include <cstring>

#include <cooperative_groups.h>

#include "sf_internal.cuh"

namespace sf {

// omega, tolerance and sweep limit of a solve, read from device memory (so a captured graph serves every solve of its
// shape); use_cap != 0: structure q also stops after cap[q] sweeps (the per-frame schedules give each structure
// its own count)
struct SorParams { double omega, tol; uint32_t max_sweeps, use_cap; };

struct SorState {
    DBuf<double> cphi;
    DBuf<float> crhs;
    DBuf<uint32_t> ccode;
    DBuf<int32_t> csid;
    DBuf<int32_t> chunk_nbr;        // 6 per chunk
    DBuf<int32_t> chunk_sid;        // the one structure a chunk's bricks belong to, -2 = several, -1 = none
    DBuf<uint32_t> work;            // chunk ids of the current solve
    DBuf<unsigned long long> resid_buf;  // [3][2][n_struct]: md, mp as f64 bits
    DBuf<uint32_t> sweeps;          // per structure
    DBuf<double> resid;             // per structure, last sweep
    DBuf<uint32_t> active0;         // per structure: 1 = solve it
    DBuf<uint32_t> st_count;        // bricks per structure
    std::vector<uint32_t> h_st_count;
    std::vector<uint32_t> st_chunk_start, st_chunk_list, all_chunks;
    // joints: 4 per static brick
    DBuf<float> j_ratio, j_bond;
    DBuf<uint8_t> j_dec;
    DBuf<uint32_t> j_crushed;
    DBuf<uint32_t> cand_flag, cand_pos, cand_list;
    DBuf<uint32_t> counters;        // joints, over, failed, crushed, maxr bits, ncand
    DBuf<uint32_t> st_req;          // requested structures list for the apply pass
    // resting-body loads
    DBuf<float> extn, share;
    DBuf<uint32_t> lcount;          // per body: bricks resting on a listed structure, bricks on the ground
    DBuf<uint64_t> lkey, lkey_alt;
    DBuf<uint32_t> lval, lval_alt;
    Work wk;
    uint64_t launches = 0;
    int occ = 1;
    Tuner tune;   // blocks per SM of the red-black kernel, keyed on log2(chunks of the solve)
    // The solve's launch sequence captured in CUDA graphs, one per launch shape (the chunk list and the active
    // flags live in device buffers the graph reads, so a graph serves every solve of its shape).
    // a graph's launch shape: the chunk count or structure count, the grid of the red-black kernel, the path, and
    // per cluster launch class its cluster count and cells a block (the structure order lives in device memory)
    struct Graph { uint32_t n_work, grid, mode; uint32_t shape[8]; cudaGraphExec_t exec; };
    // the cluster path: one thread-block cluster per structure, the structure's cells in the cluster's shared memory
    bool cl_ready = false;
    bool wide_ok = false;           // the device can run 16-block clusters of the wide structures
    std::vector<uint32_t> h_cl_n, h_cl_per, h_cl_ncl;   // per structure: cells, cells a block, blocks of its cluster
    // per structure: its height in cells, and the sweeps its last solve took (0 = none yet); the launch split puts
    // the structures expected to take longest on the larger blocks
    std::vector<uint32_t> h_st_height, h_last_sweeps;
    DBuf<uint32_t> cl_cpos, cl_off, cl_n, cl_per, cl_even, cl_list;
    DBuf<uint16_t> cl_nbr;
    uint64_t cluster_solves = 0;
    // the small structures' clusters run beside the large ones', on a second stream forked from and joined to the
    // world's stream (inside the captured graph too)
    cudaStream_t aux[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
    DBuf<SorParams> prm;
    DBuf<uint32_t> cap;             // per structure: its own sweep limit when SorParams::use_cap is set
    // the reference's per-frame schedule (src/lib.rs:1061-1079, 1268-1281): per structure its pending warm-up
    // sweeps, whether it has been solved (warmed), its settle timer and the residual of its last sweep
    std::vector<int32_t> h_warm;
    std::vector<uint8_t> h_solved;
    std::vector<float> h_settle;
    std::vector<double> h_resid;
    std::vector<Graph> graphs;
    bool graphs_ok = true;
    uint64_t graph_launches = 0;
};

const Tuner *sor_tuner(const SorState *st) { return st ? &st->tune : nullptr; }

enum : uint8_t { J_HOLD = 0, J_FATIGUE = 1, J_FAIL = 2, J_CRUSH = 3, J_ABSENT = 255 };

__device__ __forceinline__ uint32_t cell_of_static(const uint32_t *ctab, uint32_t scene, uint32_t packed, uint32_t &chunk) {
    int x, y, z;
    unpack_cell(packed, x, y, z);
    chunk = ctab[(size_t)scene * NCT + chunk_slot(x, y, z)] - 1;
    return cell_in_chunk(x, y, z);
}

// ---------------------------------------------------------------- prepare: bricks -> chunk cells
__global__ void k_sor_clear(uint32_t ncells, uint32_t *ccode, int32_t *csid) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncells) return;
    ccode[i] = 0;
    csid[i] = -1;
}

__global__ void k_sor_scatter(uint32_t ns, const uint32_t *cell, const uint32_t *scene, const uint8_t *mat,
                              const int32_t *sid, const uint32_t *nb6, const float *bond, const double *phi,
                              const float *ext, const uint32_t *ctab, double *cphi, float *crhs, uint32_t *ccode,
                              int32_t *csid) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    uint8_t mi = mat[i];
    if (mi == 0) return;
    uint32_t chunk;
    uint32_t c = cell_of_static(ctab, scene[i], cell[i], chunk);
    size_t at = (size_t)chunk * 512 + c;
    cphi[at] = phi[i];
    int32_t s = sid[i];
    if (s < 0 || mi >= SLUG) return;
    uint32_t code = 0;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        uint32_t j = nb6[(size_t)i * 6 + d];
        if (j == NONE) continue;
        uint8_t mj = mat[j];
        if (mj == 0) continue;
        float hp = (d & 1) == 0 ? bond[(size_t)i * 4 + (d >> 1)] : bond[(size_t)j * 4 + (d >> 1)];
        if (!(hp > 0.0f)) continue;
        uint32_t lm = c_mat.stiff[mi] < c_mat.stiff[mj] ? mi : mj;
        code |= lm << (4 * d);
    }
    int x, y, z;
    unpack_cell(cell[i], x, y, z);
    code |= (uint32_t)mi << 24;
    if (y == 0 && bond[(size_t)i * 4 + 3] > 0.0f) code |= 1u << 28;
    ccode[at] = code;
    csid[at] = s;
    crhs[at] = c_mat.mass[mi] + ext[i];
}

__global__ void k_sor_gather(uint32_t ns, const uint32_t *cell, const uint32_t *scene, const uint8_t *mat, const int32_t *sid,
                             const uint32_t *active, const uint32_t *ctab, const double *cphi, double *phi64, float *phi) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    int32_t s = sid[i];
    if (mat[i] == 0 || s < 0 || !active[s]) return;
    uint32_t chunk;
    uint32_t c = cell_of_static(ctab, scene[i], cell[i], chunk);
    double v = cphi[(size_t)chunk * 512 + c];
    phi64[i] = v;
    phi[i] = (float)v;
}

__global__ void k_sor_init(uint32_t nst, unsigned long long *resid_buf, uint32_t *sweeps, double *resid) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nst) return;
    for (int b = 0; b < 3; b++) {
        resid_buf[(size_t)(b * 2) * nst + s] = 0ull;
        resid_buf[(size_t)(b * 2 + 1) * nst + s] = (unsigned long long)__double_as_longlong(1.0);
    }
    sweeps[s] = 0;
    resid[s] = 0.0;
}

// ext += value, in list order (a brick listed twice gets both, in order)
__global__ void k_add_loads(uint32_t n, const uint32_t *brick, const float *value, float *ext) {
    if (blockIdx.x * blockDim.x + threadIdx.x != 0) return;
    for (uint32_t k = 0; k < n; k++) ext[brick[k]] += value[k];
}

// ---------------------------------------------------------------- the persistent red-black kernel
constexpr int SOR_BLOCK = 256;
constexpr int SOR_MAX_LOCAL_STRUCT = 8192;   // active flags kept in shared memory as bits

struct SorArgs {
    const uint32_t *cap;
    double *cphi;
    const float *crhs;
    const uint32_t *ccode;
    const int32_t *csid;
    const int32_t *chunk_nbr;
    const int32_t *chunk_sid;
    const uint32_t *work;
    uint32_t n_work;
    uint32_t n_struct;
    const uint32_t *active0;
    unsigned long long *resid_buf;
    uint32_t *sweeps;
    double *resid;
    double omega, tol;
    uint32_t max_sweeps;
    const SorParams *prm;          // when set, omega / tol / max_sweeps are read from here (a captured graph's launch
                                   // then serves every parameter set)
    GridBarrier *gb;
    uint32_t *err;
};

__device__ __forceinline__ bool is_active(const uint32_t *bits, int32_t s) { return (bits[s >> 5] >> (s & 31)) & 1u; }

// block-wide max of (d, p) for one structure, one atomic pair per block (non-negative f64 bits order as u64)
__device__ __forceinline__ void sor_flush(int32_t s, unsigned long long d, unsigned long long p, unsigned long long *md,
                                          unsigned long long *mp) {
    __shared__ unsigned long long sd[SOR_BLOCK / 32], sp[SOR_BLOCK / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
        p = max(p, __shfl_xor_sync(0xffffffffu, p, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sd[wid] = d; sp[wid] = p; }
    __syncthreads();
    if (threadIdx.x == 0 && s >= 0) {
        unsigned long long dm = 0, pm = 0;
        for (int k = 0; k < SOR_BLOCK / 32; k++) { dm = max(dm, sd[k]); pm = max(pm, sp[k]); }
        if (dm) atomicMax(&md[s], dm);
        if (pm) atomicMax(&mp[s], pm);
    }
    __syncthreads();
}

// Potentials written by other blocks during the launch are read with ld.global.cg (L2), never through L1.
// Work: chunk ids sorted by (structure, chunk); each block owns a contiguous range, so its maxima stay in
// registers while the structure is unchanged. Chunks holding bricks of several structures (chunk_sid = -2) fall
// back to per-cell atomics.
__global__ void __launch_bounds__(SOR_BLOCK) k_sor_redblack(SorArgs A) {
    __shared__ uint32_t act[SOR_MAX_LOCAL_STRUCT / 32];
    __shared__ int s_any;
    const uint32_t nst = A.n_struct;
    const uint32_t nwords = (nst + 31) / 32;
    for (uint32_t k = threadIdx.x; k < nwords; k += blockDim.x) act[k] = 0;
    __syncthreads();
    for (uint32_t s = threadIdx.x; s < nst; s += blockDim.x) if (A.active0[s]) atomicOr(&act[s >> 5], 1u << (s & 31));
    __syncthreads();
    const int t = threadIdx.x;
    const int ly = t >> 5, lz = (t >> 2) & 7, lxp = (t & 3) << 1;
    const float axis_f[3] = {0.3f, 1.0f, 0.3f};
    const uint32_t per = (A.n_work + gridDim.x - 1) / gridDim.x;
    const uint32_t w0 = min(A.n_work, blockIdx.x * per), w1 = min(A.n_work, w0 + per);
    const unsigned long long one = (unsigned long long)__double_as_longlong(1.0);
    const double omega = A.prm ? A.prm->omega : A.omega, tol = A.prm ? A.prm->tol : A.tol;
    const uint32_t max_sweeps = A.prm ? A.prm->max_sweeps : A.max_sweeps;
    for (uint32_t sweep = 0; sweep < max_sweeps; sweep++) {
        unsigned long long *md = A.resid_buf + (size_t)((sweep % 3) * 2) * nst;
        unsigned long long *mp = md + nst;
        if (blockIdx.x == 0) {
            unsigned long long *nmd = A.resid_buf + (size_t)(((sweep + 1) % 3) * 2) * nst;
            for (uint32_t s = threadIdx.x; s < nst; s += blockDim.x) { nmd[s] = 0ull; nmd[nst + s] = one; }
        }
        for (int colour = 0; colour < 2; colour++) {
            const int lx = lxp | ((ly + lz + colour) & 1);
            const int cell = (ly * 8 + lz) * 8 + lx;
            int32_t cur = -1;
            unsigned long long accd = 0, accp = 0;
            for (uint32_t wi = w0; wi < w1; wi++) {
                const uint32_t chunk = A.work[wi];
                const int32_t cs = A.chunk_sid[chunk];
                if (cs != cur) {
                    sor_flush(cur, accd, accp, md, mp);
                    cur = cs; accd = 0; accp = 0;
                }
                if (cs >= 0 && !is_active(act, cs)) continue;
                const size_t at = (size_t)chunk * 512 + cell;
                const int32_t s = A.csid[at];
                if (s < 0 || !is_active(act, s)) continue;
                const uint32_t code = A.ccode[at];
                double sk = 0.0, skp = 0.0;
#pragma unroll
                for (int d = 0; d < 6; d++) {
                    const uint32_t lm = (code >> (4 * d)) & 15u;
                    if (lm == 0) continue;
                    const int ax = d >> 1;
                    const int sg = (d & 1) ? -1 : 1;
                    int nx = lx, ny = ly, nz = lz;
                    if (ax == 0) nx += sg; else if (ax == 1) ny += sg; else nz += sg;
                    size_t nat;
                    if (nx >= 0 && nx < 8 && ny >= 0 && ny < 8 && nz >= 0 && nz < 8) {
                        nat = (size_t)chunk * 512 + (ny * 8 + nz) * 8 + nx;
                    } else {
                        const int32_t nc = A.chunk_nbr[(size_t)chunk * 6 + d];
                        if (nc < 0) { atomicOr(A.err, (unsigned)ERR_SOR_NONFINITE); continue; }
                        nat = (size_t)nc * 512 + (((ny & 7) * 8 + (nz & 7)) * 8 + (nx & 7));
                    }
                    // cond (src/lib.rs:1142): the f32 conductance, promoted
                    const double k = (double)(c_mat.stiff[lm] * axis_f[ax]);
                    sk += k;
                    skp += k * __ldcg(&A.cphi[nat]);
                }
                const uint32_t mi = (code >> 24) & 15u;
                if (code & (1u << 28)) sk += (double)c_mat.gk[mi];
                double p = __ldcg(&A.cphi[at]);
                double dabs = 0.0;
                if (sk > 0.0) {
                    const double target = ((double)A.crhs[at] + skp) / sk;
                    const double dd = omega * (target - p);
                    p += dd;
                    A.cphi[at] = p;
                    dabs = fabs(dd);
                    if (!isfinite(p)) atomicOr(A.err, (unsigned)ERR_SOR_NONFINITE);
                }
                const unsigned long long db = (unsigned long long)__double_as_longlong(dabs);
                const unsigned long long pb = p > 0.0 ? (unsigned long long)__double_as_longlong(p) : 0ull;
                if (cs >= 0) { accd = max(accd, db); accp = max(accp, pb); }
                else { if (db) atomicMax(&md[s], db); if (pb) atomicMax(&mp[s], pb); }
            }
            sor_flush(cur, accd, accp, md, mp);
            if (!grid_sync(A.gb, gridDim.x, A.err)) return;
        }
        // convergence: every block evaluates the same maxima and drops the same structures
        if (threadIdx.x == 0) s_any = 0;
        __syncthreads();
        for (uint32_t s = threadIdx.x; s < nst; s += blockDim.x) {
            if (!is_active(act, (int32_t)s)) continue;
            const double r = __longlong_as_double((long long)__ldcg(&md[s])) / __longlong_as_double((long long)__ldcg(&mp[s]));
            if (blockIdx.x == 0) { A.sweeps[s] = sweep + 1; A.resid[s] = r; }
            const uint32_t lim = (A.prm && A.prm->use_cap && A.cap) ? min(max_sweeps, A.cap[s]) : max_sweeps;
            if (r < tol || sweep + 1 >= lim) atomicAnd(&act[s >> 5], ~(1u << (s & 31)));
            else s_any = 1;
        }
        __syncthreads();
        if (!s_any) break;
    }
}

// ---------------------------------------------------------------- one cluster per structure
// A structure of up to SOR_CL x SOR_CL_CAP bricks is solved by one cluster of SOR_CL blocks that hold its cells in
// shared memory for the whole solve: cells listed in space order, split in SOR_CL contiguous ranges (one per
// block), each range with its even-parity cells first. A half-sweep updates one parity; a neighbour in another block
// of the cluster is read from that block's shared memory; a cluster barrier (hardware, no spin) separates the
// halves, and the one that ends a sweep also publishes each block's residual maxima (two barriers per sweep). The
// largest structures' clusters are listed first. Each update is the grid kernel's arithmetic on the same values in the same order, and the residual and
// stopping rule are the same, so the potentials and sweep counts are identical to the grid kernel's.
constexpr int SOR_CL = 8;                        // blocks of a structure's cluster, or SOR_CL_WIDE for large ones
constexpr int SOR_CL_WIDE = 16;                  // a non-portable cluster size: structures of SOR_CL_WIDE_MIN bricks
constexpr uint32_t SOR_CL_WIDE_MIN = 20000;
constexpr int SOR_CL_MAX_THREADS = 1024;         // threads per block: 256, 512 or 1024, picked per launch
constexpr uint32_t SOR_CL_CAP = 8192;            // cells per block: 28 B each (phi 8, rhs 4, code 4, 6 neighbours 12)
constexpr uint32_t SOR_CL_BYTES_PER_CELL = 28;
constexpr uint32_t SOR_CL_SPLIT = 1024;          // cells per block above which a structure counts as large
constexpr uint32_t CELL_ACTIVE = 1u << 31;
constexpr uint16_t NO_CELL = 0xFFFFu;

struct SorClusterArgs {
    const uint32_t *cap;                         // per structure sweep limits (when prm->use_cap)
    const uint32_t *list;                        // the structure of each cluster
    const uint32_t *off, *n, *per, *even;        // per structure; even: per (structure, block)
    const uint32_t *cpos;                        // per listed cell: its place in the chunk layout
    const uint16_t *nbr;                         // per listed cell: 6 neighbours as block rank << sh | index in block,
                                                 // sh = 13 for 8-block clusters, 12 for 16-block ones
    double *cphi;
    const float *crhs;
    const uint32_t *ccode;
    const int32_t *csid;
    uint32_t per_max;
    const SorParams *prm;
    uint32_t *sweeps;
    double *resid;
    uint32_t *err;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
// the address of the same shared-memory location in block `rank` of the cluster
__device__ __forceinline__ uint32_t mapa_shared(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ double ld_cluster_f64(uint32_t a) {
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}

// threads per block for a launch whose largest block range holds per_max cells: about two cells per thread and sweep
static unsigned sor_cl_threads(uint32_t per_max) {
    const uint32_t half = per_max / 2;
    return half > 512 ? 1024u : half > 256 ? 512u : 256u;
}

__global__ void __launch_bounds__(SOR_CL_MAX_THREADS) k_sor_cluster(SorClusterArgs A) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char sm[];
    const uint32_t P = A.per_max;
    double *phi = (double *)sm;
    float *rhs = (float *)(phi + P);
    uint32_t *code = (uint32_t *)(rhs + P);
    uint16_t *nbr = (uint16_t *)(code + P);
    // this block's maxima of sweep s in slot s & 1, published before the barrier that ends the sweep; after it,
    // warp 0 of every block reads all the cluster's blocks' slots and takes the stop decision (the same everywhere)
    __shared__ unsigned long long blk_d[2], blk_p[2];
    __shared__ unsigned long long wd[SOR_CL_MAX_THREADS / 32], wp[SOR_CL_MAX_THREADS / 32];
    __shared__ int s_stop;
    // conductances as f64: kt[2 lm + (axis is y)] = STIFF[lm] x axis factor (the f32 product, promoted), kt[32 + m]
    // = the foundation conductance of material m
    __shared__ double kt[48];
    for (uint32_t k = threadIdx.x; k < 16; k += blockDim.x) {
        const float st = k < 9 ? c_mat.stiff[k] : 0.0f;
        kt[2 * k] = (double)(st * 0.3f);
        kt[2 * k + 1] = (double)(st * 1.0f);
        kt[32 + k] = k < 9 ? (double)c_mat.gk[k] : 0.0;
    }
    const unsigned long long one = (unsigned long long)__double_as_longlong(1.0);
    const uint32_t rank = cl.block_rank(), tid = threadIdx.x;
    const uint32_t ncl = cl.num_blocks();        // 8 or 16: the structure's tables were cut for this many blocks
    const uint32_t sh = ncl == (uint32_t)SOR_CL_WIDE ? 12u : 13u, lmask = (1u << sh) - 1u;
    const uint32_t q = A.list[blockIdx.x / ncl];
    const uint32_t off = A.off[q], n = A.n[q], per = A.per[q];
    const uint32_t b0 = min(n, rank * per), b1 = min(n, b0 + per), my = b1 - b0;
    const uint32_t ev = A.even[q * SOR_CL_WIDE + rank];
    // the shared::cluster address of every block's potentials: a neighbour's is s_base[its rank] + 8 x its index
    __shared__ uint32_t s_base[SOR_CL_WIDE];
    if (tid < ncl) s_base[tid] = mapa_shared(smem_addr(phi), tid);
    for (uint32_t i = tid; i < my; i += blockDim.x) {
        const uint32_t g = off + b0 + i;
        const uint32_t at = A.cpos[g];
        phi[i] = A.cphi[at];
        rhs[i] = A.crhs[at];
        const uint32_t cd = A.csid[at] == (int32_t)q ? (A.ccode[at] | CELL_ACTIVE) : 0u;
        code[i] = cd;
        // a face without a neighbour cell of this structure has no link (link code 0, conductance 0); it reads the
        // cell's own potential, so every update does its six loads without a branch and adds zeros for the faces
        // without a link (x + 0 = x: the sums are the grid kernel's)
#pragma unroll
        for (int d = 0; d < 6; d++) {
            uint16_t nb = A.nbr[(size_t)g * 6 + d];
            if (nb == NO_CELL) {
                if ((cd & CELL_ACTIVE) && ((cd >> (4 * d)) & 15u)) atomicOr(A.err, (unsigned)ERR_SOR_NONFINITE);
                nb = (uint16_t)((rank << sh) | i);
            }
            nbr[i * 6 + d] = nb;
        }
    }
    const double omega = A.prm->omega, tol = A.prm->tol;
    const uint32_t max_sweeps = A.prm->use_cap ? min(A.prm->max_sweeps, A.cap[q]) : A.prm->max_sweeps;
    double r_last = 0.0;
    uint32_t done = 0;
    cl.sync();
    for (uint32_t sweep = 0; sweep < max_sweeps; sweep++) {
        unsigned long long accd = 0ull, accp = 0ull;
        // One cell's update: the new potential (unchanged when it has no conductance) and |dphi|. Cells of one
        // colour never read each other, so a thread computes two of them before it stores either: the two
        // dependent f64 chains (neighbour loads, divide) overlap.
        auto update = [&](uint32_t i, double &p, double &dabs) -> bool {
            const uint32_t cd = code[i];
            if (!(cd & CELL_ACTIVE)) return false;
            double pj[6];
#pragma unroll
            for (int d = 0; d < 6; d++) {
                const uint32_t g = nbr[i * 6 + d];
                pj[d] = ld_cluster_f64(s_base[g >> sh] + ((g & lmask) << 3));
            }
            double sk = 0.0, skp = 0.0;
#pragma unroll
            for (int d = 0; d < 6; d++) {
                const double k = kt[2 * ((cd >> (4 * d)) & 15u) + ((d >> 1) == 1 ? 1 : 0)];
                sk += k;
                skp += k * pj[d];
            }
            sk += (cd & (1u << 28)) ? kt[32 + ((cd >> 24) & 15u)] : 0.0;
            p = phi[i];
            dabs = 0.0;
            if (sk > 0.0) {
                const double target = ((double)rhs[i] + skp) / sk;
                const double dd = omega * (target - p);
                p += dd;
                dabs = fabs(dd);
                if (!isfinite(p)) atomicOr(A.err, (unsigned)ERR_SOR_NONFINITE);
            }
            return true;
        };
        for (int colour = 0; colour < 2; colour++) {
            const uint32_t c0 = colour ? ev : 0u, c1 = colour ? my : ev;
            for (uint32_t i = c0 + tid; i < c1; i += 2 * blockDim.x) {
                const uint32_t i2 = i + blockDim.x;
                double p1 = 0.0, d1 = 0.0, p2 = 0.0, d2 = 0.0;
                const bool a1 = update(i, p1, d1);
                const bool a2 = i2 < c1 && update(i2, p2, d2);
                if (a1) {
                    phi[i] = p1;
                    accd = max(accd, (unsigned long long)__double_as_longlong(d1));
                    if (p1 > 0.0) accp = max(accp, (unsigned long long)__double_as_longlong(p1));
                }
                if (a2) {
                    phi[i2] = p2;
                    accd = max(accd, (unsigned long long)__double_as_longlong(d2));
                    if (p2 > 0.0) accp = max(accp, (unsigned long long)__double_as_longlong(p2));
                }
            }
            if (colour == 0) cl.sync();
        }
        // the cluster's maxima of this sweep. Slot sweep & 1 is next written two sweeps later, after the next
        // sweep's first barrier, which no block passes before it has read the slot.
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            accd = max(accd, __shfl_xor_sync(0xffffffffu, accd, o));
            accp = max(accp, __shfl_xor_sync(0xffffffffu, accp, o));
        }
        if ((tid & 31) == 0) { wd[tid >> 5] = accd; wp[tid >> 5] = accp; }
        __syncthreads();
        const uint32_t slot = sweep & 1u;
        // the block's maxima: warp 0 reduces the warps' values with shuffles (max is exact in any order)
        if (tid < 32) {
            const uint32_t nw = blockDim.x / 32;
            unsigned long long dm = tid < nw ? wd[tid] : 0ull, pm = tid < nw ? wp[tid] : one;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                dm = max(dm, __shfl_xor_sync(0xffffffffu, dm, o));
                pm = max(pm, __shfl_xor_sync(0xffffffffu, pm, o));
            }
            if (tid == 0) { blk_d[slot] = dm; blk_p[slot] = pm; }
        }
        cl.sync();
        // the cluster's maxima: lane b of warp 0 reads block b's slot (the eight remote reads in flight together)
        if (tid < 32) {
            unsigned long long dm = 0ull, pm = one;
            if (tid < ncl) {
                dm = cl.map_shared_rank(blk_d, tid)[slot];
                pm = cl.map_shared_rank(blk_p, tid)[slot];
            }
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) {
                dm = max(dm, __shfl_xor_sync(0xffffffffu, dm, o));
                pm = max(pm, __shfl_xor_sync(0xffffffffu, pm, o));
            }
            if (tid == 0) {
                r_last = __longlong_as_double((long long)dm) / __longlong_as_double((long long)pm);
                s_stop = (r_last < tol || sweep + 1 >= max_sweeps) ? 1 : 0;
            }
        }
        done = sweep + 1;
        __syncthreads();
        if (s_stop) break;
    }
    for (uint32_t i = tid; i < my; i += blockDim.x)
        if (code[i] & CELL_ACTIVE) A.cphi[A.cpos[off + b0 + i]] = phi[i];
    if (rank == 0 && tid == 0 && done) { A.sweeps[q] = done; A.resid[q] = r_last; }
    cl.sync();   // every block's shared memory outlives the other blocks' reads of it
}

// ---------------------------------------------------------------- joint checks
struct StressArgs {
    uint32_t ns;
    const uint32_t *cell;
    const uint8_t *mat;
    const int32_t *sid;
    const uint32_t *nb6;
    const float *bond, *bmax, *phi;
    const uint32_t *active;
    float dt;
    int live;
    float *ratio, *bond_after;
    uint8_t *dec;
    uint32_t *crushed, *cand_flag;
};

// every joint evaluated as if nothing failed before it; failures are applied in reference order afterwards
__global__ void k_stress_eval(StressArgs A) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.ns) return;
    uint8_t mi = A.mat[i];
    int32_t s = A.sid[i];
    bool in = mi != 0 && mi < SLUG && s >= 0 && A.active[s];
    uint32_t flag = 0;
    int x, y, z;
    unpack_cell(A.cell[i], x, y, z);
    for (int a = 0; a < 3; a++) {
        size_t o = (size_t)i * 4 + a;
        uint8_t dec = J_ABSENT;
        float r = 0.0f, hpo = 0.0f;
        uint32_t kc = NONE;
        uint32_t j = in ? A.nb6[(size_t)i * 6 + a * 2] : NONE;
        if (j != NONE && A.mat[j] != 0) {
            float hp = A.bond[o];
            if (hp > 0.0f) {
                uint8_t mj = A.mat[j];
                float k = minf(c_mat.stiff[mi], c_mat.stiff[mj]) * (a == 1 ? 1.0f : 0.3f);
                float f = k * (A.phi[i] - A.phi[j]);
                float u = a == 1 ? 1.0f : 0.0f;
                float up = f > 0.0f ? maxf(u, 0.0f) : maxf(-u, 0.0f);
                float tens = minf(c_mat.tens[mi], c_mat.tens[mj]);
                float capm = 1.0f - (1.0f - tens) * up;
                r = div_rn(fabsf(f), hp * capm);
                dec = J_HOLD;
                hpo = hp;
                if (A.live && r > 1.0f) {
                    float nhp = hp - hp * A.dt * 2.2f * minf(r - 0.85f, 2.5f);
                    if (nhp < A.bmax[o] * 0.08f) {
                        if (up == 0.0f && fabsf(u) > 0.5f) { dec = J_CRUSH; kc = c_mat.capv[mj] < c_mat.capv[mi] ? j : i; }
                        else { dec = J_FAIL; hpo = 0.0f; }
                    } else { dec = J_FATIGUE; hpo = nhp; }
                    flag = 1;
                }
            }
        }
        A.ratio[o] = r; A.bond_after[o] = hpo; A.dec[o] = dec; A.crushed[o] = kc;
    }
    {
        size_t o = (size_t)i * 4 + 3;
        uint8_t dec = J_ABSENT;
        float r = 0.0f, b3 = 0.0f;
        if (in && y == 0 && A.bond[o] > 0.0f) {
            float f = c_mat.gk[mi] * A.phi[i];
            b3 = A.bond[o];
            r = div_rn(f, b3);
            dec = J_HOLD;
            if (A.live && r > 1.0f) {
                b3 = b3 - b3 * A.dt * 2.2f * (r - 0.85f);
                if (b3 < A.bmax[o] * 0.08f) { b3 = 0.0f; dec = J_FAIL; } else dec = J_FATIGUE;
                flag = 1;
            }
        }
        A.ratio[o] = r; A.bond_after[o] = b3; A.dec[o] = dec; A.crushed[o] = NONE;
    }
    A.cand_flag[i] = flag;
}

__global__ void k_stress_compact(uint32_t ns, const uint32_t *flag, const uint32_t *pos, uint32_t *list) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ns && flag[i]) list[pos[i]] = i;
}

__device__ __forceinline__ bool joint_later(uint32_t i2, int a2, uint32_t i, int a) { return i2 > i || (i2 == i && a2 > a); }

// Reference-order application of the over-stressed joints (src/lib.rs:1182-1222): a compressive crush removes a
// brick at once, so every later joint that touches it disappears, and the crushing brick's own remaining joints
// are not evaluated (stress_brick returns). The crush budget of 300 per pass turns later crushes into failures.
__global__ void k_stress_apply(const uint32_t *cand, const uint32_t *ncand_p, const uint32_t *req, uint32_t nreq,
                               const int32_t *sid, uint8_t *mat, const uint32_t *nb6, const uint32_t *cell,
                               const uint32_t *scene, const uint32_t *ctab, uint32_t *cpool, float *bond, uint8_t *dec,
                               float *bond_after, uint32_t *crushed, uint8_t *conn) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t ncand = *ncand_p;
    uint32_t crush_n = 0;
    for (uint32_t r = 0; r < nreq; r++) {
        int32_t s = (int32_t)req[r];
        for (uint32_t c = 0; c < ncand; c++) {
            uint32_t i = cand[c];
            if (sid[i] != s) continue;
            for (int a = 0; a < 4; a++) {
                size_t o = (size_t)i * 4 + a;
                uint8_t d = dec[o];
                if (d == J_ABSENT || d == J_HOLD) continue;
                if (mat[i] == 0) { dec[o] = J_ABSENT; continue; }
                if (d == J_CRUSH) {
                    if (crush_n >= 300) { d = J_FAIL; dec[o] = J_FAIL; bond_after[o] = 0.0f; crushed[o] = NONE; }
                    else {
                        crush_n++;
                        conn[s] = 1;   // a removed brick may split the structure (remove_brick, src/lib.rs:705-718)
                        uint32_t k = crushed[o];
                        mat[k] = 0;
                        uint32_t chunk;
                        uint32_t cc = cell_of_static(ctab, scene[k], cell[k], chunk);
                        cpool[(size_t)chunk * 512 + cc] = 0;
                        // the rest of brick i's joints
                        for (int a2 = a + 1; a2 < 4; a2++) dec[(size_t)i * 4 + a2] = J_ABSENT;
                        // brick k's own joints, if it comes later
                        if (k > i) for (int a2 = 0; a2 < 4; a2++) dec[(size_t)k * 4 + a2] = J_ABSENT;
                        // joints of the bricks below k along each axis, pointing at k
                        for (int a2 = 0; a2 < 3; a2++) {
                            uint32_t i2 = nb6[(size_t)k * 6 + a2 * 2 + 1];
                            if (i2 != NONE && joint_later(i2, a2, i, a)) dec[(size_t)i2 * 4 + a2] = J_ABSENT;
                        }
                        break;
                    }
                }
                bond[o] = bond_after[o];
                if (d == J_FAIL) conn[s] = 1;   // a broken joint may split the structure (src/lib.rs:1202, 1223)
            }
        }
    }
}

__global__ void k_stress_tally(uint32_t ns, const uint8_t *dec, const float *ratio, const uint32_t *nb6,
                               const int32_t *sid, const uint32_t *active, float *stress, uint32_t *counters) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    int32_t s = sid[i];
    if (s < 0 || !active[s]) return;
    uint32_t nj = 0, over = 0, fail = 0, crush = 0;
    float mr = 0.0f;
    for (int a = 0; a < 4; a++) {
        size_t o = (size_t)i * 4 + a;
        uint8_t d = dec[o];
        if (d == J_ABSENT) continue;
        float r = ratio[o];
        nj++;
        if (r > 1.0f) over++;
        if (d == J_FAIL) fail++;
        if (d == J_CRUSH) crush++;
        mr = maxf(mr, r);
        atomicMax((unsigned *)&stress[i], __float_as_uint(r));
        if (a < 3) atomicMax((unsigned *)&stress[nb6[(size_t)i * 6 + a * 2]], __float_as_uint(r));
    }
    if (nj) {
        atomicAdd(&counters[0], nj);
        if (over) atomicAdd(&counters[1], over);
        if (fail) atomicAdd(&counters[2], fail);
        if (crush) atomicAdd(&counters[3], crush);
        atomicMax(&counters[4], __float_as_uint(mr));
    }
}

__global__ void k_stress_zero(uint32_t ns, const int32_t *sid, const uint8_t *mat, const uint32_t *active, float *stress) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    int32_t s = sid[i];
    if (s >= 0 && mat[i] != 0 && active[s]) stress[i] = 0.0f;
}

// ---------------------------------------------------------------- resting-body loads (src/lib.rs:1233-1259)
// A body resting on bricks of listed structures spreads its weight over those bricks and the ground: each brick of
// the body whose cell 0.29 m below holds a static brick of a listed structure counts once (ns), each brick within
// RB + 0.05 of the ground once (nground), and every such static brick receives m / (ns + nground).
__device__ __forceinline__ uint32_t load_target(const float4 p, uint32_t sc, const uint32_t *ctab, const uint32_t *cpool,
                                                const uint8_t *smat, const int32_t *sid, const uint32_t *listed) {
    const float yy = p.y - RB - 0.02f;
    const int x = __float2int_rz(floorf(p.x / S)) + NX / 2, y = __float2int_rz(floorf(yy / S)), z = __float2int_rz(floorf(p.z / S)) + NZ / 2;
    if (!inb(x, y, z)) return NONE;
    const uint32_t t = ctab[(size_t)sc * NCT + chunk_slot(x, y, z)];
    if (t == 0) return NONE;
    const uint32_t g = cpool[(size_t)(t - 1) * 512 + cell_in_chunk(x, y, z)];
    if (g == 0) return NONE;
    const uint32_t j = g - 1;
    if (smat[j] == 0) return NONE;
    const int32_t s = sid[j];
    return (s >= 0 && listed[s]) ? j : NONE;
}

// per body: its bricks with a listed static brick below (ns) and its bricks on the ground (ng), counted brick by brick
// (a body of tens of thousands of bricks would otherwise be one thread's loop)
__global__ void k_loads_count(uint32_t nd, const uint32_t *kbody, const uint8_t *alive, const uint32_t *bscene,
                              const float4 *wpos, const uint32_t *ctab, const uint32_t *cpool, const uint8_t *smat,
                              const int32_t *sid, const uint32_t *listed, uint32_t *cnt2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = kbody[i];
    if (!alive[b]) return;
    const float4 p = wpos[i];
    if (p.y < RB + 0.05f) atomicAdd(&cnt2[2 * b + 1], 1u);
    if (load_target(p, bscene[b], ctab, cpool, smat, sid, listed) != NONE) atomicAdd(&cnt2[2 * b], 1u);
}

// a body's weight share per supported brick: m / (ns + ng), none when no brick rests on a listed structure
__global__ void k_loads_share(uint32_t nb, const uint8_t *alive, const float *m, const uint32_t *cnt2, float *share) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    float sh = 0.0f;
    if (alive[b]) {
        const uint32_t ns = cnt2[2 * b], ng = cnt2[2 * b + 1];
        if (ns) sh = div_rn(m[b], (float)(ns + ng));
    }
    share[b] = sh;
}

__global__ void k_loads_keys(uint32_t nd, uint64_t none_key, const uint32_t *kbody, const uint32_t *bscene, const float4 *wpos,
                             const float *share, const uint32_t *ctab, const uint32_t *cpool, const uint8_t *smat,
                             const int32_t *sid, const uint32_t *listed, uint64_t *key, uint32_t *val) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint32_t b = kbody[i];
    uint64_t k = none_key;
    if (share[b] > 0.0f) {
        const uint32_t j = load_target(wpos[i], bscene[b], ctab, cpool, smat, sid, listed);
        if (j != NONE) k = j;
    }
    key[i] = k;
    val[i] = i;
}

// each static brick sums its shares in body order, then brick order (the keys were sorted stably by brick id)
__global__ void k_loads_sum(uint32_t nd, uint64_t none_key, const uint64_t *key, const uint32_t *val, const uint32_t *kbody,
                            const float *share, float *extn) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nd) return;
    const uint64_t k = key[p];
    if (k >= none_key || (p > 0 && key[p - 1] == k)) return;
    float s = 0.0f;
    for (uint32_t q = p; q < nd && key[q] == k; q++) s += share[kbody[val[q]]];
    extn[k] = s;
}

__global__ void k_loads_apply(uint32_t ns, const int32_t *sid, const uint8_t *mat, const uint32_t *listed, const float *extn,
                              float *ext) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns) return;
    const int32_t s = sid[i];
    if (s < 0 || !listed[s]) return;
    ext[i] = ext[i] * 0.8f + extn[i] * 0.2f;
}

// ---------------------------------------------------------------- host side
sf_status sor_create(sf_world *w) {
    SorState *st = new SorState();
    w->sor = st;
    SF_CUDA(upload_mat_tables(w->stream));
    uint32_t nch = w->n_chunks, nst = w->n_struct;
    cudaStream_t s = w->stream;
    // chunk neighbours (host; the grid is static)
    std::vector<int32_t> nbr((size_t)nch * 6, -1);
    std::vector<uint32_t> h_ctab;
    if (nch) {
        h_ctab.resize((size_t)w->n_scenes * NCT);
        SF_CUDA(cudaMemcpyAsync(h_ctab.data(), w->ctab.p, h_ctab.size() * 4, cudaMemcpyDeviceToHost, s));
        SF_CUDA(cudaStreamSynchronize(s));
    }
    const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (uint32_t c = 0; c < nch; c++) {
        int x, y, z;
        unpack_cell(w->h_chunk_cell[c], x, y, z);
        uint32_t sc = w->h_chunk_scene[c];
        for (int d = 0; d < 6; d++) {
            int nx = x + 8 * D[d][0], ny = y + 8 * D[d][1], nz = z + 8 * D[d][2];
            if (!inb(nx, ny, nz)) continue;
            uint32_t t = h_ctab[(size_t)sc * NCT + chunk_slot(nx, ny, nz)];
            if (t) nbr[(size_t)c * 6 + d] = (int32_t)(t - 1);
        }
    }
    SF_CUDA(st->prm.alloc(1));
    SF_CUDA(st->cap.alloc(std::max<uint32_t>(nst, 1)));
    st->h_warm.assign(nst, 0);
    st->h_solved.assign(nst, 0);
    st->h_settle.assign(nst, 0.0f);
    st->h_resid.assign(nst, 0.0);
    SF_CUDA(st->chunk_nbr.alloc(nbr.size()));
    if (!nbr.empty()) SF_CUDA(cudaMemcpyAsync(st->chunk_nbr.p, nbr.data(), nbr.size() * 4, cudaMemcpyHostToDevice, s));
    // chunks of each structure
    std::vector<std::vector<uint32_t>> per(nst);
    st->h_st_count.assign(nst, 0);
    std::vector<int32_t> csole(nch, -1);
    for (uint32_t i = 0; i < w->ns; i++) {
        int32_t sid = w->h_sid[i];
        if (sid < 0) continue;
        int x, y, z;
        unpack_cell(w->h_s_cell[i], x, y, z);
        uint32_t sc = 0;
        // scene of brick i: find by static offset
        for (uint32_t q = 0; q < w->n_scenes; q++)
            if (i >= w->scenes[q].static_off && i < w->scenes[q].static_off + w->scenes[q].n_static) { sc = q; break; }
        uint32_t c = h_ctab[(size_t)sc * NCT + chunk_slot(x, y, z)] - 1;
        if (per[sid].empty() || per[sid].back() != c) per[sid].push_back(c);
        st->h_st_count[sid]++;
        csole[c] = csole[c] == -1 ? sid : (csole[c] == sid ? sid : -2);
    }
    st->st_chunk_start.assign(nst + 1, 0);
    for (uint32_t q = 0; q < nst; q++) {
        std::sort(per[q].begin(), per[q].end());
        per[q].erase(std::unique(per[q].begin(), per[q].end()), per[q].end());
        st->st_chunk_start[q + 1] = st->st_chunk_start[q] + (uint32_t)per[q].size();
        st->st_chunk_list.insert(st->st_chunk_list.end(), per[q].begin(), per[q].end());
    }
    for (uint32_t c = 0; c < nch; c++) if (csole[c] != -1) st->all_chunks.push_back(c);
    std::stable_sort(st->all_chunks.begin(), st->all_chunks.end(), [&](uint32_t x, uint32_t y) { return csole[x] < csole[y]; });
    SF_CUDA(st->chunk_sid.alloc(nch));
    if (nch) SF_CUDA(cudaMemcpyAsync(st->chunk_sid.p, csole.data(), nch * 4, cudaMemcpyHostToDevice, s));
    size_t ncell = (size_t)nch * 512;
    SF_CUDA(st->cphi.alloc(ncell)); SF_CUDA(st->crhs.alloc(ncell)); SF_CUDA(st->ccode.alloc(ncell)); SF_CUDA(st->csid.alloc(ncell));
    SF_CUDA(cudaMemsetAsync(st->cphi.p, 0, st->cphi.bytes(), s));
    SF_CUDA(cudaMemsetAsync(st->crhs.p, 0, st->crhs.bytes(), s));
    SF_CUDA(st->work.alloc(std::max<size_t>(st->all_chunks.size(), 1)));
    SF_CUDA(st->resid_buf.alloc((size_t)6 * std::max<uint32_t>(nst, 1)));
    SF_CUDA(st->sweeps.alloc(std::max<uint32_t>(nst, 1)));
    SF_CUDA(st->resid.alloc(std::max<uint32_t>(nst, 1)));
    SF_CUDA(st->active0.alloc(std::max<uint32_t>(nst, 1)));
    SF_CUDA(st->st_req.alloc(std::max<uint32_t>(nst, 1)));
    size_t nj = (size_t)std::max<uint32_t>(w->ns, 1) * 4;
    SF_CUDA(st->j_ratio.alloc(nj)); SF_CUDA(st->j_bond.alloc(nj)); SF_CUDA(st->j_dec.alloc(nj)); SF_CUDA(st->j_crushed.alloc(nj));
    SF_CUDA(cudaMemsetAsync(st->j_dec.p, 0xFF, st->j_dec.bytes(), s));
    SF_CUDA(st->cand_flag.alloc(std::max<uint32_t>(w->ns, 1) + 1));
    SF_CUDA(st->cand_pos.alloc(std::max<uint32_t>(w->ns, 1) + 1));
    SF_CUDA(st->cand_list.alloc(std::max<uint32_t>(w->ns, 1)));
    SF_CUDA(st->counters.alloc(16));
    int occ = 0;
    SF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sor_redblack, SOR_BLOCK, 0));
    st->occ = std::max(1, occ);
    {
        int c[4], n = 0;
        for (int v : {1, 2, 4, 8}) if (v <= st->occ) c[n++] = v;
        if (n == 0 || c[n - 1] != st->occ) { if (n == 4) n = 3; c[n++] = st->occ; }
        st->tune.init(c, n);
    }
    if (nst > (uint32_t)SOR_MAX_LOCAL_STRUCT) { set_error("more than %d structures", SOR_MAX_LOCAL_STRUCT); return SF_ERR_CAPACITY; }
    return SF_OK;
}

// The red-black solve of one structure (id 0) on caller-provided chunk-layout buffers: no allocation, used by the
// scratch-free entry point. Uploads this unit's material tables first (a copy to a constant symbol, no allocation).
cudaError_t sor_solve_on_buffers(const SorBuffers &B, uint32_t n_bricks, uint32_t n_chunks, float omega, float tol,
                                 uint32_t max_sweeps, int sms, cudaStream_t s) {
    cudaError_t e = upload_mat_tables(s);
    if (e != cudaSuccess) return e;
    const uint32_t ncell = n_chunks * 512;
    k_sor_clear<<<grid_for(ncell, 256), 256, 0, s>>>(ncell, B.ccode, B.csid);
    k_sor_scatter<<<grid_for(n_bricks, 256), 256, 0, s>>>(n_bricks, B.cell, B.scene, B.mat, B.sid, B.nb6, B.bond, B.phi64,
                                                          B.ext, B.ctab, B.cphi, B.crhs, B.ccode, B.csid);
    k_sor_init<<<1, 32, 0, s>>>(1, B.resid_buf, B.sweeps, B.resid);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int occ = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sor_redblack, SOR_BLOCK, 0)) != cudaSuccess) return e;
    SorArgs A;
    A.cphi = B.cphi; A.crhs = B.crhs; A.ccode = B.ccode; A.csid = B.csid; A.chunk_nbr = B.chunk_nbr; A.chunk_sid = B.chunk_sid;
    A.work = B.work; A.n_work = n_chunks; A.n_struct = 1; A.active0 = B.active0; A.resid_buf = B.resid_buf;
    A.sweeps = B.sweeps; A.resid = B.resid; A.omega = (double)omega; A.tol = (double)tol; A.max_sweeps = max_sweeps;
    A.prm = nullptr; A.cap = nullptr; A.gb = B.gb; A.err = B.err;
    unsigned grid = (unsigned)std::min<size_t>(n_chunks, (size_t)sms * std::max(occ, 1));
    void *args[] = {&A};
    if ((e = cudaLaunchCooperativeKernel((void *)k_sor_redblack, dim3(grid), dim3(SOR_BLOCK), args, 0, s)) != cudaSuccess) return e;
    k_sor_gather<<<grid_for(n_bricks, 256), 256, 0, s>>>(n_bricks, B.cell, B.scene, B.mat, B.sid, B.active0, B.ctab, B.cphi,
                                                         B.phi64, B.phi);
    return cudaGetLastError();
}

uint64_t sor_launches(const SorState *st) { return st ? st->wk.launches + st->launches : 0; }
uint64_t sor_graph_launches(const SorState *st) { return st ? st->graph_launches : 0; }
void sor_reset_launches(SorState *st) { if (st) { st->wk.launches = 0; st->launches = 0; } }

void sor_destroy(sf_world *w) {
    if (w->sor) {
        for (auto &g : w->sor->graphs) cudaGraphExecDestroy(g.exec);
        if (w->sor->fork) cudaEventDestroy(w->sor->fork);
        for (int k = 0; k < 3; k++) {
            if (w->sor->join[k]) cudaEventDestroy(w->sor->join[k]);
            if (w->sor->aux[k]) cudaStreamDestroy(w->sor->aux[k]);
        }
    }
    delete w->sor;
    w->sor = nullptr;
}

// which structures a call covers, and the chunk list of that set
static sf_status sor_select(sf_world *w, int32_t structure, std::vector<uint32_t> &act, std::vector<uint32_t> &chunks,
                            std::vector<uint32_t> &req) {
    SorState *st = w->sor;
    uint32_t nst = w->n_struct;
    act.assign(std::max<uint32_t>(nst, 1), 0);
    chunks.clear();
    req.clear();
    if (structure >= 0) {
        if ((uint32_t)structure >= nst) { set_error("structure %d does not exist", structure); return SF_ERR_ARG; }
        if (st->h_st_count[structure]) {
            act[structure] = 1;
            req.push_back((uint32_t)structure);
            chunks.assign(st->st_chunk_list.begin() + st->st_chunk_start[structure],
                          st->st_chunk_list.begin() + st->st_chunk_start[structure + 1]);
        }
    } else {
        for (uint32_t q = 0; q < nst; q++) if (st->h_st_count[q]) { act[q] = 1; req.push_back(q); }
        chunks = st->all_chunks;
    }
    return SF_OK;
}

// a list of structures (each at most once)
static sf_status sor_select_set(sf_world *w, const int32_t *ids, uint32_t n, std::vector<uint32_t> &act,
                                std::vector<uint32_t> &chunks, std::vector<uint32_t> &req) {
    SorState *st = w->sor;
    uint32_t nst = w->n_struct;
    act.assign(std::max<uint32_t>(nst, 1), 0);
    chunks.clear();
    req.clear();
    for (uint32_t k = 0; k < n; k++) {
        const int32_t q = ids[k];
        if (q < 0 || (uint32_t)q >= nst) { set_error("structure %d does not exist", q); return SF_ERR_ARG; }
        if (act[q]) { set_error("structure %d listed twice", q); return SF_ERR_ARG; }
        if (!st->h_st_count[q]) continue;
        act[q] = 1;
        req.push_back((uint32_t)q);
        chunks.insert(chunks.end(), st->st_chunk_list.begin() + st->st_chunk_start[q],
                      st->st_chunk_list.begin() + st->st_chunk_start[q + 1]);
    }
    return SF_OK;
}

// The cluster path's tables, built on its first use: each structure's bricks in lattice order (chunk slot, cell in
// chunk), cut into SOR_CL ranges with each range's even-parity cells first; every listed cell's place in the chunk
// layout and its six neighbours' indices in the list (NO_CELL for none, or a brick of another structure). A structure
// with more than 65,535 bricks takes the grid kernel.
static sf_status sor_cluster_tables(sf_world *w) {
    SorState *st = w->sor;
    SF_CUDA(cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(SOR_CL_CAP * SOR_CL_BYTES_PER_CELL)));
    SF_CUDA(cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    SF_CUDA(cudaFuncSetAttribute(k_sor_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    {
        // 16-block clusters only where the device can hold one (1,024-thread blocks with a wide structure's shared
        // memory); otherwise every structure keeps 8-block tables
        cudaLaunchConfig_t c = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = SOR_CL_WIDE; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
        c.gridDim = dim3(SOR_CL_WIDE);
        c.blockDim = dim3(SOR_CL_MAX_THREADS);
        c.dynamicSmemBytes = (size_t)4096 * SOR_CL_BYTES_PER_CELL;
        c.attrs = at;
        c.numAttrs = 1;
        int nc = 0;
        if (cudaOccupancyMaxActiveClusters(&nc, k_sor_cluster, &c) != cudaSuccess) { nc = 0; cudaGetLastError(); }
        st->wide_ok = nc > 0;
    }
    const uint32_t nst = w->n_struct, ns = w->ns;
    std::vector<uint32_t> h_ctab((size_t)w->n_scenes * NCT), h_cpool((size_t)std::max<uint32_t>(w->n_chunks, 1) * 512);
    SF_CUDA(cudaStreamSynchronize(w->stream));
    SF_CUDA(cudaMemcpy(h_ctab.data(), w->ctab.p, h_ctab.size() * 4, cudaMemcpyDeviceToHost));
    if (w->n_chunks) SF_CUDA(cudaMemcpy(h_cpool.data(), w->cpool.p, (size_t)w->n_chunks * 512 * 4, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> scene_of(ns, 0);
    for (uint32_t q = 0; q < w->n_scenes; q++)
        for (uint32_t i = 0; i < w->scenes[q].n_static; i++) scene_of[w->scenes[q].static_off + i] = q;
    std::vector<std::vector<uint32_t>> bricks(nst);
    for (uint32_t i = 0; i < ns; i++) if (w->h_sid[i] >= 0) bricks[w->h_sid[i]].push_back(i);
    auto key = [&](uint32_t i) {
        int x, y, z;
        unpack_cell(w->h_s_cell[i], x, y, z);
        return (uint64_t)chunk_slot(x, y, z) * 512 + cell_in_chunk(x, y, z);
    };
    auto cpos_of = [&](uint32_t sc, int x, int y, int z) -> uint32_t {   // (chunk << 9 | cell) or NONE
        if (!inb(x, y, z)) return NONE;
        const uint32_t t = h_ctab[(size_t)sc * NCT + chunk_slot(x, y, z)];
        return t ? ((t - 1) << 9) | cell_in_chunk(x, y, z) : NONE;
    };
    std::vector<uint32_t> idx(ns, NONE), cpos, even(std::max<size_t>((size_t)nst * SOR_CL_WIDE, 1), 0);
    std::vector<uint16_t> nbr;
    st->h_cl_n.assign(nst, 0);
    st->h_cl_per.assign(nst, 0);
    st->h_cl_ncl.assign(nst, SOR_CL);
    st->h_st_height.assign(nst, 0);
    st->h_last_sweeps.assign(nst, 0);
    std::vector<uint32_t> off(std::max<uint32_t>(nst, 1), 0), cnt(std::max<uint32_t>(nst, 1), 0), per(std::max<uint32_t>(nst, 1), 0);
    const int D[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (uint32_t q = 0; q < nst; q++) {
        // links join bricks of one structure only (a bond needs equal structure ids), so every link of a listed
        // cell ends at a listed cell
        std::vector<uint32_t> &b = bricks[q];
        if (b.empty() || b.size() >= NO_CELL) continue;
        std::sort(b.begin(), b.end(), [&](uint32_t u, uint32_t v) { return key(u) < key(v); });
        const uint32_t n = (uint32_t)b.size();
        const uint32_t ncl = (st->wide_ok && n >= SOR_CL_WIDE_MIN) ? (uint32_t)SOR_CL_WIDE : (uint32_t)SOR_CL;
        const uint32_t pr = (n + ncl - 1) / ncl, sh = ncl == (uint32_t)SOR_CL_WIDE ? 12u : 13u;
        st->h_cl_ncl[q] = ncl;
        for (uint32_t r = 0; r < ncl; r++) {
            auto lo = b.begin() + std::min(n, r * pr), hi = b.begin() + std::min(n, (r + 1) * pr);
            auto mid = std::stable_partition(lo, hi, [&](uint32_t i) {
                int x, y, z;
                unpack_cell(w->h_s_cell[i], x, y, z);
                return ((x + y + z) & 1) == 0;
            });
            even[(size_t)q * SOR_CL_WIDE + r] = (uint32_t)(mid - lo);
        }
        off[q] = (uint32_t)cpos.size();
        cnt[q] = n;
        per[q] = pr;
        for (uint32_t k = 0; k < n; k++) idx[b[k]] = k;
        for (uint32_t k = 0; k < n; k++) {
            const uint32_t i = b[k], sc = scene_of[i];
            int x, y, z;
            unpack_cell(w->h_s_cell[i], x, y, z);
            cpos.push_back(cpos_of(sc, x, y, z));
            for (int d = 0; d < 6; d++) {
                const uint32_t c = cpos_of(sc, x + D[d][0], y + D[d][1], z + D[d][2]);
                uint16_t g = NO_CELL;
                if (c != NONE) {
                    const uint32_t j1 = h_cpool[(size_t)(c >> 9) * 512 + (c & 511)];
                    if (j1 && w->h_sid[j1 - 1] == (int32_t)q) {
                        const uint32_t t = idx[j1 - 1];
                        // pr <= 8192 (8 blocks) or 4096 (16): the index fits sh bits, and the last block holds
                        // fewer than pr cells, so no neighbour packs to NO_CELL
                        g = (uint16_t)(((t / pr) << sh) | (t % pr));
                    }
                }
                nbr.push_back(g);
            }
        }
        st->h_cl_n[q] = n;
        st->h_cl_per[q] = pr;
        int ylo = NY, yhi = -1;
        for (uint32_t k = 0; k < n; k++) {
            int x, y, z;
            unpack_cell(w->h_s_cell[b[k]], x, y, z);
            ylo = std::min(ylo, y); yhi = std::max(yhi, y);
        }
        st->h_st_height[q] = (uint32_t)(yhi - ylo + 1);
    }
    // places in the chunk layout as chunk * 512 + cell
    for (uint32_t &c : cpos) c = (c >> 9) * 512 + (c & 511);
    cudaStream_t s = w->stream;
    auto up32 = [&](DBuf<uint32_t> &d, const std::vector<uint32_t> &h) -> cudaError_t {
        cudaError_t e = d.alloc(std::max<size_t>(h.size(), 1));
        if (e == cudaSuccess && !h.empty()) e = cudaMemcpyAsync(d.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, s);
        return e;
    };
    SF_CUDA(up32(st->cl_cpos, cpos));
    SF_CUDA(up32(st->cl_off, off));
    SF_CUDA(up32(st->cl_n, cnt));
    SF_CUDA(up32(st->cl_per, per));
    SF_CUDA(up32(st->cl_even, even));
    SF_CUDA(st->cl_list.alloc(std::max<uint32_t>(nst, 1)));
    SF_CUDA(st->cl_nbr.alloc(std::max<size_t>(nbr.size(), 1)));
    if (!nbr.empty()) SF_CUDA(cudaMemcpyAsync(st->cl_nbr.p, nbr.data(), nbr.size() * 2, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaStreamSynchronize(s));
    st->cl_ready = true;
    return SF_OK;
}

// caps (optional, n_struct entries): structure q stops after at most caps[q] sweeps (max_sweeps bounds them all)
static sf_status solve_impl(sf_world *w, int32_t structure, const int32_t *ids, uint32_t n_ids, float omega, float tol,
                            uint32_t max_sweeps, sf_solve_report *report, const uint32_t *caps = nullptr) {
    if (!w) return SF_ERR_ARG;
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    if (!(omega > 0.0f && omega < 2.0f)) { set_error("omega %g outside (0, 2)", (double)omega); return SF_ERR_ARG; }
    SorState *st = w->sor;
    std::vector<uint32_t> act, chunks, req;
    sf_status r = ids ? sor_select_set(w, ids, n_ids, act, chunks, req) : sor_select(w, structure, act, chunks, req);
    if (r != SF_OK) return r;
    sf_solve_report rep{};
    if (chunks.empty() || max_sweeps == 0) { if (report) *report = rep; return SF_OK; }
    cudaStream_t s = w->stream;
    uint32_t nst = w->n_struct;
    // the cluster path when every requested structure fits one cluster's shared memory
    bool use_cl = w->P.sor_cluster != 0;
    if (use_cl && !st->cl_ready) { sf_status e = sor_cluster_tables(w); if (e != SF_OK) return e; }
    uint32_t per_max = 0;
    for (uint32_t q : req) {
        if (!use_cl) break;
        if (st->h_cl_n[q] == 0 || st->h_cl_per[q] > SOR_CL_CAP) use_cl = false;
        per_max = std::max(per_max, st->h_cl_per[q]);
    }
    SF_CUDA(cudaMemcpyAsync(st->active0.p, act.data(), nst * 4, cudaMemcpyHostToDevice, s));
    std::vector<uint32_t> cl_order;
    // Launch classes of the cluster path, run side by side: W, 16-block clusters of 1,024-thread blocks (the
    // structures of SOR_CL_WIDE_MIN bricks or more, whose tables were cut for 16 blocks); L, M, S, 8-block clusters
    // of 1,024, 512 and 256 threads. A structure's solve takes its sweeps (known from its last solve; a first solve
    // guesses them from its height) times its time per sweep, modelled as a fixed 3 us plus 2.1 us per cell a thread
    // (measured: the kernel is bound by instruction issue). The 8-block structures start in S and the slowest one is
    // moved up a class while the SMs it needs are free (a W block takes an SM, L one SM, M half, S a quarter, by
    // registers); within each class the slowest clusters are listed first, so they start first.
    const int NCLS = 4;
    static const unsigned cls_threads[NCLS] = {1024u, 1024u, 512u, 256u};
    static const double cls_sm[NCLS] = {16.0, 8.0, 4.0, 2.0};
    std::vector<uint32_t> by_cls[NCLS];
    uint32_t cls_per[NCLS] = {0, 0, 0, 0};
    if (use_cl) {
        auto expect = [&](uint32_t q) -> double {
            return st->h_last_sweeps[q] ? (double)st->h_last_sweeps[q] : 60.0 * std::max<uint32_t>(st->h_st_height[q], 1);
        };
        auto t_of = [&](uint32_t q, int c) { return expect(q) * (3.0 + 2.1 * (double)st->h_cl_per[q] / cls_threads[c]); };
        std::vector<int> cls(nst, 3);
        double used = 0.0;
        for (uint32_t q : req) {
            cls[q] = st->h_cl_ncl[q] == (uint32_t)SOR_CL_WIDE ? 0 : 3;
            used += cls_sm[cls[q]];
        }
        for (;;) {
            uint32_t worst = NONE;
            for (uint32_t q : req) if (worst == NONE || t_of(q, cls[q]) > t_of(worst, cls[worst])) worst = q;
            if (worst == NONE || cls[worst] <= 1) break;   // the slowest is wide or already on 1,024 threads
            const int up = cls[worst] - 1;
            if (used - cls_sm[cls[worst]] + cls_sm[up] > (double)w->sms) break;
            used += cls_sm[up] - cls_sm[cls[worst]];
            cls[worst] = up;
        }
        for (uint32_t q : req) by_cls[cls[q]].push_back(q);
        cl_order.clear();
        for (int c = 0; c < NCLS; c++) {
            std::stable_sort(by_cls[c].begin(), by_cls[c].end(), [&](uint32_t a, uint32_t b) { return t_of(a, c) > t_of(b, c); });
            for (uint32_t q : by_cls[c]) cls_per[c] = std::max(cls_per[c], st->h_cl_per[q]);
            cl_order.insert(cl_order.end(), by_cls[c].begin(), by_cls[c].end());
        }
        SF_CUDA(cudaMemcpyAsync(st->cl_list.p, cl_order.data(), cl_order.size() * 4, cudaMemcpyHostToDevice, s));
        if (!st->fork) {
            SF_CUDA(cudaEventCreateWithFlags(&st->fork, cudaEventDisableTiming));
            for (int k = 0; k < 3; k++) {
                SF_CUDA(cudaStreamCreateWithFlags(&st->aux[k], cudaStreamNonBlocking));
                SF_CUDA(cudaEventCreateWithFlags(&st->join[k], cudaEventDisableTiming));
            }
        }
    }
    else SF_CUDA(cudaMemcpyAsync(st->work.p, chunks.data(), chunks.size() * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaEventRecord(w->ev0, s));
    size_t ncell = (size_t)w->n_chunks * 512;
    st->launches += 5;   // clear, scatter, init, red-black, gather
    SorArgs A;
    A.cphi = st->cphi.p; A.crhs = st->crhs.p; A.ccode = st->ccode.p; A.csid = st->csid.p; A.chunk_nbr = st->chunk_nbr.p;
    A.chunk_sid = st->chunk_sid.p; A.work = st->work.p; A.n_work = (uint32_t)chunks.size(); A.n_struct = nst;
    A.active0 = st->active0.p; A.resid_buf = st->resid_buf.p; A.sweeps = st->sweeps.p; A.resid = st->resid.p;
    A.omega = (double)omega; A.tol = (double)tol; A.max_sweeps = max_sweeps; A.gb = w->barrier.p; A.err = w->err.p;
    A.prm = st->prm.p;
    A.cap = st->cap.p;
    if (caps) SF_CUDA(cudaMemcpyAsync(st->cap.p, caps, (size_t)nst * 4, cudaMemcpyHostToDevice, s));
    const SorParams hp{(double)omega, (double)tol, max_sweeps, caps ? 1u : 0u};
    SF_CUDA(cudaMemcpyAsync(st->prm.p, &hp, sizeof hp, cudaMemcpyHostToDevice, s));
    int tci = -1;
    const int tb = Tuner::bucket(chunks.size());
    const unsigned per_sm = use_cl ? 1u : (unsigned)st->tune.choose(tb, tci);
    if (use_cl) tci = -1;
    unsigned grid = use_cl ? 0u : (unsigned)std::min<size_t>(chunks.size(), (size_t)w->sms * per_sm);
    const uint32_t n_launch = use_cl ? (uint32_t)req.size() : A.n_work;
    void *args[] = {&A};
    SorClusterArgs CC[NCLS];
    cudaLaunchConfig_t cfg[NCLS] = {};
    cudaLaunchAttribute cattr[NCLS][1];
    uint32_t shape[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    {
        uint32_t first = 0;
        for (int c = 0; c < NCLS; c++) {
            SorClusterArgs &X = CC[c];
            X.cap = st->cap.p;
            X.list = st->cl_list.p + first; X.off = st->cl_off.p; X.n = st->cl_n.p; X.per = st->cl_per.p;
            X.even = st->cl_even.p; X.cpos = st->cl_cpos.p; X.nbr = st->cl_nbr.p; X.cphi = st->cphi.p; X.crhs = st->crhs.p;
            X.ccode = st->ccode.p; X.csid = st->csid.p; X.per_max = cls_per[c]; X.prm = st->prm.p;
            X.sweeps = st->sweeps.p; X.resid = st->resid.p; X.err = w->err.p;
            const unsigned ncl = c == 0 ? (unsigned)SOR_CL_WIDE : (unsigned)SOR_CL;
            cattr[c][0].id = cudaLaunchAttributeClusterDimension;
            cattr[c][0].val.clusterDim.x = ncl; cattr[c][0].val.clusterDim.y = 1; cattr[c][0].val.clusterDim.z = 1;
            cfg[c].gridDim = dim3((unsigned)(by_cls[c].size() * ncl));
            cfg[c].blockDim = dim3(cls_threads[c]);
            cfg[c].dynamicSmemBytes = (size_t)cls_per[c] * SOR_CL_BYTES_PER_CELL;
            cfg[c].stream = s;
            cfg[c].attrs = cattr[c];
            cfg[c].numAttrs = 1;
            shape[2 * c] = (uint32_t)by_cls[c].size();
            shape[2 * c + 1] = cls_per[c];
            first += (uint32_t)by_cls[c].size();
        }
    }
    auto enqueue = [&]() -> cudaError_t {
        k_sor_clear<<<grid_for(ncell, 256), 256, 0, s>>>((uint32_t)ncell, st->ccode.p, st->csid.p);
        k_sor_scatter<<<grid_for(w->ns, 256), 256, 0, s>>>(w->ns, w->s_cell.p, w->s_scene.p, w->s_mat.p, w->s_sid.p,
                                                           w->s_nb6.p, w->s_bond.p, w->s_phi64.p, w->s_ext.p, w->ctab.p,
                                                           st->cphi.p, st->crhs.p, st->ccode.p, st->csid.p);
        k_sor_init<<<grid_for(nst, 256), 256, 0, s>>>(nst, st->resid_buf.p, st->sweeps.p, st->resid.p);
        cudaError_t e = cudaMemsetAsync(w->barrier.p, 0, sizeof(GridBarrier), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(w->err.p, 0, sizeof(uint32_t), s);
        if (use_cl) {
            // the classes' launches side by side, the widest first: their blocks need whole SMs (1,024 threads and
            // large shared memory) and the narrower blocks fill what is left; the first class with clusters runs on
            // the world's stream, each later one on its own stream forked after the set-up and joined back
            int first = -1, forked = 0;
            for (int c = 0; c < NCLS && e == cudaSuccess; c++) {
                if (by_cls[c].empty()) continue;
                if (first < 0) {
                    first = c;
                    e = cudaEventRecord(st->fork, s);
                    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg[c], k_sor_cluster, CC[c]);
                    continue;
                }
                cudaStream_t a = st->aux[forked];
                e = cudaStreamWaitEvent(a, st->fork, 0);
                cfg[c].stream = a;
                if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg[c], k_sor_cluster, CC[c]);
                if (e == cudaSuccess) e = cudaEventRecord(st->join[forked], a);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(s, st->join[forked], 0);
                forked++;
            }
        } else if (e == cudaSuccess) {
            e = cudaLaunchCooperativeKernel((void *)k_sor_redblack, dim3(grid), dim3(SOR_BLOCK), args, 0, s);
        }
        if (e != cudaSuccess) return e;
        k_sor_gather<<<grid_for(w->ns, 256), 256, 0, s>>>(w->ns, w->s_cell.p, w->s_scene.p, w->s_mat.p, w->s_sid.p,
                                                          st->active0.p, w->ctab.p, st->cphi.p, w->s_phi64.p, w->s_phi.p);
        return cudaGetLastError();
    };
    // replay the captured sequence for this launch shape, capturing it the first time; if the runtime refuses to
    // capture (a cooperative launch in a graph), the solve launches directly from then on
    cudaGraphExec_t ex = nullptr;
    for (auto &g : st->graphs)
        if (g.n_work == n_launch && g.grid == grid && g.mode == (use_cl ? 1u : 0u) &&
            std::memcmp(g.shape, shape, sizeof shape) == 0)
            ex = g.exec;
    if (!ex && st->graphs_ok) {
        cudaGraph_t gr = nullptr;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const cudaError_t e1 = enqueue();
            const cudaError_t e2 = cudaStreamEndCapture(s, &gr);
            if ((e1 != cudaSuccess || e2 != cudaSuccess) && gr) { cudaGraphDestroy(gr); gr = nullptr; }
        }
        if (gr) {
            if (cudaGraphInstantiate(&ex, gr, 0) != cudaSuccess) ex = nullptr;
            cudaGraphDestroy(gr);
        }
        if (!ex) { st->graphs_ok = false; cudaGetLastError(); }
        else {
            if (st->graphs.size() >= 8) { cudaGraphExecDestroy(st->graphs.front().exec); st->graphs.erase(st->graphs.begin()); }
            SorState::Graph g{};
            g.n_work = n_launch; g.grid = grid; g.mode = use_cl ? 1u : 0u; g.exec = ex;
            std::memcpy(g.shape, shape, sizeof shape);
            st->graphs.push_back(g);
        }
    }
    if (ex) { SF_CUDA(cudaGraphLaunch(ex, s)); st->graph_launches++; }
    else SF_CUDA(enqueue());
    if (use_cl) st->cluster_solves++;
    SF_CUDA(cudaEventRecord(w->ev1, s));
    SF_CUDA(cudaGetLastError());
    std::vector<uint32_t> sw(nst);
    std::vector<double> rs(nst);
    SF_CUDA(cudaMemcpyAsync(sw.data(), st->sweeps.p, nst * 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaMemcpyAsync(rs.data(), st->resid.p, nst * 8, cudaMemcpyDeviceToHost, s));
    sf_status e = read_error_word(w);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, w->ev0, w->ev1);
    rep.ms = ms;
    for (uint32_t q : req) {
        rep.structures++;
        // a solve that converged gives the structure's sweep count; one stopped by the sweep limit a lower bound
        if (!caps && q < st->h_last_sweeps.size() && e == SF_OK)
            st->h_last_sweeps[q] = rs[q] < (double)tol ? sw[q] : std::max(st->h_last_sweeps[q], sw[q]);
        if (e == SF_OK && sw[q]) st->h_resid[q] = rs[q];
        rep.max_sweeps_done = std::max(rep.max_sweeps_done, sw[q]);
        rep.brick_sweeps += (uint64_t)sw[q] * st->h_st_count[q];
        rep.max_residual = std::max(rep.max_residual, (double)rs[q]);
    }
    w->stats.graph_launches = st->graph_launches;
    w->stats.cluster_solves = st->cluster_solves;
    // per sweep, since solves of one bucket converge in different sweep counts
    if (e == SF_OK) st->tune.record(tb, tci, ms / (float)std::max<uint32_t>(rep.max_sweeps_done, 1));
    if (report) *report = rep;
    if (e == SF_OK && (w->stats.error_word & ERR_SOR_NONFINITE)) { set_error("non-finite potential (ungrounded piece?)"); return SF_ERR_VERIFY; }
    return e;
}

static sf_status check_impl(sf_world *w, int32_t structure, const int32_t *ids, uint32_t n_ids, float dt, int32_t live,
                            sf_check_report *report);
}  // namespace sf

using namespace sf;

extern "C" {

sf_status sf_structure_solve(sf_world *w, int32_t structure, float omega, float tol, uint32_t max_sweeps,
                             sf_solve_report *report) {
    return solve_impl(w, structure, nullptr, 0, omega, tol, max_sweeps, report);
}

sf_status sf_structure_warm(sf_world *w, int32_t structure) {
    if (!w || !w->sor) { set_error("no load-path state"); return SF_ERR_ARG; }
    SorState *st = w->sor;
    if (structure < 0 || (uint32_t)structure >= w->n_struct) { set_error("structure %d out of range", structure); return SF_ERR_ARG; }
    // warm_struct (src/lib.rs:1061-1066): 560 warm-up sweeps pending, once per structure
    if (st->h_solved[structure]) return SF_OK;
    st->h_solved[structure] = 1;
    st->h_warm[structure] = 560;
    st->h_settle[structure] = 1e9f;
    return SF_OK;
}

sf_status sf_structure_frame(sf_world *w, uint32_t frame, float dt, const int32_t *active, uint32_t n_active,
                             sf_frame_report *report) {
    if (!w || !w->sor || (n_active && !active)) { set_error("null argument"); return SF_ERR_ARG; }
    SorState *st = w->sor;
    const uint32_t nst = w->n_struct;
    sf_frame_report rep{};
    float ms_total = 0.0f;
    auto size_of = [&](uint32_t q) -> int64_t { return (int64_t)st->h_st_count[q]; };
    // one solve of the listed structures, structure q stopping after caps[q] sweeps (or at tol)
    auto run = [&](std::vector<uint32_t> &caps, const std::vector<int32_t> &ids, float omega, float tol) -> sf_status {
        if (ids.empty()) return SF_OK;
        uint32_t mx = 0;
        for (int32_t q : ids) mx = std::max(mx, caps[q]);
        if (mx == 0) return SF_OK;
        sf_solve_report r{};
        sf_status e = solve_impl(w, -1, ids.data(), (uint32_t)ids.size(), omega, tol, mx, &r, caps.data());
        if (e != SF_OK) return e;
        rep.brick_updates += r.brick_sweeps;
        ms_total += (float)r.ms;
        return SF_OK;
    };
    std::vector<uint32_t> caps(std::max<uint32_t>(nst, 1), 0);
    std::vector<uint32_t> sw(std::max<uint32_t>(nst, 1));
    std::vector<double> rs(std::max<uint32_t>(nst, 1));
    // structural's sweep loop (src/lib.rs:1268-1281) over the active, solved structures in the given order: every
    // structure takes its nmin sweeps at omega 1.85 (nmin from the residual of its last sweep: 1 or 0 every third
    // frame once below 1e-4, else 1 for more than 15,000 bricks, else 6), then, in order, continues while its
    // residual is at least 4e-4, it has done fewer than 90 sweeps and the shared budget of 160,000 brick-updates
    // is not spent. The nmin sweeps of all structures run in one launch (their order cannot change them); each
    // continuation runs alone, because the budget it may use depends on the structures before it.
    std::vector<int32_t> act;
    for (uint32_t k = 0; k < n_active; k++) {
        const int32_t q = active[k];
        if (q < 0 || (uint32_t)q >= nst) { set_error("structure %d out of range", q); return SF_ERR_ARG; }
        if (st->h_solved[q] && st->h_st_count[q]) act.push_back(q);
    }
    std::vector<uint32_t> nmin(std::max<uint32_t>(nst, 1), 0);
    std::vector<int32_t> first;
    for (int32_t q : act) {
        const double r = st->h_resid[q];
        nmin[q] = r < 1e-4 ? (((frame + (uint32_t)q) % 3 == 0) ? 1u : 0u) : (size_of(q) > 15000 ? 1u : 6u);
        if (nmin[q]) { caps[q] = nmin[q]; first.push_back(q); }
    }
    sf_status e = run(caps, first, 1.85f, 0.0f);
    if (e != SF_OK) return e;
    for (int32_t q : first) rep.sweeps += nmin[q];
    int64_t budget = 160000;
    for (int32_t q : act) {
        if (!nmin[q]) continue;
        const int64_t size = size_of(q);
        budget -= (int64_t)nmin[q] * size;
        uint32_t n = nmin[q];
        if (st->h_resid[q] < (double)4e-4f || n >= 90 || budget <= 0) continue;
        const uint32_t more = (uint32_t)std::min<int64_t>(90 - n, (budget + size - 1) / size);
        std::fill(caps.begin(), caps.end(), 0u);
        caps[q] = more;
        const uint64_t before = rep.brick_updates;
        e = run(caps, std::vector<int32_t>{q}, 1.85f, 4e-4f);
        if (e != SF_OK) return e;
        const uint32_t done = (uint32_t)((rep.brick_updates - before) / (uint64_t)std::max<int64_t>(size, 1));
        rep.sweeps += done;
        budget -= (int64_t)done * size;
    }
    // structural's joint pass (src/lib.rs:1323-1339): a structure's joints are judged live once it has settled and
    // its residual is below 1.5e-3; the live structures' joints are checked in structure order with one crush budget
    // (the reference's budget of 300 crushes a frame). A structure that is not live only shades its stress display in
    // the reference (no joint changes), which is left out here.
    {
        std::vector<int32_t> live_ids;
        for (int32_t q : act)
            if (st->h_settle[q] <= 0.0f && st->h_resid[q] < (double)1.5e-3f) live_ids.push_back(q);
        std::sort(live_ids.begin(), live_ids.end());
        if (!live_ids.empty()) {
            sf_check_report cr{};
            e = check_impl(w, -1, live_ids.data(), (uint32_t)live_ids.size(), dt, 1, &cr);
            if (e != SF_OK) return e;
            rep.live = (uint32_t)live_ids.size();
            rep.joints = cr.joints; rep.over = cr.over; rep.failed = cr.failed; rep.crushed = cr.crushed;
            rep.max_ratio = cr.max_ratio;
        }
    }
    // the settle timers (src/lib.rs:1334): a structure whose warm-up is over settles for 0.3 s
    for (int32_t q : act)
        if (st->h_settle[q] > 0.0f && st->h_warm[q] == 0) st->h_settle[q] -= dt;
    // warm_step (src/lib.rs:1068-1079): the pending warm-up sweeps of every structure in structure order, from a
    // budget of 120,000 brick-updates: omega 1.9 while more than 60 remain, then 1.0; no residual test. The counts
    // follow from the sizes alone, so every structure's 1.9-sweeps run in one launch and its 1.0-sweeps in another.
    std::vector<uint32_t> c19(std::max<uint32_t>(nst, 1), 0), c10(std::max<uint32_t>(nst, 1), 0);
    std::vector<int32_t> w19, w10;
    int64_t wb = 120000;
    for (uint32_t q = 0; q < nst; q++) {
        if (st->h_warm[q] <= 0 || wb <= 0 || !st->h_st_count[q]) continue;
        const int64_t size = size_of(q);
        const uint32_t k = (uint32_t)std::min<int64_t>(st->h_warm[q], (wb + size - 1) / size);
        const uint32_t hi = (uint32_t)std::max<int32_t>(0, st->h_warm[q] - 60);
        c19[q] = std::min(k, hi);
        c10[q] = k - c19[q];
        if (c19[q]) w19.push_back((int32_t)q);
        if (c10[q]) w10.push_back((int32_t)q);
        wb -= (int64_t)k * size;
        st->h_warm[q] -= (int32_t)k;
        rep.warm_sweeps += k;
        if (st->h_warm[q] == 0) st->h_settle[q] = 0.3f;
    }
    e = run(c19, w19, 1.9f, 0.0f);
    if (e != SF_OK) return e;
    e = run(c10, w10, 1.0f, 0.0f);
    if (e != SF_OK) return e;
    rep.ms = ms_total;
    if (report) *report = rep;
    return SF_OK;
}

sf_status sf_read_structure_state(sf_world *w, int32_t *warm, uint8_t *solved, float *settle, double *resid) {
    if (!w || !w->sor) { set_error("no load-path state"); return SF_ERR_ARG; }
    SorState *st = w->sor;
    for (uint32_t q = 0; q < w->n_struct; q++) {
        if (warm) warm[q] = st->h_warm[q];
        if (solved) solved[q] = st->h_solved[q];
        if (settle) settle[q] = st->h_settle[q];
        if (resid) resid[q] = st->h_resid[q];
    }
    return SF_OK;
}

sf_status sf_structure_solve_set(sf_world *w, const int32_t *structures, uint32_t n, float omega, float tol,
                                 uint32_t max_sweeps, sf_solve_report *report) {
    if (!w || (n && !structures)) { set_error("null argument"); return SF_ERR_ARG; }
    if (n == 0) { if (report) *report = sf_solve_report{}; return SF_OK; }
    return solve_impl(w, -1, structures, n, omega, tol, max_sweeps, report);
}

sf_status sf_structure_add_loads(sf_world *w, uint32_t n, const uint32_t *brick, const float *value) {
    if (!w || (n && (!brick || !value))) { set_error("null argument"); return SF_ERR_ARG; }
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    if (n == 0) return SF_OK;
    for (uint32_t k = 0; k < n; k++)
        if (brick[k] >= w->ns) { set_error("static brick %u does not exist", brick[k]); return SF_ERR_ARG; }
    DBuf<uint32_t> d_b;
    DBuf<float> d_v;
    cudaStream_t s = w->stream;
    SF_CUDA(d_b.alloc(n)); SF_CUDA(d_v.alloc(n));
    SF_CUDA(cudaMemcpyAsync(d_b.p, brick, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(d_v.p, value, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    k_add_loads<<<grid_for(n, 256), 256, 0, s>>>(n, d_b.p, d_v.p, w->s_ext.p);
    w->sor->launches++;
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

// per-structure sweeps and residuals of the last solve (n_struct entries each)
sf_status sf_read_solve_detail(sf_world *w, uint32_t *sweeps, double *resid) {
    if (!w) return SF_ERR_ARG;
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    uint32_t nst = w->n_struct;
    if (sweeps) SF_CUDA(cudaMemcpyAsync(sweeps, w->sor->sweeps.p, nst * 4, cudaMemcpyDeviceToHost, w->stream));
    if (resid) SF_CUDA(cudaMemcpyAsync(resid, w->sor->resid.p, nst * 8, cudaMemcpyDeviceToHost, w->stream));
    SF_CUDA(cudaStreamSynchronize(w->stream));
    return SF_OK;
}

sf_status sf_structure_check(sf_world *w, int32_t structure, float dt, int32_t live, sf_check_report *report) {
    return check_impl(w, structure, nullptr, 0, dt, live, report);
}

sf_status sf_structure_loads(sf_world *w, const int32_t *structures, uint32_t n_structures);

}  // extern "C"

namespace sf {
// joint checks of one structure, of all (structure -1), or of a list (ids), in structure order with one crush budget
static sf_status check_impl(sf_world *w, int32_t structure, const int32_t *ids, uint32_t n_ids, float dt, int32_t live,
                            sf_check_report *report) {
    if (!w) return SF_ERR_ARG;
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    SorState *st = w->sor;
    std::vector<uint32_t> act, chunks, req;
    sf_status r = ids ? sor_select_set(w, ids, n_ids, act, chunks, req) : sor_select(w, structure, act, chunks, req);
    if (r != SF_OK) return r;
    cudaStream_t s = w->stream;
    uint32_t ns = w->ns, nst = w->n_struct;
    sf_check_report rep{};
    if (ns == 0 || req.empty()) { if (report) *report = rep; return SF_OK; }
    SF_CUDA(cudaMemcpyAsync(st->active0.p, act.data(), nst * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemcpyAsync(st->st_req.p, req.data(), req.size() * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(cudaMemsetAsync(st->counters.p, 0, st->counters.bytes(), s));
    SF_CUDA(cudaEventRecord(w->ev0, s));
    k_stress_zero<<<grid_for(ns, 256), 256, 0, s>>>(ns, w->s_sid.p, w->s_mat.p, st->active0.p, w->s_stress.p);
    st->launches += 5;   // zero, eval, compact, apply, tally
    StressArgs A;
    A.ns = ns; A.cell = w->s_cell.p; A.mat = w->s_mat.p; A.sid = w->s_sid.p; A.nb6 = w->s_nb6.p; A.bond = w->s_bond.p;
    A.bmax = w->s_bmax.p; A.phi = w->s_phi.p; A.active = st->active0.p; A.dt = dt; A.live = live ? 1 : 0;
    A.ratio = st->j_ratio.p; A.bond_after = st->j_bond.p; A.dec = st->j_dec.p; A.crushed = st->j_crushed.p;
    A.cand_flag = st->cand_flag.p;
    k_stress_eval<<<grid_for(ns, 256), 256, 0, s>>>(A);
    SF_CUDA(exclusive_scan_u32(st->cand_flag.p, st->cand_pos.p, ns, st->counters.p + 5, st->wk, s));
    k_stress_compact<<<grid_for(ns, 256), 256, 0, s>>>(ns, st->cand_flag.p, st->cand_pos.p, st->cand_list.p);
    k_stress_apply<<<1, 32, 0, s>>>(st->cand_list.p, st->counters.p + 5, st->st_req.p, (uint32_t)req.size(), w->s_sid.p,
                                    w->s_mat.p, w->s_nb6.p, w->s_cell.p, w->s_scene.p, w->ctab.p, w->cpool.p, w->s_bond.p,
                                    st->j_dec.p, st->j_bond.p, st->j_crushed.p, w->st_conn.p);
    k_stress_tally<<<grid_for(ns, 256), 256, 0, s>>>(ns, st->j_dec.p, st->j_ratio.p, w->s_nb6.p, w->s_sid.p, st->active0.p,
                                                      w->s_stress.p, st->counters.p);
    SF_CUDA(cudaEventRecord(w->ev1, s));
    SF_CUDA(cudaGetLastError());
    uint32_t c[16];
    SF_CUDA(cudaMemcpyAsync(c, st->counters.p, sizeof c, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, w->ev0, w->ev1);
    rep.joints = c[0]; rep.over = c[1]; rep.failed = c[2]; rep.crushed = c[3];
    std::memcpy(&rep.max_ratio, &c[4], 4);
    rep.ms = ms;
    if (report) *report = rep;
    return SF_OK;
}
}  // namespace sf

extern "C" {

sf_status sf_structure_loads(sf_world *w, const int32_t *structures, uint32_t n_structures) {
    if (!w || (n_structures && !structures)) return SF_ERR_ARG;
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    SorState *st = w->sor;
    const uint32_t nst = w->n_struct, ns = w->ns, nd = w->nd, nb = w->nb;
    std::vector<uint32_t> listed(std::max<uint32_t>(nst, 1), 0);
    for (uint32_t k = 0; k < n_structures; k++) {
        if (structures[k] < 0 || (uint32_t)structures[k] >= nst) { set_error("structure %d does not exist", structures[k]); return SF_ERR_ARG; }
        listed[structures[k]] = 1;
    }
    if (ns == 0 || n_structures == 0) return SF_OK;
    cudaStream_t s = w->stream;
    SF_CUDA(st->active0.grow(listed.size()));
    SF_CUDA(cudaMemcpyAsync(st->active0.p, listed.data(), listed.size() * 4, cudaMemcpyHostToDevice, s));
    SF_CUDA(st->extn.grow(ns));
    SF_CUDA(cudaMemsetAsync(st->extn.p, 0, (size_t)ns * 4, s));
    if (nb && nd) {
        // the brick positions after the last integrate (update_cache before structural, src/lib.rs:3654)
        SF_CUDA(refresh_poses(w));
        SF_CUDA(st->share.grow(nb));
        SF_CUDA(st->lkey.grow(nd)); SF_CUDA(st->lkey_alt.grow(nd)); SF_CUDA(st->lval.grow(nd)); SF_CUDA(st->lval_alt.grow(nd));
        const uint64_t none_key = ns;
        int bits = 0;
        while (bits < 64 && (none_key >> bits)) bits++;
        SF_CUDA(st->lcount.grow((size_t)nb * 2));
        SF_CUDA(cudaMemsetAsync(st->lcount.p, 0, (size_t)nb * 8, s));
        k_loads_count<<<grid_for(nd, 256), 256, 0, s>>>(nd, w->k_body.p, w->b_alive.p, w->b_scene.p, w->k_wpos.p,
                                                        w->ctab.p, w->cpool.p, w->s_mat.p, w->s_sid.p, st->active0.p,
                                                        st->lcount.p);
        k_loads_share<<<grid_for(nb, 128), 128, 0, s>>>(nb, w->b_alive.p, w->b_m.p, st->lcount.p, st->share.p);
        k_loads_keys<<<grid_for(nd, 256), 256, 0, s>>>(nd, none_key, w->k_body.p, w->b_scene.p, w->k_wpos.p, st->share.p,
                                                       w->ctab.p, w->cpool.p, w->s_mat.p, w->s_sid.p, st->active0.p,
                                                       st->lkey.p, st->lval.p);
        SF_CUDA(radix_sort_u64(st->lkey.p, st->lval.p, st->lkey_alt.p, st->lval_alt.p, nd, bits, st->wk, s));
        k_loads_sum<<<grid_for(nd, 256), 256, 0, s>>>(nd, none_key, st->lkey.p, st->lval.p, w->k_body.p, st->share.p, st->extn.p);
        st->launches += 4;
    }
    k_loads_apply<<<grid_for(ns, 256), 256, 0, s>>>(ns, w->s_sid.p, w->s_mat.p, st->active0.p, st->extn.p, w->s_ext.p);
    st->launches++;
    SF_CUDA(cudaGetLastError());
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

sf_status sf_read_joints(sf_world *w, float *ratio4, float *bond4, uint8_t *decision4, uint32_t *crushed4) {
    if (!w) return SF_ERR_ARG;
    if (!w->sor) { set_error("this world holds no load-path state (a scene pool)"); return SF_ERR_STATE; }
    SorState *st = w->sor;
    size_t nj = (size_t)w->ns * 4;
    cudaStream_t s = w->stream;
    if (ratio4) SF_CUDA(cudaMemcpyAsync(ratio4, st->j_ratio.p, nj * 4, cudaMemcpyDeviceToHost, s));
    if (bond4) SF_CUDA(cudaMemcpyAsync(bond4, st->j_bond.p, nj * 4, cudaMemcpyDeviceToHost, s));
    if (decision4) SF_CUDA(cudaMemcpyAsync(decision4, st->j_dec.p, nj, cudaMemcpyDeviceToHost, s));
    if (crushed4) SF_CUDA(cudaMemcpyAsync(crushed4, st->j_crushed.p, nj * 4, cudaMemcpyDeviceToHost, s));
    SF_CUDA(cudaStreamSynchronize(s));
    return SF_OK;
}

}  // extern "C"

// Scans, the stable LSD radix sort, material tables and error reporting.
#include <cstdarg>
#include <mutex>

#include "sf_internal.cuh"

namespace sf {

void host_mat_tables(MatTables &t) {
    // src/lib.rs:166-183
    const float mass[9] = {0.0f, 300.0f, 230.0f, 250.0f, 60.0f, 70.0f, 2000.0f, 8.0f, 44.0f};
    const float capv[9] = {0.0f, 140000.0f, 50000.0f, 150000.0f, 1500.0f, 9000.0f, 1e12f, 1e12f, 1e12f};
    const float caph[9] = {0.0f, 12000.0f, 12000.0f, 90000.0f, 400.0f, 5000.0f, 1e12f, 1e12f, 1e12f};
    const float tens[9] = {0.0f, 0.35f, 0.1f, 0.9f, 0.5f, 0.7f, 1.0f, 1.0f, 1.0f};
    const float stiff[9] = {0.0f, 1.0f, 0.8f, 2.0f, 0.02f, 0.4f, 1.0f, 1.0f, 1.0f};
    const float duct[9] = {0.0f, 6.0f, 12.0f, 3.0f, 40.0f, 8.0f, 1.0f, 1.0f, 1.0f};
    const float eb[9] = {0.0f, 15000.0f, 12000.0f, 1.5e6f, 300.0f, 6000.0f, 1e12f, 1e12f, 1e12f};
    const float pulv[9] = {0.0f, 0.7f, 0.55f, 0.0f, 1.0f, 0.5f, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < 9; k++) {
        t.eb[k] = eb[k]; t.pulv[k] = pulv[k];
        t.mass[k] = mass[k]; t.capv[k] = capv[k]; t.caph[k] = caph[k]; t.tens[k] = tens[k]; t.stiff[k] = stiff[k];
        t.duct[k] = duct[k];
        volatile float g = GROUNDK;   // keep the product a runtime f32 multiply
        t.gk[k] = g * stiff[k];
    }
}

// the last error of the calling thread (the server's worker threads report their own)
static thread_local char g_err[512] = "";
void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

// ---------------------------------------------------------------- exclusive scan (three-phase, recursive)
constexpr int SCAN_BLOCK = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total) {
    __shared__ uint32_t warp_sums[SCAN_BLOCK / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < SCAN_BLOCK / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_BLOCK / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t before = wid ? warp_sums[wid - 1] : 0u;
    *total = warp_sums[SCAN_BLOCK / 32 - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void k_scan_reduce(const uint32_t *in, size_t n, uint32_t *sums) {
    size_t base = (size_t)blockIdx.x * SCAN_TILE;
    uint32_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
        size_t i = base + (size_t)k * SCAN_BLOCK + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}
// each thread owns SCAN_ITEMS consecutive values of the tile
__global__ void k_scan_tile(const uint32_t *in, uint32_t *out, size_t n, const uint32_t *offsets, uint32_t *d_total) {
    size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    // a full run of 8 values at 16-byte aligned arrays moves as two 16-byte words each way (the run starts at a
    // multiple of 32 bytes from the array's start); in and out may be the same array (each thread reads its run
    // before it writes it)
    static_assert(SCAN_ITEMS == 8, "the vector path moves 8 values as two uint4");
    const bool vec = base + SCAN_ITEMS <= n && ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
    if (vec) {
        const uint4 a = reinterpret_cast<const uint4 *>(in + base)[0], b = reinterpret_cast<const uint4 *>(in + base)[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) s += v[k];
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) { size_t i = base + k; v[k] = i < n ? in[i] : 0u; s += v[k]; }
    }
    uint32_t tot;
    uint32_t run = block_exclusive_scan(s, &tot) + (offsets ? offsets[blockIdx.x] : 0u);
    if (vec) {
        uint32_t o[SCAN_ITEMS];
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) { o[k] = run; run += v[k]; }
        reinterpret_cast<uint4 *>(out + base)[0] = make_uint4(o[0], o[1], o[2], o[3]);
        reinterpret_cast<uint4 *>(out + base)[1] = make_uint4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) { size_t i = base + k; if (i < n) out[i] = run; run += v[k]; }
    }
    if (d_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == SCAN_BLOCK - 1) *d_total = run;
}

static cudaError_t scan_rec(const uint32_t *in, uint32_t *out, size_t n, uint32_t *d_total, uint32_t *tmp, cudaStream_t s) {
    size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb <= 1) {
        k_scan_tile<<<1, SCAN_BLOCK, 0, s>>>(in, out, n, nullptr, d_total);
        return cudaGetLastError();
    }
    uint32_t *sums = tmp, *rest = tmp + nb;
    k_scan_reduce<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, n, sums);
    cudaError_t e = scan_rec(sums, sums, nb, nullptr, rest, s);
    if (e != cudaSuccess) return e;
    k_scan_tile<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, out, n, sums, d_total);
    return cudaGetLastError();
}

cudaError_t exclusive_scan_u32(const uint32_t *in, uint32_t *out, size_t n, uint32_t *d_total, Work &wk, cudaStream_t s) {
    if (n == 0) {
        if (d_total) return cudaMemsetAsync(d_total, 0, sizeof(uint32_t), s);
        return cudaSuccess;
    }
    size_t need = 0, m = n;
    while (m > (size_t)SCAN_TILE) { m = (m + SCAN_TILE - 1) / SCAN_TILE; need += m; }
    cudaError_t e = wk.scan_a.grow(need + 16);
    if (e != cudaSuccess) return e;
    for (size_t q = n; ; q = (q + SCAN_TILE - 1) / SCAN_TILE) { wk.launches += q > (size_t)SCAN_TILE ? 2 : 1; if (q <= (size_t)SCAN_TILE) break; }
    return scan_rec(in, out, n, d_total, wk.scan_a.p, s);
}

// ---------------------------------------------------------------- stable LSD radix sort, 8-bit digits
constexpr int RS_BLOCK = 256;
#ifndef SF_RS_ITEMS
#define SF_RS_ITEMS 8    // keys per thread of a radix-sort tile (a build-time choice: registers against tiles)
#endif
constexpr int RS_ITEMS = SF_RS_ITEMS;
constexpr int RS_TILE = RS_BLOCK * RS_ITEMS;
constexpr int RS_WARPS = RS_BLOCK / 32;

template <class K>
__global__ void k_rs_hist(const K *keys, size_t n, int shift, uint32_t *hist, unsigned nblocks) {
    __shared__ uint32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    size_t base = (size_t)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; k++) {
        size_t i = base + (size_t)k * RS_BLOCK + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(unsigned)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// Stable ranking: warp w owns the tile's keys [w * 512, (w + 1) * 512), item k of lane l being key w*512 + k*32 + l,
// so (warp, item, lane) is input order. Each warp counts its digits privately (the leader of each match group adds
// the group's size), then one prefix over (warp, digit) places every key — two block barriers per tile.
template <class K>
__global__ void __launch_bounds__(RS_BLOCK) k_rs_scatter(const K *kin, const uint32_t *vin, K *kout, uint32_t *vout,
                                                         size_t n, int shift, const uint32_t *offs, unsigned nblocks) {
    __shared__ uint32_t wcnt[RS_WARPS][256];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) wcnt[w][threadIdx.x] = 0;
    const uint32_t gbase = offs[(size_t)threadIdx.x * nblocks + blockIdx.x];
    __syncthreads();
    const size_t wbase = (size_t)blockIdx.x * RS_TILE + (size_t)wid * (RS_ITEMS * 32);
    const unsigned lt = (1u << lane) - 1u;
    K key[RS_ITEMS];
    uint32_t val[RS_ITEMS], rank[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; k++) {
        const size_t i = wbase + (size_t)k * 32 + lane;
        const bool valid = i < n;
        key[k] = valid ? kin[i] : (K)0;
        val[k] = valid ? vin[i] : 0u;
        const unsigned d = valid ? (unsigned)(key[k] >> shift) & 255u : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        uint32_t prev = 0;
        if (lane == leader && valid) { prev = wcnt[wid][d]; wcnt[wid][d] = prev + __popc(peers); }
        prev = __shfl_sync(0xffffffffu, prev, leader);
        rank[k] = prev + __popc(peers & lt);
    }
    __syncthreads();
    {
        uint32_t run = gbase;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) { const uint32_t c = wcnt[w][threadIdx.x]; wcnt[w][threadIdx.x] = run; run += c; }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RS_ITEMS; k++) {
        const size_t i = wbase + (size_t)k * 32 + lane;
        if (i < n) {
            const unsigned d = (unsigned)(key[k] >> shift) & 255u;
            const uint32_t pos = wcnt[wid][d] + rank[k];
            kout[pos] = key[k];
            vout[pos] = val[k];
        }
    }
}

template <class K>
static cudaError_t radix_sort_impl(K *keys, uint32_t *vals, K *keys_alt, uint32_t *vals_alt, size_t n, int bits, Work &wk,
                                   cudaStream_t s, bool *in_alt) {
    if (in_alt) *in_alt = false;
    if (n <= 1 || bits <= 0) return cudaSuccess;
    unsigned nblocks = (unsigned)((n + RS_TILE - 1) / RS_TILE);
    cudaError_t e = wk.hist.grow((size_t)256 * nblocks);
    if (e != cudaSuccess) return e;
    int passes = (bits + 7) / 8;
    K *ki = keys, *ko = keys_alt;
    uint32_t *vi = vals, *vo = vals_alt;
    for (int p = 0; p < passes; p++) {
        int shift = p * 8;
        k_rs_hist<K><<<nblocks, RS_BLOCK, 0, s>>>(ki, n, shift, wk.hist.p, nblocks);
        e = exclusive_scan_u32(wk.hist.p, wk.hist.p, (size_t)256 * nblocks, nullptr, wk, s);
        if (e != cudaSuccess) return e;
        k_rs_scatter<K><<<nblocks, RS_BLOCK, 0, s>>>(ki, vi, ko, vo, n, shift, wk.hist.p, nblocks);
        wk.launches += 2;
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    if (ki != keys) {
        if (in_alt) *in_alt = true;
        else {
            cudaMemcpyAsync(keys, ki, n * sizeof(K), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(vals, vi, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        }
    }
    return cudaGetLastError();
}

cudaError_t radix_sort_u64(uint64_t *keys, uint32_t *vals, uint64_t *keys_alt, uint32_t *vals_alt, size_t n, int bits,
                           Work &wk, cudaStream_t s, bool *in_alt) {
    return radix_sort_impl(keys, vals, keys_alt, vals_alt, n, bits, wk, s, in_alt);
}
cudaError_t radix_sort_u32(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt, uint32_t *vals_alt, size_t n, int bits,
                           Work &wk, cudaStream_t s, bool *in_alt) {
    return radix_sort_impl(keys, vals, keys_alt, vals_alt, n, bits < 32 ? bits : 32, wk, s, in_alt);
}

// a wait on a flag that nothing sets: it must give up after its limit and report it
__global__ void k_wait_flag(const unsigned *flag, unsigned long long limit_ns, unsigned *err) {
    if (blockIdx.x == 0 && threadIdx.x == 0) bounded_wait_while_equal(flag, 0u, limit_ns, err);
}

}  // namespace sf

extern "C" {

sf_status sf_check_wait_timeout(uint32_t limit_ms, double *waited_ms) {
    if (limit_ms == 0 || limit_ms > 2000) { sf::set_error("limit_ms %u outside 1..2000", limit_ms); return SF_ERR_ARG; }
    unsigned *d = nullptr;
    if (cudaMalloc((void **)&d, 2 * sizeof(unsigned)) != cudaSuccess) { sf::set_error("cudaMalloc failed"); return SF_ERR_CUDA; }
    unsigned err = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMemset(d, 0, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
    if (e == cudaSuccess) {
        sf::k_wait_flag<<<1, 32>>>(d, (unsigned long long)limit_ms * 1000000ull, d + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
    if (e == cudaSuccess) e = cudaMemcpy(&err, d + 1, sizeof err, cudaMemcpyDeviceToHost);
    float ms = 0.0f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (waited_ms) *waited_ms = ms;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d);
    if (e != cudaSuccess) { sf::set_error("%s", cudaGetErrorString(e)); return SF_ERR_CUDA; }
    if (err & sf::ERR_TIMEOUT) { sf::set_error("the wait gave up after %.1f ms", (double)ms); return SF_ERR_TIMEOUT; }
    return SF_OK;
}
const char *sf_last_error(void) { return sf::g_err; }
int32_t sf_version(void) { return 100; }
const char *sf_status_string(sf_status s) {
    switch (s) {
        case SF_OK: return "ok";
        case SF_ERR_ARG: return "bad argument";
        case SF_ERR_CAPACITY: return "capacity exceeded";
        case SF_ERR_CUDA: return "CUDA error";
        case SF_ERR_TIMEOUT: return "device wait timed out";
        case SF_ERR_BUDGET: return "memory budget exceeded";
        case SF_ERR_STATE: return "call out of order";
        case SF_ERR_VERIFY: return "device self-check failed";
        default: return "unknown status";
    }
}
}

// spmv.cu -- SpMV tile plans, plain SpMV launches and CSR utilities.
#include <atomic>
#include <cstdlib>
#include <map>
#include <tuple>
#include <mutex>

#include "driver.hpp"

namespace mps {
namespace {

// tile_row[t] = first row whose row_ptr is >= t * T (binary search), with
// tile_row[0] = 0 and tile_row[ntiles] = n_rows.  Rows whose nonzeros start in
// the window [tT, (t+1)T) form tile t.
__global__ void plan_tiles_kernel(const int* __restrict__ rp, int n_rows, int T, int ntiles,
                                  int* __restrict__ tile_row) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > ntiles) return;
    if (t == 0) {
        tile_row[0] = 0;
        return;
    }
    if (t == ntiles) {
        tile_row[t] = n_rows;
        return;
    }
    const long long target = (long long)t * T;
    int lo = 0, hi = n_rows;
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (rp[mid] < target)
            lo = mid + 1;
        else
            hi = mid;
    }
    tile_row[t] = lo;
}

__global__ void plan_meta_kernel(const int* __restrict__ rp, const int* __restrict__ tile_row,
                                 int ntiles, int4* __restrict__ meta) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int rs = tile_row[t], re = tile_row[t + 1];
    meta[t] = make_int4(rs, re, rp[rs], rp[re]);
}

// Largest tile of a plan: stats[0] = max nonzeros, stats[1] = max rows.
__global__ void plan_stats_kernel(const int4* __restrict__ meta, int ntiles, int* __restrict__ stats) {
    int mn = 0, mr = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
        const int4 m = meta[t];
        mn = max(mn, m.w - m.z);
        mr = max(mr, m.y - m.x);
    }
    for (int o = 16; o; o >>= 1) {
        mn = max(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(stats, mn);
        atomicMax(stats + 1, mr);
    }
}

__global__ void diag_inv_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                const float* __restrict__ v, int n, float* __restrict__ dinv) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        float d = 0.f;
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            if (ci[k] == r) d += v[k];
        dinv[r] = d != 0.f ? 1.0f / d : 1.0f;
    }
}

// (col << 32 | row) keys of every nonzero: sorting them yields the transpose.
__global__ void transpose_keys_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                      int n_rows, unsigned long long* __restrict__ keys) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x)
        for (int k = rp[r]; k < rp[r + 1]; ++k)
            keys[k] = ((unsigned long long)(unsigned)ci[k] << 32) | (unsigned)r;
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ v, __nv_bfloat16* __restrict__ o,
                                   uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        o[i] = __float2bfloat16_rn(v[i]);
}

int grid_for(uint64_t n, int nt) {
    uint64_t g = (n + nt - 1) / nt;
    const uint64_t cap = (uint64_t)num_sms() * 8;
    if (g > cap) g = cap;
    return g ? (int)g : 1;
}

}  // namespace

int default_tile_nnz(uint64_t nnz, uint32_t n_rows) {
    const double avg = n_rows ? (double)nnz / n_rows : 1.0;
    int t = (int)(kNT * (avg < 1.0 ? 1.0 : avg + 0.999));
    t = (t + 3) & ~3;
    if (t < kMinTileNnz) t = kMinTileNnz;
    if (t > 4096) t = 4096;
    return t;
}

void spmv_plan_free(SpmvPlan& p) {
    dev_free(p.d_tile_row);
    dev_free(p.d_meta);
    p = SpmvPlan{};
}

cudaError_t spmv_plan_build(CsrMat& A, int tile_nnz, cudaStream_t s, int stages, int evict_first) {
    if (tile_nnz <= 0) {
        tile_nnz = default_tile_nnz(A.nnz, A.n_rows);
        // Between one and two waves of the solver kernels (4 CTAs per SM at
        // least): larger tiles, so that every CTA takes exactly one and none
        // runs two latency chains back to back.
        const uint64_t wave = (uint64_t)num_sms() * 4;
        const uint64_t nt0 = A.nnz ? (A.nnz + tile_nnz - 1) / tile_nnz : 1;
        if (nt0 > wave && nt0 <= 2 * wave) tile_nnz = (int)((A.nnz + wave - 1) / wave);
    }
    tile_nnz = (tile_nnz + 3) & ~3;
    const uint64_t nt = A.nnz ? (A.nnz + tile_nnz - 1) / tile_nnz : 1;
    SpmvPlan p;
    p.tile_nnz = tile_nnz;
    p.ntiles = (int)nt;
    p.cap = 2 * tile_nnz + 64;
    const int cap_grid = num_sms() * 8;
    p.grid = p.ntiles < cap_grid ? p.ntiles : cap_grid;
    if (p.grid < 1) p.grid = 1;
    p.stages = stages > 0 ? stages : A.plan.stages;
    // L2 hint: by size unless a caller (autotuner, set_spmv_plan, the
    // factors following A) chose it.  A matrix well inside L2 stays there
    // between the kernels of a solve; a larger one is streamed past L2 so
    // that the gathered vector keeps its lines.
    if (evict_first >= 0) {
        p.evict_first = evict_first ? 1 : 0;
        p.evict_auto = false;
    } else if (!A.plan.evict_auto) {
        p.evict_first = A.plan.evict_first;
        p.evict_auto = false;
    } else {
        const size_t stream_bytes = (size_t)A.nnz * 8 + (size_t)A.n_rows * 4;
        p.evict_first = stream_bytes > l2_bytes() / 4 ? 1 : 0;
        p.evict_auto = true;
    }
    p.grid_s = p.ntiles < num_sms() * 6 ? p.ntiles : num_sms() * 6;
    if (p.grid_s < 1) p.grid_s = 1;
    // tile_row has 2 spare ints at the end for the plan statistics
    cudaError_t e = dev_alloc(&p.d_tile_row, (size_t)(p.ntiles + 3) * sizeof(int), s);
    if (e != cudaSuccess) return e;
    e = dev_alloc(&p.d_meta, (size_t)p.ntiles * sizeof(int4), s);
    if (e != cudaSuccess) {
        dev_free(p.d_tile_row);
        return e;
    }
    plan_tiles_kernel<<<(p.ntiles + 1 + 255) / 256, 256, 0, s>>>(A.rp, (int)A.n_rows, tile_nnz,
                                                                 p.ntiles, p.d_tile_row);
    plan_meta_kernel<<<(p.ntiles + 255) / 256, 256, 0, s>>>(A.rp, p.d_tile_row, p.ntiles, p.d_meta);
    int* d_stats = p.d_tile_row + p.ntiles + 1;
    int stats[2] = {0, 0};
    e = cudaMemsetAsync(d_stats, 0, 2 * sizeof(int), s);
    if (e == cudaSuccess) {
        plan_stats_kernel<<<grid_for(p.ntiles, 256), 256, 0, s>>>(p.d_meta, p.ntiles, d_stats);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(stats, d_stats, sizeof(stats), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dev_free(p.d_tile_row);
        dev_free(p.d_meta);
        return e;
    }
    // Staging buffers sized to the largest tile (plus the 16-byte rounding
    // of both ends), with every stage's buffer inside the 227 KB a CTA may
    // hold (1 KB kept for the kernel's static shared memory, 8 bytes per
    // staged nonzero); larger tiles take the unstaged path.
    p.max_tile_nnz = stats[0];
    p.max_tile_rows = stats[1];
    const int r_need = p.max_tile_rows + 8;
    p.rcap = ((r_need < 2048 ? r_need : 2048) + 3) & ~3;
    const int stage_bytes = (227 * 1024 - 1024) / (p.stages < 2 ? 2 : p.stages);
    int cap_lim = 2 * tile_nnz + 64;
    const int cap_smem = (stage_bytes - p.rcap * 4) / 8;
    if (cap_lim > cap_smem) cap_lim = cap_smem;
    const int cap_need = p.max_tile_nnz + 16;
    p.cap_s = (cap_need < cap_lim ? cap_need : cap_lim) & ~7;
    spmv_plan_free(A.plan);
    A.plan = p;
    return cudaSuccess;
}

template <class K>
static void smem_optin(K kernel, size_t smem) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

namespace {
std::atomic<int> g_pdl{-1};
thread_local bool t_pdl_off = false;
}  // namespace

bool pdl_enabled() {
    if (t_pdl_off) return false;
    int v = g_pdl.load();
    if (v < 0) {
        const char* e = std::getenv("MPS_PDL");
        v = (e && e[0] == '0') ? 0 : 1;
        g_pdl.store(v);
    }
    return v == 1;
}

bool pdl_suspend(bool off) {
    const bool prev = t_pdl_off;
    t_pdl_off = off;
    return prev;
}

int resident_ctas(const void* kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, size_t>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(dev, kernel, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess) n = 1;
    cache[key] = n;
    return n;
}

cudaError_t spmv_launch(const CsrMat& A, const float* x, float* y, cudaStream_t s) {
    return CsrOp{&A, nullptr}.apply(x, EpiStore{y}, s);
}

cudaError_t spmv_dot_launch(const CsrMat& A, const float* x, const float* w, float* y,
                            double* d_dot, double* partials, unsigned* counter, cudaStream_t s) {
    return CsrOp{&A, nullptr}.apply(x, EpiStoreDot{y, w, d_dot, counter, partials}, s);
}

cudaError_t diag_inv_launch(const CsrMat& A, float* dinv, cudaStream_t s) {
    diag_inv_kernel<<<grid_for(A.n_rows, 256), 256, 0, s>>>(A.rp, A.ci, A.v, (int)A.n_rows, dinv);
    return cudaGetLastError();
}

cudaError_t transpose_keys_launch(const CsrMat& A, unsigned long long* keys, cudaStream_t s) {
    transpose_keys_kernel<<<grid_for(A.n_rows, 256), 256, 0, s>>>(A.rp, A.ci, (int)A.n_rows, keys);
    return cudaGetLastError();
}

cudaError_t to_bf16_launch(const float* v, __nv_bfloat16* o, uint64_t n, cudaStream_t s) {
    f32_to_bf16_kernel<<<grid_for(n, 256), 256, 0, s>>>(v, o, n);
    return cudaGetLastError();
}

}  // namespace mps

namespace mps {
// Tile plan into caller-provided memory (used by the allocation-free entry
// point; spmv_plan_build allocates its own).
cudaError_t plan_tiles_launch(const int* rp, int n_rows, int tile_nnz, int ntiles, int* tile_row,
                              cudaStream_t s) {
    plan_tiles_kernel<<<(ntiles + 1 + 255) / 256, 256, 0, s>>>(rp, n_rows, tile_nnz, ntiles, tile_row);
    return cudaGetLastError();
}
}  // namespace mps

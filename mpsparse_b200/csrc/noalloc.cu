// noalloc.cu -- y = A x and w . y for callers that cannot allocate device
// memory.
//
// Some callers may not call cudaMalloc: a serving process that reserved its
// whole HBM budget for its own pool at start-up, or code on a latency-critical
// path where an allocation (which can synchronise the device) is not allowed.
// This entry point takes the CSR arrays and vectors as plain device pointers
// and keeps its scratch -- the SpMV tile plan, the per-CTA FP64 partial sums
// and the last-CTA counter -- in one file-scope __device__ array, so it
// allocates nothing.  Every GPU that loads this library holds that array
// (about 280 KB) until the process exits.
#include <mutex>

#include "spmv_kernels.cuh"

namespace mps {
cudaError_t plan_tiles_launch(const int* rp, int n_rows, int tile_nnz, int ntiles, int* tile_row,
                              cudaStream_t s);
int default_tile_nnz(uint64_t nnz, uint32_t n_rows);
}  // namespace mps

namespace {

constexpr int kNoAllocMaxTiles = 65536;
constexpr int kNoAllocMaxGrid = 2048;
// Default tiles hold at least kMinTileNnz nonzeros (default_tile_nnz), so
// this many nonzeros fit the static tile plan.
constexpr unsigned long long kNoAllocMaxNnz = (unsigned long long)kNoAllocMaxTiles * mps::kMinTileNnz;
static_assert(kNoAllocMaxNnz == 33554432ull, "the documented limit of mps_csr_spmv_dot_noalloc");

struct NoAllocScratch {
    double partials[kNoAllocMaxGrid];
    int tile_row[kNoAllocMaxTiles + 1];
    unsigned counter;
};

// The scratch.  In host code this name is only a host-side stand-in; its
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

std::mutex g_mu;
NoAllocScratch* g_addr[mps::kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (with that device current).
cudaError_t scratch_address(NoAllocScratch** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= mps::kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

}  // namespace

using namespace mps;

extern "C" mps_status mps_csr_spmv_dot_noalloc(const int32_t* d_row_ptr, const int32_t* d_col_ind,
                                               const float* d_vals, uint32_t n_rows,
                                               uint32_t n_cols, uint64_t nnz, const float* d_x,
                                               const float* d_w, float* d_y, double* d_dot,
                                               cudaStream_t stream) {
    if (!d_row_ptr || !d_x || !d_w || !d_y || !d_dot || (nnz && (!d_col_ind || !d_vals)))
        return fail(MPS_ERR_ARG, "spmv_dot_noalloc: null pointer");
    if (n_rows == 0 || n_cols == 0 || n_rows >= 0x7fffffffu)
        return fail(MPS_ERR_ARG, "spmv_dot_noalloc: num_rows / num_cols must be in [1, 2^31 - 1)");
    // the tile loads read col_ind and values 16 bytes at a time
    if (nnz && ((reinterpret_cast<uintptr_t>(d_col_ind) | reinterpret_cast<uintptr_t>(d_vals)) & 15))
        return fail(MPS_ERR_ARG, "spmv_dot_noalloc: d_col_ind and d_vals must be 16-byte aligned");
    if (nnz > kNoAllocMaxNnz)
        return fail(MPS_ERR_ARG, "spmv_dot_noalloc: nnz " + std::to_string(nnz) +
                                     " exceeds the allocation-free limit of " +
                                     std::to_string(kNoAllocMaxNnz) + " nonzeros");
    NoAllocScratch* scr = nullptr;
    MPS_CUDA(scratch_address(&scr));
    const int T = default_tile_nnz(nnz, n_rows);
    const int ntiles = nnz ? (int)((nnz + T - 1) / T) : 1;
    if (ntiles > kNoAllocMaxTiles)
        return fail(MPS_ERR_ARG, "spmv_dot_noalloc: matrix needs more SpMV tiles than the scratch holds");
    int grid = num_sms() * 8;
    if (grid > kNoAllocMaxGrid) grid = kNoAllocMaxGrid;
    if (grid > ntiles) grid = ntiles;
    // the last-CTA counter must start at zero
    MPS_CUDA(cudaMemsetAsync(&scr->counter, 0, sizeof(unsigned), stream));
    MPS_CUDA(plan_tiles_launch(d_row_ptr, (int)n_rows, T, ntiles, scr->tile_row, stream));
    CsrDev v{d_row_ptr, d_col_ind, d_vals, nullptr, scr->tile_row, (int)n_rows, ntiles, 2 * T + 64};
    const size_t smem = spmv_smem_bytes<float>(v);
    if (smem > 48 * 1024)
        MPS_CUDA(cudaFuncSetAttribute(spmv_tiles<float, float, false, EpiStoreDot>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    EpiStoreDot epi{d_y, d_w, d_dot, &scr->counter, scr->partials};
    spmv_tiles<float, float, false, EpiStoreDot><<<grid, kNT, smem, stream>>>(v, d_x, epi);
    MPS_CUDA(cudaGetLastError());
    return MPS_OK;
}

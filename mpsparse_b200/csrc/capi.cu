// capi.cu -- extern "C" entry points (include/mpsparse.h) for CSR handles.
#include <atomic>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "handles.hpp"

namespace mps {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
mps_status fail(mps_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}
mps_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? MPS_ERR_OOM : MPS_ERR_CUDA;
}
cudaMemPool_t lib_pool() {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(d);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = d;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[d] = pool;
    return pool;
}

namespace {
constexpr size_t kPinnedBlock = 4096;
std::mutex g_pin_mu;
std::vector<void*> g_pin_free;
std::mutex g_stream_mu;
std::map<int, std::vector<cudaStream_t>> g_stream_free;
}  // namespace

void* pinned_block_get(size_t bytes) {
    if (bytes > kPinnedBlock) return nullptr;
    void* p = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pin_mu);
        if (!g_pin_free.empty()) {
            p = g_pin_free.back();
            g_pin_free.pop_back();
        }
    }
    if (!p && cudaMallocHost(&p, kPinnedBlock) != cudaSuccess) return nullptr;
    std::memset(p, 0, kPinnedBlock);
    return p;
}
void pinned_block_put(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pin_mu);
    g_pin_free.push_back(p);
}
cudaStream_t capture_stream_get() {
    int d = 0;
    cudaGetDevice(&d);
    {
        std::lock_guard<std::mutex> lock(g_stream_mu);
        auto& v = g_stream_free[d];
        if (!v.empty()) {
            cudaStream_t s = v.back();
            v.pop_back();
            return s;
        }
    }
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    return s;
}
void capture_stream_put(cudaStream_t s) {
    if (!s) return;
    int d = 0;
    cudaGetDevice(&d);
    std::lock_guard<std::mutex> lock(g_stream_mu);
    g_stream_free[d].push_back(s);
}

// Device attributes, cached per device (a process may drive several GPUs).
static int device_attr(cudaDeviceAttr attr, std::atomic<int>* cache, int fallback) {
    int d = 0;
    cudaGetDevice(&d);
    if (d >= 0 && d < kMaxDevices) {
        const int c = cache[d].load(std::memory_order_relaxed);
        if (c) return c;
    }
    int v = 0;
    cudaDeviceGetAttribute(&v, attr, d);
    if (v <= 0) v = fallback;
    if (d >= 0 && d < kMaxDevices) cache[d].store(v, std::memory_order_relaxed);
    return v;
}

int num_sms() {
    static std::atomic<int> cache[kMaxDevices];
    return device_attr(cudaDevAttrMultiProcessorCount, cache, 148);
}

size_t l2_bytes() {
    static std::atomic<int> cache[kMaxDevices];
    return (size_t)device_attr(cudaDevAttrL2CacheSize, cache, 126 << 20);
}

mps_status device_error(unsigned err, const char* what) {
    if (err & kErrRange) return fail(MPS_ERR_RANGE, std::string(what) + ": a key lies outside [0, num_rows) x [0, num_cols)");
    if (err & kErrTimeout) return fail(MPS_ERR_TIMEOUT, std::string(what) + ": a bounded device wait gave up");
    return MPS_OK;
}

}  // namespace mps

using namespace mps;


namespace mps {

void csr_free(CsrMat& m) {
    dev_free(m.rp);
    dev_free(m.ci);
    dev_free(m.v);
    spmv_plan_free(m.plan);
    m = CsrMat{};
}

mps_status alloc_csr(CsrMat& m, uint32_t n_rows, uint32_t n_cols, uint64_t nnz,
                     unsigned* err, cudaStream_t s) {
    m.n_rows = n_rows;
    m.n_cols = n_cols;
    m.nnz = nnz;
    m.err = err;
    const size_t nz = nnz + kCsrPad;
    MPS_CUDA(dev_alloc(&m.rp, ((size_t)n_rows + 1 + kCsrPad) * sizeof(int32_t), s));
    MPS_CUDA(dev_alloc(&m.ci, nz * sizeof(int32_t), s));
    MPS_CUDA(dev_alloc(&m.v, nz * sizeof(float), s));
    return MPS_OK;
}

static mps_status check_shape(uint64_t nnz, uint32_t n_rows, uint32_t n_cols) {
    if (n_rows == 0 || n_cols == 0) return fail(MPS_ERR_ARG, "num_rows and num_cols must be positive");
    if (n_rows >= 0x7fffffffu || n_cols >= 0x7fffffffu) return fail(MPS_ERR_ARG, "num_rows / num_cols must be < 2^31 - 1");
    if (nnz >= 0x7fffff00ull) return fail(MPS_ERR_ARG, "nnz must be < 2^31 (int32 row_ptr)");
    return MPS_OK;
}

// Sort + CSR + tile plan into a fresh CsrMat (plan = false: the caller
// builds the plan afterwards, as the FSAI factors do with A's pipeline).
mps_status build_from_keys(CsrMat& m, const uint64_t* keys, const uint32_t* payload,
                                  uint64_t nnz, uint32_t n_rows, uint32_t n_cols, unsigned* d_err,
                                  cudaStream_t s, bool plan) {
    mps_status st = alloc_csr(m, n_rows, n_cols, nnz, d_err, s);
    if (st != MPS_OK) return st;
    MPS_CUDA(cudaMemsetAsync(d_err, 0, sizeof(unsigned), s));
    MPS_CUDA(sort_to_csr(keys, payload, nnz, n_rows, n_cols, m.rp, m.ci, (uint32_t*)m.v, d_err, s));
    if (plan) MPS_CUDA(spmv_plan_build(m, 0, s));
    unsigned err = 0;
    MPS_CUDA(cudaMemcpyAsync(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    return device_error(err, "COO->CSR");
}

}  // namespace mps

extern "C" {

int32_t mps_abi_version(void) { return 4; }

void mps_solve_opts_default(mps_solve_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-6;
    o->max_iter = 2000;
    o->omega = 0.01;
    o->stall_window = 400;
}

const char* mps_last_error_string(void) { return g_last_error.c_str(); }

const char* mps_status_string(mps_status s) {
    switch (s) {
        case MPS_OK: return "ok";
        case MPS_ERR_ARG: return "invalid argument";
        case MPS_ERR_CUDA: return "CUDA error";
        case MPS_ERR_OOM: return "out of device memory";
        case MPS_ERR_TIMEOUT: return "device wait timed out";
        case MPS_ERR_BREAKDOWN: return "solver breakdown";
        case MPS_ERR_RANGE: return "key out of range";
        case MPS_ERR_NOT_FINITE: return "non-finite input";
    }
    return "unknown status";
}

mps_status mps_csr_create_from_keys(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                                    uint32_t n_rows, uint32_t n_cols, mps_csr** out,
                                    cudaStream_t stream) {
    if (!out) return fail(MPS_ERR_ARG, "out is null");
    *out = nullptr;
    mps_status st = check_shape(nnz, n_rows, n_cols);
    if (st != MPS_OK) return st;
    if (nnz && (!d_keys || !d_vals)) return fail(MPS_ERR_ARG, "keys / values are null");
    mps_csr* h = new mps_csr();
    MPS_CUDA(dev_alloc(&h->d_err, 2 * sizeof(unsigned), stream));
    MPS_CUDA(cudaMemsetAsync(h->d_err, 0, 2 * sizeof(unsigned), stream));
    st = build_from_keys(h->A, d_keys, reinterpret_cast<const uint32_t*>(d_vals), nnz, n_rows,
                         n_cols, h->d_err, stream);
    if (st != MPS_OK) {
        mps_csr_destroy(h);
        return st;
    }
    *out = h;
    return MPS_OK;
}

mps_status mps_csr_create_from_csr(const int32_t* d_row_ptr, const int32_t* d_col_ind,
                                   const float* d_vals, uint32_t n_rows, uint32_t n_cols,
                                   uint64_t nnz, mps_csr** out, cudaStream_t stream) {
    if (!out) return fail(MPS_ERR_ARG, "out is null");
    *out = nullptr;
    mps_status st = check_shape(nnz, n_rows, n_cols);
    if (st != MPS_OK) return st;
    if (!d_row_ptr || (nnz && (!d_col_ind || !d_vals))) return fail(MPS_ERR_ARG, "null CSR array");
    mps_csr* h = new mps_csr();
    MPS_CUDA(dev_alloc(&h->d_err, 2 * sizeof(unsigned), stream));
    MPS_CUDA(cudaMemsetAsync(h->d_err, 0, 2 * sizeof(unsigned), stream));
    st = alloc_csr(h->A, n_rows, n_cols, nnz, h->d_err, stream);
    if (st != MPS_OK) {
        mps_csr_destroy(h);
        return st;
    }
    MPS_CUDA(cudaMemcpyAsync(h->A.rp, d_row_ptr, ((size_t)n_rows + 1) * 4, cudaMemcpyDeviceToDevice, stream));
    if (nnz) {
        MPS_CUDA(cudaMemcpyAsync(h->A.ci, d_col_ind, nnz * 4, cudaMemcpyDeviceToDevice, stream));
        MPS_CUDA(cudaMemcpyAsync(h->A.v, d_vals, nnz * 4, cudaMemcpyDeviceToDevice, stream));
    }
    cudaError_t e = spmv_plan_build(h->A, 0, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        mps_csr_destroy(h);
        return cuda_fail(e, "create_from_csr");
    }
    *out = h;
    return MPS_OK;
}

mps_status mps_test_sort_lookback_timeout(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                                          uint32_t n_rows, uint32_t n_cols, uint32_t spin_limit,
                                          uint32_t silent_tile, cudaStream_t s) {
    if (!d_keys || !d_vals || spin_limit == 0) return fail(MPS_ERR_ARG, "null argument or zero spin limit");
    mps_status st = check_shape(nnz, n_rows, n_cols);
    if (st != MPS_OK) return st;
    CsrMat m;
    unsigned* d_err = nullptr;
    MPS_CUDA(cudaMalloc(&d_err, sizeof(unsigned)));
    st = alloc_csr(m, n_rows, n_cols, nnz, d_err, s);
    cudaError_t e = cudaSuccess;
    if (st == MPS_OK) {
        e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), s);
        if (e == cudaSuccess)
            e = sort_to_csr(d_keys, reinterpret_cast<const uint32_t*>(d_vals), nnz, n_rows, n_cols, m.rp,
                            m.ci, reinterpret_cast<uint32_t*>(m.v), d_err, s, spin_limit, silent_tile);
        unsigned err = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        st = e != cudaSuccess ? cuda_fail(e, "sort (timeout test)") : device_error(err, "COO->CSR");
    }
    csr_free(m);
    cudaFree(d_err);
    return st;
}

mps_status mps_csr_set_persistent(mps_csr* h, int32_t enable) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    h->persistent = enable ? 1 : 0;
    return MPS_OK;
}

mps_status mps_csr_set_persistent_form(mps_csr* h, int32_t form) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (form < 0 || form > 3) return fail(MPS_ERR_ARG, "form must be 0 (auto), 1 (gather), 2 (window) or 3 (stream)");
    if (form != h->persist_form) {
        persist_plan_free_all(h);   // planned again, for the new choice, by the next solve
        h->persist_form = form;
    }
    return MPS_OK;
}

mps_status mps_csr_destroy(mps_csr* h) {
    if (!h) return MPS_OK;
    csr_free(h->A);
    fsai_product_free(h);
    csr_free(h->G);
    csr_free(h->Gt);
    persist_plan_free_all(h);
    dev_free(h->vb);
    dev_free(h->d_err);
    fsai_work_free(h->fw);
    h->H.destroy();
    delete h;
    return MPS_OK;
}

mps_status mps_csr_shape(const mps_csr* h, uint32_t* n_rows, uint32_t* n_cols, uint64_t* nnz) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (n_rows) *n_rows = h->A.n_rows;
    if (n_cols) *n_cols = h->A.n_cols;
    if (nnz) *nnz = h->A.nnz;
    return MPS_OK;
}

mps_status mps_csr_export(const mps_csr* h, int32_t* d_row_ptr, int32_t* d_col_ind, float* d_vals,
                          cudaStream_t s) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (d_row_ptr)
        MPS_CUDA(cudaMemcpyAsync(d_row_ptr, h->A.rp, ((size_t)h->A.n_rows + 1) * 4, cudaMemcpyDefault, s));
    if (d_col_ind && h->A.nnz)
        MPS_CUDA(cudaMemcpyAsync(d_col_ind, h->A.ci, h->A.nnz * 4, cudaMemcpyDefault, s));
    if (d_vals && h->A.nnz)
        MPS_CUDA(cudaMemcpyAsync(d_vals, h->A.v, h->A.nnz * 4, cudaMemcpyDefault, s));
    return MPS_OK;
}

mps_status mps_coo_to_csr(const uint64_t* d_keys, const float* d_vals, uint64_t nnz,
                          uint32_t n_rows, uint32_t n_cols, int32_t* d_row_ptr, int32_t* d_col_ind,
                          float* d_out_vals, cudaStream_t s) {
    mps_status st = check_shape(nnz, n_rows, n_cols);
    if (st != MPS_OK) return st;
    if (!d_row_ptr || (nnz && (!d_keys || !d_vals || !d_col_ind || !d_out_vals)))
        return fail(MPS_ERR_ARG, "null pointer");
    unsigned* d_err = nullptr;
    MPS_CUDA(stream_alloc(&d_err, sizeof(unsigned), s));
    MPS_CUDA(cudaMemsetAsync(d_err, 0, sizeof(unsigned), s));
    cudaError_t e = sort_to_csr(d_keys, reinterpret_cast<const uint32_t*>(d_vals), nnz, n_rows,
                                n_cols, d_row_ptr, d_col_ind, reinterpret_cast<uint32_t*>(d_out_vals),
                                d_err, s);
    unsigned err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_err, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "coo_to_csr");
    return device_error(err, "COO->CSR");
}

mps_status mps_csr_spmv(const mps_csr* h, const float* d_x, float* d_y, cudaStream_t s) {
    if (!h || !d_x || !d_y) return fail(MPS_ERR_ARG, "null argument");
    MPS_CUDA(spmv_launch(h->A, d_x, d_y, s));
    return MPS_OK;
}

mps_status mps_csr_set_spmv_plan(mps_csr* h, int32_t tile_nnz, int32_t stages, int32_t evict_first,
                                 cudaStream_t s) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (stages != 0 && stages != 2 && stages != 3) return fail(MPS_ERR_ARG, "stages must be 2 or 3");
    if (tile_nnz < 0 || tile_nnz > 8192) return fail(MPS_ERR_ARG, "tile_nnz must be in [0, 8192]");
    MPS_CUDA(spmv_plan_build(h->A, tile_nnz < 256 && tile_nnz > 0 ? 256 : tile_nnz, s, stages,
                             evict_first < 0 ? -1 : (evict_first ? 1 : 0)));
    MPS_CUDA(factor_plans_follow(h, s));
    h->H.drop_graphs();
    return MPS_OK;
}

mps_status mps_csr_autotune_spmv(mps_csr* h, int32_t* h_tile_nnz, int32_t* h_stages,
                                 int32_t* h_evict_first, float* h_best_us, cudaStream_t s) {
    if (!h) return fail(MPS_ERR_ARG, "null handle");
    if (h->A.nnz == 0) return MPS_OK;
    // Candidates: tile size (half, default, twice the default nonzeros per
    // tile), pipeline depth 2 / 3, L2 evict-first hint off / on; each timed
    // over 5 launches after 2 warm-ups, with x = 0 (timing only).
    const int T0 = default_tile_nnz(h->A.nnz, h->A.n_rows);
    int tiles[3] = {T0 / 2, T0, 2 * T0};
    for (int& t : tiles) t = t < 256 ? 256 : (t > 8192 ? 8192 : t);
    float* buf = nullptr;
    MPS_CUDA(cudaMalloc(&buf, ((size_t)h->A.n_cols + h->A.n_rows + 8) * sizeof(float)));
    float* x = buf;
    float* y = buf + h->A.n_cols + 4;
    cudaError_t e = cudaMemsetAsync(x, 0, (size_t)h->A.n_cols * sizeof(float), s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float best = 1e30f;
    int bt = T0, bs = h->A.plan.stages, bh = h->A.plan.evict_first;
    for (int ti = 0; ti < 3 && e == cudaSuccess; ++ti) {
        if (ti > 0 && tiles[ti] == tiles[ti - 1]) continue;
        for (int st = 2; st <= 3 && e == cudaSuccess; ++st)
            for (int hint = 0; hint <= 1 && e == cudaSuccess; ++hint) {
                e = spmv_plan_build(h->A, tiles[ti], s, st, hint);
                for (int w = 0; w < 2 && e == cudaSuccess; ++w) e = spmv_launch(h->A, x, y, s);
                if (e == cudaSuccess) e = cudaEventRecord(e0, s);
                for (int r = 0; r < 5 && e == cudaSuccess; ++r) e = spmv_launch(h->A, x, y, s);
                if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                if (e == cudaSuccess && ms < best) {
                    best = ms;
                    bt = tiles[ti];
                    bs = st;
                    bh = hint;
                }
            }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    if (e == cudaSuccess) e = spmv_plan_build(h->A, bt, s, bs, bh);
    if (e == cudaSuccess) e = factor_plans_follow(h, s);
    if (e != cudaSuccess) return cuda_fail(e, "autotune_spmv");
    h->H.drop_graphs();        // captured solves hold the old plan's launch shapes
    if (h_tile_nnz) *h_tile_nnz = bt;
    if (h_stages) *h_stages = bs;
    if (h_evict_first) *h_evict_first = bh;
    if (h_best_us) *h_best_us = best * 1e3f / 5.f;
    return MPS_OK;
}

mps_status mps_csr_spmv_dot(const mps_csr* hc, const float* d_x, const float* d_w, float* d_y,
                            double* d_dot, cudaStream_t s) {
    mps_csr* h = const_cast<mps_csr*>(hc);
    if (!h || !d_x || !d_w || !d_y || !d_dot) return fail(MPS_ERR_ARG, "null argument");
    MPS_CUDA(h->H.ensure(h->A.n_rows, s));
    MPS_CUDA(spmv_dot_launch(h->A, d_x, d_w, d_y, d_dot, h->H.ws.partials, h->H.ws.counters + 12, s));
    return MPS_OK;
}

}  // extern "C"

namespace mps {
cudaError_t factor_plans_follow(mps_csr* h, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (h->G.rp && h->G.n_rows) e = spmv_plan_build(h->G, 0, s, h->A.plan.stages, h->A.plan.evict_first);
    if (e == cudaSuccess && h->Gt.rp && h->Gt.n_rows)
        e = spmv_plan_build(h->Gt, 0, s, h->A.plan.stages, h->A.plan.evict_first);
    if (e == cudaSuccess && h->M.rp && h->M.n_rows)
        e = spmv_plan_build(h->M, 0, s, h->A.plan.stages, h->A.plan.evict_first);
    return e;
}

mps_status prepare_precond(mps_csr* h, const mps_solve_opts* o, cudaStream_t s) {
    MPS_CUDA(h->H.ensure(h->A.n_rows, s));
    const int pc = o ? o->precond : 0;
    if (pc != MPS_PRECOND_NONE && !(o && o->reference_compat)) {
        if (pc == MPS_PRECOND_FSAI && !h->has_fsai)
            return fail(MPS_ERR_ARG, "FSAI preconditioner requested but no factor was attached");
        if (pc != MPS_PRECOND_JACOBI && pc != MPS_PRECOND_FSAI)
            return fail(MPS_ERR_ARG, "unknown preconditioner");
        if (!h->H.dinv) {
            MPS_CUDA(dev_alloc(&h->H.dinv, h->H.ws.n_pad * sizeof(float), s));
            MPS_CUDA(cudaMemsetAsync(h->H.dinv, 0, h->H.ws.n_pad * sizeof(float), s));
            MPS_CUDA(diag_inv_launch(h->A, h->H.dinv, s));
            h->H.drop_graphs();   // graphs captured the previous (null) diagonal
        }
    }
    return MPS_OK;
}
}  // namespace mps

extern "C" {

// A handle's error words: [0] bounded waits of its own kernels (cleared at
// the start of each call), [1] the learned network's bounded waits, folded
// in by an attach (which does not synchronise) and reported -- then cleared
// -- by the next solve.
static mps_status solve_errors(mps_csr* h, const unsigned* e2, mps_status st, cudaStream_t s) {
    if (st != MPS_OK) return st;
    if (e2[1] & kErrTimeout) {
        cudaMemsetAsync(h->d_err + 1, 0, sizeof(unsigned), s);
        return fail(MPS_ERR_TIMEOUT, "FSAI network: a tensor-core wait gave up (in the attach before this solve)");
    }
    if (e2[0] & kErrTimeout)
        return fail(MPS_ERR_TIMEOUT, "a bounded device wait gave up (SpMV bulk copy or grid barrier)");
    return MPS_OK;
}

// Plain CG / Jacobi-PCG, BiCGSTAB or Richardson as one persistent cooperative kernel
// when A's rows (or, in the stream form, their vector windows) fit one CTA
// per SM (fsai_persistent.cu); *ran = false: not eligible, the graph form
// runs instead.  Same parameters,
// result places and report as run_solve.
static mps_status csr_persistent(SolverKind kind, mps_csr* h, const float* b, float* x,
                                 const mps_solve_opts& o, mps_solve_info* info, cudaStream_t s, bool* ran) {
    *ran = false;
    SolverHost& H = h->H;
    const size_t n = h->A.n_rows;
    SolveParams& P = *H.h_params;
    P.delta = 0.0;
    P.tol = o.tol > 0 ? o.tol : 1e-6;
    P.omega = o.omega != 0 ? o.omega : 0.01;
    P.max_iter = o.max_iter > 0 ? o.max_iter : 2000;
    P.compat = 0;
    P.precond = kind == kCG ? o.precond : 0;
    P.stall_window = o.stall_window > 0 ? o.stall_window : 400;
    MPS_CUDA(cudaMemcpyAsync(H.ws.d_params, H.h_params, sizeof(SolveParams), cudaMemcpyHostToDevice, s));
    MPS_CUDA(cudaMemcpyAsync(H.v(vB), b, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    const cudaError_t pe = kind == kCG     ? persist_cg_solve(h, s)
                           : kind == kBiCG ? persist_bicg_solve(h, s)
                                           : persist_rich_solve(h, s);
    if (pe == cudaErrorNotSupported) return MPS_OK;
    if (pe != cudaSuccess)
        return cuda_fail(pe, kind == kCG     ? "persistent CG"
                             : kind == kBiCG ? "persistent BiCGSTAB"
                                             : "persistent Richardson");
    *ran = true;
    if (kind == kRich) {   // x in vX or vXAlt by the final iteration's parity
        const int nb = ((int)n + 255) / 256;
        launch_k(copy_result, dim3(nb < 1184 ? (nb ? nb : 1) : 1184), dim3(256), 0, s, H.v(vX),
                 static_cast<const float*>(H.v(vXAlt)), H.v(vXAlt), x, (int)n, (int)kResRich,
                 static_cast<const DevScalars*>(H.ws.sc));
        MPS_CUDA(cudaGetLastError());
    } else {
        MPS_CUDA(cudaMemcpyAsync(x, H.v(vX), n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    const CsrOp op{&h->A, nullptr};
    MPS_CUDA(op.true_resid(x, H.v(vB), &H.ws.sc->true_rr, H.ws.counters + 11, H.ws.partials, s));
    MPS_CUDA(cudaMemcpyAsync(H.ws.h_sc, H.ws.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    const mps_status st = solve_report(kind, H, info, nullptr, true);
    if (info) info->persistent = 1 + h->pp_a.form;
    return st;
}

static mps_status csr_solve(SolverKind kind, mps_csr* h, const float* b, float* x,
                            const mps_solve_opts* o, mps_solve_info* info, cudaStream_t s) {
    if (!h || !b || !x) return fail(MPS_ERR_ARG, "null argument");
    if (h->A.n_rows != h->A.n_cols) return fail(MPS_ERR_ARG, "solvers need a square matrix");
    mps_status st = prepare_precond(h, kind == kCG ? o : nullptr, s);
    if (st != MPS_OK) return st;
    CsrOp op{&h->A, nullptr};
    CsrOp g{&h->G, nullptr}, gt{&h->Gt, nullptr}, mm{&h->M, nullptr};
    PrecondOps<CsrOp> pc{h->has_fsai ? &g : nullptr, h->has_fsai ? &gt : nullptr,
                         h->has_fsai && h->use_m ? &mm : nullptr};
    MPS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), s));
    mps_solve_opts oo;
    mps_solve_opts_default(&oo);
    if (o) oo = *o;
    bool ran = false;
    if (h->persistent && !oo.reference_compat && !oo.host_loop &&
        ((kind == kCG && (oo.precond == MPS_PRECOND_NONE || oo.precond == MPS_PRECOND_JACOBI)) ||
         kind == kBiCG || kind == kRich))
        st = csr_persistent(kind, h, b, x, oo, info, s, &ran);
    if (st != MPS_OK) return st;
    if (!ran) st = run_solve(kind, op, pc, h->H, b, x, o, info, s);
    unsigned err[2] = {0, 0};
    MPS_CUDA(cudaMemcpy(err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost));
    return solve_errors(h, err, st, s);
}

mps_status mps_csr_cg(mps_csr* h, const float* b, float* x, const mps_solve_opts* o,
                      mps_solve_info* info, cudaStream_t s) {
    return csr_solve(kCG, h, b, x, o, info, s);
}

mps_status mps_test_persistent_barrier_timeout(mps_csr* h, const float* d_b, float* d_x, uint32_t spin_limit,
                                               int32_t silent_cta, cudaStream_t s) {
    if (!h || !d_b || !d_x || spin_limit == 0) return fail(MPS_ERR_ARG, "null argument or zero spin limit");
    const int32_t keep = h->persistent;
    h->persistent = 1;
    h->test_spin_limit = spin_limit;
    h->test_silent_cta = silent_cta;
    mps_solve_opts o;
    mps_solve_opts_default(&o);
    o.max_iter = 50;
    mps_solve_info info{};
    mps_status st = csr_solve(kCG, h, d_b, d_x, &o, &info, s);
    h->test_spin_limit = 0;
    h->test_silent_cta = -1;
    h->persistent = keep;
    if (st == MPS_OK && !info.persistent) return fail(MPS_ERR_ARG, "the persistent form does not fit this matrix");
    return st;
}

mps_status mps_csr_bicgstab(mps_csr* h, const float* b, float* x, const mps_solve_opts* o,
                            mps_solve_info* info, cudaStream_t s) {
    return csr_solve(kBiCG, h, b, x, o, info, s);
}

mps_status mps_csr_richardson(mps_csr* h, const float* b, float* x, const mps_solve_opts* o,
                              mps_solve_info* info, cudaStream_t s) {
    return csr_solve(kRich, h, b, x, o, info, s);
}

mps_status mps_csr_set_fsai(mps_csr* h, const int32_t* d_g_row_ptr, const int32_t* d_g_col_ind,
                            const float* d_g_vals, uint64_t g_nnz, cudaStream_t s) {
    if (!h || !d_g_row_ptr || !d_g_col_ind || !d_g_vals) return fail(MPS_ERR_ARG, "null argument");
    const uint32_t n = h->A.n_rows;
    fsai_product_free(h);
    csr_free(h->G);
    csr_free(h->Gt);
    fsai_work_free(h->fw);   // a network factor (if any) is replaced
    h->has_fsai = false;
    h->H.drop_graphs();
    mps_status st = alloc_csr(h->G, n, n, g_nnz, h->d_err, s);
    if (st != MPS_OK) return st;
    MPS_CUDA(cudaMemcpyAsync(h->G.rp, d_g_row_ptr, ((size_t)n + 1) * 4, cudaMemcpyDeviceToDevice, s));
    MPS_CUDA(cudaMemcpyAsync(h->G.ci, d_g_col_ind, g_nnz * 4, cudaMemcpyDeviceToDevice, s));
    MPS_CUDA(cudaMemcpyAsync(h->G.v, d_g_vals, g_nnz * 4, cudaMemcpyDeviceToDevice, s));
    // (G's SpMV plan is built below, with G^T's, by factor_plans_follow)
    // G^T through the same radix sort on (col<<32 | row) keys.
    unsigned long long* keys = nullptr;
    MPS_CUDA(stream_alloc(&keys, (g_nnz ? g_nnz : 1) * 8, s));
    MPS_CUDA(transpose_keys_launch(h->G, keys, s));
    st = build_from_keys(h->Gt, reinterpret_cast<const uint64_t*>(keys),
                         reinterpret_cast<const uint32_t*>(h->G.v), g_nnz, n, n, h->d_err, s, false);
    cudaFreeAsync(keys, s);
    if (st != MPS_OK) return st;
    MPS_CUDA(factor_plans_follow(h, s));
    h->has_fsai = true;
    return fsai_factor_changed(h, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Mixed-precision CG with FP64 iterative refinement.
// ---------------------------------------------------------------------------
namespace mps {

// r32 = (float)(b - A x) with FP64 gathers of x and FP64 accumulation over the
// FP32 matrix values; ||b - A x||^2 in FP64.
struct EpiResid64 {
    static constexpr int NS = 1;
    const double* b;
    float* r32;
    double* out;
    unsigned* counter;
    double* partials;
    __device__ bool active() const { return true; }
    __device__ void tick() const {}
    __device__ void on_skip() const {}
    __device__ void row(int r, double s, double* acc) const {
        const double rv = b[r] - s;
        r32[r] = (float)rv;
        acc[0] += rv * rv;
    }
    __device__ void finalize(const double* tot) const { *out = tot[0]; }
};

__global__ void ir_accumulate(double* __restrict__ x, const float* __restrict__ d, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] += (double)d[i];
}

__global__ void sumsq64(const double* __restrict__ b, int n, double* out, double* part,
                        unsigned* ctr) {
    __shared__ double red[kNT / 32];
    __shared__ int last;
    double a = 0.0;
    for (int i = blockIdx.x * kNT + threadIdx.x; i < n; i += gridDim.x * kNT) a += b[i] * b[i];
    const double v = block_sum<kNT>(a, red);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
    if (!arrive_last(ctr, &last)) return;
    const double t = sum_partials<kNT>(part, gridDim.x, red);
    if (threadIdx.x == 0) *out = t;
}

}  // namespace mps

extern "C" mps_status mps_csr_cg_mixed(mps_csr* h, const double* d_b, double* d_x,
                                       const mps_ir_opts* o_in, mps_ir_info* info,
                                       cudaStream_t s) {
    if (!h || !d_b || !d_x) return fail(MPS_ERR_ARG, "null argument");
    if (h->A.n_rows != h->A.n_cols) return fail(MPS_ERR_ARG, "solvers need a square matrix");
    mps_ir_opts o{};
    if (o_in) o = *o_in;
    const double tol = o.tol > 0 ? o.tol : 1e-10;
    const bool bf16 = o.value_bits == 16;
    const double inner_tol = o.inner_tol > 0 ? o.inner_tol : (bf16 ? 0.1 : 1e-3);
    const int max_outer = o.max_outer > 0 ? o.max_outer : 50;
    const int max_inner = o.max_inner > 0 ? o.max_inner : 2000;
    if (o.value_bits != 0 && o.value_bits != 16 && o.value_bits != 32)
        return fail(MPS_ERR_ARG, "value_bits must be 16 or 32");
    mps_solve_opts io;
    mps_solve_opts_default(&io);
    io.tol = inner_tol;
    io.max_iter = max_inner;
    io.precond = o.precond;
    io.host_loop = o.host_loop;
    mps_status st = prepare_precond(h, &io, s);
    if (st != MPS_OK) return st;
    MPS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), s));
    SolverHost& H = h->H;
    const int n = (int)h->A.n_rows;
    if (bf16 && !h->vb) {
        MPS_CUDA(dev_alloc(&h->vb, (h->A.nnz + kCsrPad) * sizeof(__nv_bfloat16), s));
        MPS_CUDA(to_bf16_launch(h->A.v, h->vb, h->A.nnz, s));
    }
    double* scal = nullptr;   // [0] = ||b||^2, [1] = ||r||^2
    MPS_CUDA(stream_alloc(&scal, 2 * sizeof(double), s));
    float* r32 = H.v(vTmp0);
    float* d32 = H.v(vTmp1);
    const int g = H.vgrid();
    sumsq64<<<g, kNT, 0, s>>>(d_b, n, scal, H.ws.partials, H.ws.counters + 13);
    MPS_CUDA(cudaMemsetAsync(d_x, 0, (size_t)n * sizeof(double), s));
    CsrOp inner{&h->A, bf16 ? h->vb : nullptr};
    CsrOp gop{&h->G, nullptr}, gtop{&h->Gt, nullptr}, mop{&h->M, nullptr};
    PrecondOps<CsrOp> pc{h->has_fsai ? &gop : nullptr, h->has_fsai ? &gtop : nullptr,
                         h->has_fsai && h->use_m ? &mop : nullptr};
    const CsrDev view = h->A.view();
    const size_t smem = spmv_smem_bytes<double>(view);
    smem_optin_k(spmv_tiles<double, double, false, EpiResid64>, smem);
    int outer = 0, inner_total = 0;
    bool converged = false;
    double rel = 1.0;
    if (o.ir_mode < MPS_IR_AUTO || o.ir_mode > MPS_IR_REPLACE || (o.ir_mode == MPS_IR_REPLACE && bf16)) {
        cudaFreeAsync(scal, s);
        return fail(MPS_ERR_ARG, o.ir_mode == MPS_IR_REPLACE ? "reliable updates run on FP32 values"
                                                              : "unknown ir_mode");
    }
    if (!bf16 && o.ir_mode != MPS_IR_RESTART) {
        // Reliable updates: one FP32 PCG, x in FP64, r replaced by the FP64
        // b - A x whenever it has dropped by inner_tol; then the FP64 true
        // residual of the result for the report.  Everything is enqueued at
        // once and read back after a single synchronization (b = 0 and a
        // non-finite b are settled on the device).
        mps_solve_opts ro = io;
        ro.tol = tol;
        const long cap = (long)max_inner * max_outer;
        ro.max_iter = cap > (1L << 30) ? (1 << 30) : (int)cap;
        mps_solve_info ii{};
        int rep = 0;
        bool persisted = false;
        const bool fsai_pc = o.precond == MPS_PRECOND_FSAI && h->has_fsai && h->use_m;
        const bool plain_pc = o.precond == MPS_PRECOND_NONE || o.precond == MPS_PRECOND_JACOBI;
        if (h->persistent && !io.host_loop && (fsai_pc || plain_pc)) {
            // one cooperative kernel for the whole solve when the rows of A
            // (and M) fit one CTA per SM (fsai_persistent.cu); the parameters
            // are the ones run_solve would upload
            SolveParams& P = *H.h_params;
            P.delta = inner_tol;
            P.tol = tol;
            P.omega = 0.01;
            P.max_iter = ro.max_iter;
            P.compat = 0;
            P.precond = o.precond;
            P.stall_window = ro.stall_window > 0 ? ro.stall_window : 400;
            MPS_CUDA(cudaMemcpyAsync(H.ws.d_params, H.h_params, sizeof(SolveParams), cudaMemcpyHostToDevice, s));
            const cudaError_t pe = fsai_pc ? persist_solve(h, d_b, d_x, s) : persist_cg_solve(h, s, d_b, d_x);
            if (pe == cudaSuccess) {
                MPS_CUDA(cudaMemcpyAsync(H.ws.h_sc, H.ws.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
                persisted = true;
            } else if (pe != cudaErrorNotSupported) {
                cudaFreeAsync(scal, s);
                return cuda_fail(pe, fsai_pc ? "persistent FSAI-PCG" : "persistent CG");
            }
        }
        if (!persisted)
            st = run_solve(kCG, inner, pc, H, nullptr, nullptr, &ro, &ii, s, 0, d_b, d_x, inner_tol, &rep, true);
        if (st == MPS_OK) {
            spmv_tiles<double, double, false, EpiResid64><<<h->A.plan.grid, kNT, smem, s>>>(
                view, d_x, EpiResid64{d_b, r32, scal + 1, H.ws.counters + 14, H.ws.partials});
            st = cudaGetLastError() == cudaSuccess ? MPS_OK : cuda_fail(cudaErrorLaunchFailure, "residual");
        }
        if (st == MPS_OK) {
            unsigned* h_err = reinterpret_cast<unsigned*>(H.h_aux + 2);
            MPS_CUDA(cudaMemcpyAsync(H.h_aux, scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
            MPS_CUDA(cudaMemcpyAsync(h_err, h->d_err, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            MPS_CUDA(cudaStreamSynchronize(s));
            st = solve_report(kCG, H, &ii, &rep);
            const double bnorm = std::sqrt(H.h_aux[0]);
            rel = bnorm > 0 ? std::sqrt(H.h_aux[1]) / bnorm : std::sqrt(H.h_aux[1]);
            st = solve_errors(h, h_err, st, s);
        }
        cudaFreeAsync(scal, s);
        if (info) {
            info->outer_iters = rep;
            info->inner_iters = ii.iters;
            info->converged = ii.converged && rel <= tol;
            info->persistent = persisted ? 1 + (fsai_pc ? h->pp.form : h->pp_a.form) : 0;
            info->rel_resid = rel;
        }
        return st;
    }
    // restarted refinement: ||b|| first (the stop test runs on the host)
    double hs[2] = {0, 0};
    MPS_CUDA(cudaMemcpyAsync(hs, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    const double bnorm = std::sqrt(hs[0]);
    for (;; ++outer) {
        // FP64 outer residual r = b - A x (FP32 copy feeds the inner solve)
        spmv_tiles<double, double, false, EpiResid64><<<h->A.plan.grid, kNT, smem, s>>>(
            view, d_x, EpiResid64{d_b, r32, scal + 1, H.ws.counters + 14, H.ws.partials});
        MPS_CUDA(cudaGetLastError());
        MPS_CUDA(cudaMemcpyAsync(hs + 1, scal + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
        MPS_CUDA(cudaStreamSynchronize(s));
        rel = bnorm > 0 ? std::sqrt(hs[1]) / bnorm : std::sqrt(hs[1]);
        if (!std::isfinite(rel)) break;
        if (rel <= tol || bnorm == 0.0) {
            converged = true;
            break;
        }
        if (outer >= max_outer) break;
        mps_solve_info ii{};
        st = run_solve(kCG, inner, pc, H, r32, d32, &io, &ii, s, bf16 ? 1 : 0);
        if (st != MPS_OK) break;
        inner_total += ii.iters;
        ir_accumulate<<<g, kNT, 0, s>>>(d_x, d32, n);
        MPS_CUDA(cudaGetLastError());
        if (ii.iters == 0) break;
    }
    cudaFreeAsync(scal, s);
    {
        unsigned err[2] = {0, 0};
        MPS_CUDA(cudaMemcpy(err, h->d_err, sizeof(err), cudaMemcpyDeviceToHost));
        st = solve_errors(h, err, st, s);
    }
    if (info) {
        info->outer_iters = outer;
        info->inner_iters = inner_total;
        info->converged = converged;
        info->persistent = 0;
        info->rel_resid = rel;
    }
    return st;
}

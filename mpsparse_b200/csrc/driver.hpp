// driver.hpp -- host driver shared by the CSR and BCSR solvers: workspace,
// graph capture with a device-side WHILE loop, result and info read-back.
#pragma once
#include <type_traits>

#include "solvers.cuh"
#include "csr_stream.cuh"

namespace mps {

cudaError_t diag_inv_launch(const CsrMat& A, float* dinv, cudaStream_t s);
cudaError_t transpose_keys_launch(const CsrMat& A, unsigned long long* keys, cudaStream_t s);
cudaError_t to_bf16_launch(const float* v, __nv_bfloat16* o, uint64_t n, cudaStream_t s);
int default_tile_nnz(uint64_t nnz, uint32_t n_rows);

// Programmatic dependent launch for the solver kernels (each calls
// pdl_begin() first): the next kernel's launch overlaps the tail of the
// current one.  On unless MPS_PDL=0; a graph capture that rejects it is
// retried without it (pdl_suspend).
bool pdl_enabled();
void pdl_suspend(bool off);

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*k)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t s,
                            Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = g;
    cfg.blockDim = b;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    if (pdl_enabled()) {
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&cfg, k, args...);
}

template <class K>
inline void smem_optin_k(K kernel, size_t smem) {
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// Resident CTAs per SM of a kernel at a given dynamic shared memory size
// (cached per kernel and size).
int resident_ctas(const void* kernel, int threads, size_t smem);

// Persistent grid for a tile loop: every CTA resident at once, so the static
// tile-to-CTA assignment never runs a second wave.
template <class K>
inline int persistent_grid(K kernel, size_t smem, int ntiles) {
    const int per_sm = resident_ctas(reinterpret_cast<const void*>(kernel), kNT, smem);
    int g = num_sms() * (per_sm > 0 ? per_sm : 1);
    if (g > kMaxPartials) g = kMaxPartials;
    if (g > ntiles) g = ntiles;
    return g < 1 ? 1 : g;
}

// CSR operator: A x through the tile kernel with a given epilogue.
struct CsrOp {
    const CsrMat* A;
    const __nv_bfloat16* vb = nullptr;
    template <class Epi>
    cudaError_t apply(const float* x, const Epi& e, cudaStream_t s) const {
        const CsrStreamDev v = A->stream_view(vb);
        const int nb = A->plan.stages;
        if (vb) {
            if (nb >= 3) launch<true, 3>(v, x, e, s);
            else launch<true, 2>(v, x, e, s);
        } else {
            if (nb >= 3) launch<false, 3>(v, x, e, s);
            else launch<false, 2>(v, x, e, s);
        }
        return cudaGetLastError();
    }
    template <bool BF16, int NB, class Epi>
    static void launch(const CsrStreamDev& v, const float* x, const Epi& e, cudaStream_t s) {
        const size_t smem = NB * stream_buf_bytes<BF16>(v.cap, v.rcap);
        smem_optin_k(spmv_stream<BF16, Epi, NB>, smem);
        const int g = persistent_grid(spmv_stream<BF16, Epi, NB>, smem, v.ntiles);
        launch_k(spmv_stream<BF16, Epi, NB>, dim3(g), dim3(kNT), smem, s, v, x, e);
    }
};

enum SolverKind { kCG = 0, kBiCG = 1, kRich = 2 };
enum VecSlot { vB = 0, vX, vR, vP, vQ, vR0, vS, vT, vXAlt, vW, vTmp0, vTmp1 };

// State a handle keeps for its solvers.
struct SolverHost {
    Workspace ws;
    GraphCache graphs[32];
    GraphCache graphs_ir[4];           // reliable-update CG per preconditioner
    double* v64 = nullptr;             // reliable updates: x (FP64) | b (FP64), n_pad each
    cudaStream_t cap = nullptr;
    SolveParams* h_params = nullptr;   // pinned
    float* dinv = nullptr;             // padded
    int n = 0;

    float* v(int slot) const { return ws.vec[slot]; }
    float4* v4(int slot) const { return reinterpret_cast<float4*>(ws.vec[slot]); }
    int n4() const { return (int)(ws.n_pad / 4); }
    int vgrid() const {
        int g = (n4() + kNT - 1) / kNT;
        const int cap_g = num_sms() * 4;
        if (g > cap_g) g = cap_g;
        return g < 1 ? 1 : g;
    }
    Ctx ctx(cudaGraphConditionalHandle h, int use) const {
        return Ctx{ws.sc, ws.partials, ws.counters, h, use};
    }

    cudaError_t ensure(size_t n_rows) {
        n = (int)n_rows;
        const size_t n_pad = (n_rows + 3) & ~size_t(3);
        if (ws.sc && ws.n_pad >= n_pad) return cudaSuccess;
        release();
        cudaError_t e;
        float* block = nullptr;
        const size_t nv = sizeof(ws.vec) / sizeof(ws.vec[0]);
        if ((e = cudaMalloc(&block, nv * (n_pad ? n_pad : 4) * sizeof(float))) != cudaSuccess) return e;
        if ((e = cudaMemset(block, 0, nv * (n_pad ? n_pad : 4) * sizeof(float))) != cudaSuccess) return e;
        for (size_t i = 0; i < nv; ++i) ws.vec[i] = block + i * (n_pad ? n_pad : 4);
        if ((e = cudaMalloc(&ws.partials, 4 * kMaxPartials * sizeof(double))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&ws.counters, 16 * sizeof(unsigned))) != cudaSuccess) return e;
        if ((e = cudaMemset(ws.counters, 0, 16 * sizeof(unsigned))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&ws.sc, sizeof(DevScalars))) != cudaSuccess) return e;
        if ((e = cudaMemset(ws.sc, 0, sizeof(DevScalars))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&ws.d_params, sizeof(SolveParams))) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&ws.h_sc, sizeof(DevScalars))) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&h_params, sizeof(SolveParams))) != cudaSuccess) return e;
        if (!cap && (e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) != cudaSuccess) return e;
        ws.n_pad = n_pad ? n_pad : 4;
        return cudaSuccess;
    }
    cudaError_t ensure_ir() {
        if (v64) return cudaSuccess;
        return cudaMalloc(&v64, 2 * ws.n_pad * sizeof(double));
    }
    double* x64() const { return v64; }
    double* b64() const { return v64 + ws.n_pad; }
    void drop_graphs() {
        for (auto& g : graphs_ir) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
            g = GraphCache{};
        }
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
            g = GraphCache{};
        }
    }
    void release() {
        drop_graphs();
        if (ws.vec[0]) cudaFree(ws.vec[0]);
        if (ws.partials) cudaFree(ws.partials);
        if (ws.counters) cudaFree(ws.counters);
        if (ws.sc) cudaFree(ws.sc);
        if (ws.d_params) cudaFree(ws.d_params);
        if (ws.h_sc) cudaFreeHost(ws.h_sc);
        if (h_params) cudaFreeHost(h_params);
        if (dinv) cudaFree(dinv);
        if (v64) cudaFree(v64);
        v64 = nullptr;
        ws = Workspace{};
        h_params = nullptr;
        dinv = nullptr;
    }
    void destroy() {
        release();
        if (cap) cudaStreamDestroy(cap);
        cap = nullptr;
    }
};

// Preconditioner operators for PCG (FSAI: G and G^T as CSR).
template <class Op>
struct PrecondOps {
    const CsrOp* G = nullptr;
    const CsrOp* Gt = nullptr;
};

template <class Op>
cudaError_t launch_init(SolverKind kind, int precond, const Op& op, const PrecondOps<Op>& pc,
                        SolverHost& H, const Ctx& c, cudaStream_t s, bool ir = false) {
    const int n4 = H.n4(), g = H.vgrid();
    DevScalars* sc = H.ws.sc;
    switch (kind) {
        case kCG:
            if (ir) {
                launch_k(cg_init_ir, dim3(g), dim3(kNT), 0, s, static_cast<const double*>(H.b64()), H.x64(),
                         H.v(vR), H.v(vP), static_cast<const float*>(H.dinv), H.n,
                         static_cast<const SolveParams*>(H.ws.d_params), c);
                if (precond == MPS_PRECOND_FSAI) {
                    cudaError_t e = pc.G->apply(H.v(vR), EpiFsai1{H.v(vW), sc, c.ctr + 3, c.part}, s);
                    if (e != cudaSuccess) return e;
                    e = pc.Gt->apply(H.v(vW), EpiFsai2{H.v(vP), sc}, s);
                    if (e != cudaSuccess) return e;
                }
                break;
            }
            launch_k(cg_init, dim3(g), dim3(kNT), 0, s, H.v4(vB), H.v4(vX), H.v4(vR), H.v4(vP),
                                      reinterpret_cast<const float4*>(H.dinv), n4, H.n,
                                      H.ws.d_params, c);
            if (precond == MPS_PRECOND_FSAI) {
                cudaError_t e = pc.G->apply(H.v(vR), EpiFsai1{H.v(vW), sc, c.ctr + 3, c.part}, s);
                if (e != cudaSuccess) return e;
                e = pc.Gt->apply(H.v(vW), EpiFsai2{H.v(vP), sc}, s);
                if (e != cudaSuccess) return e;
            }
            break;
        case kBiCG:
            launch_k(bicg_init, dim3(g), dim3(kNT), 0, s, H.v4(vB), H.v4(vX), H.v4(vR), H.v4(vR0), H.v4(vP),
                                        H.v4(vQ), n4, H.n, H.ws.d_params, c);
            break;
        case kRich:
            launch_k(rich_init, dim3(g), dim3(kNT), 0, s, H.v4(vB), H.v4(vX), n4, H.n, H.ws.d_params, c);
            break;
    }
    return cudaGetLastError();
}

template <class Op>
cudaError_t launch_body(SolverKind kind, int precond, const Op& op, const PrecondOps<Op>& pc,
                        SolverHost& H, const Ctx& c, cudaStream_t s, bool ir = false) {
    const int n4 = H.n4(), g = H.vgrid();
    DevScalars* sc = H.ws.sc;
    cudaError_t e = cudaSuccess;
    const float4* dinv4 = reinterpret_cast<const float4*>(H.dinv);
    switch (kind) {
        case kCG:
            e = op.apply(H.v(vP), EpiCgPq{H.v(vQ), H.v(vP), sc, c.ctr + 1, c.part}, s);
            if (e != cudaSuccess) return e;
            if constexpr (std::is_same<Op, CsrOp>::value) {
                if (ir) {
                    const float* dv = precond ? H.dinv : nullptr;
                    launch_k(cg_update_xr_ir, dim3(g), dim3(kNT), 0, s, H.x64(), H.v(vR),
                             static_cast<const float*>(H.v(vP)), static_cast<const float*>(H.v(vQ)), dv,
                             H.n, c);
                    // FP64 true residual when a replacement is due (returns at once otherwise)
                    const CsrDev view = op.A->view();
                    const size_t smem = spmv_smem_bytes<double>(view);
                    smem_optin_k(spmv_tiles<double, double, false, EpiReplace>, smem);
                    spmv_tiles<double, double, false, EpiReplace><<<op.A->plan.grid, kNT, smem, s>>>(
                        view, H.x64(), EpiReplace{H.b64(), H.v(vR), dv, sc, c.ctr + 4, c.part});
                    if (precond == MPS_PRECOND_FSAI) {
                        e = pc.G->apply(H.v(vR), EpiFsai1{H.v(vW), sc, c.ctr + 3, c.part}, s);
                        if (e != cudaSuccess) return e;
                        e = pc.Gt->apply(H.v(vW), EpiFsai2{H.v(vP), sc, nullptr, nullptr, H.v(vR), H.dinv, c, 1}, s);
                        if (e != cudaSuccess) return e;
                    } else {
                        launch_k(cg_update_p, dim3(g), dim3(kNT), 0, s, H.v4(vP), H.v4(vR), dinv4, n4, c);
                    }
                    break;
                }
            }
            launch_k(cg_update_xr, dim3(g), dim3(kNT), 0, s, H.v4(vX), H.v4(vR), H.v4(vP), H.v4(vQ),
                                           precond ? dinv4 : nullptr, n4, c);
            if (precond == MPS_PRECOND_FSAI) {
                e = pc.G->apply(H.v(vR), EpiFsai1{H.v(vW), sc, c.ctr + 3, c.part}, s);
                if (e != cudaSuccess) return e;
                e = pc.Gt->apply(H.v(vW), EpiFsai2{H.v(vP), sc, nullptr, nullptr, H.v(vR), H.dinv, c, 1}, s);
                if (e != cudaSuccess) return e;
            } else {
                launch_k(cg_update_p, dim3(g), dim3(kNT), 0, s, H.v4(vP), H.v4(vR), dinv4, n4, c);
            }
            break;
        case kBiCG:
            launch_k(bicg_update_p, dim3(g), dim3(kNT), 0, s, H.v4(vP), H.v4(vR), H.v4(vQ), n4, c);
            e = op.apply(H.v(vP), EpiBicgV{H.v(vQ), H.v(vR0), sc, c.ctr + 5, c.part}, s);
            if (e != cudaSuccess) return e;
            launch_k(bicg_update_s, dim3(g), dim3(kNT), 0, s, H.v4(vS), H.v4(vR), H.v4(vQ), n4, c);
            e = op.apply(H.v(vS), EpiBicgT{H.v(vT), H.v(vS), sc, c.ctr + 6, c.part}, s);
            if (e != cudaSuccess) return e;
            launch_k(bicg_update_xr, dim3(g), dim3(kNT), 0, s, H.v4(vX), H.v4(vR), H.v4(vP), H.v4(vR0), H.v4(vS),
                                             H.v4(vT), H.v4(vXAlt), n4, c);
            break;
        case kRich:
            e = op.apply(H.v(vX), EpiRich{H.v(vX), H.v(vXAlt), H.v(vB), sc, c.ctr + 9, c.part, c, 0}, s);
            if (e != cudaSuccess) return e;
            e = op.apply(H.v(vXAlt), EpiRich{H.v(vXAlt), H.v(vX), H.v(vB), sc, c.ctr + 10, c.part, c, 1}, s);
            break;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

// Capture: [init kernels] -> WHILE(cond) { body kernels }.
template <class Op>
cudaError_t build_graph(SolverKind kind, int precond, const Op& op, const PrecondOps<Op>& pc,
                        SolverHost& H, GraphCache& gc, bool ir = false) {
    cudaStream_t cs = H.cap;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle h{};
    cudaGraphNode_t cn;
    cudaGraphNodeParams cp = {};
    cudaGraph_t body = nullptr;
    if ((e = cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd)) != cudaSuccess) goto abort;
    if ((e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault)) != cudaSuccess)
        goto abort;
    if ((e = launch_init(kind, precond, op, pc, H, H.ctx(h, 1), cs, ir)) != cudaSuccess) goto abort;
    if ((e = cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd)) != cudaSuccess) goto abort;
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if ((e = cudaGraphAddNode(&cn, g, deps, nd, &cp)) != cudaSuccess) goto abort;
    body = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamUpdateCaptureDependencies(cs, &cn, 1, cudaStreamSetCaptureDependencies)) !=
        cudaSuccess)
        goto abort;
    if ((e = cudaStreamEndCapture(cs, &g)) != cudaSuccess) return e;
    if ((e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    e = launch_body(kind, precond, op, pc, H, H.ctx(h, 1), cs, ir);
    {
        cudaGraph_t b2 = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cs, &b2);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    e = cudaGraphInstantiate(&gc.exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        gc = GraphCache{};
        return e;
    }
    gc.graph = g;
    return cudaSuccess;
abort:
    {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(cs, &junk);
        if (junk) cudaGraphDestroy(junk);
    }
    return e;
}

// Run one solve: b (device, n floats) -> x (device, n floats).
// Reliable-update mode (CG on a CSR only): d_b64 -> d_x64 in FP64, d_b/d_x
// unused; *replaced receives the number of residual replacements.
template <class Op>
mps_status run_solve(SolverKind kind, const Op& op, const PrecondOps<Op>& pc, SolverHost& H,
                     const float* d_b, float* d_x, const mps_solve_opts* o_in,
                     mps_solve_info* info, cudaStream_t s, int variant = 0,
                     const double* d_b64 = nullptr, double* d_x64 = nullptr, double delta = 0.0,
                     int* replaced = nullptr) {
    mps_solve_opts o;
    mps_solve_opts_default(&o);
    if (o_in) o = *o_in;
    const bool ir = d_b64 != nullptr;
    if (ir && (kind != kCG || o.reference_compat || !std::is_same<Op, CsrOp>::value))
        return fail(MPS_ERR_ARG, "reliable updates run CG on a CSR matrix");
    SolveParams& P = *H.h_params;
    P.delta = delta;
    P.tol = o.tol > 0 ? o.tol : 1e-6;
    P.omega = o.omega != 0 ? o.omega : 0.01;
    P.max_iter = o.max_iter > 0 ? o.max_iter : 2000;
    P.compat = o.reference_compat ? 1 : 0;
    P.precond = kind == kCG && !P.compat ? o.precond : 0;
    P.stall_window = o.stall_window > 0 ? o.stall_window : 400;
    const int precond = P.precond;
    MPS_CUDA(cudaMemcpyAsync(H.ws.d_params, H.h_params, sizeof(SolveParams), cudaMemcpyHostToDevice, s));
    if (ir) {
        MPS_CUDA(H.ensure_ir());
        MPS_CUDA(cudaMemcpyAsync(H.b64(), d_b64, (size_t)H.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else {
        MPS_CUDA(cudaMemcpyAsync(H.v(vB), d_b, (size_t)H.n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    if (!o.host_loop) {
        GraphCache& gc = ir ? H.graphs_ir[precond & 3] : H.graphs[(kind * 4 + precond) * 2 + (variant & 1)];
        if (!gc.exec) {
            // captured once per (solver, preconditioner) on the handle's
            // private stream; the graph only references handle-owned buffers
            cudaError_t e = build_graph(kind, precond, op, pc, H, gc, ir);
            if (e != cudaSuccess && pdl_enabled()) {   // retry with plain stream order
                cudaGetLastError();
                pdl_suspend(true);
                e = build_graph(kind, precond, op, pc, H, gc, ir);
                pdl_suspend(false);
            }
            if (e != cudaSuccess) return cuda_fail(e, "solver graph capture");
        }
        MPS_CUDA(cudaGraphLaunch(gc.exec, s));
    } else {
        MPS_CUDA(launch_init(kind, precond, op, pc, H, H.ctx({}, 0), s, ir));
        const int per_poll = 16;
        for (long it = 0;; it += per_poll) {
            for (int k = 0; k < per_poll; ++k)
                MPS_CUDA(launch_body(kind, precond, op, pc, H, H.ctx({}, 0), s, ir));
            MPS_CUDA(cudaMemcpyAsync(H.ws.h_sc, H.ws.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
            MPS_CUDA(cudaStreamSynchronize(s));
            if (H.ws.h_sc->done) break;
            if (it > 100000000L) return fail(MPS_ERR_TIMEOUT, "host loop did not stop");
        }
    }
    if (ir) {
        MPS_CUDA(cudaMemcpyAsync(d_x64, H.x64(), (size_t)H.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else {
        const int nb = (H.n + 255) / 256;
        launch_k(copy_result, dim3(nb < 1184 ? (nb ? nb : 1) : 1184), dim3(256), 0, s, H.v(vX),
                 static_cast<const float*>(H.v(vXAlt)), H.v(vXAlt), d_x, H.n,
                 kind == kRich ? kResRich : kResX, static_cast<const DevScalars*>(H.ws.sc));
        MPS_CUDA(cudaGetLastError());
    }
    MPS_CUDA(cudaMemcpyAsync(H.ws.h_sc, H.ws.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    MPS_CUDA(cudaStreamSynchronize(s));
    const DevScalars& r = *H.ws.h_sc;
    if (info) {
        info->iters = r.iter;
        info->converged = r.converged;
        info->breakdown = r.breakdown;
        info->stalled = r.stalled;
        info->compat_snapshot = r.snapshot;
        info->reserved = 0;
        const double num = kind == kCG ? r.rr : r.rnorm2;
        info->rel_resid = r.bnorm2 > 0 ? sqrt(num / r.bnorm2) : sqrt(num);
    }
    if (replaced) *replaced = r.replaced;
    if (r.err & kErrNotFinite) return fail(MPS_ERR_NOT_FINITE, "right-hand side holds NaN or Inf");
    if (r.err & kErrTimeout) return fail(MPS_ERR_TIMEOUT, "solver loop stopped by its watchdog");
    return MPS_OK;
}

}  // namespace mps

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
// retried without it (pdl_suspend, which returns the previous setting).
bool pdl_enabled();
bool pdl_suspend(bool off);

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
    // *out = ||b - A x||^2 in FP64 (the true residual of a returned x; the
    // FP32 values, never the BF16 copy).
    cudaError_t true_resid(const float* x, const float* b, double* out, unsigned* ctr, double* part,
                           cudaStream_t s) const {
        const CsrDev view = A->view();
        const size_t smem = spmv_smem_bytes<double>(view);
        smem_optin_k(spmv_tiles<float, double, false, EpiTrueResid>, smem);
        spmv_tiles<float, double, false, EpiTrueResid><<<A->plan.grid, kNT, smem, s>>>(
            view, x, EpiTrueResid{b, out, ctr, part});
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
// FSAI-PCG keeps its residual in a pair of buffers (vR, vR1) and, with
// M = G^T G, its direction too (vP, vP1); vS and vT are BiCGSTAB's and free
// during a CG solve.  vW holds w = G r (split form) or z = M r (product form).
constexpr int vR1 = vS;
constexpr int vP1 = vT;

// State a handle keeps for its solvers.
struct SolverHost {
    Workspace ws;
    GraphCache graphs[32];
    GraphCache graphs_ir[4];           // reliable-update CG per preconditioner
    double* v64 = nullptr;             // reliable updates: x (FP64) | b (FP64), n_pad each
    cudaStream_t cap = nullptr;
    cudaStream_t cap_branch = nullptr; // captures the body of an IF node
    SolveParams* h_params = nullptr;   // pinned
    double* h_aux = nullptr;           // pinned, 4 doubles: read-backs after a deferred solve
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
    Ctx ctx(cudaGraphConditionalHandle h, int use, cudaGraphConditionalHandle hif = {}) const {
        return Ctx{ws.sc, ws.partials, ws.counters, h, use, hif};
    }

    // Work vectors, FP64 partial sums, counters and scalars (device, from the
    // library pool, on stream s) and the pinned scalar mirrors.
    cudaError_t ensure(size_t n_rows, cudaStream_t s) {
        n = (int)n_rows;
        const size_t n_pad = (n_rows + 3) & ~size_t(3);
        if (ws.sc && ws.n_pad >= n_pad) return cudaSuccess;
        release();
        cudaError_t e;
        float* block = nullptr;
        const size_t nv = sizeof(ws.vec) / sizeof(ws.vec[0]);
        const size_t vbytes = nv * (n_pad ? n_pad : 4) * sizeof(float);
        if ((e = dev_alloc(&block, vbytes, s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(block, 0, vbytes, s)) != cudaSuccess) return e;
        for (size_t i = 0; i < nv; ++i) ws.vec[i] = block + i * (n_pad ? n_pad : 4);
        if ((e = dev_alloc(&ws.partials, 4 * kMaxPartials * sizeof(double), s)) != cudaSuccess) return e;
        if ((e = dev_alloc(&ws.counters, 16 * sizeof(unsigned), s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(ws.counters, 0, 16 * sizeof(unsigned), s)) != cudaSuccess) return e;
        if ((e = dev_alloc(&ws.sc, sizeof(DevScalars), s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(ws.sc, 0, sizeof(DevScalars), s)) != cudaSuccess) return e;
        if ((e = dev_alloc(&ws.d_params, sizeof(SolveParams), s)) != cudaSuccess) return e;
        static_assert(sizeof(DevScalars) + sizeof(SolveParams) + 4 * sizeof(double) + 512 <= 4096,
                      "scalar mirrors fit one pinned block");
        unsigned char* pin = static_cast<unsigned char*>(pinned_block_get(4096));
        if (!pin) return cudaErrorMemoryAllocation;
        ws.h_sc = reinterpret_cast<DevScalars*>(pin);
        h_params = reinterpret_cast<SolveParams*>(pin + ((sizeof(DevScalars) + 255) & ~size_t(255)));
        h_aux = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(h_params) +
                                          ((sizeof(SolveParams) + 255) & ~size_t(255)));
        if (!cap && !(cap = capture_stream_get())) return cudaErrorUnknown;
        if (!cap_branch && !(cap_branch = capture_stream_get())) return cudaErrorUnknown;
        ws.n_pad = n_pad ? n_pad : 4;
        return cudaSuccess;
    }
    cudaError_t ensure_ir(cudaStream_t s) {
        if (v64) return cudaSuccess;
        return dev_alloc(&v64, 2 * ws.n_pad * sizeof(double), s);
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
        dev_free(ws.vec[0]);
        dev_free(ws.partials);
        dev_free(ws.counters);
        dev_free(ws.sc);
        dev_free(ws.d_params);
        pinned_block_put(ws.h_sc);      // one block holds all three mirrors
        dev_free(dinv);
        dev_free(v64);
        v64 = nullptr;
        ws = Workspace{};
        h_params = nullptr;
        h_aux = nullptr;
        dinv = nullptr;
    }
    void destroy() {
        release();
        capture_stream_put(cap);
        capture_stream_put(cap_branch);
        cap = nullptr;
        cap_branch = nullptr;
    }
};

// Preconditioner operators for PCG (FSAI: G and G^T as CSR, and M = G^T G
// when the product form is in force).
template <class Op>
struct PrecondOps {
    const CsrOp* G = nullptr;
    const CsrOp* Gt = nullptr;
    const CsrOp* M = nullptr;
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
                if (precond == MPS_PRECOND_FSAI && pc.M)
                    return pc.M->apply(H.v(vR), EpiMz{H.v(vW), sc, c.ctr + 3, c.part, H.v(vR)}, s);
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
            if (precond == MPS_PRECOND_FSAI && pc.M)
                return pc.M->apply(H.v(vR), EpiMz{H.v(vW), sc, c.ctr + 3, c.part, H.v(vR)}, s);
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

// Replacement branch of reliable-update FSAI-PCG: r = (float)(b - A x) in
// FP64 (EpiReplace) and its G-apply (EpiFsai1R).  Both return at once unless
// a replacement is due, so the host loop may launch them every iteration;
// a graph runs them under an IF node.
inline cudaError_t launch_replace_fsai(const CsrOp& op, const PrecondOps<CsrOp>& pc, SolverHost& H,
                                       const Ctx& c, cudaStream_t s) {
    const CsrDev view = op.A->view();
    const size_t smem = spmv_smem_bytes<double>(view);
    smem_optin_k(spmv_tiles<double, double, false, EpiReplace>, smem);
    spmv_tiles<double, double, false, EpiReplace><<<op.A->plan.grid, kNT, smem, s>>>(
        view, H.x64(), EpiReplace{H.b64(), H.v(vR), H.dinv, H.ws.sc, c.ctr + 4, c.part, H.v(vR1)});
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return pc.G->apply(nullptr, EpiFsai1R{{H.v(vW), H.ws.sc, c.ctr + 3, c.part}, H.v(vR), H.v(vR1)}, s);
}

// FSAI-PCG with M = G^T G: one iteration (K1: direction + A p; K2: update +
// z = M r'), c.h being the loop the iteration runs in.  These kernels are
// launched in plain stream order: each fills every SM with its own CTAs, and
// programmatic dependent launch measured ~10% slower per iteration here
// (it does pay for the elementwise kernels of the other solvers).
inline cudaError_t launch_prod_iter(const CsrOp& op, const PrecondOps<CsrOp>& pc, SolverHost& H, const Ctx& c,
                                    cudaStream_t s, bool ir) {
    DevScalars* sc = H.ws.sc;
    const bool pdl_prev = pdl_suspend(true);
    cudaError_t e = op.apply(nullptr, EpiCgPqZ{H.v(vQ), H.v(vW), H.v(vP), H.v(vP1), H.v(vR), H.v(vR1), H.dinv,
                                               sc, c.ctr + 1, c.part}, s);
    const float* ra = H.v(vR);
    const float* rb = H.v(vR1);
    const float* pa = H.v(vP);
    const float* pb = H.v(vP1);
    if (e == cudaSuccess) {
        if (ir)
            e = pc.M->apply(nullptr, EpiFsaiM<true>{ra, rb, H.v(vQ), pa, pb, H.x64(), H.dinv, H.v(vW), sc,
                                                     c.ctr + 2, c.part, c}, s);
        else
            e = pc.M->apply(nullptr, EpiFsaiM<false>{ra, rb, H.v(vQ), pa, pb, H.v(vX), H.dinv, H.v(vW), sc,
                                                      c.ctr + 2, c.part, c}, s);
    }
    pdl_suspend(pdl_prev);
    return e;
}

// Its replacement step: r = (float)(b - A x) in FP64, then z = M r.  Both
// return at once unless a replacement is due.  c_out.h: the loop around the
// iterations and this step; c_in.h: the iterations' loop (re-armed).
inline cudaError_t launch_prod_replace(const CsrOp& op, const PrecondOps<CsrOp>& pc, SolverHost& H,
                                       const Ctx& c_out, const Ctx& c_in, cudaStream_t s) {
    const CsrDev view = op.A->view();
    const size_t smem = spmv_smem_bytes<double>(view);
    smem_optin_k(spmv_tiles<double, double, false, EpiReplace>, smem);
    spmv_tiles<double, double, false, EpiReplace><<<op.A->plan.grid, kNT, smem, s>>>(
        view, H.x64(),
        EpiReplace{H.b64(), H.v(vR), H.dinv, H.ws.sc, c_out.ctr + 4, c_out.part, H.v(vR1), c_out, 1});
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const bool pdl_prev = pdl_suspend(true);
    e = pc.M->apply(nullptr, EpiMzR{H.v(vW), H.ws.sc, c_in.ctr + 3, c_in.part, H.v(vR), H.v(vR1), c_in, 1}, s);
    pdl_suspend(pdl_prev);
    return e;
}

// During a capture on cs: append an IF node on `hif` after the captured work
// and capture fn(bs) into its body on the stream bs.
template <class F>
cudaError_t capture_if(cudaStream_t cs, cudaStream_t bs, cudaGraphConditionalHandle hif, F&& fn) {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hif;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddNode(&node, g, deps, nd, &cp)) != cudaSuccess) return e;
    if ((e = cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies)) !=
        cudaSuccess)
        return e;
    if ((e = cudaStreamBeginCaptureToGraph(bs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return e;
    e = fn(bs);
    cudaGraph_t b2 = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(bs, &b2);
    return e != cudaSuccess ? e : e2;
}

// One iteration.  branch_cap: set while capturing a graph whose reliable-update
// FSAI body holds the replacement branch under an IF node (c.hif).
template <class Op>
cudaError_t launch_body(SolverKind kind, int precond, const Op& op, const PrecondOps<Op>& pc,
                        SolverHost& H, const Ctx& c, cudaStream_t s, bool ir = false,
                        cudaStream_t branch_cap = nullptr) {
    const int n4 = H.n4(), g = H.vgrid();
    DevScalars* sc = H.ws.sc;
    cudaError_t e = cudaSuccess;
    const float4* dinv4 = reinterpret_cast<const float4*>(H.dinv);
    switch (kind) {
        case kCG:
            if constexpr (std::is_same<Op, CsrOp>::value) {
                if (precond == MPS_PRECOND_FSAI && pc.M) {
                    // product form (a reliable-update graph nests its loops:
                    // build_graph_nested; here the host loop or FP32 PCG)
                    e = launch_prod_iter(op, pc, H, c, s, ir);
                    if (e != cudaSuccess || !ir) return e;
                    return launch_prod_replace(op, pc, H, c, c, s);
                }
            }
            e = op.apply(H.v(vP), EpiCgPq{H.v(vQ), H.v(vP), sc, c.ctr + 1, c.part}, s);
            if (e != cudaSuccess) return e;
            if constexpr (std::is_same<Op, CsrOp>::value) {
                if (precond == MPS_PRECOND_FSAI) {
                    // x/r update fused into the G-apply (EpiFsaiR), then
                    // [replacement branch], then p = G^T w + beta p
                    const float* ra = H.v(vR);
                    const float* rb = H.v(vR1);
                    if (ir)
                        e = pc.G->apply(nullptr, EpiFsaiR<true>{ra, rb, H.v(vQ), H.v(vP), H.x64(), H.dinv,
                                                                 H.v(vW), sc, c.ctr + 2, c.part, c}, s);
                    else
                        e = pc.G->apply(nullptr, EpiFsaiR<false>{ra, rb, H.v(vQ), H.v(vP), H.v(vX), H.dinv,
                                                                  H.v(vW), sc, c.ctr + 2, c.part, c}, s);
                    if (e != cudaSuccess) return e;
                    bool pdl_prev = false;
                    if (ir) {
                        if (branch_cap) {
                            e = capture_if(s, branch_cap, c.hif, [&](cudaStream_t bs) {
                                return launch_replace_fsai(op, pc, H, c, bs);
                            });
                            if (e != cudaSuccess) return e;
                            // the next kernel follows the IF node: plain stream order
                            pdl_prev = pdl_suspend(true);
                        } else {
                            e = launch_replace_fsai(op, pc, H, c, s);
                            if (e != cudaSuccess) return e;
                        }
                    }
                    e = pc.Gt->apply(H.v(vW), EpiFsai2{H.v(vP), sc, nullptr, nullptr, H.v(vR), H.dinv, c, 1,
                                                       H.v(vR1)}, s);
                    if (ir && branch_cap) pdl_suspend(pdl_prev);
                    return e;
                }
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
    cudaGraphConditionalHandle hif{};
    cudaGraphNode_t cn;
    cudaGraphNodeParams cp = {};
    cudaGraph_t body = nullptr;
    // reliable-update FSAI-PCG: the replacement branch sits under an IF node
    const bool branch = ir && kind == kCG && precond == MPS_PRECOND_FSAI && !pc.M &&
                        std::is_same<Op, CsrOp>::value;
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
    if (branch &&
        (e = cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault)) != cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    if ((e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    e = launch_body(kind, precond, op, pc, H, H.ctx(h, 1, hif), cs, ir, branch ? H.cap_branch : nullptr);
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

// Reliable-update FSAI-PCG with M = G^T G:
//   [init] -> WHILE(h_out) { WHILE(h_in) { kUnroll iterations } -> replacement step }
// The inner body holds several iterations so that their kernels chain by
// programmatic dependent launch; once the solve stops or a replacement is
// due, the rest of the body returns at once.
constexpr int kUnroll = 16;   // 24.3 / 23.8 / 23.5 us per iteration at 4 / 8 / 16 (512^2)

inline cudaError_t build_graph_nested(const CsrOp& op, const PrecondOps<CsrOp>& pc, SolverHost& H,
                                      GraphCache& gc) {
    cudaStream_t cs = H.cap;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr, body_out = nullptr, body_in = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraphConditionalHandle h_out{}, h_in{};
    cudaGraphNode_t n_out, n_in;
    cudaGraphNodeParams cp = {};
    auto end_capture = [&](cudaError_t err) {   // a failed capture of the top graph
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(cs, &junk);
        if (junk) cudaGraphDestroy(junk);
        return err;
    };
    if ((e = cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd)) != cudaSuccess) return end_capture(e);
    if ((e = cudaGraphConditionalHandleCreate(&h_out, g, 0, cudaGraphCondAssignDefault)) != cudaSuccess)
        return end_capture(e);
    if ((e = launch_init(kCG, MPS_PRECOND_FSAI, op, pc, H, H.ctx(h_out, 1), cs, true)) != cudaSuccess)
        return end_capture(e);
    if ((e = cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &nd)) != cudaSuccess) return end_capture(e);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h_out;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if ((e = cudaGraphAddNode(&n_out, g, deps, nd, &cp)) != cudaSuccess) return end_capture(e);
    body_out = cp.conditional.phGraph_out[0];
    if ((e = cudaStreamUpdateCaptureDependencies(cs, &n_out, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
        return end_capture(e);
    if ((e = cudaStreamEndCapture(cs, &g)) != cudaSuccess) return e;
    // outer body: WHILE(h_in) -> replacement step
    if ((e = cudaGraphConditionalHandleCreate(&h_in, body_out, 1, cudaGraphCondAssignDefault)) != cudaSuccess ||
        (e = cudaStreamBeginCaptureToGraph(cs, body_out, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
            cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h_in;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if ((e = cudaGraphAddNode(&n_in, body_out, nullptr, 0, &cp)) == cudaSuccess) {
        body_in = cp.conditional.phGraph_out[0];
        e = cudaStreamUpdateCaptureDependencies(cs, &n_in, 1, cudaStreamSetCaptureDependencies);
    }
    if (e == cudaSuccess) {
        const bool prev = pdl_suspend(true);   // first kernel after a conditional node
        e = launch_prod_replace(op, pc, H, H.ctx(h_out, 1), H.ctx(h_in, 1), cs);
        pdl_suspend(prev);
    }
    {
        cudaGraph_t b2 = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &b2);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    // inner body: kUnroll iterations
    if ((e = cudaStreamBeginCaptureToGraph(cs, body_in, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
        cudaSuccess) {
        cudaGraphDestroy(g);
        return e;
    }
    for (int u = 0; u < kUnroll && e == cudaSuccess; ++u) e = launch_prod_iter(op, pc, H, H.ctx(h_in, 1), cs, true);
    {
        cudaGraph_t b2 = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &b2);
        if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gc.exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        gc = GraphCache{};
        return e;
    }
    gc.graph = g;
    return cudaSuccess;
}

// Run one solve: b (device, n floats) -> x (device, n floats).
// Reliable-update mode (CG on a CSR only): d_b64 -> d_x64 in FP64, d_b/d_x
// unused; *replaced receives the number of residual replacements.
// The outcome of a solve from the scalars read back into H.ws.h_sc.
// have_true: the solve ended with the FP64 true residual of its x (r.true_rr),
// which then decides `converged` (outside reference_compat); otherwise (the
// inner solve of a refinement) `converged` is the stop rule and true_resid -1.
inline mps_status solve_report(SolverKind kind, const SolverHost& H, mps_solve_info* info, int* replaced,
                               bool have_true = false) {
    const DevScalars& r = *H.ws.h_sc;
    if (info) {
        info->iters = r.iter;
        info->persistent = 0;
        info->reserved = 0;
        info->stop_rule_met = r.converged;
        info->breakdown = r.breakdown;
        info->stalled = r.stalled;
        info->compat_snapshot = r.snapshot;
        const double num = kind == kCG ? r.rr : r.rnorm2;
        info->rel_resid = r.bnorm2 > 0 ? sqrt(num / r.bnorm2) : sqrt(num);
        if (have_true) {
            info->true_resid = r.bnorm2 > 0 ? sqrt(r.true_rr / r.bnorm2) : sqrt(r.true_rr);
            info->converged = r.compat ? r.converged : (r.err == 0 && r.true_rr <= r.tol2);
        } else {
            info->true_resid = -1.0;
            info->converged = r.converged;
        }
    }
    if (replaced) *replaced = r.replaced;
    if (r.err & kErrNotFinite) return fail(MPS_ERR_NOT_FINITE, "right-hand side holds NaN or Inf");
    if (r.err & kErrTimeout) return fail(MPS_ERR_TIMEOUT, "solver loop stopped by its watchdog");
    return MPS_OK;
}

// defer: enqueue everything (the scalars' read-back into H.ws.h_sc included)
// and return without synchronizing; the caller synchronizes the stream and
// calls solve_report.
template <class Op>
mps_status run_solve(SolverKind kind, const Op& op, const PrecondOps<Op>& pc, SolverHost& H,
                     const float* d_b, float* d_x, const mps_solve_opts* o_in,
                     mps_solve_info* info, cudaStream_t s, int variant = 0,
                     const double* d_b64 = nullptr, double* d_x64 = nullptr, double delta = 0.0,
                     int* replaced = nullptr, bool defer = false) {
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
        MPS_CUDA(H.ensure_ir(s));
        MPS_CUDA(cudaMemcpyAsync(H.b64(), d_b64, (size_t)H.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else {
        MPS_CUDA(cudaMemcpyAsync(H.v(vB), d_b, (size_t)H.n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    if (!o.host_loop) {
        GraphCache& gc = ir ? H.graphs_ir[precond & 3] : H.graphs[(kind * 4 + precond) * 2 + (variant & 1)];
        if (!gc.exec) {
            // captured once per (solver, preconditioner) on the handle's
            // private stream; the graph only references handle-owned buffers
            auto build = [&]() -> cudaError_t {
                if constexpr (std::is_same<Op, CsrOp>::value) {
                    if (ir && kind == kCG && precond == MPS_PRECOND_FSAI && pc.M)
                        return build_graph_nested(op, pc, H, gc);
                }
                return build_graph(kind, precond, op, pc, H, gc, ir);
            };
            cudaError_t e = build();
            if (e != cudaSuccess && pdl_enabled()) {   // retry with plain stream order
                cudaGetLastError();
                pdl_suspend(true);
                e = build();
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
        // the FP64 true residual of the x just returned (one SpMV pass)
        MPS_CUDA(op.true_resid(d_x, H.v(vB), &H.ws.sc->true_rr, H.ws.counters + 11, H.ws.partials, s));
    }
    MPS_CUDA(cudaMemcpyAsync(H.ws.h_sc, H.ws.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
    if (defer) return MPS_OK;
    MPS_CUDA(cudaStreamSynchronize(s));
    return solve_report(kind, H, info, replaced, !ir);
}

}  // namespace mps

// torch_ext.cpp -- the PyTorch extension that mirrors the reference's modules
// on top of the C ABI (include/mpsparse.h).
//
//   spmv.csr_tensor   iterative/BiCGSTAB/spmv.cpp:892-905 (+ iter_solve of
//                     iterative/cgd/spmv.cpp:751-763 and richardson of
//                     iterative/richardson/spmv.cpp:499-512)
//   bcsr.bcsr_tensor  iterative/BiCGSTAB/bcsr.cpp:953-966
//   coo_csr.coo_csr   spmv_kernel/coo_csr/coo_csr/coo_csr/coo_to_csr.cpp:286-288
//
// Same names, argument order and in-place outputs as the reference.  Unlike
// the reference, arguments are checked (dtype, size, device) and failures
// raise RuntimeError instead of printing and continuing.  CPU tensors are
// accepted (copied to the current CUDA device and back); CUDA tensors are used
// in place.  The solvers release the GIL.
#include <torch/extension.h>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>

#include "mpsparse.h"

namespace {

void check(mps_status s, const char* what) {
    if (s != MPS_OK)
        throw std::runtime_error(std::string(what) + " failed (" + mps_status_string(s) +
                                 "): " + mps_last_error_string());
}

cudaStream_t cur_stream() { return at::cuda::getCurrentCUDAStream().stream(); }

torch::Tensor on_device(const torch::Tensor& t, at::ScalarType dt, const char* name) {
    TORCH_CHECK(t.scalar_type() == dt, name, " must be ", c10::toString(dt), ", got ",
                c10::toString(t.scalar_type()));
    torch::Tensor d = t.is_cuda() ? t : t.to(torch::kCUDA, /*non_blocking=*/false);
    return d.contiguous();
}

// Write a device result into a caller tensor (CPU or CUDA), first n entries.
void write_back(torch::Tensor& dst, const torch::Tensor& src, int64_t n) {
    auto s = src.narrow(0, 0, n);
    dst.narrow(0, 0, n).copy_(s);
}

// The persistent form a solve ran in (None: the graph form).
py::object persistent_form(int32_t p) {
    static const char* names[] = {"gather", "window", "stream"};
    if (p < 1 || p > 3) return py::none();
    return py::str(names[p - 1]);
}

py::dict info_dict(const mps_solve_info& i) {
    py::dict d;
    d["iters"] = i.iters;
    d["converged"] = (bool)i.converged;
    d["breakdown"] = (bool)i.breakdown;
    d["stalled"] = (bool)i.stalled;
    d["compat_snapshot"] = (bool)i.compat_snapshot;
    d["rel_resid"] = i.rel_resid;
    d["stop_rule_met"] = (bool)i.stop_rule_met;
    d["true_resid"] = i.true_resid;
    d["persistent"] = (bool)i.persistent;
    d["persistent_form"] = persistent_form(i.persistent);
    return d;
}

int precond_code(const std::string& p) {
    if (p == "none" || p.empty()) return MPS_PRECOND_NONE;
    if (p == "jacobi") return MPS_PRECOND_JACOBI;
    if (p == "fsai") return MPS_PRECOND_FSAI;
    throw std::invalid_argument("precond must be 'none', 'jacobi' or 'fsai'");
}

class FsaiModel {
public:
    explicit FsaiModel(c10::optional<torch::Tensor> params) {
        std::vector<float> host;
        const float* p = nullptr;
        if (params && params->defined()) {
            auto t = params->to(torch::kCPU).to(torch::kFloat32).contiguous();
            TORCH_CHECK(t.numel() == mps_fsai_param_count(), "params must hold ", mps_fsai_param_count(),
                        " floats");
            host.assign(t.data_ptr<float>(), t.data_ptr<float>() + t.numel());
            p = host.data();
        }
        check(mps_fsai_model_create(p, &m_), "fsai_model");
    }
    ~FsaiModel() { mps_fsai_model_destroy(m_); }
    torch::Tensor params() const {
        auto t = torch::empty({mps_fsai_param_count()}, torch::kFloat32);
        check(mps_fsai_model_get(m_, t.data_ptr<float>()), "params");
        return t;
    }
    void set_params(torch::Tensor p) {
        auto t = p.to(torch::kCPU).to(torch::kFloat32).contiguous();
        TORCH_CHECK(t.numel() == mps_fsai_param_count(), "wrong parameter count");
        check(mps_fsai_model_set(m_, t.data_ptr<float>()), "set_params");
    }
    torch::Tensor forward(torch::Tensor X) const {
        auto x = on_device(X, torch::kFloat32, "X");
        TORCH_CHECK(x.dim() == 2 && x.size(1) == 16, "X must be N x 16");
        auto out = torch::empty({x.size(0)}, x.options());
        check(mps_fsai_mlp_forward(m_, x.data_ptr<float>(), (uint64_t)x.size(0), out.data_ptr<float>(),
                                   cur_stream()),
              "mlp_forward");
        return out;
    }
    torch::Tensor backward(torch::Tensor X, torch::Tensor dout) const {
        auto x = on_device(X, torch::kFloat32, "X");
        auto d = on_device(dout, torch::kFloat32, "dout");
        TORCH_CHECK(x.dim() == 2 && x.size(1) == 16 && d.numel() == x.size(0), "shapes");
        auto g = torch::empty({mps_fsai_param_count()}, x.options());
        check(mps_fsai_mlp_backward(m_, x.data_ptr<float>(), d.data_ptr<float>(), (uint64_t)x.size(0),
                                    g.data_ptr<float>(), cur_stream()),
              "mlp_backward");
        return g;
    }
    // Raw passes on BF16 features, stream-ordered without a synchronisation
    // (timing, chaining); status() synchronises and reports a timed-out wait.
    void forward_bf16(torch::Tensor Xb, torch::Tensor out) const {
        TORCH_CHECK(Xb.is_cuda() && Xb.scalar_type() == torch::kBFloat16 && Xb.is_contiguous() &&
                        Xb.dim() == 2 && Xb.size(1) == 16, "Xb must be a contiguous CUDA bf16 N x 16 tensor");
        TORCH_CHECK(out.is_cuda() && out.scalar_type() == torch::kFloat32 && out.is_contiguous() &&
                        out.numel() == Xb.size(0), "out must be a contiguous CUDA float32 N tensor");
        c10::cuda::CUDAGuard g(Xb.get_device());
        check(mps_fsai_mlp_forward_bf16(m_, Xb.data_ptr(), (uint64_t)Xb.size(0), out.data_ptr<float>(),
                                        cur_stream()),
              "mlp_forward_bf16");
    }
    void backward_bf16(torch::Tensor Xb, torch::Tensor dout, torch::Tensor grad) const {
        TORCH_CHECK(Xb.is_cuda() && Xb.scalar_type() == torch::kBFloat16 && Xb.is_contiguous() &&
                        Xb.dim() == 2 && Xb.size(1) == 16, "Xb must be a contiguous CUDA bf16 N x 16 tensor");
        TORCH_CHECK(dout.is_cuda() && dout.scalar_type() == torch::kFloat32 && dout.is_contiguous() &&
                        dout.numel() == Xb.size(0), "dout must be a contiguous CUDA float32 N tensor");
        TORCH_CHECK(grad.is_cuda() && grad.scalar_type() == torch::kFloat32 && grad.is_contiguous() &&
                        grad.numel() == mps_fsai_param_count(), "grad must hold the parameter count");
        c10::cuda::CUDAGuard g(Xb.get_device());
        check(mps_fsai_mlp_backward_bf16(m_, Xb.data_ptr(), dout.data_ptr<float>(), (uint64_t)Xb.size(0),
                                         grad.data_ptr<float>(), cur_stream()),
              "mlp_backward_bf16");
    }
    void status() const { check(mps_fsai_model_status(m_, cur_stream()), "fsai model"); }
    mps_fsai_model* handle() const { return m_; }

private:
    mps_fsai_model* m_ = nullptr;
};

class CsrTensor {
public:
    CsrTensor(torch::Tensor keys, torch::Tensor values, torch::Tensor row_ptr,
              torch::Tensor col_ind, torch::Tensor out_vals, int64_t num_rows, int64_t num_cols,
              bool fill_outputs)
        : n_rows_(num_rows), n_cols_(num_cols) {
        TORCH_CHECK(num_rows > 0 && num_cols > 0, "num_rows and num_cols must be positive");
        TORCH_CHECK(keys.dim() == 1 && values.dim() == 1, "keys and values must be 1-D");
        TORCH_CHECK(keys.numel() == values.numel(), "keys and values differ in length");
        auto k = on_device(keys, torch::kInt64, "keys");
        auto v = on_device(values, torch::kFloat32, "values");
        device_ = k.get_device();
        c10::cuda::CUDAGuard g(device_);
        nnz_ = k.numel();
        check(mps_csr_create_from_keys(reinterpret_cast<const uint64_t*>(k.data_ptr<int64_t>()),
                                       v.data_ptr<float>(), (uint64_t)nnz_, (uint32_t)num_rows,
                                       (uint32_t)num_cols, &h_, cur_stream()),
              "csr_tensor");
        // The reference leaves these three tensors untouched (spmv.cpp:62-228);
        // filling them is a superset of its behaviour.
        if (fill_outputs && row_ptr.defined() && row_ptr.numel() == num_rows + 1 &&
            col_ind.numel() == nnz_ && out_vals.numel() == nnz_) {
            auto t = export_csr();
            row_ptr.copy_(std::get<0>(t));
            col_ind.copy_(std::get<1>(t));
            out_vals.copy_(std::get<2>(t));
        }
    }
    ~CsrTensor() {
        if (h_) {
            c10::cuda::CUDAGuard g(device_);
            mps_csr_destroy(h_);
        }
    }

    py::dict autotune() {
        c10::cuda::CUDAGuard g(device_);
        int32_t t = 0, st = 0, hint = 0;
        float us = 0.f;
        check(mps_csr_autotune_spmv(h_, &t, &st, &hint, &us, cur_stream()), "autotune");
        py::dict d;
        d["tile_nnz"] = t;
        d["stages"] = st;
        d["evict_first"] = hint;
        d["spmv_us"] = us;
        return d;
    }

    void set_plan(int64_t tile_nnz, int64_t stages, int64_t evict_first) {
        c10::cuda::CUDAGuard g(device_);
        check(mps_csr_set_spmv_plan(h_, (int32_t)tile_nnz, (int32_t)stages, (int32_t)evict_first,
                                    cur_stream()),
              "set_plan");
    }

    // The matrix as a torch sparse CSR tensor (int32 indices, FP32 values)
    // on the handle's device: torch's own sparse ops (matmul, to_dense,
    // autograd through torch) work on it directly.
    torch::Tensor sparse_csr() {
        auto t = export_csr();
        c10::cuda::CUDAGuard g(device_);
        return torch::sparse_csr_tensor(std::get<0>(t), std::get<1>(t), std::get<2>(t),
                                        {n_rows_, n_cols_},
                                        torch::TensorOptions().dtype(torch::kFloat32)
                                            .device(torch::kCUDA, device_));
    }
    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> export_csr() {
        c10::cuda::CUDAGuard g(device_);
        auto opt = torch::TensorOptions().device(torch::kCUDA, device_);
        auto rp = torch::empty({n_rows_ + 1}, opt.dtype(torch::kInt32));
        auto ci = torch::empty({nnz_}, opt.dtype(torch::kInt32));
        auto va = torch::empty({nnz_}, opt.dtype(torch::kFloat32));
        check(mps_csr_export(h_, rp.data_ptr<int32_t>(), ci.data_ptr<int32_t>(), va.data_ptr<float>(),
                             cur_stream()),
              "export");
        return {rp, ci, va};
    }

    // b = A x (reference: mv(x, b), spmv.cpp:491-501)
    void mv(torch::Tensor x, torch::Tensor b) {
        c10::cuda::CUDAGuard g(device_);
        TORCH_CHECK(x.numel() >= n_cols_, "x has ", x.numel(), " entries, need ", n_cols_);
        TORCH_CHECK(b.numel() >= n_rows_, "b has ", b.numel(), " entries, need ", n_rows_);
        auto xd = on_device(x, torch::kFloat32, "x");
        torch::Tensor bd = (b.is_cuda() && b.is_contiguous() && b.scalar_type() == torch::kFloat32)
                               ? b
                               : torch::empty({n_rows_}, xd.options());
        check(mps_csr_spmv(h_, xd.data_ptr<float>(), bd.data_ptr<float>(), cur_stream()), "mv");
        if (!bd.is_same(b)) write_back(b, bd, n_rows_);
    }

    // *dot = w . (A x), y = A x
    double mv_dot(torch::Tensor x, torch::Tensor w, torch::Tensor y) {
        c10::cuda::CUDAGuard g(device_);
        auto xd = on_device(x, torch::kFloat32, "x");
        auto wd = on_device(w, torch::kFloat32, "w");
        TORCH_CHECK(y.is_cuda() && y.is_contiguous() && y.scalar_type() == torch::kFloat32 &&
                        y.numel() >= n_rows_,
                    "y must be a contiguous CUDA float32 tensor of length num_rows");
        auto dot = torch::empty({1}, xd.options().dtype(torch::kFloat64));
        check(mps_csr_spmv_dot(h_, xd.data_ptr<float>(), wd.data_ptr<float>(), y.data_ptr<float>(),
                               dot.data_ptr<double>(), cur_stream()),
              "mv_dot");
        return dot.item<double>();
    }

    py::dict solve(int kind, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                   double omega, const std::string& precond, bool compat, bool host_loop,
                   int64_t stall_window) {
        c10::cuda::CUDAGuard g(device_);
        TORCH_CHECK(n_rows_ == n_cols_, "solvers need a square matrix");
        TORCH_CHECK(b.numel() >= n_rows_, "b has ", b.numel(), " entries, need ", n_rows_);
        TORCH_CHECK(x.numel() >= n_cols_, "x has ", x.numel(), " entries, need ", n_cols_);
        TORCH_CHECK(x.scalar_type() == torch::kFloat32, "x must be float32");
        auto bd = on_device(b, torch::kFloat32, "b");
        const bool direct = x.is_cuda() && x.is_contiguous();
        torch::Tensor xd = direct ? x : torch::empty({n_cols_}, bd.options());
        mps_solve_opts o;
        mps_solve_opts_default(&o);
        o.tol = tol;
        o.max_iter = (int32_t)max_iter;
        o.omega = omega;
        o.precond = precond_code(precond);
        o.reference_compat = compat ? 1 : 0;
        o.host_loop = host_loop ? 1 : 0;
        o.stall_window = (int32_t)stall_window;
        mps_solve_info info{};
        mps_status s;
        {
            py::gil_scoped_release nogil;
            cudaStream_t st = cur_stream();
            if (kind == 0)
                s = mps_csr_cg(h_, bd.data_ptr<float>(), xd.data_ptr<float>(), &o, &info, st);
            else if (kind == 1)
                s = mps_csr_bicgstab(h_, bd.data_ptr<float>(), xd.data_ptr<float>(), &o, &info, st);
            else
                s = mps_csr_richardson(h_, bd.data_ptr<float>(), xd.data_ptr<float>(), &o, &info, st);
        }
        check(s, kind == 0 ? "cgd" : kind == 1 ? "bicgstab" : "richardson");
        if (!direct) write_back(x, xd, n_cols_);
        return info_dict(info);
    }

    py::dict cg_mixed(torch::Tensor b, torch::Tensor x, double tol, double inner_tol,
                      int64_t max_outer, int64_t max_inner, int64_t value_bits,
                      const std::string& precond, bool host_loop, const std::string& ir_mode) {
        c10::cuda::CUDAGuard g(device_);
        TORCH_CHECK(b.numel() >= n_rows_ && x.numel() >= n_cols_, "b / x too short");
        auto bd = on_device(b, torch::kFloat64, "b");
        TORCH_CHECK(x.scalar_type() == torch::kFloat64, "x must be float64");
        const bool direct = x.is_cuda() && x.is_contiguous();
        torch::Tensor xd = direct ? x : torch::empty({n_cols_}, bd.options());
        mps_ir_opts o{};
        o.tol = tol;
        o.inner_tol = inner_tol;
        o.max_outer = (int32_t)max_outer;
        o.max_inner = (int32_t)max_inner;
        o.value_bits = (int32_t)value_bits;
        o.precond = precond_code(precond);
        o.host_loop = host_loop ? 1 : 0;
        if (ir_mode == "auto" || ir_mode.empty()) o.ir_mode = MPS_IR_AUTO;
        else if (ir_mode == "restart") o.ir_mode = MPS_IR_RESTART;
        else if (ir_mode == "replace") o.ir_mode = MPS_IR_REPLACE;
        else throw std::invalid_argument("ir_mode must be 'auto', 'restart' or 'replace'");
        mps_ir_info info{};
        mps_status s;
        {
            py::gil_scoped_release nogil;
            s = mps_csr_cg_mixed(h_, bd.data_ptr<double>(), xd.data_ptr<double>(), &o, &info,
                                 cur_stream());
        }
        check(s, "cg_mixed");
        if (!direct) write_back(x, xd, n_cols_);
        py::dict d;
        d["outer_iters"] = info.outer_iters;
        d["inner_iters"] = info.inner_iters;
        d["converged"] = (bool)info.converged;
        d["rel_resid"] = info.rel_resid;
        d["persistent"] = (bool)info.persistent;
        d["persistent_form"] = persistent_form(info.persistent);
        return d;
    }
    void set_persistent(bool enable, const std::string& form) {
        int f = -1;
        if (form == "auto") f = 0;
        else if (form == "gather") f = 1;
        else if (form == "window") f = 2;
        else if (form == "stream") f = 3;
        if (f < 0) throw std::invalid_argument("form must be auto, gather, window or stream");
        check(mps_csr_set_persistent(h_, enable ? 1 : 0), "set_persistent");
        check(mps_csr_set_persistent_form(h_, f), "set_persistent");
    }

    void set_fsai(torch::Tensor rp, torch::Tensor ci, torch::Tensor v) {
        c10::cuda::CUDAGuard g(device_);
        TORCH_CHECK(rp.numel() == n_rows_ + 1, "G row_ptr must have num_rows + 1 entries");
        auto r = on_device(rp, torch::kInt32, "row_ptr");
        auto c = on_device(ci, torch::kInt32, "col_ind");
        auto w = on_device(v, torch::kFloat32, "values");
        TORCH_CHECK(c.numel() == w.numel(), "col_ind / values differ in length");
        check(mps_csr_set_fsai(h_, r.data_ptr<int32_t>(), c.data_ptr<int32_t>(), w.data_ptr<float>(),
                               (uint64_t)c.numel(), cur_stream()),
              "set_fsai");
    }

    void attach_fsai(const FsaiModel& m) {
        c10::cuda::CUDAGuard g(device_);
        check(mps_fsai_attach(h_, m.handle(), cur_stream()), "attach_fsai");
    }

    // "auto" / "split" (w = G r, z = G^T w) / "product" (z = (G^T G) r)
    void set_fsai_apply(const std::string& mode) {
        c10::cuda::CUDAGuard g(device_);
        int32_t m;
        if (mode == "auto") m = MPS_FSAI_APPLY_AUTO;
        else if (mode == "split") m = MPS_FSAI_APPLY_SPLIT;
        else if (mode == "product") m = MPS_FSAI_APPLY_PRODUCT;
        else throw std::invalid_argument("mode must be 'auto', 'split' or 'product'");
        check(mps_csr_set_fsai_apply(h_, m, cur_stream()), "set_fsai_apply");
    }

    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> fsai_product() const {
        c10::cuda::CUDAGuard g(device_);
        int32_t f = -1;
        uint64_t nnz_m = 0;
        check(mps_csr_fsai_apply(h_, &f, &nnz_m), "fsai_product");
        auto o = torch::TensorOptions().device(torch::kCUDA, device_);
        auto rp = torch::empty({n_rows_ + 1}, o.dtype(torch::kInt32));
        auto ci = torch::empty({(int64_t)nnz_m}, o.dtype(torch::kInt32));
        auto v = torch::empty({(int64_t)nnz_m}, o.dtype(torch::kFloat32));
        check(mps_csr_fsai_product_get(h_, rp.data_ptr<int32_t>(), ci.data_ptr<int32_t>(),
                                       v.data_ptr<float>(), cur_stream()),
              "fsai_product");
        return {rp, ci, v};
    }

    py::dict fsai_apply() const {
        int32_t f = -1;
        uint64_t nnz_m = 0;
        check(mps_csr_fsai_apply(h_, &f, &nnz_m), "fsai_apply");
        py::dict d;
        d["form"] = f < 0 ? py::object(py::none())
                          : py::object(py::str(f == MPS_FSAI_APPLY_PRODUCT ? "product" : "split"));
        d["nnz_m"] = nnz_m;
        return d;
    }

    double fsai_train_step(FsaiModel& m, int64_t n_probes, c10::optional<torch::Tensor> extra,
                           double lr, int64_t seed) {
        c10::cuda::CUDAGuard g(device_);
        torch::Tensor e;
        int64_t ne = 0;
        if (extra && extra->defined() && extra->numel() > 0) {
            e = on_device(*extra, torch::kFloat32, "extra");
            TORCH_CHECK(e.numel() % n_rows_ == 0, "extra must be k x num_rows");
            ne = e.numel() / n_rows_;
        }
        double loss = 0;
        check(mps_fsai_train_step(m.handle(), h_, (int32_t)n_probes, ne ? e.data_ptr<float>() : nullptr,
                                  (int32_t)ne, (float)lr, (uint64_t)seed, &loss, cur_stream()),
              "fsai_train_step");
        return loss;
    }

    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> fsai_features() {
        c10::cuda::CUDAGuard g(device_);
        uint64_t nz = 0;
        check(mps_fsai_features(h_, nullptr, nullptr, nullptr, &nz, cur_stream()), "fsai_features");
        auto opt = torch::TensorOptions().device(torch::kCUDA, device_);
        auto X = torch::empty({(int64_t)nz, 16}, opt.dtype(torch::kFloat32));
        auto rp = torch::empty({n_rows_ + 1}, opt.dtype(torch::kInt32));
        auto ci = torch::empty({(int64_t)nz}, opt.dtype(torch::kInt32));
        check(mps_fsai_features(h_, X.data_ptr<float>(), rp.data_ptr<int32_t>(), ci.data_ptr<int32_t>(),
                                &nz, cur_stream()),
              "fsai_features");
        return {X, rp, ci};
    }

    torch::Tensor fsai_g_values() {
        c10::cuda::CUDAGuard g(device_);
        uint64_t nz = 0;
        check(mps_fsai_features(h_, nullptr, nullptr, nullptr, &nz, cur_stream()), "fsai_g_values");
        auto v = torch::empty({(int64_t)nz}, torch::TensorOptions().device(torch::kCUDA, device_));
        check(mps_fsai_g_values(h_, v.data_ptr<float>(), cur_stream()), "fsai_g_values");
        return v;
    }

    std::tuple<torch::Tensor, double> fsai_probe_grad(torch::Tensor V) {
        c10::cuda::CUDAGuard g(device_);
        auto v = on_device(V, torch::kFloat32, "V");
        TORCH_CHECK(v.numel() % n_rows_ == 0, "V must be k x num_rows");
        uint64_t nz = 0;
        check(mps_fsai_features(h_, nullptr, nullptr, nullptr, &nz, cur_stream()), "fsai_probe_grad");
        auto grad = torch::empty({(int64_t)nz}, v.options());
        double loss = 0;
        check(mps_fsai_probe_grad(h_, v.data_ptr<float>(), (int32_t)(v.numel() / n_rows_),
                                  grad.data_ptr<float>(), &loss, cur_stream()),
              "fsai_probe_grad");
        return {grad, loss};
    }

    int64_t nnz() const { return nnz_; }
    int64_t num_rows() const { return n_rows_; }
    int64_t num_cols() const { return n_cols_; }

private:
    mps_csr* h_ = nullptr;
    int64_t n_rows_, n_cols_, nnz_ = 0;
    int device_ = 0;
};

class BcsrTensor {
public:
    BcsrTensor(torch::Tensor keys, torch::Tensor values, torch::Tensor row_ptr,
               torch::Tensor col_ind, int64_t num_rows, int64_t num_cols, int64_t block_size)
        : n_rows_(num_rows), n_cols_(num_cols), block_(block_size) {
        TORCH_CHECK(block_size == 4 || block_size == 8, "block_size must be 4 or 8");
        TORCH_CHECK(num_rows > 0 && num_cols > 0, "num_rows and num_cols must be positive");
        nbr_ = (num_rows + block_size - 1) / block_size;
        padded_ = nbr_ * block_size;
        if (row_ptr.defined() && row_ptr.numel() > 0) {
            // pre-built BCSR arrays (bcsr.cpp:357-422)
            TORCH_CHECK(row_ptr.numel() == nbr_ + 1, "row_ptr must have ceil(num_rows/B)+1 entries");
            auto v = on_device(values, torch::kFloat32, "values");
            auto r = on_device(row_ptr, torch::kInt32, "row_ptr");
            auto c = on_device(col_ind, torch::kInt32, "col_ind");
            TORCH_CHECK(v.numel() == c.numel() * block_size * block_size,
                        "values must hold col_ind.numel() * B * B entries");
            device_ = v.get_device();
            c10::cuda::CUDAGuard g(device_);
            check(mps_bcsr_create(v.data_ptr<float>(), r.data_ptr<int32_t>(), c.data_ptr<int32_t>(),
                                  (uint64_t)c.numel(), (uint32_t)num_rows, (uint32_t)num_cols,
                                  (uint32_t)block_size, &h_, cur_stream()),
                  "bcsr_tensor");
        } else {
            // packed COO keys: BCSR built on the GPU
            auto k = on_device(keys, torch::kInt64, "keys");
            auto v = on_device(values, torch::kFloat32, "values");
            TORCH_CHECK(k.numel() == v.numel(), "keys and values differ in length");
            device_ = k.get_device();
            c10::cuda::CUDAGuard g(device_);
            check(mps_bcsr_create_from_keys(reinterpret_cast<const uint64_t*>(k.data_ptr<int64_t>()),
                                            v.data_ptr<float>(), (uint64_t)k.numel(),
                                            (uint32_t)num_rows, (uint32_t)num_cols,
                                            (uint32_t)block_size, &h_, cur_stream()),
                  "bcsr_tensor");
        }
    }
    ~BcsrTensor() {
        if (h_) {
            c10::cuda::CUDAGuard g(device_);
            mps_bcsr_destroy(h_);
        }
    }

    torch::Tensor padded(const torch::Tensor& b) {
        auto bd = on_device(b, torch::kFloat32, "b");
        if (bd.numel() == padded_) return bd;
        TORCH_CHECK(bd.numel() >= n_rows_, "vector has ", bd.numel(), " entries, need ", n_rows_);
        auto p = torch::zeros({padded_}, bd.options());
        p.narrow(0, 0, n_rows_).copy_(bd.narrow(0, 0, n_rows_));
        return p;
    }

    void mv(torch::Tensor x, torch::Tensor b) {
        c10::cuda::CUDAGuard g(device_);
        auto xd = padded(x);
        auto bd = torch::empty({padded_}, xd.options());
        check(mps_bcsr_spmv(h_, xd.data_ptr<float>(), bd.data_ptr<float>(), cur_stream()), "mv");
        write_back(b, bd, std::min<int64_t>(b.numel(), padded_));
    }

    // x is written for min(x.numel(), padded) entries: the reference copies
    // logical_rows (cgd, bcsr.cpp:716) or logical_cols (bicgstab, :942).
    py::dict solve(int kind, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                   bool compat, bool host_loop) {
        c10::cuda::CUDAGuard g(device_);
        TORCH_CHECK(x.scalar_type() == torch::kFloat32, "x must be float32");
        auto bd = padded(b);
        auto xd = torch::empty({padded_}, bd.options());
        mps_solve_opts o;
        mps_solve_opts_default(&o);
        o.tol = tol;
        o.max_iter = (int32_t)max_iter;
        o.reference_compat = compat ? 1 : 0;
        o.host_loop = host_loop ? 1 : 0;
        mps_solve_info info{};
        mps_status s;
        {
            py::gil_scoped_release nogil;
            if (kind == 0)
                s = mps_bcsr_cg(h_, bd.data_ptr<float>(), xd.data_ptr<float>(), &o, &info, cur_stream());
            else
                s = mps_bcsr_bicgstab(h_, bd.data_ptr<float>(), xd.data_ptr<float>(), &o, &info,
                                      cur_stream());
        }
        check(s, kind == 0 ? "cgd" : "bicgstab");
        const int64_t n_out = kind == 0 ? std::min<int64_t>(x.numel(), std::max(n_rows_, padded_))
                                        : std::min<int64_t>(x.numel(), padded_);
        write_back(x, xd, std::min<int64_t>(n_out, padded_));
        return info_dict(info);
    }

    // The matrix as a torch sparse BSR tensor (blocks B x B, row-major) of the
    // padded size on the handle's device.
    torch::Tensor sparse_bsr() {
        auto t = export_bcsr();
        c10::cuda::CUDAGuard g(device_);
        auto vals = std::get<2>(t).view({-1, block_, block_});
        return torch::sparse_bsr_tensor(std::get<0>(t), std::get<1>(t), vals, {padded_, padded_},
                                        torch::TensorOptions().dtype(torch::kFloat32)
                                            .device(torch::kCUDA, device_));
    }
    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> export_bcsr() {
        c10::cuda::CUDAGuard g(device_);
        uint32_t nbr, blk, pn;
        uint64_t nb;
        check(mps_bcsr_shape(h_, &nbr, &nb, &blk, &pn), "shape");
        auto opt = torch::TensorOptions().device(torch::kCUDA, device_);
        auto rp = torch::empty({(int64_t)nbr + 1}, opt.dtype(torch::kInt32));
        auto ci = torch::empty({(int64_t)nb}, opt.dtype(torch::kInt32));
        auto va = torch::empty({(int64_t)nb * blk * blk}, opt.dtype(torch::kFloat32));
        check(mps_bcsr_export(h_, rp.data_ptr<int32_t>(), ci.data_ptr<int32_t>(), va.data_ptr<float>(),
                              cur_stream()),
              "export");
        return {rp, ci, va};
    }

    int64_t padded_rows() const { return padded_; }
    int64_t num_rows() const { return n_rows_; }
    int64_t num_cols() const { return n_cols_; }
    int64_t block_size() const { return block_; }

private:
    mps_bcsr* h_ = nullptr;
    int64_t n_rows_, n_cols_, block_, nbr_ = 0, padded_ = 0;
    int device_ = 0;
};

// Batched solver over a block-diagonal stack of systems.
class BatchSolver {
public:
    BatchSolver(torch::Tensor row_ptr, torch::Tensor col_ind, torch::Tensor vals, torch::Tensor row_off) {
        auto rp = on_device(row_ptr, torch::kInt32, "row_ptr");
        auto ci = on_device(col_ind, torch::kInt32, "col_ind");
        auto v = on_device(vals, torch::kFloat32, "vals");
        auto ro = row_off.to(torch::kCPU).to(torch::kInt32).contiguous();
        n_sys_ = ro.numel() - 1;
        TORCH_CHECK(n_sys_ > 0, "row_off needs at least two entries");
        n_ = ro.data_ptr<int32_t>()[n_sys_];
        TORCH_CHECK(rp.numel() == n_ + 1, "row_ptr must have total_rows + 1 entries");
        device_ = rp.get_device();
        c10::cuda::CUDAGuard g(device_);
        check(mps_batch_create(rp.data_ptr<int32_t>(), ci.data_ptr<int32_t>(), v.data_ptr<float>(),
                               (uint64_t)ci.numel(), (uint32_t)n_, ro.data_ptr<int32_t>(), (int32_t)n_sys_,
                               &h_, cur_stream()),
              "batch");
    }
    ~BatchSolver() {
        if (h_) {
            c10::cuda::CUDAGuard g(device_);
            mps_batch_destroy(h_);
        }
    }
    void attach_fsai(const FsaiModel& m) {
        c10::cuda::CUDAGuard g(device_);
        check(mps_batch_attach_fsai(h_, m.handle(), cur_stream()), "attach_fsai");
    }
    void set_precond(torch::Tensor kinds) {
        auto k = kinds.to(torch::kCPU).to(torch::kInt8).contiguous();
        TORCH_CHECK(k.numel() == n_sys_, "one preconditioner kind per system");
        check(mps_batch_set_precond(h_, k.data_ptr<int8_t>()), "set_precond");
    }
    std::tuple<int64_t, std::vector<double>> autotune(torch::Tensor b, double tol, int64_t max_iter) {
        c10::cuda::CUDAGuard g(device_);
        auto bd = on_device(b, torch::kFloat32, "b");
        int32_t w = 0;
        float ms[6];
        check(mps_batch_autotune(h_, bd.data_ptr<float>(), tol, (int32_t)max_iter, &w, ms, cur_stream()),
              "autotune");
        return {w, std::vector<double>(ms, ms + 6)};
    }
    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> cg(torch::Tensor b, torch::Tensor x, double tol,
                                                               int64_t max_iter) {
        c10::cuda::CUDAGuard g(device_);
        auto bd = on_device(b, torch::kFloat32, "b");
        TORCH_CHECK(bd.numel() == n_ && x.numel() == n_, "b and x need total_rows entries");
        TORCH_CHECK(x.is_cuda() && x.is_contiguous() && x.scalar_type() == torch::kFloat32,
                    "x must be a contiguous CUDA float32 tensor");
        auto opt = bd.options();
        auto it = torch::empty({n_sys_}, opt.dtype(torch::kInt32));
        auto cv = torch::empty({n_sys_}, opt.dtype(torch::kInt32));
        auto rr = torch::empty({n_sys_}, opt.dtype(torch::kFloat32));
        check(mps_batch_cg(h_, bd.data_ptr<float>(), x.data_ptr<float>(), tol, (int32_t)max_iter,
                           it.data_ptr<int32_t>(), cv.data_ptr<int32_t>(), rr.data_ptr<float>(), cur_stream()),
              "batch cg");
        return {it, cv, rr};
    }
    std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> cg_mixed(torch::Tensor b, torch::Tensor x,
                                                                     double tol, double inner_tol,
                                                                     int64_t max_iter) {
        c10::cuda::CUDAGuard g(device_);
        auto bd = on_device(b, torch::kFloat32, "b");
        TORCH_CHECK(bd.numel() == n_ && x.numel() == n_, "b and x need total_rows entries");
        TORCH_CHECK(x.is_cuda() && x.is_contiguous() && x.scalar_type() == torch::kFloat64,
                    "x must be a contiguous CUDA float64 tensor");
        auto opt = bd.options();
        auto it = torch::empty({n_sys_}, opt.dtype(torch::kInt32));
        auto cv = torch::empty({n_sys_}, opt.dtype(torch::kInt32));
        auto rr = torch::empty({n_sys_}, opt.dtype(torch::kFloat32));
        check(mps_batch_cg_mixed(h_, bd.data_ptr<float>(), x.data_ptr<double>(), tol, inner_tol,
                                 (int32_t)max_iter, it.data_ptr<int32_t>(), cv.data_ptr<int32_t>(),
                                 rr.data_ptr<float>(), cur_stream()),
              "batch cg_mixed");
        return {it, cv, rr};
    }
    int64_t warps_per_system() const { return mps_batch_warps_per_system(h_); }
    int64_t uses_clusters() const { return mps_batch_uses_clusters(h_); }
    void set_clusters(int64_t n) { check(mps_batch_set_clusters(h_, (int32_t)n), "set_clusters"); }
    int64_t num_systems() const { return n_sys_; }

private:
    mps_batch* h_ = nullptr;
    int64_t n_sys_ = 0, n_ = 0;
    int device_ = 0;
};

// coo_csr.coo_csr: sort on the GPU and write the caller's three tensors.
void coo_csr_fn(torch::Tensor keys, torch::Tensor values, torch::Tensor row_ptr,
                torch::Tensor col_ind, torch::Tensor out_vals, int64_t num_rows, int64_t num_cols) {
    TORCH_CHECK(keys.numel() == values.numel(), "keys and values differ in length");
    TORCH_CHECK(row_ptr.numel() == num_rows + 1, "row_ptr must have num_rows + 1 entries");
    TORCH_CHECK(col_ind.numel() == keys.numel() && out_vals.numel() == keys.numel(),
                "col_ind / out_vals must have nnz entries");
    TORCH_CHECK(row_ptr.scalar_type() == torch::kInt32 && col_ind.scalar_type() == torch::kInt32 &&
                    out_vals.scalar_type() == torch::kFloat32,
                "row_ptr/col_ind must be int32 and out_vals float32");
    auto k = on_device(keys, torch::kInt64, "keys");
    auto v = on_device(values, torch::kFloat32, "values");
    c10::cuda::CUDAGuard g(k.get_device());
    auto opt = k.options();
    const int64_t nnz = k.numel();
    // Device outputs are written in place; host outputs through temporaries.
    auto direct = [&](const torch::Tensor& t) {
        return t.is_cuda() && t.is_contiguous() && t.get_device() == k.get_device();
    };
    const bool in_place = nnz > 0 && direct(row_ptr) && direct(col_ind) && direct(out_vals);
    auto rp = in_place ? row_ptr : torch::empty({num_rows + 1}, opt.dtype(torch::kInt32));
    auto ci = in_place ? col_ind : torch::empty({std::max<int64_t>(nnz, 1)}, opt.dtype(torch::kInt32));
    auto ov = in_place ? out_vals : torch::empty({std::max<int64_t>(nnz, 1)}, opt.dtype(torch::kFloat32));
    check(mps_coo_to_csr(reinterpret_cast<const uint64_t*>(k.data_ptr<int64_t>()), v.data_ptr<float>(),
                         (uint64_t)nnz, (uint32_t)num_rows, (uint32_t)num_cols, rp.data_ptr<int32_t>(),
                         ci.data_ptr<int32_t>(), ov.data_ptr<float>(), cur_stream()),
          "coo_csr");
    if (in_place) return;
    row_ptr.copy_(rp);
    if (nnz) {
        col_ind.copy_(ci.narrow(0, 0, nnz));
        out_vals.copy_(ov.narrow(0, 0, nnz));
    }
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
    m.doc() = "B200-native sparse iterative-solver path (drop-in for mpsparse's extensions)";
    py::class_<CsrTensor>(m, "csr_tensor")
        .def(py::init<torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor,
                      int64_t, int64_t, bool>(),
             "CSR Tensor Constructor", py::arg("keys"), py::arg("values"), py::arg("row_ptr"),
             py::arg("col_ind"), py::arg("out_vals"), py::arg("num_rows"), py::arg("num_cols"),
             py::arg("fill_outputs") = true)
        .def("mv", &CsrTensor::mv, "b = A x", py::arg("x"), py::arg("b"))
        .def("mv_dot", &CsrTensor::mv_dot, "y = A x; returns w . y", py::arg("x"), py::arg("w"),
             py::arg("y"))
        .def("cgd",
             [](CsrTensor& t, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                const std::string& precond, bool compat, bool host_loop, int64_t stall_window) {
                 return t.solve(0, b, x, tol, max_iter, 0.01, precond, compat, host_loop, stall_window);
             },
             py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6, py::arg("max_iter") = 2000,
             py::arg("precond") = "none", py::arg("reference_compat") = false,
             py::arg("host_loop") = false, py::arg("stall_window") = 400)
        .def("iter_solve",
             [](CsrTensor& t, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                const std::string& precond, bool compat) {
                 return t.solve(0, b, x, tol, max_iter, 0.01, precond, compat, false, 400);
             },
             py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6, py::arg("max_iter") = 2000,
             py::arg("precond") = "none", py::arg("reference_compat") = false)
        .def("bicgstab",
             [](CsrTensor& t, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                bool compat, bool host_loop) {
                 return t.solve(1, b, x, tol, max_iter, 0.01, "none", compat, host_loop, 400);
             },
             py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6, py::arg("max_iter") = 2000,
             py::arg("reference_compat") = false, py::arg("host_loop") = false)
        .def("richardson",
             [](CsrTensor& t, torch::Tensor b, torch::Tensor x, double omega, int64_t iters,
                double tol, bool compat, bool host_loop) {
                 return t.solve(2, b, x, tol, iters, omega, "none", compat, host_loop, 400);
             },
             py::arg("b"), py::arg("x"), py::arg("omega") = 0.01, py::arg("iters") = 1000,
             py::arg("tol") = 0.0, py::arg("reference_compat") = false,
             py::arg("host_loop") = false)
        .def("cg_mixed", &CsrTensor::cg_mixed, py::arg("b"), py::arg("x"), py::arg("tol") = 1e-10,
             py::arg("inner_tol") = 0.0, py::arg("max_outer") = 50, py::arg("max_inner") = 2000,
             py::arg("value_bits") = 32, py::arg("precond") = "none", py::arg("host_loop") = false,
             py::arg("ir_mode") = "auto")
        .def("set_fsai", &CsrTensor::set_fsai, py::arg("row_ptr"), py::arg("col_ind"),
             py::arg("values"))
        .def("attach_fsai", &CsrTensor::attach_fsai, py::arg("model"))
        .def("set_fsai_apply", &CsrTensor::set_fsai_apply, py::arg("mode"))
        .def("fsai_apply", &CsrTensor::fsai_apply)
        .def("set_persistent", &CsrTensor::set_persistent, py::arg("enable"), py::arg("form") = "auto",
             "cgd / bicgstab / cg_mixed as one persistent kernel when a CTA per SM can hold its share "
             "(default on); form: auto (window, else gather, else stream), or only gather / window / stream")
        .def("fsai_product", &CsrTensor::fsai_product)
        .def("fsai_train_step", &CsrTensor::fsai_train_step, py::arg("model"), py::arg("n_probes") = 4,
             py::arg("extra") = py::none(), py::arg("lr") = 1e-3, py::arg("seed") = 0)
        .def("fsai_features", &CsrTensor::fsai_features)
        .def("fsai_g_values", &CsrTensor::fsai_g_values)
        .def("fsai_probe_grad", &CsrTensor::fsai_probe_grad, py::arg("V"))
        .def("csr", &CsrTensor::export_csr)
        .def("sparse_csr", &CsrTensor::sparse_csr, "the matrix as a torch.sparse_csr_tensor")
        .def("set_plan", &CsrTensor::set_plan, py::arg("tile_nnz") = 0, py::arg("stages") = 0,
             py::arg("evict_first") = -1)
        .def("autotune", &CsrTensor::autotune,
             "time the SpMV tile-plan candidates on this matrix and keep the fastest")
        .def_property_readonly("nnz", &CsrTensor::nnz)
        .def_property_readonly("num_rows", &CsrTensor::num_rows)
        .def_property_readonly("num_cols", &CsrTensor::num_cols);

    py::class_<FsaiModel>(m, "fsai_model")
        .def(py::init<c10::optional<torch::Tensor>>(), py::arg("params") = py::none())
        .def("params", &FsaiModel::params)
        .def("set_params", &FsaiModel::set_params, py::arg("params"))
        .def("forward", &FsaiModel::forward, py::arg("X"))
        .def("backward", &FsaiModel::backward, py::arg("X"), py::arg("dout"))
        .def("forward_bf16", &FsaiModel::forward_bf16, py::arg("Xb"), py::arg("out"))
        .def("backward_bf16", &FsaiModel::backward_bf16, py::arg("Xb"), py::arg("dout"), py::arg("grad"))
        .def("status", &FsaiModel::status);

    py::class_<BatchSolver>(m, "batch_solver")
        .def(py::init<torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor>(), py::arg("row_ptr"),
             py::arg("col_ind"), py::arg("values"), py::arg("row_off"))
        .def("attach_fsai", &BatchSolver::attach_fsai, py::arg("model"))
        .def("set_precond", &BatchSolver::set_precond, py::arg("kinds"))
        .def("autotune", &BatchSolver::autotune, py::arg("b"), py::arg("tol") = 1e-6,
             py::arg("max_iter") = 20000)
        .def("cg", &BatchSolver::cg, py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6,
             py::arg("max_iter") = 20000)
        .def("cg_mixed", &BatchSolver::cg_mixed, py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6,
             py::arg("inner_tol") = 1e-3, py::arg("max_iter") = 20000)
        .def_property_readonly("warps_per_system", &BatchSolver::warps_per_system)
        .def_property_readonly("uses_clusters", &BatchSolver::uses_clusters)
        .def("set_clusters", &BatchSolver::set_clusters, py::arg("n_systems"))
        .def_property_readonly("num_systems", &BatchSolver::num_systems);

    py::class_<BcsrTensor>(m, "bcsr_tensor")
        .def(py::init<torch::Tensor, torch::Tensor, torch::Tensor, torch::Tensor, int64_t, int64_t,
                      int64_t>(),
             "BCSR Tensor Constructor", py::arg("keys"), py::arg("values"), py::arg("row_ptr"),
             py::arg("col_ind"), py::arg("num_rows"), py::arg("num_cols"),
             py::arg("block_size") = 4)
        .def("mv", &BcsrTensor::mv, py::arg("x"), py::arg("b"))
        .def("cgd",
             [](BcsrTensor& t, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                bool compat, bool host_loop) { return t.solve(0, b, x, tol, max_iter, compat, host_loop); },
             py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6, py::arg("max_iter") = 2000,
             py::arg("reference_compat") = false, py::arg("host_loop") = false)
        .def("bicgstab",
             [](BcsrTensor& t, torch::Tensor b, torch::Tensor x, double tol, int64_t max_iter,
                bool compat, bool host_loop) { return t.solve(1, b, x, tol, max_iter, compat, host_loop); },
             py::arg("b"), py::arg("x"), py::arg("tol") = 1e-6, py::arg("max_iter") = 2000,
             py::arg("reference_compat") = false, py::arg("host_loop") = false)
        .def("bcsr", &BcsrTensor::export_bcsr)
        .def("sparse_bsr", &BcsrTensor::sparse_bsr, "the padded matrix as a torch.sparse_bsr_tensor")
        .def_property_readonly("padded_rows", &BcsrTensor::padded_rows)
        .def_property_readonly("num_rows", &BcsrTensor::num_rows)
        .def_property_readonly("num_cols", &BcsrTensor::num_cols)
        .def_property_readonly("block_size", &BcsrTensor::block_size);

    m.def("coo_csr", &coo_csr_fn, "coo to csr", py::arg("keys"), py::arg("values"),
          py::arg("row_ptr"), py::arg("col_ind"), py::arg("out_vals"), py::arg("num_rows"),
          py::arg("num_cols"));
    m.def("abi_version", []() { return mps_abi_version(); });
    m.def("fsai_param_count", []() { return mps_fsai_param_count(); });
}

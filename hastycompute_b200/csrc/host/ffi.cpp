// TorchScript custom classes (torch.classes.HastyToeplitz.*), in the conventions of the
// reference's FFI (python/cpp/py_sense.cpp:83-96, py_batched_sense.cpp:171-190):
// tensors in and out, errors rethrown as RuntimeError.
#include <torch/custom_class.h>
#include <torch/library.h>

#include "hasty_toeplitz.hpp"

namespace hasty {
namespace ffi {

// hasty::fft::CUDANormalNufftToeplitz: construct from (coords, nmodes) or
// (nullopt, nmodes, diagonal).
class NormalNufftToeplitz : public torch::CustomClassHolder {
 public:
  NormalNufftToeplitz(const std::optional<at::Tensor>& coords, const std::vector<int64_t>& nmodes,
                      const std::optional<at::Tensor>& diagonal) {
    if (diagonal.has_value()) {
      at::Tensor d = *diagonal;
      _op = std::make_unique<fft::CUDANormalNufftToeplitz>(std::move(d), nmodes);
    } else if (coords.has_value()) {
      _op = std::make_unique<fft::CUDANormalNufftToeplitz>(*coords, nmodes);
    } else {
      throw std::runtime_error("NormalNufftToeplitz needs coords or a diagonal");
    }
  }
  at::Tensor apply(const at::Tensor& in, at::Tensor storage1, at::Tensor storage2) {
    return _op->apply(in, storage1, storage2);
  }
  void apply_add(const at::Tensor& in, at::Tensor add_to, at::Tensor storage1, at::Tensor storage2) {
    _op->apply_add(in, add_to, storage1, storage2);
  }
  void apply_addcmul(const at::Tensor& in, at::Tensor add_to, const at::Tensor& mul, at::Tensor storage1,
                     at::Tensor storage2) {
    _op->apply_addcmul(in, add_to, mul, storage1, storage2);
  }
  void apply_inplace(at::Tensor in, at::Tensor storage1, at::Tensor storage2) {
    _op->apply_inplace(in, storage1, storage2);
  }
  at::Tensor get_diagonal() { return _op->get_diagonal(); }
  // "fp32" (default) or "bf16x3" (forward x pass on the tensor cores, ny = nx = 128)
  void set_precision(const std::string& name) { _op->plan()->set_precision(name); }

 private:
  std::unique_ptr<fft::CUDANormalNufftToeplitz> _op;
};

// Toeplitz twin of HastySense.SenseNormal: same apply signature.
class SenseNormalToeplitz : public torch::CustomClassHolder {
 public:
  SenseNormalToeplitz(const std::optional<at::Tensor>& coords, const std::vector<int64_t>& nmodes,
                      const std::optional<at::Tensor>& diagonal) {
    if (diagonal.has_value()) {
      at::Tensor d = *diagonal;
      _op = std::make_unique<mri::CUDASenseNormalToeplitz>(std::move(d), nmodes);
    } else if (coords.has_value()) {
      _op = std::make_unique<mri::CUDASenseNormalToeplitz>(*coords, nmodes);
    } else {
      throw std::runtime_error("SenseNormalToeplitz needs coords or a diagonal");
    }
  }
  void apply(const at::Tensor& in, at::Tensor out, const at::Tensor& smaps, const std::vector<int64_t>& coils,
             const std::optional<at::Tensor>& imspace_storage, const std::optional<at::Tensor>& kspace_storage) {
    _op->apply(in, out, smaps, coils, imspace_storage, kspace_storage);
  }
  at::Tensor get_diagonal() { return _op->toeplitz()->get_diagonal(); }
  // "fp32" (default) or "bf16x3" (forward x pass on the tensor cores, ny = nx = 128)
  void set_precision(const std::string& name) { _op->toeplitz()->plan()->set_precision(name); }

 private:
  std::unique_ptr<mri::CUDASenseNormalToeplitz> _op;
};

// Toeplitz twin of HastyBatchedSense.BatchedSenseNormal, plus the batched CG.
class BatchedSenseNormalToeplitz : public torch::CustomClassHolder {
 public:
  BatchedSenseNormalToeplitz(const at::Tensor& diagonals, const at::Tensor& smaps,
                             const std::optional<std::vector<int64_t>>& diag_index)
      : _op(std::make_shared<mri::BatchedSenseNormalToeplitz>(diagonals, smaps,
                                                              diag_index.value_or(std::vector<int64_t>{}))) {}

  void apply(const at::Tensor& in, at::Tensor out, const std::optional<std::vector<std::vector<int64_t>>>& coils) {
    _op->apply(in, out, coils.has_value() ? *coils : all_coils(in), 0.0);
  }

  // "fp32" (default) or "bf16x3" (forward x pass on the tensor cores, ny = nx = 128)
  void set_precision(const std::string& name) { _op->plan()->set_precision(name); }

  void apply_regularized(const at::Tensor& in, at::Tensor out, double lambda,
                         const std::optional<std::vector<std::vector<int64_t>>>& coils) {
    _op->apply(in, out, coils.has_value() ? *coils : all_coils(in), lambda);
  }

  // ConjugateGradient::run on every outer batch of x (in place); returns per-system
  // iteration counts.  Raises "A was not positive definite" like the reference.
  std::vector<int64_t> cg(at::Tensor x, const at::Tensor& b, int64_t iters, double tol, double lambda,
                          const std::optional<std::vector<int64_t>>& coils) {
    std::vector<int64_t> cl;
    if (coils.has_value()) {
      cl = *coils;
    } else {
      for (int64_t c = 0; c < _op->smaps().size(0); ++c) cl.push_back(c);
    }
    auto A = std::make_shared<op::SenseNormalToeplitzOp>(_op, cl, lambda);
    op::Vector xv(x);
    op::ConjugateGradient solver(A, std::make_shared<op::Vector>(b), nullptr);
    solver.run(xv, (int)iters, tol);
    return std::vector<int64_t>(solver.iterations().begin(), solver.iterations().end());
  }

  // Preconditioned CG: as cg, with P = CirculantPreconditionerOp::Create(precond, centered,
  // nullopt, false) (batch_sense.ixx:388-390 builds it that way); precond is the diagonal
  // of CirculantPreconditionerOp::build_diagonal (centred) or, with centered = false, in FFT
  // order.  A real diagonal runs the device PCG.
  std::vector<int64_t> pcg(at::Tensor x, const at::Tensor& b, int64_t iters, double tol, double lambda,
                           const std::optional<std::vector<int64_t>>& coils, const at::Tensor& precond,
                           bool centered) {
    std::vector<int64_t> cl;
    if (coils.has_value()) {
      cl = *coils;
    } else {
      for (int64_t c = 0; c < _op->smaps().size(0); ++c) cl.push_back(c);
    }
    auto A = std::make_shared<op::SenseNormalToeplitzOp>(_op, cl, lambda);
    std::shared_ptr<op::Operator> P = mri::CirculantPreconditionerOp::Create(precond, centered, std::nullopt, false);
    op::Vector xv(x);
    op::ConjugateGradient solver(A, std::make_shared<op::Vector>(b), P);
    solver.run(xv, (int)iters, tol);
    return std::vector<int64_t>(solver.iterations().begin(), solver.iterations().end());
  }

 private:
  std::vector<std::vector<int64_t>> all_coils(const at::Tensor& in) const {
    const auto& d = _op->plan()->image_dims();
    const int64_t nouter = in.numel() / (d[0] * d[1] * d[2]);
    std::vector<int64_t> c;
    for (int64_t i = 0; i < _op->smaps().size(0); ++i) c.push_back(i);
    return std::vector<std::vector<int64_t>>(nouter, c);
  }
  std::shared_ptr<mri::BatchedSenseNormalToeplitz> _op;
};

// The binding the legacy Python driver calls (hastypy/reconstruct_util.py:410-434):
// in place on input [nenc, 1, nz, ny, nx] with diagonals [nenc, 2nz, 2ny, 2nx].
void batched_sense_toeplitz_diagonals(at::Tensor input, const std::vector<std::vector<int64_t>>& coils,
                                      const at::Tensor& smaps, const at::Tensor& diagonals,
                                      const std::optional<std::vector<at::Stream>>&) {
  mri::BatchedSenseNormalToeplitz op(diagonals, smaps);
  at::Tensor out = at::empty_like(input);
  op.apply(input, out, coils, 0.0);
  input.copy_(out);
}

}  // namespace ffi
}  // namespace hasty

TORCH_LIBRARY(HastyToeplitz, m) {
  m.class_<hasty::ffi::NormalNufftToeplitz>("NormalNufftToeplitz")
      .def(torch::init<const std::optional<at::Tensor>&, const std::vector<int64_t>&, const std::optional<at::Tensor>&>())
      .def("apply", &hasty::ffi::NormalNufftToeplitz::apply)
      .def("apply_add", &hasty::ffi::NormalNufftToeplitz::apply_add)
      .def("apply_addcmul", &hasty::ffi::NormalNufftToeplitz::apply_addcmul)
      .def("apply_inplace", &hasty::ffi::NormalNufftToeplitz::apply_inplace)
      .def("get_diagonal", &hasty::ffi::NormalNufftToeplitz::get_diagonal)
      .def("set_precision", &hasty::ffi::NormalNufftToeplitz::set_precision);

  m.class_<hasty::ffi::SenseNormalToeplitz>("SenseNormalToeplitz")
      .def(torch::init<const std::optional<at::Tensor>&, const std::vector<int64_t>&, const std::optional<at::Tensor>&>())
      .def("apply", &hasty::ffi::SenseNormalToeplitz::apply)
      .def("get_diagonal", &hasty::ffi::SenseNormalToeplitz::get_diagonal)
      .def("set_precision", &hasty::ffi::SenseNormalToeplitz::set_precision);

  m.class_<hasty::ffi::BatchedSenseNormalToeplitz>("BatchedSenseNormalToeplitz")
      .def(torch::init<const at::Tensor&, const at::Tensor&, const std::optional<std::vector<int64_t>>&>())
      .def("apply", &hasty::ffi::BatchedSenseNormalToeplitz::apply)
      .def("apply_regularized", &hasty::ffi::BatchedSenseNormalToeplitz::apply_regularized)
      .def("set_precision", &hasty::ffi::BatchedSenseNormalToeplitz::set_precision)
      .def("cg", &hasty::ffi::BatchedSenseNormalToeplitz::cg)
      .def("pcg", &hasty::ffi::BatchedSenseNormalToeplitz::pcg);

  m.def("circulant_precond_diagonal",
        [](const at::Tensor& smaps, const at::Tensor& coord, double lambda) {
          return hasty::mri::CirculantPreconditionerOp::build_diagonal(smaps, coord, std::nullopt, lambda);
        });

  m.def("batched_sense_toeplitz_diagonals", &hasty::ffi::batched_sense_toeplitz_diagonals);
}

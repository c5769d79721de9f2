// C++20 / LibTorch host layer mirroring the reference's operator API for the Toeplitz
// SENSE normal operator and its CG solver.  Every numerical call goes through the C ABI
// of libhasty_b200.so (include/hasty_b200.h); the classes own plans, workspaces and
// argument checking, and translate status codes into std::runtime_error as the
// reference does.
//
// Reference declarations mirrored (paths inside the HastyCompute project):
//   hasty::fft::CUDANormalNufftToeplitz      lib/fft/nufft.ixx:231-280
//   hasty::mri::CoilApplier / CoilManipulator lib/mri/sense.ixx:19-48
//   hasty::mri::CUDASenseNormal::apply        lib/mri/sense.ixx:274-282 (Toeplitz twin)
//   hasty::mri::BatchedSenseNormal::apply     lib/mri/batch_sense.ixx:249-279
//   hasty::op::Vector / Operator              lib/op/vec.ixx:39-119, lib/op/op.ixx:30-109
//   hasty::op::ConjugateGradient              lib/op/opalgs.ixx:36-47, opalgs.cpp:50-96
//   hasty::op::BatchedConjugateGradient       lib/op/opalgs.ixx:84-136
//   hasty::mri::CirculantPreconditionerOp     lib/mri/precond.ixx:13-37, precond.cpp:17-117
#pragma once

#include <ATen/ATen.h>

#include <functional>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

struct hb_plan;

namespace hasty {

template <typename T>
using sptr = std::shared_ptr<T>;

namespace detail {
// Owns one hb_plan (geometry + twiddle tables) for a device and image size.
class Plan {
 public:
  Plan(const std::vector<int64_t>& nmodes, c10::Device device);
  ~Plan();
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;
  hb_plan* get() const { return _p; }
  c10::Device device() const { return _device; }
  const std::vector<int64_t>& image_dims() const { return _dims; }  // {nz, ny, nx}
  std::vector<int64_t> grid_dims() const { return {2 * _dims[0], 2 * _dims[1], 2 * _dims[2]}; }
  int64_t packed_numel() const;
  at::Tensor workspace(size_t bytes) const;  // device scratch from the caching allocator
  // "fp32" (default) or "bf16x3": the forward x pass as a tensor-core contraction with
  // BF16 hi + lo operands (ny = nx = 128); applies to every later call with this plan
  void set_precision(const std::string& name);

 private:
  hb_plan* _p = nullptr;
  c10::Device _device;
  std::vector<int64_t> _dims;
};

void check(int code);               // throws std::runtime_error(hb_last_error())
void* current_stream(c10::Device device);
}  // namespace detail

namespace fft {

// Drop-in for hasty::fft::CUDANormalNufftToeplitz (nufft.ixx:231-280).
// nmodes = {ntransf(=1), nz, ny, nx}; storage tensors are [1, 2nz, 2ny, 2nx] complex64.
class CUDANormalNufftToeplitz {
 public:
  CUDANormalNufftToeplitz(const at::Tensor& coords, const std::vector<int64_t>& nmodes,
                          const std::optional<double>& tol = std::nullopt,
                          const std::optional<std::reference_wrapper<at::Tensor>>& diagonal = std::nullopt,
                          const std::optional<std::reference_wrapper<at::Tensor>>& frequency_storage = std::nullopt,
                          const std::optional<std::reference_wrapper<at::Tensor>>& input_storage = std::nullopt);

  CUDANormalNufftToeplitz(at::Tensor&& diagonal, const std::vector<int64_t>& nmodes);

  static void build_diagonal(const at::Tensor& coords, std::vector<int64_t> nmodes, double tol, at::Tensor& diagonal);
  static void build_diagonal(const at::Tensor& coords, std::vector<int64_t> nmodes, double tol, at::Tensor& diagonal,
                             at::Tensor& storage, bool storage_is_frequency);
  static void build_diagonal(const at::Tensor& coords, std::vector<int64_t> nmodes, double tol, at::Tensor& diagonal,
                             at::Tensor& frequency_storage, at::Tensor& input_storage);

  at::Tensor apply(const at::Tensor& in, at::Tensor& storage1, at::Tensor& storage2) const;
  void apply_add(const at::Tensor& in, at::Tensor& add_to, at::Tensor& storage1, at::Tensor& storage2) const;
  void apply_addcmul(const at::Tensor& in, at::Tensor& add_to, const at::Tensor& mul, at::Tensor& storage1,
                     at::Tensor& storage2) const;
  void apply_inplace(at::Tensor& in, at::Tensor& storage1, at::Tensor& storage2) const;

  at::Tensor get_diagonal();

  // internal layout read by the kernels (Re(T) / prod(2N))
  const at::Tensor& packed_diagonal() const { return _packed; }
  const std::shared_ptr<detail::Plan>& plan() const { return _plan; }
  const std::vector<int64_t>& nmodes() const { return _nmodes; }

 private:
  void init_plan(c10::Device device);
  void run(const at::Tensor& in, at::Tensor& out, int64_t ldz, int64_t ldy, const at::Tensor* mul,
           bool accumulate) const;

  std::vector<int64_t> _nmodes;
  std::shared_ptr<detail::Plan> _plan;
  at::Tensor _diagonal;  // reference layout [1, 2nz, 2ny, 2nx] complex64
  at::Tensor _packed;
  bool _created_from_diagonal = false;
};

}  // namespace fft

namespace mri {

using CoilApplier = std::function<void(at::Tensor&, int32_t)>;

// Toeplitz twin of hasty::mri::CUDASenseNormal (sense.ixx:274-282, body sense.ixx:500-578
// with the per-coil NUFFT pair replaced by CUDANormalNufftToeplitz::apply_addcmul).
class CUDASenseNormalToeplitz {
 public:
  CUDASenseNormalToeplitz(const at::Tensor& coords, const std::vector<int64_t>& nmodes);
  CUDASenseNormalToeplitz(at::Tensor&& diagonal, const std::vector<int64_t>& nmodes);
  explicit CUDASenseNormalToeplitz(std::shared_ptr<fft::CUDANormalNufftToeplitz> toeplitz);

  // out = sum_{c in coils} conj(S_c) * Top(S_c * in).  kspace_storage has no meaning for
  // the Toeplitz form and is ignored; midmanip must be absent (no k-space stage).
  // Without manipulators the whole coil loop is one fused launch sequence.
  void apply(const at::Tensor& in, at::Tensor& out, const at::Tensor& smaps, const std::vector<int64_t>& coils,
             const std::optional<at::Tensor>& imspace_storage = std::nullopt,
             const std::optional<at::Tensor>& kspace_storage = std::nullopt,
             const std::optional<CoilApplier>& premanip = std::nullopt,
             const std::optional<CoilApplier>& midmanip = std::nullopt,
             const std::optional<CoilApplier>& postmanip = std::nullopt);

  const std::shared_ptr<fft::CUDANormalNufftToeplitz>& toeplitz() const { return _top; }

 private:
  std::shared_ptr<fft::CUDANormalNufftToeplitz> _top;
};

// Batched Toeplitz SENSE normal op over outer batches (systems): the reference's
// BatchedSenseNormal::apply (batch_sense.cpp:349-450) with host staging replaced by one
// resident launch sequence.  diagonals: [ndiag, 2nz, 2ny, 2nx] (or [ndiag, 1, ...]);
// diag_index maps outer batch -> diagonal (default: outer batch i uses diagonal i, or 0
// when there is one diagonal).  in/out: [n_outer, 1, nz, ny, nx] on CPU or CUDA.
class BatchedSenseNormalToeplitz {
 public:
  BatchedSenseNormalToeplitz(const at::Tensor& diagonals, const at::Tensor& smaps,
                             std::vector<int64_t> diag_index = {});
  void apply(const at::Tensor& in, at::Tensor out, const std::vector<std::vector<int64_t>>& coils,
             double lambda = 0.0);
  const at::Tensor& packed() const { return _packed; }
  const at::Tensor& smaps() const { return _smaps; }
  const std::shared_ptr<detail::Plan>& plan() const { return _plan; }
  const std::vector<int64_t>& diag_index() const { return _diag_index; }

 private:
  std::shared_ptr<detail::Plan> _plan;
  at::Tensor _packed;  // [ndiag * packed]
  at::Tensor _smaps;
  int64_t _ndiag = 0;
  std::vector<int64_t> _diag_index;
};

}  // namespace mri

namespace op {

// Tensor-or-tree vector (vec.ixx:39-119), with what CG needs.
class Vector {
 public:
  Vector() = default;
  Vector(const at::Tensor& t) : _tensor(t) {}
  Vector(const std::vector<Vector>& children) : _children(children) {}
  bool has_children() const { return !_children.empty(); }
  const std::vector<Vector>& children() const { return _children; }
  std::vector<Vector>& children() { return _children; }
  const at::Tensor& tensor() const { return _tensor; }
  at::Tensor& tensor() { return _tensor; }
  Vector clone() const;
  Vector& operator+=(const Vector& rhs);
  Vector& operator-=(const Vector& rhs);
  friend Vector operator-(const Vector& lhs, const Vector& rhs);
  Vector scaled(const at::Tensor& s) const;  // this * s
  Vector& scale_(const at::Tensor& s);        // this *= s
  friend at::Tensor vdot(const Vector& a, const Vector& b);  // sum conj(a) b (vec.cpp:624-637)

 private:
  at::Tensor _tensor;
  std::vector<Vector> _children;
};

class Operator {
 public:
  virtual ~Operator() = default;
  virtual Vector apply(const Vector& in) const = 0;
  Vector operator()(const Vector& in) const { return apply(in); }
};

// (A^H A)_toeplitz + lambda I over one or more systems (a Vector's children).
class SenseNormalToeplitzOp : public Operator {
 public:
  SenseNormalToeplitzOp(std::shared_ptr<mri::BatchedSenseNormalToeplitz> batched, std::vector<int64_t> coils,
                        double lambda);
  Vector apply(const Vector& in) const override;
  const std::shared_ptr<mri::BatchedSenseNormalToeplitz>& batched() const { return _b; }
  const std::vector<int64_t>& coils() const { return _coils; }
  double lambda() const { return _lambda; }

 private:
  std::shared_ptr<mri::BatchedSenseNormalToeplitz> _b;
  std::vector<int64_t> _coils;
  double _lambda;
};

}  // namespace op

namespace mri {

// Drop-in for hasty::mri::CirculantPreconditionerOp (precond.ixx:13-37, precond.cpp:17-63):
//   P x = ifft(D * fft(x))                       (centered = false)
//   P x = ifftc(D * fftc(x))                     (centered = true)
//   adjointify: fft(conj(D) * ifft(x)), resp. fftc(conj(D) * ifftc(x)).
// norm may be absent, "backward", "ortho" or "forward" (the pair's scaling is 1/N for all
// three).  When D is real and the image size is one the kernels support, the operator is
// also held as the real float32 diagonal in FFT order that the device PCG reads (for even
// sizes ifftc(D * fftc(x)) = ifft(ifftshift(D) * fft(x)), and for real D the adjointified
// form is the same operator with D index-reversed), and apply() runs hb_precond_apply.
// Otherwise apply() runs the reference's ATen calls.
class CirculantPreconditionerOp : public op::Operator {
 public:
  static std::unique_ptr<CirculantPreconditionerOp> Create(at::Tensor diag, bool centered,
                                                           const std::optional<std::string>& norm, bool adjointify);
  // precond.cpp:65-117 (ported from sigpy there): 1 / (d + lambda), d the Fourier-domain
  // diagonal of sum_c S_c^H (A^H A)_toep S_c for the trajectory coord [3, K] float32,
  // built on the device by hb_precond_build (tol 1e-6); returned in the centred layout,
  // float32 [nz, ny, nx], the form the reference's loaders pass to Create(diag, true, ...)
  // (batch_sense.ixx:388-390).  Sample weights are not supported (std::runtime_error).
  static at::Tensor build_diagonal(at::Tensor smaps, at::Tensor coord,
                                   const std::optional<at::Tensor>& weights = std::nullopt,
                                   const std::optional<double>& lambda = 0.0);
  op::Vector apply(const op::Vector& in) const override;
  // Real float32 [nz, ny, nx] diagonal in FFT order for the device PCG; undefined tensor
  // when the operator has no such form.
  const at::Tensor& fft_order_diagonal() const { return _fftdiag; }

 protected:
  CirculantPreconditionerOp(at::Tensor diag, bool centered, const std::optional<std::string>& norm, bool adjointify);

 private:
  at::Tensor _diag;
  bool _centered;
  std::optional<std::string> _norm;
  bool _adjointify;
  at::Tensor _fftdiag;
  std::shared_ptr<detail::Plan> _plan;
};

}  // namespace mri

namespace op {

// ConjugateGradient(A, b, P).run(x, iter, tol)  (opalgs.cpp:50-96).
// With A a SenseNormalToeplitzOp and P absent or a CirculantPreconditionerOp with a real
// diagonal, the whole solve (all systems of x) runs on the device (fused updates, FP64
// reductions, no per-iteration host sync; preconditioned CG when P is given).  Any other
// operator runs the reference recurrences on ATen tensors.
class ConjugateGradient {
 public:
  ConjugateGradient(sptr<Operator> A, sptr<Vector> b, sptr<Operator> P);
  void run(Vector& x, int iter = 30, double tol = 0.0);
  const std::vector<int32_t>& status() const { return _status; }
  const std::vector<int32_t>& iterations() const { return _iters; }

 private:
  sptr<Operator> _A;
  sptr<Vector> _b;
  sptr<Operator> _P;
  std::vector<int32_t> _status, _iters;
};

struct ConjugateGradientLoadResult {
  sptr<Operator> A;
  Vector b;
  sptr<Operator> P;
};

// BatchedConjugateGradient (opalgs.ixx:84-136): one CG per child of x.  Children whose
// operators are SenseNormalToeplitzOps sharing one batched operator (same smaps, coils
// and lambda) are solved together in one device launch sequence.
class BatchedConjugateGradient {
 public:
  explicit BatchedConjugateGradient(std::vector<ConjugateGradientLoadResult> systems);
  void run(Vector& x, int iter = 30, double tol = 0.0);

 private:
  std::vector<ConjugateGradientLoadResult> _systems;
};

}  // namespace op
}  // namespace hasty

// Implementation of the LibTorch host layer (hasty_toeplitz.hpp).
#include "hasty_toeplitz.hpp"

#include <ATen/ops/vdot.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

#include <string>

#include "hasty_b200.h"

namespace hasty {
namespace detail {

void check(int code) {
  if (code == HB_OK) return;
  throw std::runtime_error(std::string(hb_last_error()));
}

void* current_stream(c10::Device device) {
  return (void*)c10::cuda::getCurrentCUDAStream(device.index()).stream();
}

Plan::Plan(const std::vector<int64_t>& nmodes, c10::Device device) : _device(device) {
  if (nmodes.size() != 3) throw std::runtime_error("Toeplitz plan needs three spatial dimensions");
  if (!device.is_cuda()) throw std::runtime_error("Toeplitz operators run on CUDA devices only");
  _dims = nmodes;
  check(hb_plan_create(&_p, nmodes[0], nmodes[1], nmodes[2], device.index()));
}

Plan::~Plan() {
  if (_p) hb_plan_destroy(_p);
}

int64_t Plan::packed_numel() const { return hb_diag_packed_floats(_p); }

void Plan::set_precision(const std::string& name) {
  if (name == "fp32") {
    check(hb_plan_set_precision(_p, HB_PRECISION_FP32));
  } else if (name == "bf16x3") {
    check(hb_plan_set_precision(_p, HB_PRECISION_BF16X3));
  } else {
    throw std::runtime_error("precision must be \"fp32\" or \"bf16x3\", got \"" + name + "\"");
  }
}

at::Tensor Plan::workspace(size_t bytes) const {
  return at::empty({(int64_t)std::max<size_t>(bytes, 1)}, at::TensorOptions().dtype(at::kByte).device(_device));
}

namespace {
void require(bool ok, const char* msg) {
  if (!ok) throw std::runtime_error(msg);
}

void check_image(const at::Tensor& t, const char* name, c10::Device dev, const std::vector<int64_t>& dims) {
  if (t.scalar_type() != at::kComplexFloat) throw std::runtime_error(std::string(name) + " must be complex64");
  if (t.device() != dev) throw std::runtime_error(std::string("All tensors must reside on same device (") + name + ")");
  if (!t.is_contiguous()) throw std::runtime_error(std::string(name) + " must be contiguous");
  const auto n = t.numel();
  if (n != dims[0] * dims[1] * dims[2]) throw std::runtime_error(std::string(name) + " has the wrong number of elements");
}

std::vector<int64_t> spatial(const std::vector<int64_t>& nmodes) {
  if (nmodes.size() == 4) {
    if (nmodes[0] != 1) throw std::runtime_error("only ntransf = 1 is supported");
    return {nmodes[1], nmodes[2], nmodes[3]};
  }
  if (nmodes.size() == 3) return nmodes;
  throw std::runtime_error("nmodes must be {ntransf, nz, ny, nx}");
}

at::Tensor pack_diagonals(const Plan& plan, const at::Tensor& diagonals, int64_t ndiag) {
  auto g = plan.grid_dims();
  at::Tensor d = diagonals.to(plan.device(), at::kComplexFloat).contiguous().reshape({ndiag, g[0], g[1], g[2]});
  at::Tensor packed = at::empty({ndiag * plan.packed_numel()}, at::TensorOptions().dtype(at::kFloat).device(plan.device()));
  void* st = current_stream(plan.device());
  for (int64_t i = 0; i < ndiag; ++i)
    check(hb_diag_pack(plan.get(), d[i].data_ptr(), packed.data_ptr<float>() + i * plan.packed_numel(), st));
  return packed;
}
}  // namespace
}  // namespace detail

// ============================================================ fft ==================
namespace fft {

void CUDANormalNufftToeplitz::init_plan(c10::Device device) {
  _plan = std::make_shared<detail::Plan>(detail::spatial(_nmodes), device);
}

CUDANormalNufftToeplitz::CUDANormalNufftToeplitz(const at::Tensor& coords, const std::vector<int64_t>& nmodes,
                                                 const std::optional<double>& tol,
                                                 const std::optional<std::reference_wrapper<at::Tensor>>& diagonal,
                                                 const std::optional<std::reference_wrapper<at::Tensor>>&,
                                                 const std::optional<std::reference_wrapper<at::Tensor>>&)
    : _nmodes(nmodes), _created_from_diagonal(false) {
  c10::InferenceMode guard;
  (void)tol;  // the diagonal is built exactly in FP64; the reference ignores tol too (nufft.cpp:937)
  if (coords.dim() != 2 || coords.size(0) + 1 != (int64_t)nmodes.size())
    throw std::runtime_error("coords.size(0) must match number of nmodes given");
  if (!coords.is_contiguous()) throw std::runtime_error("coords must be contiguous");
  if (coords.scalar_type() != at::kFloat) throw std::runtime_error("Unsupported type in build_diagonal");
  init_plan(coords.device());
  auto g = _plan->grid_dims();
  if (diagonal.has_value()) {
    _diagonal = diagonal->get();
  } else {
    _diagonal = at::empty({1, g[0], g[1], g[2]}, coords.options().dtype(at::kComplexFloat));
  }
  build_diagonal(coords, _nmodes, 1e-6, _diagonal);
  _packed = detail::pack_diagonals(*_plan, _diagonal, 1);
}

CUDANormalNufftToeplitz::CUDANormalNufftToeplitz(at::Tensor&& diagonal, const std::vector<int64_t>& nmodes)
    : _nmodes(nmodes), _diagonal(std::move(diagonal)), _created_from_diagonal(true) {
  c10::InferenceMode guard;
  init_plan(_diagonal.device());
  _packed = detail::pack_diagonals(*_plan, _diagonal, 1);
}

void CUDANormalNufftToeplitz::build_diagonal(const at::Tensor& coords, std::vector<int64_t> nmodes, double,
                                             at::Tensor& diagonal) {
  c10::InferenceMode guard;
  if (coords.scalar_type() != at::kFloat) throw std::runtime_error("Unsupported type in build_diagonal");
  if (!coords.is_cuda()) throw std::runtime_error("build_diagonal: coords must be a CUDA tensor");
  detail::Plan plan(detail::spatial(nmodes), coords.device());
  auto g = plan.grid_dims();
  if (diagonal.scalar_type() != at::kComplexFloat || !diagonal.is_contiguous() ||
      diagonal.numel() != g[0] * g[1] * g[2] || diagonal.device() != coords.device())
    throw std::runtime_error("diagonal must be a contiguous complex64 [1, 2nz, 2ny, 2nx] tensor on coords' device");
  at::Tensor c = coords.contiguous();
  const int64_t K = c.size(1);
  size_t nb = hb_diag_build_workspace_bytes(plan.get(), K);
  at::Tensor ws = plan.workspace(nb);
  detail::check(hb_diag_build(plan.get(), c.data_ptr<float>(), K, nullptr, diagonal.data_ptr(), ws.data_ptr(), nb,
                              detail::current_stream(plan.device())));
}

void CUDANormalNufftToeplitz::build_diagonal(const at::Tensor& coords, std::vector<int64_t> nmodes, double tol,
                                             at::Tensor& diagonal, at::Tensor&, bool) {
  build_diagonal(coords, std::move(nmodes), tol, diagonal);
}

void CUDANormalNufftToeplitz::build_diagonal(const at::Tensor& coords, std::vector<int64_t> nmodes, double tol,
                                             at::Tensor& diagonal, at::Tensor&, at::Tensor&) {
  build_diagonal(coords, std::move(nmodes), tol, diagonal);
}

void CUDANormalNufftToeplitz::run(const at::Tensor& in, at::Tensor& out, int64_t ldz, int64_t ldy,
                                  const at::Tensor* mul, bool accumulate) const {
  const auto& dims = _plan->image_dims();
  detail::check_image(in, "in", _plan->device(), dims);
  if (mul) detail::check_image(*mul, "mul", _plan->device(), dims);
  size_t nb = hb_normal_workspace_bytes(_plan->get(), 1, 1);
  at::Tensor ws = _plan->workspace(nb);
  detail::check(hb_toeplitz_apply(_plan->get(), in.data_ptr(), out.data_ptr(), ldz, ldy,
                                  mul ? mul->data_ptr() : nullptr, accumulate ? 1 : 0, _packed.data_ptr<float>(),
                                  ws.data_ptr(), nb, detail::current_stream(_plan->device())));
}

at::Tensor CUDANormalNufftToeplitz::apply(const at::Tensor& in, at::Tensor&, at::Tensor& storage2) const {
  c10::InferenceMode guard;
  auto g = _plan->grid_dims();
  const auto& d = _plan->image_dims();
  if (storage2.numel() != g[0] * g[1] * g[2] || !storage2.is_contiguous() ||
      storage2.scalar_type() != at::kComplexFloat || storage2.device() != _plan->device())
    throw std::runtime_error("storage2 must be a contiguous complex64 [1, 2nz, 2ny, 2nx] tensor on the device");
  run(in, storage2, g[1] * g[2], g[2], nullptr, false);
  using namespace at::indexing;
  at::Tensor s2 = storage2.reshape({1, g[0], g[1], g[2]});
  return s2.index({Slice(), Slice(0, d[0]), Slice(0, d[1]), Slice(0, d[2])});
}

void CUDANormalNufftToeplitz::apply_add(const at::Tensor& in, at::Tensor& add_to, at::Tensor&, at::Tensor&) const {
  c10::InferenceMode guard;
  const auto& d = _plan->image_dims();
  detail::check_image(add_to, "add_to", _plan->device(), d);
  run(in, add_to, d[1] * d[2], d[2], nullptr, true);
}

void CUDANormalNufftToeplitz::apply_addcmul(const at::Tensor& in, at::Tensor& add_to, const at::Tensor& mul,
                                            at::Tensor&, at::Tensor&) const {
  c10::InferenceMode guard;
  const auto& d = _plan->image_dims();
  detail::check_image(add_to, "add_to", _plan->device(), d);
  run(in, add_to, d[1] * d[2], d[2], &mul, true);
}

void CUDANormalNufftToeplitz::apply_inplace(at::Tensor& in, at::Tensor&, at::Tensor&) const {
  c10::InferenceMode guard;
  const auto& d = _plan->image_dims();
  run(in, in, d[1] * d[2], d[2], nullptr, false);
}

at::Tensor CUDANormalNufftToeplitz::get_diagonal() { return _diagonal; }

}  // namespace fft

// ============================================================ mri ==================
namespace mri {

CUDASenseNormalToeplitz::CUDASenseNormalToeplitz(const at::Tensor& coords, const std::vector<int64_t>& nmodes)
    : _top(std::make_shared<fft::CUDANormalNufftToeplitz>(coords, nmodes)) {}

CUDASenseNormalToeplitz::CUDASenseNormalToeplitz(at::Tensor&& diagonal, const std::vector<int64_t>& nmodes)
    : _top(std::make_shared<fft::CUDANormalNufftToeplitz>(std::move(diagonal), nmodes)) {}

CUDASenseNormalToeplitz::CUDASenseNormalToeplitz(std::shared_ptr<fft::CUDANormalNufftToeplitz> toeplitz)
    : _top(std::move(toeplitz)) {}

void CUDASenseNormalToeplitz::apply(const at::Tensor& in, at::Tensor& out, const at::Tensor& smaps,
                                    const std::vector<int64_t>& coils, const std::optional<at::Tensor>&,
                                    const std::optional<at::Tensor>&, const std::optional<CoilApplier>& premanip,
                                    const std::optional<CoilApplier>& midmanip,
                                    const std::optional<CoilApplier>& postmanip) {
  c10::InferenceMode guard;
  const auto& plan = *_top->plan();
  const auto& d = plan.image_dims();
  if (midmanip.has_value())
    throw std::runtime_error("midmanip has no meaning for the Toeplitz normal operator (there is no k-space stage)");
  detail::check_image(in, "in", plan.device(), d);
  detail::check_image(out, "out", plan.device(), d);
  if (smaps.scalar_type() != at::kComplexFloat || !smaps.is_contiguous() || smaps.device() != plan.device() ||
      smaps.dim() != 4 || smaps.size(1) != d[0] || smaps.size(2) != d[1] || smaps.size(3) != d[2])
    throw std::runtime_error("smaps must be a contiguous complex64 [ncoil, nz, ny, nx] tensor on the device");
  for (int64_t c : coils)
    if (c < 0 || c >= smaps.size(0)) throw std::runtime_error("coil index out of range");
  if (coils.empty()) {
    out.zero_();
    return;
  }
  if (!premanip.has_value() && !postmanip.has_value()) {
    size_t nb = hb_normal_workspace_bytes(plan.get(), 1, (int64_t)coils.size());
    at::Tensor ws = plan.workspace(nb);
    detail::check(hb_sense_normal_apply(plan.get(), 1, in.data_ptr(), out.data_ptr(), smaps.data_ptr(), coils.data(),
                                        (int64_t)coils.size(), _top->packed_diagonal().data_ptr<float>(), nullptr,
                                        0.f, ws.data_ptr(), nb, detail::current_stream(plan.device())));
    return;
  }
  // With coil manipulators: the reference's per-coil loop (sense.ixx:533-577), one
  // Toeplitz launch sequence per coil, manipulators applied as the reference does.
  out.zero_();
  at::Tensor imstore = at::empty_like(in);
  at::Tensor s = at::empty({0}, in.options());
  for (size_t j = 0; j < coils.size(); ++j) {
    imstore.copy_(in);
    if (premanip.has_value()) (*premanip)(imstore, (int32_t)j);
    imstore.mul_(smaps.select(0, coils[j]).reshape(imstore.sizes()));
    _top->apply_inplace(imstore, s, s);
    imstore.mul_(smaps.select(0, coils[j]).conj().reshape(imstore.sizes()));
    if (postmanip.has_value()) (*postmanip)(imstore, (int32_t)j);
    out.add_(imstore);
  }
}

BatchedSenseNormalToeplitz::BatchedSenseNormalToeplitz(const at::Tensor& diagonals, const at::Tensor& smaps,
                                                       std::vector<int64_t> diag_index)
    : _diag_index(std::move(diag_index)) {
  c10::InferenceMode guard;
  c10::Device dev = smaps.is_cuda() ? smaps.device()
                                    : (diagonals.is_cuda() ? diagonals.device() : c10::Device(c10::kCUDA, 0));
  if (smaps.dim() != 4) throw std::runtime_error("smaps must be [ncoil, nz, ny, nx]");
  _plan = std::make_shared<detail::Plan>(std::vector<int64_t>{smaps.size(1), smaps.size(2), smaps.size(3)}, dev);
  auto g = _plan->grid_dims();
  const int64_t per = g[0] * g[1] * g[2];
  if (diagonals.numel() % per != 0) throw std::runtime_error("diagonals must be [ndiag, 2nz, 2ny, 2nx]");
  _ndiag = diagonals.numel() / per;
  _packed = detail::pack_diagonals(*_plan, diagonals, _ndiag);
  _smaps = smaps.to(dev, at::kComplexFloat).contiguous();
  for (int64_t d : _diag_index)
    if (d < 0 || d >= _ndiag) throw std::runtime_error("diag_index out of range");
}

void BatchedSenseNormalToeplitz::apply(const at::Tensor& in, at::Tensor out,
                                       const std::vector<std::vector<int64_t>>& coils, double lambda) {
  c10::InferenceMode guard;
  const auto& d = _plan->image_dims();
  const int64_t nv = d[0] * d[1] * d[2];
  const int64_t nouter = in.numel() / nv;
  if (nouter * nv != in.numel() || out.numel() != in.numel())
    throw std::runtime_error("in/out must be [n_outer, 1, nz, ny, nx]");
  if ((int64_t)coils.size() != nouter) throw std::runtime_error("coils must hold one list per outer batch");
  std::vector<int64_t> didx(nouter);
  for (int64_t i = 0; i < nouter; ++i) {
    if (!_diag_index.empty()) {
      if ((int64_t)_diag_index.size() != nouter) throw std::runtime_error("diag_index must have one entry per outer batch");
      didx[i] = _diag_index[i];
    } else {
      didx[i] = _ndiag == 1 ? 0 : i;
    }
    if (didx[i] >= _ndiag) throw std::runtime_error("not enough diagonals for the outer batches");
  }
  at::Tensor xin = in.to(_plan->device(), at::kComplexFloat).contiguous().reshape({nouter, d[0], d[1], d[2]});
  const bool out_on_dev = out.device() == _plan->device() && out.is_contiguous() && out.scalar_type() == at::kComplexFloat;
  at::Tensor xo = out_on_dev ? out.reshape({nouter, d[0], d[1], d[2]}) : at::empty_like(xin);
  void* st = detail::current_stream(_plan->device());
  // group outer batches that use the same coil list into one launch sequence
  std::vector<bool> done(nouter, false);
  for (int64_t i = 0; i < nouter; ++i) {
    if (done[i]) continue;
    std::vector<int64_t> members;
    for (int64_t j = i; j < nouter; ++j)
      if (!done[j] && coils[j] == coils[i]) members.push_back(j);
    for (int64_t c : coils[i])
      if (c < 0 || c >= _smaps.size(0)) throw std::runtime_error("coil index out of range");
    if (coils[i].empty()) {
      for (int64_t j : members) { xo[j].zero_(); done[j] = true; }
      continue;
    }
    const bool contiguous_run = members.back() - members.front() + 1 == (int64_t)members.size();
    at::Tensor xs = contiguous_run ? xin.narrow(0, members.front(), members.size())
                                   : xin.index_select(0, at::tensor(members).to(xin.device()));
    at::Tensor os = contiguous_run ? xo.narrow(0, members.front(), members.size()) : at::empty_like(xs);
    std::vector<int64_t> dsub;
    for (int64_t j : members) dsub.push_back(didx[j]);
    size_t nb = hb_normal_workspace_bytes(_plan->get(), (int64_t)members.size(), (int64_t)coils[i].size());
    at::Tensor ws = _plan->workspace(nb);
    detail::check(hb_sense_normal_apply(_plan->get(), (int64_t)members.size(), xs.data_ptr(), os.data_ptr(),
                                        _smaps.data_ptr(), coils[i].data(), (int64_t)coils[i].size(),
                                        _packed.data_ptr<float>(), dsub.data(), (float)lambda, ws.data_ptr(), nb, st));
    if (!contiguous_run)
      for (size_t k = 0; k < members.size(); ++k) xo[members[k]].copy_(os[k]);
    for (int64_t j : members) done[j] = true;
  }
  if (!out_on_dev) out.copy_(xo.reshape(out.sizes()));
}

}  // namespace mri

// ============================================================ op ===================
namespace op {

Vector Vector::clone() const {
  if (!has_children()) return Vector(_tensor.clone());
  std::vector<Vector> c;
  for (const auto& ch : _children) c.push_back(ch.clone());
  return Vector(c);
}

Vector& Vector::operator+=(const Vector& rhs) {
  if (!has_children()) {
    _tensor.add_(rhs._tensor);
  } else {
    for (size_t i = 0; i < _children.size(); ++i) _children[i] += rhs._children[i];
  }
  return *this;
}

Vector& Vector::operator-=(const Vector& rhs) {
  if (!has_children()) {
    _tensor.sub_(rhs._tensor);
  } else {
    for (size_t i = 0; i < _children.size(); ++i) _children[i] -= rhs._children[i];
  }
  return *this;
}

Vector operator-(const Vector& lhs, const Vector& rhs) {
  Vector out = lhs.clone();
  out -= rhs;
  return out;
}

Vector Vector::scaled(const at::Tensor& s) const {
  Vector out = clone();
  out.scale_(s);
  return out;
}

Vector& Vector::scale_(const at::Tensor& s) {
  if (!has_children()) {
    _tensor.mul_(s);
  } else {
    for (auto& ch : _children) ch.scale_(s);
  }
  return *this;
}

at::Tensor vdot(const Vector& a, const Vector& b) {
  if (!a.has_children()) return at::vdot(a.tensor().flatten(), b.tensor().flatten());
  at::Tensor s = vdot(a.children()[0], b.children()[0]);
  for (size_t i = 1; i < a.children().size(); ++i) s = s + vdot(a.children()[i], b.children()[i]);
  return s;
}

namespace {
// Flattens a Vector (tensor or children) into a contiguous [nsys, nz, ny, nx] device tensor.
at::Tensor gather_systems(const Vector& v, const detail::Plan& plan) {
  const auto& d = plan.image_dims();
  if (!v.has_children())
    return v.tensor().to(plan.device(), at::kComplexFloat).contiguous().reshape({-1, d[0], d[1], d[2]});
  std::vector<at::Tensor> parts;
  for (const auto& ch : v.children()) parts.push_back(gather_systems(ch, plan));
  return at::cat(parts, 0);
}

void scatter_systems(Vector& v, const at::Tensor& all, int64_t& offset) {
  if (!v.has_children()) {
    const int64_t n = v.tensor().numel() / (all.numel() / all.size(0));
    v.tensor().copy_(all.narrow(0, offset, n).reshape(v.tensor().sizes()));
    offset += n;
    return;
  }
  for (auto& ch : v.children()) scatter_systems(ch, all, offset);
}

int64_t count_systems(const Vector& v, int64_t nv) {
  if (!v.has_children()) return v.tensor().numel() / nv;
  int64_t n = 0;
  for (const auto& ch : v.children()) n += count_systems(ch, nv);
  return n;
}
}  // namespace

SenseNormalToeplitzOp::SenseNormalToeplitzOp(std::shared_ptr<mri::BatchedSenseNormalToeplitz> batched,
                                             std::vector<int64_t> coils, double lambda)
    : _b(std::move(batched)), _coils(std::move(coils)), _lambda(lambda) {}

Vector SenseNormalToeplitzOp::apply(const Vector& in) const {
  const auto& plan = *_b->plan();
  at::Tensor x = gather_systems(in, plan);
  at::Tensor y = at::empty_like(x);
  std::vector<std::vector<int64_t>> coils(x.size(0), _coils);
  _b->apply(x, y, coils, _lambda);
  Vector out = in.clone();
  int64_t off = 0;
  scatter_systems(out, y, off);
  return out;
}

ConjugateGradient::ConjugateGradient(sptr<Operator> A, sptr<Vector> b, sptr<Operator> P)
    : _A(std::move(A)), _b(std::move(b)), _P(std::move(P)) {}

void ConjugateGradient::run(Vector& x, int iter, double tol) {
  c10::InferenceMode guard;
  if (iter < 1) return;
  auto top = std::dynamic_pointer_cast<SenseNormalToeplitzOp>(_A);
  if (top && !_P) {
    const auto& bat = *top->batched();
    const auto& plan = *bat.plan();
    const auto& d = plan.image_dims();
    at::Tensor xs = gather_systems(x, plan);
    at::Tensor bs = gather_systems(*_b, plan);
    const int64_t nsys = xs.size(0);
    if (bs.size(0) != nsys) throw std::runtime_error("x and b hold different numbers of systems");
    std::vector<int64_t> didx(nsys);
    for (int64_t i = 0; i < nsys; ++i)
      didx[i] = bat.diag_index().empty() ? (nsys == 1 ? 0 : i) : bat.diag_index()[i];
    _status.assign(nsys, 0);
    _iters.assign(nsys, 0);
    size_t nb = hb_cg_workspace_bytes(plan.get(), nsys, (int64_t)top->coils().size(), iter);
    at::Tensor ws = plan.workspace(nb);
    int rc = hb_cg_run(plan.get(), nsys, xs.data_ptr(), bs.data_ptr(), bat.smaps().data_ptr(), top->coils().data(),
                       (int64_t)top->coils().size(), bat.packed().data_ptr<float>(), didx.data(),
                       (float)top->lambda(), iter, tol, _status.data(), _iters.data(), ws.data_ptr(), nb,
                       detail::current_stream(plan.device()));
    int64_t off = 0;
    scatter_systems(x, xs, off);
    (void)d;
    detail::check(rc);
    return;
  }
  // generic operator: the reference recurrences on ATen tensors (opalgs.cpp:50-96)
  Vector r = *_b - _A->apply(x);
  Vector z = _P ? _P->apply(r) : r;
  Vector p = z.clone();
  at::Tensor rzold = at::real(vdot(r, z));
  double resid = std::sqrt(rzold.item<double>());
  for (int i = 0; i < iter; ++i) {
    if (resid < tol) return;
    Vector Ap = _A->apply(p);
    at::Tensor pAp = at::real(vdot(p, Ap));
    if (pAp.item<double>() <= 0.0) throw std::runtime_error("A was not positive definite");
    at::Tensor alpha = rzold / pAp;
    x += p.scaled(alpha);
    r -= Ap.scaled(alpha);
    z = _P ? _P->apply(r) : r;
    at::Tensor rznew = at::real(vdot(r, z));
    p.scale_(rznew / rzold);
    p += z;
    rzold = rznew;
    resid = std::sqrt(rzold.item<double>());
  }
}

BatchedConjugateGradient::BatchedConjugateGradient(std::vector<ConjugateGradientLoadResult> systems)
    : _systems(std::move(systems)) {}

void BatchedConjugateGradient::run(Vector& x, int iter, double tol) {
  c10::InferenceMode guard;
  auto& children = x.children();
  if (children.size() != _systems.size()) throw std::runtime_error("one load result per child of x is required");
  // fuse every system whose operator shares the first system's batched Toeplitz op
  auto first = std::dynamic_pointer_cast<SenseNormalToeplitzOp>(_systems.empty() ? nullptr : _systems[0].A);
  bool fusable = first != nullptr;
  for (const auto& s : _systems) {
    auto t = std::dynamic_pointer_cast<SenseNormalToeplitzOp>(s.A);
    if (!t || s.P || t->batched() != first->batched() || t->coils() != first->coils() || t->lambda() != first->lambda())
      fusable = false;
  }
  if (fusable) {
    const auto& bat = *first->batched();
    const auto& plan = *bat.plan();
    const int64_t nv = plan.image_dims()[0] * plan.image_dims()[1] * plan.image_dims()[2];
    std::vector<Vector> bs;
    for (const auto& s : _systems) bs.push_back(s.b);
    Vector ball(bs);
    if (count_systems(x, nv) != (int64_t)_systems.size() && bat.diag_index().size() != (size_t)count_systems(x, nv))
      throw std::runtime_error("each child of x must hold one system");
    ConjugateGradient cg(first, std::make_shared<Vector>(ball), nullptr);
    cg.run(x, iter, tol);
    return;
  }
  for (size_t i = 0; i < _systems.size(); ++i) {
    ConjugateGradient cg(_systems[i].A, std::make_shared<Vector>(_systems[i].b), _systems[i].P);
    cg.run(children[i], iter, tol);
  }
}

}  // namespace op
}  // namespace hasty

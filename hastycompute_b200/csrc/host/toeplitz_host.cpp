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

namespace {
// Device form (real float32, FFT order, on the plan's device) of a preconditioner for the
// fused PCG, or an undefined tensor when P has none (or is absent).
at::Tensor device_precond(const sptr<Operator>& P, const detail::Plan& plan) {
  auto circ = std::dynamic_pointer_cast<mri::CirculantPreconditionerOp>(P);
  if (!circ || !circ->fft_order_diagonal().defined()) return at::Tensor();
  const auto& d = plan.image_dims();
  const at::Tensor& f = circ->fft_order_diagonal();
  if (f.numel() != d[0] * d[1] * d[2]) return at::Tensor();
  return f.to(plan.device(), at::kFloat).contiguous();
}

// The whole (P)CG of every system of x on the device: hb_cg_run_systems with system i's
// diagonal and precond[i] (undefined = plain CG for that system, or one entry for all).
void device_cg(const SenseNormalToeplitzOp& top, Vector& x, const Vector& b, const std::vector<at::Tensor>& precond,
               int iter, double tol, std::vector<int32_t>& status, std::vector<int32_t>& iters) {
  const auto& bat = *top.batched();
  const auto& plan = *bat.plan();
  at::Tensor xs = gather_systems(x, plan);
  at::Tensor bs = gather_systems(b, plan);
  const int64_t nsys = xs.size(0);
  if (bs.size(0) != nsys) throw std::runtime_error("x and b hold different numbers of systems");
  if (precond.size() != 1 && (int64_t)precond.size() != nsys)
    throw std::runtime_error("one preconditioner per system (or one for all) is required");
  const int64_t nv = xs.numel() / std::max<int64_t>(nsys, 1);
  const int64_t pn = plan.packed_numel();
  std::vector<hb_system> sys(nsys);
  for (int64_t i = 0; i < nsys; ++i) {
    const int64_t di = bat.diag_index().empty() ? (nsys == 1 ? 0 : i) : bat.diag_index()[i];
    const at::Tensor& pc = precond.size() == 1 ? precond[0] : precond[i];
    hb_system q{};
    q.x = (char*)xs.data_ptr() + i * nv * 8;
    q.b = (const char*)bs.data_ptr() + i * nv * 8;
    q.smaps = bat.smaps().data_ptr();
    q.coils = top.coils().data();
    q.ncoil = (int64_t)top.coils().size();
    q.packed_diag = bat.packed().data_ptr<float>() + di * pn;
    q.lambda = (float)top.lambda();
    q.precond = pc.defined() ? pc.data_ptr<float>() : nullptr;
    sys[i] = q;
  }
  status.assign(nsys, 0);
  iters.assign(nsys, 0);
  size_t nb = hb_systems_workspace_bytes(plan.get(), nsys, nsys * (int64_t)top.coils().size(), iter);
  at::Tensor ws = plan.workspace(nb);
  int rc = hb_cg_run_systems(plan.get(), nsys, sys.data(), iter, tol, 0, status.data(), iters.data(), ws.data_ptr(),
                             nb, detail::current_stream(plan.device()));
  int64_t off = 0;
  scatter_systems(x, xs, off);
  detail::check(rc);
}
}  // namespace

void ConjugateGradient::run(Vector& x, int iter, double tol) {
  c10::InferenceMode guard;
  if (iter < 1) return;
  auto top = std::dynamic_pointer_cast<SenseNormalToeplitzOp>(_A);
  if (top) {
    at::Tensor pd = device_precond(_P, *top->batched()->plan());
    if (!_P || pd.defined()) {
      device_cg(*top, x, *_b, {pd}, iter, tol, _status, _iters);
      return;
    }
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

}  // namespace op

namespace mri {

namespace {
bool norm_ok(const std::optional<std::string>& n) {
  return !n.has_value() || *n == "backward" || *n == "ortho" || *n == "forward";
}
std::optional<c10::string_view> norm_view(const std::optional<std::string>& n) {
  return n.has_value() ? std::optional<c10::string_view>(c10::string_view(*n)) : std::nullopt;
}
}  // namespace

std::unique_ptr<CirculantPreconditionerOp> CirculantPreconditionerOp::Create(at::Tensor diag, bool centered,
                                                                             const std::optional<std::string>& norm,
                                                                             bool adjointify) {
  return std::unique_ptr<CirculantPreconditionerOp>(
      new CirculantPreconditionerOp(std::move(diag), centered, norm, adjointify));
}

CirculantPreconditionerOp::CirculantPreconditionerOp(at::Tensor diag, bool centered,
                                                     const std::optional<std::string>& norm, bool adjointify)
    : _diag(std::move(diag)), _centered(centered), _norm(norm), _adjointify(adjointify) {
  if (!norm_ok(_norm)) throw std::runtime_error("CirculantPreconditionerOp: unknown norm " + *_norm);
  // the device form: real D over a supported even image size
  at::Tensor d = _diag;
  while (d.dim() > 3 && d.size(0) == 1) d = d.squeeze(0);
  if (d.dim() != 3 || !d.is_cuda()) return;
  if (d.is_complex()) {
    if (at::any(at::imag(d) != 0).item<bool>()) return;
    d = at::real(d);
  }
  if (!hb_size_supported(d.size(0), d.size(1), d.size(2))) return;
  for (int a = 0; a < 3; ++a)
    if (d.size(a) % 2) return;
  if (_centered) d = at::fft_ifftshift(d);
  if (_adjointify) d = at::roll(at::flip(d, {0, 1, 2}), {1, 1, 1}, {0, 1, 2});  // D[-k]
  _fftdiag = d.to(at::kFloat).contiguous();
  _plan = std::make_shared<detail::Plan>(std::vector<int64_t>{d.size(0), d.size(1), d.size(2)}, d.device());
}

op::Vector CirculantPreconditionerOp::apply(const op::Vector& in) const {
  if (in.has_children()) {
    std::vector<op::Vector> out;
    for (const auto& ch : in.children()) out.push_back(apply(ch));
    return op::Vector(out);
  }
  const at::Tensor& x = in.tensor();
  if (_fftdiag.defined() && x.is_cuda() && x.device() == _fftdiag.device() && x.scalar_type() == at::kComplexFloat &&
      x.numel() == _fftdiag.numel()) {
    at::Tensor xc = x.contiguous();
    at::Tensor y = at::empty_like(xc);
    detail::check(hb_precond_apply(_plan->get(), _fftdiag.data_ptr<float>(), xc.data_ptr(), y.data_ptr(),
                                   detail::current_stream(x.device())));
    return op::Vector(y);
  }
  // the reference's own calls (precond.cpp:30-52)
  auto nv = norm_view(_norm);
  auto fftc = [&](const at::Tensor& t) { return at::fft_fftshift(at::fft_fftn(at::fft_ifftshift(t), c10::nullopt, c10::nullopt, nv)); };
  auto ifftc = [&](const at::Tensor& t) { return at::fft_fftshift(at::fft_ifftn(at::fft_ifftshift(t), c10::nullopt, c10::nullopt, nv)); };
  at::Tensor D = _diag.to(x.device());
  if (_adjointify) {
    if (_centered) return op::Vector(fftc(D.conj() * ifftc(x)));
    return op::Vector(at::fft_fftn(D.conj() * at::fft_ifftn(x, c10::nullopt, c10::nullopt, nv), c10::nullopt,
                                   c10::nullopt, nv));
  }
  if (_centered) return op::Vector(ifftc(D * fftc(x)));
  return op::Vector(at::fft_ifftn(D * at::fft_fftn(x, c10::nullopt, c10::nullopt, nv), c10::nullopt, c10::nullopt, nv));
}

at::Tensor CirculantPreconditionerOp::build_diagonal(at::Tensor smaps, at::Tensor coord,
                                                     const std::optional<at::Tensor>& weights,
                                                     const std::optional<double>& lambda) {
  c10::InferenceMode guard;
  if (weights.has_value()) throw std::runtime_error("CirculantPreconditionerOp::build_diagonal: weights not supported");
  if (smaps.dim() != 4) throw std::runtime_error("smaps must be [ncoil, nz, ny, nx]");
  if (coord.dim() != 2 || coord.size(0) != 3) throw std::runtime_error("coord must be [3, nsamples]");
  const c10::Device dev = smaps.is_cuda() ? smaps.device() : c10::Device(c10::kCUDA, 0);
  detail::Plan plan({smaps.size(1), smaps.size(2), smaps.size(3)}, dev);
  at::Tensor sm = smaps.to(dev, at::kComplexFloat).contiguous();
  at::Tensor c = coord.to(dev, at::kFloat).contiguous();
  std::vector<int64_t> coils(smaps.size(0));
  for (int64_t i = 0; i < smaps.size(0); ++i) coils[i] = i;
  at::Tensor p = at::empty({smaps.size(1), smaps.size(2), smaps.size(3)}, at::TensorOptions().dtype(at::kFloat).device(dev));
  detail::check(hb_precond_build(plan.get(), c.data_ptr<float>(), c.size(1), 1e-6, sm.data_ptr(), coils.data(),
                                 (int64_t)coils.size(), (float)lambda.value_or(0.0), p.data_ptr<float>(),
                                 detail::current_stream(dev)));
  return at::fft_fftshift(p);
}

}  // namespace mri

namespace op {

BatchedConjugateGradient::BatchedConjugateGradient(std::vector<ConjugateGradientLoadResult> systems)
    : _systems(std::move(systems)) {}

void BatchedConjugateGradient::run(Vector& x, int iter, double tol) {
  c10::InferenceMode guard;
  auto& children = x.children();
  if (children.size() != _systems.size()) throw std::runtime_error("one load result per child of x is required");
  // fuse every system whose operator shares the first system's batched Toeplitz op; each
  // may carry its own circulant preconditioner (device PCG per system)
  auto first = std::dynamic_pointer_cast<SenseNormalToeplitzOp>(_systems.empty() ? nullptr : _systems[0].A);
  bool fusable = first != nullptr;
  std::vector<at::Tensor> pre;
  for (const auto& s : _systems) {
    auto t = std::dynamic_pointer_cast<SenseNormalToeplitzOp>(s.A);
    if (!t || t->batched() != first->batched() || t->coils() != first->coils() || t->lambda() != first->lambda()) {
      fusable = false;
      break;
    }
    at::Tensor pd = device_precond(s.P, *first->batched()->plan());
    if (s.P && !pd.defined()) {
      fusable = false;
      break;
    }
    pre.push_back(pd);
  }
  if (fusable) {
    const auto& bat = *first->batched();
    const auto& plan = *bat.plan();
    const int64_t nv = plan.image_dims()[0] * plan.image_dims()[1] * plan.image_dims()[2];
    std::vector<Vector> bs;
    for (const auto& s : _systems) bs.push_back(s.b);
    Vector ball(bs);
    const int64_t ns = count_systems(x, nv);
    if (ns != (int64_t)_systems.size()) {
      if (bat.diag_index().size() != (size_t)ns) throw std::runtime_error("each child of x must hold one system");
      for (const auto& t : pre)
        if (t.defined()) throw std::runtime_error("with preconditioners each child of x must hold one system");
      pre = {at::Tensor()};
    }
    std::vector<int32_t> status, iters;
    device_cg(*first, x, ball, pre, iter, tol, status, iters);
    return;
  }
  for (size_t i = 0; i < _systems.size(); ++i) {
    ConjugateGradient cg(_systems[i].A, std::make_shared<Vector>(_systems[i].b), _systems[i].P);
    cg.run(children[i], iter, tol);
  }
}

}  // namespace op
}  // namespace hasty

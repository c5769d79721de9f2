// TorchScript custom classes torch.classes.HastyNufft.* and torch.classes.HastySVT.*, with
// the names, constructors and apply signatures of the reference's FFI
// (python/cpp/py_nufft.cpp:83-107, python/cpp/py_svt.cpp:64-73) so that the reference's
// Python wrappers (hastypy/ffi/hasty_nufft.py, hasty_svt.py) run on this library.  All
// work goes through the C ABI (include/hasty_b200.h); errors surface as RuntimeError.
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <ATen/ATen.h>
#include <torch/csrc/jit/api/compilation_unit.h>
#include <torch/custom_class.h>
#include <torch/jit.h>
#include <torch/library.h>

#include <random>
#include <string>
#include <vector>

#include "hasty_b200.h"

namespace hasty {
namespace ffi {
namespace {

void check(int code) {
  if (code != HB_OK) throw std::runtime_error(std::string(hb_last_error()));
}

void* stream_of(const at::Tensor& t) { return (void*)c10::cuda::getCurrentCUDAStream(t.device().index()).stream(); }

void require_c64_cuda(const at::Tensor& t, const char* name) {
  if (!t.is_cuda() || t.scalar_type() != at::kComplexFloat || !t.is_contiguous())
    throw std::runtime_error(std::string(name) + " must be a contiguous complex64 CUDA tensor");
}

}  // namespace

// NufftOptions(type, positive?, tol?)  (nufft.ixx:26-70; defaults: type 1 positive, type 2
// negative, tol 1e-5)
class NufftOptions : public torch::CustomClassHolder {
 public:
  NufftOptions(int64_t type, const std::optional<bool>& positive, const std::optional<double>& tol) : type(type) {
    if (type != 1 && type != 2) throw std::runtime_error("Only Nufft Type 1 and Type 2 is supported");
    this->positive = positive.has_value() ? *positive : (type == 1);
    this->tol = tol.has_value() ? *tol : 1e-5;
  }
  int64_t type;
  bool positive;
  double tol;
};

// Nufft(coords, nmodes = [ntransf, nz, ny, nx], opts).apply(in, out)  (CUDANufft,
// nufft.cpp:540-767): type 1 maps [ntransf, nfreq] -> nmodes, type 2 the reverse.
class Nufft : public torch::CustomClassHolder {
 public:
  Nufft(const at::Tensor& coords, const std::vector<int64_t>& nmodes, const c10::intrusive_ptr<NufftOptions>& opts)
      : _opts(opts), _nmodes(nmodes) {
    // [ntransf, nz, ny, nx], [ntransf, ny, nx] or [ntransf, nx] (the reference's 3-D, 2-D and
    // 1-D plans) with coords [ndim, nfreq]
    const int64_t d = (int64_t)nmodes.size() - 1;
    if (d < 1 || d > 3) throw std::runtime_error("nmodes must be [ntransf, nz, ny, nx], [ntransf, ny, nx] or [ntransf, nx]");
    if (!coords.is_cuda() || coords.scalar_type() != at::kFloat || coords.dim() != 2 || coords.size(0) != d)
      throw std::runtime_error("Coordinates did not reside in cuda device as float32 [ndim, nfreq]");
    for (int64_t a = 1; a <= d; ++a)
      if (d < 3 && nmodes[a] == 1) throw std::runtime_error("a transformed axis needs more than one mode");
    _coords = coords.contiguous();
    _nfreq = _coords.size(1);
    c10::cuda::CUDAGuard g(_coords.device());
    const int maxbatch = (int)std::max<int64_t>(1, std::min<int64_t>(nmodes[0], 16));
    const int64_t nz = d == 3 ? nmodes[1] : 1, ny = d >= 2 ? nmodes[d - 1] : 1, nx = nmodes[d];
    check(hb_nufft_create(&_plan, nz, ny, nx, _coords.data_ptr<float>(), _nfreq, opts->tol, maxbatch,
                          _coords.device().index(), stream_of(_coords)));
  }
  ~Nufft() override {
    if (_plan) hb_nufft_destroy(_plan);
  }
  void apply(const at::Tensor& in, at::Tensor out) {
    require_c64_cuda(in, "in");
    require_c64_cuda(out, "out");
    c10::cuda::CUDAGuard g(_coords.device());
    const int isign = _opts->positive ? 1 : -1;
    if (_opts->type == 1) {
      if (out.sizes() != at::IntArrayRef(_nmodes)) throw std::runtime_error("out.sizes() must equal nmodes given at construct");
      if (in.sizes() != at::IntArrayRef({_nmodes[0], _nfreq}))
        throw std::runtime_error("in tensor must match ntransf in first dim and nfreq in second dim");
      check(hb_nufft_type1(_plan, in.data_ptr(), out.data_ptr(), _nmodes[0], isign, stream_of(in)));
    } else {
      if (in.sizes() != at::IntArrayRef(_nmodes)) throw std::runtime_error("in.sizes() must equal nmodes given at construct");
      if (out.sizes() != at::IntArrayRef({_nmodes[0], _nfreq}))
        throw std::runtime_error("out tensor must match ntransf in first dim and nfreq in second dim");
      check(hb_nufft_type2(_plan, in.data_ptr(), out.data_ptr(), _nmodes[0], isign, stream_of(in)));
    }
  }

 private:
  c10::intrusive_ptr<NufftOptions> _opts;
  std::vector<int64_t> _nmodes;
  at::Tensor _coords;
  int64_t _nfreq = 0;
  hb_nufft* _plan = nullptr;
};

// FunctionLambda(script, entry, captures).apply(inout) (python/cpp/py_interface.cpp:6-15):
// a TorchScript function compiled from `script`, called as entry(inout, captures).  The
// reference passes it to NufftNormal.apply to act on the k-space data between the two
// transforms.
class FunctionLambda : public torch::CustomClassHolder {
 public:
  FunctionLambda(const std::string& script, const std::string& entry, const std::vector<at::Tensor>& captures)
      : _cunit(torch::jit::compile(script)), _entry(entry), _captures(captures) {}
  void apply(const std::vector<at::Tensor>& inout) const {
    _cunit->run_method(_entry, c10::List<at::Tensor>(inout), c10::List<at::Tensor>(_captures));
  }

 private:
  std::shared_ptr<torch::jit::CompilationUnit> _cunit;
  std::string _entry;
  std::vector<at::Tensor> _captures;
};

// NufftNormal(coords, nmodes, forward_opts, backward_opts).apply(in, out, storage, func_between)
// (CUDANufftNormal, nufft.cpp:785-920; binding py_nufft.cpp:96-107): out = backward(f(forward(in))),
// storage [ntransf, nfreq] holds the k-space data in between and f, when given, is a
// FunctionLambda applied to it in place (the identity otherwise).
class NufftNormal : public torch::CustomClassHolder {
 public:
  NufftNormal(const at::Tensor& coords, const std::vector<int64_t>& nmodes,
              const c10::intrusive_ptr<NufftOptions>& fwd, const c10::intrusive_ptr<NufftOptions>& bwd)
      : _fwd(c10::make_intrusive<Nufft>(coords, nmodes, fwd)), _bwd(c10::make_intrusive<Nufft>(coords, nmodes, bwd)) {
    if (fwd->type != 2 || bwd->type != 1) throw std::runtime_error("NufftNormal needs a type-2 forward and a type-1 backward");
  }
  void apply(const at::Tensor& in, at::Tensor out, at::Tensor storage,
             const std::optional<c10::intrusive_ptr<FunctionLambda>>& func_between) {
    _fwd->apply(in, storage);
    if (func_between.has_value() && *func_between) (*func_between)->apply({storage});
    _bwd->apply(storage, out);
  }

 private:
  c10::intrusive_ptr<Nufft> _fwd, _bwd;
};

// ---- block SVT (svt.cpp:268-490) ----
namespace {

// Greedy partition into waves of non-overlapping blocks (one voxel-occupancy grid per wave)
std::vector<std::vector<int32_t>> waves_of(const std::vector<std::array<int64_t, 3>>& corners,
                                           const std::array<int64_t, 3>& b, const std::array<int64_t, 3>& S) {
  std::vector<std::vector<int32_t>> waves;
  std::vector<std::vector<char>> occ;
  const int64_t vol = S[0] * S[1] * S[2];
  for (const auto& c : corners) {
    size_t w = 0;
    for (; w < waves.size(); ++w) {
      bool free = true;
      for (int64_t i = 0; i < b[0] && free; ++i)
        for (int64_t j = 0; j < b[1] && free; ++j)
          for (int64_t k = 0; k < b[2] && free; ++k)
            if (occ[w][((c[0] + i) * S[1] + c[1] + j) * S[2] + c[2] + k]) free = false;
      if (free) break;
    }
    if (w == waves.size()) {
      waves.emplace_back();
      occ.emplace_back(vol, 0);
    }
    for (int64_t i = 0; i < b[0]; ++i)
      for (int64_t j = 0; j < b[1]; ++j)
        for (int64_t k = 0; k < b[2]; ++k) occ[w][((c[0] + i) * S[1] + c[1] + j) * S[2] + c[2] + k] = 1;
    waves[w].insert(waves[w].end(), {(int32_t)c[0], (int32_t)c[1], (int32_t)c[2]});
  }
  return waves;
}

// Thresholds the blocks of every wave of `in` [d0, d1, S0, S1, S2] (a CPU tensor is moved
// to the current CUDA device and back, as the reference moves its blocks).
void run_waves(at::Tensor in, const std::vector<std::vector<int32_t>>& waves, const std::array<int64_t, 3>& b,
               double thresh, bool soft) {
  if (in.dim() != 5 || in.scalar_type() != at::kComplexFloat)
    throw std::runtime_error("SVT input must be complex64 [d0, d1, S0, S1, S2]");
  at::Tensor work = in.is_cuda() ? in : in.to(at::Device(at::kCUDA, c10::cuda::current_device()));
  if (!work.is_contiguous()) work = work.contiguous();
  c10::cuda::CUDAGuard g(work.device());
  for (const auto& w : waves) {
    at::Tensor c = at::from_blob((void*)w.data(), {(int64_t)w.size()}, at::kInt).to(work.device());
    check(hb_svt_blocks(work.data_ptr(), work.size(0), work.size(1), work.size(2), work.size(3), work.size(4), b[0],
                        b[1], b[2], c.data_ptr<int32_t>(), (int64_t)w.size() / 3, thresh, soft ? 1 : 0,
                        stream_of(work)));
  }
  if (!work.is_same(in)) in.copy_(work);
}

}  // namespace

class Random3DBlocksSVT : public torch::CustomClassHolder {
 public:
  explicit Random3DBlocksSVT(const std::optional<std::vector<at::Stream>>&) {}
  void apply(at::Tensor in, int64_t nblocks, const std::vector<int64_t>& block_shape, double thresh, bool soft) {
    if (block_shape.size() != 3 || in.dim() != 5) throw std::runtime_error("3-D blocks of a 5-D input expected");
    const std::array<int64_t, 3> b{block_shape[0], block_shape[1], block_shape[2]};
    const std::array<int64_t, 3> S{in.size(2), in.size(3), in.size(4)};
    std::vector<std::array<int64_t, 3>> corners;
    for (int64_t i = 0; i < nblocks; ++i) {
      std::array<int64_t, 3> c{};
      for (int d = 0; d < 3; ++d) c[d] = std::uniform_int_distribution<int64_t>(0, S[d] - b[d])(_gen);
      corners.push_back(c);
    }
    run_waves(in, waves_of(corners, b, S), b, thresh, soft);
  }

 private:
  std::mt19937_64 _gen{0x5eed};
};

class Normal3DBlocksSVT : public torch::CustomClassHolder {
 public:
  explicit Normal3DBlocksSVT(const std::optional<std::vector<at::Stream>>&) {}
  void apply(at::Tensor in, const std::vector<int64_t>& block_strides, const std::vector<int64_t>& block_shape,
             int64_t block_iter, double thresh, bool soft) {
    if (block_iter < 1) throw std::runtime_error("Can't perform Normal3DBlocksSVT with block_iter < 1");
    if (block_shape.size() != 3 || block_strides.size() != 3 || in.dim() != 5)
      throw std::runtime_error("3-D blocks of a 5-D input expected");
    const std::array<int64_t, 3> b{block_shape[0], block_shape[1], block_shape[2]};
    const std::array<int64_t, 3> S{in.size(2), in.size(3), in.size(4)};
    for (int64_t it = 0; it < block_iter; ++it) {
      int64_t sh[3] = {0, 0, 0};
      if (it > 0)
        for (int d = 0; d < 3; ++d) sh[d] = std::uniform_int_distribution<int64_t>(0, b[d])(_gen);
      std::vector<std::array<int64_t, 3>> corners;
      for (int64_t n0 = 0; n0 < S[0] / block_strides[0]; ++n0) {
        const int64_t s0 = n0 * block_strides[0] + sh[0];
        if (s0 + b[0] >= S[0]) continue;  // a block ending on the last index is skipped, svt.cpp:395-420
        for (int64_t n1 = 0; n1 < S[1] / block_strides[1]; ++n1) {
          const int64_t s1 = n1 * block_strides[1] + sh[1];
          if (s1 + b[1] >= S[1]) continue;
          for (int64_t n2 = 0; n2 < S[2] / block_strides[2]; ++n2) {
            const int64_t s2 = n2 * block_strides[2] + sh[2];
            if (s2 + b[2] >= S[2]) continue;
            corners.push_back({s0, s1, s2});
          }
        }
      }
      run_waves(in, waves_of(corners, b, S), b, thresh, soft);
    }
  }

 private:
  std::mt19937_64 _gen{0x5eed};
};

}  // namespace ffi
}  // namespace hasty

// registered first: NufftNormal.apply takes a FunctionLambda (static initialisation runs in
// definition order within this file)
TORCH_LIBRARY(HastyInterface, hi) {
  hi.class_<hasty::ffi::FunctionLambda>("FunctionLambda")
      .def(torch::init<const std::string&, const std::string&, const std::vector<at::Tensor>&>())
      .def("apply", &hasty::ffi::FunctionLambda::apply);
}

TORCH_LIBRARY(HastyNufft, hn) {
  hn.class_<hasty::ffi::NufftOptions>("NufftOptions")
      .def(torch::init<int64_t, const std::optional<bool>&, const std::optional<double>&>());
  hn.class_<hasty::ffi::Nufft>("Nufft")
      .def(torch::init<const at::Tensor&, const std::vector<int64_t>&,
                       const c10::intrusive_ptr<hasty::ffi::NufftOptions>&>())
      .def("apply", &hasty::ffi::Nufft::apply);
  hn.class_<hasty::ffi::NufftNormal>("NufftNormal")
      .def(torch::init<const at::Tensor&, const std::vector<int64_t>&, const c10::intrusive_ptr<hasty::ffi::NufftOptions>&,
                       const c10::intrusive_ptr<hasty::ffi::NufftOptions>&>())
      .def("apply", &hasty::ffi::NufftNormal::apply);
}

TORCH_LIBRARY(HastySVT, hsvt) {
  hsvt.class_<hasty::ffi::Random3DBlocksSVT>("Random3DBlocksSVT")
      .def(torch::init<const std::optional<std::vector<at::Stream>>&>())
      .def("apply", &hasty::ffi::Random3DBlocksSVT::apply);
  hsvt.class_<hasty::ffi::Normal3DBlocksSVT>("Normal3DBlocksSVT")
      .def(torch::init<const std::optional<std::vector<at::Stream>>&>())
      .def("apply", &hasty::ffi::Normal3DBlocksSVT::apply);
}

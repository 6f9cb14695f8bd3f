// Drives the reference's own CUDA restriction (src/cuda/cuda-elem-restriction.cu,
// include/cuda/cuda-elem-restriction.hpp) through its public API, for the GPU
// baseline of the restriction stages and bitwise parity checks.  Test and
// benchmark infrastructure only: built by `make -C oracle refcuda` into
// oracle/_ref/libfemrefcuda.so, from the reference sources where they lie.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "cuda/cuda-elem-restriction.hpp"
#include "elem-restriction.hpp"

namespace {
thread_local std::string g_err;

struct Handle {
  fem::cuda::ElemRestriction r;
  fem::cuda::DeviceArray<double> l, e;  // an L-vector and an E-vector the applies read and write
};

template <class F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return 1;
  }
}
}  // namespace

extern "C" {

const char* refcuda_last_error() { return g_err.c_str(); }

// A device restriction from host offsets (deterministic != 0: the reference's
// transpose-map scatter), with its L- and E-vectors allocated.
int refcuda_create(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size, const int* offsets,
                   int deterministic, void** out) {
  return guarded([&] {
    fem::ElemRestriction host;
    fem::elem_restriction_create(num_elem, elem_size, num_comp, comp_stride, l_size,
                                 std::vector<int>(offsets, offsets + int64_t(num_elem) * elem_size), host);
    auto* h = new Handle;
    try {
      fem::cuda::elem_restriction_create(
          host, deterministic ? fem::cuda::ScatterMode::Deterministic : fem::cuda::ScatterMode::Atomic, h->r);
      h->l.resize(size_t(h->r.l_size));
      h->e.resize(size_t(h->r.e_size));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int refcuda_set_l(void* h, const double* host) {
  return guarded([&] {
    auto* p = static_cast<Handle*>(h);
    p->l.copy_from_host(std::vector<double>(host, host + p->l.size()));
  });
}

int refcuda_set_e(void* h, const double* host) {
  return guarded([&] {
    auto* p = static_cast<Handle*>(h);
    p->e.copy_from_host(std::vector<double>(host, host + p->e.size()));
  });
}

int refcuda_zero_l(void* h) {
  return guarded([&] { static_cast<Handle*>(h)->l.zero(); });
}

// NoTranspose: e = gather(l).  Transpose: l += scatter(e).  Asynchronous
// (the reference launches on the default stream).
int refcuda_apply(void* h, int transpose) {
  return guarded([&] {
    auto* p = static_cast<Handle*>(h);
    if (transpose)
      fem::cuda::elem_restriction_apply(p->r, fem::ContractMode::Transpose, p->e, p->l);
    else
      fem::cuda::elem_restriction_apply(p->r, fem::ContractMode::NoTranspose, p->l, p->e);
  });
}

int refcuda_get_l(void* h, double* host) {
  return guarded([&] {
    auto* p = static_cast<Handle*>(h);
    std::vector<double> v;
    p->l.copy_to_host(v);
    std::memcpy(host, v.data(), v.size() * sizeof(double));
  });
}

int refcuda_get_e(void* h, double* host) {
  return guarded([&] {
    auto* p = static_cast<Handle*>(h);
    std::vector<double> v;
    p->e.copy_to_host(v);
    std::memcpy(host, v.data(), v.size() * sizeof(double));
  });
}

int refcuda_sizes(void* h, int64_t* l_size, int64_t* e_size) {
  return guarded([&] {
    auto* p = static_cast<Handle*>(h);
    *l_size = int64_t(p->l.size());
    *e_size = int64_t(p->e.size());
  });
}

int refcuda_destroy(void* h) {
  return guarded([&] { delete static_cast<Handle*>(h); });
}

}  // extern "C"

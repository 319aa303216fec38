// common.hpp -- status codes, CUDA error plumbing and device buffers.
//
// Every public entry point returns an int status and never exits the process
// (the reference prints and calls exit(); see src/block_tensor_inst.cpp:233-246).
#pragma once
#include <cuda_runtime.h>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sadmrg.h"

namespace sadmrg {

using dcmplex = std::complex<double>;

// Status codes are the C ABI's (include/sadmrg.h): SADMRG_OK, SADMRG_ERR_*.

// Exception type used internally; converted to a status at the C boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define SADMRG_CUDA(call)                                                         \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      throw ::sadmrg::Error(SADMRG_ERR_CUDA,                            \
                            std::string(#call " -> ") + cudaGetErrorString(e_)); \
  } while (0)

#define SADMRG_REQUIRE(cond, code, msg)                     \
  do {                                                      \
    if (!(cond)) throw ::sadmrg::Error((code), (msg));      \
  } while (0)

template <class S> struct ScalarInfo;
template <> struct ScalarInfo<double> { static constexpr bool cplx = false; };
template <> struct ScalarInfo<dcmplex> { static constexpr bool cplx = true; };

inline double real_of(double x) { return x; }
inline double real_of(dcmplex x) { return x.real(); }
inline double conj_of(double x) { return x; }
inline dcmplex conj_of(dcmplex x) { return std::conj(x); }

// Stream-ordered device buffer (cudaMallocAsync on the owning stream).
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t s) { alloc(bytes, s); }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p_ = o.p_; n_ = o.n_; s_ = o.s_; o.p_ = nullptr; o.n_ = 0; }
    return *this;
  }
  void alloc(size_t bytes, cudaStream_t s) {
    release();
    s_ = s;
    n_ = bytes;
    if (bytes == 0) return;
    cudaError_t e = cudaMallocAsync(&p_, bytes, s);
    if (e != cudaSuccess) {
      p_ = nullptr; n_ = 0;
      throw Error(SADMRG_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    }
  }
  void release() {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr; n_ = 0;
  }
  void* get() const { return p_; }
  size_t bytes() const { return n_; }
  template <class T> T* as() const { return static_cast<T*>(p_); }

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};

}  // namespace sadmrg

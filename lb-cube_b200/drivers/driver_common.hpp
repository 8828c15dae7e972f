// Shared pieces of the engine's ports of LB-Cube's two drivers (lbm_sim,
// lbm_reaction_sim): command-line helpers with the reference drivers' checks
// and messages (src/main.cpp:75-196, src/simulate_reaction.cpp:87-166), device
// buffers owned by the driver, and a kernel timer.
//
// The ports call only the engine's C ABI (include/lbcube_b200.h) and the CUDA
// runtime. They run on the GPU only.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lbcube_b200.h"

namespace lbport {

inline void check_cuda(cudaError_t error, const std::string& context) {
  if (error != cudaSuccess) throw std::runtime_error(context + ": " + cudaGetErrorString(error));
}

// An engine call's cudaError_t (returned as int).
inline void check_engine(int code, const std::string& context) {
  check_cuda(static_cast<cudaError_t>(code), context);
}

inline std::size_t parse_size_arg(const std::vector<std::string>& args, std::size_t& i) {
  if (i + 1 >= args.size()) throw std::invalid_argument("missing value for " + args[i]);
  const std::size_t value = std::stoull(args[++i]);
  if (value == 0) throw std::invalid_argument(args[i - 1] + " must be greater than zero");
  return value;
}

inline int parse_int_arg(const std::vector<std::string>& args, std::size_t& i) {
  if (i + 1 >= args.size()) throw std::invalid_argument("missing value for " + args[i]);
  return std::stoi(args[++i]);
}

inline double parse_real_arg(const std::vector<std::string>& args, std::size_t& i) {
  if (i + 1 >= args.size()) throw std::invalid_argument("missing value for " + args[i]);
  return std::stod(args[++i]);
}

// "-cpu" selects the reference's CPU path, which this port does not carry.
inline void reject_cpu() {
  throw std::invalid_argument(
      "this port runs the engine on the GPU only; the CPU path is the reference's own driver");
}

// A device array owned by the driver (the engine's launchers never allocate).
template <class T>
class DeviceArray {
 public:
  explicit DeviceArray(std::size_t count) : count_(count) {
    check_cuda(cudaMalloc(reinterpret_cast<void**>(&ptr_), count * sizeof(T)), "cudaMalloc");
  }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { cudaFree(ptr_); }
  T* get() const { return ptr_; }
  std::size_t count() const { return count_; }
  std::size_t bytes() const { return count_ * sizeof(T); }
  void upload(const std::vector<T>& host) {
    check_cuda(cudaMemcpy(ptr_, host.data(), bytes(), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  }
  std::vector<T> download(std::size_t count) const {
    std::vector<T> host(count);
    check_cuda(cudaMemcpy(host.data(), ptr_, count * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
    return host;
  }

 private:
  T* ptr_{};
  std::size_t count_{};
};

// Device time of the stepping launches only: CUDA events bracket each run of
// steps between two outputs on the driver's stream.
class KernelTimer {
 public:
  explicit KernelTimer(cudaStream_t s) : stream_(s) {
    check_cuda(cudaEventCreate(&start_), "cudaEventCreate");
    check_cuda(cudaEventCreate(&stop_), "cudaEventCreate");
  }
  KernelTimer(const KernelTimer&) = delete;
  KernelTimer& operator=(const KernelTimer&) = delete;
  ~KernelTimer() {
    cudaEventDestroy(start_);
    cudaEventDestroy(stop_);
  }
  void begin() { check_cuda(cudaEventRecord(start_, stream_), "cudaEventRecord"); }
  void end() {
    check_cuda(cudaEventRecord(stop_, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(stop_), "cudaEventSynchronize");
    float ms = 0.0f;
    check_cuda(cudaEventElapsedTime(&ms, start_, stop_), "cudaEventElapsedTime");
    seconds_ += 1e-3 * static_cast<double>(ms);
  }
  double seconds() const { return seconds_; }

 private:
  cudaStream_t stream_;
  cudaEvent_t start_{}, stop_{};
  double seconds_ = 0.0;
};

}  // namespace lbport

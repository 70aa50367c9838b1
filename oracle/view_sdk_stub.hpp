// view_sdk_stub.hpp - test infrastructure: just enough of the Holoscan SDK's
// declarations for the reference demo's view operator
// (applications/isp/src/view_op.cu, view_op.hpp) to compile, so that its
// view kernel can be built from its own source and run beside this
// library's (view_ref_shim.cu). The operator around the kernel compiles
// against these stubs but never runs: none of them does anything. The names
// and shapes are the ones that source uses (the SDK itself is not present
// here); nothing else is declared.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

// DLPack's type descriptor, as the SDK's headers bring it in.
struct DLDataType {
  std::uint8_t code;
  std::uint8_t bits;
  std::uint16_t lanes;
};
enum DLDataTypeCode : std::uint8_t { kDLInt = 0, kDLUInt = 1, kDLFloat = 2 };

namespace holoscan {

enum class ErrorCode { kInvalidArgument, kFailure };
struct Error {
  ErrorCode code{};
  std::string message;
};

template <class E>
struct unexpected {
  E error;
};
template <class E>
unexpected<std::decay_t<E>> make_unexpected(E&& e) {
  return {std::forward<E>(e)};
}

template <class T, class E>
class expected {
 public:
  expected() = default;
  expected(T v) : v_(std::move(v)), ok_(true) {}
  template <class G>
  expected(unexpected<G> u) : e_(std::move(u.error)) {}
  explicit operator bool() const { return ok_; }
  T* operator->() { return &v_; }
  const T* operator->() const { return &v_; }
  T& operator*() & { return v_; }
  T&& operator*() && { return std::move(v_); }
  E error() && { return std::move(e_); }

 private:
  T v_{};
  E e_{};
  bool ok_ = false;
};

template <class E>
class expected<void, E> {
 public:
  expected() = default;
  template <class G>
  expected(unexpected<G> u) : e_(std::move(u.error)), ok_(false) {}
  explicit operator bool() const { return ok_; }
  E error() && { return std::move(e_); }

 private:
  E e_{};
  bool ok_ = true;
};

namespace schema {
enum ImageEncoding { ImageEncoding_RGB8 = 0, ImageEncoding_RAW = 1 };
struct Tensor {
  const std::int64_t* strides() const { return nullptr; }
  void* data() const { return nullptr; }
  template <class T>
  T* data_as() const {
    return nullptr;
  }
};
struct ImageT {
  std::shared_ptr<Tensor> data;
  int width = 0;
  int height = 0;
  ImageEncoding encoding = ImageEncoding_RGB8;
};
}  // namespace schema

enum class MemoryKind { kHost, kCudaDevice };
enum class TensorStridePolicy { kContiguousOnly };
enum class TensorOutputStorage { kRuntimePool };
struct TensorRepresentation {
  MemoryKind memory_kind{};
  DLDataType dtype{};
  unsigned rank = 0;
  TensorStridePolicy strides{};
};
struct TensorBounds {
  std::uint64_t bytes = 0;
};
inline TensorBounds tensor_bounds(std::uint64_t bytes) { return {bytes}; }
struct TensorOutputSpec {
  TensorRepresentation representation;
  TensorBounds bounds;
  TensorOutputStorage storage{};
};
struct SchemaId {
  const char* name = "";
};
template <class T>
SchemaId schema_identity() {
  return {};
}
struct PayloadOptions {
  SchemaId schema;
};

struct OutputSpec {
  OutputSpec& produces_tensor(const TensorOutputSpec&) { return *this; }
  OutputSpec& payload_options(const PayloadOptions&) { return *this; }
};
struct OperatorSpec {
  template <class P>
  void input(P&, const char*) {}
  template <class P>
  OutputSpec output(P&, const char*) {
    return {};
  }
};

struct CudaStreamRef {
  cudaStream_t get() const { return nullptr; }
};
struct ExecutionContext {
  CudaStreamRef cuda_stream() const { return {}; }
};

template <class T>
struct Sample {
  T data;
};

namespace sensor_io {
struct Provenance {};
template <class T>
Provenance derive_from(const Sample<T>&) {
  return {};
}
}  // namespace sensor_io

struct TensorWriter {
  template <class T>
  T* data_as() const {
    return nullptr;
  }
  expected<void, Error> commit() && { return {}; }
};
struct TensorLoan {
  expected<TensorWriter, Error> write(cudaStream_t) { return TensorWriter{}; }
};
struct TensorLoanRequest {
  std::array<std::int64_t, 3> shape{};
  DLDataType dtype{};
};

template <class T>
struct Input {
  expected<Sample<T>, Error> receive() { return Sample<T>{}; }
};
template <class T>
struct Output {
  expected<TensorLoan, Error> allocate_tensor(const TensorLoanRequest&) { return TensorLoan{}; }
  expected<void, Error> emit_tensor(TensorLoan, T, sensor_io::Provenance) { return {}; }
};

struct PortRef {
  template <class T>
  PortRef(const Input<T>&) {}
};
struct PortList {
  std::vector<PortRef> ports;
};
struct OnAligned {
  PortList ports;
  std::chrono::nanoseconds window{};
};
struct Exact {};
struct Contract {
  void trigger(const OnAligned&) {}
  template <class P>
  void input(P&, const Exact&) {}
};

template <class... Ts>
class Operator {
 public:
  virtual ~Operator() = default;
  virtual void setup(OperatorSpec&) {}
  virtual Contract contract() const { return {}; }
  virtual expected<void, Error> compute(ExecutionContext&) { return {}; }
};

}  // namespace holoscan

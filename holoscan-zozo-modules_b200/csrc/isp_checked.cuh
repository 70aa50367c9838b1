// isp_checked.cuh - the pointers of the ISP kernels, and their bounds-checked
// form (the ISP_CHECKED build).
//
// Every shared- and global-memory array the ISP kernels index (the frame's
// raw samples, output rows, tables, histograms, scratch, and each region of a
// CTA's shared memory) is held as a Span<T>. In the regular build Span<T> is
// T*, so the code compiles to exactly what it would with plain pointers. With
// ISP_CHECKED defined (libisp_b200_checked.so) a Span carries the bytes it may
// touch, and every access through it (p[i], *p, p->f, a vector view of it,
// the destination of a copy into it) is checked first: an access outside
// them is not made (a store goes to a sink, a load reads the sink), and the
// violation is counted in device memory with the first offending address,
// where isp_b200_checked_violations() reads and clears it (the record lives
// in the pipeline's scratch, so it needs no allocation of its own). Nothing
// traps.
// This is the stand-in for running the reference's tests under
// compute-sanitizer (modules/isp/tests/CMakeLists.txt:34-50).
#pragma once

#include <cstddef>
#include <cstdint>
#include <type_traits>

namespace isp_b200 {

#ifdef ISP_CHECKED

// Violations since the last read, in a pipeline's scratch (Scratch::check):
// their count, the first one's address, size and bounds, and the sink that
// refused accesses use (16-byte aligned; the widest access is 16 bytes).
struct CheckRecord {
  unsigned int count;
  unsigned int bytes;
  unsigned long long address;
  unsigned long long lo;
  unsigned long long hi;
  uint4 sink[16];
};

// The record of spans built without one (Span(nullptr)): an access through
// such a span is refused and counted here rather than dereferencing null.
static __device__ CheckRecord g_unowned_check;

static __device__ __noinline__ CheckRecord* check_failed(CheckRecord* rec, const void* at, size_t bytes,
                                                         const void* lo, const void* hi) {
  if (rec == nullptr) rec = &g_unowned_check;
  if (atomicAdd(&rec->count, 1U) == 0U) {
    rec->bytes = static_cast<unsigned int>(bytes);
    rec->address = reinterpret_cast<unsigned long long>(at);
    rec->lo = reinterpret_cast<unsigned long long>(lo);
    rec->hi = reinterpret_cast<unsigned long long>(hi);
  }
  return rec;
}

// The check of one access, out of line: each access adds a call rather than
// a branch to the (fully inlined) kernels, which keeps the checked build's
// compile time near the regular build's. Returns the address to use.
static __device__ __noinline__ void* check_access(const void* q, size_t bytes, const char* lo, const char* hi,
                                                  CheckRecord* rec) {
  const char* c = static_cast<const char*>(q);
  if (c < lo || c + bytes > hi || c + bytes < c) return check_failed(rec, q, bytes, lo, hi)->sink;
  return const_cast<void*>(q);
}

template <class T>
struct Span {
  T* p;
  const char* lo;  // the bytes [lo, hi) may be accessed
  const char* hi;
  CheckRecord* rec;  // where violations are counted

  Span() = default;
  __host__ __device__ Span(std::nullptr_t) : p(nullptr), lo(nullptr), hi(nullptr), rec(nullptr) {}
  __host__ __device__ Span(T* ptr, const void* lo_, const void* hi_, CheckRecord* r)
      : p(ptr), lo(static_cast<const char*>(lo_)), hi(static_cast<const char*>(hi_)), rec(r) {}
  template <class U, class = std::enable_if_t<std::is_convertible<U*, T*>::value>>
  __host__ __device__ Span(const Span<U>& o) : p(o.p), lo(o.lo), hi(o.hi), rec(o.rec) {}

  // The address of `bytes` bytes at q, or of the sink when they fall outside.
  __device__ __forceinline__ T* at(T* q, size_t bytes) const {
    return static_cast<T*>(check_access(q, bytes, lo, hi, rec));
  }
  __device__ __forceinline__ T& operator[](ptrdiff_t i) const { return *at(p + i, sizeof(T)); }
  __device__ __forceinline__ T& operator*() const { return *at(p, sizeof(T)); }
  __device__ __forceinline__ T* operator->() const { return at(p, sizeof(T)); }
  __host__ __device__ Span operator+(ptrdiff_t i) const { return Span(p + i, lo, hi, rec); }
  __host__ __device__ Span operator-(ptrdiff_t i) const { return Span(p - i, lo, hi, rec); }
  __host__ __device__ Span& operator+=(ptrdiff_t i) {
    p += i;
    return *this;
  }
  __host__ __device__ bool operator==(std::nullptr_t) const { return p == nullptr; }
  __host__ __device__ bool operator!=(std::nullptr_t) const { return p != nullptr; }
};

// A Span over `count` elements at ptr, counting into rec. A null ptr gives a
// null span that still counts into rec: an access through it is refused and
// reported like any other.
template <class T>
__host__ __device__ inline Span<T> make_span(T* ptr, size_t count, CheckRecord* rec) {
  return ptr == nullptr ? Span<T>(nullptr, nullptr, nullptr, rec) : Span<T>(ptr, ptr, ptr + count, rec);
}
// The same bytes viewed as U (for vector loads and stores, and carving).
template <class U, class T>
__host__ __device__ inline Span<U> span_cast(const Span<T>& s) {
  return Span<U>(reinterpret_cast<U*>(s.p), s.lo, s.hi, s.rec);
}
// The address of `count` elements at s, checked (for copies the hardware
// makes: TMA boxes, cp.async); the sink when they fall outside.
template <class T>
__device__ __forceinline__ T* span_range(const Span<T>& s, size_t count) {
  return s.at(s.p, count * sizeof(T));
}
// The unchecked address (comparisons, and addresses that are not accessed).
template <class T>
__host__ __device__ inline T* span_ptr(const Span<T>& s) {
  return s.p;
}
// Where a span counts its violations.
template <class T>
__host__ __device__ inline CheckRecord* span_rec(const Span<T>& s) {
  return s.rec;
}
// `count` elements at ptr, a part of what `parent` covers (an array member
// of the object a span points to), counting where the parent counts.
template <class T, class U>
__host__ __device__ inline Span<T> sub_span(const Span<U>& parent, T* ptr, size_t count) {
  return Span<T>(ptr, ptr, ptr + count, parent.rec);
}
// `bytes` bytes at byte `offset` of a CTA's shared memory, as T.
template <class T>
__device__ __forceinline__ Span<T> carve_span(unsigned char* base, int offset, int bytes, CheckRecord* rec) {
  return Span<T>(reinterpret_cast<T*>(base + offset), base + offset, base + offset + bytes, rec);
}

#else

template <class T>
using Span = T*;

struct CheckRecord;

template <class T>
__host__ __device__ inline T* make_span(T* ptr, size_t, CheckRecord*) {
  return ptr;
}
template <class U, class T>
__host__ __device__ inline U* span_cast(T* p) {
  return reinterpret_cast<U*>(p);
}
template <class T>
__device__ __forceinline__ T* span_range(T* p, size_t) {
  return p;
}
template <class T>
__host__ __device__ inline T* span_ptr(T* p) {
  return p;
}
template <class T>
__host__ __device__ inline CheckRecord* span_rec(T*) {
  return nullptr;
}
template <class T, class U>
__host__ __device__ inline T* sub_span(U*, T* ptr, size_t) {
  return ptr;
}
template <class T>
__device__ __forceinline__ T* carve_span(unsigned char* base, int offset, int, CheckRecord*) {
  return reinterpret_cast<T*>(base + offset);
}

#endif

}  // namespace isp_b200

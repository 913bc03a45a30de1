// Stand-in for the reference's model/main_header.h and the parts of YAKL and
// Kokkos that the reference dynamical core uses (TEST INFRASTRUCTURE ONLY).
//
// The reference's dycore headers (model/modules/dynamics_rk.h,
// helpers/WenoLimiter.h, helpers/TransformMatrices.h and core/MultipleFields.h)
// are compiled unchanged against this file, from where they lie, by the
// `ref` target of oracle/Makefile.  Their external dependencies (YAKL, Kokkos, MPI,
// PNetCDF, yaml-cpp) are empty submodules in the reference tree, so this shim
// supplies, for one host process:
//   * yakl::SArray     -- fixed-size array, C order, (i,j,...) indexing
//   * yakl::Array      -- reference-counted C-order N-d array with views
//   * yakl::c::parallel_for over SimpleBounds (OpenMP on the host cores)
//   * yakl::intrinsics::matmul_cr (column-row matrix products) and sum
//   * no-op timers and a no-op SimplePNetCDF (output hooks are registered,
//     never called)
//   * Kokkos::abort / endrun throwing std::runtime_error.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <typeinfo>
#include <vector>

#define KOKKOS_INLINE_FUNCTION inline
#define YAKL_INLINE inline
#define KOKKOS_LAMBDA [=]
#define YAKL_LAMBDA [=]
#define YAKL_AUTO_LABEL() "porturb_ref_shim"

typedef double real;
inline constexpr real operator"" _fp(long double x) { return static_cast<real>(x); }
int constexpr max_fields = 50;

typedef long long MPI_Offset;
typedef int MPI_Op;
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

namespace Kokkos {
inline void abort(const char *msg) { throw std::runtime_error(std::string("Kokkos::abort: ") + msg); }
inline void fence() {}
// One thread: the atomic add is a plain add, in the loop's index order.
template <class T>
inline void atomic_add(T *dst, T v) { *dst += v; }
}  // namespace Kokkos

// A local name for a member the kernel lambda captures by value in yakl.
#define YAKL_SCOPE(local, expr) auto &local = expr

inline void endrun(std::string msg = "") { throw std::runtime_error("endrun: " + msg); }

namespace yakl {

int constexpr memDevice = 1;
int constexpr memHost = 2;
int constexpr styleC = 1;

struct Colon {};
Colon constexpr COLON{};

inline void timer_start(const char *) {}
inline void timer_stop(const char *) {}

// ---------------------------------------------------------------------------
template <class T, int RANK, size_t D0, size_t D1 = 1, size_t D2 = 1, size_t D3 = 1>
class SArray {
 public:
  T myData[D0 * D1 * D2 * D3];
  SArray() = default;
  SArray(T v) { for (auto &x : myData) x = v; }
  SArray &operator=(T v) { for (auto &x : myData) x = v; return *this; }
  // Like YAKL, element access is a const member returning a mutable
  // reference (MultipleFields.h relies on this).
  T &operator()(unsigned i0) const { return at(i0); }
  T &operator()(unsigned i0, unsigned i1) const { return at(i0 * D1 + i1); }
  T &operator()(unsigned i0, unsigned i1, unsigned i2) const { return at((i0 * D1 + i1) * D2 + i2); }
  T &operator()(unsigned i0, unsigned i1, unsigned i2, unsigned i3) const { return at(((i0 * D1 + i1) * D2 + i2) * D3 + i3); }
  T &at(unsigned i) const { return const_cast<T &>(myData[i]); }
  static int constexpr get_rank() { return RANK; }
  static size_t constexpr size() { return D0 * D1 * D2 * D3; }
  T *data() { return myData; }
};

// ---------------------------------------------------------------------------
template <class T, int RANK, int MEM, int STYLE>
class Array {
 public:
  typedef typename std::remove_cv<T>::type type;
  std::shared_ptr<type> owner;
  type *ptr = nullptr;
  size_t dims[RANK > 0 ? RANK : 1] = {};
  std::string myname;

  Array() = default;
  template <class... I>
  Array(const char *label, I... d) {
    static_assert(sizeof...(I) == RANK, "wrong number of dimensions");
    myname = label;
    size_t v[] = {size_t(d)...};
    for (int i = 0; i < RANK; i++) dims[i] = v[i];
    allocate();
  }
  Array(const char *label, std::vector<int> const &d) {
    myname = label;
    for (int i = 0; i < RANK; i++) dims[i] = d[i];
    allocate();
  }
  void allocate() {
    size_t n = size();
    owner = std::shared_ptr<type>(new type[n > 0 ? n : 1](), std::default_delete<type[]>());
    ptr = owner.get();
  }
  // Conversion from the non-const to the const element type.
  template <class U, typename = typename std::enable_if<std::is_same<typename std::remove_cv<U>::type, type>::value &&
                                                        !std::is_same<U, T>::value>::type>
  Array(Array<U, RANK, MEM, STYLE> const &rhs) : owner(rhs.owner), ptr(rhs.ptr), myname(rhs.myname) {
    for (int i = 0; i < RANK; i++) dims[i] = rhs.dims[i];
  }

  size_t size() const { size_t n = 1; for (int i = 0; i < RANK; i++) n *= dims[i]; return n; }
  size_t extent(int i) const { return dims[i]; }
  const char *label() const { return myname.c_str(); }
  T *data() const { return ptr; }
  bool initialized() const { return ptr != nullptr; }
  static int constexpr get_rank() { return RANK; }

  template <class... I>
  T &operator()(I... idx) const {
    static_assert(sizeof...(I) == RANK, "wrong number of indices");
    size_t v[] = {size_t(idx)...};
    size_t off = 0;
    for (int i = 0; i < RANK; i++) off = off * dims[i] + v[i];
    return ptr[off];
  }

  Array const &operator=(T v) const { for (size_t i = 0; i < size(); i++) ptr[i] = v; return *this; }
  Array &operator=(Array const &) = default;
  Array(Array const &) = default;

  template <class U, int M2>
  void deep_copy_to(Array<U, RANK, M2, STYLE> const &dst) const {
    if (dst.size() != size()) Kokkos::abort("deep_copy_to: size mismatch");
    std::memcpy((void *)dst.ptr, (const void *)ptr, size() * sizeof(type));
  }
  Array<type, RANK, memHost, STYLE> createHostCopy() const { return copy_as<memHost>(); }
  template <class U = type>
  Array<U, RANK, memDevice, STYLE> createDeviceCopy() const { return copy_as<memDevice>(); }
  Array<type, RANK, memHost, STYLE> createHostObject() const { return object_as<memHost>(); }
  Array<type, RANK, memDevice, STYLE> createDeviceObject() const { return object_as<memDevice>(); }
  template <int M2>
  Array<type, RANK, M2, STYLE> object_as() const {
    Array<type, RANK, M2, STYLE> r;
    r.myname = myname;
    for (int i = 0; i < RANK; i++) r.dims[i] = dims[i];
    r.allocate();
    return r;
  }
  template <int M2>
  Array<type, RANK, M2, STYLE> copy_as() const {
    auto r = object_as<M2>();
    std::memcpy((void *)r.ptr, (const void *)ptr, size() * sizeof(type));
    return r;
  }

  // slice<N>(i0, ..., placeholders): fix the leading RANK-N indices and view
  // the trailing N dimensions (C order, so the view is contiguous).
  template <int N, class... I>
  Array<T, N, MEM, STYLE> slice(I... idx) const {
    static_assert(sizeof...(I) == RANK, "slice needs one argument per dimension");
    size_t v[] = {slice_index(idx)...};
    size_t off = 0;
    for (int i = 0; i < RANK; i++) off = off * dims[i] + (i < RANK - N ? v[i] : 0);
    Array<T, N, MEM, STYLE> r;
    r.owner = owner;
    r.ptr = ptr + off;
    r.myname = myname;
    for (int i = 0; i < N; i++) r.dims[i] = dims[RANK - N + i];
    return r;
  }
  static size_t slice_index(Colon) { return 0; }
  template <class U>
  static size_t slice_index(U i) { return size_t(i); }
};

// ---------------------------------------------------------------------------
namespace c {
template <int N>
struct SimpleBounds {
  int n[N];
  template <class... I>
  SimpleBounds(I... d) : n{int(d)...} { static_assert(sizeof...(I) == N, "bounds rank"); }
};
// Bounds: each dimension is a count n (indices 0..n-1) or an inclusive
// range {lo, hi} (yakl's LBnd without stride).
struct LBnd {
  int l, u;
  LBnd(int n) : l(0), u(n - 1) {}
  LBnd(size_t n) : l(0), u(int(n) - 1) {}
  LBnd(std::initializer_list<int> b) : l(*b.begin()), u(*(b.begin() + 1)) {}
};
template <int N>
struct Bounds {
  LBnd b[N];
  Bounds(LBnd a) : b{a} {}
  Bounds(LBnd a, LBnd c) : b{a, c} {}
  Bounds(LBnd a, LBnd c, LBnd d) : b{a, c, d} {}
  Bounds(LBnd a, LBnd c, LBnd d, LBnd e) : b{a, c, d, e} {}
};

template <class F>
void parallel_for(const char *, int n, F const &f) {
#pragma omp parallel for
  for (int i = 0; i < n; i++) f(i);
}
template <class F>
void parallel_for(int n, F const &f) { parallel_for("", n, f); }
template <class F>
void parallel_for(const char *, SimpleBounds<1> const &b, F const &f) { parallel_for("", b.n[0], f); }
template <class F>
void parallel_for(const char *, SimpleBounds<2> const &b, F const &f) {
#pragma omp parallel for collapse(2)
  for (int i0 = 0; i0 < b.n[0]; i0++)
    for (int i1 = 0; i1 < b.n[1]; i1++) f(i0, i1);
}
template <class F>
void parallel_for(const char *, SimpleBounds<3> const &b, F const &f) {
#pragma omp parallel for collapse(2)
  for (int i0 = 0; i0 < b.n[0]; i0++)
    for (int i1 = 0; i1 < b.n[1]; i1++)
      for (int i2 = 0; i2 < b.n[2]; i2++) f(i0, i1, i2);
}
template <class F>
void parallel_for(const char *, SimpleBounds<4> const &b, F const &f) {
#pragma omp parallel for collapse(2)
  for (int i0 = 0; i0 < b.n[0]; i0++)
    for (int i1 = 0; i1 < b.n[1]; i1++)
      for (int i2 = 0; i2 < b.n[2]; i2++)
        for (int i3 = 0; i3 < b.n[3]; i3++) f(i0, i1, i2, i3);
}
template <class F, int N>
void parallel_for(SimpleBounds<N> const &b, F const &f) { parallel_for("", b, f); }
template <class F>
void parallel_for(const char *, Bounds<1> const &b, F const &f) {
#pragma omp parallel for
  for (int i0 = b.b[0].l; i0 <= b.b[0].u; i0++) f(i0);
}
template <class F>
void parallel_for(const char *, Bounds<2> const &b, F const &f) {
#pragma omp parallel for collapse(2)
  for (int i0 = b.b[0].l; i0 <= b.b[0].u; i0++)
    for (int i1 = b.b[1].l; i1 <= b.b[1].u; i1++) f(i0, i1);
}
template <class F>
void parallel_for(const char *, Bounds<3> const &b, F const &f) {
#pragma omp parallel for collapse(2)
  for (int i0 = b.b[0].l; i0 <= b.b[0].u; i0++)
    for (int i1 = b.b[1].l; i1 <= b.b[1].u; i1++)
      for (int i2 = b.b[2].l; i2 <= b.b[2].u; i2++) f(i0, i1, i2);
}
template <class F, int N>
void parallel_for(Bounds<N> const &b, F const &f) { parallel_for("", b, f); }
}  // namespace c

namespace intrinsics {
// Sum of all elements in memory order (yakl's sum is a parallel reduction
// whose order is unspecified; one order has to be picked at one rank).
template <class T, int N, int M, int S>
typename std::remove_cv<T>::type sum(Array<T, N, M, S> const &a) {
  typename std::remove_cv<T>::type s = 0;
  for (size_t i = 0; i < a.size(); i++) s += a.data()[i];
  return s;
}
// Column-row storage: A(col,row).  C = A*B as matrices, C(c,r) = sum_k A(k,r) B(c,k).
template <class T, size_t CA, size_t RA, size_t CB>
SArray<T, 2, CB, RA> matmul_cr(SArray<T, 2, CA, RA> const &A, SArray<T, 2, CB, CA> const &B) {
  SArray<T, 2, CB, RA> C;
  for (unsigned r = 0; r < RA; r++)
    for (unsigned cc = 0; cc < CB; cc++) {
      T tmp = 0;
      for (unsigned k = 0; k < CA; k++) tmp += A(k, r) * B(cc, k);
      C(cc, r) = tmp;
    }
  return C;
}
template <class T, size_t CA, size_t RA>
SArray<T, 1, RA> matmul_cr(SArray<T, 2, CA, RA> const &A, SArray<T, 1, CA> const &v) {
  SArray<T, 1, RA> r;
  for (unsigned i = 0; i < RA; i++) {
    T tmp = 0;
    for (unsigned k = 0; k < CA; k++) tmp += A(k, i) * v(k);
    r(i) = tmp;
  }
  return r;
}
}  // namespace intrinsics

struct SimplePNetCDF {
  void redef() {}
  void enddef() {}
  void begin_indep_data() {}
  void end_indep_data() {}
  void create_dim(std::string, size_t) {}
  template <class T>
  void create_var(std::string, std::vector<std::string>) {}
  template <class A>
  void write(A const &, std::string) {}
  template <class A>
  void write_all(A const &, std::string, std::vector<MPI_Offset> const &) {}
  template <class A>
  void read_all(A const &, std::string, std::vector<MPI_Offset> const &) {}
};

}  // namespace yakl

using yakl::Array;
using yakl::memDevice;
using yakl::memHost;
using yakl::SArray;
using yakl::styleC;

#define PU_SHIM_TYPEDEFS(T, N)                                  \
  typedef Array<T, 1, memDevice, styleC> N##1d;                 \
  typedef Array<T, 2, memDevice, styleC> N##2d;                 \
  typedef Array<T, 3, memDevice, styleC> N##3d;                 \
  typedef Array<T, 4, memDevice, styleC> N##4d;                 \
  typedef Array<T, 5, memDevice, styleC> N##5d;                 \
  typedef Array<T const, 1, memDevice, styleC> N##Const1d;      \
  typedef Array<T const, 2, memDevice, styleC> N##Const2d;      \
  typedef Array<T const, 3, memDevice, styleC> N##Const3d;      \
  typedef Array<T const, 4, memDevice, styleC> N##Const4d;      \
  typedef Array<T const, 5, memDevice, styleC> N##Const5d;      \
  typedef Array<T, 1, memHost, styleC> N##Host1d;               \
  typedef Array<T, 2, memHost, styleC> N##Host2d;               \
  typedef Array<T, 3, memHost, styleC> N##Host3d;
PU_SHIM_TYPEDEFS(real, real)
PU_SHIM_TYPEDEFS(float, float)
PU_SHIM_TYPEDEFS(int, int)
PU_SHIM_TYPEDEFS(bool, bool)
#undef PU_SHIM_TYPEDEFS

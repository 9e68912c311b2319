// Minimal stand-ins for the AMReX types that PeleMP's spray physics headers
// use, so that those headers (Source/PP_Spray/SprayFuelData.H, Drag.H,
// SprayInterpolation.H, WallFunctions.H, BreakupSplash/AhamedSplash.H,
// BreakupSplash/SBData.H) compile as plain host C++ for the oracle's
// reference build.  TEST INFRASTRUCTURE, written for this project: the
// semantics follow AMReX's documented behaviour (element-wise RealVect
// arithmetic, floor() to IntVect, inclusive Box bounds, Array4 indexing);
// AMReX itself is not part of PeleMP and is not used.
#ifndef PMP_REF_SHIM_AMREX_H
#define PMP_REF_SHIM_AMREX_H

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#define AMREX_SPACEDIM 3
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_HOST
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_D_DECL(a, b, c) a, b, c
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_D_PICK(a, b, c) c

namespace amrex {
using Real = double;

template <class T>
constexpr const T& min(const T& a, const T& b) noexcept
{
  return std::min(a, b);
}
template <class T>
constexpr const T& max(const T& a, const T& b) noexcept
{
  return std::max(a, b);
}

template <class... Ts>
inline void ignore_unused(const Ts&...)
{
}

struct RefAbort : std::runtime_error {
  explicit RefAbort(const std::string& s) : std::runtime_error(s) {}
};
[[noreturn]] inline void Abort(const std::string& msg) { throw RefAbort(msg); }

template <class T, int N>
struct GpuArray {
  T arr[N];
  T& operator[](int i) noexcept { return arr[i]; }
  const T& operator[](int i) const noexcept { return arr[i]; }
  T* data() noexcept { return arr; }
  const T* data() const noexcept { return arr; }
};

struct IntVect {
  int vect[3] = {0, 0, 0};
  IntVect() = default;
  IntVect(int i, int j, int k) : vect{i, j, k} {}
  int& operator[](int i) noexcept { return vect[i]; }
  const int& operator[](int i) const noexcept { return vect[i]; }
  static IntVect TheZeroVector() { return IntVect(0, 0, 0); }
};

struct RealVect {
  Real vect[3] = {0., 0., 0.};
  RealVect() = default;
  RealVect(Real a, Real b, Real c) : vect{a, b, c} {}
  Real& operator[](int i) noexcept { return vect[i]; }
  const Real& operator[](int i) const noexcept { return vect[i]; }
  static RealVect TheZeroVector() { return RealVect(0., 0., 0.); }
  RealVect& operator+=(const RealVect& p)
  {
    for (int d = 0; d < 3; ++d) {
      vect[d] += p.vect[d];
    }
    return *this;
  }
  RealVect& operator-=(const RealVect& p)
  {
    for (int d = 0; d < 3; ++d) {
      vect[d] -= p.vect[d];
    }
    return *this;
  }
  RealVect& operator*=(Real s)
  {
    for (int d = 0; d < 3; ++d) {
      vect[d] *= s;
    }
    return *this;
  }
  RealVect& operator/=(Real s)
  {
    for (int d = 0; d < 3; ++d) {
      vect[d] /= s;
    }
    return *this;
  }
  Real radSquared() const
  {
    return vect[0] * vect[0] + vect[1] * vect[1] + vect[2] * vect[2];
  }
  Real vectorLength() const { return std::sqrt(radSquared()); }
  Real dotProduct(const RealVect& a) const
  {
    return vect[0] * a[0] + vect[1] * a[1] + vect[2] * a[2];
  }
  RealVect crossProduct(const RealVect& a) const
  {
    return RealVect(
      vect[1] * a[2] - vect[2] * a[1], vect[2] * a[0] - vect[0] * a[2],
      vect[0] * a[1] - vect[1] * a[0]);
  }
  RealVect operator-() const { return RealVect(-vect[0], -vect[1], -vect[2]); }
  IntVect floor() const
  {
    return IntVect(
      static_cast<int>(std::floor(vect[0])), static_cast<int>(std::floor(vect[1])),
      static_cast<int>(std::floor(vect[2])));
  }
};

inline RealVect operator+(const RealVect& a, const RealVect& b)
{
  return RealVect(a[0] + b[0], a[1] + b[1], a[2] + b[2]);
}
inline RealVect operator-(const RealVect& a, const RealVect& b)
{
  return RealVect(a[0] - b[0], a[1] - b[1], a[2] - b[2]);
}
inline RealVect operator*(const RealVect& a, const RealVect& b)
{
  return RealVect(a[0] * b[0], a[1] * b[1], a[2] * b[2]);
}
inline RealVect operator/(const RealVect& a, const RealVect& b)
{
  return RealVect(a[0] / b[0], a[1] / b[1], a[2] / b[2]);
}
inline RealVect operator+(const RealVect& a, Real s)
{
  return RealVect(a[0] + s, a[1] + s, a[2] + s);
}
inline RealVect operator-(const RealVect& a, Real s)
{
  return RealVect(a[0] - s, a[1] - s, a[2] - s);
}
inline RealVect operator*(const RealVect& a, Real s)
{
  return RealVect(a[0] * s, a[1] * s, a[2] * s);
}
inline RealVect operator/(const RealVect& a, Real s)
{
  return RealVect(a[0] / s, a[1] / s, a[2] / s);
}
inline RealVect operator*(Real s, const RealVect& a)
{
  return RealVect(s * a[0], s * a[1], s * a[2]);
}
inline RealVect operator-(Real s, const RealVect& a)
{
  return RealVect(s - a[0], s - a[1], s - a[2]);
}
inline RealVect operator+(Real s, const RealVect& a)
{
  return RealVect(s + a[0], s + a[1], s + a[2]);
}
inline RealVect operator-(const RealVect& a, const IntVect& b)
{
  return RealVect(
    a[0] - static_cast<Real>(b[0]), a[1] - static_cast<Real>(b[1]),
    a[2] - static_cast<Real>(b[2]));
}

struct Box {
  IntVect lo, hi;
  Box() = default;
  Box(const IntVect& l, const IntVect& h) : lo(l), hi(h) {}
  bool contains(const IntVect& p) const
  {
    for (int d = 0; d < 3; ++d) {
      if (p[d] < lo[d] || p[d] > hi[d]) {
        return false;
      }
    }
    return true;
  }
  bool contains(const Box& b) const { return contains(b.lo) && contains(b.hi); }
  Box& grow(int n)
  {
    for (int d = 0; d < 3; ++d) {
      lo[d] -= n;
      hi[d] += n;
    }
    return *this;
  }
  Box& growLo(int dir, int n)
  {
    lo[dir] -= n;
    return *this;
  }
  Box& growHi(int dir, int n)
  {
    hi[dir] += n;
    return *this;
  }
};

template <class T>
struct Array4 {
  T* p = nullptr;
  int lo[3] = {0, 0, 0};
  long long jstride = 0, kstride = 0, nstride = 0;
  T& operator()(const IntVect& iv, int n = 0) const
  {
    return p[(iv[0] - lo[0]) + (iv[1] - lo[1]) * jstride + (iv[2] - lo[2]) * kstride +
             n * nstride];
  }
  T& operator()(int i, int j, int k, int n = 0) const { return (*this)(IntVect(i, j, k), n); }
};

namespace Math {
inline Real floor(Real x) { return std::floor(x); }
inline Real abs(Real x) { return std::abs(x); }
} // namespace Math

namespace Gpu {
template <class T>
using HostVector = std::vector<T>;
template <class T>
using DeviceVector = std::vector<T>;
struct HostToDevice {};
struct DeviceToHost {};
static constexpr HostToDevice hostToDevice{};
static constexpr DeviceToHost deviceToHost{};
template <class Tag, class It, class Out>
inline void copyAsync(Tag, It b, It e, Out o)
{
  std::copy(b, e, o);
}
template <class Tag, class It, class Out>
inline void copy(Tag, It b, It e, Out o)
{
  std::copy(b, e, o);
}
inline void streamSynchronize() {}
namespace Device {
inline void streamSynchronize() {}
} // namespace Device
} // namespace Gpu
} // namespace amrex

#endif

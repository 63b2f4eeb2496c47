// The handful of Kokkos and Cabana names that CabanaPD user programs touch
// (execution/memory space tags, Kokkos::Array, reducer tags, the lambda
// macros), as plain C++ / CUDA stand-ins. Nothing here runs kernels: the
// CabanaPD front end launches its own.
#pragma once

#include <cmath>
#include <cstddef>
#include <limits>

#if defined(__CUDACC__)
#define CPD_HD __host__ __device__
#define KOKKOS_LAMBDA [=] __host__ __device__
#else
#define CPD_HD
#define KOKKOS_LAMBDA [=]
#endif
#define KOKKOS_INLINE_FUNCTION CPD_HD inline
#define KOKKOS_FUNCTION CPD_HD

namespace Kokkos {

template <class T, std::size_t N>
struct Array {
    T v[N];
    CPD_HD T& operator[](std::size_t i) { return v[i]; }
    CPD_HD const T& operator[](std::size_t i) const { return v[i]; }
    CPD_HD static constexpr std::size_t size() { return N; }
};

struct HostSpace;
struct Serial {
    using execution_space = Serial;
    using memory_space = HostSpace;
};
struct HostSpace {
    using execution_space = Serial;
    using memory_space = HostSpace;
};
struct CudaSpace;
struct Cuda {
    using execution_space = Cuda;
    using memory_space = CudaSpace;
};
struct CudaSpace {
    using execution_space = Cuda;
    using memory_space = CudaSpace;
};
using DefaultExecutionSpace = Cuda;
using DefaultHostExecutionSpace = Serial;

// Reducer tags for CabanaPD::createOutputTimeSeries: identity and join of
// Kokkos::Max / Kokkos::Sum / Kokkos::Min.
template <class T>
struct Max {
    using value_type = T;
    static T identity() { return std::numeric_limits<T>::lowest(); }
    static T join(T a, T b) { return a > b ? a : b; }
};
template <class T>
struct Min {
    using value_type = T;
    static T identity() { return std::numeric_limits<T>::max(); }
    static T join(T a, T b) { return a < b ? a : b; }
};
template <class T>
struct Sum {
    using value_type = T;
    static T identity() { return T(0); }
    static T join(T a, T b) { return a + b; }
};

inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}
inline void fence() {}

using std::abs;
using std::atan2;
using std::cos;
using std::exp;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;

namespace numbers {
template <class T>
constexpr T pi_v = T(3.14159265358979323846);
constexpr double pi = 3.14159265358979323846;
}  // namespace numbers

}  // namespace Kokkos

namespace Cabana {
struct InitUniform {};
struct InitRandom {};
}  // namespace Cabana

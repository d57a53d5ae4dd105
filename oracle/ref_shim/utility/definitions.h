// ORACLE — test infrastructure only. Stand-in for the reference's
// src/utility/definitions.h when the reference's host initial partitioner
// (src/initial_partitioning/kway_partitioner/kway_core.h, namespace
// GPU_HeiPa::ModifiedMetis, plain C++) is compiled on its own by
// oracle/build_ref.py. The real header pulls in Kokkos, which is not
// available; kway_core.h needs from it only the scalar type names and the
// few Kokkos names used by its two wrapper functions (kway_core.h:1547-1589),
// which the oracle never calls. These stand-ins let those wrappers compile.
#pragma once
#include <cstddef>
#include <cstdint>
#include <utility>
#include <vector>

namespace GPU_HeiPa {
typedef int32_t s32;
typedef int64_t s64;
typedef uint32_t u32;
typedef uint64_t u64;
typedef float f32;
typedef double f64;
typedef u32 vertex_t;
typedef s32 weight_t;
typedef u32 partition_t;

// A host array with the View call syntax used by the wrappers.
template<typename T>
struct ShimView {
    std::vector<T> v;
    ShimView() = default;
    template<typename A>
    ShimView(A, size_t n) : v(n) {}
    T &operator()(size_t i) { return v[i]; }
    const T &operator()(size_t i) const { return v[i]; }
    size_t extent(int) const { return v.size(); }
};

using HostPartition = ShimView<partition_t>;
struct DeviceExecutionSpace {};
}  // namespace GPU_HeiPa

namespace Kokkos {
struct WithoutInitializingTag {};
constexpr WithoutInitializingTag WithoutInitializing{};
template<typename... A>
inline int view_alloc(A...) { return 0; }
template<typename T>
inline GPU_HeiPa::ShimView<T> subview(GPU_HeiPa::ShimView<T> &v, std::pair<size_t, size_t>) { return v; }
template<typename A, typename B>
inline void deep_copy(A &, const B &) {}
inline void fence() {}
}  // namespace Kokkos

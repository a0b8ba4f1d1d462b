// Stand-ins for the CUSP containers and solvers that appear in the reference's
// host drivers, so its kernel files compile for the per-kernel parity tests.
// The drivers are never called; only the __global__ kernels are launched
// (test infrastructure).
#pragma once
#include <cstddef>
#include <thrust/device_vector.h>
namespace cusp {
struct device_memory {};
struct host_memory {};
template <typename T, typename Mem>
struct array1d : public thrust::device_vector<T> {
    array1d() {}
    explicit array1d(size_t n) : thrust::device_vector<T>(n) {}
    array1d(size_t n, T v) : thrust::device_vector<T>(n, v) {}
};
template <typename I, typename T, typename Mem>
struct dia_matrix {
    size_t num_rows = 0, num_cols = 0;
};
template <typename T, typename Mem>
struct identity_operator {
    size_t num_rows = 0, num_cols = 0;
    identity_operator() {}
    identity_operator(size_t r, size_t c) : num_rows(r), num_cols(c) {}
    void resize(size_t r, size_t c, T) { num_rows = r; num_cols = c; }
};
template <typename T>
struct monitor {
    template <typename V>
    monitor(const V &, size_t, double, double = 0.0, bool = false) {}
};
namespace krylov {
template <class A, class V, class Mo, class Pr>
void bicgstab(A &, V &, V &, Mo &, Pr &) {}
template <class A, class V, class Mo, class Pr>
void cg(A &, V &, V &, Mo &, Pr &) {}
}  // namespace krylov
namespace gallery {
template <class Mx>
void poisson5pt(Mx &, int, int) {}
template <class Mx>
void poisson7pt(Mx &, int, int, int) {}
}  // namespace gallery
}  // namespace cusp

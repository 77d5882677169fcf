// common.cuh — shared device/host helpers of the multislice engine.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace ms {

// complex types per real precision
template <class R> struct CplxT;
template <> struct CplxT<float> { using type = float2; };
template <> struct CplxT<double> { using type = double2; };
template <class R> using cplx = typename CplxT<R>::type;

template <class R> __host__ __device__ __forceinline__ cplx<R> mk(R re, R im) { cplx<R> c; c.x = re; c.y = im; return c; }

template <class C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <class C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {   // a * conj(b)
    C r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}
template <class C, class R> __host__ __device__ __forceinline__ C cscale(C a, R s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
template <class C> __host__ __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class C> __host__ __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void check(cudaError_t e, const char *what, const char *file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
        throw CudaError(buf);
    }
}
#define MS_CUDA(x) ::ms::check((x), #x, __FILE__, __LINE__)

}  // namespace ms

// ref_shim.h — lets g++ compile the reference's OpenCL C kernels (kernels/*_d.cl) for the CPU.
// TEST INFRASTRUCTURE ONLY (oracle/_ref). Included ahead of each kernel file by oracle/build_ref.py.
//
// OpenCL C -> C++: address-space qualifiers vanish, double2 is a struct, work-item functions read a
// thread-local work-item descriptor, barrier() is a real barrier across the threads emulating one work
// group (ref_host.cpp), and the builtins the kernels call map to the C library (native_ prefixes are
// already stripped by the build, as clTEM does when native functions are off, kernels.h:41-42).
#pragma once

#include <barrier>
#include <cfloat>
#include <cmath>
#include <cstddef>

struct double2 {
    double x, y;
};
inline double2 make_double2(double a, double b) { return double2{a, b}; }
inline double2 operator*(double s, double2 a) { return double2{s * a.x, s * a.y}; }
inline double2 operator*(double2 a, double s) { return double2{a.x * s, a.y * s}; }
inline double2 operator/(double2 a, double s) { return double2{a.x / s, a.y / s}; }

struct RefWorkItem {
    size_t gid[2], lid[2], grp[2], lsz[2], gsz[2];
};
extern thread_local RefWorkItem ref_wi;
extern thread_local std::barrier<> *ref_bar;

inline size_t get_global_id(int d) { return ref_wi.gid[d]; }
inline size_t get_local_id(int d) { return ref_wi.lid[d]; }
inline size_t get_group_id(int d) { return ref_wi.grp[d]; }
inline size_t get_local_size(int d) { return ref_wi.lsz[d]; }
inline size_t get_global_size(int d) { return ref_wi.gsz[d]; }
inline void ref_barrier() { ref_bar->arrive_and_wait(); }

#define __kernel
#define __global
#define global
#define __constant const
#define __local
#define restrict __restrict__
#define CLK_LOCAL_MEM_FENCE 1
#define barrier(x) ref_barrier()

inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
// OpenCL C 1.2 section 6.12.4
inline double smoothstep(double e0, double e1, double x) {
    double t = std::fmin(std::fmax((x - e0) / (e1 - e0), 0.0), 1.0);
    return t * t * (3.0 - 2.0 * t);
}
using std::ceil;
using std::cos;
using std::exp;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
using std::tan;

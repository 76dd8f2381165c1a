// OpenCL C on the host: just enough of the language for the reference's
// Barnes-Hut OpenCL kernels (Morton codes, bitonic sort, Karras build) to
// compile as C++ and run on the CPU. TEST INFRASTRUCTURE ONLY.
// Address-space qualifiers vanish (host memory is one space); work-item ids
// come from the emulator in cl_runner.cpp, and barrier() hands control to the
// next work-item of the work-group (the emulator runs a group's work-items as
// coroutines).
#pragma once
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <sys/types.h>

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef unsigned long ulong;  // 64 bits on LP64, as in OpenCL

struct uint2 {
    uint x, y;  // little-endian halves of a ulong: x the low 32 bits
};
struct double2 {
    double x, y;
};
struct double3 {
    double x, y, z;
};

#define __kernel
#define __global
#define __constant const
#define __local
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

namespace clemu {
struct Item {
    size_t gid, lid, grp, lsize, gsize;
};
extern Item cur;
void barrier_wait();
}  // namespace clemu

inline size_t get_global_id(uint) { return clemu::cur.gid; }
inline size_t get_local_id(uint) { return clemu::cur.lid; }
inline size_t get_group_id(uint) { return clemu::cur.grp; }
inline size_t get_local_size(uint) { return clemu::cur.lsize; }
inline size_t get_global_size(uint) { return clemu::cur.gsize; }
inline void barrier(int) { clemu::barrier_wait(); }
inline uint clz(uint x) { return x ? (uint)__builtin_clz(x) : 32u; }
inline double3 vload3(size_t i, const double* p) { return double3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
inline void vstore3(double3 v, size_t i, double* p) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

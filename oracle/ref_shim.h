// ref_shim.h - TEST INFRASTRUCTURE ONLY: lets the reference's device traversal header (accel/traverse.cuh) compile
// as host C++ so the oracle can run the reference's own traversal arithmetic on the CPU. Provides the CUDA
// bit-cast and bit-count intrinsics it uses, implemented with memcpy and compiler builtins.
#pragma once
#include <cuda_runtime.h>
#include <cstring>
#ifndef __CUDACC__
static inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
static inline unsigned __float_as_uint(float f) { unsigned u; std::memcpy(&u, &f, 4); return u; }
static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline float __uint_as_float(unsigned u) { float f; std::memcpy(&f, &u, 4); return f; }
static inline int __ffs(unsigned x) { return __builtin_ffs((int)x); }
static inline int __popc(unsigned x) { return __builtin_popcount(x); }
#endif

/*
 * prelude.h -- lets the reference's CUDA C kernels compile as host C++ so
 * the reference itself can be run on CPU cores to pin the oracle.
 * TEST INFRASTRUCTURE ONLY (oracle/).  Force-included (-include) before the
 * reference's kern.cu by oracle/build_ref.py; the reference sources are
 * compiled where they lie, through symlinks, and are not modified.
 *
 * Kernel launches become loops over the launch grid in ref_driver.cpp; the
 * built-in index variables are thread-local so OpenMP threads can each run
 * a block.  The reference kernels use no shared memory and no barriers.
 */
#ifndef REF_EMU_PRELUDE_H
#define REF_EMU_PRELUDE_H
#include <cmath>
#include <cstdio>
#include <cstdlib>
#define __CUDACC__ 1
#define __global__
#define __device__
#define __host__
#define __align__(x) __attribute__((aligned(x)))
struct emu_dim3 {
  unsigned x, y, z;
};
extern thread_local emu_dim3 blockIdx;
extern thread_local emu_dim3 threadIdx;
extern thread_local emu_dim3 blockDim;
using std::cos;
using std::exp;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
using std::tan;
#endif

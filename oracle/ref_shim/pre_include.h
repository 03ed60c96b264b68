// ORACLE PIN SHIM — TEST INFRASTRUCTURE ONLY.
// Pre-included when the reference updater is compiled for sm_100a (oracle/Makefile, target `ref`).
// The reference's helper header uses the warp intrinsics of CUDA < 9 (__shfl, __shfl_down,
// __shfl_xor, __ballot), which are errors on sm_70 and later. None of them is reached by the
// sweep; they are mapped to their *_sync forms over the full warp so the header compiles.
#pragma once
#include <cuda_runtime.h>
#define __shfl(...) __shfl_sync(0xffffffffu, __VA_ARGS__)
#define __shfl_down(...) __shfl_down_sync(0xffffffffu, __VA_ARGS__)
#define __shfl_xor(...) __shfl_xor_sync(0xffffffffu, __VA_ARGS__)
#define __ballot(x) __ballot_sync(0xffffffffu, (x))

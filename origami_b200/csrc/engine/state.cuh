// Whole-engine state transfer: the real atoms of every system (systems in
// order, n in all) as AoS triples <-> the padded SoA device layout, through
// `map` (real index -> padded index).  Positions and velocities are FP64;
// forces are the engine's 64-bit fixed-point accumulators, moved bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ogk {

void launch_gather_xyz(const double* a, const double* b, const double* c, const int32_t* map, int64_t n,
                       double* out, cudaStream_t s);
void launch_scatter_xyz(const double* in, const int32_t* map, int64_t n, double* a, double* b, double* c,
                        cudaStream_t s);
void launch_gather_fixed(const unsigned long long* a, const unsigned long long* b, const unsigned long long* c,
                         const int32_t* map, int64_t n, int64_t* out, cudaStream_t s);
void launch_scatter_fixed(const int64_t* in, const int32_t* map, int64_t n, unsigned long long* a,
                          unsigned long long* b, unsigned long long* c, cudaStream_t s);

}  // namespace ogk

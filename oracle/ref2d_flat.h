// Pre-include for building the reference 2D solver from its own, unmodified sources (checker
// only): 2D-solver/include/parsing.h never defines the flat(i, j, Nx) index helper that
// common/filterABC.h and 2D-solver/core/functions.cuh call. This is the row-major node index
// those files assume (j * Nx + i, as 3D-solver/include/parsing3D.h:49-51 defines it in 3D).
#pragma once
#include <cstddef>
__host__ __device__ inline size_t flat(int i, int j, int Nx) { return (size_t)j * (size_t)Nx + (size_t)i; }

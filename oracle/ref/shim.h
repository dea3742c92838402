/*
 * Forced-include shim for compiling the unmodified reference sources
 * (al0vya/gpu-mwdg2 source/) with nvcc 12.9 on Linux.
 *
 * - utilities/cuda_utils.cuh:9-10 declares `cudaError_t sync()`, which clashes
 *   with glibc's `int sync(void)` from <unistd.h>; the reference's function is
 *   renamed by the macro below after <unistd.h> has been seen.
 * - classes/Details.cu:100 uses std::max({...}) without including <algorithm>.
 *
 * This header is part of the oracle build recipe (test infrastructure only).
 */
#pragma once
#include <unistd.h>
#include <algorithm>
#include <initializer_list>
#define sync ref_sync

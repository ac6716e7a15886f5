// TEST INFRASTRUCTURE: lets the reference's GPU test suite
// (tests/test_cuda_solver.cu, which includes "cuda_solver.cuh") compile
// against this library's drop-in API instead of the reference's GPU solver.
#pragma once
#include "adrt/cuda_solver.hpp"

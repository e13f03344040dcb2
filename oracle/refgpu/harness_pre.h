// Force-included (nvcc -include) ahead of one of the reference's own GPU programs,
// gpu_cuda/shared/<algorithm>.cu, compiled unchanged from the reference checkout.  TEST
// INFRASTRUCTURE ONLY: the programs built with it run the reference's kernels as a second oracle
// on a B200; nothing in the product links them.
//
// It changes no line of the reference.  It includes every header the reference includes (their
// include guards then make the reference's own #includes no-ops), and afterwards renames three
// identifiers for the rest of the translation unit:
//   * cudaMalloc / cudaFree -> tga_ref_malloc / tga_ref_free (harness_main.cu), which forward to the
//     runtime and record each device allocation with the reference source line that made it, so
//     the harness can copy a buffer back before it is freed (or after main returns, if it is
//     never freed) -- the reference keeps its results in such buffers and prints none of them;
//   * main -> tga_ref_main, called by the harness's own main.
#pragma once
#include <assert.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <device_launch_parameters.h>
#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/fill.h>
#include <thrust/host_vector.h>
#include <thrust/transform_scan.h>

#include <chrono>
#include <fstream>
#include <iostream>
#include <vector>

cudaError_t tga_ref_malloc(void** p, size_t n, int line);
cudaError_t tga_ref_free(void* p, int line);

#define cudaMalloc(p, n) tga_ref_malloc((void**)(p), (size_t)(n), __LINE__)
#define cudaFree(p) tga_ref_free((void*)(p), __LINE__)
#define main tga_ref_main

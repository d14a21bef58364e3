// remora/cuda.hpp -- the B200 (sm_100a) cuda_tag device for Remora.
//
// Include this header BEFORE <remora/remora.hpp> (or any other Remora header that
// defines expressions or kernels): Remora binds kernel calls by qualified name at the
// point where its templates are defined, so the cuda_tag overloads must be declared
// first. The host code compiles with any C++14 compiler (no CUDA toolkit, no __NVCC__:
// defining __NVCC__ would pull in Remora's HIP backend) and links libremora_cuda.so.
//
//   #include <remora/cuda.hpp>
//   #include <remora/remora.hpp>
//   using namespace remora;
//   matrix<double, column_major, cuda_tag> A = copy_to_device(A_cpu, cuda_tag());
//   cholesky_decomposition<matrix<double, column_major, cuda_tag>> chol(A);
//   chol.solve(B, left());
//   matrix<double> X = copy_to_cpu(B);
#ifndef REMORA_CUDA_HPP
#define REMORA_CUDA_HPP

#if defined(__NVCC__) || defined(__HCC__)
#error "compile cuda_tag host code with the host compiler: Remora includes its HIP backend under __NVCC__/__HCC__"
#endif

#include "cuda/fwd.hpp"
#include <remora/remora.hpp>
#include "cuda/device.hpp"
#include "cuda/dense.hpp"
#include "cuda/copy.hpp"
#include "cuda/kernels.hpp"

#endif

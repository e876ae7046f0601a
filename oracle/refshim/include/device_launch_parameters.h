/* Stand-in: blockIdx/threadIdx/blockDim come from ref_shim.h when the
 * reference kernels are compiled as host code. Oracle test infrastructure only. */
#pragma once

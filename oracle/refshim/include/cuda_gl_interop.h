/* Stand-in for CUDA's GL interop header: the reference kernels that include
 * it use nothing from it, and there is no OpenGL on these machines.
 * Oracle test infrastructure only. */
#pragma once

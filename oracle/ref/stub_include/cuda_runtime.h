/* Empty stand-in for <cuda_runtime.h>: the reference's decoder headers include it, but
 * compiled as host C++ for the CPU oracle they need nothing from it. */
#pragma once

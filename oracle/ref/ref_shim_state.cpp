// TEST INFRASTRUCTURE ONLY: storage for the emulated thread/block index.
#include "host_shim.h"
thread_local fls_shim_idx3 fls_shim_thread_idx {0, 0, 0};
thread_local fls_shim_idx3 fls_shim_block_idx {0, 0, 0};

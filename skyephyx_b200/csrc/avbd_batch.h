// Builds of the batched persistent kernel.  Each build is compiled in its own
// translation unit (avbd_batch_v.cu with AVBD_BATCH_ID = 1..7) so the library
// compiles in parallel; the host side reaches them through these getters.
#pragma once
#include "avbd_common.cuh"

namespace avbd {

// k_batch_step(world, order, nlive, queue): one step of every listed scene.
using BatchKernel = void (*)(World, const int*, const int*, int*);

BatchKernel batch_kernel_v1();   // 256 threads, about 156 registers
BatchKernel batch_kernel_v2();   // 256 threads, 128 registers
BatchKernel batch_kernel_v3();   // 256 threads, 80 registers
BatchKernel batch_kernel_v4();   // 256 threads, 64 registers
BatchKernel batch_kernel_v5();   // 512 threads, 128 registers
BatchKernel batch_kernel_v6();   // 512 threads, 64 registers
BatchKernel batch_kernel_v7();   // 1024 threads, 64 registers

}  // namespace avbd

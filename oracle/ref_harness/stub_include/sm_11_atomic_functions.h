/* Empty stand-in for the CUDA-1.x header that neiglist.cu:23 includes and that
 * CUDA 12.9 no longer ships; the reference kernels use no atomics from it. */
#pragma once

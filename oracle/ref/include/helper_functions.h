/* Empty stand-in for the CUDA-samples helper_functions.h that the reference
 * includes (MCGPU-PET.h:173-176); the reference uses nothing from it.
 * Test infrastructure for the oracle/_ref build only. */
#pragma once

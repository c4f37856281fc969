// Build-only stand-in for the OptiX function-table header.
//
// Test infrastructure: Native/denoiser.cuh includes this header and then
// renames the table symbol. The OptiX SDK is not present on this machine, and
// the OptiX denoiser is a closed library that the product replaces, so the
// reference's RtDenoise is compiled against stubs that report an error.
#pragma once
#include <cstddef>

#define OPTIX_FUNCTION_TABLE_SYMBOL g_optixFunctionTable
struct OptixFunctionTable { void* unused; };

// Declarations-only stand-ins for the OptiX names that FliX's index header
// mentions.  TEST INFRASTRUCTURE ONLY.
//
// FliX's bucket layer (build_bucket_layer_only, insert, remove,
// lookups_ordered, lookups_successor, rebuild_bucket_layer_only in
// FliX/impl_cg_rtx_index_updates.cuh:1711-2677) is plain CUDA, but the same
// header also defines the ray-tracing index layer, so it names OptiX types and
// functions in code the bucket layer never reaches:
//   - `extern optix_wrapper optix` (FliX/impl_cg_rtx_index_updates.cuh:52),
//   - `rebuild_structures` / `build_structures` returning an
//     OptixTraversableHandle (:531, :934) and calling
//     cg::build_compacted_as_from_representatives (:637, :1051),
//   - std::optional<optix_pipeline> with emplace(...) (:1451, :2056),
//   - OPTIX_CHECK(optixLaunch(...)) in lookup() (:2622).
// Those names only have to parse.  Nothing here is defined: the shim library
// is linked with -z defs, so if any bucket-layer path reached one of them the
// link would fail instead of producing a library that calls OptiX.
// The one helper that IS defined, atomicAdd on `unsigned long`, is the overload
// the reference takes from its un-vendored cudahelpers library for
// compute_total_keys_in_structure (:134); it forwards to the 64-bit atomicAdd.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

typedef unsigned long long OptixTraversableHandle;
typedef struct OptixDeviceContext_opaque *OptixDeviceContext;
typedef struct OptixPipeline_opaque *OptixPipeline;
typedef int OptixResult;
struct OptixShaderBindingTable;

struct optix_wrapper {
  OptixDeviceContext optix_context;
};

struct optix_pipeline {
  optix_wrapper *optix;
  OptixPipeline pipeline;
  OptixShaderBindingTable *sbt;
  optix_pipeline(optix_wrapper *, const char *, const char *, const char *);
};

OptixResult optixLaunch(OptixPipeline, cudaStream_t, CUdeviceptr, size_t, OptixShaderBindingTable **,
                        unsigned, unsigned, unsigned);

#define OPTIX_CHECK(call) { (void)(call); }

namespace cg {
template <typename key_type, typename... Args>
OptixTraversableHandle build_compacted_as_from_representatives(Args &&...);
}

__device__ __forceinline__ unsigned long atomicAdd(unsigned long *address, unsigned long value) {
  static_assert(sizeof(unsigned long) == sizeof(unsigned long long), "LP64 only");
  return (unsigned long)atomicAdd((unsigned long long *)address, (unsigned long long)value);
}

// NVTX domain tag used by lookup()/lookup_cuda(); the nvtx3 headers come from
// FliX's own nvtx_stub folder.
#include <nvtx3/nvtx3.hpp>
struct nvtx_rtx_domain {
  static constexpr char const *name{"rtx"};
};

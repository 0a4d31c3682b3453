// BSDF readback probe (re_bsdf_probe): the device BSDF of the Shade kernels,
// evaluated and sampled on a batch of caller-supplied queries, one thread per
// query.  Counterpart of the reference's readback probe
// resources/shaders/integrators/pbr_sampling_probe.hlsl:9-102, with the
// context, parameters, directions and random triple chosen per query.
#include <cuda_runtime.h>

#include <cstdint>

#include "bsdf.cuh"
#include "re_b200.h"
#include "runtime.h"

static_assert(sizeof(re_bsdf_query) == 160, "re_bsdf_query is ten float4");
static_assert(sizeof(re_bsdf_probe_result) == 128, "re_bsdf_probe_result is eight float4");

namespace re {
namespace {

__device__ __forceinline__ f3 xyz(float4 v) { return mk(v.x, v.y, v.z); }

__global__ void __launch_bounds__(128) k_bsdf_probe(const float4* __restrict__ q, uint32_t n, float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4* r = q + size_t(i) * 10u;
    float4 v[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = r[k];
    BsdfContext c;
    c.ng = xyz(v[0]);
    c.eta_i = v[0].w;
    c.ns = xyz(v[1]);
    c.eta_t = v[1].w;
    c.tangent = xyz(v[2]);
    c.transport = __float_as_uint(v[2].w);
    BsdfParams p;
    p.base_color = xyz(v[3]);
    p.metallic = v[3].w;
    p.f0 = xyz(v[4]);
    p.roughness = v[4].w;
    p.cond_eta = xyz(v[5]);
    p.transmission = v[5].w;
    p.cond_k = xyz(v[6]);
    p.model = __float_as_uint(v[6].w);
    p.lobes = __float_as_uint(v[7].w);
    p.complex_fresnel = __float_as_uint(v[8].w);
    const f3 wo = xyz(v[7]), wi = xyz(v[8]), u = xyz(v[9]);
    const BsdfEval e = bsdf_evaluate<false>(c, p, wo, wi);
    const BsdfSample s = bsdf_sample<false>(c, p, wo, u);
    float pdf_at = 0.f;
    if (s.valid && !s.delta) {
        const BsdfEval e2 = bsdf_evaluate<false>(c, p, wo, s.dir);
        pdf_at = (e2.valid && e2.measure == kMeasureSolidAngle) ? e2.pdf : 0.f;
    }
    float4* o = out + size_t(i) * 8u;
    o[0] = make_float4(e.value.x, e.value.y, e.value.z, e.pdf);
    o[1] = make_float4(e.diffuse.x, e.diffuse.y, e.diffuse.z, __uint_as_float(e.measure));
    o[2] = make_float4(e.specular.x, e.specular.y, e.specular.z, __uint_as_float(e.lobe));
    o[3] = make_float4(s.dir.x, s.dir.y, s.dir.z, s.pdf);
    o[4] = make_float4(s.value.x, s.value.y, s.value.z, s.eta);
    o[5] = make_float4(s.diffuse.x, s.diffuse.y, s.diffuse.z, __uint_as_float(s.measure));
    o[6] = make_float4(s.specular.x, s.specular.y, s.specular.z, __uint_as_float(s.lobe));
    o[7] = make_float4(__uint_as_float(e.valid ? 1u : 0u), __uint_as_float(s.delta ? 1u : 0u),
                       __uint_as_float(s.valid ? 1u : 0u), pdf_at);
}

}  // namespace
}  // namespace re

extern "C" RE_API re_status re_bsdf_probe(const re_bsdf_query* queries, uint32_t count, re_bsdf_probe_result* results,
                                          uint32_t memory, void* stream) {
    using namespace re;
    if (count == 0) return clear_error();
    if (queries == nullptr || results == nullptr) return set_error(RE_INVALID_ARGUMENT, "null argument");
    if ((reinterpret_cast<uintptr_t>(queries) & 15u) != 0 || (reinterpret_cast<uintptr_t>(results) & 15u) != 0)
        return set_error(RE_INVALID_ARGUMENT, "re_bsdf_probe: queries and results must be 16-byte aligned");
    if (memory != RE_MEMORY_HOST && memory != RE_MEMORY_DEVICE)
        return set_error(RE_INVALID_ARGUMENT, "re_bsdf_probe: unknown memory kind");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t blocks = (count + 127u) / 128u;
    if (memory == RE_MEMORY_DEVICE) {
        k_bsdf_probe<<<blocks, 128, 0, st>>>(reinterpret_cast<const float4*>(queries), count,
                                             reinterpret_cast<float4*>(results));
        RE_CUDA_TRY(cudaGetLastError());
        return clear_error();
    }
    DeviceBuffer dq, dr;
    RE_CUDA_TRY(dq.reserve(size_t(count) * sizeof(re_bsdf_query)));
    RE_CUDA_TRY(dr.reserve(size_t(count) * sizeof(re_bsdf_probe_result)));
    RE_CUDA_TRY(cudaMemcpyAsync(dq.ptr, queries, size_t(count) * sizeof(re_bsdf_query), cudaMemcpyHostToDevice, st));
    k_bsdf_probe<<<blocks, 128, 0, st>>>(static_cast<const float4*>(dq.ptr), count, static_cast<float4*>(dr.ptr));
    RE_CUDA_TRY(cudaGetLastError());
    RE_CUDA_TRY(cudaMemcpyAsync(results, dr.ptr, size_t(count) * sizeof(re_bsdf_probe_result), cudaMemcpyDeviceToHost,
                                st));
    RE_CUDA_TRY(cudaStreamSynchronize(st));
    return clear_error();
}

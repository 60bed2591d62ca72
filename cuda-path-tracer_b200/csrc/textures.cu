// Texture objects for albedo and normal maps, and a sampling entry for tests.
#include <cuda_runtime.h>
#include <string.h>
#include "cpt.h"
#include "cpt_internal.h"

// Scene::upload(textureArrays) (Scene.cu:57-81) creates one texture object per image
// with normalized coordinates, linear filtering, normalized-float reads and the
// default (wrap) address mode. This creates the same sampler over a single-level
// RGBA8 array, which is what tex2D reads from the reference's mipmapped arrays.
extern "C" int cpt_texture_create(const uint8_t* rgba8, uint32_t width, uint32_t height, cudaTextureObject_t* out)
{
    CPT_RANGE("cpt_texture_create");
    if (!rgba8 || !out || width == 0 || height == 0) return CPT_ERR_INVALID_ARGUMENT;
    *out = 0;
    const cudaChannelFormatDesc fmt = cudaCreateChannelDesc<uchar4>();
    cudaArray_t arr = nullptr;
    if (cudaMallocArray(&arr, &fmt, width, height) != cudaSuccess) return CPT_ERR_CUDA;
    const size_t pitch = 4 * (size_t)width;
    if (cudaMemcpy2DToArray(arr, 0, 0, rgba8, pitch, pitch, height, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFreeArray(arr);
        return CPT_ERR_CUDA;
    }
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeNormalizedFloat;
    td.normalizedCoords = 1;
    if (cudaCreateTextureObject(out, &res, &td, nullptr) != cudaSuccess) {
        cudaFreeArray(arr);
        *out = 0;
        return CPT_ERR_CUDA;
    }
    return CPT_OK;
}

extern "C" void cpt_texture_destroy(cudaTextureObject_t tex)
{
    if (!tex) return;
    cudaResourceDesc res;
    const bool have = cudaGetTextureObjectResourceDesc(&res, tex) == cudaSuccess;
    cudaDestroyTextureObject(tex);
    if (have && res.resType == cudaResourceTypeArray && res.res.array.array) cudaFreeArray(res.res.array.array);
}

namespace cpt {

__global__ void k_texture_sample(cudaTextureObject_t tex, const float2* __restrict__ uv, uint32_t n,
                                 float4* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = tex2D<float4>(tex, uv[i].x, uv[i].y);
}

}  // namespace cpt

extern "C" int cpt_texture_sample(cudaTextureObject_t tex, const float* uv, uint32_t n, float* rgba_out,
                                  cudaStream_t stream)
{
    if (!tex || (n && (!uv || !rgba_out))) return CPT_ERR_INVALID_ARGUMENT;
    if (!n) return CPT_OK;
    cpt::k_texture_sample<<<(n + 255) / 256, 256, 0, stream>>>(tex, reinterpret_cast<const float2*>(uv), n,
                                                              reinterpret_cast<float4*>(rgba_out));
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

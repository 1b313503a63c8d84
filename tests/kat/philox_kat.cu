// Test-only: device curand Philox4_32_10 output for pinning the oracle's Philox stream.
// For each subsequence s: curand_init(1234, s, 0) followed by the draw schedule
// uniform4, uniform4, uniform, uniform4, uniform (14 floats), then for each offset in
// offsets[]: curand_init(1234, s, offset) and one uniform4.
#include <cstdint>
#include <curand_kernel.h>

__global__ void kat_kernel(const unsigned long long* subseq, int n, const unsigned* offsets, int nOff, float* sched, float* reinit,
                           unsigned* words)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandStatePhilox4_32_10_t st;
    curand_init(1234ull, subseq[i], 0ull, &st);
    float* o = sched + (size_t)i * 14;
    float4 a = curand_uniform4(&st);
    float4 b = curand_uniform4(&st);
    float c = curand_uniform(&st);
    float4 d = curand_uniform4(&st);
    float e = curand_uniform(&st);
    o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    o[4] = b.x; o[5] = b.y; o[6] = b.z; o[7] = b.w;
    o[8] = c;
    o[9] = d.x; o[10] = d.y; o[11] = d.z; o[12] = d.w;
    o[13] = e;
    for (int k = 0; k < nOff; k++)
    {
        curandStatePhilox4_32_10_t r;
        curand_init(1234ull, subseq[i], offsets[k], &r);
        float4 u = curand_uniform4(&r);
        float* q = reinit + ((size_t)i * nOff + k) * 4;
        q[0] = u.x; q[1] = u.y; q[2] = u.z; q[3] = u.w;
    }
    curandStatePhilox4_32_10_t w;
    curand_init(1234ull, subseq[i], 0ull, &w);
    uint4 x = curand4(&w);
    uint4 y = curand4(&w);
    unsigned* wo = words + (size_t)i * 8;
    wo[0] = x.x; wo[1] = x.y; wo[2] = x.z; wo[3] = x.w;
    wo[4] = y.x; wo[5] = y.y; wo[6] = y.z; wo[7] = y.w;
}

extern "C" int philox_kat(const unsigned long long* subseq, int n, const unsigned* offsets, int nOff, float* sched, float* reinit,
                          unsigned* words)
{
    kat_kernel<<<(n + 127) / 128, 128>>>(subseq, n, offsets, nOff, sched, reinit, words);
    if (cudaGetLastError() != cudaSuccess) return 1;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// Test-only: samples of a texture created with the renderer's descriptors (clamp, linear
// filter, normalised coordinates), to pin the oracle's texture sampling against the hardware.
// format: 0 = u8 sRGB, 1 = u8 linear, 2 = f32; channels 1 or 4.
__global__ void texture_kat_kernel(cudaTextureObject_t tex, int channels, const float* uv, int n, float* out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (channels == 1)
        out[i] = tex2D<float>(tex, uv[2 * i], uv[2 * i + 1]);
    else
    {
        float4 v = tex2D<float4>(tex, uv[2 * i], uv[2 * i + 1]);
        out[4 * i] = v.x; out[4 * i + 1] = v.y; out[4 * i + 2] = v.z; out[4 * i + 3] = v.w;
    }
}

extern "C" int texture_kat(const void* texels, int width, int height, int channels, int format, const float* uvHost, int n, float* outHost)
{
    const bool u8 = format != 2;
    cudaChannelFormatDesc cd = u8 ? (channels == 1 ? cudaCreateChannelDesc<uchar1>() : cudaCreateChannelDesc<uchar4>())
                                  : (channels == 1 ? cudaCreateChannelDesc<float1>() : cudaCreateChannelDesc<float4>());
    cudaArray_t arr;
    if (cudaMallocArray(&arr, &cd, width, height) != cudaSuccess) return 1;
    size_t pitch = (size_t)width * channels * (u8 ? 1 : 4);
    if (cudaMemcpy2DToArray(arr, 0, 0, texels, pitch, pitch, height, cudaMemcpyHostToDevice) != cudaSuccess) return 2;
    cudaResourceDesc res{};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = arr;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.normalizedCoords = 1;
    td.sRGB = format == 0 ? 1 : 0;
    td.readMode = u8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
    cudaTextureObject_t tex;
    if (cudaCreateTextureObject(&tex, &res, &td, nullptr) != cudaSuccess) return 3;
    float *uvD, *outD;
    cudaMalloc(&uvD, sizeof(float) * 2 * n);
    cudaMalloc(&outD, sizeof(float) * channels * n);
    cudaMemcpy(uvD, uvHost, sizeof(float) * 2 * n, cudaMemcpyHostToDevice);
    texture_kat_kernel<<<(n + 127) / 128, 128>>>(tex, channels, uvD, n, outD);
    int rc = cudaDeviceSynchronize() == cudaSuccess ? 0 : 4;
    cudaMemcpy(outHost, outD, sizeof(float) * channels * n, cudaMemcpyDeviceToHost);
    cudaFree(uvD);
    cudaFree(outD);
    cudaDestroyTextureObject(tex);
    cudaFreeArray(arr);
    return rc;
}

// tex2d_shim.cpp -- Tex2D<float> (CUDA/Tex2D.h) for the reference's GPU
// backprojector, written for g++.
//
// The reference defines these members in CUDA/Tex2DFloat.cpp without the
// `template<>` prefix an explicit specialisation needs, which MSVC accepts and
// g++ rejects, so that one file is restated here with the same behaviour
// (CUDA/Tex2DFloat.cpp:15-134): a width x height float cudaArray, a texture
// object on it with unnormalised coordinates, linear filtering, clamped
// addressing and element reads; Set copies a dense host image into the array.
#include <sstream>
#include <string>

#include <cuda_runtime.h>

#include "CUDA/ErrorChecking.h"
#include "CUDA/Tex2D.h"
#include "Common/Exception.h"

namespace JEngine {

template <>
void Tex2D<float>::Malloc() {
    cudaChannelFormatDesc desc = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    const cudaError_t e = cudaMallocArray(&pArrayOnDevice, &desc, width, height);
    if (e == cudaErrorMemoryAllocation) {
        std::stringstream ss;
        ss << "CUDA failed to malloc " << width * height * sizeof(float) << " bytes of array memory";
        ThrowExceptionAndLog(ss.str());
    } else if (e != cudaSuccess) {
        ThrowExceptionAndLog(cudaGetErrorString(e));
    }
}

template <>
void Tex2D<float>::CreateObject() {
    cudaResourceDesc res{};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = pArrayOnDevice;
    cudaTextureDesc td{};
    td.normalizedCoords = 0;
    td.filterMode = cudaFilterModeLinear;
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.readMode = cudaReadModeElementType;
    CUDA_SAFE_CALL(cudaCreateTextureObject(&textureObject, &res, &td, nullptr));
}

template <>
Tex2D<float>::Tex2D(const size_t w, const size_t h) : width(w), height(h), pArrayOnDevice(nullptr) {
    Malloc();
    CreateObject();
}

template <>
Tex2D<float>::Tex2D(const Tex2D<float>& o) : width(o.width), height(o.height), pArrayOnDevice(nullptr) {
    Malloc();
    CreateObject();
    CUDA_SAFE_CALL(cudaMemcpy2DArrayToArray(pArrayOnDevice, 0, 0, o.pArrayOnDevice, 0, 0, width * sizeof(float),
                                            height, cudaMemcpyDeviceToDevice));
}

template <>
Tex2D<float>::Tex2D(Tex2D<float>&& o) noexcept
    : width(o.width), height(o.height), pArrayOnDevice(o.pArrayOnDevice), textureObject(o.textureObject) {
    o.pArrayOnDevice = nullptr;
    o.textureObject = 0;
}

template <>
Tex2D<float>::~Tex2D() {
    if (textureObject) cudaDestroyTextureObject(textureObject);
    if (pArrayOnDevice) cudaFreeArray(pArrayOnDevice);
}

template <>
void Tex2D<float>::Set(const float* src, cudaStream_t s) {
    CUDA_SAFE_CALL(cudaMemcpy2DToArrayAsync(pArrayOnDevice, 0, 0, src, width * sizeof(float), width * sizeof(float),
                                            height, cudaMemcpyHostToDevice, s));
}

template <>
void Tex2D<float>::Set(const float* src) {
    CUDA_SAFE_CALL(cudaMemcpy2DToArray(pArrayOnDevice, 0, 0, src, width * sizeof(float), width * sizeof(float),
                                       height, cudaMemcpyHostToDevice));
}

}  // namespace JEngine

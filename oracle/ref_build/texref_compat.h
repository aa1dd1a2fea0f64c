// Compatibility header force-included (nvcc -include) when the reference's
// unmodified projector sources are compiled for the parity pin.
//
// The reference kernels (model/ConeBeamLayers/{Standard,Beijing}/plug/kernel/
// {forward,backward}Kernel.cu) use CUDA *texture references*:
//   texture<float, cudaTextureType3D, cudaReadModeElementType> t;   (global)
//   t.addressMode[i] = ...; t.filterMode = ...; t.normalized = ...;  (host)
//   cudaBindTextureToArray(t, array, desc); cudaUnbindTexture(t);   (host)
//   tex3D(t, x, y, z)                                               (device)
// CUDA 12 removed that API. This header supplies the same names on top of
// texture *objects* with identical sampling state (address mode, filter mode,
// unnormalised coordinates), so the reference's arithmetic is compiled as is.
// It is test infrastructure: only the oracle build recipe uses it.
#pragma once
#include <torch/extension.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdio.h>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct dtvref_texref {
  enum cudaTextureAddressMode addressMode[3];
  enum cudaTextureFilterMode filterMode;
  int normalized;
  cudaTextureObject_t obj;
};

// The reference declares its texture reference at file scope without a
// memory-space qualifier and touches it from host and device code alike;
// managed memory is the one space both sides can name directly.
#define texture __managed__ dtvref_texref

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ inline T tex3D(const dtvref_texref<T, Dim, Mode>& t, float x, float y, float z) {
  return ::tex3D<T>(t.obj, x, y, z);
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaBindTextureToArray(dtvref_texref<T, Dim, Mode>& t, cudaArray_t array,
                                          const cudaChannelFormatDesc&) {
  cudaResourceDesc res;
  memset(&res, 0, sizeof(res));
  res.resType = cudaResourceTypeArray;
  res.res.array.array = array;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  for (int i = 0; i < 3; ++i) td.addressMode[i] = t.addressMode[i];
  td.filterMode = t.filterMode;
  td.readMode = Mode;
  td.normalizedCoords = t.normalized;
  cudaTextureObject_t obj = 0;
  cudaError_t e = cudaCreateTextureObject(&obj, &res, &td, nullptr);
  t.obj = obj;
  return e;
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaUnbindTexture(dtvref_texref<T, Dim, Mode>& t) {
  // Kernels launched on this texture may still be running: finish them before
  // the object goes away (the legacy unbind was ordered the same way).
  cudaError_t e = cudaDeviceSynchronize();
  if (t.obj) cudaDestroyTextureObject(t.obj);
  t.obj = 0;
  return e;
}

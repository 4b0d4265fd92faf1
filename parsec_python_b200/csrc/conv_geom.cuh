// Geometry of one 3-D convolution of the learned-start network and the
// 8-channel gather of its "virtual input" (shared by the CUDA-core kernels in
// unet.cu and the tensor-core forward in conv_tc.cu).
//
// Activations are channels-last BF16 tensors [voxel][C] on a grid with x
// fastest (voxel = x + nx (y + ny z)), C a multiple of 8.  The virtual input
// of Cin = Ca + Cs channels is the first Ca from tensor A -- nearest-neighbour
// upsampled x2 when `up` is set -- and the last Cs from the skip tensor S at
// the virtual input's own resolution.
#pragma once

#include "psc_internal.cuh"

#include <cuda_bf16.h>

struct ConvGeom {
  int nxi, nyi, nzi;   // virtual input grid
  int nxa, nya, nza;   // grid of A (the virtual grid halved when up)
  int up;
  int Ca, Cs, Cin;
  int nxo, nyo, nzo;   // output grid
  int stride, ksize, Cout;
};

// 8 channels [c0, c0+8) of the virtual input at voxel (x, y, z) (inside the grid)
__device__ __forceinline__ uint4 conv_vin8(const __nv_bfloat16* A, const __nv_bfloat16* S, const ConvGeom& g,
                                           int x, int y, int z, int c0) {
  if (c0 < g.Ca) {
    long va;
    if (g.up) va = (x >> 1) + (long)g.nxa * ((y >> 1) + (long)g.nya * (z >> 1));
    else va = x + (long)g.nxa * (y + (long)g.nya * z);
    return *reinterpret_cast<const uint4*>(A + va * g.Ca + c0);
  }
  const long vs = x + (long)g.nxi * (y + (long)g.nyi * z);
  return *reinterpret_cast<const uint4*>(S + vs * g.Cs + (c0 - g.Ca));
}

// tensor-core forward (conv_tc.cu); the caller has validated the geometry
int psc_conv_tc_forward(psc_ctx* ctx, const ConvGeom& g, const __nv_bfloat16* a, const __nv_bfloat16* s,
                        const __nv_bfloat16* w, const float* bias, int act, __nv_bfloat16* o, float* out32,
                        cudaStream_t st);

// Learned initial density: BF16 3-D convolution kernels (forward, backward
// data, backward weights) with FP32 accumulation, the loss and the Adam step.
//
// The reference only consumes a predicted density (it reads a file in
// V_ion/pseudoDiag_ML4Den_poisson.py:12-586 and renormalises it); the network
// that produces it is new here.  Activations are channels-last BF16 tensors
// [voxel][C] on a grid with x fastest (voxel = x + nx (y + ny z)), C a
// multiple of 8.  Weights are BF16 [tap][Cin][Cout] (tap = dx + 3 (dy + 3 dz)
// for 3x3x3 kernels, one tap for 1x1x1), biases FP32.  Gradients are FP32.
//
// One convolution reads a "virtual input" of Cin = Ca + Cs channels: the
// first Ca from tensor A -- nearest-neighbour upsampled x2 when `up` is set,
// which is how the decoder grows back to the finer grid -- and the last Cs
// from the skip tensor S at the virtual input's own resolution.  So the
// upsample and the concatenation of an encoder-decoder are never written out.
// Stride 2 halves the grid (output dims ceil(n/2)), padding is 1 for 3x3x3.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <cuda_bf16.h>

#include "conv_geom.cuh"

namespace {

__device__ __forceinline__ void unpack8(const uint4 u, float* f) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float2 t = __bfloat1622float2(h[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

constexpr int FWD_NT = 128;
constexpr float LEAK = 0.0625f;   // leaky-ReLU slope below zero
constexpr int WTILE = 256;   // weights staged per tap: input-chunk x output-chunk = 256 floats (27 KB for 27 taps)

}  // namespace

// ---------------------------------------------------------------------------
// forward: out[o][co] = act(b[co] + sum_tap sum_ci vin(o s + tap - pad)[ci] W[tap][ci][co])
// act: 0 identity, 1 ReLU, 2 leaky ReLU (slope 1/16 below zero).
// One thread per output voxel, COT output channels per CTA (blockIdx.y).
// ---------------------------------------------------------------------------
template <int COT>
__global__ void __launch_bounds__(FWD_NT)
k_conv_fwd(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ S,
           const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias, ConvGeom g, int act,
           __nv_bfloat16* __restrict__ out, float* __restrict__ out32) {
  constexpr int CIN_CHUNK = WTILE / COT;
  __shared__ __align__(16) float ws[27 * WTILE];
  const int taps = g.ksize * g.ksize * g.ksize;
  const int pad = g.ksize / 2;
  const int co0 = blockIdx.y * COT;
  const long nvo = (long)g.nxo * g.nyo * g.nzo;
  const long vo = (long)blockIdx.x * FWD_NT + threadIdx.x;
  const bool valid = vo < nvo;
  int xo = 0, yo = 0, zo = 0;
  if (valid) {
    xo = (int)(vo % g.nxo);
    const long r = vo / g.nxo;
    yo = (int)(r % g.nyo);
    zo = (int)(r / g.nyo);
  }
  float acc[COT];
#pragma unroll
  for (int j = 0; j < COT; ++j) acc[j] = bias[co0 + j];
  for (int cc = 0; cc < g.Cin; cc += CIN_CHUNK) {
    const int cn = min(CIN_CHUNK, g.Cin - cc);
    __syncthreads();
    for (int e = threadIdx.x; e < taps * cn * COT; e += FWD_NT) {
      const int co = e % COT;
      const int r = e / COT;
      const int ci = r % cn, tap = r / cn;
      ws[(tap * CIN_CHUNK + ci) * COT + co] =
          __bfloat162float(W[((long)tap * g.Cin + cc + ci) * g.Cout + co0 + co]);
    }
    __syncthreads();
    if (!valid) continue;
    for (int tap = 0; tap < taps; ++tap) {
      const int dx = tap % g.ksize, dy = (tap / g.ksize) % g.ksize, dz = tap / (g.ksize * g.ksize);
      const int xi = xo * g.stride + dx - pad, yi = yo * g.stride + dy - pad, zi = zo * g.stride + dz - pad;
      if (xi < 0 || yi < 0 || zi < 0 || xi >= g.nxi || yi >= g.nyi || zi >= g.nzi) continue;
      for (int c8 = 0; c8 < cn; c8 += 8) {
        float x[8];
        unpack8(conv_vin8(A, S, g, xi, yi, zi, cc + c8), x);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float* wr = ws + (tap * CIN_CHUNK + c8 + j) * COT;
#pragma unroll
          for (int co = 0; co < COT; co += 4) {
            const float4 w4 = *reinterpret_cast<const float4*>(wr + co);
            acc[co] = fmaf(x[j], w4.x, acc[co]);
            acc[co + 1] = fmaf(x[j], w4.y, acc[co + 1]);
            acc[co + 2] = fmaf(x[j], w4.z, acc[co + 2]);
            acc[co + 3] = fmaf(x[j], w4.w, acc[co + 3]);
          }
        }
      }
    }
  }
  if (!valid) return;
#pragma unroll
  for (int j = 0; j < COT; ++j) {
    const float a = acc[j];
    const float v = act == 1 ? fmaxf(a, 0.0f) : (act == 2 ? (a > 0.0f ? a : LEAK * a) : a);
    out[vo * g.Cout + co0 + j] = __float2bfloat16_rn(v);
    if (out32) out32[vo * g.Cout + co0 + j] = v;
  }
}

// ---------------------------------------------------------------------------
// backward data: dvin[v][ci] = sum_tap sum_co gm[o(v,tap)][co] W[tap][ci][co]
// where o s + tap - pad = v.  One thread per virtual-input voxel, CIT input
// channels per CTA; the output channels are walked in chunks of 256 / CIT.
// ---------------------------------------------------------------------------
template <int CIT>
__global__ void __launch_bounds__(FWD_NT)
k_conv_bwd_data(const float* __restrict__ gm, const __nv_bfloat16* __restrict__ W, ConvGeom g,
                float* __restrict__ dvin) {
  constexpr int COUT_CHUNK = WTILE / CIT;
  __shared__ __align__(16) float ws[27 * WTILE];
  const int taps = g.ksize * g.ksize * g.ksize;
  const int pad = g.ksize / 2;
  const int ci0 = blockIdx.y * CIT;
  const long nvi = (long)g.nxi * g.nyi * g.nzi;
  const long v = (long)blockIdx.x * FWD_NT + threadIdx.x;
  const bool valid = v < nvi;
  int x = 0, y = 0, z = 0;
  if (valid) {
    x = (int)(v % g.nxi);
    const long r = v / g.nxi;
    y = (int)(r % g.nyi);
    z = (int)(r / g.nyi);
  }
  float acc[CIT];
#pragma unroll
  for (int j = 0; j < CIT; ++j) acc[j] = 0.0f;
  for (int oc = 0; oc < g.Cout; oc += COUT_CHUNK) {
    const int on = min(COUT_CHUNK, g.Cout - oc);
    __syncthreads();
    for (int e = threadIdx.x; e < taps * on * CIT; e += FWD_NT) {
      const int ci = e % CIT;
      const int r = e / CIT;
      const int co = r % on, tap = r / on;
      ws[(tap * COUT_CHUNK + co) * CIT + ci] = __bfloat162float(W[((long)tap * g.Cin + ci0 + ci) * g.Cout + oc + co]);
    }
    __syncthreads();
    if (!valid) continue;
    for (int tap = 0; tap < taps; ++tap) {
      const int dx = tap % g.ksize, dy = (tap / g.ksize) % g.ksize, dz = tap / (g.ksize * g.ksize);
      // o s = v - d + pad
      const int ax = x - dx + pad, ay = y - dy + pad, az = z - dz + pad;
      if (ax < 0 || ay < 0 || az < 0) continue;
      if (g.stride == 2 && ((ax | ay | az) & 1)) continue;
      const int ox = ax / g.stride, oy = ay / g.stride, oz = az / g.stride;
      if (ox >= g.nxo || oy >= g.nyo || oz >= g.nzo) continue;
      const float* gp = gm + (ox + (long)g.nxo * (oy + (long)g.nyo * oz)) * g.Cout + oc;
      for (int co4 = 0; co4 < on; co4 += 4) {
        const float4 g4 = *reinterpret_cast<const float4*>(gp + co4);
        const float gv[4] = {g4.x, g4.y, g4.z, g4.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float* wr = ws + (tap * COUT_CHUNK + co4 + j) * CIT;
#pragma unroll
          for (int ci = 0; ci < CIT; ci += 4) {
            const float4 w4 = *reinterpret_cast<const float4*>(wr + ci);
            acc[ci] = fmaf(gv[j], w4.x, acc[ci]);
            acc[ci + 1] = fmaf(gv[j], w4.y, acc[ci + 1]);
            acc[ci + 2] = fmaf(gv[j], w4.z, acc[ci + 2]);
            acc[ci + 3] = fmaf(gv[j], w4.w, acc[ci + 3]);
          }
        }
      }
    }
  }
  if (!valid) return;
#pragma unroll
  for (int j = 0; j < CIT; ++j) dvin[v * g.Cin + ci0 + j] = acc[j];
}

// ---------------------------------------------------------------------------
// backward weights: part[chunk][tap][ci][co] = sum over the chunk's output
// voxels of vin(o s + tap - pad)[ci] gm[o][co].  A CTA owns one tap, a 16x16
// (ci, co) tile and one voxel chunk; it stages 64 voxels at a time.
// ---------------------------------------------------------------------------
constexpr int BW_NT = 256;
constexpr int BW_STAGE = 64;

__global__ void __launch_bounds__(BW_NT)
k_conv_bwd_w(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ S,
             const float* __restrict__ gm, ConvGeom g, int vchunk, float* __restrict__ part) {
  __shared__ float xs[BW_STAGE][17];
  __shared__ float gs[BW_STAGE][17];
  const int taps = g.ksize * g.ksize * g.ksize;
  const int pad = g.ksize / 2;
  const int nci = (g.Cin + 15) / 16, nco = (g.Cout + 15) / 16;
  int t = blockIdx.y;
  const int cot = t % nco;
  t /= nco;
  const int cit = t % nci;
  const int tap = t / nci;
  const int ci0 = cit * 16, co0 = cot * 16;
  const int dx = tap % g.ksize, dy = (tap / g.ksize) % g.ksize, dz = tap / (g.ksize * g.ksize);
  const long nvo = (long)g.nxo * g.nyo * g.nzo;
  const long v_begin = (long)blockIdx.x * vchunk;
  const long v_end = min(nvo, v_begin + vchunk);
  const int tci = threadIdx.x >> 4, tco = threadIdx.x & 15;
  float acc = 0.0f;
  for (long v0 = v_begin; v0 < v_end; v0 += BW_STAGE) {
    __syncthreads();
    // stage inputs: 64 voxels x two groups of 8 channels (threads 0..127)
    if (threadIdx.x < 2 * BW_STAGE) {
      const int j = threadIdx.x >> 1, half = threadIdx.x & 1;
      const long vo = v0 + j;
      const int c0 = ci0 + 8 * half;
      float x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (vo < v_end && c0 < g.Cin) {
        const int xo = (int)(vo % g.nxo);
        const long r = vo / g.nxo;
        const int yo = (int)(r % g.nyo), zo = (int)(r / g.nyo);
        const int xi = xo * g.stride + dx - pad, yi = yo * g.stride + dy - pad, zi = zo * g.stride + dz - pad;
        if (xi >= 0 && yi >= 0 && zi >= 0 && xi < g.nxi && yi < g.nyi && zi < g.nzi)
          unpack8(conv_vin8(A, S, g, xi, yi, zi, c0), x);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) xs[j][8 * half + i] = x[i];
    } else {
      // stage gradients: 64 voxels x 16 channels as float4 (threads 128..255, two each)
      for (int q = threadIdx.x - 2 * BW_STAGE; q < BW_STAGE * 4; q += BW_NT - 2 * BW_STAGE) {
        const int j = q >> 2, c4 = (q & 3) * 4;
        const long vo = v0 + j;
        float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (vo < v_end && co0 + c4 < g.Cout) g4 = *reinterpret_cast<const float4*>(gm + vo * g.Cout + co0 + c4);
        gs[j][c4] = g4.x;
        gs[j][c4 + 1] = g4.y;
        gs[j][c4 + 2] = g4.z;
        gs[j][c4 + 3] = g4.w;
      }
    }
    __syncthreads();
#pragma unroll 16
    for (int j = 0; j < BW_STAGE; ++j) acc = fmaf(xs[j][tci], gs[j][tco], acc);
  }
  const int ci = ci0 + tci, co = co0 + tco;
  if (ci < g.Cin && co < g.Cout) part[(((long)blockIdx.x * taps + tap) * g.Cin + ci) * g.Cout + co] = acc;
}

// dW[e] = sum_chunk part[chunk][e] in chunk order
__global__ void k_sum_chunks(const float* __restrict__ part, int nchunk, long nw, float* __restrict__ dW) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nw; e += (long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < nchunk; ++c) s += part[(long)c * nw + e];
    dW[e] = s;
  }
}

// bias gradient partials: per CTA (voxel chunk) and channel, then summed by
// k_sum_chunks.  256 threads = R rows x Cout channels (Cout <= 256); row r
// sums voxels v0 + r, v0 + r + R, ...; the rows are combined in order.
__global__ void __launch_bounds__(256)
k_bias_partial(const float* __restrict__ gm, long nvo, int Cout, int vchunk, float* __restrict__ part) {
  __shared__ float sh[256];
  const long v0 = (long)blockIdx.x * vchunk;
  const long v1 = min(nvo, v0 + vchunk);
  const int R = 256 / Cout;
  const int co = threadIdx.x % Cout, r = threadIdx.x / Cout;
  float s = 0.0f;
  if (r < R)
    for (long v = v0 + r; v < v1; v += R) s += gm[v * Cout + co];
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < Cout) {
    float t = 0.0f;
    for (int q = 0; q < R; ++q) t += sh[q * Cout + threadIdx.x];
    part[(long)blockIdx.x * Cout + threadIdx.x] = t;
  }
}

// gm = g * act'(pre) from the BF16 activation (out > 0 exactly when pre > 0):
// 1 above zero, 0 (ReLU) or the leak slope (leaky ReLU) below
__global__ void k_relu_grad(const float* __restrict__ gin, const __nv_bfloat16* __restrict__ out, long n,
                            float below, float* __restrict__ gm) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    gm[i] = __bfloat162float(out[i]) > 0.0f ? gin[i] : below * gin[i];
}

// Split the virtual-input gradient: dA (+)= pool(dvin[:, :Ca]) (sum over the
// 8 fine voxels of each coarse one when up), dS (+)= dvin[:, Ca:].
__global__ void k_split_grad_a(const float* __restrict__ dvin, ConvGeom g, int accumulate, float* __restrict__ dA) {
  const long na = (long)g.nxa * g.nya * g.nza * g.Ca;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < na; e += (long)gridDim.x * blockDim.x) {
    const int c = (int)(e % g.Ca);
    const long va = e / g.Ca;
    float s = 0.0f;
    if (g.up) {
      const int xa = (int)(va % g.nxa);
      const long r = va / g.nxa;
      const int ya = (int)(r % g.nya), za = (int)(r / g.nya);
      for (int d = 0; d < 8; ++d) {
        const int x = 2 * xa + (d & 1), y = 2 * ya + ((d >> 1) & 1), z = 2 * za + (d >> 2);
        if (x < g.nxi && y < g.nyi && z < g.nzi)
          s += dvin[(x + (long)g.nxi * (y + (long)g.nyi * z)) * g.Cin + c];
      }
    } else {
      s = dvin[va * g.Cin + c];
    }
    dA[e] = accumulate ? dA[e] + s : s;
  }
}

__global__ void k_split_grad_s(const float* __restrict__ dvin, ConvGeom g, int accumulate, float* __restrict__ dS) {
  const long ns = (long)g.nxi * g.nyi * g.nzi * g.Cs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < ns; e += (long)gridDim.x * blockDim.x) {
    const int c = (int)(e % g.Cs);
    const long v = e / g.Cs;
    const float s = dvin[v * g.Cin + g.Ca + c];
    dS[e] = accumulate ? dS[e] + s : s;
  }
}

// MSE on channel 0 of a [n][C] FP32 prediction: per-CTA partial of sum (y-t)^2
// and the gradient 2 (y - t) / n on channel 0 (0 elsewhere).
__global__ void __launch_bounds__(256)
k_mse(const float* __restrict__ y, int C, const float* __restrict__ t, long n, float* __restrict__ grad,
      double* __restrict__ part) {
  __shared__ double sh[8];
  double s = 0.0;
  const float inv = 2.0f / (float)n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float d = y[i * C] - t[i];
    s += (double)d * d;
    grad[i * C] = inv * d;
    for (int c = 1; c < C; ++c) grad[i * C + c] = 0.0f;
  }
  s = psc_block_sum<double, 256>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_mse_final(const double* __restrict__ part, int np, long n, double* __restrict__ loss) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < np; ++i) s += part[i];
    *loss = s / (double)n;
  }
}

// Adam (Kingma & Ba 2015) on FP32 master weights; the BF16 copy used by the
// convolutions is refreshed in the same pass.
__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ grad,
                       float* __restrict__ m, float* __restrict__ v, long n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void k_f32_to_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16_rn(x[i]);
}

// Network input: channels-last BF16 [n][8]: ch0 = a0 * x0, ch1 = a1 * x1, rest 0
__global__ void k_pack_input(const double* __restrict__ x0, const double* __restrict__ x1, long n, double a0,
                             double a1, __nv_bfloat16* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    out[i * 8] = __float2bfloat16_rn((float)(a0 * x0[i]));
    out[i * 8 + 1] = __float2bfloat16_rn((float)(a1 * x1[i]));
#pragma unroll
    for (int c = 2; c < 8; ++c) out[i * 8 + c] = __float2bfloat16_rn(0.0f);
  }
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {
int geom_from(psc_ctx* ctx, const int* gi, ConvGeom& g) {
  g.nxi = gi[0]; g.nyi = gi[1]; g.nzi = gi[2];
  g.nxa = gi[3]; g.nya = gi[4]; g.nza = gi[5];
  g.up = gi[6];
  g.Ca = gi[7]; g.Cs = gi[8];
  g.Cin = g.Ca + g.Cs;
  g.nxo = gi[9]; g.nyo = gi[10]; g.nzo = gi[11];
  g.stride = gi[12]; g.ksize = gi[13]; g.Cout = gi[14];
  PSC_REQUIRE(ctx, g.Ca > 0 && g.Ca % 8 == 0 && g.Cs >= 0 && g.Cs % 8 == 0 && g.Cout % 8 == 0 && g.Cout > 0,
              "conv3d: channel counts must be positive multiples of 8");
  PSC_REQUIRE(ctx, g.stride == 1 || g.stride == 2, "conv3d: stride must be 1 or 2");
  PSC_REQUIRE(ctx, g.ksize == 1 || g.ksize == 3, "conv3d: kernel size must be 1 or 3");
  PSC_REQUIRE(ctx, g.nxi > 0 && g.nyi > 0 && g.nzi > 0 && g.nxo > 0 && g.nyo > 0 && g.nzo > 0,
              "conv3d: empty grid");
  const int ex = g.stride == 1 ? g.nxi : (g.nxi + 1) / 2;
  const int ey = g.stride == 1 ? g.nyi : (g.nyi + 1) / 2;
  const int ez = g.stride == 1 ? g.nzi : (g.nzi + 1) / 2;
  PSC_REQUIRE(ctx, g.nxo == ex && g.nyo == ey && g.nzo == ez, "conv3d: output grid does not match stride");
  PSC_REQUIRE(ctx, g.ksize == 3 || g.stride == 1, "conv3d: 1x1x1 kernels take stride 1");
  PSC_REQUIRE(ctx, g.Cout <= 256, "conv3d: at most 256 output channels");
  if (g.up) {
    PSC_REQUIRE(ctx, g.nxa == (g.nxi + 1) / 2 && g.nya == (g.nyi + 1) / 2 && g.nza == (g.nzi + 1) / 2,
                "conv3d: A must be the virtual grid halved (rounded up) when up = 1");
  } else {
    PSC_REQUIRE(ctx, g.nxa == g.nxi && g.nya == g.nyi && g.nza == g.nzi, "conv3d: A must match the input grid");
  }
  return 0;
}
}  // namespace

extern "C" int psc_conv3d_fwd(psc_ctx* ctx, const int* geom, const void* A, const void* S, const void* W,
                              const float* bias, int act, void* out, float* out32, void* stream) {
  if (!ctx) return 2;
  ConvGeom g;
  if (int rc = geom_from(ctx, geom, g)) return rc;
  PSC_REQUIRE(ctx, act >= 0 && act <= 2, "conv3d_fwd: act must be 0 (identity), 1 (ReLU) or 2 (leaky ReLU)");
  PSC_REQUIRE(ctx, A && W && bias && out && (g.Cs == 0 || S), "conv3d_fwd: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const long nvo = (long)g.nxo * g.nyo * g.nzo;
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* s = static_cast<const __nv_bfloat16*>(S);
  const auto* w = static_cast<const __nv_bfloat16*>(W);
  auto* o = static_cast<__nv_bfloat16*>(out);
  // the tensor cores where a layer has 32 or more output channels; the
  // full-grid layers with 8 (N padded to 16) are gather-bound and faster on
  // the CUDA cores (90^3: 636 against 779 us for the widest of them)
  if (ctx->conv_tc == 2 || (ctx->conv_tc == 1 && g.Cout >= 32))
    return psc_conv_tc_forward(ctx, g, a, s, w, bias, act, o, out32, st);
  if (g.Cout % 16 == 0) {
    dim3 grid(psc_div_up(nvo, FWD_NT), g.Cout / 16);
    k_conv_fwd<16><<<grid, FWD_NT, 0, st>>>(a, s, w, bias, g, act, o, out32);
  } else {
    dim3 grid(psc_div_up(nvo, FWD_NT), g.Cout / 8);
    k_conv_fwd<8><<<grid, FWD_NT, 0, st>>>(a, s, w, bias, g, act, o, out32);
  }
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_conv3d_bwd(psc_ctx* ctx, const int* geom, const void* A, const void* S, const void* W,
                              const float* gout, const void* out, int act, float* gm, float* dvin, float* dA,
                              int acc_a, float* dS, int acc_s, float* dW, float* dB, float* work, long work_floats,
                              void* stream) {
  if (!ctx) return 2;
  ConvGeom g;
  if (int rc = geom_from(ctx, geom, g)) return rc;
  PSC_REQUIRE(ctx, act >= 0 && act <= 2 && (act == 0 || out), "conv3d_bwd: bad activation arguments");
  PSC_REQUIRE(ctx, A && W && gout && gm && dW && dB && work && (g.Cs == 0 || S), "conv3d_bwd: NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const long nvo = (long)g.nxo * g.nyo * g.nzo;
  const long nvi = (long)g.nxi * g.nyi * g.nzi;
  const int taps = g.ksize * g.ksize * g.ksize;
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* s = static_cast<const __nv_bfloat16*>(S);
  const auto* w = static_cast<const __nv_bfloat16*>(W);
  // 1. output gradient through the activation
  if (act != 0) {
    k_relu_grad<<<148 * 8, 256, 0, st>>>(gout, static_cast<const __nv_bfloat16*>(out), nvo * g.Cout,
                                         act == 2 ? LEAK : 0.0f, gm);
    PSC_LAUNCH_CHECK(ctx);
  } else if (gm != gout) {
    PSC_CUDA(ctx, cudaMemcpyAsync(gm, gout, nvo * g.Cout * sizeof(float), cudaMemcpyDeviceToDevice, st));
  }
  // 2. weight and bias gradients (partials in `work`, summed in chunk order)
  const long nw = (long)taps * g.Cin * g.Cout;
  int vchunk = 4096;
  int nchunk = psc_div_up(nvo, vchunk);
  while ((long)nchunk * nw > work_floats && vchunk < (1 << 26)) {
    vchunk *= 2;
    nchunk = psc_div_up(nvo, vchunk);
  }
  PSC_REQUIRE(ctx, (long)nchunk * nw <= work_floats && (long)nchunk * g.Cout <= work_floats,
              "conv3d_bwd: work buffer too small");
  {
    const int nci = (g.Cin + 15) / 16, nco = (g.Cout + 15) / 16;
    dim3 grid(nchunk, taps * nci * nco);
    k_conv_bwd_w<<<grid, BW_NT, 0, st>>>(a, s, gm, g, vchunk, work);
    PSC_LAUNCH_CHECK(ctx);
    k_sum_chunks<<<psc_div_up(nw, 256), 256, 0, st>>>(work, nchunk, nw, dW);
    PSC_LAUNCH_CHECK(ctx);
    k_bias_partial<<<nchunk, 256, 0, st>>>(gm, nvo, g.Cout, vchunk, work);
    PSC_LAUNCH_CHECK(ctx);
    k_sum_chunks<<<1, 256, 0, st>>>(work, nchunk, g.Cout, dB);
    PSC_LAUNCH_CHECK(ctx);
  }
  // 3. input gradient, split into dA and dS
  if (dvin) {
    if (g.Cin % 16 == 0) {
      dim3 grid(psc_div_up(nvi, FWD_NT), g.Cin / 16);
      k_conv_bwd_data<16><<<grid, FWD_NT, 0, st>>>(gm, w, g, dvin);
    } else {
      dim3 grid(psc_div_up(nvi, FWD_NT), g.Cin / 8);
      k_conv_bwd_data<8><<<grid, FWD_NT, 0, st>>>(gm, w, g, dvin);
    }
    PSC_LAUNCH_CHECK(ctx);
    if (dA) {
      k_split_grad_a<<<148 * 8, 256, 0, st>>>(dvin, g, acc_a, dA);
      PSC_LAUNCH_CHECK(ctx);
    }
    if (dS && g.Cs > 0) {
      k_split_grad_s<<<148 * 8, 256, 0, st>>>(dvin, g, acc_s, dS);
      PSC_LAUNCH_CHECK(ctx);
    }
  }
  return 0;
}

extern "C" int psc_mse_loss(psc_ctx* ctx, const float* y, int C, const float* target, long n, float* grad,
                            double* loss_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, y && target && grad && loss_dev && n > 0 && C >= 1, "mse: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  double* part = ctx->red_partial;
  k_mse<<<PSC_RED_BLOCKS, 256, 0, st>>>(y, C, target, n, grad, part);
  PSC_LAUNCH_CHECK(ctx);
  k_mse_final<<<1, 32, 0, st>>>(part, PSC_RED_BLOCKS, n, loss_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_adam_step(psc_ctx* ctx, float* w, void* wb, const float* grad, float* m, float* v, long n,
                             float lr, float b1, float b2, float eps, int step, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, w && grad && m && v && n > 0 && step >= 1, "adam: bad arguments");
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<psc_div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(w, static_cast<__nv_bfloat16*>(wb), grad, m, v, n,
                                                               lr, b1, b2, eps, c1, c2);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_f32_to_bf16(psc_ctx* ctx, const float* x, void* y, long n, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, x && y && n >= 0, "f32_to_bf16: bad arguments");
  if (n == 0) return 0;
  k_f32_to_bf16<<<psc_div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(x, static_cast<__nv_bfloat16*>(y), n);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_pack_input(psc_ctx* ctx, const double* x0, const double* x1, double a0, double a1, void* out,
                              void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, x0 && x1 && out, "pack_input: NULL pointer");
  k_pack_input<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(x0, x1, ctx->n, a0, a1, static_cast<__nv_bfloat16*>(out));
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

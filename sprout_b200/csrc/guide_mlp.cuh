// The guiding network on one tile of 128 samples per thread block: forward pass, loss
// gradient at the outputs, backward pass with per-block weight-gradient partials.
//
// Operands live in shared memory as BF16 in the K-major "core matrix" layout of the tensor
// cores (8 rows x 8 elements = 128 contiguous bytes per core matrix, core matrices K-fastest):
// element (r, k) of an R x K operand sits at ((r/8)*(K/8) + k/8)*64 + (r%8)*8 + k%8.  The
// products here run on the CUDA cores with FP32 accumulation.  Blocks are 256 threads.
#pragma once

#include <cuda_bf16.h>

#include "guide.cuh"

namespace spb::guide {

constexpr int Block = 256;

__device__ __forceinline__ int tiled(int r, int k, int K) {
    return (((r >> 3) * (K >> 3) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

// Padded row count of a layer's weight tile (outputs rounded up to 16).
__host__ __device__ constexpr int padded_out(int l) { return (out_dim(l) + 15) & ~15; }
__host__ __device__ constexpr int weight_tile_offset(int l) {
    int o = 0;
    for (int k = 0; k < l; ++k) {
        o += padded_out(k) * in_dim(k);
    }
    return o;
}
constexpr int Weight_tile_elems = weight_tile_offset(Layers);  // 17,408 BF16
constexpr int Bias_count        = 4 * Width + Outputs;          // 296
constexpr int Out_stride        = Outputs + 1;  // FP32 rows padded by one word (bank spread)

struct Net_smem {
    __nv_bfloat16 w[Weight_tile_elems];  // all layers' weights, tiled
    float         b[Bias_count];         // all layers' biases
};

// Loads the BF16 weights (packed per layer, out x in row-major) and FP32 biases (from the
// packed parameter vector) into shared memory.
__device__ inline void load_net(Net_smem& s, __nv_bfloat16 const* __restrict__ wbf,
                                float const* __restrict__ params) {
    int src = 0;
    for (int l = 0; l < Layers; ++l) {
        int const K = in_dim(l), N = out_dim(l), P = padded_out(l);
        __nv_bfloat16* dst = s.w + weight_tile_offset(l);
        for (int i = threadIdx.x; i < P * K; i += Block) {
            int const n = i / K, k = i % K;
            dst[tiled(n, k, K)] = n < N ? wbf[src + n * K + k] : __float2bfloat16(0.f);
        }
        src += N * K;
    }
    int bo = 0;
    for (int l = 0; l < Layers; ++l) {
        for (int i = threadIdx.x; i < out_dim(l); i += Block) {
            s.b[bo + i] = params[bias_offset(l) + i];
        }
        bo += out_dim(l);
    }
}

__host__ __device__ constexpr int bias_slot(int l) {
    int o = 0;
    for (int k = 0; k < l; ++k) {
        o += out_dim(k);
    }
    return o;
}

// out = act(A W^T + b) for the tile: A (128 x K, tiled BF16), W (P x K, tiled BF16).  Hidden
// layers write ReLU'd BF16 into `act` (128 x N, tiled); the last layer writes FP32 into
// `out` (128 rows of Out_stride floats).  Thread t computes row t % 128, half t / 128 of the
// columns.
template <int K, int N, bool Last>
__device__ inline void layer_forward(__nv_bfloat16 const* A, __nv_bfloat16 const* W, float const* b,
                                     __nv_bfloat16* act, float* out) {
    int const r  = threadIdx.x & (Tile - 1);
    int const n0 = (threadIdx.x >> 7) * (N / 2);
    float     a[K];
#pragma unroll
    for (int k = 0; k < K; k += 8) {
        uint4 const v = *reinterpret_cast<uint4 const*>(A + tiled(r, k, K));
        __nv_bfloat162 const* h = reinterpret_cast<__nv_bfloat162 const*>(&v);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float2 const f = __bfloat1622float2(h[j]);
            a[k + 2 * j]     = f.x;
            a[k + 2 * j + 1] = f.y;
        }
    }
    for (int n = n0; n < n0 + N / 2; ++n) {
        float acc = b[n];
#pragma unroll
        for (int k = 0; k < K; k += 8) {
            uint4 const v = *reinterpret_cast<uint4 const*>(W + tiled(n, k, K));
            __nv_bfloat162 const* h = reinterpret_cast<__nv_bfloat162 const*>(&v);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float2 const f = __bfloat1622float2(h[j]);
                acc            = fmaf(a[k + 2 * j], f.x, acc);
                acc            = fmaf(a[k + 2 * j + 1], f.y, acc);
            }
        }
        if (Last) {
            out[r * Out_stride + n] = acc;
        } else {
            act[tiled(r, n, N)] = __float2bfloat16(fmaxf(acc, 0.f));
        }
    }
}

// Forward through all layers: acts[0] holds the tile's inputs (128 x 32, tiled); acts[1..4]
// receive the hidden activations; out the 40 outputs per sample.  Ends with a barrier.
__device__ inline void forward(Net_smem const& s, __nv_bfloat16* const acts[Layers], float* out) {
    layer_forward<Inputs, Width, false>(acts[0], s.w + weight_tile_offset(0), s.b + bias_slot(0), acts[1], nullptr);
    __syncthreads();
    layer_forward<Width, Width, false>(acts[1], s.w + weight_tile_offset(1), s.b + bias_slot(1), acts[2], nullptr);
    __syncthreads();
    layer_forward<Width, Width, false>(acts[2], s.w + weight_tile_offset(2), s.b + bias_slot(2), acts[3], nullptr);
    __syncthreads();
    layer_forward<Width, Width, false>(acts[3], s.w + weight_tile_offset(3), s.b + bias_slot(3), acts[4], nullptr);
    __syncthreads();
    layer_forward<Width, Outputs, true>(acts[4], s.w + weight_tile_offset(4), s.b + bias_slot(4), nullptr, out);
    __syncthreads();
}

// Gradient of scale * (-log q(d)) with respect to one sample's 40 outputs o (mixture from
// guide.cuh; the log-concentration has zero gradient where it is clamped).
__device__ inline void output_gradient(float const* o, shading::V3 d, float scale, float* g) {
    Lobe lobes[Lobes];
    mixture(o, lobes);
    float v[Lobes];
    float q = 0.f;
    for (int j = 0; j < Lobes; ++j) {
        v[j] = vmf_pdf(lobes[j], d);
        q += lobes[j].weight * v[j];
    }
    q = fmaxf(q, 1e-30f);
    for (int j = 0; j < Lobes; ++j) {
        float const r     = lobes[j].weight * v[j] / q;
        float const kappa = lobes[j].kappa;
        float const c     = shading::dot(lobes[j].mu, d);
        g[32 + j]         = scale * (lobes[j].weight - r);
        float const lk    = o[4 * j + 3];
        if (lk > Log_kappa_min && lk < Log_kappa_max) {
            float const x2   = 2.f * kappa;
            float const dlog = 1.f - x2 / expm1f(x2) + kappa * (c - 1.f);
            g[4 * j + 3]     = -scale * r * dlog;
        } else {
            g[4 * j + 3] = 0.f;
        }
        float const m0 = o[4 * j], m1 = o[4 * j + 1], m2 = o[4 * j + 2];
        float const l2 = m0 * m0 + m1 * m1 + m2 * m2;
        float const f  = l2 > 1e-20f ? -scale * r * kappa * rsqrtf(l2) : 0.f;
        g[4 * j]       = f * (d.x - lobes[j].mu.x * c);
        g[4 * j + 1]   = f * (d.y - lobes[j].mu.y * c);
        g[4 * j + 2]   = f * (d.z - lobes[j].mu.z * c);
    }
}

// Backward through layer l of the tile.  dz: d loss / d z_l (128 rows of N + 1 floats).
// Writes this block's sums of the weight and bias gradients to gw (N x K) and gb (N) and, when
// dz_prev is given, d loss / d z_{l-1} (128 rows of K + 1 floats; ReLU mask from A > 0).
// A: the layer's input activations (128 x K, tiled BF16); W: its weights (tiled).
template <int K, int N>
__device__ inline void layer_backward(__nv_bfloat16 const* A, __nv_bfloat16 const* W, float const* dz,
                                      float* dz_prev, float* gw, float* gb) {
    constexpr int S      = N + 1;
    constexpr int groups = Block / K;
    int const     k      = threadIdx.x % K;
    for (int n = threadIdx.x / K; n < N; n += groups) {
        float acc = 0.f;
        for (int r = 0; r < Tile; ++r) {
            acc = fmaf(dz[r * S + n], __bfloat162float(A[tiled(r, k, K)]), acc);
        }
        gw[n * K + k] = acc;
    }
    for (int n = threadIdx.x; n < N; n += Block) {
        float acc = 0.f;
        for (int r = 0; r < Tile; ++r) {
            acc += dz[r * S + n];
        }
        gb[n] = acc;
    }
    if (dz_prev) {
        int const r  = threadIdx.x & (Tile - 1);
        int const k0 = (threadIdx.x >> 7) * (K / 2);
        for (int kk = k0; kk < k0 + K / 2; ++kk) {
            float acc = 0.f;
            for (int n = 0; n < N; ++n) {
                acc = fmaf(dz[r * S + n], __bfloat162float(W[tiled(n, kk, K)]), acc);
            }
            dz_prev[r * (K + 1) + kk] = __bfloat162float(A[tiled(r, kk, K)]) > 0.f ? acc : 0.f;
        }
    }
}

}  // namespace spb::guide

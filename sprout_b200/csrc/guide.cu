// Path-guiding network kernels (guide_mlp.cuh): batched forward, per-block gradient partials
// with a deterministic reduction, Adam, and the C-ABI entry points that expose the forward
// pass and the gradient to tests.  The renderer's use (inference per path vertex, training on
// the tracer's own samples) is in render.cu; the network's state is guide::Network.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/sprout_b200.h"
#include "common.hpp"
#include "guide.hpp"
#include "guide_mlp.cuh"

namespace spb::guide {

namespace {

// Shared memory of the tile kernels: the network, the five layer inputs (BF16, tiled) and two
// FP32 gradient / output buffers of 128 rows of up to 65 floats.
struct Train_smem {
    Net_smem      net;
    __nv_bfloat16 a0[Tile * Inputs];
    __nv_bfloat16 a[4][Tile * Width];
    float         za[Tile * (Width + 1)];
    float         zb[Tile * (Width + 1)];
    uint64_t      mbar;       // tensor-core completion barrier
    uint32_t      tmem_slot;  // accumulator address written by tcgen05.alloc
};

// Loads rows [base, base + 128) of an n x 32 FP32 input matrix into the tiled BF16 a0 (rows
// past n are zero).
__device__ inline void load_inputs(__nv_bfloat16* a0, float const* __restrict__ in, uint64_t base, uint64_t n) {
    for (int i = threadIdx.x; i < Tile * Inputs; i += Block) {
        int const      r = i / Inputs, k = i % Inputs;
        uint64_t const g = base + r;
        a0[tiled(r, k, Inputs)] = __float2bfloat16(g < n ? in[g * Inputs + k] : 0.f);
    }
}

// Forward pass on the tensor cores (the renderer's inference path, guide_mlp.cuh).
__global__ void __launch_bounds__(Block) k_forward(__nv_bfloat16 const* wbf, float const* params,
                                                   float const* in, uint64_t n, float* out, uint32_t* error) {
    extern __shared__ __align__(16) unsigned char raw[];
    Train_smem& s = *reinterpret_cast<Train_smem*>(raw);
    load_net(s.net, wbf, params);
    uint64_t const base = uint64_t(blockIdx.x) * Tile;
    load_inputs(s.a0, in, base, n);
    fence_async_smem();
    Tmem_tile tm = tc_setup(&s.tmem_slot, &s.mbar, error);
    __nv_bfloat16* const acts[Layers] = {s.a0, s.a[0], s.a[1], s.a[2], s.a[3]};
    forward_tc(s.net, acts, s.za, tm);
    tc_teardown(tm);
    for (int i = threadIdx.x; i < Tile * Outputs; i += Block) {
        int const      r = i / Outputs, j = i % Outputs;
        uint64_t const g = base + r;
        if (g < n) {
            out[g * Outputs + j] = s.za[r * Out_stride + j];
        }
    }
}

// ---- training on the tensor cores ----
// A persistent kernel: one block per SM walks tiles of 128 samples.  Per tile: forward as in
// inference (keeping every layer's input), the loss gradient at the outputs, then per layer l
// from the last: dW_l += dZ_l^T A_l (M = 128 over the neurons, padded with zero rows; both
// operands MN-major) and dA_l = dZ_l W_l (M = 128 over the samples; dZ K-major, W MN-major),
// committed together; dZ_{l-1} = dA_l masked by ReLU.  Every layer's dW accumulator stays in
// tensor memory across the block's tiles and is written out once, as the block's partial sum.
// dZ is held as BF16 in a 128 x 128 tiled buffer whose columns past the layer's width stay 0;
// bias gradients are summed in FP32 before the rounding (warp reductions, then shared memory).
constexpr int Zw = 128;  // dZ buffer width

struct Train_tc_smem {
    Net_smem      net;
    __nv_bfloat16 a0[Tile * Inputs];
    __nv_bfloat16 a[4][Tile * Width];
    __nv_bfloat16 z[2][Tile * Zw];
    float         gb[Bias_count];
    float         red[2][8][32];  // per-warp column sums, alternating between layers
    float         qpart[2][Tile];  // each half's share of the mixture density per sample
    uint64_t      mbar;
    uint32_t      tmem_slot;
};

// TMEM columns: [0, 64) the forward / dA accumulator; then each layer's dW accumulator.
constexpr uint32_t Train_tmem_columns = 512;
__host__ __device__ constexpr uint32_t dw_column(int l) {
    return l == 0 ? 64u : 96u + 64u * uint32_t(l - 1);  // 64 (32 wide), 96, 160, 224, 288 (64 wide)
}

// Sum over a warp's 32 lanes (rows) of each of its 32 registers (columns), by recursive halving:
// afterwards v[0] of lane j holds the total of column j.
__device__ inline float warp_column_sums(float v[32]) {
    int const lane = threadIdx.x & 31;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        bool const upper = lane & w;
#pragma unroll
        for (int i = 0; i < w; ++i) {
            float const send = upper ? v[i] : v[i + w];
            float const keep = upper ? v[i + w] : v[i];
            v[i]             = keep + __shfl_xor_sync(0xFFFFFFFFu, send, w);
        }
    }
    return v[0];
}

// The output layer of a training tile, by all threads, after its MMA was issued: thread t
// takes sample r = t % 128 and lobes 4h..4h+3 (h = t / 128).  From the accumulator plus bias it
// forms the mixture (softmax weights of all lobes; unit mean and concentration of its own),
// adds its lobes' share of q(d) = sum_j w_j vMF_j(d), exchanges it with the other half, and
// writes the gradient of scale * (-log q(d)) with respect to its 20 outputs as BF16 dZ
// columns (columns 40..63 are cleared); the log-concentration has zero gradient where it is
// clamped.  The per-warp column sums of the FP32 gradient go to red (the output bias
// gradient).  Ends with a barrier.
__device__ inline void finish_output_gradient(Train_tc_smem& s, float const* b, shading::V3 d, float scale,
                                              float (&red)[8][32], Tmem_tile& tm) {
    if (!mbar_wait(tm.mbar, tm.phase)) {
        *tm.error = 1u;
    }
    tm.phase ^= 1u;
    tc_fence_after();
    int const      warp  = threadIdx.x >> 5;
    int const      r     = threadIdx.x & (Tile - 1);
    int const      h     = threadIdx.x >> 7;
    uint32_t const lanes = uint32_t(32 * (warp & 3)) << 16;
    float          o[16], logit[Lobes];
    tmem_ld16(tm.tmem + lanes + uint32_t(16 * h), o);
    tmem_ld8(tm.tmem + lanes + 32u, logit);
    float mx = -3.4e38f;
#pragma unroll
    for (int j = 0; j < Lobes; ++j) {
        logit[j] += b[32 + j];
        mx = fmaxf(mx, logit[j]);
    }
    float sum = 0.f, w[4];
#pragma unroll
    for (int j = 0; j < Lobes; ++j) {
        float const e = expf(logit[j] - mx);
        sum += e;
        if (j / 4 == h) {
            w[j % 4] = e;
        }
    }
    float mu[4][3], kappa[4], c[4], v[4], q = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            o[4 * j + k] += b[16 * h + 4 * j + k];
        }
        w[j] /= sum;
        float const l2  = o[4 * j] * o[4 * j] + o[4 * j + 1] * o[4 * j + 1] + o[4 * j + 2] * o[4 * j + 2];
        float const inv = l2 > 1e-20f ? 1.f / sqrtf(l2) : 0.f;
        mu[j][0]        = l2 > 1e-20f ? inv * o[4 * j] : 0.f;
        mu[j][1]        = l2 > 1e-20f ? inv * o[4 * j + 1] : 0.f;
        mu[j][2]        = l2 > 1e-20f ? inv * o[4 * j + 2] : 1.f;
        kappa[j]        = expf(fminf(fmaxf(o[4 * j + 3], Log_kappa_min), Log_kappa_max));
        c[j]            = mu[j][0] * d.x + mu[j][1] * d.y + mu[j][2] * d.z;
        float const nrm = kappa[j] / (2.f * 3.14159265358979f * -expm1f(-2.f * kappa[j]));
        v[j]            = nrm * expf(kappa[j] * (c[j] - 1.f));
        q += w[j] * v[j];
    }
    s.qpart[h][r] = q;
    __syncthreads();
    q = fmaxf(s.qpart[0][r] + s.qpart[1][r], 1e-30f);
    float g[32];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float const rj = w[j] * v[j] / q;
        g[16 + j]      = scale * (w[j] - rj);
        float const lk = o[4 * j + 3];
        if (lk > Log_kappa_min && lk < Log_kappa_max) {
            float const x2 = 2.f * kappa[j];
            g[4 * j + 3]   = -scale * rj * (1.f - x2 / expm1f(x2) + kappa[j] * (c[j] - 1.f));
        } else {
            g[4 * j + 3] = 0.f;
        }
        float const l2 = o[4 * j] * o[4 * j] + o[4 * j + 1] * o[4 * j + 1] + o[4 * j + 2] * o[4 * j + 2];
        float const f  = l2 > 1e-20f ? -scale * rj * kappa[j] * rsqrtf(l2) : 0.f;
        g[4 * j]       = f * (d.x - mu[j][0] * c[j]);
        g[4 * j + 1]   = f * (d.y - mu[j][1] * c[j]);
        g[4 * j + 2]   = f * (d.z - mu[j][2] * c[j]);
    }
    // dZ row r: lobe columns 16h..16h+15, logit columns 32+4h..32+4h+3, zeros in 40..63
    __nv_bfloat162 hv[8];
#pragma unroll
    for (int q2 = 0; q2 < 8; ++q2) {
        hv[q2] = __floats2bfloat162_rn(g[2 * q2], g[2 * q2 + 1]);
    }
    *reinterpret_cast<uint4*>(&s.z[0][tiled(r, 16 * h, Zw)])     = *reinterpret_cast<uint4*>(hv);
    *reinterpret_cast<uint4*>(&s.z[0][tiled(r, 16 * h + 8, Zw)]) = *reinterpret_cast<uint4*>(hv + 4);
    __nv_bfloat162 const lg[2] = {__floats2bfloat162_rn(g[16], g[17]), __floats2bfloat162_rn(g[18], g[19])};
    *reinterpret_cast<uint2*>(&s.z[0][tiled(r, 32 + 4 * h, Zw)]) = *reinterpret_cast<uint2 const*>(lg);
    uint4 const zero = make_uint4(0u, 0u, 0u, 0u);
    if (h == 0) {
        *reinterpret_cast<uint4*>(&s.z[0][tiled(r, 40, Zw)]) = zero;
        *reinterpret_cast<uint4*>(&s.z[0][tiled(r, 48, Zw)]) = zero;
    } else {
        *reinterpret_cast<uint4*>(&s.z[0][tiled(r, 56, Zw)]) = zero;
    }
    fence_async_smem();
#pragma unroll
    for (int k = 20; k < 32; ++k) {
        g[k] = 0.f;
    }
    red[warp][threadIdx.x & 31] = warp_column_sums(g);
    tc_fence_before();
    __syncthreads();
}

// Issues the layer's dW (accumulating unless `fresh`) and, when with_da, its dA; thread 0.
template <int K, int N>
__device__ inline void backward_mma(uint32_t tmem, uint32_t dw_col, __nv_bfloat16 const* z, __nv_bfloat16 const* act,
                                    __nv_bfloat16 const* w, bool with_da, bool fresh, uint32_t mbar) {
    constexpr int P = (N + 15) & ~15;
    tc_fence_after();
    uint32_t const zs = smem_u32(z), as = smem_u32(act), ws = smem_u32(w);
    // dW[n][k] += sum_r dZ[r][n] A[r][k]: A operand dZ^T (MN-major: n groups 128 B apart, r groups
    // Zw * 16 B apart), B operand A_l (MN-major: k groups 128 B, r groups K * 16 B).
#pragma unroll
    for (int s = 0; s < Tile / 16; ++s) {
        umma_bf16(tmem + dw_col, operand_desc(zs + 2u * Zw * 16u * s, Zw * 16u, 128u),
                  operand_desc(as + 2u * K * 16u * s, K * 16u, 128u), instr_desc(Tile, K, true, true),
                  (fresh && s == 0) ? 0u : 1u);
    }
    if (with_da) {
        // dA[r][k] = sum_n dZ[r][n] W[n][k]: A operand dZ (K-major over n), B operand W_l
        // (MN-major: k groups 128 B, n groups K * 16 B).
#pragma unroll
        for (int s = 0; s < P / 16; ++s) {
            umma_bf16(tmem, operand_desc(zs + 256u * s, 128u, Zw * 16u),
                      operand_desc(ws + 2u * K * 16u * s, K * 16u, 128u), instr_desc(Tile, K, false, true), s > 0);
        }
    }
    umma_commit(mbar);
}

// Inputs: Tiled_inputs, BF16 tiles of 128 samples in operand order (8 KB each); else FP32,
// 32 per sample.
template <bool Tiled_inputs>
__global__ void __launch_bounds__(Block) k_gradients_tc(__nv_bfloat16 const* wbf, float const* params,
                                                        void const* in, float const* dirs, float const* scale,
                                                        uint64_t n, uint32_t tiles, float* partial, uint32_t* error) {
    extern __shared__ __align__(16) unsigned char raw[];
    Train_tc_smem& s = *reinterpret_cast<Train_tc_smem*>(raw);
    load_net(s.net, wbf, params);
    for (int i = threadIdx.x; i < 2 * Tile * Zw / 8; i += Block) {
        reinterpret_cast<uint4*>(s.z)[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    for (int i = threadIdx.x; i < Bias_count; i += Block) {
        s.gb[i] = 0.f;
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem_slot)),
                     "r"(Train_tmem_columns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s.mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    Tmem_tile tm{s.tmem_slot, smem_u32(&s.mbar), 0u, error};

    __nv_bfloat16* const acts[Layers] = {s.a0, s.a[0], s.a[1], s.a[2], s.a[3]};
    int const            r     = threadIdx.x & (Tile - 1);
    int const            warp  = threadIdx.x >> 5;
    int const            lane  = threadIdx.x & 31;
    uint32_t const       lanes = uint32_t(32 * (warp & 3)) << 16;
    bool                 fresh = true;  // no dW accumulated yet
#pragma unroll 1
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        uint64_t const base = uint64_t(tile) * Tile;
        if constexpr (Tiled_inputs) {
            uint4 const* const src = static_cast<uint4 const*>(in) + uint64_t(tile) * (Tile * Inputs / 8);
            uint4* const       dst = reinterpret_cast<uint4*>(s.a0);
            dst[threadIdx.x]         = src[threadIdx.x];
            dst[Block + threadIdx.x] = src[Block + threadIdx.x];
        } else {
            load_inputs(s.a0, static_cast<float const*>(in), base, n);
        }
        uint64_t const   g     = base + r;
        float const      sc    = g < n ? scale[g] : 0.f;
        shading::V3 const d    = g < n ? shading::v3(dirs[3 * g], dirs[3 * g + 1], dirs[3 * g + 2])
                                       : shading::v3(0.f, 0.f, 1.f);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // forward (hidden layers), then the output layer and the loss gradient -> dZ_4
        layer_forward_tc<Inputs, Width, false>(acts[0], s.net.w + weight_tile_offset(0), s.net.b + bias_slot(0),
                                               acts[1], Smem_outputs{nullptr}, tm);
#pragma unroll
        for (int l = 1; l < Layers - 1; ++l) {
            layer_forward_tc<Width, Width, false>(acts[l], s.net.w + weight_tile_offset(l), s.net.b + bias_slot(l),
                                                  acts[l + 1], Smem_outputs{nullptr}, tm);
        }
        issue_layer<Width, Outputs>(acts[4], s.net.w + weight_tile_offset(4), tm);
        finish_output_gradient(s, s.net.b + bias_slot(4), d, sc, s.red[1], tm);
        if (threadIdx.x < Outputs) {
            // output bias gradient: column c lies in half h at local column lc
            int const c  = threadIdx.x;
            int const h  = c < 32 ? c / 16 : (c - 32) / 4;
            int const lc = c < 32 ? c % 16 : 16 + (c - 32) % 4;
            s.gb[bias_slot(4) + c] += s.red[1][4 * h][lc] + s.red[1][4 * h + 1][lc] + s.red[1][4 * h + 2][lc] +
                                      s.red[1][4 * h + 3][lc];
        }

        int cur = 0;  // dZ buffer of the current layer
#pragma unroll 1
        for (int l = Layers - 1; l >= 0; --l) {
            if (threadIdx.x == 0) {
                __nv_bfloat16 const* w = s.net.w + weight_tile_offset(l);
                if (l == 4) {
                    backward_mma<Width, Outputs>(tm.tmem, dw_column(l), s.z[cur], acts[l], w, true, fresh, tm.mbar);
                } else if (l > 0) {
                    backward_mma<Width, Width>(tm.tmem, dw_column(l), s.z[cur], acts[l], w, true, fresh, tm.mbar);
                } else {
                    backward_mma<Inputs, Width>(tm.tmem, dw_column(l), s.z[cur], acts[l], w, false, fresh, tm.mbar);
                }
            }
            if (!mbar_wait(tm.mbar, tm.phase)) {
                *tm.error = 1u;
            }
            tm.phase ^= 1u;
            tc_fence_after();
            if (l > 0) {
                // dZ_{l-1} = dA masked by the ReLU of layer l's input (K = 64 columns: thread
                // row r, half t / 128).
                int const nxt = cur ^ 1;
                int const k0  = (threadIdx.x >> 7) * (Width / 2);
                float     v[32];
                tmem_ld32(tm.tmem + lanes + uint32_t(k0), v);
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    __nv_bfloat162 h[4];
                    uint4 const    in8 = *reinterpret_cast<uint4 const*>(&acts[l][tiled(r, k0 + j, Width)]);
                    __nv_bfloat16 const* a8 = reinterpret_cast<__nv_bfloat16 const*>(&in8);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (!(__bfloat162float(a8[q]) > 0.f)) {
                            v[j + q] = 0.f;
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        h[q] = __floats2bfloat162_rn(v[j + 2 * q], v[j + 2 * q + 1]);
                    }
                    *reinterpret_cast<uint4*>(&s.z[nxt][tiled(r, k0 + j, Zw)]) = *reinterpret_cast<uint4*>(h);
                }
                fence_async_smem();
                s.red[l & 1][warp][lane] = warp_column_sums(v);
                cur = nxt;
            }
            tc_fence_before();
            __syncthreads();
            if (l > 0 && threadIdx.x < Width) {
                // bias gradient of layer l - 1: column c = t, from the four warps on its half
                int const c = threadIdx.x, h = c >> 5;
                float const(&red)[8][32] = s.red[l & 1];
                s.gb[bias_slot(l - 1) + c] += red[4 * h][c & 31] + red[4 * h + 1][c & 31] + red[4 * h + 2][c & 31] +
                                              red[4 * h + 3][c & 31];
            }
        }
        fresh = false;
    }

    // The block's partial sums: dW from tensor memory (thread row n, half of the columns),
    // biases from shared memory.
    float* const pout = partial + uint64_t(blockIdx.x) * Parameters;
    __syncthreads();
#pragma unroll 1
    for (int l = 0; l < Layers; ++l) {
        int const K  = in_dim(l), N = out_dim(l);
        int const k0 = (threadIdx.x >> 7) * (K / 2);
        float     v[32];
        if (K == Width) {
            tmem_ld32(tm.tmem + lanes + dw_column(l) + uint32_t(k0), v);
        } else {
            tmem_ld8(tm.tmem + lanes + dw_column(l) + uint32_t(k0), v);
            tmem_ld8(tm.tmem + lanes + dw_column(l) + uint32_t(k0) + 8u, v + 8);
        }
        if (r < N) {
            float* const dst = pout + weight_offset(l) + r * K + k0;
            for (int i = 0; i < K / 2; ++i) {
                dst[i] = fresh ? 0.f : v[i];
            }
        }
    }
    for (int l = 0; l < Layers; ++l) {
        for (int i = threadIdx.x; i < out_dim(l); i += Block) {
            pout[bias_offset(l) + i] = s.gb[bias_slot(l) + i];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm.tmem), "r"(Train_tmem_columns));
    }
}

// grads[p] = sum over blocks of partial[b][p], in block order (deterministic); divided by the
// total of weight_parts when given (the batch's loss weights, summed in a fixed order).
__global__ void k_reduce(float const* partial, uint32_t blocks, float const* weight_parts, uint32_t num_parts,
                         float* grads, uint32_t* step_counter) {
    if (step_counter && blockIdx.x == 0 && threadIdx.x == 0) {
        ++*step_counter;  // the Adam step that follows (k_adam_counted reads it)
    }
    __shared__ float total;
    if (threadIdx.x < 32) {
        float acc = 0.f;
        if (weight_parts) {
            for (uint32_t i = threadIdx.x; i < num_parts; i += 32) {
                acc += weight_parts[i];
            }
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        }
        if (threadIdx.x == 0) {
            total = acc;
        }
    }
    __syncthreads();
    uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= uint32_t(Parameters)) {
        return;
    }
    float acc = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) {
        acc += partial[uint64_t(b) * Parameters + p];
    }
    grads[p] = !weight_parts ? acc : (total > 0.f ? acc / total : 0.f);
}

// Index of parameter p in the BF16 weight array, or -1 for a bias.
__device__ inline int bf16_index(int p) {
    int w = 0;
    for (int l = 0; l < Layers; ++l) {
        if (p < weight_offset(l + 1)) {
            return p < bias_offset(l) ? w + (p - weight_offset(l)) : -1;
        }
        w += out_dim(l) * in_dim(l);
    }
    return -1;
}

__global__ void k_to_bf16(float const* params, __nv_bfloat16* wbf) {
    int const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < Parameters) {
        int const i = bf16_index(p);
        if (i >= 0) {
            wbf[i] = __float2bfloat16(params[p]);
        }
    }
}

// Adam (Kingma and Ba 2015) on the FP32 master parameters; refreshes the BF16 weights.
__global__ void k_adam(float* params, float* m, float* v, float const* grads, float lr, float c1, float c2,
                       __nv_bfloat16* wbf) {
    int const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Parameters) {
        return;
    }
    float const g  = grads[p];
    float const mm = 0.9f * m[p] + 0.1f * g;
    float const vv = 0.999f * v[p] + 0.001f * g * g;
    m[p]           = mm;
    v[p]           = vv;
    float const w  = params[p] - lr * (mm * c1) / (sqrtf(vv * c2) + 1e-8f);
    params[p]      = w;
    int const i    = bf16_index(p);
    if (i >= 0) {
        wbf[i] = __float2bfloat16(w);
    }
}

// Adam with its step count in device memory (counted by k_reduce), so that training steps can
// be replayed from a captured graph; block 0 also advances `advance` (the caller's batch
// counter) when given, after every reader of it has run.
__global__ void k_adam_counted(float* params, float* m, float* v, float const* grads, float lr,
                               uint32_t const* step_counter, uint32_t* advance, __nv_bfloat16* wbf) {
    int const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (advance && p == 0) {
        ++*advance;
    }
    if (p >= Parameters) {
        return;
    }
    float const step = float(max(*step_counter, 1u));
    float const c1   = 1.f / (1.f - powf(0.9f, step));
    float const c2   = 1.f / (1.f - powf(0.999f, step));
    float const g    = grads[p];
    float const mm   = 0.9f * m[p] + 0.1f * g;
    float const vv   = 0.999f * v[p] + 0.001f * g * g;
    m[p]             = mm;
    v[p]             = vv;
    float const w    = params[p] - lr * (mm * c1) / (sqrtf(vv * c2) + 1e-8f);
    params[p]        = w;
    int const i      = bf16_index(p);
    if (i >= 0) {
        wbf[i] = __float2bfloat16(w);
    }
}

}  // namespace

size_t tile_smem_bytes() {
    return sizeof(Train_smem);
}

namespace {

template <typename T>
void release(T*& p) {
    if (p) {
        cudaFree(p);
        p = nullptr;
    }
}

int set_kernel_attributes() {
    static int const status = [] {
        int const bytes = int(tile_smem_bytes());
        cudaError_t e   = cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e == cudaSuccess) {
            e = cudaFuncSetAttribute(k_gradients_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(sizeof(Train_tc_smem)));
        }
        if (e == cudaSuccess) {
            e = cudaFuncSetAttribute(k_gradients_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(sizeof(Train_tc_smem)));
        }
        return int(e);
    }();
    return status;
}

}  // namespace

Network::~Network() {
    release(params_);
    release(m_);
    release(v_);
    release(grads_);
    release(wbf_);
    release(partial_);
    release(error_);
    release(step_dev_);
}

int Network::init(uint32_t seed) {
    // He-uniform weights (limit sqrt(6 / fan_in)), zero biases.
    std::vector<float> host(Parameters, 0.f);
    std::mt19937       g(seed);
    for (int l = 0; l < Layers; ++l) {
        std::uniform_real_distribution<float> u(-std::sqrt(6.f / in_dim(l)), std::sqrt(6.f / in_dim(l)));
        for (int i = 0; i < out_dim(l) * in_dim(l); ++i) {
            host[weight_offset(l) + i] = u(g);
        }
    }
    return set_parameters(host.data());
}

int Network::set_parameters(float const* host) {
    if (int const e = set_kernel_attributes()) {
        return e;
    }
    size_t const bytes = Parameters * sizeof(float);
    for (float** p : {&params_, &m_, &v_, &grads_}) {
        if (!*p) {
            if (cudaError_t const e = cudaMalloc(p, bytes)) {
                return e;
            }
        }
    }
    if (!wbf_) {
        if (cudaError_t const e = cudaMalloc(&wbf_, Parameters * sizeof(__nv_bfloat16))) {
            return e;
        }
    }
    if (!step_dev_) {
        if (cudaError_t const e = cudaMalloc(&step_dev_, sizeof(uint32_t))) {
            return e;
        }
    }
    cudaError_t e = cudaMemcpy(params_, host, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m_, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(v_, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(grads_, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(step_dev_, 0, sizeof(uint32_t));
    if (e != cudaSuccess) {
        return e;
    }
    step_ = 0;
    k_to_bf16<<<(Parameters + 255) / 256, 256>>>(params_, wbf_);
    return cudaGetLastError();
}

bool Network::timed_out() const {
    uint32_t flag = 0;
    if (error_) {
        cudaMemcpy(&flag, error_, sizeof(flag), cudaMemcpyDeviceToHost);
    }
    return flag != 0;
}

int Network::get_parameters(float* host) const {
    return cudaMemcpy(host, params_, Parameters * sizeof(float), cudaMemcpyDeviceToHost);
}

int Network::forward(float const* inputs, uint64_t n, float* outputs, cudaStream_t stream) {
    if (n == 0) {
        return 0;
    }
    uint64_t const blocks = (n + Tile - 1) / Tile;
    if (!error_) {
        if (cudaError_t const e = cudaMalloc(&error_, sizeof(uint32_t))) {
            return e;
        }
    }
    cudaError_t e = cudaMemsetAsync(error_, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) {
        return e;
    }
    k_forward<<<unsigned(blocks), Block, tile_smem_bytes(), stream>>>(wbf_, params_, inputs, n, outputs, error_);
    uint32_t flag = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, error_, sizeof(flag), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && flag) {
        return int(cudaErrorLaunchTimeout);  // a tensor-core completion wait ran out
    }
    return e;
}

int Network::gradients(float const* inputs, float const* dirs, float const* scale, uint64_t n,
                       cudaStream_t stream) {
    return run_gradients(inputs, false, dirs, scale, n, nullptr, 0, stream);
}

int Network::gradients_tiled(__nv_bfloat16 const* tiles, float const* dirs, float const* weights, uint64_t n,
                             float const* weight_parts, uint32_t num_parts, cudaStream_t stream) {
    return run_gradients(tiles, true, dirs, weights, n, weight_parts, num_parts, stream);
}

int Network::run_gradients(void const* inputs, bool tiled, float const* dirs, float const* scale, uint64_t n,
                           float const* weight_parts, uint32_t num_parts, cudaStream_t stream) {
    uint64_t const blocks = (n + Tile - 1) / Tile;
    if (blocks == 0) {
        return cudaMemsetAsync(grads_, 0, Parameters * sizeof(float), stream);
    }
    if (int const e = prepare_gradients(n)) {
        return e;
    }
    // one persistent block per SM (at most one per tile)
    uint32_t const grid = uint32_t(std::min<uint64_t>(blocks, partial_blocks_));
    if (tiled) {
        k_gradients_tc<true><<<grid, Block, sizeof(Train_tc_smem), stream>>>(wbf_, params_, inputs, dirs, scale, n,
                                                                             uint32_t(blocks), partial_, error_);
    } else {
        k_gradients_tc<false><<<grid, Block, sizeof(Train_tc_smem), stream>>>(wbf_, params_, inputs, dirs, scale, n,
                                                                              uint32_t(blocks), partial_, error_);
    }
    k_reduce<<<(Parameters + 255) / 256, 256, 0, stream>>>(partial_, grid, weight_parts, num_parts, grads_,
                                                           tiled ? step_dev_ : nullptr);
    return cudaGetLastError();
}

int Network::adam_counted(float lr, uint32_t* advance, cudaStream_t stream) {
    k_adam_counted<<<(Parameters + 255) / 256, 256, 0, stream>>>(params_, m_, v_, grads_, lr, step_dev_, advance,
                                                                 wbf_);
    return cudaGetLastError();
}

int Network::prepare_gradients(uint64_t n) {
    static int const sms = [] {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        return std::max(count, 1);
    }();
    uint64_t const grid = std::min<uint64_t>((n + Tile - 1) / Tile, uint64_t(sms));
    if (grid > partial_blocks_) {
        release(partial_);
        if (cudaError_t const e = cudaMalloc(&partial_, size_t(grid) * Parameters * sizeof(float))) {
            partial_blocks_ = 0;
            return e;
        }
        partial_blocks_ = grid;
    }
    if (!error_) {
        if (cudaError_t const e = cudaMalloc(&error_, sizeof(uint32_t))) {
            return e;
        }
        if (cudaError_t const e = cudaMemset(error_, 0, sizeof(uint32_t))) {
            return e;
        }
    }
    return cudaSuccess;
}

int Network::adam(float lr, cudaStream_t stream) {
    ++step_;
    float const c1 = 1.f / (1.f - std::pow(0.9f, float(step_)));
    float const c2 = 1.f / (1.f - std::pow(0.999f, float(step_)));
    k_adam<<<(Parameters + 255) / 256, 256, 0, stream>>>(params_, m_, v_, grads_, lr, c1, c2, wbf_);
    return cudaGetLastError();
}

}  // namespace spb::guide

// ---- C ABI (include/sprout_b200.h): the network's forward pass and gradient on host data ----

namespace {

template <typename T>
struct Device_copy {
    T*  p = nullptr;
    int status = 0;
    Device_copy(T const* host, size_t count) {
        status = cudaMalloc(&p, count * sizeof(T) + 16);
        if (status == 0 && host) {
            status = cudaMemcpy(p, host, count * sizeof(T), cudaMemcpyHostToDevice);
        }
    }
    ~Device_copy() {
        if (p) {
            cudaFree(p);
        }
    }
};

int32_t cuda_status(int e, char const* what) {
    if (e != 0) {
        return spb::fail(SPB_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(cudaError_t(e)));
    }
    return SPB_OK;
}

}  // namespace

SPB_API int32_t spb_guide_parameter_count(uint32_t* count) {
    if (!count) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_guide_parameter_count: null argument");
    }
    *count = uint32_t(spb::guide::Parameters);
    return SPB_OK;
}

SPB_API int32_t spb_guide_forward(float const* params, float const* inputs, uint64_t n, float* outputs) {
    using namespace spb::guide;
    if (!params || (n && (!inputs || !outputs))) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_guide_forward: null argument");
    }
    Network net;
    if (int32_t const s = cuda_status(net.set_parameters(params), "spb_guide_forward")) {
        return s;
    }
    Device_copy<float> in(inputs, n * Inputs), out(nullptr, n * Outputs);
    if (int32_t const s = cuda_status(in.status ? in.status : out.status, "spb_guide_forward")) {
        return s;
    }
    int e = net.forward(in.p, n, out.p, nullptr);
    if (e == 0) {
        e = cudaMemcpy(outputs, out.p, n * Outputs * sizeof(float), cudaMemcpyDeviceToHost);
    }
    return cuda_status(e, "spb_guide_forward");
}

SPB_API int32_t spb_guide_gradients(float const* params, float const* inputs, float const* directions,
                                    float const* weights, uint64_t n, float* gradient) {
    using namespace spb::guide;
    if (!params || !gradient || (n && (!inputs || !directions || !weights))) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_guide_gradients: null argument");
    }
    Network net;
    if (int32_t const s = cuda_status(net.set_parameters(params), "spb_guide_gradients")) {
        return s;
    }
    std::vector<float> scale(n);
    for (uint64_t i = 0; i < n; ++i) {
        scale[i] = weights[i] / float(n);
    }
    Device_copy<float> in(inputs, n * Inputs), dirs(directions, n * 3), sc(scale.data(), n);
    int e = in.status ? in.status : (dirs.status ? dirs.status : sc.status);
    if (e == 0) {
        e = net.gradients(in.p, dirs.p, sc.p, n, nullptr);
    }
    if (e == 0) {
        e = cudaMemcpy(gradient, net.gradient(), Parameters * sizeof(float), cudaMemcpyDeviceToHost);
    }
    if (e == 0 && net.timed_out()) {
        return spb::fail(SPB_ERROR_CUDA, "spb_guide_gradients: a tensor-core completion wait ran out");
    }
    return cuda_status(e, "spb_guide_gradients");
}

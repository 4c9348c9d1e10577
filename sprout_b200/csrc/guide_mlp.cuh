// The guiding network on one tile of 128 samples per thread block: weights in shared memory,
// the forward pass on the tensor cores (tcgen05), the loss gradient at the outputs.  The
// backward pass is in guide.cu.
//
// Operands live in shared memory as BF16 in the K-major "core matrix" layout of the tensor
// cores (8 rows x 8 elements = 128 contiguous bytes per core matrix, core matrices K-fastest):
// element (r, k) of an R x K operand sits at ((r/8)*(K/8) + k/8)*64 + (r%8)*8 + k%8.
// Accumulation is FP32.  Blocks are 256 threads.
#pragma once

#include <cuda_bf16.h>

#include <cstring>

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
#pragma unroll
    for (int l = 0; l < Layers; ++l) {
        // 16-byte chunks: 8 consecutive inputs of one output row, one core-matrix row
        constexpr uint4 zero = {0u, 0u, 0u, 0u};
        int const       K = in_dim(l), N = out_dim(l), P = padded_out(l);
        __nv_bfloat16*  dst = s.w + weight_tile_offset(l);
        for (int i = threadIdx.x; i < P * K / 8; i += Block) {
            int const n = i / (K / 8), k = 8 * (i % (K / 8));
            *reinterpret_cast<uint4*>(dst + tiled(n, k, K)) =
                n < N ? *reinterpret_cast<uint4 const*>(wbf + src + n * K + k) : zero;
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

// ---- the products on the tensor cores (tcgen05, sm_100a) ----
// One M = 128 tile per layer: the layer's input tile (A, K-major) times its weights (B, K-major)
// accumulated in FP32 in tensor memory (TMEM) by tcgen05.mma (kind::f16, BF16 operands), issued
// by thread 0 in K steps of 16, completion signalled by tcgen05.commit on an mbarrier.  Each
// warp then reads its 32-lane quarter of the accumulator (row = lane) with tcgen05.ld; bias,
// ReLU and the BF16 store for the next layer follow as on the CUDA cores.  Operand descriptors:
// the tiled layout above is the canonical K-major layout without swizzle, leading byte offset
// 128 (the next 8 columns), stride byte offset K * 16 (the next 8 rows).
struct Tmem_tile {
    uint32_t  tmem;   // accumulator: lane 0 of its first column
    uint32_t  mbar;   // shared-memory address of the completion mbarrier
    uint32_t  phase;  // parity of the next completion
    uint32_t* error;  // set to 1 when a completion wait runs out
};

__device__ __forceinline__ uint32_t smem_u32(void const* p) {
    return uint32_t(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle, version 1 (sm_100); offsets in bytes.
__device__ __forceinline__ uint64_t operand_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, M x N, K- or MN-major.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n, bool a_mn = false, bool b_mn = false) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
           (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    uint32_t const mask = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(mask));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes this thread's shared-memory stores visible to the tensor cores' operand reads.
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    return done != 0;
}

// Waits (bounded) for the mbarrier to complete the given phase; false if it never did.  Called
// by whole warps: lane 0 polls, then every lane observes the completed phase itself.
__device__ inline bool mbar_wait(uint32_t mbar, uint32_t phase) {
    bool done = false;
    if ((threadIdx.x & 31) == 0) {
        for (uint32_t i = 0; i < (1u << 22) && !done; ++i) {
            done = mbar_try_wait(mbar, phase);
        }
    }
    __syncwarp();
    return mbar_try_wait(mbar, phase);
}

// 32 / 8 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float v[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

// (max(x, 0), max(y, 0)) rounded to BF16 (x in the low half), in one conversion instruction.
__device__ __forceinline__ __nv_bfloat162 relu_bf16x2(float x, float y) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(y), "f"(x));
    __nv_bfloat162 h;
    std::memcpy(&h, &r, sizeof(r));
    return h;
}

// Stores the 40 outputs of sample r into shared memory (Out_stride floats per sample).
struct Smem_outputs {
    float* out;
    __device__ void operator()(int r, float const (&v)[Outputs]) const {
#pragma unroll
        for (int n = 0; n < Outputs; ++n) {
            out[r * Out_stride + n] = v[n];
        }
    }
};

// One layer on the tensor cores, in two halves.  issue_layer (thread 0): the layer's MMAs into
// the tile's accumulator and a commit to its mbarrier; precondition: A and W are in shared
// memory, every writer fenced its stores for the async proxy, and a block barrier (after
// tc_fence_before) followed.  finish_layer (all threads): waits for the commit, adds the bias,
// applies ReLU and stores the BF16 activations (the last layer: store(r, outputs) by thread
// r < Tile), then fences and ends with a barrier, after which the next layer may be issued.
template <int K, int N>
__device__ inline void issue_layer(__nv_bfloat16 const* A, __nv_bfloat16 const* W, Tmem_tile const& tm) {
    constexpr int P = (N + 15) & ~15;
    if (threadIdx.x == 0) {
        tc_fence_after();
        uint32_t const a0 = smem_u32(A);
        uint32_t const b0 = smem_u32(W);
#pragma unroll
        for (int k = 0; k < K / 16; ++k) {
            umma_bf16(tm.tmem, operand_desc(a0 + 256u * k, 128u, K * 16u), operand_desc(b0 + 256u * k, 128u, K * 16u),
                      instr_desc(Tile, P), k > 0 ? 1u : 0u);
        }
        umma_commit(tm.mbar);
    }
}

template <int N, bool Last, class Store>
__device__ inline void finish_layer(float const* b, __nv_bfloat16* act, Store const& store, Tmem_tile& tm) {
    if (!mbar_wait(tm.mbar, tm.phase)) {
        *tm.error = 1u;
    }
    tm.phase ^= 1u;
    tc_fence_after();
    int const      warp  = threadIdx.x >> 5;
    int const      r     = threadIdx.x & (Tile - 1);
    uint32_t const lanes = uint32_t(32 * (warp & 3)) << 16;
    if constexpr (Last) {
        if (threadIdx.x < Tile) {
            float v[Outputs];
            tmem_ld32(tm.tmem + lanes, v);
            tmem_ld8(tm.tmem + lanes + 32u, v + 32);
#pragma unroll
            for (int n = 0; n < Outputs; ++n) {
                v[n] += b[n];
            }
            store(r, v);
        }
    } else {
        int const n0 = (threadIdx.x >> 7) * (N / 2);  // N = 64: 32 columns per thread
        float     v[32];
        tmem_ld32(tm.tmem + lanes + uint32_t(n0), v);
#pragma unroll
        for (int j = 0; j < 32; j += 8) {
            __nv_bfloat162 h[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                h[q] = relu_bf16x2(v[j + 2 * q] + b[n0 + j + 2 * q], v[j + 2 * q + 1] + b[n0 + j + 2 * q + 1]);
            }
            *reinterpret_cast<uint4*>(act + tiled(r, n0 + j, N)) = *reinterpret_cast<uint4*>(h);
        }
        fence_async_smem();
    }
    tc_fence_before();
    __syncthreads();
}

// Both halves: one layer, results stored, ending with a barrier.
template <int K, int N, bool Last, class Store = Smem_outputs>
__device__ inline void layer_forward_tc(__nv_bfloat16 const* A, __nv_bfloat16 const* W, float const* b,
                                        __nv_bfloat16* act, Store const& store, Tmem_tile& tm) {
    issue_layer<K, N>(A, W, tm);
    finish_layer<N, Last>(b, act, store, tm);
}

// Forward through all layers: acts[0] holds the tile's inputs (128 x 32, tiled); acts[1..4]
// receive the hidden activations (acts may alternate between two buffers); store(r, outputs)
// takes each sample's 40 outputs.  Same entry conditions as layer_forward_tc.
template <class Store>
__device__ inline void forward_tc(Net_smem const& s, __nv_bfloat16* const acts[Layers], Store const& store,
                                  Tmem_tile& tm) {
    layer_forward_tc<Inputs, Width, false>(acts[0], s.w + weight_tile_offset(0), s.b + bias_slot(0), acts[1], store, tm);
    layer_forward_tc<Width, Width, false>(acts[1], s.w + weight_tile_offset(1), s.b + bias_slot(1), acts[2], store, tm);
    layer_forward_tc<Width, Width, false>(acts[2], s.w + weight_tile_offset(2), s.b + bias_slot(2), acts[3], store, tm);
    layer_forward_tc<Width, Width, false>(acts[3], s.w + weight_tile_offset(3), s.b + bias_slot(3), acts[4], store, tm);
    layer_forward_tc<Width, Outputs, true>(acts[4], s.w + weight_tile_offset(4), s.b + bias_slot(4), nullptr, store, tm);
}

// The same with the outputs stored in shared memory (128 rows of Out_stride floats).
__device__ inline void forward_tc(Net_smem const& s, __nv_bfloat16* const acts[Layers], float* out, Tmem_tile& tm) {
    forward_tc(s, acts, Smem_outputs{out}, tm);
}

// TMEM columns for one accumulator tile (64 FP32 columns, a power of two >= 32).
constexpr uint32_t Tmem_columns = 64;

// Block set-up for tensor-core tiles: warp 0 allocates the accumulator, thread 0 initialises
// the mbarrier; `slot` and `bar` live in shared memory.  Ends with a barrier.
__device__ inline Tmem_tile tc_setup(uint32_t* slot, uint64_t* bar, uint32_t* error) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                     "r"(Tmem_columns));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return Tmem_tile{*slot, smem_u32(bar), 0u, error};
}

// Releases the accumulator (warp 0; after the last tcgen05.ld of every warp and a barrier).
__device__ inline void tc_teardown(Tmem_tile const& tm) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm.tmem), "r"(Tmem_columns));
    }
}

}  // namespace spb::guide

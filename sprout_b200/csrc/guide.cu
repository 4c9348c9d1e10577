// Path-guiding network kernels (guide_mlp.cuh): batched forward, per-block gradient partials
// with a deterministic reduction, Adam, and the C-ABI entry points that expose the forward
// pass and the gradient to tests.  The renderer's use (inference per path vertex, training on
// the tracer's own samples) is in render.cu; the network's state is guide::Network.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

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

// Gradient partials of one tile: loss sum_i scale_i * (-log q(d_i | x_i)) over the tile's
// samples; writes Parameters floats per block to partial.
__global__ void __launch_bounds__(Block) k_gradients(__nv_bfloat16 const* wbf, float const* params,
                                                     float const* in, float const* dirs, float const* scale,
                                                     uint64_t n, float* partial) {
    extern __shared__ __align__(16) unsigned char raw[];
    Train_smem& s = *reinterpret_cast<Train_smem*>(raw);
    load_net(s.net, wbf, params);
    uint64_t const base = uint64_t(blockIdx.x) * Tile;
    load_inputs(s.a0, in, base, n);
    __syncthreads();
    __nv_bfloat16* const acts[Layers] = {s.a0, s.a[0], s.a[1], s.a[2], s.a[3]};
    forward(s.net, acts, s.zb);
    if (threadIdx.x < Tile) {
        int const      r = threadIdx.x;
        uint64_t const g = base + r;
        float*         o = s.za + r * Out_stride;
        if (g < n) {
            output_gradient(s.zb + r * Out_stride,
                            shading::v3(dirs[3 * g], dirs[3 * g + 1], dirs[3 * g + 2]), scale[g], o);
        } else {
            for (int j = 0; j < Outputs; ++j) {
                o[j] = 0.f;
            }
        }
    }
    __syncthreads();
    float* const p = partial + uint64_t(blockIdx.x) * Parameters;
    Net_smem const& net = s.net;
    layer_backward<Width, Outputs>(acts[4], net.w + weight_tile_offset(4), s.za, s.zb,
                                   p + weight_offset(4), p + bias_offset(4));
    __syncthreads();
    layer_backward<Width, Width>(acts[3], net.w + weight_tile_offset(3), s.zb, s.za,
                                 p + weight_offset(3), p + bias_offset(3));
    __syncthreads();
    layer_backward<Width, Width>(acts[2], net.w + weight_tile_offset(2), s.za, s.zb,
                                 p + weight_offset(2), p + bias_offset(2));
    __syncthreads();
    layer_backward<Width, Width>(acts[1], net.w + weight_tile_offset(1), s.zb, s.za,
                                 p + weight_offset(1), p + bias_offset(1));
    __syncthreads();
    layer_backward<Inputs, Width>(acts[0], net.w + weight_tile_offset(0), s.za, nullptr,
                                  p + weight_offset(0), p + bias_offset(0));
}

// grads[p] = sum over blocks of partial[b][p], in block order (deterministic).
__global__ void k_reduce(float const* partial, uint32_t blocks, float* grads) {
    uint32_t const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= uint32_t(Parameters)) {
        return;
    }
    float acc = 0.f;
    for (uint32_t b = 0; b < blocks; ++b) {
        acc += partial[uint64_t(b) * Parameters + p];
    }
    grads[p] = acc;
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
            e = cudaFuncSetAttribute(k_gradients, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
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
    cudaError_t e = cudaMemcpy(params_, host, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m_, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(v_, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(grads_, 0, bytes);
    if (e != cudaSuccess) {
        return e;
    }
    step_ = 0;
    k_to_bf16<<<(Parameters + 255) / 256, 256>>>(params_, wbf_);
    return cudaGetLastError();
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
    uint64_t const blocks = (n + Tile - 1) / Tile;
    if (blocks == 0) {
        return cudaMemsetAsync(grads_, 0, Parameters * sizeof(float), stream);
    }
    if (blocks > partial_blocks_) {
        release(partial_);
        if (cudaError_t const e = cudaMalloc(&partial_, blocks * Parameters * sizeof(float))) {
            partial_blocks_ = 0;
            return e;
        }
        partial_blocks_ = blocks;
    }
    k_gradients<<<unsigned(blocks), Block, tile_smem_bytes(), stream>>>(wbf_, params_, inputs, dirs, scale, n,
                                                                        partial_);
    k_reduce<<<(Parameters + 255) / 256, 256, 0, stream>>>(partial_, uint32_t(blocks), grads_);
    return cudaGetLastError();
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
    return cuda_status(e, "spb_guide_gradients");
}

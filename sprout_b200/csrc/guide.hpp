// Host side of the path-guiding network: its state on the device (FP32 master parameters,
// Adam moments, BF16 weights) and the training step.  Kernels in guide.cu.
#pragma once

#include <cuda_bf16.h>

#include <cstddef>
#include <cstdint>

namespace spb::guide {

// Shared memory of the forward / gradient tile kernels (176 KB).
size_t tile_smem_bytes();

class Network {
  public:
    Network() = default;
    ~Network();
    Network(Network const&)            = delete;
    Network& operator=(Network const&) = delete;

    // Allocates the state and initialises the parameters (He-uniform weights, zero biases,
    // seeded); 0 or a cudaError_t.
    int init(uint32_t seed);
    // Replaces the parameters (host FP32, Parameters values); resets Adam.
    int set_parameters(float const* host);
    int get_parameters(float* host) const;

    // Forward pass over n encoded inputs (device, n x 32 FP32) into n x 40 device outputs, on
    // the tensor cores; waits for completion.
    int forward(float const* inputs, uint64_t n, float* outputs, cudaStream_t stream);
    // Gradient of sum_i scale_i * (-log q(d_i | x_i)) into the device gradient buffer.
    int gradients(float const* inputs, float const* dirs, float const* scale, uint64_t n, cudaStream_t stream);
    // The same for the renderer's batches: inputs as BF16 tiles of 128 samples in the tensor
    // cores' operand order (zero rows past n), and the loss sum_i w_i (-log q) / sum_i w_i with
    // sum_i w_i the total of weight_parts (num_parts partial sums).
    int gradients_tiled(__nv_bfloat16 const* tiles, float const* dirs, float const* weights, uint64_t n,
                        float const* weight_parts, uint32_t num_parts, cudaStream_t stream);
    // One Adam step with the current gradient.
    int adam(float lr, cudaStream_t stream);
    // One Adam step after gradients_tiled(), with the step count kept in device memory (each
    // gradients_tiled() call counts one), so that the pair can be replayed from a captured
    // graph; increments *advance (if given) once the step has run.
    int adam_counted(float lr, uint32_t* advance, cudaStream_t stream);
    // Allocates what gradients_tiled() on n samples needs, so that no allocation happens while
    // a stream is being captured.
    int prepare_gradients(uint64_t n);

    float const*         gradient() const { return grads_; }
    // True once a tensor-core completion wait of forward() or gradients() ran out.
    bool                 timed_out() const;
    uint32_t*            error_flag() const { return error_; }
    __nv_bfloat16 const* weights() const { return wbf_; }
    float const*         parameters() const { return params_; }

  private:
    int run_gradients(void const* inputs, bool tiled, float const* dirs, float const* scale, uint64_t n,
                      float const* weight_parts, uint32_t num_parts, cudaStream_t stream);

    float*         params_  = nullptr;
    float*         m_       = nullptr;
    float*         v_       = nullptr;
    float*         grads_   = nullptr;
    __nv_bfloat16* wbf_     = nullptr;
    float*         partial_ = nullptr;
    uint64_t       partial_blocks_ = 0;
    uint32_t       step_    = 0;
    uint32_t*      error_   = nullptr;  // set by a tensor-core wait that ran out
    uint32_t*      step_dev_ = nullptr;  // Adam steps taken through gradients_tiled()
};

}  // namespace spb::guide

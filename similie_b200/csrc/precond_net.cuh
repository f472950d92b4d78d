// precond_net.cuh -- the learned multilevel convolutional preconditioner of
// the 2D magnetostatics solve: network definition, batched workspace and the
// host-side interface the solver and the C API use.
//
// Preconditioner M(r) for a batch of residuals (FP32, node grids x fastest):
//   e1 = w D^-1 r                      (Jacobi step, w = 0.8)
//   r1 = r - K e1
//   s  = rms(D^-1/2 r1)
//   x  = pool2x2([D^-1/2 r1 / s, log(nu) / log(1000)])   (2-channel image, half resolution)
//   v  = s * D^-1/2 up2x2(net(x)), zero on the Dirichlet boundary
// The symmetric diagonal scaling carries the 1/nu amplitude of the error in
// low-reluctivity (high-permeability) regions, so the network sees an
// operator of much lower contrast.
//   e2 = e1 + v
//   M(r) = e2 + w D^-1 (r - K e2)      (Jacobi step)
// The network is a U-Net over levels of halving resolution down to a
// coarsest grid of at least 8 x 8: a 2->32 input convolution, per coarser
// level a 2x2 average pool followed by two 32->32 convolutions (down, enc),
// per level on the way up a 32->32 convolution of skip + nearest-upsampled
// coarse features (dec), and a 32->1 output convolution; all 3x3, ReLU
// after every convolution but the last.  Levels 1, 2 and 3 have their own
// weights; deeper levels reuse the level-3 weights.  Activations and the
// 32->32 weights are BF16, accumulation FP32 (tensor cores, tcgen05).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "sil_b200.h"

namespace sil {
namespace nn {

constexpr int kCh = 32;
constexpr int kTaps = 9;
constexpr int kBigW = kCh * kTaps * kCh;   // 9216 weights of one 32->32 convolution
constexpr int kBigParams = kBigW + kCh;    // + bias
constexpr int kNumBig = 9;                 // down/enc/dec x 3 weight levels
constexpr int kInW = kCh * kTaps * 2;      // 576
constexpr int kOutW = kTaps * kCh;         // 288
constexpr int kOffIn = 0;
constexpr int kOffBig = kInW + kCh;                         // 608
constexpr int kOffOut = kOffBig + kNumBig * kBigParams;     // 83840
constexpr int kNumParams = kOffOut + kOutW + 1;             // 84129
constexpr int kMaxImages = 64;
constexpr float kOmega = 0.8f;

// Index of a 32->32 convolution in the parameter list.
__host__ __device__ constexpr int big_index(int kind, int weight_level) { return weight_level * 3 + kind; }
enum BigKind { kDown = 0, kEnc = 1, kDec = 2 };

// One sample of a batch: an nx x ny node grid, x fastest, at `offset` in the
// batch's flat node arrays.
struct Sample
{
    int32_t nx, ny;
    int64_t offset;
};

class Workspace;

// Network parameters (FP32 master copy, BF16 tensor-core copies) and the
// Adam state; workspaces are cached per batch geometry.
class Net
{
public:
    Net();
    ~Net();
    sil_status init(uint64_t seed, cudaStream_t stream);
    sil_status set_params(float const* host, cudaStream_t stream);
    sil_status get_params(float* host, cudaStream_t stream);
    // Refresh the BF16 copies after the master weights changed.
    sil_status refresh(cudaStream_t stream);

    // Workspace of a batch geometry (allocated once, before any stream capture).
    sil_status prepare(std::vector<Sample> const& samples, cudaStream_t stream, Workspace** out);
    // Declare nu (device, FP32 per node) fixed for the forward passes that
    // follow on this workspace: the log(nu) input channel is formed once and
    // reused while forward() is given the same nu pointer; NULL ends it.  A
    // caller that changes nu in place must call this again.
    sil_status set_static_nu(Workspace* w, float const* nu, cudaStream_t stream);
    // out = M(r) on a prepared workspace: kernel launches only (capturable).
    // dinv: inverse operator diagonal per node (FP32), or NULL.  active
    // (device, one int per sample, or NULL): samples whose entry is 0 at
    // launch time are skipped, their out left unwritten.
    sil_status forward(Workspace* w, float const* nu, float const* dinv, float const* r, float* out,
                       cudaStream_t stream, int const* active = nullptr);
    // out = M(r) for a batch (device FP32 node arrays, nu FP32 per node).
    sil_status apply(std::vector<Sample> const& samples, float const* nu, float const* r, float* out, cudaStream_t stream,
                     int const* active = nullptr);
    // Loss 1 - (u.b)^2 / ((u.K u)(x.b)) with u = M(b), mean over the batch,
    // and its gradient with respect to every parameter (into grad, device).
    sil_status loss_grad(std::vector<Sample> const& samples, float const* nu, float const* b, float const* x,
                         double* loss, std::vector<double>* per_sample, cudaStream_t stream);
    // One Adam step on the gradient of loss_grad.
    sil_status adam_step(float lr, cudaStream_t stream);
    // Copy a buffer of the most recent workspace to the host as FP32
    // (0 h, 1 p, 2 g per level; 3 dh, 4 dg; 5 features, 6 network output,
    // 7 preconditioned vector, 8 network output gradient).
    sil_status debug_fetch(int which, int level, float* host, int64_t count, cudaStream_t stream);

    float* params = nullptr;   // device FP32 [kNumParams]
    float* grad = nullptr;     // device FP32 [kNumParams]
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    void* wbf = nullptr;       // device BF16 forward weights [kNumBig][32][9][32]
    void* wbf_t = nullptr;     // device BF16 transposed weights for the data gradient
    int adam_t = 0;
    int* error_flag = nullptr;
    Workspace* workspace(std::vector<Sample> const& samples, cudaStream_t stream, sil_status* st);

private:
    std::vector<std::unique_ptr<Workspace>> cache_;
};

} // namespace nn
} // namespace sil

struct sil_precond_s
{
    sil::nn::Net net;
};

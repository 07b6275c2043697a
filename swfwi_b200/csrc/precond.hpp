// Learned preconditioner: a small convolutional encoder-decoder that maps
// (raw gradient, current velocity, source illumination) on the model
// interior to an update direction for the FWI line search.
//
// The network has no counterpart in the reference; it sits beside the
// plain FWI epoch (src/fwi/fwiframework.cpp:269-356), which stays both the
// fallback and the arbiter of every proposed step.
//
// Architecture (4 levels, widths c0..c3, default 16/32/64/64):
//   x (3 channels, zero-padded to 16)
//   e0a,e0b: 3x3 conv 16->c0->c0, ReLU              -> s0   (H x W)
//   pool 2x2; e1a,e1b: c0->c1->c1                    -> s1   (H/2)
//   pool;     e2a,e2b: c1->c2->c2                    -> s2   (H/4)
//   pool;     ba,bb:   c2->c3->c3                    -> b3   (H/8)
//   up 2x, concat s2; d2a,d2b: c3+c2 -> c2 -> c2     -> u2
//   up 2x, concat s1; d1a,d1b: c2+c1 -> c1 -> c1     -> u1
//   up 2x, concat s0; d0a,d0b: c1+c0 -> c0 -> c0     -> u0
//   out: 1x1 conv c0 -> 1 (no activation, FP32)
// Activations and conv weights are BF16 (NHWC, weights [co][ky][kx][ci]);
// every product accumulates in FP32 on the tensor cores (tcgen05.mma
// kind::f16, BF16 operands, accumulators in tensor memory); master weights,
// Adam moments, gradients, the loss and the output layer are FP32.  H and W
// must be multiples of 8; every width a multiple of 16, at most 128.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>
#include <vector>
#include "common.hpp"

namespace swfwi {

struct ConvSpec {
  int cin, cout;
  long long w_off, b_off;   // floats into the flat parameter vector
};

class Preconditioner {
 public:
  explicit Preconditioner(const int widths[4]);
  static constexpr int kConvs = 14;
  static constexpr int kInCh = 16;   // input channels after padding (3 used)

  long long num_params() const { return nparam_; }
  const std::vector<ConvSpec> &convs() const { return conv_; }
  long long out_w_off() const { return out_w_; }
  long long out_b_off() const { return out_b_; }

  void set_stream(cudaStream_t s) { st_ = s; }
  void set_params(const float *host);
  void get_params(float *host);
  void get_grads(float *host);
  void reset_optimizer();

  // Raw network on device tensors: x [N][H][W][3] FP32 -> y [N][H][W] FP32.
  void forward(const float *x, float *y, int N, int H, int W);
  // Mean-square loss of the last forward against t [N][H][W] (FP32) and the
  // parameter gradient (overwritten); returns the loss.
  double backward(const float *t);
  // Adam on the parameter gradient (bias-corrected; step counted here).
  void adam_step(float lr, float beta1 = 0.9f, float beta2 = 0.999f, float eps = 1e-8f);
  // forward + backward + adam; returns the loss before the step.
  double train_step(const float *x, const float *t, int N, int H, int W, float lr);

  // Features of a padded model grid (caller layout [nxpad][nzpad]): the
  // interior [bx0, nxpad-bxn) x [bz0, nzpad-bzn) as an image of
  // Hp x Wp = roundup(nx,8) x roundup(nz,8) pixels, rows along x, columns
  // along depth; zero outside the interior.  x3 [Hp][Wp][3]:
  //   0: gradient / its RMS; 1: (vt - mean) / std;
  //   2: (log10(illum / max illum + 1e-6) + 3) / 3.
  void features(const float *grad, const float *vel, const float *illum, int nxpad, int nzpad,
                int bx0, int bxn, int bz0, int bzn, float *x3);
  // Training target: the interior of dv scaled to unit RMS, t [Hp][Wp].
  void target(const float *dv, int nxpad, int nzpad, int bx0, int bxn, int bz0, int bzn, float *t);
  // Direction on the padded grid from a network output y [Hp][Wp]: zero
  // outside the interior.
  void scatter(const float *y, int nxpad, int nzpad, int bx0, int bxn, int bz0, int bzn,
               float *dir);
  // features -> forward -> scatter.
  void propose(const float *grad, const float *vel, const float *illum, int nxpad, int nzpad,
               int bx0, int bxn, int bz0, int bzn, float *dir);

 private:
  cudaStream_t st_ = nullptr;
  int w_[4];
  std::vector<ConvSpec> conv_;
  long long out_w_ = 0, out_b_ = 0, nparam_ = 0;
  DevBuf<float> params_, grads_, m_, v_;
  DevBuf<__nv_bfloat16> wbf_, wflip_;
  long long step_ = 0;
  // activations of the last forward
  int N_ = 0, H_ = 0, W_ = 0;
  DevBuf<__nv_bfloat16> x16_, a0_, s0_, p0_, a1_, s1_, p1_, a2_, s2_, p2_, a3_, b3_, cat2_, a4_, u2_,
      cat1_, a5_, u1_, cat0_, a6_, u0_;
  DevBuf<float> y_;
  // backward scratch
  DevBuf<float> dy_, dA_, dB_, dS0_, dS1_, dS2_, dLow_, dCat_;
  DevBuf<__nv_bfloat16> dz_;
  DevBuf<float> part_;   // per-chunk / per-block partial sums of the gradients
  DevBuf<double> red_;
  DevBuf<float> feat_, outimg_;

  void refresh_bf16();
  // interior statistics of a, b, c into red_[0..3] (fixed summation order)
  void stats(const float *a, const float *b, const float *c, int nzpad, int x0, int z0, int nx, int nz);
  void conv_fwd(int l, const __nv_bfloat16 *in, __nv_bfloat16 *out, long long P, int H, int W);
  // dY (FP32, layer output grad) -> parameter grads; dX (FP32, may be null)
  void conv_bwd(int l, const __nv_bfloat16 *in, const __nv_bfloat16 *out, const float *dY, float *dX,
                int H, int W);
};

// Device launches used by the class and the tests.
void launch_conv3x3(const __nv_bfloat16 *in, int cin, const __nv_bfloat16 *w, const float *bias,
                    void *out, bool out_f32, bool accum, int cout, int N, int H, int W,
                    cudaStream_t st);
// dw [cout][3][3][cin] (overwritten) from per-chunk partials in scratch
// (at least conv3x3_wgrad_scratch floats), summed in a fixed order.
size_t conv3x3_wgrad_scratch(int cout, int cin, int N, int H, int W);
void launch_conv3x3_wgrad(const __nv_bfloat16 *dz, int cout, const __nv_bfloat16 *x, int cin,
                          float *dw, float *scratch, size_t scratch_floats, int N, int H, int W,
                          cudaStream_t st);
// Illumination: illum[x*nzpad + z] += sum over n slots of p^2 (pitched
// fields at fstride).
void launch_illum_accum(float *illum, const float *p, long long fstride, int n, int nxpad, int nzpad,
                        int pitch, cudaStream_t st);

}  // namespace swfwi

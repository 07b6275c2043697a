// The propagator: swfwi's Damp4t10d on the GPU, plus batched whole-shot
// forward modelling and gradients.  Host C++ over the kernels in
// kernels.cu / stencil.cuh.
#pragma once
#include <atomic>
#include <mutex>
#include <vector>
#include "common.hpp"
#include "kernels.cuh"

namespace swfwi {

// Process-wide timing of stencil launches (CUDA events on the launching
// stream) and their algorithmic work, read by benchmarks.
struct StepTimer {
  std::atomic<bool> enabled{false};
  std::mutex mu;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  size_t used = 0;
  long long launches = 0;
  double points = 0, bytes = 0;
  void reset();
  void read(double &ms, long long &n, double &pts, double &b);
};
StepTimer &step_timer();
void timed_step(int arith, bool damped, int tx, const StepArgs &a, int n, cudaStream_t st);

// A regular line of points (src/common/shot-position.cpp:11-41).
struct Line {
  int szbeg, sxbeg, jsz, jsx, n;
  int z(int i) const { return szbeg + i * jsz; }
  int x(int i) const { return sxbeg + i * jsx; }
};

// Device work space for a batch of wavefields, grown on demand.
template <typename T>
struct Work {
  DevBuf<T> p0, p1, g0, g1, image, strips;
  DevBuf<float> dcal, obs, res, vsrc;   // [slot][nt][ng]
  DevBuf<int> win, slot_shot, slot_row;
  DevBuf<double> partials, obj;
};

class Propagator {
 public:
  Propagator(const Line &src, const Line &geo, float dt, float dx, float fm, int nb, int nt);
  ~Propagator();

  // ---- geometry ----
  int nx, nz, nb, nt, ns, ng, ngmax;
  float dt, dx, fm;
  int bx0, bxn, bz0, bzn;
  int nxpad, nzpad;
  long long fstride;   // floats between batched fields (aligned)
  int bsize;           // strip floats per step
  int half_len;        // direct-arrival mute half window (samples)

  void set_stream(cudaStream_t s);
  cudaStream_t stream() const { return st_; }
  int arith = ARITH_REF;
  int strip_format = SWFWI_STRIP_F32;
  int tile_tx = 32;

  void set_receivers_per_shot(const int *offsets, const int *gx, const int *gz);
  void set_dims(int nxpad, int nzpad);   // padded grid; uploads geometry
  void expand_domain(const float *vel, float *exvel) const;   // host
  void bind_velocity(const float *exvel_dev);
  const float *velocity() const { return vel_; }

  // ---- reference-compatible single-field operations (device pointers) ----
  void step_forward(float *p0, float *p1);
  void step_backward(float *p0, float *p1);
  void manip_source(float *p, const float *src, int shot_id, int sign);
  void add_receiver_source(float *p, const float *vsrc_it);
  void record_seis(float *seis, const float *p);
  void write_bndry(float *bndr, const float *p, int it);
  void read_bndry(const float *bndr, float *p, int it);
  void mask_gradient(float *g);
  void scale_gradient(float *g);
  void refill_boundary(float *v);
  void remove_direct_arrival(float *data, int shot_id, const float *vel = nullptr);
  void fwi_forward(const float *wlt, float *dcal, int shot_id);
  void ess_forward(const float *encsrc, float *dcal, const float *vel = nullptr);

  // ---- batched ----
  // dcal [n][nt][ng] for shots ids[0..n) (host list).
  void forward_batch(const float *wlt, float *dcal, const int *ids, int n,
                     const float *vel = nullptr);
  // Gradient loop of FwiFramework::epoch for the listed shots; grad
  // overwritten (or accumulated if accumulate); obj[n] host.
  // rows (host, optional): the dobs row of each listed shot (default: the
  // shot id itself).
  void gradient_batch(const float *wlt, const float *dobs, const int *ids, int n, float *grad,
                      double *obj, bool accumulate = false, const int *rows = nullptr);
  // Trial objective: sum over listed shots of |mute_obs - mute_cal(vel)|^2
  // with the observed data muted with the bound velocity (host result).
  double trial_objective_fwi(const float *wlt, const float *dobs, const int *ids, int n,
                             const float *trial_vel);
  // Encoded supershot pieces.
  void calgradient_ess(const float *encsrc, const float *vsrc, float *grad);
  void calgradient_fwi(const float *wlt, const float *vsrc, float *grad, int shot_id);
  void calgradient_fwi_f64(const float *vel, const double *wlt, const double *vsrc, double *grad,
                           int shot_id);
  void fwi_forward_f64(const float *vel, const double *wlt, double *dcal, int shot_id);

  // Max shots per batch that fit the device memory budget.
  int max_batch() const;

  // host mirrors of geometry (padded coordinates)
  std::vector<int> h_src_x, h_src_z, h_geo_x, h_geo_z;
  std::vector<int> h_rec_x, h_rec_z;   // [ns][ngmax], -1 padded
  std::vector<int> h_rec_count;

 private:
  cudaStream_t st_ = nullptr, own_st_ = nullptr;
  const float *vel_ = nullptr;
  DevBuf<float> rcp_;
  const float *rcp_for_ = nullptr;
  DevBuf<int> d_src_pos_, d_src_x_, d_src_z_;
  DevBuf<int> d_geo_pos_, d_geo_x_, d_geo_z_;
  DevBuf<int> d_rec_pos_, d_rec_x_, d_rec_z_;
  DevBuf<int> d_win1_;
  DevBuf<double> d_scalar_;
  DevBuf<float> trial_rcp_;
  Work<float> w_;
  Work<double> wd_;

  void upload_geometry();
  const float *rcp_of(const float *vel);
  StepArgs step_args(void *prev, const void *curr, const void *velrcp, int n) const;

  // Runs the forward time loop for n slots already described by src/rec
  // point sets.  Source values: vals + it*it_stride + slot*slot_stride +
  // i*i_stride.
  template <typename T>
  void run_forward(Work<T> &w, int n, PointSet src, const T *vals, long long it_stride,
                   long long slot_stride, int i_stride, PointSet rec, int ngrec, T *dcal,
                   bool save_strips, const void *velrcp);
  template <typename T>
  void run_backward(Work<T> &w, int n, PointSet src, const T *vals, long long it_stride,
                    long long slot_stride, int i_stride, PointSet rec, int ngrec, const T *vsrc,
                    const void *velrcp_damped);
  template <typename T>
  void ensure_work(Work<T> &w, int n, bool strips, int ngrec);
};

}  // namespace swfwi

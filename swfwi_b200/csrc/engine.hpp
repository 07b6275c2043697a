// The propagator: swfwi's Damp4t10d on the GPU, plus batched whole-shot
// forward modelling and gradients.  Host C++ over the kernels in
// kernels.cu / stencil.cuh / stream.cuh.
//
// Wavefields the propagator owns are stored with rows of `pitch` floats
// (nzpad + 8 rounded up to 8) behind an 8-float origin offset, so every row
// and every 4-depth group starts on a 16-byte boundary and the streaming step
// can move rows with TMA bulk copies; pointers to them passed to kernels are
// origins (slot start + 8).  Arrays the caller owns keep the reference's
// [nxpad][nzpad] layout.
#pragma once
#include <algorithm>
#include <atomic>
#include <functional>
#include <memory>
#include <mutex>
#include <vector>
#include "common.hpp"
#include "kernels.cuh"

namespace swfwi {

// Process-wide timing of stencil launches (CUDA events on the launching
// stream) and their algorithmic work, read by benchmarks.  While enabled,
// every launch's work is counted and every period-th launch is timed.
struct StepTimer {
  // What a captured time loop contributes each time its graph is replayed:
  // its stencil launches' count and work, its kernel launches, and the
  // event pairs (graph event-record nodes) of its timed stencil launches,
  // whose times are added up after each replay.
  struct Capture {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pairs;
    long long launches = 0, kernels = 0;
    double points = 0, bytes = 0;
    bool pending = false;   // replayed, times not yet added
    ~Capture();
  };
  std::atomic<bool> enabled{false};
  std::atomic<int> period{1};
  std::mutex mu;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pool;
  size_t used = 0;
  long long launches = 0;
  double points = 0, bytes = 0;
  double graph_ms = 0;          // times of replayed graphs' timed launches
  long long graph_timed = 0;
  std::vector<Capture *> replayed;
  void reset();
  // ms: the timed launches' total; n: launches counted; timed: launches timed
  void read(double &ms, long long &n, double &pts, double &b, long long &timed);
  // Opens the timing of one launch over n fields of pts interior points
  // reading nvel velocity models, el bytes an element; returns the event to
  // record after the launch with close() (null when timing is off).
  cudaEvent_t open(cudaStream_t st, double pts, int n, int nvel, int el);
  void close(cudaEvent_t done, cudaStream_t st);
  // Stream capture of a time loop begins / ends (the kernels the capture
  // counted are taken back; each replay adds them).
  void begin_capture(Capture *c);
  void end_capture();
  // A captured loop was launched: add its counts; its times are added once
  // its launch is complete (at its next replay or at read()).
  void replay(Capture *c);
  void forget(Capture *c);   // before a capture is destroyed
 private:
  void harvest(Capture *c);   // mu held
};
StepTimer &step_timer();

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
  DevBuf<uint16_t> qstrips;   // 16-bit strips [slot][nt][bsize] (FP32 fields, F16/BF16 format)
  DevBuf<float> qscale;       // their scales [slot][nt]
  // checkpoint snapshots (reconstruction by snapshots): pairs of whole
  // fields [snapshot][2][slot][fstride] in T, or 16-bit [snapshot][2][slot]
  // [nxpad * pitch] with scales [snapshot][2][slot]; the re-forward ring of
  // snap_every + 1 fields [ring slot][slot][fstride]
  DevBuf<T> snaps, ring;
  DevBuf<uint16_t> qsnaps;
  DevBuf<float> qsnap_scale, snap_pmax;
  DevBuf<float> dcal, res, vsrc;   // [slot][nt][ngmax]
  DevBuf<int> win, win2, slot_shot, slot_row;
  DevBuf<PtLine> src_lines, rec_lines;   // fused epilogue lines [slot]
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
  int pitch;           // floats per row of propagator-owned fields
  long long fstride;   // floats between batched fields (multiple of 64)
  int bsize;           // strip floats per step
  int half_len;        // direct-arrival mute half window (samples)

  void set_stream(cudaStream_t s);
  cudaStream_t stream() const { return st_; }
  int arith = ARITH_REF;
  int strip_format = SWFWI_STRIP_F32;
  // How the backward sweep gets the source field: SWFWI_RECON_STRIPS
  // (back-propagation with the saved boundary strips, the reference's
  // method) or SWFWI_RECON_SNAPSHOTS (the forward saves both fields every
  // snap_every steps in snap_format; the backward re-runs each segment
  // forward from its snapshot into a ring of fields).
  int recon = SWFWI_RECON_STRIPS;
  int snap_every = 64;
  int snap_format = SWFWI_STRIP_F32;
  int stream_kernel = 6;      // 1: warp-specialised, 5: register-queue warps, 6: two-row register queue (FAST)
  int stream_bz = 120;        // output depths per CTA (120 for kernel 5; 120, 248 or 376 for kernel 1)
  int stream_xchunk = 0;      // rows per CTA (per warp task for kernel 5); 0: automatic
  int stream_depth = 3;       // rows ahead (3 or 7)
  int stream_shot_major = 0;  // launch order: 0 = shots fastest
  bool fuse = false;          // fused time loops where they apply
  // Source illumination: while set, the forward sweeps that save strips
  // add sum over slots of p^2 into illum [nxpad][nzpad] every illum_every
  // steps (the caller zeroes it).
  float *illum = nullptr;
  int illum_every = 4;
  // CUDA graphs for the time loops of the forward and backward sweeps:
  // 0 never, 1 when a step is small enough to be launch-bound (n fields x
  // nxpad x nzpad at most kGraphMaxPoints), 2 for every step size; never
  // while stencil launches are being timed.
  int graphs = 1;
  static constexpr double kGraphMaxPoints = 8e6;

  void set_receivers_per_shot(const int *offsets, const int *gx, const int *gz);
  void set_dims(int nxpad, int nzpad);   // padded grid; uploads geometry
  void expand_domain(const float *vel, float *exvel) const;   // host
  void bind_velocity(const float *exvel_dev);
  // Forget the bound velocity if it is v (its owner is going away).
  void unbind_velocity(const float *v) {
    if (vel_ == v) {
      vel_ = nullptr;
      rcp_for_ = nullptr;
    }
  }
  const float *velocity() const { return vel_; }

  // ---- reference-compatible single-field operations (device pointers,
  // caller layout [nxpad][nzpad]) ----
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
  // The HA loop of EnkfAnalyze::calGainMatrix (enkfanalyze.cpp:207-236):
  // EssForwardModeling of the encoded supershot with each of n velocities
  // (vels [n][nxpad*nzpad], caller layout), the seismograms transposed to
  // the analysis matrix's column order: hona [n][ng*nt], row ig*nt + it.
  void ess_forward_members(const float *encsrc, const float *vels, int n, float *hona);

  // ---- batched ----
  // dcal [n][nt][ngmax] for shots ids[0..n) (host list).
  void forward_batch(const float *wlt, float *dcal, const int *ids, int n,
                     const float *vel = nullptr);
  // Gradient loop of FwiFramework::epoch for the listed shots; grad
  // overwritten (or accumulated); obj[n] host.  rows (host, optional): the
  // dobs row of each listed shot (default: the shot id).
  // before_residual (optional) runs on the host after each batch's forward
  // sweep is enqueued and before its residual is (a caller's upload of the
  // observed data can overlap the sweep).
  void gradient_batch(const float *wlt, const float *dobs, const int *ids, int n, float *grad,
                      double *obj, bool accumulate = false, const int *rows = nullptr,
                      const std::function<void()> *before_residual = nullptr);
  // Trial objective: sum over listed shots of |mute(obs) - mute(cal(vel))|^2,
  // the observed data muted with the bound velocity (host result).
  double trial_objective_fwi(const float *wlt, const float *dobs, const int *ids, int n,
                             const float *trial_vel);
  void calgradient_ess(const float *encsrc, const float *vsrc, float *grad);
  void calgradient_fwi(const float *wlt, const float *vsrc, float *grad, int shot_id);
  void calgradient_fwi_f64(const float *vel, const double *wlt, const double *vsrc, double *grad,
                           int shot_id);
  void calgradient_ess_f64(const float *vel, const double *encsrc, const double *vsrc, double *grad);
  void fwi_forward_f64(const float *vel, const double *wlt, double *dcal, int shot_id);

  // Max shots per batch that fit the device memory budget.
  int max_batch() const;
  // Raises SWFWI_ERR_TIMEOUT if a kernel's bounded wait gave up (syncs).
  void check_device_error();

  // host mirrors of geometry (unpadded coordinates)
  std::vector<int> h_src_x, h_src_z, h_geo_x, h_geo_z;
  std::vector<int> h_rec_x, h_rec_z;   // [ns][ngmax], -1 padded
  std::vector<int> h_rec_count;

 private:
  cudaStream_t st_ = nullptr;   // 0 = the legacy default stream
  const float *vel_ = nullptr;
  DevBuf<float> rcp_;           // pitched 1/vt of the bound velocity
  const float *rcp_for_ = nullptr;
  DevBuf<float> trial_rcp_;
  DevBuf<float> members_rcp_;   // per-member reciprocals of ess_forward_members
  long long vel_stride_ = 0;    // floats between slots' velocity reciprocals (0: one model)
  DevBuf<int> d_err_;
  DevBuf<float> damp_x_, damp_z_;   // per-axis sponge ramps (streaming step)
  DevBuf<float2> coef_x_;           // each row's FAST ramp coefficients (streaming step)
  // positions in the caller's layout (x*nzpad + z) ...
  DevBuf<int> d_src_pos_, d_geo_pos_;
  // ... and in the propagator's pitched layout (x*pitch + z)
  DevBuf<int> d_src_pos_p_, d_geo_pos_p_, d_rec_pos_p_;
  // padded coordinates for the mute windows
  DevBuf<int> d_src_x_, d_src_z_, d_geo_x_, d_geo_z_, d_rec_x_, d_rec_z_;
  DevBuf<int> d_win1_;
  Work<float> w_;
  Work<double> wd_;

  void upload_geometry();
  const float *rcp_of(const float *vel);
  void step_fields(int ar, bool damped, void *prev, const void *curr, const void *velrcp, int n,
                   const Epilogue *epi = nullptr, void *out = nullptr);
  // Checkpoint snapshots: how many a forward sweep saves, and their save /
  // restore (snapshot m holds the pair (p0, p1) after forward step
  // (m + 1) * snap_every - 1).
  int snapshot_count() const { return recon == SWFWI_RECON_SNAPSHOTS ? (nt - 1) / std::max(snap_every, 1) : 0; }
  template <typename T>
  void save_snapshot(Work<T> &w, int n, int m, const T *a, const T *b);
  template <typename T>
  void restore_snapshot(Work<T> &w, int n, int m, T *a, T *b);
  // Point lines (padded coordinates) for the fused forward epilogue; false
  // when the points do not form a regular line.
  bool line_of(const int *xs, const int *zs, int n, PtLine &out) const;
  bool shot_lines(const int *ids, int k, bool per_shot_receivers, std::vector<PtLine> &src,
                  std::vector<PtLine> &rec) const;
  bool ess_lines(int k, std::vector<PtLine> &src, std::vector<PtLine> &rec) const;

  // Forward time loop for n slots.  Source values:
  // vals + it*it_stride + slot*slot_stride + i*i_stride.
  template <typename T>
  void run_forward(Work<T> &w, int n, PointSet src, const T *vals, long long it_stride,
                   long long slot_stride, int i_stride, PointSet rec, int ngrec, T *dcal,
                   bool save_strips, const void *velrcp);
  // Backward sweep with imaging into w.image (not cleared here).
  template <typename T>
  // With per-slot horizontal lines, FP32 fields and fusion on: the source
  // back-step also subtracts the source and images, the receiver step also
  // injects the next residual.  sum_images (FAST arithmetic, separate
  // launches only): every slot images into slot 0's image, one pass per
  // step.  Returns true when the images were summed that way.
  bool run_backward(Work<T> &w, int n, PointSet src, const T *vals, long long it_stride,
                    long long slot_stride, int i_stride, PointSet rec, int ngrec, const T *vsrc,
                    const void *velrcp, const std::vector<PtLine> *src_lines = nullptr,
                    const std::vector<PtLine> *rec_lines = nullptr, bool sum_images = false);
  template <typename T>
  void ensure_work(Work<T> &w, int n, bool strips);
  // Runs body (launches on st_ only, no allocation or synchronisation):
  // directly, or as a CUDA graph launched on st_.  which: 0 forward loop,
  // 1 backward loop.  key lists everything the loop's launches depend on
  // (pointers, sizes, settings); a cached graph with the same key is
  // relaunched without running body, else body is captured on a private
  // stream into a new graph (up to kGraphCache per loop kind).
  template <typename F>
  void run_loop(int which, double points_per_step, const std::vector<long long> &key, F &&body);
  struct LoopGraph {
    std::vector<long long> key;
    cudaGraphExec_t exec = nullptr;
    std::unique_ptr<StepTimer::Capture> timing;   // its launches' counts and timed event pairs
  };
  static constexpr size_t kGraphCache = 4;
  cudaStream_t cap_ = nullptr;
  std::vector<LoopGraph> gcache_[2];
  bool loop_warm_[2] = {false, false};
  // settings every loop launch depends on, for graph keys
  void loop_key_common(std::vector<long long> &k) const;
  // copies between the caller's [nxpad][nzpad] layout and pitched rows
  template <typename T>
  void to_pitched(T *dst, const T *src);
  template <typename T>
  void from_pitched(T *dst, const T *src);
};

}  // namespace swfwi

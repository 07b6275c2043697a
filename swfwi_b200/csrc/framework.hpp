// FWI drivers over the propagator: the plain per-shot framework
// (src/fwi/fwiframework.cpp), the encoded-source framework
// (src/essfwi/essfwiframework.cpp) and their step-length search
// (src/essfwi/updatesteplenop.cpp) and velocity update
// (src/essfwi/updatevelop.cpp).
#pragma once
#include <cstdint>
#include <functional>
#include <vector>
#include "engine.hpp"

namespace swfwi {

// RandomCodes (src/common/random-code.cpp:2-22): Boost.Random minstd_rand
// (x <- 48271 x mod 2^31-1, seed 0 -> 1) mapped to {0,1} by Boost's
// uniform_int bucketing (bucket = (brange+1)/2 over the engine range
// [1, 2^31-2]), then to -1/+1.
class RandomCodes {
 public:
  explicit RandomCodes(int seed);
  std::vector<int> gen_plus1_minus1(int n);

 private:
  uint64_t x_;
  int draw();
};

// parabolaVertex (src/common/parabola-vertex.cpp:12-33).
void parabola_vertex(float x1, float y1, float x2, float y2, float x3, float y3, float max_alpha3,
                     float &xv, float &yv);

// The step-length search of UpdateSteplenOp (updatesteplenop.cpp:25-285)
// over an objective function of the step.
struct StepSearch {
  int nita = 0;
  float maxdv = 0;
  bool preserved_init = false;
  float preserved_alpha = 0;
  // last search, for inspection: its (alpha, objective) triple and vertex,
  // and how many trial objectives (forward sweeps over all shots) it ran
  float alpha[4] = {0, 0, 0, 0}, obj[4] = {0, 0, 0, 0};
  int trials = 0;
  // calsteplen: returns the step; objval receives its objective
  float calsteplen(const std::function<float(float)> &f, float obj_val1, float max_alpha3,
                   float &objval);
};

class Preconditioner;

class FwiRunner {
 public:
  FwiRunner(Propagator &p, const float *exvel_host, float vmin, float vmax, int nita, float maxdv,
            const float *wlt_host, const float *dobs_host, bool encoded);
  ~FwiRunner() { p_.unbind_velocity(vel_.get()); }
  void epoch(int iter);
  float update_obj = 0, init_obj = 0;
  void get_velocity(float *host);
  void set_velocity(const float *host);   // the member moved by an EnKF analysis
  void write_vel(float *host);   // sfWriteVel without the file
  StepSearch search;

  // Learned preconditioner (not owned; null = plain FWI).  With a network
  // set, each plain epoch first searches along the network's direction with
  // its own copy of the step-length search and takes that step only when
  // the search confirms an objective decrease (its vertex objective and an
  // evaluated trial both below the current objective); otherwise it takes
  // the plain step.  After a learned step the next CG direction restarts.
  void set_preconditioner(Preconditioner *net) {
    SWFWI_REQUIRE(!net || !encoded_, "the learned step applies to plain FWI");
    net_ = net;
  }
  // Accumulate the source illumination during the gradient's forward sweep
  // (always on while a network is set).
  void set_collect_illumination(bool on) { collect_illum_ = on; }
  // EssFwiRegu (src/unused/essfwiregu.cpp:667-776) for an encoded
  // framework: each objective adds lx Wx2 + lz Wz2 of the model
  // (ReguFactor, src/unused/ReguFactor.cpp), the gradient adds the factor's
  // gradient before the mask, it is not depth-scaled, and the direction is
  // the gradient itself (gradUpdator :66-68).  lx = lz = 0 turns it off.
  void set_regularization(float lx, float lz);
  void get_gradient(float *host);       // the last epoch's gradient
  void get_illumination(float *host);   // the last epoch's illumination
  int last_step_learned = 0, learned_tried = 0, learned_accepted = 0;
  // A learned step must lower the objective by at least this fraction
  // (0: any confirmed decrease).
  float learned_min_decrease = 0.0f;
  // Stop proposing learned steps after this many rejections (0: never):
  // the network helps most early in a run, and a rejected proposal costs
  // its trial forwards.
  int learned_patience = 0;
  int learned_rejected = 0;
  StepSearch learned_search;

 private:
  Propagator &p_;
  bool encoded_;
  float vmin_t_, vmax_t_;   // UpdateVelOp bounds in transformed units
  int n_;                   // nxpad*nzpad
  DevBuf<float> vel_, trial_, g_, g0_, dir_, wlt_, dobs_, encsrc_, encobs_, dcal_, vsrc_, res_;
  DevBuf<int> codes_;
  DevBuf<float> illum_, ldir_;
  Preconditioner *net_ = nullptr;
  bool collect_illum_ = false;
  bool restart_cg_ = false;
  bool try_learned_step(float obj1);
  float regu_lx_ = 0.0f, regu_lz_ = 0.0f;
  DevBuf<double> regu_scratch_;
  bool regu_ = false;
  void regu_epoch(int iter);
  float regu_term(const float *vel);
  DevBuf<double> scratch_;
  RandomCodes codes_gen_;
  std::vector<int> ids_;
  void update_grad(int iter);
  void plain_epoch(int iter);
  void ess_epoch(int iter);
  double sumsq(const float *x, long long n);
};

}  // namespace swfwi

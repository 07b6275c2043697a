// Propagator: Damp4t10d on the GPU (src/modeling/damp4t10d.cpp) and the
// batched shot loops of the FWI frameworks.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <utility>
#include "engine.hpp"
#include "precond.hpp"

namespace swfwi {

namespace {
constexpr int kPartials = 256;   // FP64 partial sums per slot in reductions
long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }
}  // namespace

// ---- stencil launch timing (CUDA events around each step launch) -------
StepTimer &step_timer() {
  static StepTimer t;
  return t;
}

namespace {
// the capture in progress on this thread, and its thread's launch count at
// its start
thread_local StepTimer::Capture *t_capturing = nullptr;
thread_local long long t_capture_notes0 = 0;
}  // namespace

StepTimer::Capture::~Capture() {
  for (auto &e : pairs) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
}

void StepTimer::reset() {
  std::lock_guard<std::mutex> g(mu);
  used = 0;
  launches = 0;
  points = bytes = 0;
  graph_ms = 0;
  graph_timed = 0;
  for (Capture *c : replayed) c->pending = false;   // launched before the reset: not counted
  replayed.clear();
  g_kernel_launches.store(0);
}

void StepTimer::harvest(Capture *c) {
  if (!c->pending) return;
  for (auto &e : c->pairs) {
    SWFWI_CUDA(cudaEventSynchronize(e.second));
    float t = 0;
    SWFWI_CUDA(cudaEventElapsedTime(&t, e.first, e.second));
    graph_ms += t;
  }
  graph_timed += (long long)c->pairs.size();
  c->pending = false;
}

void StepTimer::read(double &ms, long long &n, double &pts, double &b, long long &timed) {
  std::lock_guard<std::mutex> g(mu);
  for (Capture *c : replayed) harvest(c);
  replayed.clear();
  ms = graph_ms;
  for (size_t i = 0; i < used; i++) {
    SWFWI_CUDA(cudaEventSynchronize(pool[i].second));
    float t = 0;
    SWFWI_CUDA(cudaEventElapsedTime(&t, pool[i].first, pool[i].second));
    ms += t;
  }
  n = launches;
  pts = points;
  b = bytes;
  timed = (long long)used + graph_timed;
}

// Algorithmic work of one step launch: every interior point of every field
// is updated (read current and previous, write next: 3 elements), and each
// velocity model the launch uses is read once.  Inside a capture the work
// goes to the capture (added per replay) and a timed launch gets its own
// event pair, recorded as graph nodes.
cudaEvent_t StepTimer::open(cudaStream_t st, double pts, int n, int nvel, int el) {
  if (!enabled.load(std::memory_order_relaxed)) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  Capture *c = t_capturing;
  const long long k = c ? c->launches++ : launches++;
  (c ? c->points : points) += pts * n;
  (c ? c->bytes : bytes) += pts * n * 3 * el + pts * el * nvel;
  const int per = std::max(period.load(std::memory_order_relaxed), 1);
  if (k % per != 0) return nullptr;
  if (c) {
    cudaEvent_t x, y;
    SWFWI_CUDA(cudaEventCreate(&x));
    SWFWI_CUDA(cudaEventCreate(&y));
    c->pairs.emplace_back(x, y);
    SWFWI_CUDA(cudaEventRecordWithFlags(x, st, cudaEventRecordExternal));
    return y;
  }
  if (used == pool.size()) {
    cudaEvent_t x, y;
    SWFWI_CUDA(cudaEventCreate(&x));
    SWFWI_CUDA(cudaEventCreate(&y));
    pool.emplace_back(x, y);
  }
  auto ev = pool[used++];
  SWFWI_CUDA(cudaEventRecord(ev.first, st));
  return ev.second;
}

void StepTimer::close(cudaEvent_t done, cudaStream_t st) {
  if (!done) return;
  if (t_capturing) SWFWI_CUDA(cudaEventRecordWithFlags(done, st, cudaEventRecordExternal));
  else SWFWI_CUDA(cudaEventRecord(done, st));
}

void StepTimer::begin_capture(Capture *c) {
  t_capturing = c;
  t_capture_notes0 = thread_launches();
}

void StepTimer::end_capture() {
  if (t_capturing) {
    t_capturing->kernels = thread_launches() - t_capture_notes0;
    g_kernel_launches.fetch_sub(t_capturing->kernels);
  }
  t_capturing = nullptr;
}

void StepTimer::replay(Capture *c) {
  std::lock_guard<std::mutex> g(mu);
  harvest(c);   // the previous replay's times, before this one overwrites them
  launches += c->launches;
  points += c->points;
  bytes += c->bytes;
  g_kernel_launches.fetch_add(c->kernels);
  if (!c->pairs.empty()) {
    c->pending = true;
    if (std::find(replayed.begin(), replayed.end(), c) == replayed.end()) replayed.push_back(c);
  }
}

void StepTimer::forget(Capture *c) {
  std::lock_guard<std::mutex> g(mu);
  harvest(c);
  replayed.erase(std::remove(replayed.begin(), replayed.end(), c), replayed.end());
  if (t_capturing == c) t_capturing = nullptr;
}

Propagator::Propagator(const Line &src, const Line &geo, float dt_, float dx_, float fm_, int nb_,
                       int nt_)
    : nx(0), nz(0), nb(nb_), nt(nt_), ns(src.n), ng(geo.n), ngmax(geo.n), dt(dt_), dx(dx_),
      fm(fm_), nxpad(0), nzpad(0), pitch(0), fstride(0), bsize(0) {
  SWFWI_REQUIRE(nb_ >= 0 && nt_ > 0 && src.n > 0 && geo.n > 0, "bad propagator sizes");
  SWFWI_REQUIRE(dt_ > 0 && dx_ > 0 && fm_ > 0, "dt, dx, fm must be positive");
  // Damp4t10d::Damp4t10d (damp4t10d.cpp:367-376)
  bz0 = 6;
  bx0 = bxn = bzn = nb_ + 6;
  // fwiRemoveDirectArrival: t_width = 1.5 / fm in double stored as float,
  // half_len = t_width / dt truncated (damp4t10d.cpp:322, 391).
  float t_width = (float)(1.5 / (double)fm_);
  half_len = (int)(t_width / dt_);
  h_src_x.resize(ns);
  h_src_z.resize(ns);
  for (int i = 0; i < ns; i++) {
    h_src_x[i] = src.x(i);
    h_src_z[i] = src.z(i);
  }
  h_geo_x.resize(ng);
  h_geo_z.resize(ng);
  for (int i = 0; i < ng; i++) {
    h_geo_x[i] = geo.x(i);
    h_geo_z[i] = geo.z(i);
  }
  h_rec_count.assign(ns, ng);
  h_rec_x.resize((size_t)ns * ng);
  h_rec_z.resize((size_t)ns * ng);
  for (int s = 0; s < ns; s++)
    for (int i = 0; i < ng; i++) {
      h_rec_x[(size_t)s * ng + i] = h_geo_x[i];
      h_rec_z[(size_t)s * ng + i] = h_geo_z[i];
    }
  d_err_.resize(1);
  SWFWI_CUDA(cudaMemset(d_err_.get(), 0, sizeof(int)));
}

// the handle owns no stream: work goes to the caller's (default: legacy stream 0)
Propagator::~Propagator() {
  for (auto &c : gcache_)
    for (LoopGraph &g : c) {
      if (g.timing) step_timer().forget(g.timing.get());
      if (g.exec) cudaGraphExecDestroy(g.exec);
    }
  if (cap_) cudaStreamDestroy(cap_);
}

void Propagator::loop_key_common(std::vector<long long> &k) const {
  const long long v[] = {nxpad, nzpad, pitch, fstride, bsize, bx0, nt, arith, strip_format, stream_kernel,
                         stream_bz, stream_xchunk, stream_depth, stream_shot_major, fuse ? 1 : 0,
                         reinterpret_cast<long long>(illum), illum_every, vel_stride_,
                         reinterpret_cast<long long>(damp_x_.get()), reinterpret_cast<long long>(damp_z_.get()),
                         reinterpret_cast<long long>(d_err_.get())};
  k.insert(k.end(), std::begin(v), std::end(v));
}

template <typename F>
void Propagator::run_loop(int which, double points_per_step, const std::vector<long long> &key_in, F &&body) {
  // mode 1 captures from a loop's second use (a loop run once costs no
  // capture), mode 2 from its first
  const bool use = graphs > 0 && (loop_warm_[which] || graphs == 2) &&
                   (graphs == 2 || points_per_step <= kGraphMaxPoints);
  loop_warm_[which] = true;
  if (!use) {
    body();
    return;
  }
  // a graph captured with stencil timing off has no event nodes: the key
  // carries the timing setting
  std::vector<long long> key = key_in;
  const StepTimer &tm = step_timer();
  key.push_back(tm.enabled.load(std::memory_order_relaxed) ? tm.period.load(std::memory_order_relaxed) : 0);
  std::vector<LoopGraph> &cache = gcache_[which];
  for (size_t i = 0; i < cache.size(); i++)
    if (cache[i].key == key) {
      if (i) std::swap(cache[i], cache[0]);   // most recent first
      SWFWI_CUDA(cudaGraphLaunch(cache[0].exec, st_));
      step_timer().replay(cache[0].timing.get());
      return;
    }
  if (!cap_) SWFWI_CUDA(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking));
  cudaStream_t user = st_;
  cudaGraph_t g = nullptr;
  LoopGraph e;
  e.key = key;
  e.timing.reset(new StepTimer::Capture);
  SWFWI_CUDA(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal));
  st_ = cap_;
  step_timer().begin_capture(e.timing.get());
  try {
    body();
  } catch (...) {
    step_timer().end_capture();
    st_ = user;
    cudaStreamEndCapture(cap_, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  step_timer().end_capture();
  st_ = user;
  SWFWI_CUDA(cudaStreamEndCapture(cap_, &g));
  cudaError_t err = cudaGraphInstantiate(&e.exec, g, 0);
  cudaGraphDestroy(g);
  SWFWI_CUDA(err);
  if (cache.size() >= kGraphCache) {
    if (cache.back().timing) step_timer().forget(cache.back().timing.get());
    cudaGraphExecDestroy(cache.back().exec);
    cache.pop_back();
  }
  cache.insert(cache.begin(), std::move(e));
  SWFWI_CUDA(cudaGraphLaunch(cache[0].exec, st_));
  step_timer().replay(cache[0].timing.get());
}

void Propagator::set_stream(cudaStream_t s) { st_ = s; }

void Propagator::set_receivers_per_shot(const int *offsets, const int *gx, const int *gz) {
  SWFWI_REQUIRE(offsets && gx && gz, "null receiver arrays");
  SWFWI_REQUIRE(offsets[0] == 0, "offsets[0] must be 0");
  int m = 0;
  for (int s = 0; s < ns; s++) {
    int c = offsets[s + 1] - offsets[s];
    SWFWI_REQUIRE(c > 0, "every shot needs at least one receiver");
    m = std::max(m, c);
  }
  ngmax = m;
  h_rec_count.resize(ns);
  h_rec_x.assign((size_t)ns * ngmax, -1);
  h_rec_z.assign((size_t)ns * ngmax, -1);
  for (int s = 0; s < ns; s++) {
    h_rec_count[s] = offsets[s + 1] - offsets[s];
    for (int i = 0; i < h_rec_count[s]; i++) {
      h_rec_x[(size_t)s * ngmax + i] = gx[offsets[s] + i];
      h_rec_z[(size_t)s * ngmax + i] = gz[offsets[s] + i];
    }
  }
  if (nxpad) upload_geometry();
}

// expandDomain (damp4t10d.cpp:138-151): edge replication by nb
// (expandBndry :96-124, free surface on top), transform
// v -> dx^2/(v^2 dt^2) (transvel :126-130), then a 6-cell halo all round
// (expandForStencil/fillForStencil :47-94).  Host float arithmetic in the
// reference's order.
void Propagator::expand_domain(const float *v, float *out) const {
  SWFWI_REQUIRE(nx > 0 && nz > 0, "model size unknown");
  int nxb = nx + 2 * nb, nzb = nz + nb;
  std::vector<float> b((size_t)nxb * nzb);
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) b[(size_t)(nb + ix) * nzb + iz] = v[(size_t)ix * nz + iz];
  for (int ix = 0; ix < nb; ix++)
    for (int iz = 0; iz < nz; iz++) {
      b[(size_t)ix * nzb + iz] = v[iz];
      b[(size_t)(nb + nx + ix) * nzb + iz] = v[(size_t)(nx - 1) * nz + iz];
    }
  for (int ix = 0; ix < nxb; ix++)
    for (int iz = 0; iz < nb; iz++) b[(size_t)ix * nzb + nz + iz] = b[(size_t)ix * nzb + nz - 1];
  for (float &x : b) x = (dx * dx) / (x * x * dt * dt);
  const int h = 6;
  int nzp = nzb + 2 * h, nxp = nxb + 2 * h;
  for (int ix = h; ix < nxb + h; ix++)
    for (int iz = h; iz < nzb + h; iz++)
      out[(size_t)ix * nzp + iz] = b[(size_t)(ix - h) * nzb + (iz - h)];
  for (int ix = h; ix < nxb + h; ix++) {
    for (int iz = 0; iz < h; iz++) out[(size_t)ix * nzp + iz] = out[(size_t)ix * nzp + h];
    for (int iz = nzb + h; iz < nzp; iz++) out[(size_t)ix * nzp + iz] = out[(size_t)ix * nzp + nzb + h - 1];
  }
  for (int iz = 0; iz < nzp; iz++) {
    for (int ix = 0; ix < h; ix++) out[(size_t)ix * nzp + iz] = out[(size_t)h * nzp + iz];
    for (int ix = nxb + h; ix < nxp; ix++) out[(size_t)ix * nzp + iz] = out[(size_t)(nxb + h - 1) * nzp + iz];
  }
}

void Propagator::upload_geometry() {
  std::vector<int> sp(ns), spp(ns), sx(ns), sz(ns), gp(ng), gpp(ng), gxp(ng), gzp(ng);
  auto inside = [&](int x, int z) { return x >= 6 && x < nxpad - 6 && z >= 6 && z < nzpad - 6; };
  for (int i = 0; i < ns; i++) {
    sx[i] = h_src_x[i] + bx0;
    sz[i] = h_src_z[i] + bz0;
    SWFWI_REQUIRE(inside(sx[i], sz[i]), "source outside the computing zone");
    sp[i] = sx[i] * nzpad + sz[i];
    spp[i] = sx[i] * pitch + sz[i];
  }
  for (int i = 0; i < ng; i++) {
    gxp[i] = h_geo_x[i] + bx0;
    gzp[i] = h_geo_z[i] + bz0;
    SWFWI_REQUIRE(inside(gxp[i], gzp[i]), "receiver outside the computing zone");
    gp[i] = gxp[i] * nzpad + gzp[i];
    gpp[i] = gxp[i] * pitch + gzp[i];
  }
  size_t nr = (size_t)ns * ngmax;
  std::vector<int> rpp(nr, -1), rx(nr, -1), rz(nr, -1);
  for (size_t k = 0; k < nr; k++) {
    if (h_rec_x[k] < 0) continue;
    rx[k] = h_rec_x[k] + bx0;
    rz[k] = h_rec_z[k] + bz0;
    SWFWI_REQUIRE(inside(rx[k], rz[k]), "receiver outside the computing zone");
    rpp[k] = rx[k] * pitch + rz[k];
  }
  // Positions within one injection set must be distinct (the reference adds
  // sequentially; the device adds in parallel).
  {
    std::vector<int> t = sp;
    std::sort(t.begin(), t.end());
    SWFWI_REQUIRE(std::adjacent_find(t.begin(), t.end()) == t.end(), "duplicate source positions");
    t = gp;
    std::sort(t.begin(), t.end());
    SWFWI_REQUIRE(std::adjacent_find(t.begin(), t.end()) == t.end(), "duplicate receiver positions");
    for (int s = 0; s < ns; s++) {
      std::vector<int> r(rpp.begin() + (size_t)s * ngmax, rpp.begin() + (size_t)(s + 1) * ngmax);
      r.erase(std::remove(r.begin(), r.end(), -1), r.end());
      std::sort(r.begin(), r.end());
      SWFWI_REQUIRE(std::adjacent_find(r.begin(), r.end()) == r.end(), "duplicate receiver positions");
    }
  }
  d_src_pos_.upload(sp, st_);
  d_src_pos_p_.upload(spp, st_);
  d_src_x_.upload(sx, st_);
  d_src_z_.upload(sz, st_);
  d_geo_pos_.upload(gp, st_);
  d_geo_pos_p_.upload(gpp, st_);
  d_geo_x_.upload(gxp, st_);
  d_geo_z_.upload(gzp, st_);
  d_rec_pos_p_.upload(rpp, st_);
  d_rec_x_.upload(rx, st_);
  d_rec_z_.upload(rz, st_);
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

// Called once the padded size is known (from expandDomain or a bind).
void Propagator::set_dims(int nxpad_, int nzpad_) {
  SWFWI_REQUIRE(nxpad_ > 2 * bx0 && nzpad_ > bz0 + bzn, "grid smaller than its padding");
  if (nxpad == nxpad_ && nzpad == nzpad_) return;
  nxpad = nxpad_;
  nzpad = nzpad_;
  nx = nxpad - 2 * nb - 12;
  nz = nzpad - nb - 12;
  // rows keep 8 spare floats before depth 0 (the origin offset) and end on a
  // 32-byte boundary; slots hold the origin offset plus all rows
  pitch = (int)round_up(nzpad + kStreamCoff, 8);
  fstride = round_up((long long)nxpad * pitch + 2 * kStreamCoff, 64);
  damp_x_.resize(nxpad);
  damp_z_.resize(nzpad);
  coef_x_.resize(nxpad);
  launch_damp_tables(damp_x_.get(), damp_z_.get(), coef_x_.get(), nxpad, nzpad, bx0, st_);
  bsize = strip_size(nxpad, nzpad, bx0);
  rcp_for_ = nullptr;
  upload_geometry();
}

void Propagator::bind_velocity(const float *exvel) {
  SWFWI_REQUIRE(exvel != nullptr, "null velocity");
  SWFWI_REQUIRE(nxpad > 12 && nzpad > 12, "padded size unknown");
  vel_ = exvel;
  rcp_for_ = nullptr;   // contents may have changed: recompute 1/vt lazily
}

const float *Propagator::rcp_of(const float *vel) {
  SWFWI_REQUIRE(vel != nullptr, "no velocity bound");
  size_t n = (size_t)nxpad * pitch;
  if (vel == vel_) {
    if (rcp_for_ != vel_) {
      rcp_.resize(n + 2 * kStreamCoff);
      launch_pitched_reciprocal(rcp_.get() + kStreamCoff, vel_, nxpad, nzpad, pitch, st_);
      rcp_for_ = vel_;
    }
    return rcp_.get() + kStreamCoff;
  }
  trial_rcp_.resize(n + 2 * kStreamCoff);
  launch_pitched_reciprocal(trial_rcp_.get() + kStreamCoff, vel, nxpad, nzpad, pitch, st_);
  return trial_rcp_.get() + kStreamCoff;
}

void Propagator::check_device_error() {
  int e = 0;
  SWFWI_CUDA(cudaMemcpyAsync(&e, d_err_.get(), sizeof(int), cudaMemcpyDeviceToHost, st_));
  SWFWI_CUDA(cudaStreamSynchronize(st_));
  if (e) {
    SWFWI_CUDA(cudaMemsetAsync(d_err_.get(), 0, sizeof(int), st_));
    throw Error(SWFWI_ERR_TIMEOUT, "a stencil kernel's bounded wait on its row pipeline gave up");
  }
}

// One FD step for n propagator-owned fields (pitched rows, fstride apart,
// one velocity model): the streaming TMA kernel for float arithmetics, the
// shared-memory tile kernel for FP64.
void Propagator::step_fields(int ar, bool damped, void *prev, const void *curr, const void *velrcp,
                             int n, const Epilogue *epi, void *out) {
  double pts = (double)(nxpad - 12) * (nzpad - 12);
  if (ar == ARITH_F64) {
    cudaEvent_t done = step_timer().open(st_, pts, n, 1, 8);
    StepArgs a;
    a.prev = prev;
    a.out = out;
    a.curr = curr;
    a.vel = velrcp;
    a.nx = nxpad;
    a.nz = nzpad;
    a.pitch = pitch;
    a.bx0 = bx0;
    a.shot_stride = fstride;
    a.vel_stride = 0;
    a.shots_per_vel = std::max(n, 1);
    launch_step(ARITH_F64, damped, true, 32, a, n, st_);
    step_timer().close(done, st_);
    return;
  }
  cudaEvent_t done = step_timer().open(st_, pts, n, vel_stride_ ? n : 1, 4);
  StreamArgs a;
  a.prev = static_cast<float *>(prev);
  a.out = static_cast<float *>(out);
  a.curr = static_cast<const float *>(curr);
  a.rcp = static_cast<const float *>(velrcp);
  a.damp_x = damp_x_.get();
  a.coef_x = coef_x_.get();
  a.ramp = bx0;   // launch_damp_tables ramp length
  a.epi = epi ? *epi : Epilogue{};
  a.damp_z = damp_z_.get();
  a.nx = nxpad;
  a.nz = nzpad;
  a.pitch = pitch;
  a.shot_stride = fstride;
  a.vel_stride = vel_stride_;
  a.shots_per_vel = vel_stride_ ? 1 : std::max(n, 1);
  a.xchunk = stream_xchunk;
  a.shot_major = stream_shot_major;
  a.err = d_err_.get();
  if (epi) {
    // the fused step is the warp-specialised kernel with 376-deep bands
    if (stream_kernel != 1 || a.xchunk <= 0) a.xchunk = 64;
    launch_ws_step(ar, damped, 376, stream_kernel == 1 ? stream_depth : 3, a, n, st_);
  } else if (stream_kernel == 6 && ar == ARITH_FAST) {
    launch_rq2_step(damped, a, n, st_);   // xchunk 0: automatic
  } else if (stream_kernel == 5 || stream_kernel == 6) {
    // kernel 6 runs FAST arithmetic only: REF takes kernel 5
    launch_rq_step(ar, damped, stream_kernel == 6 ? 3 : stream_depth, a, n, st_);   // xchunk 0: automatic
  } else {
    if (a.xchunk <= 0) a.xchunk = 64;
    launch_ws_step(ar, damped, stream_bz, stream_depth, a, n, st_);
  }
  step_timer().close(done, st_);
}

// ---- single-field operations on caller arrays ([nxpad][nzpad]) ---------
namespace {
StepArgs caller_args(float *p0, const float *p1, const float *vel, int nxpad, int nzpad, int bx0) {
  StepArgs a;
  a.prev = p0;
  a.curr = p1;
  a.vel = vel;
  a.nx = nxpad;
  a.nz = nzpad;
  a.pitch = nzpad;
  a.bx0 = bx0;
  a.shot_stride = 0;
  a.vel_stride = 0;
  a.shots_per_vel = 1;
  return a;
}
}  // namespace

void Propagator::step_forward(float *p0, float *p1) {
  SWFWI_REQUIRE(p0 && p1 && vel_, "null field or no velocity");
  cudaEvent_t done = step_timer().open(st_, (double)(nxpad - 12) * (nzpad - 12), 1, 1, 4);
  launch_step(arith, true, false, 32, caller_args(p0, p1, vel_, nxpad, nzpad, bx0), 1, st_);
  step_timer().close(done, st_);
}

void Propagator::step_backward(float *p0, float *p1) {
  SWFWI_REQUIRE(p0 && p1 && vel_, "null field or no velocity");
  cudaEvent_t done = step_timer().open(st_, (double)(nxpad - 12) * (nzpad - 12), 1, 1, 4);
  launch_step(arith, false, false, 32, caller_args(p0, p1, vel_, nxpad, nzpad, bx0), 1, st_);
  step_timer().close(done, st_);
}

void Propagator::manip_source(float *p, const float *src, int shot_id, int sign) {
  SWFWI_REQUIRE(p && src, "null pointer");
  SWFWI_REQUIRE(shot_id >= -1 && shot_id < ns, "shot id out of range");
  PointSet ps;
  if (shot_id >= 0) ps = {d_src_pos_.get() + shot_id, 1, nullptr};
  else ps = {d_src_pos_.get(), ns, nullptr};
  launch_inject<float>(p, 0, 1, ps, src, 0, 1, sign, st_);
}

void Propagator::add_receiver_source(float *p, const float *vsrc_it) {
  SWFWI_REQUIRE(p && vsrc_it, "null pointer");
  launch_inject<float>(p, 0, 1, PointSet{d_geo_pos_.get(), ng, nullptr}, vsrc_it, 0, 1, +1, st_);
}

void Propagator::record_seis(float *seis, const float *p) {
  SWFWI_REQUIRE(seis && p, "null pointer");
  launch_record<float>(seis, 0, p, 0, 1, PointSet{d_geo_pos_.get(), ng, nullptr}, st_);
}

void Propagator::write_bndry(float *bndr, const float *p, int it) {
  SWFWI_REQUIRE(bndr && p && it >= 0, "bad strip arguments");
  launch_strip_write<float>(bndr + (long long)it * bsize, 0, p, 0, 1, nxpad, nzpad, bx0, nzpad, st_);
}

void Propagator::read_bndry(const float *bndr, float *p, int it) {
  SWFWI_REQUIRE(bndr && p && it >= 0, "bad strip arguments");
  launch_strip_read<float>(bndr + (long long)it * bsize, 0, p, 0, 1, nxpad, nzpad, bx0, nzpad, st_);
}

namespace {
__global__ void k_mask(float *g, int nxpad, int nzpad, int bx0, int bz0, int bxn, int bzn) {
  int n = nxpad * nzpad;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    int ix = q / nzpad, iz = q - ix * nzpad;
    if (ix < bx0 || iz < bz0 || ix >= nxpad - bxn || iz >= nzpad - bzn) g[q] = 0.f;
  }
}
__global__ void k_scale(float *g, int nxpad, int nzpad, int bx0, int bz0, int bxn, int bzn) {
  int nzi = nzpad - bz0 - bzn;
  int nxi = nxpad - bx0 - bxn;
  int n = nxi * nzi;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    int ix = q / nzi, iz = q - ix * nzi;
    if (iz < 1) continue;
    float *p = g + (long long)(ix + bx0) * nzpad + iz + bz0;
    *p = __fmul_rn(*p, __fsqrt_rn((float)iz));
  }
}
}  // namespace

void Propagator::mask_gradient(float *g) {
  SWFWI_REQUIRE(g, "null gradient");
  k_mask<<<592, 256, 0, st_>>>(g, nxpad, nzpad, bx0, bz0, bxn, bzn);
  g_kernel_launches++;
}

void Propagator::scale_gradient(float *g) {
  SWFWI_REQUIRE(g, "null gradient");
  k_scale<<<592, 256, 0, st_>>>(g, nxpad, nzpad, bx0, bz0, bxn, bzn);
  g_kernel_launches++;
}

void Propagator::refill_boundary(float *v) {
  SWFWI_REQUIRE(v, "null array");
  launch_refill_boundary(v, nxpad, nzpad, bz0, bzn, bx0, bxn, st_);
}

void Propagator::remove_direct_arrival(float *data, int shot_id, const float *vel) {
  SWFWI_REQUIRE(data, "null data");
  SWFWI_REQUIRE(shot_id >= -1 && shot_id < ns, "shot id out of range");
  const float *v = vel ? vel : vel_;
  SWFWI_REQUIRE(v, "no velocity bound");
  int s = shot_id < 0 ? 0 : shot_id;   // removeDirectArrival uses source 0
  d_win1_.resize((size_t)2 * ng);
  launch_mute_windows(d_win1_.get(), v, nxpad, nzpad, d_src_x_.get() + s, d_src_z_.get() + s,
                      d_geo_x_.get(), d_geo_z_.get(), 0, ng, nullptr, half_len, nt, 1, st_);
  launch_apply_mute(data, 0, d_win1_.get(), nt, ng, 1, st_);
}

// ---- time loops ----------------------------------------------------------
template <typename T>
void Propagator::ensure_work(Work<T> &w, int n, bool strips) {
  size_t f = (size_t)n * fstride;
  w.p0.resize(f);
  w.p1.resize(f);
  if (strips && recon == SWFWI_RECON_SNAPSHOTS) {
    const size_t m = (size_t)snapshot_count();
    if (sizeof(T) == 4 && snap_format != SWFWI_STRIP_F32) {
      w.qsnaps.resize(m * 2 * n * (size_t)nxpad * pitch);
      w.qsnap_scale.resize(m * 2 * n);
      w.snap_pmax.resize((size_t)n * kSnapParts);
    } else {
      w.snaps.resize(m * 2 * f);
    }
    // the kernels never write a field's border, coordinate margin or tail:
    // zero once, they stay zero through restores and out-of-place steps
    w.ring.resize((size_t)(snap_every + 1) * f);
    w.ring.zero(st_);
  } else if (strips) {
    if (sizeof(T) == 4 && strip_format != SWFWI_STRIP_F32) {
      w.qstrips.resize((size_t)n * nt * bsize);
      w.qscale.resize((size_t)n * nt);
    } else {
      w.strips.resize((size_t)n * nt * bsize);
    }
  }
  w.partials.resize((size_t)n * kPartials);
  w.obj.resize(n);
}

bool Propagator::line_of(const int *xs, const int *zs, int n, PtLine &out) const {
  if (n <= 0) return false;
  out = PtLine{xs[0] + bx0, zs[0] + bz0, 0, 0, n};
  if (n == 1) return true;
  out.jx = xs[1] - xs[0];
  out.jz = zs[1] - zs[0];
  if (out.jx == 0 && out.jz == 0) return false;
  for (int i = 2; i < n; i++)
    if (xs[i] - xs[i - 1] != out.jx || zs[i] - zs[i - 1] != out.jz) return false;
  return true;
}

// The fused steps inject at a line's single depth: horizontal lines or points.
static bool injectable(const std::vector<PtLine> &ls) {
  for (const PtLine &l : ls)
    if (!(l.n == 1 || l.jz == 0)) return false;
  return true;
}

bool Propagator::shot_lines(const int *ids, int k, bool per_shot_receivers, std::vector<PtLine> &src,
                            std::vector<PtLine> &rec) const {
  src.resize(k);
  rec.resize(k);
  for (int j = 0; j < k; j++) {
    const int s = ids[j];
    if (!line_of(&h_src_x[s], &h_src_z[s], 1, src[j])) return false;
    const bool ok = per_shot_receivers
                        ? line_of(&h_rec_x[(size_t)s * ngmax], &h_rec_z[(size_t)s * ngmax], h_rec_count[s], rec[j])
                        : line_of(h_geo_x.data(), h_geo_z.data(), ng, rec[j]);
    if (!ok) return false;
  }
  return true;
}

bool Propagator::ess_lines(int k, std::vector<PtLine> &src, std::vector<PtLine> &rec) const {
  PtLine s, r;
  if (!line_of(h_src_x.data(), h_src_z.data(), ns, s) || !line_of(h_geo_x.data(), h_geo_z.data(), ng, r))
    return false;
  src.assign(k, s);
  rec.assign(k, r);
  return true;
}

// Snapshot m: the pair (a, b) = (p0, p1) after forward step
// (m + 1) * snap_every - 1, every slot's whole field (F32 or the element
// type: a copy of the n slots' contiguous fields; 16-bit: the values from
// each origin over nxpad x pitch, one scale per field, slot and snapshot).
template <typename T>
void Propagator::save_snapshot(Work<T> &w, int n, int m, const T *a, const T *b) {
  const long long f = (long long)n * fstride;
  const T *src[2] = {a, b};
  for (int k = 0; k < 2; k++) {
    if (sizeof(T) == 4 && snap_format != SWFWI_STRIP_F32) {
      const long long count = (long long)nxpad * pitch;
      launch_field_write_q(snap_format, w.qsnaps.get() + ((long long)m * 2 + k) * n * count,
                           w.qsnap_scale.get() + ((long long)m * 2 + k) * n, 1, w.snap_pmax.get(),
                           reinterpret_cast<const float *>(src[k]), fstride, count, n, st_);
    } else {
      SWFWI_CUDA(cudaMemcpyAsync(w.snaps.get() + ((long long)m * 2 + k) * f, src[k] - kStreamCoff, f * sizeof(T),
                                 cudaMemcpyDeviceToDevice, st_));
    }
  }
}

template <typename T>
void Propagator::restore_snapshot(Work<T> &w, int n, int m, T *a, T *b) {
  const long long f = (long long)n * fstride;
  T *dst[2] = {a, b};
  for (int k = 0; k < 2; k++) {
    if (sizeof(T) == 4 && snap_format != SWFWI_STRIP_F32) {
      const long long count = (long long)nxpad * pitch;
      launch_field_read_q(snap_format, w.qsnaps.get() + ((long long)m * 2 + k) * n * count,
                          w.qsnap_scale.get() + ((long long)m * 2 + k) * n, 1, reinterpret_cast<float *>(dst[k]),
                          fstride, count, n, st_);
    } else {
      SWFWI_CUDA(cudaMemcpyAsync(dst[k] - kStreamCoff, w.snaps.get() + ((long long)m * 2 + k) * f, f * sizeof(T),
                                 cudaMemcpyDeviceToDevice, st_));
    }
  }
}

template <typename T>
void Propagator::run_forward(Work<T> &w, int n, PointSet src, const T *vals, long long it_stride,
                             long long slot_stride, int i_stride, PointSet rec, int ngrec, T *dcal,
                             bool save_strips, const void *velrcp) {
  ensure_work(w, n, save_strips);
  T *p0 = w.p0.get() + kStreamCoff, *p1 = w.p1.get() + kStreamCoff;
  w.p0.zero(st_);
  w.p1.zero(st_);
  int ar = sizeof(T) == 8 ? (int)ARITH_F64 : arith;
  long long bstride = (long long)nt * bsize;
  std::vector<long long> key = {
      (long long)sizeof(T), n, reinterpret_cast<long long>(src.pos), src.per_shot,
      reinterpret_cast<long long>(src.slot_shot), reinterpret_cast<long long>(vals), it_stride, slot_stride,
      i_stride, reinterpret_cast<long long>(rec.pos), rec.per_shot, reinterpret_cast<long long>(rec.slot_shot),
      ngrec, reinterpret_cast<long long>(dcal), save_strips ? 1 : 0, reinterpret_cast<long long>(velrcp),
      reinterpret_cast<long long>(p0), reinterpret_cast<long long>(p1),
      reinterpret_cast<long long>(w.strips.get()), reinterpret_cast<long long>(w.qstrips.get()),
      reinterpret_cast<long long>(w.qscale.get())};
  // checkpoint snapshots instead of strips
  const bool gradient_sweep = save_strips;
  const int nsnap = save_strips ? snapshot_count() : 0;
  if (save_strips && recon == SWFWI_RECON_SNAPSHOTS) {
    save_strips = false;
    for (long long v : {(long long)recon, (long long)snap_every, (long long)snap_format,
                        reinterpret_cast<long long>(w.snaps.get()), reinterpret_cast<long long>(w.qsnaps.get()),
                        reinterpret_cast<long long>(w.qsnap_scale.get())})
      key.push_back(v);
  }
  loop_key_common(key);
  const bool qstrips = save_strips && sizeof(T) == 4 && strip_format != SWFWI_STRIP_F32;
  run_loop(0, (double)n * nxpad * nzpad, key, [&] {
  // addSource -> stepForward -> swap -> recordSeis / writeBndry
  // (damp4t10d.cpp:283-288, fwiframework.cpp:137-144); the record, the FP32
  // strips and the next step's addSource share one launch
  launch_inject<T>(p1, fstride, n, src, vals, slot_stride, i_stride, +1, st_);
  for (int it = 0; it < nt; it++) {
    step_fields(ar, true, p0, p1, velrcp, n);
    std::swap(p0, p1);
    const bool more = it + 1 < nt;
    launch_after_forward<T>(dcal ? dcal + (long long)it * ngrec : nullptr, (long long)nt * ngrec, p0, rec,
                            save_strips && !qstrips ? w.strips.get() + (long long)it * bsize : nullptr, bstride,
                            nxpad, nzpad, bx0, pitch, more ? p1 : nullptr, src,
                            more ? vals + (long long)(it + 1) * it_stride : nullptr, slot_stride, i_stride,
                            fstride, n, st_);
    if (qstrips)
      launch_strip_write_q(strip_format, w.qstrips.get() + (long long)it * bsize, bstride, w.qscale.get() + it,
                           nt, reinterpret_cast<const float *>(p0), fstride, n, nxpad, nzpad, bx0, pitch, st_);
    if (nsnap > 0 && (it + 1) % snap_every == 0 && (it + 1) / snap_every <= nsnap)
      save_snapshot(w, n, (it + 1) / snap_every - 1, p0, p1);
    if (gradient_sweep && sizeof(T) == 4 && illum && it % std::max(illum_every, 1) == 0)
      launch_illum_accum(illum, reinterpret_cast<const float *>(p0), fstride, n, nxpad, nzpad, pitch, st_);
  }
  });
  // leave the final (current, next) pair for a backward sweep: every step
  // swaps the pair once (decided by nt alone, since a replayed graph does
  // not run the loop's host code)
  if (nt % 2 == 1) std::swap(w.p0, w.p1);
}

template <typename T>
bool Propagator::run_backward(Work<T> &w, int n, PointSet src, const T *vals, long long it_stride,
                              long long slot_stride, int i_stride, PointSet rec, int ngrec,
                              const T *vsrc, const void *velrcp, const std::vector<PtLine> *src_lines,
                              const std::vector<PtLine> *rec_lines, bool sum_images) {
  size_t f = (size_t)n * fstride;
  w.g0.resize(f);
  w.g1.resize(f);
  w.g0.zero(st_);
  w.g1.zero(st_);
  T *sp0 = w.p0.get() + kStreamCoff, *sp1 = w.p1.get() + kStreamCoff;
  T *gp0 = w.g0.get() + kStreamCoff, *gp1 = w.g1.get() + kStreamCoff;
  int ar = sizeof(T) == 8 ? (int)ARITH_F64 : arith;
  long long bstride = (long long)nt * bsize;
  // image every point of the pitched field, nxpad rows of pitch floats from
  // kStreamCoff on: (slot j) j*fstride + kStreamCoff + [0, nxpad*pitch)
  // stays inside the slot's fstride floats
  const int npts = nxpad * pitch;
  std::vector<long long> key = {
      (long long)sizeof(T), n, reinterpret_cast<long long>(src.pos), src.per_shot,
      reinterpret_cast<long long>(src.slot_shot), reinterpret_cast<long long>(vals), it_stride, slot_stride,
      i_stride, reinterpret_cast<long long>(rec.pos), rec.per_shot, reinterpret_cast<long long>(rec.slot_shot),
      ngrec, reinterpret_cast<long long>(vsrc), reinterpret_cast<long long>(velrcp),
      reinterpret_cast<long long>(sp0), reinterpret_cast<long long>(sp1), reinterpret_cast<long long>(gp0),
      reinterpret_cast<long long>(gp1), reinterpret_cast<long long>(w.image.get()),
      reinterpret_cast<long long>(w.strips.get()), reinterpret_cast<long long>(w.qstrips.get()),
      reinterpret_cast<long long>(w.qscale.get()), reinterpret_cast<long long>(w.src_lines.get()),
      reinterpret_cast<long long>(w.rec_lines.get()), (long long)(dt * 1e9)};
  if (recon == SWFWI_RECON_SNAPSHOTS) {
    // Checkpointing: the image at backward step it uses the forward field
    // of step it-1 (what the strips' back-propagation rebuilds in the
    // interior, its source terms aside), taken from a re-run of its segment
    // of snap_every steps from the segment's snapshot.  Ring slot r holds
    // the field of forward step seg * snap_every + r - 1; each re-run step
    // writes a fresh slot (out-of-place) and adds the next source as the
    // forward does.
    const int K = snap_every;
    const bool summed = sum_images && sizeof(T) == 4 && ar == ARITH_FAST;
    for (long long v : {(long long)(3 + (summed ? 1 : 0)), (long long)K, (long long)snap_format,
                        reinterpret_cast<long long>(w.snaps.get()), reinterpret_cast<long long>(w.qsnaps.get()),
                        reinterpret_cast<long long>(w.qsnap_scale.get()), reinterpret_cast<long long>(w.ring.get())})
      key.push_back(v);
    loop_key_common(key);
    const long long block = (long long)n * fstride;
    auto ring_at = [&](int r) { return w.ring.get() + (long long)r * block + kStreamCoff; };
    run_loop(1, (double)n * nxpad * nzpad, key, [&] {
    int seg_cur = -1;
    for (int it = nt - 1; it >= 0; it--) {
      // receivers, as below: addSource -> stepForward -> swap
      launch_inject<T>(gp1, fstride, n, rec, vsrc + (long long)it * ngrec, (long long)nt * ngrec, 1, +1, st_);
      step_fields(ar, true, gp0, gp1, velrcp, n);
      std::swap(gp0, gp1);
      float t = dt * (float)it;
      float scale;
      if ((double)t > 0.4) scale = 1.0f;
      else if ((double)t > 0.3) scale = (float)(((double)t - 0.3) / 0.1);
      else break;
      const int j = it - 1;   // t > 0.3 keeps it >= 1
      const int seg = j / K;
      if (seg != seg_cur) {
        const int a0 = seg * K, b0 = std::min(a0 + K, nt);
        if (seg == 0) {   // the forward's start: zero fields, then the first source
          SWFWI_CUDA(cudaMemsetAsync(ring_at(0) - kStreamCoff, 0, 2 * block * sizeof(T), st_));
          launch_inject<T>(ring_at(1), fstride, n, src, vals, slot_stride, i_stride, +1, st_);
        } else {
          restore_snapshot(w, n, seg - 1, ring_at(0), ring_at(1));
        }
        for (int jj = a0; jj + 1 < b0; jj++) {
          T *nextf = ring_at(jj - a0 + 2);
          step_fields(ar, true, ring_at(jj - a0), ring_at(jj - a0 + 1), velrcp, n, nullptr, nextf);
          launch_inject<T>(nextf, fstride, n, src, vals + (long long)(jj + 1) * it_stride, slot_stride, i_stride,
                           +1, st_);
        }
        seg_cur = seg;
      }
      const T *sf = ring_at(j - seg * K + 1);
      if (summed)
        launch_image_sum(reinterpret_cast<float *>(w.image.get()) + kStreamCoff, reinterpret_cast<const float *>(sf),
                         reinterpret_cast<const float *>(gp0), fstride, n, bx0, nxpad - bxn, bz0, nzpad - bzn, pitch,
                         scale, st_);
      else
        launch_image<T>(w.image.get() + kStreamCoff, fstride, sf, gp0, fstride, n, npts, scale, st_);
    }
    });
    return summed;
  }
  const bool fused = fuse && sizeof(T) == 4 && src_lines && rec_lines && (int)src_lines->size() == n &&
                     (int)rec_lines->size() == n && injectable(*src_lines) && injectable(*rec_lines);
  if (fused) {
    // two launches and the strip restore per step: the source back-step
    // also subtracts the source and images, the receiver step also injects
    // the next residual
    w.src_lines.upload(*src_lines, st_);
    w.rec_lines.upload(*rec_lines, st_);
    key.push_back(1);   // fused
    key.push_back(reinterpret_cast<long long>(w.src_lines.get()));
    key.push_back(reinterpret_cast<long long>(w.rec_lines.get()));
    float *image = reinterpret_cast<float *>(w.image.get()) + kStreamCoff;
    launch_inject<T>(gp1, fstride, n, rec, vsrc + (long long)(nt - 1) * ngrec, (long long)nt * ngrec, 1, +1,
                     st_);
    loop_key_common(key);
    run_loop(1, (double)n * nxpad * nzpad, key, [&] {
    for (int it = nt - 1; it >= 0; it--) {
      launch_strip_read<T>(w.strips.get() + (long long)it * bsize, bstride, sp0, fstride, n, nxpad, nzpad, bx0,
                           pitch, st_);
      std::swap(sp0, sp1);
      float t = dt * (float)it;
      float scale = 0.0f;
      bool last = false;
      if ((double)t > 0.4) scale = 1.0f;
      else if ((double)t > 0.3) scale = (float)(((double)t - 0.3) / 0.1);
      else last = true;   // the reference's loop breaks after this step, before imaging
      Epilogue e{};
      e.src = w.src_lines.get();
      e.sub = reinterpret_cast<const float *>(vals) + (long long)it * it_stride;
      e.sub_slot_stride = slot_stride;
      e.sub_stride = i_stride;
      if (!last) {
        e.image = image;
        e.gcurr = reinterpret_cast<const float *>(gp1);
        e.scale = scale;
      }
      step_fields(ar, false, sp0, sp1, velrcp, n, &e);
      Epilogue r{};
      r.src = w.rec_lines.get();
      if (!last && it >= 1) {
        r.inj = reinterpret_cast<const float *>(vsrc) + (long long)(it - 1) * ngrec;
        r.inj_slot_stride = (long long)nt * ngrec;
        r.inj_stride = 1;
      }
      step_fields(ar, true, gp0, gp1, velrcp, n, r.inj ? &r : nullptr);
      std::swap(gp0, gp1);
      if (last) break;
    }
    });
    return false;
  }
  const bool summed = sum_images && sizeof(T) == 4 && ar == ARITH_FAST;
  key.push_back(summed ? 2 : 0);   // separate launches (2: one summed image)
  loop_key_common(key);
  // With the summed image (interior cells only), step it-1's FP32 strip
  // restore, which writes boundary cells of the field the source
  // subtraction of step it writes, rides in that launch.
  const bool fold_strips = summed && strip_format == SWFWI_STRIP_F32;
  run_loop(1, (double)n * nxpad * nzpad, key, [&] {
  if (fold_strips)
    launch_strip_read<T>(w.strips.get() + (long long)(nt - 1) * bsize, bstride, sp0, fstride, n, nxpad, nzpad, bx0,
                         pitch, st_);
  for (int it = nt - 1; it >= 0; it--) {
    // fwiframework.cpp:146-176: readBndry -> swap -> stepBackward ->
    // subSource; receiver addSource -> stepForward -> swap; image.
    if (sizeof(T) == 4 && strip_format != SWFWI_STRIP_F32)
      launch_strip_read_q(strip_format, w.qstrips.get() + (long long)it * bsize, bstride,
                          w.qscale.get() + it, nt, reinterpret_cast<float *>(sp0), fstride, n, nxpad,
                          nzpad, bx0, pitch, st_);
    else if (!fold_strips)
      launch_strip_read<T>(w.strips.get() + (long long)it * bsize, bstride, sp0, fstride, n, nxpad,
                           nzpad, bx0, pitch, st_);
    std::swap(sp0, sp1);
    step_fields(ar, false, sp0, sp1, velrcp, n);
    const bool next_strip = fold_strips && it > 0;
    launch_inject2<T>(sp0, src, vals + (long long)it * it_stride, slot_stride, i_stride, -1, gp1, rec,
                      vsrc + (long long)it * ngrec, (long long)nt * ngrec, 1, +1, fstride, n, st_,
                      next_strip ? w.strips.get() + (long long)(it - 1) * bsize : nullptr, bstride, nxpad, nzpad,
                      bx0, pitch);
    step_fields(ar, true, gp0, gp1, velrcp, n);
    std::swap(gp0, gp1);
    float t = dt * (float)it;
    float scale;
    if ((double)t > 0.4) scale = 1.0f;
    else if ((double)t > 0.3) scale = (float)(((double)t - 0.3) / 0.1);
    else break;
    if (summed)   // only the gradient's unmasked region (maskGradient, damp4t10d.cpp:216-226) is used
      launch_image_sum(reinterpret_cast<float *>(w.image.get()) + kStreamCoff, reinterpret_cast<const float *>(sp0),
                       reinterpret_cast<const float *>(gp0), fstride, n, bx0, nxpad - bxn, bz0, nzpad - bzn, pitch,
                       scale, st_);
    else
      launch_image<T>(w.image.get() + kStreamCoff, fstride, sp0, gp0, fstride, n, npts, scale, st_);
  }
  });
  return summed;
}

template <typename T>
void Propagator::to_pitched(T *dst, const T *src) {
  SWFWI_CUDA(cudaMemcpy2DAsync(dst, sizeof(T) * pitch, src, sizeof(T) * nzpad, sizeof(T) * nzpad,
                               nxpad, cudaMemcpyDeviceToDevice, st_));
}

template <typename T>
void Propagator::from_pitched(T *dst, const T *src) {
  SWFWI_CUDA(cudaMemcpy2DAsync(dst, sizeof(T) * nzpad, src, sizeof(T) * pitch, sizeof(T) * nzpad,
                               nxpad, cudaMemcpyDeviceToDevice, st_));
}

void Propagator::fwi_forward(const float *wlt, float *dcal, int shot_id) {
  SWFWI_REQUIRE(wlt && dcal, "null pointer");
  SWFWI_REQUIRE(shot_id >= 0 && shot_id < ns, "shot id out of range");
  PointSet src{d_src_pos_p_.get() + shot_id, 1, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  run_forward<float>(w_, 1, src, wlt, 1, 0, 0, rec, ng, dcal, false, rcp_of(vel_));
}

void Propagator::ess_forward(const float *encsrc, float *dcal, const float *vel) {
  SWFWI_REQUIRE(encsrc && dcal, "null pointer");
  PointSet src{d_src_pos_p_.get(), ns, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  run_forward<float>(w_, 1, src, encsrc, ns, 0, 1, rec, ng, dcal, false, rcp_of(vel ? vel : vel_));
}

void Propagator::ess_forward_members(const float *encsrc, const float *vels, int n, float *hona) {
  SWFWI_REQUIRE(encsrc && vels && hona && n > 0, "bad member batch arguments");
  SWFWI_REQUIRE(nxpad > 12 && nzpad > 12, "grid size not set");
  const long long per = (long long)nxpad * pitch;        // floats per member reciprocal
  const long long vsz = (long long)nxpad * nzpad;
  int mb = max_batch();
  for (int c0 = 0; c0 < n; c0 += mb) {
    int k = std::min(mb, n - c0);
    members_rcp_.resize((size_t)k * per + 2 * kStreamCoff);
    float *rcp = members_rcp_.get() + kStreamCoff;
    for (int i = 0; i < k; i++)
      launch_pitched_reciprocal(rcp + i * per, vels + (c0 + i) * vsz, nxpad, nzpad, pitch, st_);
    std::vector<int> zeros(k, 0);                        // every slot: the one encoded supershot
    w_.slot_shot.upload(zeros.data(), k, st_);
    PointSet src{d_src_pos_p_.get(), ns, w_.slot_shot.get()};
    PointSet rec{d_geo_pos_p_.get(), ng, w_.slot_shot.get()};
    w_.dcal.resize((size_t)k * nt * ng);
    struct Restore {
      long long &v;
      ~Restore() { v = 0; }
    } restore{vel_stride_};
    vel_stride_ = per;
    run_forward<float>(w_, k, src, encsrc, ns, 0, 1, rec, ng, w_.dcal.get(), false, rcp);
    vel_stride_ = 0;
    // EssForwardModeling's dcal [nt][ng] -> the matrix column order [ng][nt]
    launch_transpose_traces(hona + (long long)c0 * nt * ng, w_.dcal.get(), nt, ng, k, st_);
  }
  check_device_error();
}

int Propagator::max_batch() const {
  size_t freeb = 0, total = 0;
  if (cudaMemGetInfo(&freeb, &total) != cudaSuccess) return 1;
  // per slot: p0, p1, g0, g1, image fields; strips; dcal, res, vsrc data
  const double strip_bytes = strip_format == SWFWI_STRIP_F32 ? 4.0 : 2.0;
  // reconstruction storage: strips, or snapshots plus the re-forward ring
  const double recon_bytes =
      recon == SWFWI_RECON_SNAPSHOTS
          ? 2.0 * snapshot_count() * (snap_format == SWFWI_STRIP_F32 ? 4.0 * fstride : 2.0 * nxpad * pitch) +
                (snap_every + 1.0) * fstride * 4
          : (double)nt * bsize * strip_bytes;
  double per = 5.0 * fstride * 4 + recon_bytes + 3.0 * nt * ngmax * 4 + 4096;
  double budget = 0.85 * (double)freeb;
  // memory already held by this propagator's work space counts as free
  budget += (double)(w_.p0.capacity() + w_.p1.capacity() + w_.g0.capacity() + w_.g1.capacity() +
                     w_.image.capacity() + w_.strips.capacity() + w_.dcal.capacity() +
                     w_.res.capacity() + w_.vsrc.capacity() + w_.snaps.capacity() + w_.ring.capacity()) * 4 +
            (double)(w_.qstrips.capacity() + w_.qsnaps.capacity()) * 2;
  int m = (int)(budget / per);
  return std::max(1, std::min(m, ns));
}

void Propagator::forward_batch(const float *wlt, float *dcal, const int *ids, int n,
                               const float *vel) {
  SWFWI_REQUIRE(wlt && dcal && ids && n > 0, "bad batch arguments");
  for (int i = 0; i < n; i++) SWFWI_REQUIRE(ids[i] >= 0 && ids[i] < ns, "shot id out of range");
  const float *rcp = rcp_of(vel ? vel : vel_);
  int mb = max_batch();
  for (int c0 = 0; c0 < n; c0 += mb) {
    int k = std::min(mb, n - c0);
    w_.slot_shot.upload(ids + c0, k, st_);
    PointSet src{d_src_pos_p_.get(), 1, w_.slot_shot.get()};
    PointSet rec{d_rec_pos_p_.get(), ngmax, w_.slot_shot.get()};
    run_forward<float>(w_, k, src, wlt, 1, 0, 0, rec, ngmax, dcal + (long long)c0 * nt * ngmax,
                       false, rcp);
  }
}

void Propagator::gradient_batch(const float *wlt, const float *dobs, const int *ids, int n,
                                float *grad, double *obj, bool accumulate, const int *rows,
                                const std::function<void()> *before_residual) {
  SWFWI_REQUIRE(wlt && dobs && ids && grad && n > 0, "bad batch arguments");
  for (int i = 0; i < n; i++) SWFWI_REQUIRE(ids[i] >= 0 && ids[i] < ns, "shot id out of range");
  const float *rcp = rcp_of(vel_);
  int mb = max_batch();
  long long dn = (long long)nt * ngmax;
  for (int c0 = 0; c0 < n; c0 += mb) {
    int k = std::min(mb, n - c0);
    w_.slot_shot.upload(ids + c0, k, st_);
    const int *ss = w_.slot_shot.get();
    const int *rr = ss;
    if (rows) {
      w_.slot_row.upload(rows + c0, k, st_);
      rr = w_.slot_row.get();
    }
    PointSet src{d_src_pos_p_.get(), 1, ss};
    PointSet rec{d_rec_pos_p_.get(), ngmax, ss};
    w_.dcal.resize((size_t)k * dn);
    w_.res.resize((size_t)k * dn);
    w_.vsrc.resize((size_t)k * dn);
    w_.win.resize((size_t)k * ngmax * 2);
    w_.image.resize((size_t)k * fstride);
    w_.image.zero(st_);
    // FwiForwardModeling and calgradient's forward sweep model the same
    // field from the same source: one sweep records dcal and saves strips.
    std::vector<PtLine> sl, rl;
    const bool lines = shot_lines(ids + c0, k, true, sl, rl);
    run_forward<float>(w_, k, src, wlt, 1, 0, 0, rec, ngmax, w_.dcal.get(), true, rcp);
    launch_mute_windows(w_.win.get(), vel_, nxpad, nzpad, d_src_x_.get(), d_src_z_.get(),
                        d_rec_x_.get(), d_rec_z_.get(), ngmax, ngmax, ss, half_len, nt, k, st_);
    if (before_residual && c0 == 0) (*before_residual)();
    launch_muted_residual(w_.res.get(), dobs, dn, rr, w_.dcal.get(), w_.win.get(), w_.win.get(), nt,
                          ngmax, k, st_);
    launch_sumsq_f64(w_.obj.get(), w_.res.get(), dn, k, w_.partials.get(), kPartials, st_);
    launch_trans_vsrc(w_.vsrc.get(), w_.res.get(), nt, ngmax, k, st_);
    // FAST arithmetic images all shots of the batch into one image (one
    // read-modify-write a step for the whole batch)
    const bool summed = run_backward<float>(w_, k, src, wlt, 1, 0, 0, rec, ngmax, w_.vsrc.get(), rcp,
                                            lines ? &sl : nullptr, lines ? &rl : nullptr, arith == ARITH_FAST);
    launch_finalize_gradient(grad, w_.image.get() + kStreamCoff, fstride, summed ? 1 : k, nxpad, nzpad, bx0,
                             pitch, (accumulate || c0 > 0) ? 1 : 0, st_);
    if (obj) {
      SWFWI_CUDA(cudaMemcpyAsync(obj + c0, w_.obj.get(), sizeof(double) * k, cudaMemcpyDeviceToHost,
                                 st_));
    }
  }
  if (obj) check_device_error();
}

double Propagator::trial_objective_fwi(const float *wlt, const float *dobs, const int *ids, int n,
                                       const float *trial_vel) {
  SWFWI_REQUIRE(wlt && dobs && ids && trial_vel && n > 0, "bad trial arguments");
  const float *rcp = rcp_of(trial_vel);
  int mb = max_batch();
  long long dn = (long long)nt * ngmax;
  std::vector<double> h;
  double total = 0.0;
  for (int c0 = 0; c0 < n; c0 += mb) {
    int k = std::min(mb, n - c0);
    w_.slot_shot.upload(ids + c0, k, st_);
    const int *ss = w_.slot_shot.get();
    PointSet src{d_src_pos_p_.get(), 1, ss};
    PointSet rec{d_rec_pos_p_.get(), ngmax, ss};
    w_.dcal.resize((size_t)k * dn);
    w_.res.resize((size_t)k * dn);
    w_.win.resize((size_t)k * ngmax * 2);
    w_.win2.resize((size_t)k * ngmax * 2);
    run_forward<float>(w_, k, src, wlt, 1, 0, 0, rec, ngmax, w_.dcal.get(), false, rcp);
    // modelled data muted with the trial velocity, observed data with the
    // current one (updatesteplenop.cpp:77 and essfwiframework.cpp:205)
    launch_mute_windows(w_.win.get(), trial_vel, nxpad, nzpad, d_src_x_.get(), d_src_z_.get(),
                        d_rec_x_.get(), d_rec_z_.get(), ngmax, ngmax, ss, half_len, nt, k, st_);
    launch_mute_windows(w_.win2.get(), vel_, nxpad, nzpad, d_src_x_.get(), d_src_z_.get(),
                        d_rec_x_.get(), d_rec_z_.get(), ngmax, ngmax, ss, half_len, nt, k, st_);
    launch_muted_residual(w_.res.get(), dobs, dn, ss, w_.dcal.get(), w_.win2.get(), w_.win.get(), nt,
                          ngmax, k, st_);
    launch_sumsq_f64(w_.obj.get(), w_.res.get(), dn, k, w_.partials.get(), kPartials, st_);
    h.resize(k);
    SWFWI_CUDA(cudaMemcpyAsync(h.data(), w_.obj.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, st_));
    check_device_error();
    for (int i = 0; i < k; i++) total += h[i];
  }
  return total;
}

void Propagator::calgradient_ess(const float *encsrc, const float *vsrc, float *grad) {
  SWFWI_REQUIRE(encsrc && vsrc && grad, "null pointer");
  const float *rcp = rcp_of(vel_);
  PointSet src{d_src_pos_p_.get(), ns, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  w_.image.resize((size_t)fstride);
  w_.image.zero(st_);
  to_pitched(w_.image.get() + kStreamCoff, grad);
  std::vector<PtLine> sl, rl;
  const bool lines = ess_lines(1, sl, rl);
  run_forward<float>(w_, 1, src, encsrc, ns, 0, 1, rec, ng, nullptr, true, rcp);
  run_backward<float>(w_, 1, src, encsrc, ns, 0, 1, rec, ng, vsrc, rcp, lines ? &sl : nullptr,
                      lines ? &rl : nullptr);
  from_pitched(grad, w_.image.get() + kStreamCoff);
}

void Propagator::calgradient_fwi(const float *wlt, const float *vsrc, float *grad, int shot_id) {
  SWFWI_REQUIRE(wlt && vsrc && grad, "null pointer");
  SWFWI_REQUIRE(shot_id >= 0 && shot_id < ns, "shot id out of range");
  const float *rcp = rcp_of(vel_);
  PointSet src{d_src_pos_p_.get() + shot_id, 1, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  w_.image.resize((size_t)fstride);
  w_.image.zero(st_);
  to_pitched(w_.image.get() + kStreamCoff, grad);
  std::vector<PtLine> sl, rl;
  const bool lines = shot_lines(&shot_id, 1, false, sl, rl);
  run_forward<float>(w_, 1, src, wlt, 1, 0, 0, rec, ng, nullptr, true, rcp);
  run_backward<float>(w_, 1, src, wlt, 1, 0, 0, rec, ng, vsrc, rcp, lines ? &sl : nullptr,
                      lines ? &rl : nullptr);
  from_pitched(grad, w_.image.get() + kStreamCoff);
}

void Propagator::calgradient_fwi_f64(const float *vel, const double *wlt, const double *vsrc,
                                     double *grad, int shot_id) {
  SWFWI_REQUIRE(vel && wlt && vsrc && grad, "null pointer");
  SWFWI_REQUIRE(shot_id >= 0 && shot_id < ns, "shot id out of range");
  DevBuf<double> r64((size_t)nxpad * pitch + 2 * kStreamCoff);
  launch_to_f64_reciprocal(r64.get() + kStreamCoff, vel, nxpad, nzpad, pitch, st_);
  PointSet src{d_src_pos_p_.get() + shot_id, 1, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  wd_.image.resize((size_t)fstride);
  wd_.image.zero(st_);
  to_pitched(wd_.image.get() + kStreamCoff, grad);
  run_forward<double>(wd_, 1, src, wlt, 1, 0, 0, rec, ng, nullptr, true, r64.get() + kStreamCoff);
  run_backward<double>(wd_, 1, src, wlt, 1, 0, 0, rec, ng, vsrc, r64.get() + kStreamCoff);
  from_pitched(grad, wd_.image.get() + kStreamCoff);
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

void Propagator::calgradient_ess_f64(const float *vel, const double *encsrc, const double *vsrc,
                                     double *grad) {
  SWFWI_REQUIRE(vel && encsrc && vsrc && grad, "null pointer");
  DevBuf<double> r64((size_t)nxpad * pitch + 2 * kStreamCoff);
  launch_to_f64_reciprocal(r64.get() + kStreamCoff, vel, nxpad, nzpad, pitch, st_);
  PointSet src{d_src_pos_p_.get(), ns, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  wd_.image.resize((size_t)fstride);
  wd_.image.zero(st_);
  to_pitched(wd_.image.get() + kStreamCoff, grad);
  run_forward<double>(wd_, 1, src, encsrc, ns, 0, 1, rec, ng, nullptr, true, r64.get() + kStreamCoff);
  run_backward<double>(wd_, 1, src, encsrc, ns, 0, 1, rec, ng, vsrc, r64.get() + kStreamCoff);
  from_pitched(grad, wd_.image.get() + kStreamCoff);
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

void Propagator::fwi_forward_f64(const float *vel, const double *wlt, double *dcal, int shot_id) {
  SWFWI_REQUIRE(vel && wlt && dcal, "null pointer");
  SWFWI_REQUIRE(shot_id >= 0 && shot_id < ns, "shot id out of range");
  DevBuf<double> r64((size_t)nxpad * pitch + 2 * kStreamCoff);
  launch_to_f64_reciprocal(r64.get() + kStreamCoff, vel, nxpad, nzpad, pitch, st_);
  PointSet src{d_src_pos_p_.get() + shot_id, 1, nullptr};
  PointSet rec{d_geo_pos_p_.get(), ng, nullptr};
  run_forward<double>(wd_, 1, src, wlt, 1, 0, 0, rec, ng, dcal, false, r64.get() + kStreamCoff);
  SWFWI_CUDA(cudaStreamSynchronize(st_));
}

}  // namespace swfwi

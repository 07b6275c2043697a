// Test driver: the call sequence of the reference's FWI drivers
// (src/tool/main-fwi-damp.cpp:145-212, main-essfwi-damp.cpp:145-211) with
// their RSF readers and writers replaced by raw float files, compiled
// against the C++ classes in include/swfwi and run on the GPU.
//
//   fwi_driver <plain|ess> vinit.bin dobs.bin out_prefix nx nz nt ns ng
//              dx dt fm nb sxbeg jsx szbeg gxbeg jgx gzbeg vmin vmax nita
//              maxdv niter
//
// Writes out_prefix.objs (init obj, then each epoch's update obj),
// out_prefix.exvel (the bound padded transformed model after the last
// epoch) and out_prefix.vel (writeVel: interior model in m/s).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "damp4t10d.h"
#include "essfwiframework.h"
#include "fwiframework.h"
#include "ricker-wavelet.h"
#include "shot-position.h"
#include "updatevelop.h"

static std::vector<float> read_floats(const char *path, size_t n) {
  std::vector<float> v(n);
  FILE *f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), sizeof(float), n, f) != n) {
    std::fprintf(stderr, "cannot read %zu floats from %s\n", n, path);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

static void write_floats(const std::string &path, const std::vector<float> &v) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(v.data(), sizeof(float), v.size(), f) != v.size()) std::exit(3);
  std::fclose(f);
}

template <class Framework, class StepOp, class VelOp>
static int run(Damp4t10d &fmMethod, const std::vector<float> &wlt, const std::vector<float> &dobs, float vmin,
               float vmax, float dx, float dt, int nita, float maxdv, int niter, const std::string &out) {
  VelOp updatevelop(vmin, vmax, dx, dt);
  StepOp updateSteplenOp(fmMethod, updatevelop, nita, maxdv);
  Framework fwi(fmMethod, updateSteplenOp, updatevelop, wlt, dobs);
  std::vector<float> objs;
  for (int iter = 0; iter < niter; iter++) {
    fwi.epoch(iter);
    if (iter == 0) objs.push_back(fwi.getInitObj());
    objs.push_back(fwi.getUpdateObj());
  }
  write_floats(out + ".objs", objs);
  write_floats(out + ".exvel", fmMethod.getVelocity().dat);
  write_floats(out + ".vel", fwi.writeVel());
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 25) {
    std::fprintf(stderr, "usage: see the header of fwi_driver.cpp\n");
    return 1;
  }
  const std::string kind = argv[1];
  int a = 5;
  auto I = [&]() { return std::atoi(argv[a++]); };
  auto F = [&]() { return (float)std::atof(argv[a++]); };
  const int nx = I(), nz = I(), nt = I(), ns = I(), ng = I();
  const float dx = F(), dt = F(), fm = F();
  const int nb = I(), sxbeg = I(), jsx = I(), szbeg = I(), gxbeg = I(), jgx = I(), gzbeg = I();
  const float vmin = F(), vmax = F();
  const int nita = I();
  const float maxdv = F();
  const int niter = I();
  try {
    ShotPosition allSrcPos(szbeg, sxbeg, 0, jsx, ns, nz);
    ShotPosition allGeoPos(gzbeg, gxbeg, 0, jgx, ng, nz);
    Damp4t10d fmMethod(allSrcPos, allGeoPos, dt, dx, fm, nb, nt);
    Velocity v0(read_floats(argv[2], (size_t)nx * nz), nx, nz);
    Velocity exvel = fmMethod.expandDomain(v0);
    fmMethod.bindVelocity(exvel);
    std::vector<float> wlt(nt);
    rickerWavelet(&wlt[0], nt, fm, dt, 1.0f);
    std::vector<float> dobs = read_floats(argv[3], (size_t)ns * nt * ng);
    if (kind == "plain")
      return run<FwiFramework, FwiUpdateSteplenOp, FwiUpdateVelOp>(fmMethod, wlt, dobs, vmin, vmax, dx, dt, nita,
                                                                    maxdv, niter, argv[4]);
    return run<EssFwiFramework, UpdateSteplenOp, UpdateVelOp>(fmMethod, wlt, dobs, vmin, vmax, dx, dt, nita, maxdv,
                                                              niter, argv[4]);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 4;
  }
}

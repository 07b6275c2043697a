// The ensemble Kalman analysis of swfwi's EnFWI (src/enfwi/enkfanalyze.cpp)
// on the GPU, in FP64.
//
// calGainMatrix (enkfanalyze.cpp:185-341) forms, over rows = nt*ng data
// samples and N members, HA' = HA - rowmean(HA), the perturbed data
// D = dobs + pert, gamma = pert - rowmean(pert), band = HA' + gamma, the SVD
// band = U S V', and the N x N gain t4 = HA'^T U SSqInv U^T (D - HA) with
// SSqInv = diag(1/s_i^2) for the first clipPosition(S) singular values.
// With U = band V S^-1 that is
//   t4 = X2 V diag(s_i^-4, i < clip) V^T X3,
//   X1 = band^T band,  X2 = HA'^T band,  X3 = band^T (D - HA),
// and s_i^2, V the eigenpairs of X1.  The three N x N cross products are
// the only work over the data (O(rows N^2)); one fused pass forms them row
// by row (row means, perturbation, band and residual never reach HBM), a
// fixed-order reduction sums the per-CTA partials, and the N x N eigen
// problem and products run on the host (cyclic Jacobi in double).
//
// analyze (enkfanalyze.cpp:57-111) then moves each member by
// A' t4 (A' = members - their float mean), in physical velocity.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>
#include "common.hpp"

namespace swfwi {
namespace {

constexpr int kMaxMembers = 64;   // members per analysis (one 64 x 64 tile)
constexpr int kRowsPerChunk = 16;
constexpr int kThreads = 256;

// ---- counter-based normal draws (Philox4x32-10 of Salmon et al. 2011,
// "Parallel random numbers: as easy as 1, 2, 3"; Box-Muller transform)
__device__ __forceinline__ void philox_round(uint32_t (&c)[4], const uint32_t (&k)[2]) {
  const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;
  const uint32_t hi0 = __umulhi(m0, c[0]), lo0 = m0 * c[0];
  const uint32_t hi1 = __umulhi(m1, c[2]), lo1 = m1 * c[2];
  const uint32_t n0 = hi1 ^ c[1] ^ k[0], n1 = lo1, n2 = hi0 ^ c[3] ^ k[1], n3 = lo0;
  c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
}

__device__ __forceinline__ double normal_draw(unsigned long long seed, unsigned long long index) {
  uint32_t c[4] = {(uint32_t)index, (uint32_t)(index >> 32), 0u, 0u};
  uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
#pragma unroll
  for (int r = 0; r < 10; r++) {
    philox_round(c, k);
    k[0] += 0x9E3779B9u;
    k[1] += 0xBB67AE85u;
  }
  const double u1 = ((double)c[0] + 1.0) * 2.3283064365386963e-10;   // (0, 1]
  const double u2 = (double)c[1] * 2.3283064365386963e-10;           // [0, 1)
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// ---- max |HA'| as initPerturbation picks it: the first element (member-
// major order) whose float |x| is largest.  key = float bits of |x| above
// the inverted element index, so the largest key is that element.
__global__ void k_maxkey(unsigned long long *best, const float *hona, long long rows, int n) {
  unsigned long long mine = 0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
       r += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += (double)hona[i * rows + r];
    const double mean = s / n;
    for (int i = 0; i < n; i++) {
      const double x = (double)hona[i * rows + r] - mean;
      const uint32_t key = __float_as_uint(fabsf((float)x));
      const uint32_t inv = 0xFFFFFFFFu - (uint32_t)(i * rows + r);
      const unsigned long long v = ((unsigned long long)key << 32) | inv;
      mine = v > mine ? v : mine;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, mine, o);
    mine = other > mine ? other : mine;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(best, mine);
}

__global__ void k_value_at(double *out, const unsigned long long *best, const float *hona, long long rows,
                           int n) {
  const uint32_t idx = 0xFFFFFFFFu - (uint32_t)(*best & 0xFFFFFFFFull);
  const long long r = idx % rows;
  const int i0 = (int)(idx / rows);
  double s = 0.0;
  for (int i = 0; i < n; i++) s += (double)hona[i * rows + r];
  *out = fabs((double)hona[i0 * rows + r] - s / n);
}

// ---- the three cross products, one pass over the rows.  A CTA takes 16
// rows at a time: it stages the members' HA and perturbation of those rows
// in shared memory, forms the row means in member order (as initGamma
// sums), then HA', band and D - HA; each thread accumulates a 4 x 4 tile of
// X1, X2 and X3 over the rows.  partials[cta][3][64][64].
template <bool DRAW>
__global__ void __launch_bounds__(kThreads)
k_cross(double *partials, const float *hona, const float *dobs, const double *z, long long rows, int n,
        double sigma, unsigned long long seed) {
  __shared__ double sh[kRowsPerChunk][kMaxMembers];   // HA, then HA'
  __shared__ double sp[kRowsPerChunk][kMaxMembers];   // perturbation, then band
  __shared__ double st[kRowsPerChunk][kMaxMembers];   // D - HA
  __shared__ double mh[kRowsPerChunk], mp[kRowsPerChunk];
  const int t = threadIdx.x, ta = t >> 4, tb = t & 15, lr = t & 15;
  double a1[4][4] = {}, a2[4][4] = {}, a3[4][4] = {};
  for (long long r0 = (long long)blockIdx.x * kRowsPerChunk; r0 < rows;
       r0 += (long long)gridDim.x * kRowsPerChunk) {
    const long long r = r0 + lr;
    const bool rok = r < rows;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = (t >> 4) + 16 * q;
      double h = 0.0, p = 0.0;
      if (rok && i < n) {
        h = (double)hona[i * rows + r];
        p = sigma * (DRAW ? normal_draw(seed, (unsigned long long)(i * rows + r)) : z[i * rows + r]);
      }
      sh[lr][i] = h;
      sp[lr][i] = p;
    }
    __syncthreads();
    if (t < kRowsPerChunk) {
      double a = 0.0, b = 0.0;
      for (int i = 0; i < n; i++) {
        a += sh[t][i];
        b += sp[t][i];
      }
      mh[t] = a / n;
      mp[t] = b / n;
    }
    __syncthreads();
    const double d = rok ? (double)dobs[r] : 0.0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = (t >> 4) + 16 * q;
      double hap = 0.0, band = 0.0, res = 0.0;
      if (rok && i < n) {
        const double h = sh[lr][i], p = sp[lr][i];
        hap = h - mh[lr];
        band = hap + (p - mp[lr]);
        res = (d + p) - h;
      }
      sh[lr][i] = hap;
      sp[lr][i] = band;
      st[lr][i] = res;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kRowsPerChunk; rr++) {
      double ga[4], ha[4], gb[4], tb4[4];
#pragma unroll
      for (int x = 0; x < 4; x++) {
        ga[x] = sp[rr][4 * ta + x];
        ha[x] = sh[rr][4 * ta + x];
        gb[x] = sp[rr][4 * tb + x];
        tb4[x] = st[rr][4 * tb + x];
      }
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) {
          a1[x][y] = fma(ga[x], gb[y], a1[x][y]);
          a2[x][y] = fma(ha[x], gb[y], a2[x][y]);
          a3[x][y] = fma(ga[x], tb4[y], a3[x][y]);
        }
    }
    __syncthreads();
  }
  double *out = partials + (long long)blockIdx.x * 3 * kMaxMembers * kMaxMembers;
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) {
      const int e = (4 * ta + x) * kMaxMembers + 4 * tb + y;
      out[e] = a1[x][y];
      out[kMaxMembers * kMaxMembers + e] = a2[x][y];
      out[2 * kMaxMembers * kMaxMembers + e] = a3[x][y];
    }
}

// Sum of the per-CTA partials in CTA order (deterministic).
__global__ void k_sum_partials(double *x, const double *partials, int nparts) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = 3 * kMaxMembers * kMaxMembers;
  if (e >= m) return;
  double s = 0.0;
  for (int b = 0; b < nparts; b++) s += partials[(long long)b * m + e];
  x[e] = s;
}

// ---- analyze's update, one thread per model point: the members' float
// mean (createAMean, enkfanalyze.cpp:568-580), A' in double, A' t4, and
// v <- velTrans(velRecover(v) + (A' t4)_i) (enkfanalyze.cpp:72-108).
__global__ void __launch_bounds__(kThreads)
k_update(float *vels, long long model, int n, const double *t4, float dx, float dt) {
  __shared__ double g[kMaxMembers * kMaxMembers];   // t4 column-major: row j, col i at i*n + j
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) g[e] = t4[e];
  __syncthreads();
  const float dx2 = __fmul_rn(dx, dx), dt2 = __fmul_rn(dt, dt);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < model;
       p += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int j = 0; j < n; j++) s = __fadd_rn(s, vels[j * model + p]);
    const float mean = __fdiv_rn(s, (float)n);
    // every member's A' t4 from the values before any of them is written
    double t5s[kMaxMembers];
    for (int i = 0; i < n; i++) {
      double t5 = 0.0;
      for (int j = 0; j < n; j++) t5 = fma((double)vels[j * model + p] - (double)mean, g[i * n + j], t5);
      t5s[i] = t5;
    }
    for (int i = 0; i < n; i++) {
      const float vi = vels[i * model + p];
      const float phys = __fsqrt_rn(__fdiv_rn(dx2, __fmul_rn(dt2, vi)));
      const float upd = (float)((double)phys + t5s[i]);
      vels[i * model + p] = __fdiv_rn(dx2, __fmul_rn(__fmul_rn(dt2, upd), upd));
    }
  }
}

__global__ void k_mean(float *mean, const float *vels, long long model, int n) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < model;
       p += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int j = 0; j < n; j++) s = __fadd_rn(s, vels[j * model + p]);
    mean[p] = __fdiv_rn(s, (float)n);
  }
}

unsigned grid_of(long long n, int per) {
  long long g = (n + per - 1) / per;
  return (unsigned)std::max(1LL, std::min(g, 4096LL));
}

// Cyclic Jacobi eigen decomposition of the symmetric n x n matrix a
// (row-major; destroyed): w eigenvalues, column k of v (row-major) the
// k-th eigenvector.
void jacobi_eigen(int n, std::vector<double> &a, std::vector<double> &w, std::vector<double> &v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) v[(size_t)i * n + i] = 1.0;
  auto A = [&](int i, int j) -> double & { return a[(size_t)i * n + j]; };
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        tot += A(i, j) * A(i, j);
        if (i != j) off += A(i, j) * A(i, j);
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const double apq = A(p, q);
        if (apq == 0.0) continue;
        const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
        const double tt = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(tt * tt + 1.0), s = tt * c;
        for (int k = 0; k < n; k++) {   // columns p, q
          const double akp = A(k, p), akq = A(k, q);
          A(k, p) = c * akp - s * akq;
          A(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {   // rows p, q
          const double apk = A(p, k), aqk = A(q, k);
          A(p, k) = c * apk - s * aqk;
          A(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < n; k++) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = A(i, i);
}

// clipPosition (src/enfwi/Matrix.cpp:170-185).
int clip_position(const std::vector<double> &s) {
  const double rel = (double)0.001f;
  const int n = (int)s.size();
  double sum = 0.0;
  int pos;
  for (pos = 0; pos < n - 1; pos++) {
    sum += std::fabs(s[pos]);
    if (rel / (1 - rel) * sum > (n - pos + 1) * s[pos + 1]) break;
  }
  return pos + 1;
}

}  // namespace
}  // namespace swfwi

using namespace swfwi;

extern "C" int swfwi_enkf_gain_matrix(const float *hona, const float *dobs, const double *z, long long rows,
                                      int n, float sigfac, double *sigma, unsigned long long seed,
                                      double *t4, int *clip, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(hona && dobs && sigma && t4, "null pointer");
    SWFWI_REQUIRE(n >= 2 && n <= kMaxMembers, "members must be 2..64");
    SWFWI_REQUIRE(rows > 0 && rows * n < 0xFFFFFFFFLL, "rows x members must be below 2^32");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (!(*sigma > 0.0)) {
      // initPerturbation's first call: sigma = max|HA'| * sigmaFactor
      DevBuf<unsigned long long> best(1);
      DevBuf<double> val(1);
      SWFWI_CUDA(cudaMemsetAsync(best.get(), 0, sizeof(unsigned long long), st));
      k_maxkey<<<grid_of(rows, kThreads), kThreads, 0, st>>>(best.get(), hona, rows, n);
      k_value_at<<<1, 1, 0, st>>>(val.get(), best.get(), hona, rows, n);
      SWFWI_CUDA(cudaGetLastError());
      double mx = 0.0;
      SWFWI_CUDA(cudaMemcpyAsync(&mx, val.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
      SWFWI_CUDA(cudaStreamSynchronize(st));
      *sigma = mx * (double)sigfac;
    }
    int dev = 0, sms = 148;
    SWFWI_CUDA(cudaGetDevice(&dev));
    SWFWI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long long chunks = (rows + kRowsPerChunk - 1) / kRowsPerChunk;
    const int nparts = (int)std::min<long long>(chunks, 2LL * sms);
    const int m = 3 * kMaxMembers * kMaxMembers;
    DevBuf<double> partials((size_t)nparts * m), x(m);
    if (z)
      k_cross<false><<<nparts, kThreads, 0, st>>>(partials.get(), hona, dobs, z, rows, n, *sigma, seed);
    else
      k_cross<true><<<nparts, kThreads, 0, st>>>(partials.get(), hona, dobs, nullptr, rows, n, *sigma, seed);
    k_sum_partials<<<(m + 255) / 256, 256, 0, st>>>(x.get(), partials.get(), nparts);
    SWFWI_CUDA(cudaGetLastError());
    std::vector<double> hx(m);
    SWFWI_CUDA(cudaMemcpyAsync(hx.data(), x.get(), sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
    for (double e : hx)
      if (!std::isfinite(e)) throw Error(SWFWI_ERR_NONFINITE, "non-finite data in the analysis");

    // X1's eigenpairs in descending order: s_i^2 and V
    const int K = kMaxMembers;
    std::vector<double> a((size_t)n * n), w, v;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) a[(size_t)i * n + j] = hx[(size_t)i * K + j];
    jacobi_eigen(n, a, w, v);
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](int p, int q) { return w[p] > w[q]; });
    std::vector<double> s(n);
    for (int i = 0; i < n; i++) s[i] = std::sqrt(std::max(w[ord[i]], 0.0));
    const int c = clip_position(s);
    if (clip) *clip = c;
    // t4 = X2 V diag(s^-4) V^T X3 over the kept singular values
    std::vector<double> left((size_t)n * c, 0.0), right((size_t)c * n, 0.0);
    for (int k = 0; k < c; k++) {
      const int col = ord[k];
      const double wk = 1.0 / (s[k] * s[k] * s[k] * s[k]);
      for (int i = 0; i < n; i++) {
        double l = 0.0, r = 0.0;
        for (int j = 0; j < n; j++) {
          l += hx[(size_t)K * K + (size_t)i * K + j] * v[(size_t)j * n + col];       // (X2 V)[i][k]
          r += v[(size_t)j * n + col] * hx[2 * (size_t)K * K + (size_t)j * K + i];   // (V^T X3)[k][i]
        }
        left[(size_t)i * c + k] = l * wk;
        right[(size_t)k * n + i] = r;
      }
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        double e = 0.0;
        for (int k = 0; k < c; k++) e += left[(size_t)i * c + k] * right[(size_t)k * n + j];
        t4[(size_t)j * n + i] = e;   // column-major, as the reference's Matrix
      }
  });
}

extern "C" int swfwi_enkf_update(float *vels, long long model_size, int n, const double *t4, float dx,
                                 float dt, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(vels && t4 && model_size > 0, "bad update arguments");
    SWFWI_REQUIRE(n >= 2 && n <= kMaxMembers, "members must be 2..64");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    DevBuf<double> g((size_t)n * n);
    SWFWI_CUDA(cudaMemcpyAsync(g.get(), t4, sizeof(double) * n * n, cudaMemcpyHostToDevice, st));
    k_update<<<grid_of(model_size, kThreads), kThreads, 0, st>>>(vels, model_size, n, g.get(), dx, dt);
    SWFWI_CUDA(cudaGetLastError());
    SWFWI_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int swfwi_enkf_mean(float *mean, const float *vels, long long model_size, int n, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(mean && vels && model_size > 0 && n >= 1, "bad mean arguments");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_mean<<<grid_of(model_size, kThreads), kThreads, 0, st>>>(mean, vels, model_size, n);
    SWFWI_CUDA(cudaGetLastError());
  });
}

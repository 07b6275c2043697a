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
// fixed-order reduction sums the per-CTA partials, and one CTA solves the
// N x N eigen problem (parallel-ordered two-sided Jacobi in FP64 shared
// memory), sorts it, applies clipPosition and forms t4, which stays in
// device memory for the member update.
//
// analyze (enkfanalyze.cpp:57-111) then moves each member by
// A' t4 (A' = members - their float mean), in physical velocity.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>
#include "common.hpp"
#include "kernels.cuh"

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

// sigma = |HA'| of that element times the perturbation factor
// (initPerturbation, enkfanalyze.cpp:621-635)
__global__ void k_value_at(double *sigma, const unsigned long long *best, const float *hona, long long rows,
                           int n, float sigfac) {
  const uint32_t idx = 0xFFFFFFFFu - (uint32_t)(*best & 0xFFFFFFFFull);
  const long long r = idx % rows;
  const int i0 = (int)(idx / rows);
  double s = 0.0;
  for (int i = 0; i < n; i++) s += (double)hona[i * rows + r];
  *sigma = fabs((double)hona[i0 * rows + r] - s / n) * (double)sigfac;
}

// ---- the three cross products, one pass over the rows.  A CTA takes 16
// rows at a time: it stages the members' HA and perturbation of those rows
// in shared memory, forms the row means in member order (as initGamma
// sums), then HA', band and D - HA; each thread accumulates a 4 x 4 tile of
// X1, X2 and X3 over the rows.  partials[cta][3][64][64].
template <bool DRAW>
__global__ void __launch_bounds__(kThreads)
k_cross(double *partials, const float *hona, const float *dobs, const double *z, long long rows, int n,
        const double *sigma_dev, unsigned long long seed) {
  const double sigma = *sigma_dev;
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
__device__ __forceinline__ void update_members(float *vels, long long model, int n, const double *t4, float dx,
                                               float dt) {
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

__global__ void __launch_bounds__(kThreads)
k_update(float *vels, long long model, int n, const double *t4, float dx, float dt) {
  update_members(vels, model, n, t4, dx, dt);
}

// the same after a device-side gain: nothing moves if the gain was not finite
__global__ void __launch_bounds__(kThreads)
k_update_guarded(float *vels, long long model, int n, const double *t4, float dx, float dt, const int *status) {
  if (status[1]) return;
  update_members(vels, model, n, t4, dx, dt);
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

// ---- the gain from the cross products, one CTA.  x = [X1 | X2 | X3],
// each K x K row-major (K = kMaxMembers), first n x n used.
//
// Eigenpairs of the symmetric X1 by two-sided Jacobi in the round-robin
// (tournament) ordering: each round rotates n/2 disjoint index pairs at
// once (all column rotations, then all row rotations: A <- J^T A J with J
// the product of the round's plane rotations), n-1 rounds a sweep; a pair's
// angle comes from its own 2 x 2 block, which no other rotation of the
// round touches.  Sweeps stop when the off-diagonal square sum is at most
// 1e-30 of the total (or after 100).  Eigenvalues sorted descending (ties
// by index), s_k = sqrt(max(lambda_k, 0)), c = clipPosition(s)
// (src/enfwi/Matrix.cpp:170-185), then
//   t4 = (X2 V_c diag(s^-4)) (V_c^T X3),  written column-major (the
// reference's Matrix): t4[j*n + i] = row i, column j.
// status[0] = c, status[1] = 1 if any cross product is not finite.
constexpr int kGainThreads = 256;
constexpr int kLd = kMaxMembers + 1;   // padded row stride in shared memory

__host__ __device__ constexpr size_t gain_smem_bytes() {
  return sizeof(double) * (3 * kMaxMembers * kLd + 4 * kMaxMembers + 2 * kGainThreads) +
         sizeof(int) * (3 * kMaxMembers + 2 * (kMaxMembers / 2) + 4);
}

__device__ double block_sum_fixed(double v, double *red) {
  // fixed-order tree over the CTA's threads (deterministic)
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = kGainThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kGainThreads)
k_gain(double *t4, int *status, const double *x, int n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *A = reinterpret_cast<double *>(smem_raw);        // X1, then left = X2 V diag(s^-4)
  double *V = A + kMaxMembers * kLd;                        // eigenvectors (columns)
  double *R = V + kMaxMembers * kLd;                        // right = V^T X3
  double *w = R + kMaxMembers * kLd;                        // eigenvalues
  double *sv = w + kMaxMembers;                             // sorted singular values
  double *cs = sv + kMaxMembers;                            // rotation cosines [n/2]
  double *sn = cs + kMaxMembers;                            // rotation sines [n/2]
  double *red = sn + kMaxMembers;                           // [2 * kGainThreads]
  int *ord = reinterpret_cast<int *>(red + 2 * kGainThreads);
  int *perm = ord + kMaxMembers;                            // tournament positions
  int *pp = perm + kMaxMembers, *pq = pp + kMaxMembers / 2;
  int *flag = pq + kMaxMembers / 2;
  const int tid = threadIdx.x;
  const int K = kMaxMembers;
  const int m = (n + 1) & ~1;            // even number of tournament players (n odd: one idle)
  const int half = m / 2;

  if (tid == 0) *flag = 0;
  __syncthreads();
  for (int e = tid; e < n * n; e += kGainThreads) {
    const int i = e / n, j = e - i * n;
    const double a = x[i * K + j], b = x[K * K + i * K + j], c = x[2 * K * K + i * K + j];
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) *flag = 1;
    A[i * kLd + j] = a;
    V[i * kLd + j] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  if (*flag) {
    if (tid == 0) {
      status[0] = 0;
      status[1] = 1;
    }
    return;
  }

  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int e = tid; e < n * n; e += kGainThreads) {
      const int i = e / n, j = e - i * n;
      const double a = A[i * kLd + j];
      tot += a * a;
      if (i != j) off += a * a;
    }
    off = block_sum_fixed(off, red);
    tot = block_sum_fixed(tot, red + kGainThreads);
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int round = 0; round < m - 1; round++) {
      // pair k of this round: player m-1 meets player `round`, the others
      // (round + k, round - k) modulo m-1
      if (tid < half) {
        int p, q;
        if (tid == 0) {
          p = round;
          q = m - 1;
        } else {
          p = (round + tid) % (m - 1);
          q = (round - tid + (m - 1)) % (m - 1);
        }
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        double c = 1.0, sg = 0.0;
        if (q < n) {
          const double apq = A[p * kLd + q];
          if (apq != 0.0) {
            const double theta = (A[q * kLd + q] - A[p * kLd + p]) / (2.0 * apq);
            const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(tt * tt + 1.0);
            sg = tt * c;
          }
        }
        pp[tid] = p;
        pq[tid] = q < n ? q : p;   // an idle player's pair rotates nothing
        cs[tid] = c;
        sn[tid] = q < n ? sg : 0.0;
      }
      __syncthreads();
      // columns p, q of A and V
      for (int e = tid; e < half * n; e += kGainThreads) {
        const int k = e / half, pr = e - k * half;
        const int p = pp[pr], q = pq[pr];
        if (p == q) continue;
        const double c = cs[pr], sg = sn[pr];
        const double akp = A[k * kLd + p], akq = A[k * kLd + q];
        A[k * kLd + p] = c * akp - sg * akq;
        A[k * kLd + q] = sg * akp + c * akq;
        const double vkp = V[k * kLd + p], vkq = V[k * kLd + q];
        V[k * kLd + p] = c * vkp - sg * vkq;
        V[k * kLd + q] = sg * vkp + c * vkq;
      }
      __syncthreads();
      // rows p, q of A
      for (int e = tid; e < half * n; e += kGainThreads) {
        const int k = e / half, pr = e - k * half;
        const int p = pp[pr], q = pq[pr];
        if (p == q) continue;
        const double c = cs[pr], sg = sn[pr];
        const double apk = A[p * kLd + k], aqk = A[q * kLd + k];
        A[p * kLd + k] = c * apk - sg * aqk;
        A[q * kLd + k] = sg * apk + c * aqk;
      }
      __syncthreads();
    }
  }
  // descending order of the eigenvalues, ties by index
  if (tid < n) w[tid] = A[tid * kLd + tid];
  __syncthreads();
  if (tid < n) {
    int rank = 0;
    const double wi = w[tid];
    for (int j = 0; j < n; j++) rank += (w[j] > wi || (w[j] == wi && j < tid)) ? 1 : 0;
    ord[rank] = tid;
  }
  __syncthreads();
  if (tid < n) sv[tid] = sqrt(fmax(w[ord[tid]], 0.0));
  __syncthreads();
  if (tid == 0) {
    // clipPosition (Matrix.cpp:170-185); relativeError is a float literal
    const double rel = (double)0.001f;
    double sum = 0.0;
    int pos;
    for (pos = 0; pos < n - 1; pos++) {
      sum += fabs(sv[pos]);
      if (rel / (1 - rel) * sum > (n - pos + 1) * sv[pos + 1]) break;
    }
    flag[0] = pos + 1;
  }
  __syncthreads();
  const int c = flag[0];
  // left[i][k] = (X2 V)[i][ord[k]] s_k^-4 (into A); right[k][i] = (V^T X3)[ord[k]][i]
  for (int e = tid; e < n * c; e += kGainThreads) {
    const int i = e / c, k = e - i * c;
    const int col = ord[k];
    double l = 0.0, r = 0.0;
    for (int j = 0; j < n; j++) {
      l += x[K * K + i * K + j] * V[j * kLd + col];
      r += V[j * kLd + col] * x[2 * K * K + j * K + i];
    }
    const double s2 = sv[k] * sv[k];
    A[i * kLd + k] = l * (1.0 / (s2 * s2));
    R[k * kLd + i] = r;
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += kGainThreads) {
    const int j = e / n, i = e - j * n;
    double acc = 0.0;
    for (int k = 0; k < c; k++) acc += A[i * kLd + k] * R[k * kLd + j];
    t4[j * n + i] = acc;
  }
  if (tid == 0) {
    status[0] = c;
    status[1] = 0;
  }
}

// Device memory of one analysis, held by the caller until its results are
// back (freeing it earlier would synchronise the device mid-analysis).
struct GainScratch {
  DevBuf<unsigned long long> best;
  DevBuf<double> sigma, partials, x, t4;
  DevBuf<int> status;   // [0] clip, [1] non-finite cross products
};

// The analysis's device part: sigma (first call), cross products, gain into
// sc.t4 [n*n] (column-major), sc.status, sc.sigma.
void gain_on_device(const float *hona, const float *dobs, const double *z, long long rows, int n, float sigfac,
                    double sigma_in, unsigned long long seed, GainScratch &sc, cudaStream_t st) {
  sc.sigma.resize(1);
  sc.t4.resize((size_t)n * n);
  sc.status.resize(2);
  if (!(sigma_in > 0.0)) {
    // initPerturbation's first call: sigma = max|HA'| * sigmaFactor
    sc.best.resize(1);
    SWFWI_CUDA(cudaMemsetAsync(sc.best.get(), 0, sizeof(unsigned long long), st));
    k_maxkey<<<grid_of(rows, kThreads), kThreads, 0, st>>>(sc.best.get(), hona, rows, n);
    note_launch();
    k_value_at<<<1, 1, 0, st>>>(sc.sigma.get(), sc.best.get(), hona, rows, n, sigfac);
    note_launch();
  } else {
    SWFWI_CUDA(cudaMemcpyAsync(sc.sigma.get(), &sigma_in, sizeof(double), cudaMemcpyHostToDevice, st));
  }
  int dev = 0, sms = 148;
  SWFWI_CUDA(cudaGetDevice(&dev));
  SWFWI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long chunks = (rows + kRowsPerChunk - 1) / kRowsPerChunk;
  const int nparts = (int)std::min<long long>(chunks, 2LL * sms);
  const int m = 3 * kMaxMembers * kMaxMembers;
  sc.partials.resize((size_t)nparts * m);
  sc.x.resize(m);
  if (z)
    k_cross<false><<<nparts, kThreads, 0, st>>>(sc.partials.get(), hona, dobs, z, rows, n, sc.sigma.get(), seed);
  else
    k_cross<true><<<nparts, kThreads, 0, st>>>(sc.partials.get(), hona, dobs, nullptr, rows, n, sc.sigma.get(),
                                               seed);
  note_launch();
  k_sum_partials<<<(m + 255) / 256, 256, 0, st>>>(sc.x.get(), sc.partials.get(), nparts);
  note_launch();
  // once (thread-safe static init)
  static const cudaError_t attr =
      cudaFuncSetAttribute(k_gain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gain_smem_bytes());
  SWFWI_CUDA(attr);
  k_gain<<<1, kGainThreads, gain_smem_bytes(), st>>>(sc.t4.get(), sc.status.get(), sc.x.get(), n);
  note_launch();
  SWFWI_CUDA(cudaGetLastError());
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
    GainScratch sc;
    gain_on_device(hona, dobs, z, rows, n, sigfac, *sigma, seed, sc, st);
    int hs[2] = {0, 0};
    SWFWI_CUDA(cudaMemcpyAsync(hs, sc.status.get(), sizeof(hs), cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaMemcpyAsync(sigma, sc.sigma.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaMemcpyAsync(t4, sc.t4.get(), sizeof(double) * n * n, cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
    if (hs[1]) throw Error(SWFWI_ERR_NONFINITE, "non-finite data in the analysis");
    if (clip) *clip = hs[0];
  });
}

extern "C" int swfwi_enkf_analyze(const float *hona, const float *dobs, const double *z, long long rows, int n,
                                  float sigfac, double *sigma, unsigned long long seed, float *vels,
                                  long long model_size, float dx, float dt, double *t4_out, int *clip,
                                  void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(hona && dobs && sigma && vels && model_size > 0, "null pointer or empty model");
    SWFWI_REQUIRE(n >= 2 && n <= kMaxMembers, "members must be 2..64");
    SWFWI_REQUIRE(rows > 0 && rows * n < 0xFFFFFFFFLL, "rows x members must be below 2^32");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    GainScratch sc;
    gain_on_device(hona, dobs, z, rows, n, sigfac, *sigma, seed, sc, st);
    // a non-finite gain leaves the members unchanged: the update skips when
    // status[1] is set
    k_update_guarded<<<grid_of(model_size, kThreads), kThreads, 0, st>>>(vels, model_size, n, sc.t4.get(), dx, dt,
                                                                         sc.status.get());
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
    int hs[2] = {0, 0};
    SWFWI_CUDA(cudaMemcpyAsync(hs, sc.status.get(), sizeof(hs), cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaMemcpyAsync(sigma, sc.sigma.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    if (t4_out)
      SWFWI_CUDA(cudaMemcpyAsync(t4_out, sc.t4.get(), sizeof(double) * n * n, cudaMemcpyDeviceToHost, st));
    SWFWI_CUDA(cudaStreamSynchronize(st));
    if (hs[1]) throw Error(SWFWI_ERR_NONFINITE, "non-finite data in the analysis");
    if (clip) *clip = hs[0];
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
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
    SWFWI_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int swfwi_enkf_mean(float *mean, const float *vels, long long model_size, int n, void *stream) {
  return guarded([&] {
    SWFWI_REQUIRE(mean && vels && model_size > 0 && n >= 1, "bad mean arguments");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_mean<<<grid_of(model_size, kThreads), kThreads, 0, st>>>(mean, vels, model_size, n);
    note_launch();
    SWFWI_CUDA(cudaGetLastError());
  });
}

// tseg_fit.cu — the per-sample half of a time-segmentation fit (`fit`, tseg.rs:185-227) on the
// device, in FP64.  For one fit with segment count L over a rate grid of g rates z_k = (-d_k, w_k):
//   y_j[k] = e^{-d_k tau_j} cos(w_k tau_j),  y_j[g + k] = e^{-d_k tau_j} sin(w_k tau_j)
//   c_r = (left_r . y_j) / sig_r,  x_j = sum_r c_r right_r           (the factored solve)
//   b_sum = max_j sum_l |x_j[l] + i x_j[L + l]|
//   err   = max_{j,k} |y_j[k] + i y_j[g + k] - sum_i cols_i[k, g + k] x_j[i]|
// The host keeps the factorisation (one-sided Jacobi on the 2L columns) and the search over L
// and m; this file does the part whose cost grows with the samples (thousands of sample times x
// hundreds of rates x 2L columns, about 90 % of a host plan).
//
// Each block takes TJ consecutive sample times.  Every dot product, the solve and the residual
// run in the host fit's summation order (one thread per sum, sequential over its terms) and
// this file is compiled without multiply-add contraction, so a device fit differs from the host
// one only where CUDA's exp / sin / cos / hypot round differently from the host's.  The
// coefficients b are determined only to the conditioning of the truncated least-squares problem
// (a one-ulp change of y moves b by ~1e-5 in directions the rate grid does not see); the plan's
// L and m, and b_sum and the bound to ~1e-6, are what the two fits share.  The maxima reduce
// through atomicMax on the bit patterns of non-negative doubles: order-free, so every run gives
// the same figures.
#include <algorithm>
#include <cstring>

#include "mrsim_internal.h"
#include "spiral_host.h"

namespace mrsim {
namespace {

constexpr int kFitThreads = 256;
constexpr size_t kFitSmemBudget = 200 * 1024;

struct FitArgs {
  const double* tau;     // [n_tau] sample times (ms)
  const double2* rate;   // [g] (-d, w): decay (1/ms, negated) and angular frequency (rad/ms)
  const double* left;    // [R][2g] left singular vectors kept by the truncation
  const double* right;   // [R][2L] right singular vectors
  const double* sig;     // [R] singular values
  const double* cols;    // [2L][2g] the fit's columns e^{z_k tau_l} (re rows, then the -im / re pairs)
  double* b;             // [n_tau][L][2]
  unsigned long long* maxes;  // [0] b_sum, [1] err, as the bits of non-negative doubles
  int n_tau, g, R, L, TJ;
};

__global__ void __launch_bounds__(kFitThreads) tseg_fit_kernel(FitArgs a) {
  extern __shared__ double smem[];
  const int g2 = 2 * a.g, l2 = 2 * a.L, TJ = a.TJ;
  double* y = smem;                        // [TJ][2g]
  double* c = y + (size_t)TJ * g2;         // [TJ][R]
  double* x = c + (size_t)TJ * a.R;        // [TJ][2L]
  double* red = x + (size_t)TJ * l2;       // [TJ][32] warp maxima
  const int j0 = blockIdx.x * TJ;
  const int nt = min(TJ, a.n_tau - j0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  // the right-hand sides of the block's sample times
  for (int e = tid; e < nt * a.g; e += kFitThreads) {
    const int t = e / a.g, k = e - t * a.g;
    const double tj = a.tau[j0 + t];
    const double2 r = a.rate[k];
    const double mag = exp(r.x * tj);
    double s, co;
    sincos(r.y * tj, &s, &co);
    y[(size_t)t * g2 + k] = co * mag;
    y[(size_t)t * g2 + a.g + k] = s * mag;
  }
  __syncthreads();
  // c[t][r] = (left_r . y_t) / sig_r, one thread per (t, r), summed over k in order
  for (int e = tid; e < nt * a.R; e += kFitThreads) {
    const int r = e / nt, t = e - r * nt;
    const double* lr = a.left + (size_t)r * g2;
    const double* yt = y + (size_t)t * g2;
    double acc = 0.0;
    for (int k = 0; k < g2; ++k) acc += __ldg(lr + k) * yt[k];
    c[t * a.R + r] = acc / a.sig[r];
  }
  __syncthreads();
  // x[t][i] = sum_r c[t][r] right_r[i], in r order
  for (int e = tid; e < nt * l2; e += kFitThreads) {
    const int t = e / l2, i = e - t * l2;
    double acc = 0.0;
    for (int r = 0; r < a.R; ++r) acc += c[t * a.R + r] * __ldg(a.right + (size_t)r * l2 + i);
    x[t * l2 + i] = acc;
  }
  __syncthreads();
  // b and b_sum
  for (int e = tid; e < nt * a.L; e += kFitThreads) {
    const int t = e / a.L, i = e - t * a.L;
    double* bj = a.b + ((size_t)(j0 + t) * a.L + i) * 2;
    bj[0] = x[t * l2 + i];
    bj[1] = x[t * l2 + a.L + i];
  }
  if (tid < nt) {
    double s = 0.0;
    for (int i = 0; i < a.L; ++i) s += hypot(x[tid * l2 + i], x[tid * l2 + a.L + i]);
    atomicMax(a.maxes, (unsigned long long)__double_as_longlong(s));
  }
  // residual over the rate grid: one thread per rate, every sample time of the block
  double emax[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) emax[t] = 0.0;
  for (int k = tid; k < a.g; k += kFitThreads) {
    double re[8], im[8];
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (t < nt) {
        re[t] = y[(size_t)t * g2 + k];
        im[t] = y[(size_t)t * g2 + a.g + k];
      }
    for (int i = 0; i < l2; ++i) {
      const double cr = __ldg(a.cols + (size_t)i * g2 + k), ci = __ldg(a.cols + (size_t)i * g2 + a.g + k);
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < nt) {
          const double xi = x[t * l2 + i];
          re[t] -= cr * xi;
          im[t] -= ci * xi;
        }
    }
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (t < nt) emax[t] = fmax(emax[t], hypot(re[t], im[t]));
  }
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    double v = emax[t];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0 && t < nt) red[t * 32 + warp] = v;
  }
  __syncthreads();
  if (tid < nt) {
    double v = 0.0;
    for (int w = 0; w < kFitThreads / 32; ++w) v = fmax(v, red[tid * 32 + w]);
    atomicMax(a.maxes + 1, (unsigned long long)__double_as_longlong(v));
  }
}

template <class T>
void grow(T*& p, size_t& cap, size_t n) {
  if (n <= cap) return;
  if (p) MRSIM_CUDA(cudaFree(p));
  p = nullptr;
  cap = 0;
  MRSIM_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  cap = n;
}

}  // namespace

struct TsegDevice::Bufs {
  double* tau = nullptr;
  double2* rate = nullptr;
  double *left = nullptr, *right = nullptr, *sig = nullptr, *cols = nullptr, *b = nullptr;
  unsigned long long* maxes = nullptr;
  size_t c_tau = 0, c_rate = 0, c_left = 0, c_right = 0, c_sig = 0, c_cols = 0, c_b = 0, c_max = 0;
  std::vector<double> stage;  // host staging of the flattened factors
};

TsegDevice::TsegDevice(cudaStream_t st) : st_(st), d_(new Bufs) {}

TsegDevice::~TsegDevice() {
  for (void* p : {(void*)d_->tau, (void*)d_->rate, (void*)d_->left, (void*)d_->right, (void*)d_->sig,
                  (void*)d_->cols, (void*)d_->b, (void*)d_->maxes})
    if (p) cudaFree(p);
  delete d_;
}

void TsegDevice::set_times(const std::vector<double>& tau) {
  n_tau_ = (int)tau.size();
  grow(d_->tau, d_->c_tau, tau.size());
  if (!tau.empty())
    MRSIM_CUDA(cudaMemcpyAsync(d_->tau, tau.data(), tau.size() * sizeof(double), cudaMemcpyHostToDevice, st_));
}

void TsegDevice::fit(const std::vector<std::pair<double, double>>& rates, const std::vector<std::vector<double>>& cols,
                     const std::vector<std::vector<double>>& left, const std::vector<std::vector<double>>& right,
                     const std::vector<double>& sig, int l, double* b_sum, double* err) {
  const int g = (int)rates.size(), R = (int)sig.size(), l2 = 2 * l;
  const size_t g2 = 2 * (size_t)g;
  l_ = l;
  *b_sum = 0.0;
  *err = 0.0;
  if (n_tau_ == 0) return;
  // flatten: rates, left [R][2g], right [R][2L], sig [R], cols [2L][2g] into one staging vector
  std::vector<double>& s = d_->stage;
  s.assign(2 * (size_t)g + (size_t)R * g2 + (size_t)R * l2 + R + (size_t)l2 * g2, 0.0);
  double* p = s.data();
  for (int k = 0; k < g; ++k) {
    p[2 * k] = rates[k].first;
    p[2 * k + 1] = rates[k].second;
  }
  p += 2 * (size_t)g;
  double* pl = p;
  for (int r = 0; r < R; ++r) std::memcpy(p + (size_t)r * g2, left[r].data(), g2 * sizeof(double));
  p += (size_t)R * g2;
  double* pr = p;
  for (int r = 0; r < R; ++r) std::memcpy(p + (size_t)r * l2, right[r].data(), (size_t)l2 * sizeof(double));
  p += (size_t)R * l2;
  double* ps = p;
  std::memcpy(p, sig.data(), (size_t)R * sizeof(double));
  p += R;
  double* pc = p;
  for (int i = 0; i < l2; ++i) std::memcpy(p + (size_t)i * g2, cols[i].data(), g2 * sizeof(double));
  grow(d_->rate, d_->c_rate, (size_t)g);
  grow(d_->left, d_->c_left, (size_t)R * g2);
  grow(d_->right, d_->c_right, (size_t)R * l2);
  grow(d_->sig, d_->c_sig, (size_t)R);
  grow(d_->cols, d_->c_cols, (size_t)l2 * g2);
  grow(d_->b, d_->c_b, (size_t)n_tau_ * l2);
  grow(d_->maxes, d_->c_max, 2);
  MRSIM_CUDA(cudaMemcpyAsync(d_->rate, s.data(), (size_t)g * sizeof(double2), cudaMemcpyHostToDevice, st_));
  MRSIM_CUDA(cudaMemcpyAsync(d_->left, pl, (size_t)R * g2 * sizeof(double), cudaMemcpyHostToDevice, st_));
  MRSIM_CUDA(cudaMemcpyAsync(d_->right, pr, (size_t)R * l2 * sizeof(double), cudaMemcpyHostToDevice, st_));
  MRSIM_CUDA(cudaMemcpyAsync(d_->sig, ps, (size_t)R * sizeof(double), cudaMemcpyHostToDevice, st_));
  MRSIM_CUDA(cudaMemcpyAsync(d_->cols, pc, (size_t)l2 * g2 * sizeof(double), cudaMemcpyHostToDevice, st_));
  MRSIM_CUDA(cudaMemsetAsync(d_->maxes, 0, 2 * sizeof(unsigned long long), st_));
  // sample times per block: as many (up to 8) as the shared memory holds
  int TJ = 8;
  auto smem_of = [&](int tj) { return ((size_t)tj * (g2 + R + l2 + 32)) * sizeof(double); };
  while (TJ > 1 && smem_of(TJ) > kFitSmemBudget) TJ /= 2;
  const size_t smem = smem_of(TJ);
  if (smem > 227 * 1024) fail("the time segmentation's rate grid is too large for the device fit");
  MRSIM_CUDA(cudaFuncSetAttribute(tseg_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  FitArgs a;
  a.tau = d_->tau;
  a.rate = d_->rate;
  a.left = d_->left;
  a.right = d_->right;
  a.sig = d_->sig;
  a.cols = d_->cols;
  a.b = d_->b;
  a.maxes = d_->maxes;
  a.n_tau = n_tau_;
  a.g = g;
  a.R = R;
  a.L = l;
  a.TJ = TJ;
  tseg_fit_kernel<<<(n_tau_ + TJ - 1) / TJ, kFitThreads, smem, st_>>>(a);
  MRSIM_CUDA(cudaGetLastError());
  unsigned long long m[2];
  MRSIM_CUDA(cudaMemcpyAsync(m, d_->maxes, sizeof m, cudaMemcpyDeviceToHost, st_));
  MRSIM_CUDA(cudaStreamSynchronize(st_));
  std::memcpy(b_sum, &m[0], sizeof(double));
  std::memcpy(err, &m[1], sizeof(double));
}

void TsegDevice::fetch_b(std::vector<double>& b) const {
  b.resize((size_t)n_tau_ * 2 * l_);
  if (b.empty()) return;
  MRSIM_CUDA(cudaMemcpyAsync(b.data(), d_->b, b.size() * sizeof(double), cudaMemcpyDeviceToHost, st_));
  MRSIM_CUDA(cudaStreamSynchronize(st_));
}

}  // namespace mrsim

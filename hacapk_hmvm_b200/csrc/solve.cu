// Krylov solvers on a resident plan: the callers of the HMVM.
//
// BiCGSTAB restates HACApK_bicgstab_lfmtx (src_lhdump/m_HACApK_solve.f90:
// 977-1028), van der Vorst's BiCGSTAB with the shadow residual r0 = b - A u0:
// per step two H-matrix products (hmvm_b200_apply on the device-resident
// matrix) and five inner products.  GCR(m) restates HACApK_gcrm_lfmtx
// (m_HACApK_solve.f90:1277-1342): one product per step, search directions
// A-orthogonalised against the last m (restarted cyclically).  All vectors
// stay on the device; the inner products are summed in a fixed order
// (per-block partial sums, then one block), so a solve is repeatable bit for
// bit; their values come back to the host for the scalars and the stopping
// test ||r|| / ||b|| < eps.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "hmvm_b200.h"

namespace hmvm {
int set_error(int status, const std::string& msg);
}
using hmvm::set_error;

namespace {

constexpr int kDotBlocks = 256;
constexpr int kDotThreads = 256;

// part[b * 2 + j] = sum over the block's strided elements of x_j . y_j
template <typename T>
__global__ void dot2_partial(const T* __restrict__ x0, const T* __restrict__ y0, const T* __restrict__ x1,
                             const T* __restrict__ y1, int n, double* __restrict__ part) {
  __shared__ double s0[kDotThreads], s1[kDotThreads];
  double a0 = 0.0, a1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    a0 += (double)x0[i] * (double)y0[i];
    if (x1) a1 += (double)x1[i] * (double)y1[i];
  }
  s0[threadIdx.x] = a0;
  s1[threadIdx.x] = a1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}
__global__ void dot2_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  __shared__ double s0[kDotBlocks], s1[kDotBlocks];
  const int t = threadIdx.x;
  s0[t] = t < nb ? part[2 * t] : 0.0;
  s1[t] = t < nb ? part[2 * t + 1] : 0.0;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w) {
      s0[t] += s0[t + w];
      s1[t] += s1[t + w];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[0] = s0[0];
    out[1] = s1[0];
  }
}

// part[(j * kDotBlocks + b)] = block b's partial sum of x_j . y, x_j = x + j * ldx
template <typename T>
__global__ void dotm_partial(const T* __restrict__ x, size_t ldx, const T* __restrict__ y, int n,
                             double* __restrict__ part) {
  __shared__ double s[kDotThreads];
  const T* xj = x + blockIdx.y * ldx;
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    a += (double)xj[i] * (double)y[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = s[0];
}
// out[j] = sum of part[j * nb .. j * nb + nb), one block per j
__global__ void dotm_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  __shared__ double s[kDotBlocks];
  const int t = threadIdx.x;
  s[t] = t < nb ? part[blockIdx.x * nb + t] : 0.0;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w) s[t] += s[t + w];
    __syncthreads();
  }
  if (t == 0) out[blockIdx.x] = s[0];
}

constexpr int kMaxRestart = 64;
struct Betas {
  double b[kMaxRestart];
};
// GCR direction update, per element in the reference's order
// (m_HACApK_solve.f90:1331-1337): for il = 0..k-1,
//   p_new += beta_il * p_il,  ap_new += beta_il * ap_il,
// where slot `self` is p_new / ap_new itself (the restart step, at which the
// new direction reuses the oldest slot) and reads its current value.
template <typename T>
__global__ void gcr_update(T* __restrict__ p, T* __restrict__ ap, size_t ld, int k, int self, Betas be, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T* pn = p + (size_t)self * ld;
    T* an = ap + (size_t)self * ld;
    T vp = pn[i], va = an[i];
    for (int il = 0; il < k; il++) {
      const T wp = il == self ? vp : p[il * ld + i];
      const T wa = il == self ? va : ap[il * ld + i];
      vp = (T)((double)vp + be.b[il] * (double)wp);
      va = (T)((double)va + be.b[il] * (double)wa);
    }
    pn[i] = vp;
    an[i] = va;
  }
}

// z = x + a * y + b * w (w may be NULL)
template <typename T>
__global__ void axpbyz(T* __restrict__ z, const T* __restrict__ x, double a, const T* __restrict__ y, double b,
                       const T* __restrict__ w, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = (double)x[i] + a * (double)y[i];
    if (w) v += b * (double)w[i];
    z[i] = (T)v;
  }
}

template <typename T>
struct Solver {
  hmvm_plan* plan;
  int n;
  cudaStream_t st;
  double* part;  // [2 * kDotBlocks + 2]
  double host[2];

  int dot2(const T* x0, const T* y0, const T* x1, const T* y1, double* d0, double* d1) {
    dot2_partial<T><<<kDotBlocks, kDotThreads, 0, st>>>(x0, y0, x1, y1, n, part);
    dot2_final<<<1, kDotBlocks, 0, st>>>(part, kDotBlocks, part + 2 * kDotBlocks);
    if (cudaMemcpyAsync(host, part + 2 * kDotBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return set_error(HMVM_ECUDA, "bicgstab: inner products");
    *d0 = host[0];
    if (d1) *d1 = host[1];
    return HMVM_OK;
  }
  void lin(T* z, const T* x, double a, const T* y, double b = 0.0, const T* w = nullptr) {
    axpbyz<T><<<(n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184, 256, 0, st>>>(z, x, a, y, b, w, n);
  }
};

template <typename T>
int bicgstab_t(hmvm_plan* plan, int n, const T* b, T* u, int max_steps, double eps, int32_t* steps_out,
               double* relres_out, cudaStream_t st) {
  T* buf = nullptr;
  double* part = nullptr;
  // r, shadow, p, t, kp (= p), akp, akt, and a copy slot
  if (cudaMalloc(&buf, sizeof(T) * (size_t)n * 7) != cudaSuccess ||
      cudaMalloc(&part, sizeof(double) * (2 * kDotBlocks + 2)) != cudaSuccess) {
    if (buf) cudaFree(buf);
    cudaGetLastError();
    return set_error(HMVM_ENOMEM, "bicgstab: device vectors");
  }
  T *r = buf, *sh = buf + n, *p = buf + 2 * (size_t)n, *t = buf + 3 * (size_t)n, *akp = buf + 4 * (size_t)n,
    *akt = buf + 5 * (size_t)n, *kt = buf + 6 * (size_t)n;
  Solver<T> s{plan, n, st, part, {0, 0}};
  int rc = HMVM_OK;
  double bb = 0, rr = 0, relres = 0;
  int steps = 0;
  cudaMemsetAsync(p, 0, sizeof(T) * n, st);
  cudaMemsetAsync(akp, 0, sizeof(T) * n, st);
  // r = b - A u; shadow = r
  rc = hmvm_b200_apply(plan, u, akt, st);
  if (!rc) {
    s.lin(r, b, -1.0, akt);
    cudaMemcpyAsync(sh, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
    rc = s.dot2(b, b, r, r, &bb, &rr);
  }
  const double bnorm = std::sqrt(bb);
  relres = bnorm > 0 ? std::sqrt(rr) / bnorm : 0.0;
  double alpha = 0, beta = 0, zeta = 0, nom_old = 1;
  while (!rc && relres >= eps && steps < max_steps) {
    // p = r + beta (p - zeta akp)
    s.lin(p, r, beta, p, -beta * zeta, akp);
    rc = hmvm_b200_apply(plan, p, akp, st);
    if (rc) break;
    double nom, den;
    rc = s.dot2(sh, r, sh, akp, &nom, &den);
    if (rc) break;
    if (den == 0.0) {
      rc = set_error(HMVM_EINVAL, "bicgstab: breakdown (shadow residual orthogonal to A p)");
      break;
    }
    alpha = nom / den;
    nom_old = nom;
    s.lin(t, r, -alpha, akp);  // t = r - alpha akp
    cudaMemcpyAsync(kt, t, sizeof(T) * n, cudaMemcpyDeviceToDevice, st);
    rc = hmvm_b200_apply(plan, kt, akt, st);
    if (rc) break;
    double znom, zden;
    rc = s.dot2(akt, t, akt, akt, &znom, &zden);
    if (rc) break;
    zeta = zden != 0.0 ? znom / zden : 0.0;
    s.lin(u, u, alpha, p, zeta, kt);    // u += alpha p + zeta t
    s.lin(r, t, -zeta, akt);            // r = t - zeta akt
    double shr;
    rc = s.dot2(sh, r, r, r, &shr, &rr);
    if (rc) break;
    if (zeta == 0.0 || nom_old == 0.0) {
      steps++;
      relres = std::sqrt(rr) / bnorm;
      rc = set_error(HMVM_EINVAL, "bicgstab: breakdown (zeta or rho vanished)");
      break;
    }
    beta = alpha / zeta * shr / nom_old;
    relres = std::sqrt(rr) / bnorm;
    steps++;
  }
  cudaStreamSynchronize(st);
  cudaFree(buf);
  cudaFree(part);
  if (steps_out) *steps_out = steps;
  if (relres_out) *relres_out = relres;
  if (!rc) rc = hmvm_b200_plan_status(plan);
  return rc;
}

template <typename T>
int gcrm_t(hmvm_plan* plan, int n, const T* b, T* u, int max_steps, int m, double eps, int32_t* steps_out,
           double* relres_out, cudaStream_t st) {
  T* buf = nullptr;
  double* part = nullptr;
  // r, ar, then the m directions p and their products ap
  const size_t ld = (size_t)n;
  if (cudaMalloc(&buf, sizeof(T) * ld * (2 + 2 * (size_t)m)) != cudaSuccess ||
      cudaMalloc(&part, sizeof(double) * ((size_t)kDotBlocks * (m + 2) + m + 2)) != cudaSuccess) {
    if (buf) cudaFree(buf);
    cudaGetLastError();
    return set_error(HMVM_ENOMEM, "gcrm: device vectors");
  }
  T *r = buf, *ar = buf + ld, *p = buf + 2 * ld, *ap = buf + (2 + (size_t)m) * ld;
  double* dots = part + (size_t)kDotBlocks * (m + 2);
  Solver<T> s{plan, n, st, part, {0, 0}};
  std::vector<double> capap(m, 0.0), hd(m, 0.0);
  int rc = HMVM_OK;
  double bb = 0, rr = 0, relres = 0;
  int steps = 0;
  // r = b - A u; p_0 = r
  rc = hmvm_b200_apply(plan, u, ar, st);
  if (!rc) {
    s.lin(r, b, -1.0, ar);
    cudaMemcpyAsync(p, r, sizeof(T) * ld, cudaMemcpyDeviceToDevice, st);
    rc = s.dot2(b, b, r, r, &bb, &rr);
  }
  const double bnorm = std::sqrt(bb);
  relres = bnorm > 0 ? std::sqrt(rr) / bnorm : 0.0;
  if (!rc && relres >= eps && max_steps > 0) rc = hmvm_b200_apply(plan, p, ap, st);  // ap_0 = A p_0
  for (int in = 1; !rc && relres >= eps && in <= max_steps; in++) {
    const int ik = (in - 1) % m;
    T* q = ap + (size_t)ik * ld;
    double nom, qq;
    rc = s.dot2(q, r, q, q, &nom, &qq);
    if (rc) break;
    if (qq == 0.0) {
      rc = set_error(HMVM_EINVAL, "gcrm: breakdown (A p vanished)");
      break;
    }
    capap[ik] = qq;
    const double alpha = nom / qq;
    s.lin(u, u, alpha, p + (size_t)ik * ld);  // u += alpha p_ik
    s.lin(r, r, -alpha, q);                   // r -= alpha ap_ik
    rc = s.dot2(r, r, nullptr, nullptr, &rr, nullptr);
    if (rc) break;
    relres = std::sqrt(rr) / bnorm;
    steps = in;
    if (relres < eps || in == max_steps) break;
    rc = hmvm_b200_apply(plan, r, ar, st);  // ar = A r
    if (rc) break;
    const int ikn = in % m;
    cudaMemcpyAsync(p + (size_t)ikn * ld, r, sizeof(T) * ld, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(ap + (size_t)ikn * ld, ar, sizeof(T) * ld, cudaMemcpyDeviceToDevice, st);
    // beta_il = -(ap_il . ar) / capap_il for il = 0..ik, all against the same ar
    const int k = ik + 1;
    dotm_partial<T><<<dim3(kDotBlocks, k), kDotThreads, 0, st>>>(ap, ld, ar, n, part);
    dotm_final<<<k, kDotBlocks, 0, st>>>(part, kDotBlocks, dots);
    if (cudaMemcpyAsync(hd.data(), dots, sizeof(double) * k, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      rc = set_error(HMVM_ECUDA, "gcrm: inner products");
      break;
    }
    Betas be;
    for (int il = 0; il < k; il++) be.b[il] = -hd[il] / capap[il];
    gcr_update<T><<<(n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184, 256, 0, st>>>(p, ap, ld, k, ikn, be, n);
  }
  cudaStreamSynchronize(st);
  cudaFree(buf);
  cudaFree(part);
  if (steps_out) *steps_out = steps;
  if (relres_out) *relres_out = relres;
  if (!rc) rc = hmvm_b200_plan_status(plan);
  return rc;
}

}  // namespace

extern "C" int hmvm_b200_bicgstab(hmvm_plan* plan, const void* b_dev, void* u_dev, int32_t max_steps, double eps,
                                  int32_t* steps, double* relres, void* stream) {
  hmvm_plan_info info;
  int rc = hmvm_b200_plan_get_info(plan, &info);
  if (rc) return rc;
  if (info.nd > 0 && (!b_dev || !u_dev)) return set_error(HMVM_EINVAL, "b or u is NULL");
  if (max_steps < 0 || !(eps >= 0.0)) return set_error(HMVM_EINVAL, "max_steps < 0 or eps not >= 0");
  if (info.nd == 0) {
    if (steps) *steps = 0;
    if (relres) *relres = 0.0;
    return HMVM_OK;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  if (cudaSetDevice(info.device) != cudaSuccess) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (info.precision == HMVM_FP32)
    rc = bicgstab_t<float>(plan, info.nd, static_cast<const float*>(b_dev), static_cast<float*>(u_dev), max_steps,
                           eps, steps, relres, st);
  else
    rc = bicgstab_t<double>(plan, info.nd, static_cast<const double*>(b_dev), static_cast<double*>(u_dev), max_steps,
                            eps, steps, relres, st);
  cudaSetDevice(cur);
  return rc;
}

extern "C" int hmvm_b200_gcrm(hmvm_plan* plan, const void* b_dev, void* u_dev, int32_t max_steps, int32_t restart,
                              double eps, int32_t* steps, double* relres, void* stream) {
  hmvm_plan_info info;
  int rc = hmvm_b200_plan_get_info(plan, &info);
  if (rc) return rc;
  if (info.nd > 0 && (!b_dev || !u_dev)) return set_error(HMVM_EINVAL, "b or u is NULL");
  if (max_steps < 0 || !(eps >= 0.0)) return set_error(HMVM_EINVAL, "max_steps < 0 or eps not >= 0");
  if (restart < 1 || restart > kMaxRestart) return set_error(HMVM_EINVAL, "restart must be in 1..64");
  if (info.nd == 0) {
    if (steps) *steps = 0;
    if (relres) *relres = 0.0;
    return HMVM_OK;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  if (cudaSetDevice(info.device) != cudaSuccess) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (info.precision == HMVM_FP32)
    rc = gcrm_t<float>(plan, info.nd, static_cast<const float*>(b_dev), static_cast<float*>(u_dev), max_steps,
                       restart, eps, steps, relres, st);
  else
    rc = gcrm_t<double>(plan, info.nd, static_cast<const double*>(b_dev), static_cast<double*>(u_dev), max_steps,
                        restart, eps, steps, relres, st);
  cudaSetDevice(cur);
  return rc;
}

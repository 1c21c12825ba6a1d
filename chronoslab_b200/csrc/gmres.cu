// Right-preconditioned restarted GMRES on the GPU with the V-cycle as the
// preconditioner: the gmres_RIGHT.m caller (LinearSolver/GMRES_CJ/
// gmres_RIGHT.m:7-650) of the reference, with its stopping logic -- implicit
// residual test, confirmation by the explicit residual, up to maxmsteps more
// steps, stagnation test, restart from the iterate of minimal residual,
// flags 0-3 and iter = [outer inner].
//
// The Krylov basis is orthogonalised by classical Gram-Schmidt applied twice
// (CGS2) instead of the reference's Householder reflectors: both give the
// Arnoldi relation to working accuracy and the same iterates in exact
// arithmetic, and CGS2 needs two batched passes over the basis per step
// instead of a sequence of dependent reflector applications.  The projections
// V^T w are reduced deterministically (fixed tiles, fixed order), and the
// Hessenberg matrix, Givens rotations and least-squares solves live on the
// host (at most restart columns).
#include <cmath>
#include <functional>
#include <limits>
#include <vector>

#include "hier.h"

namespace chronos {

namespace {

constexpr int kMdotThreads = 256;
constexpr int kMdotRows = kMdotThreads * 8;   // rows per block tile

// part[b * k + j] = sum over block b's rows of V[:, j] w.
__global__ void k_mdot_part(int n, int k, const double *__restrict__ V, int64_t ldv,
                            const double *__restrict__ w, double *__restrict__ part) {
  __shared__ double sm[32];
  const int r0 = blockIdx.x * kMdotRows;
  double wr[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int r = r0 + u * kMdotThreads + threadIdx.x;
    wr[u] = r < n ? w[r] : 0.0;
  }
  for (int j = 0; j < k; ++j) {
    const double *Vj = V + (int64_t)j * ldv;
    double s = 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = r0 + u * kMdotThreads + threadIdx.x;
      if (r < n) s += Vj[r] * wr[u];
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) part[(int64_t)blockIdx.x * k + j] = s;
  }
}

// h[j] = sum over blocks b (in order of b) of part[b * k + j]; one block per j.
__global__ void k_mdot_fin(int nb, int k, const double *__restrict__ part, double *__restrict__ h) {
  __shared__ double sm[32];
  const int j = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[(int64_t)b * k + j];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) h[j] = s;
}

// w += sign * V[:, 0:k] h
__global__ void k_basis_combine(int n, int k, const double *__restrict__ V, int64_t ldv,
                                const double *__restrict__ h, double sign, double *__restrict__ w) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < k; ++j) s += V[r + (int64_t)j * ldv] * h[j];
    w[r] += sign * s;
  }
}

__global__ void k_all_finite(int n, const double *__restrict__ v, int *__restrict__ bad) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    if (!isfinite(v[r])) *bad = 1;
}

// Back substitution R z = y (R upper triangular, column-major, leading dim ld).
std::vector<double> solve_upper(const std::vector<double> &R, int ld, int k,
                                const std::vector<double> &y) {
  std::vector<double> z(y.begin(), y.begin() + k);
  for (int i = k - 1; i >= 0; --i) {
    double s = z[i];
    for (int c = i + 1; c < k; ++c) s -= R[(size_t)c * ld + i] * z[c];
    z[i] = s / R[(size_t)i * ld + i];
  }
  return z;
}

}  // namespace

void gmres_right_device(Hier &h, const std::function<void(const double *, double *)> &apply_op,
                        const double *b, double *x, int restart, double tol, int maxit,
                        GmresResult &res) {
  cudaStream_t st = h.st;
  const int n = h.levels[0].n;
  const double eps = std::numeric_limits<double>::epsilon();
  const int outer = std::max(maxit, 0);
  const int inner = std::min(std::max(restart, 0), n);                 // :143-157
  DBuf<double> scratch(256);
  auto dot = [&](const double *a, const double *c) { return device_dot(n, a, c, scratch.get(), st); };
  auto norm = [&](const double *a) { return std::sqrt(std::max(dot(a, a), 0.0)); };
  res = GmresResult{};
  const double n2b = norm(b);
  if (n2b == 0.0) {                                                     // :160-172
    CHRONOS_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    res.flag = 0;
    res.relres = 0.0;
    res.resvec.assign(1, 0.0);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    return;
  }
  const int64_t ld = n;
  DBuf<double> V((size_t)(inner + 1) * n), r(n), w(n), z(n), xm(n), xmin(n), part, hd(inner + 2);
  DBuf<int> bad(1);
  const int nb = (int)ceil_div(n, kMdotRows);
  part.alloc((size_t)nb * (inner + 1) + 1);
  const int eg = (int)std::min<int64_t>(ceil_div(n, 256), (int64_t)num_sms() * 16);
  auto copy = [&](const double *src, double *dst) {
    CHRONOS_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  };
  auto residual = [&](const double *xv, double *rv) {                   // rv = b - A xv
    apply_op(xv, rv);
    device_axpby(n, 1.0, b, -1.0, rv, st);
  };
  // z = V[:, 0:k] y
  auto combine = [&](const std::vector<double> &y, int k, double *out) {
    CHRONOS_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * n, st));
    if (k <= 0) return;
    hd.upload(y.data(), k, st);
    k_basis_combine<<<eg, 256, 0, st>>>(n, k, V.get(), ld, hd.get(), 1.0, out);
    CHRONOS_CHECK_LAUNCH();
  };
  auto finite = [&](const double *v) {
    bad.zero(st);
    k_all_finite<<<eg, 256, 0, st>>>(n, v, bad.get());
    CHRONOS_CHECK_LAUNCH();
    int bh = 0;
    CHRONOS_CUDA(cudaMemcpyAsync(&bh, bad.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    return bh == 0;
  };
  // CGS2 projection of w on V[:, 0:k]: w -= V h twice, hsum = h1 + h2
  std::vector<double> hcol(inner + 1), htmp(inner + 1);
  auto project = [&](int k) {
    std::fill(hcol.begin(), hcol.end(), 0.0);
    for (int pass = 0; pass < 2; ++pass) {
      k_mdot_part<<<nb, kMdotThreads, 0, st>>>(n, k, V.get(), ld, w.get(), part.get());
      CHRONOS_CHECK_LAUNCH();
      k_mdot_fin<<<k, 256, 0, st>>>(nb, k, part.get(), hd.get());
      CHRONOS_CHECK_LAUNCH();
      k_basis_combine<<<eg, 256, 0, st>>>(n, k, V.get(), ld, hd.get(), -1.0, w.get());
      CHRONOS_CHECK_LAUNCH();
      hd.download(htmp.data(), k, st);
      CHRONOS_CUDA(cudaStreamSynchronize(st));
      for (int j = 0; j < k; ++j) hcol[j] += htmp[j];
    }
  };

  int flag = 1;
  copy(x, xmin.get());
  int imin = 0, jmin = 0;
  const double tolb = tol * n2b;
  int stag = 0, moresteps = 0, minupdated = 0;
  const int maxmsteps = std::min({n / 50, 5, n - maxit});               // :221
  const int maxstagsteps = 3;
  residual(x, r.get());                                                 // :226
  double normr = norm(r.get());
  if (normr <= tolb) {                                                  // :227-237
    res.flag = 0;
    res.relres = normr / n2b;
    res.resvec.assign(1, normr);
    CHRONOS_CUDA(cudaStreamSynchronize(st));
    return;
  }
  std::vector<double> resvec((size_t)inner * outer + 1, 0.0);
  resvec[0] = normr;
  double normrmin = normr, normr_act = normr;
  std::vector<double> R((size_t)inner * inner, 0.0), cs(inner, 0.0), sn(inner, 0.0),
      g(inner + 1, 0.0);
  int it_out = 0, it_in = 0, outiter = 0, initer = 0;
  bool have_xm = false;
  std::vector<double> yprev;
  for (outiter = 1; outiter <= outer; ++outiter) {                      // :302
    normr = norm(r.get());
    // v_0 = r / ||r||; g = ||r|| e_1
    device_scale_copy(n, 1.0 / normr, r.get(), V.get(), st);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = normr;
    have_xm = false;
    initer = 0;
    for (int k = 1; k <= inner; ++k) {                                  // :317
      initer = k;
      double *vk = V.get() + (int64_t)(k - 1) * ld;
      h.vcycle(vk, z.get(), nullptr, nullptr);                          // :332-352
      if (!finite(z.get())) { flag = 2; break; }
      apply_op(z.get(), w.get());
      project(k);                                                       // :353-378
      const double hk1 = norm(w.get());
      if (hk1 != 0.0) device_scale_copy(n, 1.0 / hk1, w.get(), V.get() + (int64_t)k * ld, st);
      // previous rotations, then the new one (:380-395)
      for (int c = 0; c < k - 1; ++c) {
        const double t = hcol[c];
        hcol[c] = cs[c] * t + sn[c] * hcol[c + 1];
        hcol[c + 1] = -sn[c] * t + cs[c] * hcol[c + 1];
      }
      double hkk = hcol[k - 1];
      const double rho = std::hypot(hkk, hk1);
      if (rho != 0.0) {
        cs[k - 1] = hkk / rho;
        sn[k - 1] = hk1 / rho;
      } else {
        cs[k - 1] = 1.0;
        sn[k - 1] = 0.0;
      }
      g[k] = -sn[k - 1] * g[k - 1];
      g[k - 1] = cs[k - 1] * g[k - 1];
      hcol[k - 1] = rho;
      for (int i = 0; i < inner; ++i) R[(size_t)(k - 1) * inner + i] = i < k ? hcol[i] : 0.0;
      normr = std::fabs(g[k]);                                          // :396-406
      resvec[(size_t)(outiter - 1) * inner + k] = normr;
      normr_act = normr;
      if (normr <= tolb || stag >= maxstagsteps || moresteps) {         // :409
        // xm = x + M (V y) with y = R \ g.  The reference updates xm
        // incrementally from the previous y (the same vector in exact
        // arithmetic) and counts a stagnation step when the update's
        // coefficients are below eps times the iterate's norm; V is
        // orthonormal, so coefficient norms are vector norms.
        const std::vector<double> y = solve_upper(R, inner, k, g);
        double nadd = 0.0;
        for (int i = 0; i < k; ++i) {
          const double d = y[i] - (have_xm && i < (int)yprev.size() ? yprev[i] : 0.0);
          nadd += d * d;
        }
        nadd = std::sqrt(nadd);
        const double nref = have_xm ? norm(xm.get()) : norm(x);
        stag = (nadd < eps * nref) ? stag + 1 : 0;
        yprev = y;
        combine(y, k, z.get());
        h.vcycle(z.get(), w.get(), nullptr, nullptr);
        if (!finite(w.get())) { flag = 2; break; }
        copy(x, xm.get());
        device_axpby(n, 1.0, w.get(), 1.0, xm.get(), st);
        have_xm = true;
        residual(xm.get(), r.get());                                    // :477-484
        const double nr = norm(r.get());
        if (nr <= tol * n2b) {
          copy(xm.get(), x);
          flag = 0;
          it_out = outiter;
          it_in = k;
          break;
        }
        normr_act = nr;
        resvec[(size_t)(outiter - 1) * inner + k] = normr_act;
        if (normr_act <= normrmin) {                                    // :496-508
          normrmin = normr_act;
          imin = outiter;
          jmin = k;
          copy(xm.get(), xmin.get());
          minupdated = 1;
        }
        if (normr_act <= tolb) {
          copy(xm.get(), x);
          flag = 0;
          it_out = outiter;
          it_in = k;
          break;
        }
        if (stag >= maxstagsteps && moresteps == 0) stag = 0;           // :515-531
        ++moresteps;
        if (moresteps >= maxmsteps) {
          flag = 3;
          it_out = outiter;
          it_in = k;
          break;
        }
      }
      if (normr_act <= normrmin) {                                      // :534-545
        normrmin = normr_act;
        imin = outiter;
        jmin = k;
        minupdated = 1;
      }
      if (stag >= maxstagsteps) { flag = 3; break; }
      if (hk1 == 0.0) break;                                            // exact solution space
    }
    if (flag != 0) {                                                    // :552-590
      const int idx = minupdated ? jmin : initer;
      if (idx > 0) {
        const std::vector<double> y = solve_upper(R, inner, idx, g);
        combine(y, idx, z.get());
        h.vcycle(z.get(), w.get(), nullptr, nullptr);
        if (!finite(w.get())) { flag = 2; break; }
        device_axpby(n, 1.0, w.get(), 1.0, x, st);
      }
      copy(x, xmin.get());
      residual(x, r.get());
      normr_act = norm(r.get());
    }
    if (normr_act <= normrmin) {                                        // :591-597
      copy(x, xmin.get());
      normrmin = normr_act;
      imin = outiter;
      jmin = initer;
    }
    if (flag == 3) break;
    if (normr_act <= tolb) {
      flag = 0;
      it_out = outiter;
      it_in = initer;
      break;
    }
    minupdated = 0;
  }
  if (outiter > outer) outiter = outer;
  res.relres = normr_act / n2b;                                         // :637-644
  if (flag != 0) {
    copy(xmin.get(), x);
    it_out = imin;
    it_in = jmin;
  }
  res.flag = flag;
  res.outer = it_out;
  res.inner = it_in;
  const size_t last = (size_t)std::max(outiter - 1, 0) * inner + initer + 1;  // :645-648
  resvec.resize(std::min(last, resvec.size()));
  if (flag == 2 && initer != 0 && !resvec.empty()) resvec.pop_back();
  res.resvec = std::move(resvec);
  CHRONOS_CUDA(cudaStreamSynchronize(st));
}

}  // namespace chronos

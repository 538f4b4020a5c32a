// OrbitIntegration on the device: phase-space grid, per-orbit radial time
// integral (Omega_1), azimuthal phase integral (Omega_2), subsampled
// trajectory (w1, r, theta), Jacobian of (Rc, v) -> (E, L) and the
// Toomre-Zang distribution function with its E and L derivatives.
//
// Follows src/KalnajsLogSpiral/OrbitIntegration.jl:102-382 and
// src/KalnajsLogSpiral/Models.jl:40-169 of the reference.  One CTA per
// orbit; the reference's sequential cumsum over nw points
// (OrbitIntegration.jl:277-294) becomes a chunked block-wide prefix scan:
// each thread sums a contiguous chunk, the chunk sums are scanned, and a
// second pass re-evaluates the chunk to emit the running sums at the
// subsample points 1:nwai:nw.
//
// This translation unit is compiled without FMA contraction (-fmad=false)
// and keeps the reference's association order: v_r^2 = 2(E - ln x) x^2 - L^2
// cancels like 1/e^2 near the turning points of near-circular orbits, so a
// one-ulp change in any term moves Omega_1 by up to ~1e-10 relative.
#include "kls_internal.cuh"
#include <cmath>
#include <vector>

namespace {

constexpr int ORB_THREADS = 512;

struct OrbitParams {
  int NR, Ne, nw, nwa, nwai, Ia_last;
  double Rc_min, Rc_max, v_min;
  double L0, q1, qz, sigma_r0, DF_const;
  int n_zang;
  double dw;
  int quad_v;          // KLS_QUAD_* rule of the v grid (never DEFAULT here)
};

// trapezoid weight of point i of a sequence (OrbitIntegration.jl:63-74)
__host__ __device__ double trap_w(double xm, double x0, double xp, int i, int n) {
  if (n < 2) return 0.0;
  if (i == 0) return (xp - x0) / 2;
  if (i == n - 1) return (x0 - xm) / 2;
  return (xp - xm) / 2;
}

// Weight of point i of an n-point uniform grid x(.) under `rule`:
// KLS_QUAD_TRAPEZOID (OrbitIntegration.jl:63-74), KLS_QUAD_SIMPSON
// (OrbitIntegration.jl:79-95: the trapezoid rule for n < 3 or even n) or
// KLS_QUAD_BOOLE (2h/45 (7, 32, 12, 32, 14, ..., 7) for n = 4k + 1 >= 5,
// else the Simpson rule; NL_julia_boole.jl:186-217).
template <typename X>
__host__ __device__ double quad_w(int rule, const X& x, int i, int n) {
  auto trap = [&]() {
    double xm = i > 0 ? x(i - 1) : 0.0, xp = i < n - 1 ? x(i + 1) : 0.0;
    return trap_w(xm, x(i), xp, i, n);
  };
  if (rule == KLS_QUAD_TRAPEZOID) return trap();
  if (rule == KLS_QUAD_BOOLE && n >= 5 && (n - 1) % 4 == 0) {
    double dx = x(1) - x(0);
    double f = 2 * dx / 45;
    if (i == 0 || i == n - 1) return 7 * f;
    int r = i % 4;
    return r == 0 ? 14 * f : (r == 2 ? 12 * f : 32 * f);
  }
  if (n < 3 || (n % 2) == 0) return trap();
  double dx = x(1) - x(0);
  if (i == 0 || i == n - 1) return dx / 3;
  return (i % 2 == 1) ? 4 * dx / 3 : 2 * dx / 3;
}

// S_e weight of v point ie (OrbitIntegration.jl:119-123; Simpson unless the
// configuration selects another rule)
__device__ double v_weight(const OrbitParams& P, int ie) {
  auto v = [&](int i) { return kls_lin(P.v_min, 1.0, P.Ne, i); };
  return quad_w(P.quad_v, v, ie, P.Ne);
}

__device__ double taper(const OrbitParams& P, double L) {
  if (P.n_zang == 0) return 1.0;
  double La = fabs(L);
  if (La < 1e-12) return 0.0;
  return 1.0 / (1.0 + pow(P.L0 / La, (double)P.n_zang));
}

__device__ double df0(const OrbitParams& P, double E, double L) {
  double La = fabs(L);
  if (La < 1e-12) return 0.0;
  double s2 = P.sigma_r0 * P.sigma_r0;
  double r = P.DF_const * exp(-E / s2) * pow(La, P.qz) * taper(P, L);
  return isfinite(r) ? r : 0.0;
}

// Radial-integrand pieces at point i of the w grid: x, svr (time) and
// svr_phi (phase) before endpoint extrapolation.
struct PointVals { double x, svr, svp; };

__device__ __forceinline__ PointVals point_vals(double rs, double drs, double E, double L2,
                                                bool nonradial, double cw, double sw) {
  PointVals v;
  v.x = rs - drs * cw;
  if (nonradial) {
    // (2 (E - V(x))) * x^2 - L^2, the reference's association order
    double vr2 = 2.0 * (E - log(v.x)) * (v.x * v.x) - L2;
    double rvr = sqrt(fmax(0.0, vr2));
    v.svr = sw * v.x / rvr;
    v.svp = sw / rvr;
  } else {
    double vr2 = 2.0 * (E - log(v.x));
    double vr = sqrt(fmax(0.0, vr2));
    v.svr = sw / vr;
    v.svp = 0.0;
  }
  return v;
}

template <typename T>
__device__ T block_exclusive_scan(T val, T* sh, T* total) {
  // sh: blockDim.x entries
  int t = threadIdx.x;
  sh[t] = val;
  __syncthreads();
  for (int off = 1; off < blockDim.x; off <<= 1) {
    T add = (t >= off) ? sh[t - off] : T(0);
    __syncthreads();
    sh[t] += add;
    __syncthreads();
  }
  T incl = sh[t];
  if (total) *total = sh[blockDim.x - 1];
  __syncthreads();
  return incl - val;  // exclusive
}

// table read, guarded in the bounds-checked build (plain t[i] otherwise)
#define ORB_TAB(t, i) KLS_LD(KLS_IB((i), P.nw, KS_ORBIT_TABLE), t[i], 0.0)

__global__ void __launch_bounds__(ORB_THREADS)
orbit_kernel(OrbitParams P, const double* __restrict__ cosw, const double* __restrict__ sinw,
             const double* __restrict__ rc_tab, const double* __restrict__ SRC,
             double* __restrict__ of, int NPh, int* __restrict__ valid,
             double* __restrict__ w1o, double* __restrict__ rao, double* __restrict__ phao) {
  __shared__ double sh_t[ORB_THREADS];
  __shared__ double sh_p[ORB_THREADS];
  __shared__ double sh_misc[4];
  const int p = blockIdx.x;
  const int iR = p % P.NR, ie = p / P.NR;
  const int tid = threadIdx.x;

  // ---- grid scalars (OrbitIntegration.jl:102-170), computed redundantly
  const double Rc = KLS_LD(KLS_IB(iR, P.NR, KS_ORBIT_TABLE), rc_tab[iR], 0.0);
  double v = kls_lin(P.v_min, 1.0, P.Ne, ie);
  if (fabs(v) < 1e-14) v = 1e-12;
  const double sg = (v > 0) ? 1.0 : ((v < 0) ? -1.0 : 0.0);
  const double ecc = 1.0 - fabs(v);
  const double R1 = Rc * (1.0 - ecc), R2 = Rc * (1.0 + ecc);
  double E;
  if (fabs(R2 * R2 - R1 * R1) > 1e-14) {
    E = (log(R2) * (R2 * R2) - log(R1) * (R1 * R1)) / (R2 * R2 - R1 * R1);
  } else {
    E = Rc * (1.0 / Rc) / 2 + log(Rc);
  }
  if (!isfinite(E)) E = log(R2);
  double L2 = 2.0 * (E - log(R2)) * (R2 * R2);
  if (L2 < 1e-14) L2 = 0.0;
  const double L = sqrt(L2) * sg;

  const double kap = sqrt(2.0) / Rc, Om = 1.0 / Rc;
  const int nw = P.nw, nwa = P.nwa, nwai = P.nwai;
  double* w1p = w1o + (size_t)p * nwa;
  double* rap = rao + (size_t)p * nwa;
  double* php = phao + (size_t)p * nwa;
  bool fin = true;
  double Om1 = 0.0, Om2 = 0.0;

  if (fabs(ecc) < 1e-10 || ecc < 0.01) {
    // circular (:222-229) and epicyclic (:232-241) branches
    Om1 = kap;
    Om2 = Om * sg;
    const bool circ = fabs(ecc) < 1e-10;
    const double a_j = (R2 - R1) / 2;
    for (int j = tid; j < nwa; j += blockDim.x) {
      int i = j * nwai;
      double wa = kls_lin(1e-8, KLS_PI - 1e-8, nw, i);
      double r, ph;
      if (circ) {
        r = Rc;
        ph = wa * Om2 / Om1;
      } else {
        r = Rc - a_j * ORB_TAB(cosw, i);
        ph = wa * Om2 / Om1 + 2 * Om / kap * a_j / Rc * ORB_TAB(sinw, i) * sg;
      }
      KLS_UNLESS(KLS_IB((int64_t)p * nwa + j, (int64_t)NPh * nwa, KS_ORBIT_SAMPLES), continue)
      w1p[j] = wa; rap[j] = r; php[j] = ph;
      fin = fin && isfinite(wa) && isfinite(r) && isfinite(ph);
    }
  } else {
    // general orbit (:244-302)
    const double rs = (R1 + R2) / 2, drs = (R2 - R1) / 2;
    const bool nonradial = L2 > 1e-12;
    const bool phase_int = (fabs(1.0 - ecc) > 1e-10) && nonradial;
    const double dtc = drs * P.dw;
    // svr / svr_phi with the reference's endpoint extrapolation
    auto vals_at = [&](int i, double& x, double& svr, double& svp) {
      PointVals a = point_vals(rs, drs, E, L2, nonradial, ORB_TAB(cosw, i), ORB_TAB(sinw, i));
      x = a.x; svr = a.svr; svp = a.svp;
      if (i == 0 || i == nw - 1) {
        int i1 = (i == 0) ? 1 : nw - 2, i2 = (i == 0) ? 2 : nw - 3;
        PointVals b = point_vals(rs, drs, E, L2, nonradial, ORB_TAB(cosw, i1), ORB_TAB(sinw, i1));
        PointVals c = point_vals(rs, drs, E, L2, nonradial, ORB_TAB(cosw, i2), ORB_TAB(sinw, i2));
        if (i == nw - 1 || nonradial) svr = 2.0 * b.svr - c.svr;
        svp = 2.0 * b.svp - c.svp;
      }
    };
    const int chunk = (nw + blockDim.x - 1) / blockDim.x;
    const int i0 = tid * chunk, i1 = min(nw, i0 + chunk);
    // pass 1: chunk sums of dt2 and dt4
    double st = 0.0, sp = 0.0;
    if (i0 < i1) {
      double x, svr, svp;
      double prev_t = 0.0, prev_p = 0.0;
      if (i0 > 0) {
        vals_at(i0 - 1, x, svr, svp);
        prev_t = dtc * svr;
        prev_p = dtc * svp / x;
      }
      for (int i = i0; i < i1; ++i) {
        vals_at(i, x, svr, svp);
        double dt1 = dtc * svr, dt3 = dtc * svp / x;
        if (i > 0) { st += (prev_t + dt1) / 2; sp += (prev_p + dt3) / 2; }
        prev_t = dt1; prev_p = dt3;
      }
    }
    double tot_t, tot_p;
    double pre_t = block_exclusive_scan(st, sh_t, &tot_t);
    double pre_p = block_exclusive_scan(sp, sh_p, &tot_p);
    Om1 = KLS_PI / tot_t;
    // pass 2: running sums at subsample points
    if (i0 < i1) {
      double x, svr, svp;
      double prev_t = 0.0, prev_p = 0.0;
      double rt = pre_t, rp = pre_p;
      if (i0 > 0) {
        vals_at(i0 - 1, x, svr, svp);
        prev_t = dtc * svr;
        prev_p = dtc * svp / x;
      }
      for (int i = i0; i < i1; ++i) {
        vals_at(i, x, svr, svp);
        double dt1 = dtc * svr, dt3 = dtc * svp / x;
        if (i > 0) { rt += (prev_t + dt1) / 2; rp += (prev_p + dt3) / 2; }
        prev_t = dt1; prev_p = dt3;
        if (i % nwai == 0 && i <= P.Ia_last) {
          int j = i / nwai;
          double ph;
          if (phase_int) ph = L * rp;
          else ph = (j == 0) ? 0.0 : (KLS_PI / 2) * 1.0 * sg;
          double wv = rt * Om1;
          KLS_UNLESS(KLS_IB((int64_t)p * nwa + j, (int64_t)NPh * nwa, KS_ORBIT_SAMPLES), continue)
          w1p[j] = wv; rap[j] = x; php[j] = ph;
          fin = fin && isfinite(wv) && isfinite(x) && isfinite(ph);
          if (i == P.Ia_last) sh_misc[0] = ph;
        }
      }
    }
    __syncthreads();
    Om2 = Om1 * sh_misc[0] / KLS_PI;
  }
  int all_fin = __syncthreads_and(fin ? 1 : 0);

  if (tid == 0) {
    // Jacobian (OrbitIntegration.jl:341-382)
    double jac = 0.0;
    if (fabs(R2 - R1) > 1e-12 && fabs(L) > 1e-12) {
      double V1 = log(R1), V2 = log(R2), dV1 = 1.0 / R1, dV2 = 1.0 / R2;
      double t1 = 2 * (E - V1) * R1 - dV1 * (R1 * R1);
      double t2 = 2 * (E - V2) * R2 - dV2 * (R2 * R2);
      double den = R2 * R2 - R1 * R1;
      double dj = fabs(t1 * t2 / den);
      jac = 2 * dj * Rc / Om1 / fabs(L);
    }
    if (fabs(L) <= 1e-12) {
      double DelE = 2.0 * (E - log(R1));
      jac = sqrt(fmax(DelE, 0.0)) * (1.0 / R2) * 2 * Rc / Om1;
      if (!isfinite(jac)) jac = 0.0;
    }
    // DF and derivatives (Models.jl:137-169), NaN -> 0 (:331-333)
    double F0 = df0(P, E, L);
    double FE = -F0 / (P.sigma_r0 * P.sigma_r0);
    double FL = 0.0;
    if (fabs(L) >= 1e-12) FL = F0 * (P.qz + P.n_zang - P.n_zang * taper(P, L)) / fabs(L);
    if (!isfinite(F0)) F0 = 0.0;
    if (!isfinite(FE)) FE = 0.0;
    if (!isfinite(FL)) FL = 0.0;
    // S_e quadrature weight (OrbitIntegration.jl:119-123); S_RC from the host
    double src = KLS_LD(KLS_IB(iR, P.NR, KS_ORBIT_TABLE), SRC[iR], 0.0);
    double se = v_weight(P, ie);
    double vals[OF_COUNT] = {Rc, ecc, v, R1, R2, E, L, L2, sg, se,
                             Om1, Om2, jac, F0, FE, FL, src * se * jac};
    for (int f = 0; f < OF_COUNT; ++f)
      KLS_IF(KLS_IB((int64_t)f * NPh + p, (int64_t)OF_COUNT * NPh, KS_ORBIT_FIELDS))
      of[(size_t)f * NPh + p] = vals[f];
    double ratio = Om2 / Om1;
    KLS_IF(KLS_IB(p, NPh, KS_ORBIT_FIELDS)) valid[p] = (all_fin && isfinite(ratio)) ? 1 : 0;
  }
}

}  // namespace

int kls_run_orbits(kls_ctx* c) {
  const kls_config& k = c->cfg;
  OrbitParams P{};
  P.NR = c->NR; P.Ne = c->Ne; P.nw = c->nw; P.nwa = c->nwa; P.nwai = c->nwai;
  P.Ia_last = (c->nwa - 1) * c->nwai;
  P.Rc_min = k.Rc_min; P.Rc_max = k.Rc_max; P.v_min = k.v_min;
  P.L0 = k.L0; P.q1 = k.q1; P.qz = k.q1 - 1.0; P.n_zang = k.n_zang;
  P.sigma_r0 = 1.0 / std::sqrt(k.q1);
  // DF normalisation (Models.jl:53-54), Gamma of a real argument
  P.DF_const = 1.0 / (2.0 * KLS_PI * std::pow(2.0, P.qz / 2.0) * std::sqrt(KLS_PI) *
                      std::tgamma((P.qz + 1.0) / 2.0) * std::pow(P.sigma_r0, P.qz + 2.0));
  P.quad_v = k.quad_v == KLS_QUAD_DEFAULT ? KLS_QUAD_SIMPSON : k.quad_v;
  double w0 = kls_lin(1e-8, KLS_PI - 1e-8, c->nw, 0);
  double w1 = kls_lin(1e-8, KLS_PI - 1e-8, c->nw, 1);
  P.dw = w1 - w0;

  // Tables shared by every orbit, from the host C library: the w grid's cos
  // and sin, the log-spaced guiding-centre radii and their trapezoid weights
  // S_RC = Rc * trapz(ln Rc) (OrbitIntegration.jl:111-113, :188-193).  Near
  // a turning point x = rs - drs cos w cancels catastrophically, so the table
  // values, not just their accuracy, decide the last bits of Omega_1.
  std::vector<double> cw(c->nw), sw(c->nw), rc(c->NR), src(c->NR);
  for (int i = 0; i < c->nw; ++i) {
    double w = kls_lin(1e-8, KLS_PI - 1e-8, c->nw, i);
    cw[i] = std::cos(w);
    sw[i] = std::sin(w);
  }
  const double la = std::log10(k.Rc_min), lb = std::log10(k.Rc_max);
  for (int i = 0; i < c->NR; ++i) rc[i] = std::pow(10.0, kls_lin(la, lb, c->NR, i));
  {
    // S_RC = Rc * (weights on ln Rc): trapezoid unless configured
    std::vector<double> u(c->NR);
    for (int i = 0; i < c->NR; ++i) u[i] = std::log(rc[i]);
    const int rule = k.quad_rc == KLS_QUAD_DEFAULT ? KLS_QUAD_TRAPEZOID : k.quad_rc;
    auto x = [&](int i) { return u[i]; };
    for (int i = 0; i < c->NR; ++i) src[i] = rc[i] * quad_w(rule, x, i, c->NR);
  }
  KLS_CK(c, cudaMemcpyAsync(c->d_cosw, cw.data(), c->nw * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
  KLS_CK(c, cudaMemcpyAsync(c->d_sinw, sw.data(), c->nw * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
  KLS_CK(c, cudaMemcpyAsync(c->d_rc, rc.data(), c->NR * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
  KLS_CK(c, cudaMemcpyAsync(c->d_SRC, src.data(), c->NR * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
  kls_pre_mark(c, 0);
  orbit_kernel<<<c->NPh, ORB_THREADS, 0, c->stream>>>(P, c->d_cosw, c->d_sinw, c->d_rc, c->d_SRC,
                                                      c->d_of, c->NPh, c->d_valid, c->d_w1,
                                                      c->d_ra, c->d_pha);
  KLS_LAUNCHED(c);
  kls_pre_mark(c, 1);
  // the host vectors must outlive the asynchronous copies
  KLS_CK(c, cudaStreamSynchronize(c->stream));
  return KLS_OK;
}

int kls_upload_alpha(kls_ctx* c) {
  // alpha grid and its weights (BasisFunctions.jl:106-107: trapezoid unless
  // configured)
  std::vector<double> a(c->Na), d(c->Na);
  for (int i = 0; i < c->Na; ++i) a[i] = kls_lin(-c->cfg.alpha_max, c->cfg.alpha_max, c->Na, i);
  const int rule =
      c->cfg.quad_alpha == KLS_QUAD_DEFAULT ? KLS_QUAD_TRAPEZOID : c->cfg.quad_alpha;
  auto x = [&](int i) { return a[i]; };
  for (int i = 0; i < c->Na; ++i) d[i] = quad_w(rule, x, i, c->Na);
  KLS_CK(c, cudaMemcpy(c->d_alpha, a.data(), c->Na * sizeof(double), cudaMemcpyHostToDevice));
  KLS_CK(c, cudaMemcpy(c->d_dalpha, d.data(), c->Na * sizeof(double), cudaMemcpyHostToDevice));
  return KLS_OK;
}

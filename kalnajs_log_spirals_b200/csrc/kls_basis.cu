// BasisFunctions on the device.
//
// * W_l(alpha; J) table (BasisFunctions.jl:199-266, Eq. 41):
//     W[p, a, l] = (1/pi) sum_k Sw1_k cos(l w1_k + m phi_k) r_k^{-1/2} e^{-i alpha_a ln r_k}
//   evaluated per orbit as the product C[l,k] E[k,a] of a real matrix
//   C = Sw1_k cos(l w1_k + m phi_k) and a complex matrix
//   E = r_k^{-1/2} e^{-i alpha ln r_k}, on the FP64 tensor pipe (DMMA
//   m8n8k4).  C and E are generated in shared memory per 16-sample chunk:
//   each thread evaluates one anchor sincos and advances by complex rotation
//   over a short run (4 harmonics for C, 8 alphas for E), so the
//   transcendental cost is a small fraction of the contraction.
//   Orbits with non-finite samples are zero rows (BasisFunctions.jl:224-226);
//   non-finite generated factors are zeroed (BasisFunctions.jl:248).
// * N_m(alpha) (BasisFunctions.jl:281-304, Eq. 46) through ln|Gamma(z)|:
//   Re[G(z1)G(z2)/(G(z3)G(z4))] = |G(z1)|^2/|G(z3)|^2 since z2 = conj(z1),
//   z4 = conj(z3).  ln|Gamma| uses Stirling's asymptotic series
//   (Bernoulli-number coefficients) after the upward recurrence
//   Gamma(z+1) = z Gamma(z) moves Re z above 15.
// * Per-row resonant data, row k = il*NPh + p (BasisFunctions.jl:127-153):
//   G_k = DJ_p * F0l[p,l], F0l = (l Om1 + m Om2) FE + m FL,
//   Omega_res = l Om1 + m Om2.
#include "kls_internal.cuh"
#include <cmath>

namespace {

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// ---- W table kernel --------------------------------------------------------
constexpr int WL_LB = 32;      // harmonics per CTA
constexpr int WL_AB = 64;      // alphas per CTA
constexpr int WL_BK = 16;      // samples per chunk
constexpr int WL_SC = WL_BK + 4;   // smem row stride of C [l][k] (== 4 mod 16)
constexpr int WL_SE = WL_AB + 4;   // smem row stride of E [k][a]
constexpr int WL_THREADS = 128;

struct WlParams {
  int NPh, nwa, Na, Na_pad, n_l, l_min, m;
  double astep;          // alpha grid step
};

// orbit p's sample k, guarded in the bounds-checked build (plain t[k] otherwise)
#define WL_SMP(t, k) \
  KLS_LD(KLS_IB((int64_t)p * nwa + (k), (int64_t)NPh * nwa, KS_WL_SAMPLES), t[k], 0.0)

__global__ void __launch_bounds__(WL_THREADS)
wl_kernel(WlParams P, const double* __restrict__ of, const int* __restrict__ valid,
          const double* __restrict__ w1g, const double* __restrict__ rag,
          const double* __restrict__ phag, const double* __restrict__ alpha,
          double* __restrict__ Wre, double* __restrict__ Wim) {
  __shared__ double sC[WL_LB * WL_SC];
  __shared__ double sEr[WL_BK * WL_SE];
  __shared__ double sEi[WL_BK * WL_SE];
  // one orbit's (l block, alpha block) CTAs are consecutive in launch order,
  // so its w1 / r / theta samples are read from DRAM once and then from L2
  const int nlb = (P.n_l + WL_LB - 1) / WL_LB, nab = P.Na_pad / WL_AB;
  const int p = (int)(blockIdx.x / (unsigned)(nlb * nab));
  const int lb = (int)((blockIdx.x / (unsigned)nab) % (unsigned)nlb);
  const int ab = (int)(blockIdx.x % (unsigned)nab);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NPh = P.NPh, nwa = P.nwa;
  const double* w1 = w1g + (size_t)p * nwa;
  const double* ra = rag + (size_t)p * nwa;
  const double* pha = phag + (size_t)p * nwa;
  const bool ok = KLS_LD(KLS_IB(p, NPh, KS_WL_SAMPLES), valid[p] != 0, false);
  const double ratio = KLS_LD(KLS_IB(p, NPh, KS_WL_SAMPLES),
                              of[(size_t)OF_OM2 * NPh + p] / of[(size_t)OF_OM1 * NPh + p], 0.0);

  // accumulators: warp covers all 32 harmonics (4 m-tiles) x 16 alphas (2 n-tiles)
  double accR[4][2][2], accI[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      accR[i][j][0] = accR[i][j][1] = 0.0;
      accI[i][j][0] = accI[i][j][1] = 0.0;
    }

  // generator assignment: 16 samples x 8 sub-runs
  const int gk = tid & 15, gsub = tid >> 4;       // gsub 0..7
  const int l_first = lb * WL_LB + gsub * 4;       // C: 4 harmonics
  const int a_first = ab * WL_AB + gsub * 8;       // E: 8 alphas

  if (ok) {
    for (int k0 = 0; k0 < nwa; k0 += WL_BK) {
      // ---- generate C and E for samples k0..k0+15
      const int k = k0 + gk;
      if (k < nwa) {
        double wk = WL_SMP(w1, k), rk = WL_SMP(ra, k);
        double wm = k > 0 ? WL_SMP(w1, k - 1) : 0.0, wp = k < nwa - 1 ? WL_SMP(w1, k + 1) : 0.0;
        double sw;
        if (nwa < 2) sw = 0.0;
        else if (k == 0) sw = (wp - wk) / 2;
        else if (k == nwa - 1) sw = (wk - wm) / 2;
        else sw = (wp - wm) / 2;
        double phi = ratio * wk - WL_SMP(pha, k);
        // C: cos(l w1 + m phi), anchor at l_first, rotate by w1
        double th = (double)(P.l_min + l_first) * wk + (double)P.m * phi;
        double s, c, ss, cs;
        sincos(th, &s, &c);
        sincos(wk, &ss, &cs);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          double v = sw * c;
          if (!isfinite(v)) v = 0.0;
          sC[(gsub * 4 + j) * WL_SC + gk] = (l_first + j < P.n_l) ? v : 0.0;
          double cn = c * cs - s * ss;
          s = s * cs + c * ss;
          c = cn;
        }
        // E: r^{-1/2} e^{-i alpha ln r}, anchor at a_first, rotate by -astep ln r
        double lr = log(rk);
        double isq = 1.0 / sqrt(rk);
        double ta = -KLS_LD(KLS_IB(min(a_first, P.Na - 1), P.Na, KS_WL_SAMPLES),
                            alpha[min(a_first, P.Na - 1)], 0.0) * lr;
        sincos(ta, &s, &c);
        sincos(-P.astep * lr, &ss, &cs);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          double er = c * isq, ei = s * isq;
          if (!(isfinite(er) && isfinite(ei))) { er = 0.0; ei = 0.0; }
          bool in = a_first + j < P.Na;
          sEr[gk * WL_SE + gsub * 8 + j] = in ? er : 0.0;
          sEi[gk * WL_SE + gsub * 8 + j] = in ? ei : 0.0;
          double cn = c * cs - s * ss;
          s = s * cs + c * ss;
          c = cn;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) sC[(gsub * 4 + j) * WL_SC + gk] = 0.0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          sEr[gk * WL_SE + gsub * 8 + j] = 0.0;
          sEi[gk * WL_SE + gsub * 8 + j] = 0.0;
        }
      }
      __syncthreads();
      // ---- 4 k-steps of m8n8k4
#pragma unroll
      for (int kk = 0; kk < WL_BK; kk += 4) {
        double a[4], br[2], bi[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = sC[(i * 8 + (lane >> 2)) * WL_SC + kk + (lane & 3)];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          int col = warp * 16 + j * 8 + (lane >> 2);
          br[j] = sEr[(kk + (lane & 3)) * WL_SE + col];
          bi[j] = sEi[(kk + (lane & 3)) * WL_SE + col];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            dmma(accR[i][j][0], accR[i][j][1], a[i], br[j]);
            dmma(accI[i][j][0], accI[i][j][1], a[i], bi[j]);
          }
      }
      __syncthreads();
    }
  }
  // ---- epilogue: W / pi into rows il*NPh + p
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int il = lb * WL_LB + i * 8 + (lane >> 2);
    if (il >= P.n_l) continue;
    size_t row = ((size_t)il * NPh + p) * P.Na_pad;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      int a0 = ab * WL_AB + warp * 16 + j * 8 + 2 * (lane & 3);
      double r0 = accR[i][j][0] / KLS_PI, r1 = accR[i][j][1] / KLS_PI;
      double i0 = accI[i][j][0] / KLS_PI, i1 = accI[i][j][1] / KLS_PI;
      if (a0 >= P.Na) { r0 = 0.0; i0 = 0.0; }
      if (a0 + 1 >= P.Na) { r1 = 0.0; i1 = 0.0; }
      KLS_UNLESS(KLS_IB((int64_t)row + a0 + 1, (int64_t)P.n_l * NPh * P.Na_pad, KS_WL_OUT),
                 continue)
      *reinterpret_cast<double2*>(Wre + row + a0) = make_double2(r0, r1);
      *reinterpret_cast<double2*>(Wim + row + a0) = make_double2(i0, i1);
    }
  }
}

// ---- alpha grid and N_m(alpha) ------------------------------------------
// ln|Gamma(x + iy)| for x > 0 (Stirling series after upward recurrence).
__device__ double ln_abs_gamma(double x, double y) {
  double acc = 0.0;
  while (x < 15.0) {
    acc -= 0.5 * log(x * x + y * y);   // ln|z|
    x += 1.0;
  }
  // lnGamma(w) ~ (w - 1/2) ln w - w + ln(2 pi)/2 + sum_k c_k / w^(2k-1)
  double r = hypot(x, y), th = atan2(y, x);
  double lnr = log(r);
  double re = (x - 0.5) * lnr - y * th - x + 0.91893853320467274178;  // ln(2pi)/2
  // coefficients B_2k / (2k (2k-1)), k = 1..10
  const double cf[10] = {1.0 / 12.0,       -1.0 / 360.0,      1.0 / 1260.0,
                         -1.0 / 1680.0,    1.0 / 1188.0,      -691.0 / 360360.0,
                         1.0 / 156.0,      -3617.0 / 122400.0, 43867.0 / 244188.0,
                         -174611.0 / 125400.0};
  // 1/w = conj(w)/|w|^2 ; powers 1/w^(2k-1)
  double ir = x / (r * r), ii = -y / (r * r);            // 1/w
  double i2r = ir * ir - ii * ii, i2i = 2 * ir * ii;     // 1/w^2
  double pr = ir, pi = ii;
  for (int k = 0; k < 10; ++k) {
    re += cf[k] * pr;
    double nr = pr * i2r - pi * i2i;
    pi = pr * i2i + pi * i2r;
    pr = nr;
  }
  return re + acc;
}

// N_m(alpha) = |Gamma(z1)|^2 / |Gamma(z3)|^2 * pi * d_alpha,
// z1 = (m + 1/2 + i alpha)/2, z3 = (m + 3/2 + i alpha)/2
__global__ void n_kernel(int Na, int m, const double* __restrict__ alpha,
                         const double* __restrict__ dalpha, double* __restrict__ Nk) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Na) return;
  KLS_UNLESS(KLS_IB(i, Na, KS_NKERNEL), return)
  double a = alpha[i];
  double l1 = ln_abs_gamma((m + 0.5) / 2, a / 2);
  double l3 = ln_abs_gamma((m + 1.5) / 2, a / 2);
  Nk[i] = exp(2.0 * (l1 - l3)) * KLS_PI * dalpha[i];
}

__global__ void rows_kernel(int NPh, int n_l, int l_min, int m, int64_t K, int64_t K_pad,
                            const double* __restrict__ of, double* __restrict__ Gk,
                            double* __restrict__ Ok, double* __restrict__ F0l) {
  int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K_pad) return;
  KLS_UNLESS(KLS_IB(k, K_pad, KS_ROWS), return)
  if (k >= K) { Gk[k] = 0.0; Ok[k] = 0.0; F0l[k] = 0.0; return; }
  int il = (int)(k / NPh), p = (int)(k % NPh);
  KLS_UNLESS(KLS_IB((int64_t)OF_DJ * NPh + p, (int64_t)OF_COUNT * NPh, KS_ROWS), return)
  double l = (double)(l_min + il);
  double om1 = of[(size_t)OF_OM1 * NPh + p], om2 = of[(size_t)OF_OM2 * NPh + p];
  double FE = of[(size_t)OF_FE * NPh + p], FL = of[(size_t)OF_FL * NPh + p];
  double DJ = of[(size_t)OF_DJ * NPh + p];
  double ores = l * om1 + m * om2;
  double f0l = ores * FE + m * FL;
  Gk[k] = DJ * f0l;
  Ok[k] = ores;
  F0l[k] = f0l;
}

}  // namespace

int kls_run_basis(kls_ctx* c) {
  const kls_config& k = c->cfg;
  int r = kls_upload_alpha(c);
  if (r) return r;
  n_kernel<<<(c->Na + 127) / 128, 128, 0, c->stream>>>(c->Na, k.m, c->d_alpha, c->d_dalpha,
                                                      c->d_N);
  KLS_LAUNCHED(c);
  rows_kernel<<<(unsigned)((c->K_pad + 255) / 256), 256, 0, c->stream>>>(
      c->NPh, c->n_l, k.l_min, k.m, c->K, c->K_pad, c->d_of, c->d_Gk, c->d_Ok, c->d_F0l);
  KLS_LAUNCHED(c);
  // zero the padding rows of the table (rows K..K_pad-1)
  size_t pad_rows = (size_t)(c->K_pad - c->K);
  if (pad_rows) {
    KLS_CK(c, cudaMemsetAsync(c->d_Wre + (size_t)c->K * c->Na_pad, 0,
                              pad_rows * c->Na_pad * sizeof(double), c->stream));
    KLS_CK(c, cudaMemsetAsync(c->d_Wim + (size_t)c->K * c->Na_pad, 0,
                              pad_rows * c->Na_pad * sizeof(double), c->stream));
  }
  WlParams P{};
  P.NPh = c->NPh; P.nwa = c->nwa; P.Na = c->Na; P.Na_pad = c->Na_pad; P.n_l = c->n_l;
  P.l_min = k.l_min; P.m = k.m;
  P.astep = c->Na > 1 ? (2.0 * k.alpha_max) / (double)(c->Na - 1) : 0.0;
  dim3 grid((unsigned)c->NPh * ((c->n_l + WL_LB - 1) / WL_LB) * (c->Na_pad / WL_AB));
  kls_pre_mark(c, 2);
  wl_kernel<<<grid, WL_THREADS, 0, c->stream>>>(P, c->d_of, c->d_valid, c->d_w1, c->d_ra,
                                                c->d_pha, c->d_alpha, c->d_Wre, c->d_Wim);
  KLS_LAUNCHED(c);
  kls_pre_mark(c, 3);
  return KLS_OK;
}

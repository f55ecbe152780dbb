// Grid construction on the GPU: Gauss-Legendre nodes (FP64, double-double
// residuals), the Wigner d^l_{mn}(theta_j) recurrence (one thread per
// (m, theta_j) chain, exponent-scaled start values), and the compact table
// forms (BF16 hi/mid/lo planes, Ozaki INT8 slices with per-column
// power-of-two scales).
//
// Replaces GaussLegendreGrid's constructor (GaussLegendreGrid.h:38-73), the
// GaussQuad node computation it calls (:47-49) and Wigner::ComputeAll /
// Compute (Wigner.h:24-95, 289-486).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "gsht_internal.cuh"

namespace gsht {
namespace {

// ---------------------------------------------------------------------------
// Double-double helpers (Dekker/Knuth error-free transformations).
// ---------------------------------------------------------------------------
struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
__device__ __forceinline__ dd quick_two_sum(double a, double b) {
  double s = a + b;
  return {s, b - (s - a)};
}
__device__ __forceinline__ dd two_prod(double a, double b) {
  double p = a * b;
  return {p, fma(a, b, -p)};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  s.lo += a.lo + b.lo;
  return quick_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ dd dd_mul_d(dd a, double b) {
  dd p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ dd dd_div_d(dd a, double b) {
  double q1 = a.hi / b;
  dd p = two_prod(q1, b);
  double r = ((a.hi - p.hi) - p.lo + a.lo) / b;
  return quick_two_sum(q1, r);
}

// P_n(x), P_{n-1}(x) and P_{n-2}(x) by the three-term recurrence
// (k+1) P_{k+1} = (2k+1) x P_k - k P_{k-1}, in double-double.
__device__ void legendre_dd(int n, double x, dd* pn, dd* pnm1, dd* pnm2) {
  dd p0 = {1.0, 0.0}, p1 = {x, 0.0}, pm = {0.0, 0.0};
  for (int k = 1; k < n; k++) {
    dd t = dd_mul(two_prod(x, (double)(2 * k + 1)), p1);
    dd u = dd_mul_d(p0, (double)k);
    dd p2 = dd_div_d(dd_add(t, dd_neg(u)), (double)(k + 1));
    pm = p0;
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pnm1 = p0;
  *pnm2 = pm;
}

// One thread per node pair (x_i, x_{n-1-i} = -x_i): Newton on P_n from the
// asymptotic guess, residuals in double-double so that the iteration settles
// on the double nearest the root; theta = acos(-x) (GaussLegendreGrid.h:48).
// The weight w = 2 (1 - r^2) / (n P_{n-1}(r))^2 is taken at the root r, not
// at its double rounding x: with delta = r - x = -P_n(x)/P_n'(x) (first order,
// P_n in double-double), P_{n-1}(r) = P_{n-1}(x) + P_{n-1}'(x) delta and
// 1 - r^2 = (1 - x)(1 + x) - 2 x delta. Near the poles P_n' ~ n^2, so the
// uncorrected form would be off by ~1e-8 relative at lmax 1024.
__global__ void k_gl_nodes(int n, double* theta, double* weight) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (n + 1) / 2) return;
  double x = -cospi((i + 0.75) / (n + 0.5));
  dd pn, pnm1, pnm2;
  for (int it = 0; it < 60; it++) {
    legendre_dd(n, x, &pn, &pnm1, &pnm2);
    const double dp = n * (x * pn.hi - pnm1.hi) / (x * x - 1.0);
    const double xn = x - pn.hi / dp;
    if (xn == x) break;
    x = xn;
  }
  if (2 * i + 1 == n) x = 0.0;
  legendre_dd(n, x, &pn, &pnm1, &pnm2);
  double w = 2.0;
  if (n >= 2) {
    const double dp = n * (x * pn.hi - pnm1.hi) / (x * x - 1.0);
    const double delta = -(pn.hi + pn.lo) / dp;
    const double dq = (n - 1) * (x * pnm1.hi - pnm2.hi) / (x * x - 1.0);
    const double q = n * (pnm1.hi + (pnm1.lo + dq * delta));
    const double omr2 = (1.0 - x) * (1.0 + x) - 2.0 * x * delta;
    w = 2.0 * omr2 / (q * q);
  }
  // North node: theta = acos(-x) with -x in (0, 1]. South node: theta =
  // acos(x) = pi - acos(-x), formed with a split pi.
  const double tn = acos(-x);
  const double pi_hi = 3.141592653589793116;
  const double pi_lo = 1.2246467991473532e-16;
  dd s = two_sum(pi_hi, -tn);
  const double ts = s.hi + (s.lo + pi_lo);
  theta[i] = tn;
  theta[n - 1 - i] = ts;
  weight[i] = w;
  weight[n - 1 - i] = w;
}

// ---------------------------------------------------------------------------
// Exponent-extended numbers f * 2^e (Fukushima-style X-numbers) for the
// start values, which underflow double near the poles at high degree.
// ---------------------------------------------------------------------------
struct xnum {
  double f;
  int e;
};
__device__ __forceinline__ void xnorm(xnum& a) {
  if (a.f != 0.0 && (fabs(a.f) < 0x1p-400 || fabs(a.f) > 0x1p400)) {
    int k;
    a.f = frexp(a.f, &k);
    a.e += k;
  }
}
__device__ __forceinline__ void xmul(xnum& a, double b) {
  a.f *= b;
  xnorm(a);
}

// Start values of the l-recurrence for every order m >= 0 at colatitude
// theta_j: d^{l0}_{mn}(theta_j), l0 = max(m, |n|). For m >= |n| these are the
// boundary values d^m_{mn} (WignerMaxOrder, Wigner.h:82-85), generated by the
// exact ratio d^{m+1}_{m+1,n} / d^m_{mn} = -sqrt((2m+2)(2m+1)/((m+1+n)(m+1-n)))
// sin(theta/2) cos(theta/2) from d^{|n|}_{|n|,n}; for m < |n| they are the
// row l = |n| (WignerMax/MinUpperIndex, Wigner.h:87-95), generated downward in
// m. Products of exact ratios replace the reference's exp(lgamma ...) form,
// which loses ~|argument| ulps and underflows for L >~ 1930.
__global__ void k_wigner_start(int L, int n, int nTheta, int thetaPad,
                               const double* __restrict__ theta,
                               double* __restrict__ start_f,
                               int* __restrict__ start_e) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nTheta) return;
  const int na = n < 0 ? -n : n;
  double s, c;
  sincos(0.5 * theta[j], &s, &c);
  // d^{|n|}_{|n|,n} = c^{2n} (n >= 0) or s^{2|n|} (n < 0).
  xnum v = {1.0, 0};
  const double base = n >= 0 ? c : s;
  for (int k = 0; k < 2 * na; k++) xmul(v, base);
  auto store = [&](int m, const xnum& x) {
    const size_t o = (size_t)m * thetaPad + j;
    start_f[o] = x.f;
    start_e[o] = x.e;
  };
  store(na, v);
  xnum u = v;
  for (int m = na; m < L; m++) {
    const double r = sqrt((double)(2 * m + 2) * (double)(2 * m + 1) /
                          ((double)(m + 1 + n) * (double)(m + 1 - n)));
    xmul(u, -r * s * c);
    store(m + 1, u);
  }
  // Orders m < |n| at degree |n|, downward from m = |n|.
  u = v;
  for (int m = na; m > 0; m--) {
    const double r = sqrt((double)(na + m) / (double)(na - m + 1));
    if (n >= 0) {
      xmul(u, r * (s / c));
    } else {
      xmul(u, -r * (c / s));
    }
    store(m - 1, u);
  }
}

// Coefficients of step k = l - l0 of the l-recurrence (Wigner.h:347-472) for
// order m >= 0 and upper index n: d^l = (a cos(theta) - b) d^{l-1} - g d^{l-2}
// for k >= 1, and the normalisation of degree l (Ortho: sqrt(2l+1)/(2 sqrt(pi)),
// FourPi: 1; Wigner.h:475-485). Step 0 (the start value) has a = b = g = 0.
// Shared by the table build and the on-the-fly recurrence of the transforms.
__device__ __forceinline__ void chain_coefficients(int n, int m, int l, int k, int ortho,
                                                   double* a, double* b, double* g,
                                                   double* nrm) {
  const int na = n < 0 ? -n : n;
  *nrm = ortho ? sqrt((double)(2 * l + 1)) * 0.28209479177387814347 : 1.0;
  *a = 0.0;
  *b = 0.0;
  *g = 0.0;
  if (k == 1) {
    if (m <= na) {
      // Row |n|+1, interior orders (Wigner.h:365-373).
      const double sg = n < 0 ? -1.0 : 1.0;
      const double c0 = (2.0 * l - 1.0) * rsqrt((double)(l + na)) *
                        rsqrt((double)(l - m)) * rsqrt((double)(l + m));
      *a = c0 * l;
      *b = c0 * sg * m;
    } else {
      // One-term recursion at m = l - 1 (Wigner.h:406-413, 448-457).
      const double c0 = (2.0 * l - 1.0) * rsqrt((double)(l - n)) *
                        rsqrt((double)(l + n)) * rsqrt((double)(l - m)) *
                        rsqrt((double)(l + m)) / (double)(l - 1);
      *a = c0 * l * (l - 1.0);
      *b = c0 * (double)m * (double)n;
    }
  } else if (k >= 2) {
    // Two-term recursion (Wigner.h:428-445).
    const double inl = rsqrt((double)(l - n)) * rsqrt((double)(l + n));
    const double dn = rsqrt((double)(l - m)) * rsqrt((double)(l + m));
    *a = (2.0 * l - 1.0) * l * inl * dn;
    *b = (2.0 * l - 1.0) * n * inl / (l - 1.0) * m * dn;
    *g = l * sqrt((double)(l - 1 - n)) * sqrt((double)(l - 1 + n)) * inl / (l - 1.0) *
         sqrt((double)(l - 1 - m)) * sqrt((double)(l - 1 + m)) * dn;
  }
}

// The l-recurrence (Wigner.h:347-472) for one order m per block (blockIdx.y)
// and one colatitude per thread. Per-degree coefficients are computed once per
// block into shared memory; the chain runs in exponent-extended form until its
// values enter the normal double range. Values are written Ortho-normalised
// (factor sqrt(2l+1)/(2 sqrt(pi)), Wigner.h:475-485).
__global__ void __launch_bounds__(128) k_wigner_chain(
    int L, int n, int nTheta, int thetaPad, int ortho, const double* __restrict__ theta,
    const double* __restrict__ start_f, const int* __restrict__ start_e,
    const long long* __restrict__ row_off, double* __restrict__ table) {
  extern __shared__ double sh[];
  const int m = (int)blockIdx.y;
  const int na = n < 0 ? -n : n;
  const int l0 = m > na ? m : na;
  const int K = L - l0 + 1;
  double* a = sh;          // f1 = a_l cos(theta) - b_l
  double* b = sh + K;
  double* g = sh + 2 * K;  // f2
  double* nrm = sh + 3 * K;
  for (int k = threadIdx.x; k < K; k += blockDim.x)
    chain_coefficients(n, m, l0 + k, k, ortho, &a[k], &b[k], &g[k], &nrm[k]);
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= thetaPad) return;
  double* out = table + (size_t)row_off[m] * thetaPad + j;
  if (j >= nTheta) {
    for (int k = 0; k < K; k++) out[(size_t)k * thetaPad] = 0.0;
    return;
  }
  const double cs = cos(theta[j]);
  // Exponent-extended chain: value = p * 2^E with E a multiple of 512.
  int ef = 0;
  const double f0 = frexp(start_f[(size_t)m * thetaPad + j], &ef);  // [0.5, 1)
  const int e0 = start_e[(size_t)m * thetaPad + j] + ef;  // value = f0 2^e0
  int E = 0;
  if (f0 != 0.0 && e0 < -900) E = -512 * ((-900 - e0 + 511) / 512);
  double p1 = ldexp(f0, e0 - E), p2 = 0.0;
  auto emit = [&](int k, double p) {
    const double v = (E == 0) ? p : ldexp(p, E);
    out[(size_t)k * thetaPad] = v * nrm[k];
  };
  emit(0, p1);
  for (int k = 1; k < K; k++) {
    const double p = (a[k] * cs - b[k]) * p1 - g[k] * p2;
    p2 = p1;
    p1 = p;
    if (E < 0 && fabs(p1) >= 0x1p-100) {
      p1 = ldexp(p1, -512);
      p2 = ldexp(p2, -512);
      E += 512;
    }
    emit(k, p1);
  }
}

// BF16 hi/mid/lo planes: x = hi + mid + lo + O(2^-24 |x|).
__global__ void k_split_bf16(size_t count, const double* __restrict__ t64,
                             __nv_bfloat16* __restrict__ tbf,
                             size_t plane) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    const double x = t64[i];
    const __nv_bfloat16 h = __double2bfloat16(x);
    const double r1 = x - (double)__bfloat162float(h);
    const __nv_bfloat16 md = __double2bfloat16(r1);
    const double r2 = r1 - (double)__bfloat162float(md);
    tbf[i] = h;
    tbf[plane + i] = md;
    tbf[2 * plane + i] = __double2bfloat16(r2);
  }
}

// Ozaki slices per (m, theta_j) column: sigma = 2^e with max_l |d| < sigma,
// d / sigma = sum_s S_s 2^{-7 s}, S_s in [-127, 127] by truncation (each
// residual keeps the sign of the value, so no slice overflows).
__global__ void k_slice_i8(int L, int n, int thetaPad,
                           const long long* __restrict__ row_off,
                           const double* __restrict__ t64,
                           int8_t* __restrict__ ti8, size_t plane,
                           int* __restrict__ col_exp) {
  const int m = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= thetaPad) return;
  const int na = n < 0 ? -n : n;
  const int l0 = m > na ? m : na;
  const int K = L - l0 + 1;
  const size_t base = (size_t)row_off[m] * thetaPad + j;
  double mx = 0.0;
  for (int k = 0; k < K; k++) mx = fmax(mx, fabs(t64[base + (size_t)k * thetaPad]));
  int e = 0;
  if (mx > 0.0) {
    frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1) => mx < 2^e
  }
  col_exp[(size_t)m * thetaPad + j] = e;
  for (int k = 0; k < K; k++) {
    double y = ldexp(t64[base + (size_t)k * thetaPad], -e);  // |y| < 1
    for (int s = 0; s < kTableSlices; s++) {
      y *= 128.0;
      const double q = trunc(y);
      y -= q;
      ti8[s * plane + base + (size_t)k * thetaPad] = (int8_t)q;
    }
  }
}

// Column j of the FP64 table, one value per row (the rows of order m at
// row_off[m]..).
__global__ void k_table_column(long long rows, int thetaPad, int j, const double* __restrict__ t64,
                               double* __restrict__ col) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < rows) col[r] = t64[(size_t)r * thetaPad + j];
}

}  // namespace

gsht_status build_nodes(gsht_grid* g) {
  const int nt = g->n_theta;
  GSHT_CUDA(dev_malloc(&g->d_theta, sizeof(double) * g->theta_pad));
  GSHT_CUDA(dev_malloc(&g->d_weight, sizeof(double) * g->theta_pad));
  GSHT_CUDA(cudaMemset(g->d_theta, 0, sizeof(double) * g->theta_pad));
  GSHT_CUDA(cudaMemset(g->d_weight, 0, sizeof(double) * g->theta_pad));
  const int pairs = (nt + 1) / 2;
  k_gl_nodes<<<(pairs + 127) / 128, 128>>>(nt, g->d_theta, g->d_weight);
  GSHT_LAUNCH_CHECK("k_gl_nodes");
  g->h_theta.resize(nt);
  g->h_weight.resize(nt);
  GSHT_CUDA(cudaMemcpy(g->h_theta.data(), g->d_theta, sizeof(double) * nt,
                       cudaMemcpyDeviceToHost));
  GSHT_CUDA(cudaMemcpy(g->h_weight.data(), g->d_weight, sizeof(double) * nt,
                       cudaMemcpyDeviceToHost));
  return GSHT_OK;
}

// Table of upper index t->n for orders 0..L at nTheta colatitudes (device
// array theta, pitch thetaPad), in the layout described in gsht_internal.cuh.
static gsht_status compute_table(int L, int nTheta, int thetaPad, const double* d_theta,
                                 int ortho, Table* t, cudaStream_t s) {
  const int tp = thetaPad, na = t->n < 0 ? -t->n : t->n;
  t->row_off.assign(L + 2, 0);
  for (int m = 0; m <= L; m++) {
    const int l0 = m > na ? m : na;
    t->row_off[m + 1] = t->row_off[m] + (L - l0 + 1);
  }
  t->rows = t->row_off[L + 1];
  GSHT_CUDA(dev_malloc(&t->d_row_off, sizeof(long long) * (L + 2)));
  GSHT_CUDA(cudaMemcpy(t->d_row_off, t->row_off.data(),
                       sizeof(long long) * (L + 2), cudaMemcpyHostToDevice));
  const size_t elems = (size_t)(t->rows + kTablePadRows) * tp;
  if (dev_malloc(&t->t64, sizeof(double) * elems) != cudaSuccess) {
    cudaGetLastError();
    return fail(GSHT_ERR_OOM, "table allocation of %zu bytes failed",
                sizeof(double) * elems);
  }
  GSHT_CUDA(cudaMemsetAsync(t->t64, 0, sizeof(double) * elems, s));
  ScopedDev<double> start_f;
  ScopedDev<int> start_e;
  GSHT_CUDA(dev_malloc(&start_f.p, sizeof(double) * (size_t)(L + 1) * tp));
  GSHT_CUDA(dev_malloc(&start_e.p, sizeof(int) * (size_t)(L + 1) * tp));
  k_wigner_start<<<(nTheta + 127) / 128, 128, 0, s>>>(L, t->n, nTheta, tp, d_theta, start_f.p,
                                                      start_e.p);
  GSHT_LAUNCH_CHECK("k_wigner_start");
  const size_t shmem = sizeof(double) * 4 * (L + 1);
  if (shmem > 48 * 1024) {
    GSHT_CUDA(cudaFuncSetAttribute(k_wigner_chain,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)shmem));
  }
  dim3 grid((tp + 127) / 128, L + 1);
  k_wigner_chain<<<grid, 128, shmem, s>>>(L, t->n, nTheta, tp, ortho, d_theta, start_f.p,
                                          start_e.p, t->d_row_off, t->t64);
  GSHT_LAUNCH_CHECK("k_wigner_chain");
  GSHT_CUDA(cudaStreamSynchronize(s));
  return GSHT_OK;
}

gsht_status build_table(gsht_grid* g, Table* t, cudaStream_t s) {
  return compute_table(g->L, g->n_theta, g->theta_pad, g->d_theta, 1, t, s);
}

// Recurrence-form coefficients per table row (m, k). The recurrence
// d_k = (a_k c - b_k) d_{k-1} - g_k d_{k-2} (c = cos theta) is carried for
// e_k = d_k / s_k with s_0 = s_1 = 1, s_k = g_k s_{k-2}, which turns it into
// e_k = (a'_k c - b'_k) e_{k-1} - e_{k-2}, a'_k = a_k s_{k-1} / s_k (same for
// b): two FMAs per step instead of three. Stored: (a'_k, b'_k) and the
// factor sc_k = norm_k s_k that turns e_k into the normalised value; step 0 is
// (a', b') = (0, -1), so that with the initial state e_{-1} = 0, e_{-2} =
// -d_0 every step runs the same update. One thread per order m (the s_k are a
// running product over k).
__global__ void k_rec_coefficients(int L, int n, int ortho, const long long* __restrict__ row_off,
                                   double2* __restrict__ ab, double* __restrict__ sc) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > L) return;
  const int na = n < 0 ? -n : n;
  const int l0 = m > na ? m : na;
  const int K = L - l0 + 1;
  const size_t r0 = (size_t)row_off[m];
  double s1 = 1.0, s2 = 1.0;  // s_{k-1}, s_{k-2}
  for (int k = 0; k < K; k++) {
    double a, b, g, nrm;
    chain_coefficients(n, m, l0 + k, k, ortho, &a, &b, &g, &nrm);
    double sk = 1.0;
    if (k == 0) {
      a = 0.0;
      b = -1.0;
    } else if (k >= 2) {
      sk = g * s2;
      const double r = s1 / sk;
      a *= r;
      b *= r;
    }
    ab[r0 + k] = make_double2(a, b);
    sc[r0 + k] = nrm * sk;
    s2 = s1;
    s1 = sk;
  }
}

gsht_status build_recurrence(gsht_grid* g, Table* t, cudaStream_t s) {
  const int L = g->L, tp = g->theta_pad, na = t->n < 0 ? -t->n : t->n;
  if (!t->d_row_off) {
    t->row_off.assign(L + 2, 0);
    for (int m = 0; m <= L; m++) {
      const int l0 = m > na ? m : na;
      t->row_off[m + 1] = t->row_off[m] + (L - l0 + 1);
    }
    t->rows = t->row_off[L + 1];
    GSHT_CUDA(dev_malloc(&t->d_row_off, sizeof(long long) * (L + 2)));
    GSHT_CUDA(cudaMemcpy(t->d_row_off, t->row_off.data(), sizeof(long long) * (L + 2),
                         cudaMemcpyHostToDevice));
  }
  if (dev_malloc(&t->rec_f, sizeof(double) * (size_t)(L + 1) * tp) != cudaSuccess ||
      dev_malloc(&t->rec_e, sizeof(int) * (size_t)(L + 1) * tp) != cudaSuccess ||
      dev_malloc(&t->rec_ab, sizeof(double2) * (size_t)t->rows) != cudaSuccess ||
      dev_malloc(&t->rec_sc, sizeof(double) * (size_t)t->rows) != cudaSuccess) {
    cudaGetLastError();
    return fail(GSHT_ERR_OOM, "recurrence form allocation failed");
  }
  k_wigner_start<<<(g->n_theta + 127) / 128, 128, 0, s>>>(L, t->n, g->n_theta, tp, g->d_theta,
                                                          t->rec_f, t->rec_e);
  GSHT_LAUNCH_CHECK("k_wigner_start");
  k_rec_coefficients<<<(L + 1 + 127) / 128, 128, 0, s>>>(L, t->n, 1, t->d_row_off, t->rec_ab,
                                                          t->rec_sc);
  GSHT_LAUNCH_CHECK("k_rec_coefficients");
  GSHT_CUDA(cudaStreamSynchronize(s));
  return GSHT_OK;
}

gsht_status build_forms(gsht_grid* g, Table* t, cudaStream_t s) {
  const int L = g->L, tp = g->theta_pad;
  const size_t plane = (size_t)(t->rows + kTablePadRows) * tp;
  if (g->forms & GSHT_FORM_BF16X3) {
    if (dev_malloc(&t->tbf, sizeof(__nv_bfloat16) * 3 * plane) != cudaSuccess) {
      cudaGetLastError();
      return fail(GSHT_ERR_OOM, "BF16 table allocation failed");
    }
    GSHT_CUDA(cudaMemsetAsync(t->tbf, 0, sizeof(__nv_bfloat16) * 3 * plane, s));
    k_split_bf16<<<148 * 8, 256, 0, s>>>((size_t)t->rows * tp, t->t64, t->tbf,
                                         plane);
    GSHT_LAUNCH_CHECK("k_split_bf16");
  }
  if (g->forms & GSHT_FORM_OZAKI) {
    if (dev_malloc(&t->ti8, (size_t)kTableSlices * plane) != cudaSuccess) {
      cudaGetLastError();
      return fail(GSHT_ERR_OOM, "INT8 slice allocation failed");
    }
    GSHT_CUDA(cudaMemsetAsync(t->ti8, 0, (size_t)kTableSlices * plane, s));
    GSHT_CUDA(dev_malloc(&t->i8_exp, sizeof(int) * (size_t)(L + 1) * tp));
    dim3 grid((tp + 127) / 128, L + 1);
    k_slice_i8<<<grid, 128, 0, s>>>(L, t->n, tp, t->d_row_off, t->t64, t->ti8,
                                    plane, t->i8_exp);
    GSHT_LAUNCH_CHECK("k_slice_i8");
    if (g->n_theta % 128 == 1) {
      if (dev_malloc(&t->tail64, sizeof(double) * (size_t)t->rows) != cudaSuccess) {
        cudaGetLastError();
        return fail(GSHT_ERR_OOM, "table column allocation failed");
      }
      k_table_column<<<(unsigned)((t->rows + 255) / 256), 256, 0, s>>>(t->rows, tp,
                                                                       g->n_theta - 1, t->t64,
                                                                       t->tail64);
      GSHT_LAUNCH_CHECK("k_table_column");
    }
  }
  GSHT_CUDA(cudaStreamSynchronize(s));
  return GSHT_OK;
}

gsht_status wigner_compute(int lmax, int mmax, int nmax, int mrange, int nrange, int norm,
                           int row_major, const double* theta, int ntheta, double* out,
                           long* count) {
  const bool allM = mrange == GSHT_RANGE_ALL;
  const int nmin = nrange == GSHT_RANGE_ALL ? -nmax : (nrange == GSHT_RANGE_NONNEGATIVE ? 0 : nmax);
  const int mm = mmax < lmax ? mmax : lmax;
  // Block size of GSHIndices<MRange>(lmax, mmax, n) (Indexing.h:104-131).
  auto block = [&](int n) {
    const long na = n < 0 ? -n : n;
    long size = 0;
    for (long l = na; l <= lmax; l++) {
      const long ml = l < mm ? l : mm;
      size += allM ? 2 * ml + 1 : ml + 1;
    }
    return size;
  };
  long total = 0;
  for (int n = nmin; n <= nmax; n++) total += block(n) * ntheta;
  if (count) *count = total;
  if (!out) return GSHT_OK;
  const int tp = (int)round_up(ntheta, kThetaPad);
  ScopedDev<double> dTheta;
  GSHT_CUDA(dev_malloc(&dTheta.p, sizeof(double) * tp));
  double* d_theta = dTheta.p;
  GSHT_CUDA(cudaMemset(d_theta, 0, sizeof(double) * tp));
  GSHT_CUDA(cudaMemcpy(d_theta, theta, sizeof(double) * ntheta, cudaMemcpyHostToDevice));
  // Negative orders at n come from the table of -n: d^l_{-m,n} = (-1)^{m+n} d^l_{m,-n}.
  std::vector<std::vector<double>> host(2 * nmax + 1);
  std::vector<Table> tabs(2 * nmax + 1);
  gsht_status st = GSHT_OK;
  auto need = [&](int n) { return n >= nmin || (allM && -n >= nmin); };
  for (int n = -nmax; n <= nmax && st == GSHT_OK; n++) {
    if (!need(n)) continue;
    Table* t = &tabs[n + nmax];
    t->n = n;
    st = compute_table(lmax, ntheta, tp, d_theta, norm == 0 ? 1 : 0, t, nullptr);
    if (st != GSHT_OK) break;
    host[n + nmax].resize((size_t)t->rows * tp);
    if (cudaMemcpy(host[n + nmax].data(), t->t64, sizeof(double) * host[n + nmax].size(),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      st = cuda_fail(cudaGetLastError(), "wigner table download");
  }
  if (st == GSHT_OK) {
    const int nn = nmax - nmin + 1;
    long off = 0;
    for (int bi = 0; bi < nn * ntheta; bi++) {
      // ColumnMajor: n outer, angle inner; RowMajor: angle outer, n inner.
      const int n = row_major ? nmin + bi % nn : nmin + bi / ntheta;
      const int it = row_major ? bi / nn : bi % ntheta;
      const int na = n < 0 ? -n : n;
      for (int l = na; l <= lmax; l++) {
        const int ml = l < mm ? l : mm;
        for (int m = allM ? -ml : 0; m <= ml; m++) {
          const int am = m < 0 ? -m : m;
          const int nsrc = m >= 0 ? n : -n;
          const Table& t = tabs[nsrc + nmax];
          const int nsa = nsrc < 0 ? -nsrc : nsrc;
          const int l0 = am > nsa ? am : nsa;
          double v = host[nsrc + nmax][(size_t)(t.row_off[am] + (l - l0)) * tp + it];
          if (m < 0 && ((am + n) & 1)) v = -v;
          out[off++] = v;
        }
      }
    }
  }
  for (auto& t : tabs) free_table(&t);
  return st;
}

void free_table(Table* t) {
  dev_free(t->d_row_off);
  dev_free(t->t64);
  dev_free(t->tbf);
  dev_free(t->ti8);
  dev_free(t->i8_exp);
  dev_free(t->tail64);
  dev_free(t->rec_f);
  dev_free(t->rec_e);
  dev_free(t->rec_ab);
  dev_free(t->rec_sc);
  *t = Table{};
}

}  // namespace gsht

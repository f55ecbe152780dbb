// Longitudinal (ring) FFT stage, fused with the order-major reordering.
//
// Replaces the per-ring FFTWpp plans of GaussLegendreGrid.h:148-174 (forward:
// c2c Forward or r2c) and :266-320 (inverse: c2c Backward or c2r), including
// the bin <-> order map (m >= 0 -> bin m, m < 0 -> bin nPhi + m, :189-206 and
// :294-311) and, for the forward direction, the quadrature factor
// w_j * 2 pi / nPhi (:177-178) folded into the spectrum.
//
// Spectral buffer layout (shared with the Legendre stage):
//   spec[((m * SGN + sgn) * count + f) * thetaPad + j]  (complex double)
// for orders m = 0..lmax, sgn 0 for +m and 1 for -m (SGN = 2 for complex
// fields, 1 for real ones). Entries of -m are stored at the mirrored
// colatitude index nTheta-1-theta, which lets the Legendre stage contract +m
// and -m against the same table columns (d^l_{-m,n}(pi - theta) =
// (-1)^{l+n} d^l_{mn}(theta)).
//
// One thread block transforms one ring entirely in shared memory with a
// self-sorting (Stockham) mixed-radix FFT: radix-4 and radix-2 butterflies,
// plus a generic radix-p DFT for odd factors, so every even nPhi works.
// Real fields use the half-length complex FFT with the standard pre/post
// twiddle (pack even/odd samples as real/imaginary parts).
#include <cstring>
#include <type_traits>

#include <cstdlib>

#include "gsht_internal.cuh"
#include "tc_common.cuh"

namespace gsht {
namespace {

constexpr int kMaxStages = 40;

struct FftPlan {
  int n;                    // transform length
  int tw_stride;            // twiddle table index step: table length / n
  int stages;
  int radix[kMaxStages];
};

FftPlan make_plan(int n, int tableLen) {
  FftPlan p{};
  p.n = n;
  p.tw_stride = tableLen / n;
  int m = n, s = 0;
  while (m % 4 == 0) { p.radix[s++] = 4; m /= 4; }
  while (m % 2 == 0) { p.radix[s++] = 2; m /= 2; }
  for (int q = 3; m > 1; q += 2) {
    while (m % q == 0) { p.radix[s++] = q; m /= q; }
  }
  p.stages = s;
  return p;
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
// Spectral buffer elements: FP64 (double2) or FP32 (float2) complex.
template <typename T>
__device__ __forceinline__ T from_d2(double2 v);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// Multiply by sign * i.
__device__ __forceinline__ double2 cmul_si(double2 a, int sign) {
  return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// exp(sign 2 pi i t / n) from the table exp(-2 pi i u / tableLen).
__device__ __forceinline__ double2 twiddle(const double2* __restrict__ tw, int t,
                                           int stride, int sign) {
  double2 w = __ldg(tw + (size_t)t * stride);
  return sign < 0 ? w : cconj(w);
}

// FP32 complex arithmetic of the FP32-spectrum path (the three-pass kernels
// with float2 spectra run their butterflies in FP32: the BF16x3 form they
// serve keeps ~1e-6, and FP32 halves the shared-memory bytes per point and
// runs on the FP32 pipe).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cmul_si(float2 a, int sign) {
  return sign > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
__device__ __forceinline__ float2 twiddle(const float2* __restrict__ tw, int t, int stride,
                                          int sign) {
  float2 w = __ldg(tw + (size_t)t * stride);
  return sign < 0 ? w : cconj(w);
}
// Complex value of compute type C from a stored one.
template <typename C>
__device__ __forceinline__ C to_c(double2 v);
template <>
__device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 to_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <typename C>
__device__ __forceinline__ C to_c(float2 v);
template <>
__device__ __forceinline__ double2 to_c<double2>(float2 v) { return make_double2(v.x, v.y); }
template <>
__device__ __forceinline__ float2 to_c<float2>(float2 v) { return v; }

// Stockham FFT of length plan.n on buffer a (scratch b); returns the buffer
// holding the result. All threads of the block must call it.
__device__ double2* fft_block(double2* a, double2* b, const FftPlan& plan,
                              const double2* __restrict__ tw, int sign) {
  const int n = plan.n;
  int l = n, m = 1;
  double2* src = a;
  double2* dst = b;
  for (int s = 0; s < plan.stages; s++) {
    const int p = plan.radix[s];
    l /= p;
    const int nb = n / p;
    if (p == 4) {
      for (int idx = threadIdx.x; idx < nb; idx += blockDim.x) {
        const int j = idx / m, k = idx - j * m;
        const int base = k + j * m;
        const double2 c0 = src[base], c1 = src[base + l * m];
        const double2 c2 = src[base + 2 * l * m], c3 = src[base + 3 * l * m];
        const double2 s02 = cadd(c0, c2), d02 = csub(c0, c2);
        const double2 s13 = cadd(c1, c3), d13 = cmul_si(csub(c1, c3), sign);
        const int o = k + 4 * j * m;
        dst[o] = cadd(s02, s13);
        const int t = j * m;
        dst[o + m] = t ? cmul(cadd(d02, d13), twiddle(tw, t, plan.tw_stride, sign)) : cadd(d02, d13);
        dst[o + 2 * m] = t ? cmul(csub(s02, s13), twiddle(tw, 2 * t, plan.tw_stride, sign)) : csub(s02, s13);
        dst[o + 3 * m] = t ? cmul(csub(d02, d13), twiddle(tw, 3 * t, plan.tw_stride, sign)) : csub(d02, d13);
      }
    } else if (p == 2) {
      for (int idx = threadIdx.x; idx < nb; idx += blockDim.x) {
        const int j = idx / m, k = idx - j * m;
        const int base = k + j * m;
        const double2 c0 = src[base], c1 = src[base + l * m];
        const int o = k + 2 * j * m;
        dst[o] = cadd(c0, c1);
        const int t = j * m;
        dst[o + m] = t ? cmul(csub(c0, c1), twiddle(tw, t, plan.tw_stride, sign)) : csub(c0, c1);
      }
    } else {
      const int np = n / p;
      for (int idx = threadIdx.x; idx < nb; idx += blockDim.x) {
        const int j = idx / m, k = idx - j * m;
        const int base = k + j * m;
        const int o = k + p * j * m;
        for (int r = 0; r < p; r++) {
          double2 acc = src[base];
          for (int q = 1; q < p; q++) {
            const int t = (q * r * np) % n;
            acc = cadd(acc, cmul(src[base + q * l * m], twiddle(tw, t, plan.tw_stride, sign)));
          }
          const int t = (j * r * m) % n;
          dst[o + r * m] = t ? cmul(acc, twiddle(tw, t, plan.tw_stride, sign)) : acc;
        }
      }
    }
    m *= p;
    double2* tmp = src;
    src = dst;
    dst = tmp;
    __syncthreads();
  }
  return src;
}

// Inverse: spectrum -> ring values. Block (j, f).
template <bool kReal>
__global__ void __launch_bounds__(256) k_fft_inverse(
    FftPlan plan, int L, int lmax, int nTheta, int thetaPad, int count,
    const double2* __restrict__ spec, const double2* __restrict__ tw,
    double* __restrict__ out, RingRange rr) {
  extern __shared__ double2 smem[];
  const int j = blockIdx.x + rr.jBegin, f = blockIdx.y;
  const int nPhi = 2 * L;
  const int sgnCount = kReal ? 1 : 2;
  double2* a = smem;
  double2* b = smem + plan.n;
  auto S = [&](int m, int sgn, int jj) {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  if (!kReal) {
    const int jm = nTheta - 1 - j;
    for (int bin = threadIdx.x; bin < nPhi; bin += blockDim.x) {
      double2 x = make_double2(0.0, 0.0);
      if (bin <= lmax) x = S(bin, 0, j);
      if (bin >= nPhi - lmax) x = cadd(x, S(nPhi - bin, 1, jm));
      a[bin] = x;
    }
    __syncthreads();
    const double2* r = fft_block(a, b, plan, tw, +1);
    double2* o = reinterpret_cast<double2*>(rr.grid(out, f, 2 * (size_t)nTheta * nPhi)) + (size_t)j * nPhi;
    for (int k = threadIdx.x; k < nPhi; k += blockDim.x) o[k] = r[k];
  } else {
    // Bins X[0..M], M = L (Nyquist); imaginary parts of X[0], X[M] dropped.
    const int M = L;
    for (int bin = threadIdx.x; bin < M; bin += blockDim.x) {
      const int bc = M - bin;
      double2 x0 = bin <= lmax ? S(bin, 0, j) : make_double2(0.0, 0.0);
      double2 x1 = bc <= lmax ? S(bc, 0, j) : make_double2(0.0, 0.0);
      if (bin == 0) x0.y = 0.0;
      if (bc == M) x1.y = 0.0;
      // Z[b] = (X[b] + conj X[M-b]) + i w^b (X[b] - conj X[M-b]), w = e^{+2 pi i/N}
      const double2 xc = cconj(x1);
      const double2 w = twiddle(tw, bin, 1, +1);
      a[bin] = cadd(cadd(x0, xc), cmul_si(cmul(w, csub(x0, xc)), +1));
    }
    __syncthreads();
    const double2* r = fft_block(a, b, plan, tw, +1);
    double2* o = reinterpret_cast<double2*>(rr.grid(out, f, (size_t)nTheta * nPhi) + (size_t)j * nPhi);
    for (int k = threadIdx.x; k < M; k += blockDim.x) o[k] = r[k];
  }
}

// Forward: ring values -> weighted spectrum. Block (j, f).
template <bool kReal>
__global__ void __launch_bounds__(256) k_fft_forward(
    FftPlan plan, int L, int lmax, int nTheta, int thetaPad, int count,
    const double* __restrict__ in, const double* __restrict__ weight,
    const double2* __restrict__ tw, double2* __restrict__ spec, RingRange rr) {
  extern __shared__ double2 smem[];
  const int j = blockIdx.x + rr.jBegin, f = blockIdx.y;
  const int nPhi = 2 * L;
  const int sgnCount = kReal ? 1 : 2;
  double2* a = smem;
  double2* b = smem + plan.n;
  const double scale = weight[j] * (6.283185307179586477 / nPhi);
  auto S = [&](int m, int sgn, int jj) -> double2& {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  if (j == nTheta - 1) {
    // The colatitude padding [nTheta, thetaPad) is part of the contraction
    // length of the forward Legendre stage and must hold zeros.
    const int padW = thetaPad - nTheta;
    for (int i = threadIdx.x; i < (lmax + 1) * sgnCount * padW; i += blockDim.x) {
      const int q = i / padW, jj = nTheta + (i - q * padW);
      S(q / sgnCount, q % sgnCount, jj) = make_double2(0.0, 0.0);
    }
  }
  if (!kReal) {
    const double2* x = reinterpret_cast<const double2*>(rr.grid(in, f, 2 * (size_t)nTheta * nPhi)) + (size_t)j * nPhi;
    for (int k = threadIdx.x; k < nPhi; k += blockDim.x) a[k] = x[k];
    __syncthreads();
    const double2* r = fft_block(a, b, plan, tw, -1);
    const int jm = nTheta - 1 - j;
    for (int m = threadIdx.x; m <= lmax; m += blockDim.x) {
      S(m, 0, j) = cscale(r[m], scale);
      S(m, 1, jm) = m ? cscale(r[nPhi - m], scale) : make_double2(0.0, 0.0);
    }
  } else {
    const int M = L;
    const double2* x = reinterpret_cast<const double2*>(rr.grid(in, f, (size_t)nTheta * nPhi) + (size_t)j * nPhi);
    for (int k = threadIdx.x; k < M; k += blockDim.x) a[k] = x[k];
    __syncthreads();
    const double2* r = fft_block(a, b, plan, tw, -1);
    // X[b] = (Z[b] + conj Z[M-b])/2 - (i/2) w^b (Z[b] - conj Z[M-b]),
    // w = e^{-2 pi i/N}, Z[M] = Z[0].
    for (int m = threadIdx.x; m <= lmax; m += blockDim.x) {
      const double2 z0 = r[m == M ? 0 : m];
      const double2 zc = cconj(r[m == 0 ? 0 : M - m]);
      const double2 w = twiddle(tw, m, 1, -1);
      const double2 e = cscale(cadd(z0, zc), 0.5);
      const double2 od = cscale(cmul_si(csub(z0, zc), -1), 0.5);
      S(m, 0, j) = cscale(cadd(e, cmul(w, od)), scale);
    }
  }
}

// ---------------------------------------------------------------------------
// Register-staged path: R rings per block, every thread owns kVPT points;
// each Stockham stage loads its butterflies' inputs into registers, syncs,
// and writes the outputs back in place (one buffer of R*n points). Radices
// 8, 4, 2 and 3; lengths whose factorisation has other primes use the
// generic path above.
// ---------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ void dft_reg(double2 (&c)[P], int sign);

template <>
__device__ __forceinline__ void dft_reg<2>(double2 (&c)[2], int) {
  const double2 a = cadd(c[0], c[1]), b = csub(c[0], c[1]);
  c[0] = a;
  c[1] = b;
}

template <>
__device__ __forceinline__ void dft_reg<4>(double2 (&c)[4], int sign) {
  const double2 s02 = cadd(c[0], c[2]), d02 = csub(c[0], c[2]);
  const double2 s13 = cadd(c[1], c[3]), d13 = cmul_si(csub(c[1], c[3]), sign);
  c[0] = cadd(s02, s13);
  c[1] = cadd(d02, d13);
  c[2] = csub(s02, s13);
  c[3] = csub(d02, d13);
}

template <>
__device__ __forceinline__ void dft_reg<8>(double2 (&c)[8], int sign) {
  double2 e[4] = {c[0], c[2], c[4], c[6]};
  double2 o[4] = {c[1], c[3], c[5], c[7]};
  dft_reg<4>(e, sign);
  dft_reg<4>(o, sign);
  const double h = 0.70710678118654752440;  // 1/sqrt(2)
  const double sg = (double)sign;
  // o[r] *= exp(sign 2 pi i r / 8), r = 1..3
  o[1] = make_double2(h * (o[1].x - sg * o[1].y), h * (o[1].y + sg * o[1].x));
  o[2] = cmul_si(o[2], sign);
  o[3] = make_double2(h * (-o[3].x - sg * o[3].y), h * (-o[3].y + sg * o[3].x));
#pragma unroll
  for (int r = 0; r < 4; r++) {
    c[r] = cadd(e[r], o[r]);
    c[r + 4] = csub(e[r], o[r]);
  }
}

// 16 = 4 x 4: DFT4 over n1 of x[4 n1 + n2] for each n2, twiddle
// W16^(n2 k1), DFT4 over n2; output k = k1 + 4 k2.
template <>
__device__ __forceinline__ void dft_reg<16>(double2 (&c)[16], int sign) {
  const double sg = (double)sign;
  const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;  // cos, sin(pi/8)
  const double h = 0.70710678118654752440;
  double2 a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    double2 t[4] = {c[n2], c[4 + n2], c[8 + n2], c[12 + n2]};
    dft_reg<4>(t, sign);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) a[n2][k1] = t[k1];
  }
  // W16^e = (cos(2 pi e / 16), sign sin(2 pi e / 16)) for e = n2 k1.
  a[1][1] = cmul(a[1][1], make_double2(c1, sg * s1));
  a[1][2] = cmul(a[1][2], make_double2(h, sg * h));
  a[1][3] = cmul(a[1][3], make_double2(s1, sg * c1));
  a[2][1] = cmul(a[2][1], make_double2(h, sg * h));
  a[2][2] = cmul_si(a[2][2], sign);
  a[2][3] = cmul(a[2][3], make_double2(-h, sg * h));
  a[3][1] = cmul(a[3][1], make_double2(s1, sg * c1));
  a[3][2] = cmul(a[3][2], make_double2(-h, sg * h));
  a[3][3] = cmul(a[3][3], make_double2(-c1, -sg * s1));
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    double2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    dft_reg<4>(t, sign);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) c[k1 + 4 * k2] = t[k2];
  }
}

template <>
__device__ __forceinline__ void dft_reg<3>(double2 (&c)[3], int sign) {
  const double s3 = 0.86602540378443864676;  // sqrt(3)/2
  const double2 t = cadd(c[1], c[2]);
  const double2 u = cmul_si(csub(c[1], c[2]), sign);
  const double2 x0 = cadd(c[0], t);
  const double2 b = make_double2(c[0].x - 0.5 * t.x, c[0].y - 0.5 * t.y);
  c[0] = x0;
  c[1] = make_double2(b.x + s3 * u.x, b.y + s3 * u.y);
  c[2] = make_double2(b.x - s3 * u.x, b.y - s3 * u.y);
}

// Shared-memory index of point u in the register path: one 16-byte pad per
// 8 points, so that the strided accesses of early Stockham stages (lane
// stride 8 points) hit distinct bank groups.
__device__ __forceinline__ int pad8(int u) { return u + (u >> 3); }

template <int P, int NB>
__device__ __forceinline__ void reg_stage(double2* buf, int n, int l, int m,
                                          const double2* __restrict__ tw, int twStride,
                                          int sign) {
  const int nbr = n / P;
  double2 v[NB][P];
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int idx = threadIdx.x + b * 256;
    const int ring = idx / nbr, bi = idx - ring * nbr;
    const int j = bi / m, k = bi - j * m;
    const int src = ring * n + k + j * m;
#pragma unroll
    for (int q = 0; q < P; q++) v[b][q] = buf[pad8(src + q * l * m)];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int idx = threadIdx.x + b * 256;
    const int ring = idx / nbr, bi = idx - ring * nbr;
    const int j = bi / m, k = bi - j * m;
    dft_reg<P>(v[b], sign);
    const int t = j * m;
    if (t) {
#pragma unroll
      for (int r = 1; r < P; r++) v[b][r] = cmul(v[b][r], twiddle(tw, t * r, twStride, sign));
    }
    const int dst = ring * n + k + j * P * m;
#pragma unroll
    for (int r = 0; r < P; r++) buf[pad8(dst + r * m)] = v[b][r];
  }
  __syncthreads();
}

template <int kVPT>
__device__ void fft_reg(double2* buf, const FftPlan& plan, const double2* __restrict__ tw,
                        int sign) {
  const int n = plan.n;
  int l = n, m = 1;
  for (int s = 0; s < plan.stages; s++) {
    const int p = plan.radix[s];
    l /= p;
    if (p == 8) {
      if constexpr (kVPT % 8 == 0) reg_stage<8, kVPT / 8>(buf, n, l, m, tw, plan.tw_stride, sign);
    } else if (p == 4) {
      reg_stage<4, kVPT / 4>(buf, n, l, m, tw, plan.tw_stride, sign);
    } else if (p == 2) {
      reg_stage<2, kVPT / 2>(buf, n, l, m, tw, plan.tw_stride, sign);
    } else {
      if constexpr (kVPT % 3 == 0) reg_stage<3, kVPT / 3>(buf, n, l, m, tw, plan.tw_stride, sign);
    }
    m *= p;
  }
}

// Inverse, R rings per block: block (ring group, field).
template <bool kReal, int kVPT>
__global__ void __launch_bounds__(256) k_fft_inverse_reg(
    FftPlan plan, int R, int L, int lmax, int nTheta, int thetaPad, int count,
    const double2* __restrict__ spec, const double2* __restrict__ tw,
    double* __restrict__ out, RingRange rr) {
  extern __shared__ double2 smem[];
  const int j0 = (blockIdx.x + rr.jBegin / R) * R, f = blockIdx.y;
  const int nPhi = 2 * L, n = plan.n;
  const int sgnCount = kReal ? 1 : 2;
  auto S = [&](int m, int sgn, int jj) {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  if (!kReal) {
    for (int e = threadIdx.x; e < R * nPhi; e += 256) {
      const int r = e % R, bin = e / R;
      const int j = j0 + r;
      double2 x = make_double2(0.0, 0.0);
      if (j < nTheta) {
        if (bin <= lmax) x = S(bin, 0, j);
        if (bin >= nPhi - lmax) x = cadd(x, S(nPhi - bin, 1, nTheta - 1 - j));
      }
      smem[pad8(r * n + bin)] = x;
    }
  } else {
    const int M = L;
    for (int e = threadIdx.x; e < R * M; e += 256) {
      const int r = e % R, bin = e / R;
      const int j = j0 + r;
      double2 z = make_double2(0.0, 0.0);
      if (j < nTheta) {
        const int bc = M - bin;
        double2 x0 = bin <= lmax ? S(bin, 0, j) : make_double2(0.0, 0.0);
        double2 x1 = bc <= lmax ? S(bc, 0, j) : make_double2(0.0, 0.0);
        if (bin == 0) x0.y = 0.0;
        if (bc == M) x1.y = 0.0;
        const double2 xc = cconj(x1);
        const double2 w = twiddle(tw, bin, 1, +1);
        z = cadd(cadd(x0, xc), cmul_si(cmul(w, csub(x0, xc)), +1));
      }
      smem[pad8(r * n + bin)] = z;
    }
  }
  __syncthreads();
  fft_reg<kVPT>(smem, plan, tw, +1);
  for (int e = threadIdx.x; e < R * n; e += 256) {
    const int r = e / n, k = e - r * n;
    const int j = j0 + r;
    if (!rr.has(j)) continue;
    if (!kReal) {
      reinterpret_cast<double2*>(rr.grid(out, f, 2 * (size_t)nTheta * nPhi))[(size_t)j * nPhi + k] = smem[pad8(e)];
    } else {
      reinterpret_cast<double2*>(rr.grid(out, f, (size_t)nTheta * nPhi) + (size_t)j * nPhi)[k] = smem[pad8(e)];
    }
  }
}

// Forward, R rings per block.
template <bool kReal, int kVPT>
__global__ void __launch_bounds__(256) k_fft_forward_reg(
    FftPlan plan, int R, int L, int lmax, int nTheta, int thetaPad, int count,
    const double* __restrict__ in, const double* __restrict__ weight,
    const double2* __restrict__ tw, double2* __restrict__ spec, RingRange rr) {
  extern __shared__ double2 smem[];
  const int j0 = (blockIdx.x + rr.jBegin / R) * R, f = blockIdx.y;
  const int nPhi = 2 * L, n = plan.n;
  const int sgnCount = kReal ? 1 : 2;
  auto S = [&](int m, int sgn, int jj) -> double2& {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  if (j0 <= nTheta - 1 && nTheta - 1 < j0 + R) {
    const int padW = thetaPad - nTheta;
    for (int i = threadIdx.x; i < (lmax + 1) * sgnCount * padW; i += 256) {
      const int q = i / padW, jj = nTheta + (i - q * padW);
      S(q / sgnCount, q % sgnCount, jj) = make_double2(0.0, 0.0);
    }
  }
  for (int e = threadIdx.x; e < R * n; e += 256) {
    const int r = e / n, k = e - r * n;
    const int j = j0 + r;
    double2 x = make_double2(0.0, 0.0);
    if (j < nTheta) {
      if (!kReal) {
        x = reinterpret_cast<const double2*>(rr.grid(in, f, 2 * (size_t)nTheta * nPhi))[(size_t)j * nPhi + k];
      } else {
        x = reinterpret_cast<const double2*>(rr.grid(in, f, (size_t)nTheta * nPhi) + (size_t)j * nPhi)[k];
      }
    }
    smem[pad8(e)] = x;
  }
  __syncthreads();
  fft_reg<kVPT>(smem, plan, tw, -1);
  const double twoPiOverN = 6.283185307179586477 / nPhi;
  for (int e = threadIdx.x; e < R * (lmax + 1); e += 256) {
    const int r = e % R, m = e / R;
    const int j = j0 + r;
    if (!rr.has(j)) continue;
    const double scale = weight[j] * twoPiOverN;
    auto X = [&](int b) { return smem[pad8(r * n + b)]; };
    if (!kReal) {
      S(m, 0, j) = cscale(X(m), scale);
      S(m, 1, nTheta - 1 - j) = m ? cscale(X(nPhi - m), scale) : make_double2(0.0, 0.0);
    } else {
      const int M = L;
      const double2 z0 = X(m == M ? 0 : m);
      const double2 zc = cconj(X(m == 0 ? 0 : M - m));
      const double2 w = twiddle(tw, m, 1, -1);
      const double2 ev = cscale(cadd(z0, zc), 0.5);
      const double2 od = cscale(cmul_si(csub(z0, zc), -1), 0.5);
      S(m, 0, j) = cscale(cadd(ev, cmul(w, od)), scale);
    }
  }
}

// ---------------------------------------------------------------------------
// Power-of-two lengths with everything compile-time: N points per ring,
// R = 4096 / N rings per block (16 points per thread), radix-8 stages then one
// radix-4 or radix-2 stage; indices by shifts and masks. Used for rings of
// 32..128 points; longer power-of-two rings take the three-pass path below.
// Ring r's point u
// sits at r * RS + u + u / 8, which keeps both the in-ring strided accesses
// and the ring-interleaved gathers conflict-free. Global loads are issued
// all at once per thread before any shared-memory store.
// ---------------------------------------------------------------------------
template <int N>
struct P2 {
  static constexpr int kPoints = N > 4096 ? N : 4096;
  static constexpr int kVPT = kPoints / 256;
  static constexpr int R = kPoints / N;
  // Ring stride: in the ring-interleaved gathers a quarter warp touches
  // min(R, 8) rings x max(1, 8 / R) consecutive points; RS = 8 / R (mod 8) for
  // R < 8 and RS odd otherwise puts those eight 16-byte accesses in eight
  // different bank groups.
  static constexpr int RS = N + N / 8 + (R < 8 ? 8 / R : 1);
  static constexpr int kSmem = R * RS;  // double2 units
  __device__ __forceinline__ static int at(int ring, int u) { return ring * RS + u + (u >> 3); }
};

__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x / 2); }

template <int N, int P, int M>
__device__ __forceinline__ void p2_stage(double2* buf, const double2* __restrict__ tw,
                                         int twStride, int sign) {
  constexpr int L = N / (P * M);
  constexpr int NBR = N / P;  // butterflies per ring
  constexpr int NB = P2<N>::kVPT / P;  // butterflies per thread
  double2 v[NB][P];
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int idx = threadIdx.x + b * 256;
    const int ring = idx >> ilog2(NBR), bi = idx & (NBR - 1);
    const int j = bi >> ilog2(M), k = bi & (M - 1);
#pragma unroll
    for (int q = 0; q < P; q++) v[b][q] = buf[P2<N>::at(ring, k + j * M + q * L * M)];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const int idx = threadIdx.x + b * 256;
    const int ring = idx >> ilog2(NBR), bi = idx & (NBR - 1);
    const int j = bi >> ilog2(M), k = bi & (M - 1);
    dft_reg<P>(v[b], sign);
    const int t = j * M;
    if (L > 1 && t) {
#pragma unroll
      for (int r = 1; r < P; r++) v[b][r] = cmul(v[b][r], twiddle(tw, t * r, twStride, sign));
    }
#pragma unroll
    for (int r = 0; r < P; r++) buf[P2<N>::at(ring, k + j * P * M + r * M)] = v[b][r];
  }
  __syncthreads();
}

template <int N, int M>
__device__ __forceinline__ void p2_fft(double2* buf, const double2* __restrict__ tw, int twStride,
                                       int sign) {
  constexpr int rem = N / M;
  constexpr int P = rem % 8 == 0 ? 8 : (rem % 4 == 0 ? 4 : 2);
  p2_stage<N, P, M>(buf, tw, twStride, sign);
  if constexpr (M * P < N) p2_fft<N, M * P>(buf, tw, twStride, sign);
}

template <bool kReal, int N>
__global__ void __launch_bounds__(256) k_fft_inverse_p2(
    int L, int lmax, int nTheta, int thetaPad, int count, const double2* __restrict__ spec,
    const double2* __restrict__ tw, double* __restrict__ out, RingRange rr) {
  extern __shared__ double2 smem[];
  constexpr int R = P2<N>::R;
  const int j0 = (blockIdx.x + rr.jBegin / R) * R, f = blockIdx.y;
  const int nPhi = 2 * L;
  const int sgnCount = kReal ? 1 : 2;
  const int twStride = nPhi / N;
  auto S = [&](int m, int sgn, int jj) {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  constexpr int kPer = R * N / 256;  // points per thread (16)
  double2 xv[kPer];
#pragma unroll
  for (int it = 0; it < kPer; it++) {
    const int e = threadIdx.x + it * 256;
    const int r = e & (R - 1), bin = e >> ilog2(R);
    const int j = j0 + r;
    double2 x = make_double2(0.0, 0.0);
    if (j < nTheta) {
      if (!kReal) {
        if (bin <= lmax) x = S(bin, 0, j);
        if (bin >= nPhi - lmax) x = cadd(x, S(nPhi - bin, 1, nTheta - 1 - j));
      } else {
        const int M = L, bc = M - bin;
        double2 x0 = bin <= lmax ? S(bin, 0, j) : make_double2(0.0, 0.0);
        double2 x1 = bc <= lmax ? S(bc, 0, j) : make_double2(0.0, 0.0);
        if (bin == 0) x0.y = 0.0;
        if (bc == M) x1.y = 0.0;
        const double2 xc = cconj(x1);
        const double2 w = twiddle(tw, bin, 1, +1);
        x = cadd(cadd(x0, xc), cmul_si(cmul(w, csub(x0, xc)), +1));
      }
    }
    xv[it] = x;
  }
#pragma unroll
  for (int it = 0; it < kPer; it++) {
    const int e = threadIdx.x + it * 256;
    smem[P2<N>::at(e & (R - 1), e >> ilog2(R))] = xv[it];
  }
  __syncthreads();
  p2_fft<N, 1>(smem, tw, twStride, +1);
  for (int e = threadIdx.x; e < R * N; e += 256) {
    const int r = e >> ilog2(N), k = e & (N - 1);
    const int j = j0 + r;
    if (!rr.has(j)) continue;
    if (!kReal) {
      reinterpret_cast<double2*>(rr.grid(out, f, 2 * (size_t)nTheta * nPhi))[(size_t)j * nPhi + k] = smem[P2<N>::at(r, k)];
    } else {
      reinterpret_cast<double2*>(rr.grid(out, f, (size_t)nTheta * nPhi) + (size_t)j * nPhi)[k] = smem[P2<N>::at(r, k)];
    }
  }
}

template <bool kReal, int N>
__global__ void __launch_bounds__(256) k_fft_forward_p2(
    int L, int lmax, int nTheta, int thetaPad, int count, const double* __restrict__ in,
    const double* __restrict__ weight, const double2* __restrict__ tw,
    double2* __restrict__ spec, RingRange rr) {
  extern __shared__ double2 smem[];
  constexpr int R = P2<N>::R;
  const int j0 = (blockIdx.x + rr.jBegin / R) * R, f = blockIdx.y;
  const int nPhi = 2 * L;
  const int sgnCount = kReal ? 1 : 2;
  const int twStride = nPhi / N;
  auto S = [&](int m, int sgn, int jj) -> double2& {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  if (j0 <= nTheta - 1 && nTheta - 1 < j0 + R) {
    const int padW = thetaPad - nTheta;
    for (int i = threadIdx.x; i < (lmax + 1) * sgnCount * padW; i += 256) {
      const int q = i / padW, jj = nTheta + (i - q * padW);
      S(q / sgnCount, q % sgnCount, jj) = make_double2(0.0, 0.0);
    }
  }
  constexpr int kPer = R * N / 256;
  double2 xv[kPer];
#pragma unroll
  for (int it = 0; it < kPer; it++) {
    const int e = threadIdx.x + it * 256;
    const int r = e >> ilog2(N), k = e & (N - 1);
    const int j = j0 + r;
    double2 x = make_double2(0.0, 0.0);
    if (j < nTheta) {
      x = kReal ? reinterpret_cast<const double2*>(rr.grid(in, f, (size_t)nTheta * nPhi) + (size_t)j * nPhi)[k]
                : reinterpret_cast<const double2*>(rr.grid(in, f, 2 * (size_t)nTheta * nPhi))[(size_t)j * nPhi + k];
    }
    xv[it] = x;
  }
#pragma unroll
  for (int it = 0; it < kPer; it++) {
    const int e = threadIdx.x + it * 256;
    smem[P2<N>::at(e >> ilog2(N), e & (N - 1))] = xv[it];
  }
  __syncthreads();
  p2_fft<N, 1>(smem, tw, twStride, -1);
  const double twoPiOverN = 6.283185307179586477 / nPhi;
  for (int e = threadIdx.x; e < R * (lmax + 1); e += 256) {
    const int r = e & (R - 1), m = e >> ilog2(R);
    const int j = j0 + r;
    if (!rr.has(j)) continue;
    const double scale = weight[j] * twoPiOverN;
    auto X = [&](int b) { return smem[P2<N>::at(r, b)]; };
    if (!kReal) {
      S(m, 0, j) = cscale(X(m), scale);
      S(m, 1, nTheta - 1 - j) = m ? cscale(X(nPhi - m), scale) : make_double2(0.0, 0.0);
    } else {
      const int M = L;
      const double2 z0 = X(m == M ? 0 : m);
      const double2 zc = cconj(X(m == 0 ? 0 : M - m));
      const double2 w = twiddle(tw, m, 1, -1);
      const double2 ev = cscale(cadd(z0, zc), 0.5);
      const double2 od = cscale(cmul_si(csub(z0, zc), -1), 0.5);
      S(m, 0, j) = cscale(cadd(ev, cmul(w, od)), scale);
    }
  }
}

// FP32 register DFTs of length 2, 4, 8, 16: the same operations as the FP64
// specialisations above, in float2.
template <int P>
__device__ __forceinline__ void dft_reg(float2 (&c)[P], int sign) {
  if constexpr (P == 2) {
    const float2 a = cadd(c[0], c[1]), b = csub(c[0], c[1]);
    c[0] = a;
    c[1] = b;
  } else if constexpr (P == 4) {
    const float2 s02 = cadd(c[0], c[2]), d02 = csub(c[0], c[2]);
    const float2 s13 = cadd(c[1], c[3]), d13 = cmul_si(csub(c[1], c[3]), sign);
    c[0] = cadd(s02, s13);
    c[1] = cadd(d02, d13);
    c[2] = csub(s02, s13);
    c[3] = csub(d02, d13);
  } else if constexpr (P == 8) {
    float2 e[4] = {c[0], c[2], c[4], c[6]};
    float2 o[4] = {c[1], c[3], c[5], c[7]};
    dft_reg<4>(e, sign);
    dft_reg<4>(o, sign);
    const float h = 0.70710678118654752440f;
    const float sg = (float)sign;
    o[1] = make_float2(h * (o[1].x - sg * o[1].y), h * (o[1].y + sg * o[1].x));
    o[2] = cmul_si(o[2], sign);
    o[3] = make_float2(h * (-o[3].x - sg * o[3].y), h * (-o[3].y + sg * o[3].x));
#pragma unroll
    for (int r = 0; r < 4; r++) {
      c[r] = cadd(e[r], o[r]);
      c[r + 4] = csub(e[r], o[r]);
    }
  } else {
    static_assert(P == 16, "FP32 register DFTs: 2, 4, 8, 16");
    const float sg = (float)sign;
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float h = 0.70710678118654752440f;
    float2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
      float2 t[4] = {c[n2], c[4 + n2], c[8 + n2], c[12 + n2]};
      dft_reg<4>(t, sign);
#pragma unroll
      for (int k1 = 0; k1 < 4; k1++) a[n2][k1] = t[k1];
    }
    a[1][1] = cmul(a[1][1], make_float2(c1, sg * s1));
    a[1][2] = cmul(a[1][2], make_float2(h, sg * h));
    a[1][3] = cmul(a[1][3], make_float2(s1, sg * c1));
    a[2][1] = cmul(a[2][1], make_float2(h, sg * h));
    a[2][2] = cmul_si(a[2][2], sign);
    a[2][3] = cmul(a[2][3], make_float2(-h, sg * h));
    a[3][1] = cmul(a[3][1], make_float2(s1, sg * c1));
    a[3][2] = cmul(a[3][2], make_float2(-h, sg * h));
    a[3][3] = cmul(a[3][3], make_float2(-c1, -sg * s1));
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
      float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      dft_reg<4>(t, sign);
#pragma unroll
      for (int k2 = 0; k2 < 4; k2++) c[k1 + 4 * k2] = t[k2];
    }
  }
}

// ---------------------------------------------------------------------------
// Three-pass power-of-two path (rings of 256..4096 points). A block holds
// 4096 points (R = 4096 / N rings), 16 per thread, and runs the Stockham
// stages 16 x ... with radix-16/8/4 register butterflies: the first stage
// works directly on the values loaded from global memory, the last one writes
// its results straight to global memory, so shared memory is crossed only
// between stages (two round trips for N = 2048 instead of five). Twiddles of
// a butterfly are built from at most three table loads (w^t, w^4t, w^8t) by
// complex products, each power at most four products deep. Ring r's point u
// sits at r * RS + u + u / 16: with RS = N + N/16 + 8/R every stage's loads
// and stores, in both the ring-major and the ring-interleaved thread maps,
// are free of bank conflicts (checked by enumeration of the quarter-warp
// access sets).
// ---------------------------------------------------------------------------
template <int N, int kPts>
struct P3 {
  static constexpr int kPoints = N > kPts ? N : kPts;
  static constexpr int kThreads = kPoints / 16;
  static constexpr int R = kPoints / N;
  static constexpr int RS = N + N / 16 + (R > 8 ? 1 : (R > 1 ? 8 / R : 0));
  static constexpr int kSmem = R * RS;  // complex elements
  __device__ __forceinline__ static int at(int ring, int u) { return ring * RS + u + (u >> 4); }
};

// Radix of the stage that follows M points of already combined length.
template <int N, int M>
struct P3Radix {
  static constexpr int rem = N / M;
  static constexpr int P = M == 1 ? 16
                           : ((rem % 16 == 0 && rem / 16 != 2) ? 16
                              : (rem % 8 == 0 ? 8 : (rem % 4 == 0 ? 4 : 2)));
};

// Blocks per SM the three-pass kernels are compiled for: two of 4096 FP64
// points (128 registers a thread; one of 8192), three of 4096 FP32 points
// (85 registers) and two of 8192 (64).
template <int kPts, typename C>
constexpr int p3_min_blocks() {
  return sizeof(C) == 16 ? 8192 / kPts : (kPts >= 8192 ? 2 : 3);
}

// v[r] *= w^(t r), w = exp(sign 2 pi i / N) from the table at stride twStride.
template <int P, typename C>
__device__ __forceinline__ void p3_twiddle(C (&v)[P], const C* __restrict__ tw, int t,
                                           int twStride, int sign) {
  if (t == 0) return;
  const C a = twiddle(tw, t, twStride, sign);
  v[1] = cmul(v[1], a);
  if constexpr (P > 2) {
    const C a2 = cmul(a, a), a3 = cmul(a2, a);
    v[2] = cmul(v[2], a2);
    v[3] = cmul(v[3], a3);
    if constexpr (P > 4) {
      const C b = twiddle(tw, 4 * t, twStride, sign);
      const C b1 = cmul(b, a), b2 = cmul(b, a2), b3 = cmul(b, a3);
      v[4] = cmul(v[4], b);
      v[5] = cmul(v[5], b1);
      v[6] = cmul(v[6], b2);
      v[7] = cmul(v[7], b3);
      if constexpr (P > 8) {
        const C c = twiddle(tw, 8 * t, twStride, sign);
        v[8] = cmul(v[8], c);
        v[9] = cmul(v[9], cmul(c, a));
        v[10] = cmul(v[10], cmul(c, a2));
        v[11] = cmul(v[11], cmul(c, a3));
        v[12] = cmul(v[12], cmul(c, b));
        v[13] = cmul(v[13], cmul(c, b1));
        v[14] = cmul(v[14], cmul(c, b2));
        v[15] = cmul(v[15], cmul(c, b3));
      }
    }
  }
}

// Middle stages (every stage after the first and before the last), in place.
template <int N, int kPts, int M, typename C>
__device__ __forceinline__ void p3_middle(C* buf, const C* __restrict__ tw, int twStride,
                                          int sign) {
  constexpr int P = P3Radix<N, M>::P;
  if constexpr (M * P < N) {
    constexpr int L = N / (P * M);
    constexpr int NBR = N / P;
    constexpr int NB = 16 / P;
    C v[NB][P];
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const int g = threadIdx.x + b * P3<N, kPts>::kThreads;
      const int ring = g >> ilog2(NBR), bi = g & (NBR - 1);
      const int j = bi >> ilog2(M), k = bi & (M - 1);
#pragma unroll
      for (int q = 0; q < P; q++) v[b][q] = buf[P3<N, kPts>::at(ring, k + j * M + q * L * M)];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const int g = threadIdx.x + b * P3<N, kPts>::kThreads;
      const int ring = g >> ilog2(NBR), bi = g & (NBR - 1);
      const int j = bi >> ilog2(M), k = bi & (M - 1);
      dft_reg<P>(v[b], sign);
      p3_twiddle<P>(v[b], tw, j * M, twStride, sign);
#pragma unroll
      for (int r = 0; r < P; r++) buf[P3<N, kPts>::at(ring, k + j * P * M + r * M)] = v[b][r];
    }
    __syncthreads();
    p3_middle<N, kPts, M * P, C>(buf, tw, twStride, sign);
  }
}

// Combined length before the last stage.
template <int N, int M = 1>
__host__ __device__ constexpr int p3_last_m() {
  constexpr int P = P3Radix<N, M>::P;
  if constexpr (M * P >= N) return M;
  else return p3_last_m<N, M * P>();
}

// Spectral rows per TMA box of the inverse's staged loads.
constexpr int kSpecBox = 64;

// kTma: the block's spectral rows (orders 0..lmax for each sign, R
// colatitudes each; the -m rows at the mirrored colatitudes) are brought into
// a staging buffer by 4-D TMA boxes of kSpecBox rows, so the strided 16R-byte
// row segments cost no load instructions or registers; the first stage
// reads them from there. The kernel is then persistent: a block walks the
// work items (ring group, field) with stride gridDim.x, and as soon as the
// first stage has read an item's rows it starts the TMA of its next item's
// rows, which arrive while the middle and last stages run. Without kTma,
// one block per item, and the first stage loads from global memory.
//
// SpecT: double2 (the FP64 layout above) or float2, the spectra of the
// BF16x3 form, which keeps its -m rows at their own colatitudes (no mirror:
// the Legendre epilogue and operand preparation of that form apply it), so
// both signs' TMA boxes start at colatitude j0.
//
// C: the butterflies' precision (double2, or float2 with float2 spectra);
// the grid is written in FP64.
template <bool kReal, int N, bool kTma, int kPts, typename SpecT, typename C>
__global__ void __launch_bounds__(kPts / 16, p3_min_blocks<kPts, C>()) k_fft_inverse_p3(
    const __grid_constant__ CUtensorMap specMap, int L, int lmax, int nTheta, int thetaPad,
    int count, const SpecT* __restrict__ spec, const C* __restrict__ tw,
    double* __restrict__ out, int* err, int stageOff, RingRange rr, int nGroups) {
  constexpr bool kMir = std::is_same<SpecT, double2>::value;
  // TMA destinations want 128-byte alignment: round the dynamic base up (the
  // launch adds 128 bytes of slack plus the barrier word after the buffers).
  extern __shared__ unsigned char p3_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(p3_raw) + 127) & ~uintptr_t(127));
  C* smem = reinterpret_cast<C*>(base);
  constexpr int R = P3<N, kPts>::R;
  const int nPhi = 2 * L;
  const int sgnCount = kReal ? 1 : 2;
  const int twStride = nPhi / N;
  const int nbox = (lmax + 1 + kSpecBox - 1) / kSpecBox;
  const int M1 = nbox * kSpecBox;  // staged rows per sign
  // stageOff: byte offset of the staging buffer. The barrier word lies
  // past both buffers (which may overlap).
  SpecT* staged = reinterpret_cast<SpecT*>(base + stageOff);
  constexpr size_t kFftBytes = (sizeof(C) * P3<N, kPts>::kSmem + 127) / 128 * 128;
  const size_t stageEnd = (size_t)stageOff + (size_t)sgnCount * M1 * R * sizeof(SpecT);
  uint64_t& bar =
      *reinterpret_cast<uint64_t*>(base + (stageEnd > kFftBytes ? stageEnd : kFftBytes));
  const int items = kTma ? nGroups * count : 1;
  // Colatitude of an item's first ring, and its field.
  auto item = [&](int w, int& j0, int& f) {
    if constexpr (kTma) {
      const int grp = w % nGroups;
      f = w / nGroups;
      j0 = (grp + rr.jBegin / R) * R;
    } else {
      j0 = (blockIdx.x + rr.jBegin / R) * R;
      f = blockIdx.y;
    }
  };
  auto fetch = [&](int w) {  // one thread: the TMA boxes of item w
    int j0, f;
    item(w, j0, f);
    tc::mbar_arrive_expect_tx(&bar, (uint32_t)(sgnCount * M1 * R * sizeof(SpecT)));
    for (int sg = 0; sg < sgnCount; sg++) {
      // Colatitudes j0.. (sign 0, and sign 1 without mirror) or their mirror
      // images nTheta-j0-R.. (sign 1, FP64 layout).
      const int x = 2 * ((sg == 0 || !kMir) ? j0 : nTheta - j0 - R);
      for (int b = 0; b < nbox; b++)
        tc::tma_load_4d(staged + (size_t)(sg * M1 + b * kSpecBox) * R, &specMap, &bar, x, f, sg,
                        b * kSpecBox);
    }
  };
  if constexpr (kTma) {
    if (threadIdx.x == 0) {
      tc::mbar_init(&bar, 1);
      tc::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && (int)blockIdx.x < items) {
      tc::prefetch_tmap(&specMap);
      fetch(blockIdx.x);
    }
  }
  int it = 0;
  for (int w = kTma ? (int)blockIdx.x : 0; w < items; w += kTma ? (int)gridDim.x : 1, it++) {
    int j0, f;
    item(w, j0, f);
    auto S = [&](int m, int sgn, int jj) {
      return to_c<C>(spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj]);
    };
    if constexpr (kTma) {
      // Every thread leaves together if the rows do not arrive in time.
      const bool ok = tc::mbar_wait(&bar, it & 1, err, 21);
      if (__syncthreads_or(!ok)) break;
    }
    // First stage (radix 16, M = 1), rings interleaved across lanes so that
    // lanes 0..R-1 read R consecutive colatitudes of one spectral row.
    {
      const int r = threadIdx.x & (R - 1), jj = threadIdx.x >> ilog2(R);
      const int th = j0 + r;
      C v[16];
      // Row m of sign sg (staged): colatitude j0 + r is element r, its mirror
      // nTheta-1-(j0+r) element R-1-r.
      auto T = [&](int m, int sg) {
        return to_c<C>(sg == 0 ? staged[(size_t)m * R + r]
                               : staged[(size_t)(M1 + m) * R + (kMir ? R - 1 - r : r)]);
      };
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int bin = jj + q * (N / 16);
        C x{};
        if (kTma || th < nTheta) {
          if (!kReal) {
            if (bin <= lmax) x = kTma ? T(bin, 0) : S(bin, 0, th);
            if (bin >= nPhi - lmax)
              x = cadd(x, kTma ? T(nPhi - bin, 1) : S(nPhi - bin, 1, kMir ? nTheta - 1 - th : th));
          } else {
            const int M = L, bc = M - bin;
            C x0 = bin <= lmax ? (kTma ? T(bin, 0) : S(bin, 0, th)) : C{};
            C x1 = bc <= lmax ? (kTma ? T(bc, 0) : S(bc, 0, th)) : C{};
            if (bin == 0) x0.y = 0;
            if (bc == M) x1.y = 0;
            const C xc = cconj(x1);
            const C w2 = twiddle(tw, bin, 1, +1);
            x = cadd(cadd(x0, xc), cmul_si(cmul(w2, csub(x0, xc)), +1));
          }
        }
        v[q] = x;
      }
      // The staging buffer is read and the previous item's last stage has
      // read the FFT buffer: start the next item's rows (a block has a next
      // item only when the staging buffer is its own), then fill the FFT
      // buffer.
      __syncthreads();
      if constexpr (kTma) {
        if (threadIdx.x == 0 && w + (int)gridDim.x < items) {
          tc::fence_proxy_async();
          fetch(w + gridDim.x);
        }
      }
      dft_reg<16>(v, +1);
      p3_twiddle<16>(v, tw, jj, twStride, +1);
#pragma unroll
      for (int q = 0; q < 16; q++) smem[P3<N, kPts>::at(r, jj * 16 + q)] = v[q];
    }
    __syncthreads();
    p3_middle<N, kPts, 16>(smem, tw, twStride, +1);
    // Last stage (L = 1, no twiddles), ring-major so that lanes write
    // consecutive longitudes.
    constexpr int M = p3_last_m<N>();
    constexpr int P = N / M;
    constexpr int NB = 16 / P;
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const int g = threadIdx.x + b * P3<N, kPts>::kThreads;
      const int ring = g >> ilog2(M), k = g & (M - 1);
      C v[P];
#pragma unroll
      for (int q = 0; q < P; q++) v[q] = smem[P3<N, kPts>::at(ring, k + q * M)];
      dft_reg<P>(v, +1);
      const int th = j0 + ring;
      if (rr.has(th)) {
        double2* row = kReal ? reinterpret_cast<double2*>(rr.grid(out, f, (size_t)nTheta * nPhi) + (size_t)th * nPhi)
                             : reinterpret_cast<double2*>(rr.grid(out, f, 2 * (size_t)nTheta * nPhi)) + (size_t)th * nPhi;
#pragma unroll
        for (int r = 0; r < P; r++) row[k + r * M] = to_c<double2>(v[r]);
      }
    }
  }
}

// SpecT as for the inverse: float2 spectra keep the -m rows unmirrored.
template <bool kReal, int N, int kPts, typename SpecT>
__global__ void __launch_bounds__(kPts / 16, p3_min_blocks<kPts, SpecT>()) k_fft_forward_p3(
    int L, int lmax, int nTheta, int thetaPad, int count, const double* __restrict__ in,
    const double* __restrict__ weight, const SpecT* __restrict__ tw,
    SpecT* __restrict__ spec, RingRange rr) {
  using C = SpecT;  // butterflies in the spectra's precision
  constexpr bool kMir = std::is_same<SpecT, double2>::value;
  extern __shared__ unsigned char p3f_raw[];
  C* smem = reinterpret_cast<C*>(p3f_raw);
  constexpr int R = P3<N, kPts>::R;
  const int j0 = (blockIdx.x + rr.jBegin / R) * R, f = blockIdx.y;
  const int nPhi = 2 * L;
  const int sgnCount = kReal ? 1 : 2;
  const int twStride = nPhi / N;
  auto S = [&](int m, int sgn, int jj) -> SpecT& {
    return spec[((size_t)(m * sgnCount + sgn) * count + f) * thetaPad + jj];
  };
  if (j0 <= nTheta - 1 && nTheta - 1 < j0 + R) {
    const int padW = thetaPad - nTheta;
    for (int i = threadIdx.x; i < (lmax + 1) * sgnCount * padW; i += P3<N, kPts>::kThreads) {
      const int q = i / padW, jj = nTheta + (i - q * padW);
      S(q / sgnCount, q % sgnCount, jj) = from_d2<SpecT>(make_double2(0.0, 0.0));
    }
  }
  // First stage, ring-major: lanes read consecutive longitudes.
  {
    constexpr int NBR = N / 16;
    const int ring = threadIdx.x >> ilog2(NBR), jj = threadIdx.x & (NBR - 1);
    const int th = j0 + ring;
    C v[16];
    const double2* row = kReal ? reinterpret_cast<const double2*>(rr.grid(in, f, (size_t)nTheta * nPhi) + (size_t)th * nPhi)
                               : reinterpret_cast<const double2*>(rr.grid(in, f, 2 * (size_t)nTheta * nPhi)) + (size_t)th * nPhi;
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = th < nTheta ? to_c<C>(row[jj + q * NBR]) : C{};
    dft_reg<16>(v, -1);
    p3_twiddle<16>(v, tw, jj, twStride, -1);
#pragma unroll
    for (int q = 0; q < 16; q++) smem[P3<N, kPts>::at(ring, jj * 16 + q)] = v[q];
  }
  __syncthreads();
  p3_middle<N, kPts, 16>(smem, tw, twStride, -1);
  constexpr int M = p3_last_m<N>();
  constexpr int P = N / M;
  constexpr int NB = 16 / P;
  const double twoPiOverN = 6.283185307179586477 / nPhi;
  if constexpr (!kReal) {
    // Last stage with rings interleaved across lanes: lanes 0..R-1 write R
    // consecutive colatitudes of one spectral row.
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const int g = threadIdx.x + b * P3<N, kPts>::kThreads;
      const int ring = g & (R - 1), k = g >> ilog2(R);
      C v[P];
#pragma unroll
      for (int q = 0; q < P; q++) v[q] = smem[P3<N, kPts>::at(ring, k + q * M)];
      dft_reg<P>(v, -1);
      const int th = j0 + ring;
      if (rr.has(th)) {
        const double scale = weight[th] * twoPiOverN;
#pragma unroll
        for (int r = 0; r < P; r++) {
          const int bin = k + r * M;
          const C x = cscale(v[r], scale);
          const int thm = kMir ? nTheta - 1 - th : th;
          if (bin <= lmax) S(bin, 0, th) = x;
          if (bin == 0) S(0, 1, thm) = C{};
          else if (bin >= nPhi - lmax) S(nPhi - bin, 1, thm) = x;
        }
      }
    }
  } else {
    C v[NB][P];
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const int g = threadIdx.x + b * P3<N, kPts>::kThreads;
      const int ring = g >> ilog2(M), k = g & (M - 1);
#pragma unroll
      for (int q = 0; q < P; q++) v[b][q] = smem[P3<N, kPts>::at(ring, k + q * M)];
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const int g = threadIdx.x + b * P3<N, kPts>::kThreads;
      const int ring = g >> ilog2(M), k = g & (M - 1);
      dft_reg<P>(v[b], -1);
#pragma unroll
      for (int r = 0; r < P; r++) smem[P3<N, kPts>::at(ring, k + r * M)] = v[b][r];
    }
    __syncthreads();
    // Real field: unpack the half-length transform, X(m) from z(m) and
    // conj z(M - m), M = nPhi / 2.
    for (int e = threadIdx.x; e < R * (lmax + 1); e += P3<N, kPts>::kThreads) {
      const int r = e & (R - 1), m = e >> ilog2(R);
      const int th = j0 + r;
      if (!rr.has(th)) continue;
      const double scale = weight[th] * twoPiOverN;
      const int Mh = L;
      const C z0 = smem[P3<N, kPts>::at(r, m == Mh ? 0 : m)];
      const C zc = cconj(smem[P3<N, kPts>::at(r, m == 0 ? 0 : Mh - m)]);
      const C w = twiddle(tw, m, 1, -1);
      const C ev = cscale(cadd(z0, zc), 0.5);
      const C od = cscale(cmul_si(csub(z0, zc), -1), 0.5);
      S(m, 0, th) = cscale(cadd(ev, cmul(w, od)), scale);
    }
  }
}

// Tensor map of the spectral buffer as FP64 or FP32 [m][sign][field][2 *
// thetaPad] with a 2R x 1 x 1 x kSpecBox box (R colatitudes of kSpecBox
// rows).
template <typename SpecT>
bool spec_map(CUtensorMap* map, const SpecT* spec, int thetaPad, int count, int sgnCount,
              int lmax, int R) {
  tc::EncodeTiledFn fn = tc::encode_fn();
  if (!fn) return false;
  constexpr cuuint64_t kE = sizeof(SpecT) / 2;  // bytes per real component
  const cuuint64_t tp2 = 2 * (cuuint64_t)thetaPad;
  cuuint64_t dims[4] = {tp2, (cuuint64_t)count, (cuuint64_t)sgnCount, (cuuint64_t)lmax + 1};
  cuuint64_t strides[3] = {tp2 * kE, tp2 * kE * count, tp2 * kE * count * sgnCount};
  cuuint32_t box[4] = {(cuuint32_t)(2 * R), 1, 1, kSpecBox};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUtensorMapDataType dt =
      kE == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(map, dt, 4, const_cast<SpecT*>(spec), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Blocks of R rings covering the colatitudes of rr.
inline unsigned ring_blocks(RingRange rr, int R) {
  return (unsigned)((rr.jEnd + R - 1) / R - rr.jBegin / R);
}

// Butterflies of the inverse with FP32 spectra: FP64 by default. Measured at
// lmax 1024, 64 fields: 0.93 ms; FP32 butterflies 1.07 ms at the three blocks
// per SM their smaller FFT buffer allows (0.88 ms when held to two; faster
// at 16 fields, 0.18 against 0.22 ms), for a larger error against the FP64
// path (8.3e-7 against 8.1e-7). GSHT_FFT_INV_FP32=1 selects the FP32 ones
// for comparisons.
bool fp32_inverse_butterflies() {
  const char* e = getenv("GSHT_FFT_INV_FP32");
  return e && e[0] == '1';
}

template <int N, int kPts, typename SpecT, typename C>
gsht_status launch_p3_inverse(const gsht_grid* g, int lmax, int is_real, int count,
                              const void* src, void* dst, cudaStream_t s, RingRange rr) {
  constexpr int kThr = P3<N, kPts>::kThreads;
  size_t shmem = sizeof(C) * P3<N, kPts>::kSmem;  // FFT buffer of the butterflies' precision
  constexpr int R = P3<N, kPts>::R;
  dim3 grid(ring_blocks(rr, R), count);
  const C* tw = std::is_same<C, float2>::value ? reinterpret_cast<const C*>(g->d_twiddle32)
                                               : reinterpret_cast<const C*>(g->d_twiddle);
  {
    const SpecT* spec = static_cast<const SpecT*>(src);
    double* out = static_cast<double*>(dst);
    // Staged spectral rows: sign x ceil((lmax+1)/kSpecBox) boxes x R colatitudes.
    const int sgnCount = is_real ? 1 : 2;
    const size_t staged =
        sizeof(SpecT) * sgnCount * (size_t)((lmax + kSpecBox) / kSpecBox) * kSpecBox * R;
    CUtensorMap map{};
    // TMA boxes start at x = 2 j0 components: 16-byte aligned for FP64
    // always, for FP32 when R (and so j0) is even; the box is 2R components.
    // With a staging buffer of its own after the FFT buffer (128-byte
    // aligned, then the barrier word; 128 bytes of slack align the dynamic
    // base), the kernel runs persistent with the next item's rows in flight,
    // as long as two blocks still fit on an SM (the FP32 spectra of the
    // BF16x3 form). Otherwise (FP64 spectra, twice the bytes) the staging
    // shares the FFT buffer and each block takes one item.
    const bool aligned = sizeof(SpecT) == 16 || R % 2 == 0;
    const size_t fftBytes = (shmem + 127) / 128 * 128;
    const bool tma = aligned && staged + 16 + 128 <= 227 * 1024 &&
                     spec_map(&map, spec, g->theta_pad, count, sgnCount, lmax, R);
    const bool ahead = tma && fftBytes + staged + 16 + 128 <= 113 * 1024;
    const int stageOff = ahead ? (int)fftBytes : 0;  // bytes
    shmem = (ahead ? fftBytes + staged : (fftBytes > staged ? fftBytes : staged)) + 16 + 128;
    const int groups = (int)ring_blocks(rr, R);
    if (tma) {
      auto k = is_real ? k_fft_inverse_p3<true, N, true, kPts, SpecT, C>
                       : k_fft_inverse_p3<false, N, true, kPts, SpecT, C>;
      GSHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
      const long items = (long)groups * count;
      long blocks = items;
      if (ahead) {
        int sms = 148, per = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kThr, shmem) != cudaSuccess ||
            per < 1) {
          cudaGetLastError();
          per = 1;
        }
        if (blocks > (long)sms * per) blocks = (long)sms * per;
      }
      k<<<(unsigned)blocks, kThr, shmem, s>>>(map, g->L, lmax, g->n_theta, g->theta_pad, count,
                                              spec, tw, out, g->d_err, stageOff, rr, groups);
    } else {
      auto k = is_real ? k_fft_inverse_p3<true, N, false, kPts, SpecT, C>
                       : k_fft_inverse_p3<false, N, false, kPts, SpecT, C>;
      GSHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
      k<<<grid, kThr, shmem, s>>>(map, g->L, lmax, g->n_theta, g->theta_pad, count, spec, tw, out,
                                  g->d_err, stageOff, rr, groups);
    }
    GSHT_LAUNCH_CHECK("k_fft_inverse_p3");
  }
  return GSHT_OK;
}

template <int N, int kPts, typename SpecT>
gsht_status launch_p3_dir(const gsht_grid* g, int dir, int lmax, int is_real, int count,
                          const void* src, void* dst, cudaStream_t s, RingRange rr) {
  constexpr int kThr = P3<N, kPts>::kThreads;
  // Forward: butterflies in the spectra's precision.
  size_t shmem = sizeof(SpecT) * P3<N, kPts>::kSmem;
  constexpr int R = P3<N, kPts>::R;
  dim3 grid(ring_blocks(rr, R), count);
  const SpecT* tw = std::is_same<SpecT, float2>::value
                        ? reinterpret_cast<const SpecT*>(g->d_twiddle32)
                        : reinterpret_cast<const SpecT*>(g->d_twiddle);
  if (dir == 1) {
    if (std::is_same<SpecT, float2>::value && fp32_inverse_butterflies())
      return launch_p3_inverse<N, kPts, SpecT, SpecT>(g, lmax, is_real, count, src, dst, s, rr);
    return launch_p3_inverse<N, kPts, SpecT, double2>(g, lmax, is_real, count, src, dst, s, rr);
  } else {
    auto k = is_real ? k_fft_forward_p3<true, N, kPts, SpecT> : k_fft_forward_p3<false, N, kPts, SpecT>;
    GSHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k<<<grid, kThr, shmem, s>>>(g->L, lmax, g->n_theta, g->theta_pad, count,
                                static_cast<const double*>(src), g->d_weight, tw,
                                static_cast<SpecT*>(dst), rr);
    GSHT_LAUNCH_CHECK("k_fft_forward_p3");
  }
  return GSHT_OK;
}

// Points per block of the three-pass kernels for ring length N: 4096 (two
// blocks of 256 threads per SM), except the forward at N = 2048, whose
// spectral rows are written 4 colatitudes (64 B) at a time from 8192-point
// blocks of 512 threads (1.07 against 1.19 ms at lmax 1024, 64 fields).
// Measured and not kept: 2048-point blocks (one ring, 16 B row segments)
// ran 2x slower at N = 2048; 8192-point blocks made the inverse at N = 2048
// (1.30 ms) and both directions at N = 1024 slower.
template <int N, bool kForward>
constexpr int p3_points() {
  return (kForward && N == 2048) ? 8192 : 4096;
}

template <int N, typename SpecT = double2>
gsht_status launch_p3(const gsht_grid* g, int dir, int lmax, int is_real, int count,
                      const void* src, void* dst, cudaStream_t s, RingRange rr) {
  if (dir == 0)
    return launch_p3_dir<N, p3_points<N, true>(), SpecT>(g, dir, lmax, is_real, count, src, dst, s,
                                                         rr);
  return launch_p3_dir<N, p3_points<N, false>(), SpecT>(g, dir, lmax, is_real, count, src, dst, s,
                                                        rr);
}

template <int N>
gsht_status launch_p2(const gsht_grid* g, int dir, int lmax, int is_real, int count,
                      const double* src, double* dst, cudaStream_t s, RingRange rr) {
  const size_t shmem = sizeof(double2) * P2<N>::kSmem;
  dim3 grid(ring_blocks(rr, P2<N>::R), count);
  const double2* tw = reinterpret_cast<const double2*>(g->d_twiddle);
  if (dir == 1) {
    auto k = is_real ? k_fft_inverse_p2<true, N> : k_fft_inverse_p2<false, N>;
    GSHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k<<<grid, 256, shmem, s>>>(g->L, lmax, g->n_theta, g->theta_pad, count,
                               reinterpret_cast<const double2*>(src), tw, dst, rr);
    GSHT_LAUNCH_CHECK("k_fft_inverse_p2");
  } else {
    auto k = is_real ? k_fft_forward_p2<true, N> : k_fft_forward_p2<false, N>;
    GSHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k<<<grid, 256, shmem, s>>>(g->L, lmax, g->n_theta, g->theta_pad, count, src, g->d_weight,
                               tw, reinterpret_cast<double2*>(dst), rr);
    GSHT_LAUNCH_CHECK("k_fft_forward_p2");
  }
  return GSHT_OK;
}

// Power-of-two paths if n is one of the compiled lengths; *used = false otherwise.
gsht_status fft_p2(const gsht_grid* g, int n, int dir, int lmax, int is_real, int count,
                   const double* src, double* dst, cudaStream_t s, bool* used, RingRange rr) {
  *used = true;
  switch (n) {
    case 32: return launch_p2<32>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 64: return launch_p2<64>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 128: return launch_p2<128>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 256: return launch_p3<256>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 512: return launch_p3<512>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 1024: return launch_p3<1024>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 2048: return launch_p3<2048>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 4096: return launch_p3<4096>(g, dir, lmax, is_real, count, src, dst, s, rr);
    default: *used = false; return GSHT_OK;
  }
}

// Register-path configuration for a transform length: points per thread
// kVPT in {16, 24, 32} and rings per block R = kVPT * 256 / n, or 0 if the
// length needs the generic path.
struct RegConfig {
  int vpt = 0, rings = 0;
  FftPlan plan{};
};

RegConfig reg_config(int n, int tableLen) {
  RegConfig c;
  FftPlan p{};
  p.n = n;
  p.tw_stride = tableLen / n;
  int m = n, s = 0;
  while (m % 8 == 0) { p.radix[s++] = 8; m /= 8; }
  while (m % 4 == 0) { p.radix[s++] = 4; m /= 4; }
  while (m % 2 == 0) { p.radix[s++] = 2; m /= 2; }
  while (m % 3 == 0) { p.radix[s++] = 3; m /= 3; }
  if (m != 1 || n < 8) return c;
  p.stages = s;
  for (int vpt : {16, 24, 32}) {
    if ((vpt * 256) % n) continue;
    bool ok = true;
    for (int i = 0; i < s; i++) ok = ok && (vpt % p.radix[i] == 0);
    if (!ok) continue;
    c.vpt = vpt;
    c.rings = vpt * 256 / n;
    c.plan = p;
    return c;
  }
  return c;
}

template <int kVPT>
gsht_status launch_inverse_reg(const gsht_grid* g, const RegConfig& c, int lmax, int is_real,
                               int count, const double* spec, double* out, cudaStream_t s,
                               RingRange rr) {
  const size_t shmem = sizeof(double2) * (kVPT * 256 + kVPT * 32);
  dim3 grid(ring_blocks(rr, c.rings), count);
  auto kr = is_real ? k_fft_inverse_reg<true, kVPT> : k_fft_inverse_reg<false, kVPT>;
  GSHT_CUDA(cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  kr<<<grid, 256, shmem, s>>>(c.plan, c.rings, g->L, lmax, g->n_theta, g->theta_pad, count,
                              reinterpret_cast<const double2*>(spec),
                              reinterpret_cast<const double2*>(g->d_twiddle), out, rr);
  GSHT_LAUNCH_CHECK("k_fft_inverse_reg");
  return GSHT_OK;
}

template <int kVPT>
gsht_status launch_forward_reg(const gsht_grid* g, const RegConfig& c, int lmax, int is_real,
                               int count, const double* in, double* spec, cudaStream_t s,
                               RingRange rr) {
  const size_t shmem = sizeof(double2) * (kVPT * 256 + kVPT * 32);
  dim3 grid(ring_blocks(rr, c.rings), count);
  auto kf = is_real ? k_fft_forward_reg<true, kVPT> : k_fft_forward_reg<false, kVPT>;
  GSHT_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  kf<<<grid, 256, shmem, s>>>(c.plan, c.rings, g->L, lmax, g->n_theta, g->theta_pad, count,
                              in, g->d_weight, reinterpret_cast<const double2*>(g->d_twiddle),
                              reinterpret_cast<double2*>(spec), rr);
  GSHT_LAUNCH_CHECK("k_fft_forward_reg");
  return GSHT_OK;
}

}  // namespace

gsht_status fft_inverse(const gsht_grid* g, int lmax, int is_real, int count,
                        const double* spec, double* out, cudaStream_t s, RingRange rr) {
  rr = resolve(rr, g->n_theta);
  if (rr.jBegin >= rr.jEnd) return GSHT_OK;
  const int N = g->n_phi;
  bool used = false;
  gsht_status st =
      fft_p2(g, is_real ? N / 2 : N, 1, lmax, is_real, count, spec, out, s, &used, rr);
  if (used) return st;
  const RegConfig rc = reg_config(is_real ? N / 2 : N, N);
  if (rc.vpt == 16) return launch_inverse_reg<16>(g, rc, lmax, is_real, count, spec, out, s, rr);
  if (rc.vpt == 24) return launch_inverse_reg<24>(g, rc, lmax, is_real, count, spec, out, s, rr);
  if (rc.vpt == 32) return launch_inverse_reg<32>(g, rc, lmax, is_real, count, spec, out, s, rr);
  const FftPlan plan = make_plan(is_real ? N / 2 : N, N);
  const size_t shmem = sizeof(double2) * 2 * plan.n;
  dim3 grid(rr.jEnd - rr.jBegin, count);
  if (is_real) {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_inverse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_inverse<true><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count,
        reinterpret_cast<const double2*>(spec),
        reinterpret_cast<const double2*>(g->d_twiddle), out, rr);
  } else {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_inverse<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_inverse<false><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count,
        reinterpret_cast<const double2*>(spec),
        reinterpret_cast<const double2*>(g->d_twiddle), out, rr);
  }
  GSHT_LAUNCH_CHECK("k_fft_inverse");
  return GSHT_OK;
}

gsht_status fft_forward(const gsht_grid* g, int lmax, int is_real, int count,
                        const double* in, double* spec, cudaStream_t s, RingRange rr) {
  rr = resolve(rr, g->n_theta);
  if (rr.jBegin >= rr.jEnd) return GSHT_OK;
  const int N = g->n_phi;
  bool used = false;
  gsht_status st = fft_p2(g, is_real ? N / 2 : N, 0, lmax, is_real, count, in, spec, s, &used, rr);
  if (used) return st;
  const RegConfig rc = reg_config(is_real ? N / 2 : N, N);
  if (rc.vpt == 16) return launch_forward_reg<16>(g, rc, lmax, is_real, count, in, spec, s, rr);
  if (rc.vpt == 24) return launch_forward_reg<24>(g, rc, lmax, is_real, count, in, spec, s, rr);
  if (rc.vpt == 32) return launch_forward_reg<32>(g, rc, lmax, is_real, count, in, spec, s, rr);
  const FftPlan plan = make_plan(is_real ? N / 2 : N, N);
  const size_t shmem = sizeof(double2) * 2 * plan.n;
  dim3 grid(rr.jEnd - rr.jBegin, count);
  if (is_real) {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_forward<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_forward<true><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count, in, g->d_weight,
        reinterpret_cast<const double2*>(g->d_twiddle),
        reinterpret_cast<double2*>(spec), rr);
  } else {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_forward<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_forward<false><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count, in, g->d_weight,
        reinterpret_cast<const double2*>(g->d_twiddle),
        reinterpret_cast<double2*>(spec), rr);
  }
  GSHT_LAUNCH_CHECK("k_fft_forward");
  return GSHT_OK;
}

bool fft_spec32_supported(const gsht_grid* g, int is_real) {
  const int n = is_real ? g->n_phi / 2 : g->n_phi;
  return n >= 256 && n <= 4096 && (n & (n - 1)) == 0;
}

// The three-pass kernels with FP32 spectra (unmirrored -m rows); only for the
// ring lengths fft_spec32_supported accepts.
gsht_status fft_spec32(const gsht_grid* g, int dir, int lmax, int is_real, int count,
                       const void* src, void* dst, cudaStream_t s, double* const* fields) {
  RingRange rr = resolve(RingRange{}, g->n_theta);
  rr.fields = fields;
  switch (is_real ? g->n_phi / 2 : g->n_phi) {
    case 256: return launch_p3<256, float2>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 512: return launch_p3<512, float2>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 1024: return launch_p3<1024, float2>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 2048: return launch_p3<2048, float2>(g, dir, lmax, is_real, count, src, dst, s, rr);
    case 4096: return launch_p3<4096, float2>(g, dir, lmax, is_real, count, src, dst, s, rr);
    default: return fail(GSHT_ERR_UNSUPPORTED, "no FP32-spectrum FFT for this ring length");
  }
}

gsht_status fft_inverse32(const gsht_grid* g, int lmax, int is_real, int count, const float* spec,
                          double* out, cudaStream_t s, double* const* fields) {
  return fft_spec32(g, 1, lmax, is_real, count, spec, out, s, fields);
}

gsht_status fft_forward32(const gsht_grid* g, int lmax, int is_real, int count, const double* in,
                          float* spec, cudaStream_t s, double* const* fields) {
  return fft_spec32(g, 0, lmax, is_real, count, in, spec, s, fields);
}

}  // namespace gsht

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

#include "gsht_internal.cuh"

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
    double* __restrict__ out) {
  extern __shared__ double2 smem[];
  const int j = blockIdx.x, f = blockIdx.y;
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
    double2* o = reinterpret_cast<double2*>(out) + ((size_t)f * nTheta + j) * nPhi;
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
    double2* o = reinterpret_cast<double2*>(out + ((size_t)f * nTheta + j) * nPhi);
    for (int k = threadIdx.x; k < M; k += blockDim.x) o[k] = r[k];
  }
}

// Forward: ring values -> weighted spectrum. Block (j, f).
template <bool kReal>
__global__ void __launch_bounds__(256) k_fft_forward(
    FftPlan plan, int L, int lmax, int nTheta, int thetaPad, int count,
    const double* __restrict__ in, const double* __restrict__ weight,
    const double2* __restrict__ tw, double2* __restrict__ spec) {
  extern __shared__ double2 smem[];
  const int j = blockIdx.x, f = blockIdx.y;
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
    const double2* x = reinterpret_cast<const double2*>(in) + ((size_t)f * nTheta + j) * nPhi;
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
    const double2* x = reinterpret_cast<const double2*>(in + ((size_t)f * nTheta + j) * nPhi);
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
    double* __restrict__ out) {
  extern __shared__ double2 smem[];
  const int j0 = blockIdx.x * R, f = blockIdx.y;
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
    if (j >= nTheta) continue;
    if (!kReal) {
      reinterpret_cast<double2*>(out)[((size_t)f * nTheta + j) * nPhi + k] = smem[pad8(e)];
    } else {
      reinterpret_cast<double2*>(out + ((size_t)f * nTheta + j) * nPhi)[k] = smem[pad8(e)];
    }
  }
}

// Forward, R rings per block.
template <bool kReal, int kVPT>
__global__ void __launch_bounds__(256) k_fft_forward_reg(
    FftPlan plan, int R, int L, int lmax, int nTheta, int thetaPad, int count,
    const double* __restrict__ in, const double* __restrict__ weight,
    const double2* __restrict__ tw, double2* __restrict__ spec) {
  extern __shared__ double2 smem[];
  const int j0 = blockIdx.x * R, f = blockIdx.y;
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
        x = reinterpret_cast<const double2*>(in)[((size_t)f * nTheta + j) * nPhi + k];
      } else {
        x = reinterpret_cast<const double2*>(in + ((size_t)f * nTheta + j) * nPhi)[k];
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
    if (j >= nTheta) continue;
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
                               int count, const double* spec, double* out, cudaStream_t s) {
  const size_t shmem = sizeof(double2) * (kVPT * 256 + kVPT * 32);
  dim3 grid((g->n_theta + c.rings - 1) / c.rings, count);
  auto kr = is_real ? k_fft_inverse_reg<true, kVPT> : k_fft_inverse_reg<false, kVPT>;
  GSHT_CUDA(cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  kr<<<grid, 256, shmem, s>>>(c.plan, c.rings, g->L, lmax, g->n_theta, g->theta_pad, count,
                              reinterpret_cast<const double2*>(spec),
                              reinterpret_cast<const double2*>(g->d_twiddle), out);
  GSHT_LAUNCH_CHECK("k_fft_inverse_reg");
  return GSHT_OK;
}

template <int kVPT>
gsht_status launch_forward_reg(const gsht_grid* g, const RegConfig& c, int lmax, int is_real,
                               int count, const double* in, double* spec, cudaStream_t s) {
  const size_t shmem = sizeof(double2) * (kVPT * 256 + kVPT * 32);
  dim3 grid((g->n_theta + c.rings - 1) / c.rings, count);
  auto kf = is_real ? k_fft_forward_reg<true, kVPT> : k_fft_forward_reg<false, kVPT>;
  GSHT_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  kf<<<grid, 256, shmem, s>>>(c.plan, c.rings, g->L, lmax, g->n_theta, g->theta_pad, count,
                              in, g->d_weight, reinterpret_cast<const double2*>(g->d_twiddle),
                              reinterpret_cast<double2*>(spec));
  GSHT_LAUNCH_CHECK("k_fft_forward_reg");
  return GSHT_OK;
}

}  // namespace

gsht_status fft_inverse(const gsht_grid* g, int lmax, int is_real, int count,
                        const double* spec, double* out, cudaStream_t s) {
  const int N = g->n_phi;
  const RegConfig rc = reg_config(is_real ? N / 2 : N, N);
  if (rc.vpt == 16) return launch_inverse_reg<16>(g, rc, lmax, is_real, count, spec, out, s);
  if (rc.vpt == 24) return launch_inverse_reg<24>(g, rc, lmax, is_real, count, spec, out, s);
  if (rc.vpt == 32) return launch_inverse_reg<32>(g, rc, lmax, is_real, count, spec, out, s);
  const FftPlan plan = make_plan(is_real ? N / 2 : N, N);
  const size_t shmem = sizeof(double2) * 2 * plan.n;
  dim3 grid(g->n_theta, count);
  if (is_real) {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_inverse<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_inverse<true><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count,
        reinterpret_cast<const double2*>(spec),
        reinterpret_cast<const double2*>(g->d_twiddle), out);
  } else {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_inverse<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_inverse<false><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count,
        reinterpret_cast<const double2*>(spec),
        reinterpret_cast<const double2*>(g->d_twiddle), out);
  }
  GSHT_LAUNCH_CHECK("k_fft_inverse");
  return GSHT_OK;
}

gsht_status fft_forward(const gsht_grid* g, int lmax, int is_real, int count,
                        const double* in, double* spec, cudaStream_t s) {
  const int N = g->n_phi;
  const RegConfig rc = reg_config(is_real ? N / 2 : N, N);
  if (rc.vpt == 16) return launch_forward_reg<16>(g, rc, lmax, is_real, count, in, spec, s);
  if (rc.vpt == 24) return launch_forward_reg<24>(g, rc, lmax, is_real, count, in, spec, s);
  if (rc.vpt == 32) return launch_forward_reg<32>(g, rc, lmax, is_real, count, in, spec, s);
  const FftPlan plan = make_plan(is_real ? N / 2 : N, N);
  const size_t shmem = sizeof(double2) * 2 * plan.n;
  dim3 grid(g->n_theta, count);
  if (is_real) {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_forward<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_forward<true><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count, in, g->d_weight,
        reinterpret_cast<const double2*>(g->d_twiddle),
        reinterpret_cast<double2*>(spec));
  } else {
    if (shmem > 48 * 1024)
      GSHT_CUDA(cudaFuncSetAttribute(k_fft_forward<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
    k_fft_forward<false><<<grid, 256, shmem, s>>>(
        plan, g->L, lmax, g->n_theta, g->theta_pad, count, in, g->d_weight,
        reinterpret_cast<const double2*>(g->d_twiddle),
        reinterpret_cast<double2*>(spec));
  }
  GSHT_LAUNCH_CHECK("k_fft_forward");
  return GSHT_OK;
}

}  // namespace gsht

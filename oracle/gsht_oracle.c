/*
 * CPU restatement of the reference's Gauss-Legendre GSHT path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle: tests and the smoke
 * check compare the GPU results against it, and the CPU-baseline leg of the
 * benchmark times it. The product (libgsht_cuda.so) never links, loads or
 * calls it.
 *
 * It restates, function by function, the reference's algorithm:
 *   orc_gl_nodes      GaussQuad::LegendrePolynomial::GaussQuadrature (the
 *                     unpinned da380/GaussQuad@main dependency, CMakeLists.txt
 *                     :37-42; published Newton-on-P_n construction) followed by
 *                     the acos(-x) map of GaussLegendreGrid.h:47-49.
 *   orc_wigner_block  Wigner::Compute for one (n, theta), Ortho normalisation,
 *                     mMax = lMax (Wigner.h:24-95 start values, :317-472
 *                     recurrence, :475-485 normalisation), in the reference's
 *                     GSHIndices<All> block layout (Indexing.h:104-116,143-146).
 *   orc_fft           FFTW's unnormalised DFT conventions, which the reference
 *                     reaches through da380/FFTWpp@main (CMakeLists.txt:45-50):
 *                     sign -1 forward, +1 backward; computed in long double by
 *                     a recursive mixed-radix decimation in time.
 *   orc_forward       GaussLegendreGrid::ForwardTransformation
 *                     (GaussLegendreGrid.h:108-217), accumulating into out.
 *   orc_inverse       GaussLegendreGrid::InverseTransformation
 *                     (GaussLegendreGrid.h:222-321).
 * Pinned against the reference headers compiled in place (oracle/_ref) and
 * against the committed fixtures in tests/golden (generated from that build).
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef long double complex cplx_ld;

static const long double kPiL = 3.141592653589793238462643383279502884L;

/* ---------------------------------------------------------------------- */
/* Gauss-Legendre nodes: Newton on P_n, long double, ascending x.          */
/* ---------------------------------------------------------------------- */
static void legendre_pair(int n, long double x, long double *pn,
                          long double *pnm1) {
  long double p0 = 1, p1 = x;
  for (int k = 1; k < n; k++) {
    long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
    p0 = p1;
    p1 = p2;
  }
  *pn = p1;
  *pnm1 = p0;
}

/* theta[i] = acos(-x_i), w[i] the Gauss weights (GaussLegendreGrid.h:47-49). */
int orc_gl_nodes(int n, double *theta, double *w) {
  if (n < 1) return 1;
  for (int i = 0; i < (n + 1) / 2; i++) {
    long double x = -cosl(kPiL * (i + 0.75L) / (n + 0.5L));
    long double pn, pnm1, dp;
    for (int it = 0; it < 20; it++) {
      legendre_pair(n, x, &pn, &pnm1);
      dp = n * (x * pn - pnm1) / (x * x - 1);
      long double dx = pn / dp;
      x -= dx;
      if (fabsl(dx) <= 1e-19L) break;
    }
    legendre_pair(n, x, &pn, &pnm1);
    dp = n * (x * pn - pnm1) / (x * x - 1);
    if (2 * i + 1 == n) x = 0;
    long double wi = 2 / ((1 - x * x) * dp * dp);
    double xd = (double)x;
    theta[i] = acos(-xd);
    theta[n - 1 - i] = acos(xd);
    w[i] = w[n - 1 - i] = (double)wi;
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Wigner d^l_{mn}(theta), Ortho, one (n, theta) block, GSHIndices<All>.   */
/* ---------------------------------------------------------------------- */
typedef struct {
  double logSinHalf, logCosHalf;
  int atLeft, atRight;
} wig_args; /* WignerDetails::Arguments, Wigner.h:24-50 */

static wig_args make_args(double theta) {
  wig_args a;
  double s = sin(0.5 * theta), c = cos(0.5 * theta);
  a.atLeft = s < DBL_MIN;
  a.atRight = c < DBL_MIN;
  a.logSinHalf = a.atLeft ? 0.0 : log(s);
  a.logCosHalf = a.atRight ? 0.0 : log(c);
  return a;
}

/* WignerMinOrder, Wigner.h:52-80. */
static double min_order(int l, int n, const wig_args *a) {
  if (l == 0) return 1.0;
  if (a->atLeft) return n == -l ? 1.0 : 0.0;
  if (a->atRight) return n == l ? 1.0 : 0.0;
  double fl = l, fn = n;
  return exp(0.5 * (lgamma(2 * fl + 1) - lgamma(fl - fn + 1) -
                    lgamma(fl + fn + 1)) +
             (fl + fn) * a->logSinHalf + (fl - fn) * a->logCosHalf);
}

static double minus_one_pow(int k) { return (k % 2) ? -1.0 : 1.0; }

/* WignerMaxOrder / MinUpperIndex / MaxUpperIndex, Wigner.h:82-95. */
static double max_order(int l, int n, const wig_args *a) {
  return minus_one_pow(n + l) * min_order(l, -n, a);
}
static double min_upper(int l, int m, const wig_args *a) {
  return max_order(l, -m, a);
}
static double max_upper(int l, int m, const wig_args *a) {
  return min_order(l, -m, a);
}

/* Offset of degree l in a GSHIndices<All>(L, L, n) block (Indexing.h:104-116). */
static long off_all(int l, int n) { return (long)l * l - (long)n * n; }

/* Writes the block d[l][m], l = |n|..L, m = -l..l, at out[off_all(l,n)+m+l].
 * Follows Wigner::Compute (Wigner.h:317-486) with mMax = lMax = L. */
int orc_wigner_block(int L, int n, double theta, double *out) {
  const int na = abs(n);
  if (L < 0 || na > L) return 1;
  const int nsq = 2 * L + 2;
  double *sq = (double *)malloc(sizeof(double) * nsq);
  double *sqi = (double *)malloc(sizeof(double) * nsq);
  for (int k = 0; k < nsq; k++) { /* PreCompute, Wigner.h:289-303 */
    sq[k] = sqrt((double)k);
    sqi[k] = sq[k] > 0 ? 1.0 / sq[k] : 0.0;
  }
  const wig_args a = make_args(theta);
  const double cs = cos(theta);
#define D(l, m) out[off_all((l), n) + (m) + (l)]
  { /* l == |n|: closed forms (Wigner.h:330-344) */
    const int l = na;
    for (int m = -l; m <= l; m++)
      D(l, m) = n >= 0 ? max_upper(l, m, &a) : min_upper(l, m, &a);
  }
  if (na < L) { /* l == |n|+1 (Wigner.h:347-383) */
    const int l = na + 1;
    D(l, -l) = min_order(l, n, &a);
    const double alpha = (2 * l - 1) * l * cs * sqi[l + na];
    const double beta = (n < 0 ? -1 : 1) * (2 * l - 1) * sqi[l + na];
    for (int m = -na; m <= na; m++) {
      const double f1 = (alpha - beta * m) * sqi[l - m] * sqi[l + m];
      D(l, m) = f1 * D(l - 1, m);
    }
    D(l, l) = max_order(l, n, &a);
  }
  /* Products are associated left to right exactly as the reference writes
   * them, so that the restatement reproduces its rounding. */
  for (int l = na + 2; l <= L; l++) { /* Wigner.h:386-472 */
    D(l, -l) = min_order(l, n, &a);
    {
      const int m = -l + 1;
      const double f1 = (2 * l - 1) * (l * (l - 1) * cs - m * n) *
                        sqi[l - n] * sqi[l + n] * sqi[l - m] * sqi[l + m] /
                        (double)(l - 1);
      D(l, m) = f1 * D(l - 1, m);
    }
    const double alpha = (2 * l - 1) * l * cs * sqi[l - n] * sqi[l + n];
    const double beta =
        (2 * l - 1) * n * sqi[l - n] * sqi[l + n] / (double)(l - 1);
    const double gamma = l * sq[l - 1 - n] * sq[l - 1 + n] * sqi[l - n] *
                         sqi[l + n] / (double)(l - 1);
    for (int m = -l + 2; m <= l - 2; m++) {
      const double denom = sqi[l - m] * sqi[l + m];
      const double f1 = (alpha - beta * m) * denom;
      const double f2 = gamma * sq[l - 1 - m] * sq[l - 1 + m] * denom;
      D(l, m) = f1 * D(l - 1, m) - f2 * D(l - 2, m);
    }
    {
      const int m = l - 1;
      const double f1 = (2 * l - 1) * (l * (l - 1) * cs - m * n) *
                        sqi[l - n] * sqi[l + n] * sqi[l - m] * sqi[l + m] /
                        (double)(l - 1);
      D(l, m) = f1 * D(l - 1, m);
    }
    D(l, l) = max_order(l, n, &a);
  }
  { /* Ortho normalisation, Wigner.h:475-485 */
    const double factor = (double)(1.0L / sqrtl(kPiL)) / 2.0;
    for (int l = na; l <= L; l++) {
      const double s = factor * sqrt((double)(2 * l + 1));
      for (int m = -l; m <= l; m++) D(l, m) = s * D(l, m);
    }
  }
#undef D
  free(sq);
  free(sqi);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Unnormalised DFT, FFTW conventions, long double mixed radix.           */
/* ---------------------------------------------------------------------- */
/* out[k] = sum_{j<n} in[j*stride] * tw[(j*k*tws) % N], tw[t] = e^{sign 2 pi i t/N} */
static void dft_rec(cplx_ld *out, const cplx_ld *in, size_t n, size_t stride,
                    const cplx_ld *tw, size_t N, size_t tws, cplx_ld *tmp) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  size_t p = 2;
  while (n % p) p++;
  const size_t m = n / p;
  for (size_t q = 0; q < p; q++)
    dft_rec(out + q * m, in + q * stride, m, stride * p, tw, N, tws * p, tmp);
  for (size_t k = 0; k < m; k++) {
    for (size_t q = 0; q < p; q++)
      tmp[q] = out[q * m + k] * tw[(q * k * tws) % N];
    for (size_t r = 0; r < p; r++) {
      cplx_ld s = 0;
      for (size_t q = 0; q < p; q++) s += tmp[q] * tw[(q * r * m * tws) % N];
      out[k + r * m] = s;
    }
    /* All p inputs of this k were read into tmp before any output was
     * written, and the outputs land on the same p slots. */
  }
}

/* In-place transform of n complex doubles (interleaved); sign -1 or +1. */
void orc_fft(int n, int sign, double *x) {
  if (n <= 1) return;
  cplx_ld *in = (cplx_ld *)malloc(sizeof(cplx_ld) * n);
  cplx_ld *out = (cplx_ld *)malloc(sizeof(cplx_ld) * n);
  cplx_ld *tw = (cplx_ld *)malloc(sizeof(cplx_ld) * n);
  cplx_ld *tmp = (cplx_ld *)malloc(sizeof(cplx_ld) * n);
  for (int t = 0; t < n; t++) {
    long double a = 2 * kPiL * t / n;
    tw[t] = cosl(a) + (sign < 0 ? -1.0L : 1.0L) * sinl(a) * I;
    in[t] = x[2 * t] + x[2 * t + 1] * I;
  }
  dft_rec(out, in, (size_t)n, 1, tw, (size_t)n, 1, tmp);
  for (int t = 0; t < n; t++) {
    x[2 * t] = (double)creall(out[t]);
    x[2 * t + 1] = (double)cimagl(out[t]);
  }
  free(in);
  free(out);
  free(tw);
  free(tmp);
}

/* Size of GSHIndices<All> / <NonNegative>(lmax, lmax, n) (Indexing.h:148-150). */
long orc_size_all(int lmax, int n) {
  return (long)(lmax + 1) * (lmax + 1) - (long)n * n;
}
long orc_size_nonneg(int lmax, int n) {
  const long na = labs((long)n);
  return (long)(lmax + 1) * (lmax + 2) / 2 - na * (na + 1) / 2;
}
static long off_nonneg(int l, int n) {
  const long na = labs((long)n);
  return (long)l * (l + 1) / 2 - na * (na + 1) / 2;
}

/* ---------------------------------------------------------------------- */
/* ForwardTransformation, GaussLegendreGrid.h:108-217 (out += ...).        */
/* in: nTheta x nPhi ring-major grid (real, or complex interleaved);       */
/* out: coefficients, complex interleaved.                                 */
/* ---------------------------------------------------------------------- */
int orc_forward(int L, int lmax, int n, int isReal, const double *in,
                double *out) {
  if (L < 1 || lmax < 0 || lmax > L || abs(n) > lmax) return 1;
  const double invSqrtPi2 = (double)(1.0L / sqrtl(kPiL)) / 2.0;
  if (lmax == 0) { /* :136-140 */
    out[0] = (isReal ? in[0] : in[0]) * invSqrtPi2;
    out[1] = isReal ? 0.0 : in[1] * invSqrtPi2;
    return 0;
  }
  const int nTheta = L + 1, nPhi = 2 * L;
  double *theta = (double *)malloc(sizeof(double) * nTheta);
  double *wq = (double *)malloc(sizeof(double) * nTheta);
  double *d = (double *)malloc(sizeof(double) * orc_size_all(L, n));
  double *F = (double *)malloc(sizeof(double) * 2 * nPhi);
  orc_gl_nodes(nTheta, theta, wq);
  const double scale = (double)(2 * kPiL) / nPhi; /* :144-145 */
  for (int it = 0; it < nTheta; it++) {
    for (int k = 0; k < nPhi; k++) { /* FFT the ring, :165-174 */
      const long g = (long)it * nPhi + k;
      F[2 * k] = isReal ? in[g] : in[2 * g];
      F[2 * k + 1] = isReal ? 0.0 : in[2 * g + 1];
    }
    orc_fft(nPhi, -1, F);
    orc_wigner_block(L, n, theta[it], d);
    const double w = wq[it] * scale; /* :177-178 */
    for (int l = abs(n); l <= lmax; l++) {
      for (int m = isReal ? 0 : -l; m <= l; m++) {
        const double dv = d[off_all(l, n) + m + l];
        const int bin = m >= 0 ? m : nPhi + m; /* :189-206 */
        const long o = isReal ? off_nonneg(l, n) + m : off_all(l, n) + m + l;
        out[2 * o] += dv * F[2 * bin] * w;
        out[2 * o + 1] += dv * F[2 * bin + 1] * w;
      }
    }
    if (!isReal && lmax == L) { /* zero the (L, L) coefficient, :209-215 */
      const long last = orc_size_all(lmax, n) - 1;
      out[2 * last] = 0.0;
      out[2 * last + 1] = 0.0;
    }
  }
  free(theta);
  free(wq);
  free(d);
  free(F);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* InverseTransformation, GaussLegendreGrid.h:222-321.                     */
/* ---------------------------------------------------------------------- */
int orc_inverse(int L, int lmax, int n, int isReal, const double *in,
                double *out) {
  if (L < 1 || lmax < 0 || lmax > L || abs(n) > lmax) return 1;
  if (lmax == 0) { /* :251-260 */
    const double f = 2.0 / ((double)(1.0L / sqrtl(kPiL)));
    if (isReal) {
      out[0] = in[0] * f;
    } else {
      out[0] = in[0] * f;
      out[1] = in[1] * f;
    }
    return 0;
  }
  const int nTheta = L + 1, nPhi = 2 * L;
  double *theta = (double *)malloc(sizeof(double) * nTheta);
  double *wq = (double *)malloc(sizeof(double) * nTheta);
  double *d = (double *)malloc(sizeof(double) * orc_size_all(L, n));
  double *G = (double *)malloc(sizeof(double) * 2 * nPhi);
  orc_gl_nodes(nTheta, theta, wq);
  for (int it = 0; it < nTheta; it++) {
    memset(G, 0, sizeof(double) * 2 * nPhi); /* :282 */
    orc_wigner_block(L, n, theta[it], d);
    for (int l = abs(n); l <= lmax; l++) { /* :292-312 */
      for (int m = isReal ? 0 : -l; m <= l; m++) {
        const double dv = d[off_all(l, n) + m + l];
        const int bin = m >= 0 ? m : nPhi + m;
        const long o = isReal ? off_nonneg(l, n) + m : off_all(l, n) + m + l;
        G[2 * bin] += in[2 * o] * dv;
        G[2 * bin + 1] += in[2 * o + 1] * dv;
      }
    }
    if (isReal) {
      /* c2r: Hermitian extension of bins 0..nPhi/2, imaginary parts of bin 0
       * and bin nPhi/2 ignored (FFTW convention). */
      G[1] = 0.0;
      G[2 * L + 1] = 0.0;
      for (int k = 1; k < L; k++) {
        G[2 * (nPhi - k)] = G[2 * k];
        G[2 * (nPhi - k) + 1] = -G[2 * k + 1];
      }
    }
    orc_fft(nPhi, +1, G); /* :314-319 */
    for (int k = 0; k < nPhi; k++) {
      const long g = (long)it * nPhi + k;
      if (isReal) {
        out[g] = G[2 * k];
      } else {
        out[2 * g] = G[2 * k];
        out[2 * g + 1] = G[2 * k + 1];
      }
    }
  }
  free(theta);
  free(wq);
  free(d);
  free(G);
  return 0;
}

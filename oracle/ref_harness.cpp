// C-ABI harness over the UNMODIFIED reference headers (GSHTrans/Core), compiled
// in place from the reference tree with the FFTWpp/GaussQuad stand-ins in
// oracle/shim. TEST INFRASTRUCTURE ONLY: the product never links this; tests,
// the smoke check and the CPU baseline leg of the benchmark load it as the
// checker / reference arm.
//
// Every entry point forwards to the reference's own methods:
//   GaussLegendreGrid ctor                 GaussLegendreGrid.h:38-73
//   ForwardTransformation (+= semantics)   GaussLegendreGrid.h:108-217
//   InverseTransformation                  GaussLegendreGrid.h:222-321
//   Wigner table views operator[](n, iθ)   Wigner.h:241-244
//   CoLatitudes / CoLatitudeWeights        GaussLegendreGrid.h:89-92
// Real = double or long double; long double results are rounded to double on
// the way out (they serve as the accuracy yardstick).
#include <GSHTrans/Core>
#include <omp.h>

#include <algorithm>
#include <complex>
#include <cstdint>
#include <memory>
#include <mutex>
#include <numbers>
#include <span>
#include <vector>

namespace {

using namespace GSHTrans;

struct GridHolderBase {
  virtual ~GridHolderBase() = default;
  virtual int NTheta() const = 0;
  virtual int NPhi() const = 0;
  virtual void Nodes(double* theta, double* w) const = 0;
  virtual int Forward(int lmax, int n, int isReal, const double* in,
                      double* out) const = 0;
  virtual int Inverse(int lmax, int n, int isReal, const double* in,
                      double* out) const = 0;
  virtual long WignerBlock(int n, int iTheta, double* out) const = 0;
};

template <typename Real, typename MRange, typename NRange>
struct GridHolder final : GridHolderBase {
  using Grid = GaussLegendreGrid<Real, MRange, NRange>;
  using Complex = std::complex<Real>;
  using Table = Wigner<Real, Ortho, MRange, NRange, Multiple, ColumnMajor>;
  Grid grid;
  // A second table with the grid's own template arguments, so that host-side
  // views of d^l_{mn}(θ_j) can be returned (the grid keeps its table
  // private). Built on first use only: it doubles the memory.
  mutable std::unique_ptr<Table> wigner;
  mutable std::once_flag wignerOnce;
  int lMax;
  int nMax;

  GridHolder(int l, int nMaxIn)
      : grid(l, nMaxIn, FFTWpp::Estimate), lMax{l}, nMax{nMaxIn} {}

  int NTheta() const override {
    return static_cast<int>(grid.NumberOfCoLatitudes());
  }
  int NPhi() const override {
    return static_cast<int>(grid.NumberOfLongitudes());
  }
  void Nodes(double* theta, double* w) const override {
    int i = 0;
    for (auto t : grid.CoLatitudes()) theta[i++] = static_cast<double>(t);
    i = 0;
    for (auto x : grid.CoLatitudeWeights()) w[i++] = static_cast<double>(x);
  }

  bool ValidN(int n) const {
    for (auto k : grid.UpperIndices())
      if (k == n) return true;
    return false;
  }

  // Runs fn(span) over `count` values of type T viewing the double buffer
  // `buf` (complex values interleaved re/im). For Real == double the span
  // aliases the caller's buffer; for long double the values are staged.
  template <typename T, typename Fn>
  static void WithSpan(double* buf, std::size_t count, bool copyIn,
                       bool copyOut, Fn&& fn) {
    if constexpr (std::same_as<Real, double>) {
      auto span = std::span<T>(reinterpret_cast<T*>(buf), count);
      fn(span);
    } else {
      constexpr std::size_t w = sizeof(T) / sizeof(Real);
      std::vector<T> stage(count);
      auto* raw = reinterpret_cast<Real*>(stage.data());
      if (copyIn)
        for (std::size_t i = 0; i < count * w; i++) raw[i] = buf[i];
      auto span = std::span<T>(stage);
      fn(span);
      if (copyOut)
        for (std::size_t i = 0; i < count * w; i++)
          buf[i] = static_cast<double>(raw[i]);
    }
  }

  int Forward(int lmax, int n, int isReal, const double* in,
              double* out) const override {
    if (lmax < 0 || lmax > lMax || std::abs(n) > lmax || !ValidN(n)) return 1;
    const auto fieldSize = static_cast<std::size_t>(grid.FieldSize());
    auto* inMut = const_cast<double*>(in);
    if (isReal) {
      const auto outSize = static_cast<std::size_t>(
          GSHIndices<NonNegative>(lmax, lmax, n).Size());
      WithSpan<Real>(inMut, fieldSize, true, false, [&](auto inSpan) {
        WithSpan<Complex>(out, outSize, true, true, [&](auto outSpan) {
          grid.ForwardTransformation(lmax, n, std::span<const Real>(inSpan),
                                     outSpan);
        });
      });
      return 0;
    }
    if constexpr (!std::same_as<MRange, All>) {
      return 2;
    } else {
      const auto outSize =
          static_cast<std::size_t>(GSHIndices<All>(lmax, lmax, n).Size());
      WithSpan<Complex>(inMut, fieldSize, true, false, [&](auto inSpan) {
        WithSpan<Complex>(out, outSize, true, true, [&](auto outSpan) {
          grid.ForwardTransformation(lmax, n, std::span<const Complex>(inSpan),
                                     outSpan);
        });
      });
      return 0;
    }
  }

  int Inverse(int lmax, int n, int isReal, const double* in,
              double* out) const override {
    if (lmax < 0 || lmax > lMax || std::abs(n) > lmax || !ValidN(n)) return 1;
    const auto fieldSize = static_cast<std::size_t>(grid.FieldSize());
    auto* inMut = const_cast<double*>(in);
    if (isReal) {
      const auto inSize = static_cast<std::size_t>(
          GSHIndices<NonNegative>(lmax, lmax, n).Size());
      WithSpan<Complex>(inMut, inSize, true, false, [&](auto inSpan) {
        WithSpan<Real>(out, fieldSize, true, true, [&](auto outSpan) {
          grid.InverseTransformation(lmax, n, std::span<const Complex>(inSpan),
                                     outSpan);
        });
      });
      return 0;
    }
    if constexpr (!std::same_as<MRange, All>) {
      return 2;
    } else {
      const auto inSize =
          static_cast<std::size_t>(GSHIndices<All>(lmax, lmax, n).Size());
      WithSpan<Complex>(inMut, inSize, true, false, [&](auto inSpan) {
        WithSpan<Complex>(out, fieldSize, true, true, [&](auto outSpan) {
          grid.InverseTransformation(lmax, n, std::span<const Complex>(inSpan),
                                     outSpan);
        });
      });
      return 0;
    }
  }

  long WignerBlock(int n, int iTheta, double* out) const override {
    if (!ValidN(n) || iTheta < 0 || iTheta >= NTheta()) return -1;
    std::call_once(wignerOnce, [this] {
      auto theta = std::vector<Real>(grid.CoLatitudes().begin(),
                                     grid.CoLatitudes().end());
      wigner = std::make_unique<Table>(lMax, lMax, nMax, theta);
    });
    auto d = (*wigner)[n, iTheta];
    long i = 0;
    for (auto x : d) {
      if (out) out[i] = static_cast<double>(x);
      i++;
    }
    return i;
  }
};

template <typename Real>
GridHolderBase* MakeGrid(int lmax, int nmax, int mrange, int nrange) {
  if (mrange == 0) {
    if (nrange == 0) return new GridHolder<Real, All, All>(lmax, nmax);
    if (nrange == 1) return new GridHolder<Real, All, NonNegative>(lmax, nmax);
    return new GridHolder<Real, All, Single>(lmax, nmax);
  }
  if (nrange == 0) return new GridHolder<Real, NonNegative, All>(lmax, nmax);
  if (nrange == 1)
    return new GridHolder<Real, NonNegative, NonNegative>(lmax, nmax);
  return new GridHolder<Real, NonNegative, Single>(lmax, nmax);
}

}  // namespace

extern "C" {

// mrange: 0 All, 1 NonNegative. nrange: 0 All, 1 NonNegative, 2 Single.
void* ref_grid_create(int lmax, int nmax, int mrange, int nrange,
                      int longDouble) {
  if (lmax < 1 || nmax < 0 || nmax > lmax) return nullptr;
  if (longDouble) return MakeGrid<long double>(lmax, nmax, mrange, nrange);
  return MakeGrid<double>(lmax, nmax, mrange, nrange);
}

void ref_grid_destroy(void* h) { delete static_cast<GridHolderBase*>(h); }

int ref_grid_ntheta(void* h) { return static_cast<GridHolderBase*>(h)->NTheta(); }
int ref_grid_nphi(void* h) { return static_cast<GridHolderBase*>(h)->NPhi(); }

void ref_grid_nodes(void* h, double* theta, double* w) {
  static_cast<GridHolderBase*>(h)->Nodes(theta, w);
}

// in: grid values (real, or complex interleaved re/im); out: coefficients,
// complex interleaved, ACCUMULATED into as the reference does.
int ref_forward(void* h, int lmax, int n, int isReal, const double* in,
                double* out) {
  return static_cast<GridHolderBase*>(h)->Forward(lmax, n, isReal, in, out);
}

int ref_inverse(void* h, int lmax, int n, int isReal, const double* in,
                double* out) {
  return static_cast<GridHolderBase*>(h)->Inverse(lmax, n, isReal, in, out);
}

// Copies the reference's table block for (n, iTheta); returns its length
// (out may be null to query the length).
long ref_wigner_block(void* h, int n, int iTheta, double* out) {
  return static_cast<GridHolderBase*>(h)->WignerBlock(n, iTheta, out);
}

// Wigner<Real, Norm, All, All>(lMax, mMax, nMax, theta) for one angle
// (the form used by tests/CheckAdditionTheorem.h:27); writes the blocks for
// n = -nMax..nMax back to back and returns the total length.
long ref_wigner_single(int lmax, int mmax, int nmax, double theta, int fourPi,
                       int longDouble, double* out) {
  auto run = [&](auto tag, auto norm) -> long {
    using Real = decltype(tag);
    using Norm = decltype(norm);
    auto d = Wigner<Real, Norm, All, All>(lmax, mmax, nmax,
                                          static_cast<Real>(theta));
    long i = 0;
    for (auto n : d.UpperIndices()) {
      for (auto x : d[n]) {
        if (out) out[i] = static_cast<double>(x);
        i++;
      }
    }
    return i;
  };
  if (longDouble) {
    return fourPi ? run((long double)0, FourPi{}) : run((long double)0, Ortho{});
  }
  return fourPi ? run(0.0, FourPi{}) : run(0.0, Ortho{});
}

// Reference CPU arm of the benchmark: for each of nfields fields, one
// InverseTransformation then one ForwardTransformation (the reference's own
// round-trip usage, tests/CheckCoeff2Coeff.h:70-75), OpenMP over fields.
// coefIn/coefOut: nfields * coefSize complex; gridScratch: nfields * fieldSize
// (real or complex). Returns 0 on success.
int ref_roundtrip_batch(void* h, int lmax, int n, int isReal, int nfields,
                        const double* coefIn, double* coefOut,
                        double* gridScratch, long coefSize, long fieldSize,
                        int nthreads) {
  auto* g = static_cast<GridHolderBase*>(h);
  const long gridDoubles = fieldSize * (isReal ? 1 : 2);
  int bad = 0;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) reduction(+ : bad)
  for (int f = 0; f < nfields; f++) {
    bad += g->Inverse(lmax, n, isReal, coefIn + 2 * coefSize * f,
                      gridScratch + gridDoubles * f);
    bad += g->Forward(lmax, n, isReal, gridScratch + gridDoubles * f,
                      coefOut + 2 * coefSize * f);
  }
  return bad;
}

int ref_max_threads() { return omp_get_max_threads(); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Transforms at degrees whose whole table does not fit in host memory (lmax
// 2048: 68.8 GB in double, twice that in long double). The reference's own
// Wigner<Real, Ortho, All, Single, Multiple, ColumnMajor> is built on chunks
// of colatitudes and the loops of InverseTransformation
// (GaussLegendreGrid.h:281-320) and ForwardTransformation
// (GaussLegendreGrid.h:163-216) are restated per chunk, in the reference's
// order of operations, so that the results equal those of a whole
// GaussLegendreGrid<Real, All, Single> bit for bit (checked at small
// degrees). The grid's colatitudes and weights come from the same quadrature
// and map as its constructor (GaussLegendreGrid.h:47-49). Real = long double
// is the accuracy yardstick; Real = double reproduces the reference's FP64
// values where the whole grid cannot be built. Both transforms take lmax
// equal to the grid's degree (the whole field) and one upper index n.
// ---------------------------------------------------------------------------
namespace {

template <typename Real>
GaussQuad::Quadrature1D<Real> ChunkedQuadrature(int lmax) {
  auto q = GaussQuad::LegendrePolynomial<Real>{}.GaussQuadrature(lmax + 1);
  q.Transform([](auto x) { return std::acos(-x); },
              [](auto) -> Real { return 1; });
  return q;
}

template <typename Real>
int ChunkedInverseRings(int lmax, int n, int isReal, const double* coef,
                        int nRings, const int* rings, double* out) {
  using Complex = std::complex<Real>;
  using ChunkTable = Wigner<Real, Ortho, All, Single, Multiple, ColumnMajor>;
  if (lmax < 1 || std::abs(n) > lmax || nRings < 1) return 1;
  const auto quad = ChunkedQuadrature<Real>(lmax);
  std::vector<Real> theta(nRings);
  for (int i = 0; i < nRings; i++) {
    if (rings[i] < 0 || rings[i] > lmax) return 1;
    theta[i] = quad.Points()[rings[i]];
  }
  const ChunkTable table(lmax, lmax, n, theta);
  const int nPhi = 2 * lmax;
  const auto size = static_cast<std::size_t>(
      isReal ? GSHIndices<NonNegative>(lmax, lmax, n).Size()
             : GSHIndices<All>(lmax, lmax, n).Size());
  std::vector<Complex> in(size);
  for (std::size_t i = 0; i < size; i++)
    in[i] = Complex(coef[2 * i], coef[2 * i + 1]);

  if (isReal) {
    auto inWork = FFTWpp::vector<Complex>(nPhi / 2 + 1);
    auto outWork = FFTWpp::vector<Real>(nPhi);
    auto plan = FFTWpp::Ranges::Plan(FFTWpp::Ranges::View(inWork),
                                     FFTWpp::Ranges::View(outWork),
                                     FFTWpp::Estimate);
    for (int i = 0; i < nRings; i++) {
      std::ranges::fill(inWork, Complex(0));
      auto d = table[n, i];
      auto inIter = in.begin();
      auto wigIter = d.begin();
      for (auto l : d.Degrees()) {
        auto dl = d[l];
        auto workIter = inWork.begin();
        std::advance(wigIter, l);
        for ([[maybe_unused]] auto m : dl.NonNegativeOrders()) {
          *workIter++ += *inIter++ * *wigIter++;
        }
      }
      plan.Execute();
      for (int k = 0; k < nPhi; k++)
        out[static_cast<std::size_t>(i) * nPhi + k] =
            static_cast<double>(outWork[k]);
    }
    return 0;
  }
  auto inWork = FFTWpp::vector<Complex>(nPhi);
  auto outWork = FFTWpp::vector<Complex>(nPhi);
  auto plan = FFTWpp::Ranges::Plan(FFTWpp::Ranges::View(inWork),
                                   FFTWpp::Ranges::View(outWork),
                                   FFTWpp::Estimate, FFTWpp::Backward);
  for (int i = 0; i < nRings; i++) {
    std::ranges::fill(inWork, Complex(0));
    auto d = table[n, i];
    auto inIter = in.begin();
    auto wigIter = d.begin();
    for (auto l : d.Degrees()) {
      auto dl = d[l];
      auto workIter = std::prev(inWork.end(), l);
      for ([[maybe_unused]] auto m : dl.NegativeOrders()) {
        *workIter++ += *inIter++ * *wigIter++;
      }
      workIter = inWork.begin();
      for ([[maybe_unused]] auto m : dl.NonNegativeOrders()) {
        *workIter++ += *inIter++ * *wigIter++;
      }
    }
    plan.Execute();
    for (int k = 0; k < nPhi; k++) {
      const auto o = 2 * (static_cast<std::size_t>(i) * nPhi + k);
      out[o] = static_cast<double>(outWork[k].real());
      out[o + 1] = static_cast<double>(outWork[k].imag());
    }
  }
  return 0;
}

template <typename Real>
int ChunkedForwardOrders(int lmax, int n, int isReal, const double* grid,
                         int nOrders, const int* orders, int chunk,
                         double* out) {
  using Complex = std::complex<Real>;
  using ChunkTable = Wigner<Real, Ortho, All, Single, Multiple, ColumnMajor>;
  if (lmax < 1 || std::abs(n) > lmax || nOrders < 1 || chunk < 1) return 1;
  std::vector<std::size_t> start(nOrders + 1, 0);
  for (int k = 0; k < nOrders; k++) {
    const int m = orders[k];
    if (std::abs(m) > lmax || (isReal && m < 0)) return 1;
    const int l0 = std::max(std::abs(m), std::abs(n));
    start[k + 1] = start[k] + static_cast<std::size_t>(lmax - l0 + 1);
  }
  std::vector<Complex> acc(start[nOrders], Complex(0));
  const auto quad = ChunkedQuadrature<Real>(lmax);
  const int nTheta = lmax + 1;
  const int nPhi = 2 * lmax;
  const Real scaleFactor = static_cast<Real>(2) * std::numbers::pi_v<Real> /
                           static_cast<Real>(nPhi);

  auto inReal = FFTWpp::vector<Real>(nPhi);
  auto inCplx = FFTWpp::vector<Complex>(nPhi);
  auto outWork = FFTWpp::vector<Complex>(isReal ? nPhi / 2 + 1 : nPhi);
  auto planReal = FFTWpp::Ranges::Plan(FFTWpp::Ranges::View(inReal),
                                       FFTWpp::Ranges::View(outWork),
                                       FFTWpp::Estimate);
  auto planCplx = FFTWpp::Ranges::Plan(FFTWpp::Ranges::View(inCplx),
                                       FFTWpp::Ranges::View(outWork),
                                       FFTWpp::Estimate, FFTWpp::Forward);

  for (int c0 = 0; c0 < nTheta; c0 += chunk) {
    const int cn = std::min(chunk, nTheta - c0);
    std::vector<Real> theta(quad.Points().begin() + c0,
                            quad.Points().begin() + c0 + cn);
    const ChunkTable table(lmax, lmax, n, theta);
    for (int i = 0; i < cn; i++) {
      const int iTheta = c0 + i;
      const auto ring = static_cast<std::size_t>(iTheta) * nPhi;
      if (isReal) {
        for (int k = 0; k < nPhi; k++) inReal[k] = grid[ring + k];
        planReal.Execute();
      } else {
        for (int k = 0; k < nPhi; k++)
          inCplx[k] = Complex(grid[2 * (ring + k)], grid[2 * (ring + k) + 1]);
        planCplx.Execute();
      }
      auto d = table[n, i];
      const Real w = quad.W(iTheta) * scaleFactor;
      for (int k = 0; k < nOrders; k++) {
        const int m = orders[k];
        const int l0 = std::max(std::abs(m), std::abs(n));
        const auto bin = m < 0 ? nPhi + m : m;
        for (int l = l0; l <= lmax; l++) {
          acc[start[k] + (l - l0)] += d[l][m] * outWork[bin] * w;
        }
      }
      if (!isReal) {
        for (int k = 0; k < nOrders; k++)
          if (orders[k] == lmax) acc[start[k + 1] - 1] = 0;
      }
    }
  }
  for (std::size_t i = 0; i < acc.size(); i++) {
    out[2 * i] = static_cast<double>(acc[i].real());
    out[2 * i + 1] = static_cast<double>(acc[i].imag());
  }
  return 0;
}

}  // namespace

extern "C" {

// Colatitudes and weights of the grid of degree lmax (nTheta = lmax + 1
// values each), computed in long double or double and returned as double.
void ref_chunked_nodes(int lmax, int longDouble, double* theta, double* w) {
  auto run = [&](auto q) {
    for (int i = 0; i <= lmax; i++) {
      theta[i] = static_cast<double>(q.Points()[i]);
      w[i] = static_cast<double>(q.W(i));
    }
  };
  if (longDouble) {
    run(ChunkedQuadrature<long double>(lmax));
  } else {
    run(ChunkedQuadrature<double>(lmax));
  }
}

// InverseTransformation on the rings listed in `rings` only
// (GaussLegendreGrid.h:281-320 for each listed iTheta). coef: the packed
// coefficients (GSHIndices<All> for a complex field, <NonNegative> for a real
// one), complex interleaved. out: nRings rings of nPhi = 2 lmax values (real,
// or complex interleaved), in the order of `rings`. Returns 0 on success.
int ref_chunked_inverse_rings(int lmax, int n, int isReal, int longDouble,
                              const double* coef, int nRings, const int* rings,
                              double* out) {
  return longDouble ? ChunkedInverseRings<long double>(lmax, n, isReal, coef,
                                                       nRings, rings, out)
                    : ChunkedInverseRings<double>(lmax, n, isReal, coef,
                                                  nRings, rings, out);
}

// ForwardTransformation restricted to the orders listed in `orders`
// (GaussLegendreGrid.h:163-216: every ring's FFT, weight and table block,
// accumulated over iTheta in ascending order; the table is rebuilt for each
// chunk of `chunk` colatitudes). grid: nTheta x nPhi values (real, or complex
// interleaved). out: for each listed order m in turn, the coefficients
// c_{l,m} for l = max(|m|, |n|)..lmax, complex interleaved; c_{lmax,lmax} is
// zeroed as the reference does for complex fields. Real fields take orders
// m >= 0 only. Returns 0 on success.
int ref_chunked_forward_orders(int lmax, int n, int isReal, int longDouble,
                               const double* grid, int nOrders,
                               const int* orders, int chunk, double* out) {
  return longDouble
             ? ChunkedForwardOrders<long double>(lmax, n, isReal, grid,
                                                 nOrders, orders, chunk, out)
             : ChunkedForwardOrders<double>(lmax, n, isReal, grid, nOrders,
                                            orders, chunk, out);
}

}  // extern "C"

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

#include <complex>
#include <cstdint>
#include <memory>
#include <mutex>
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

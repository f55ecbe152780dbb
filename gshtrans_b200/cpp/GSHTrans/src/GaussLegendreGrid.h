// GaussLegendreGrid on the GPU (reference: GaussLegendreGrid.h:24-333).
// Construction computes the Gauss-Legendre nodes and the Wigner tables of all
// upper indices on the device; the transforms run there (C ABI of
// libgsht_cuda.so). Same template parameters, member names, argument meaning
// and semantics as the reference: ForwardTransformation accumulates into its
// output and zeroes c_{L,L} for complex fields; InverseTransformation
// overwrites the grid values; lMax may be below the grid degree.
#ifndef GSHT_B200_GAUSS_LEGENDRE_GRID_H
#define GSHT_B200_GAUSS_LEGENDRE_GRID_H

#include <complex>
#include <numbers>
#include <ranges>
#include <vector>

#include "Backend.h"
#include "GridBase.h"

namespace GSHTrans {

// Legendre-stage precision of a grid's transforms (an extension of the
// reference interface): FP64 is the drop-in default. Recurrence is FP64 with
// no stored table: the grid keeps only the l-recurrence's start values and
// coefficients, and the transforms generate the Wigner values as they go.
// BF16x3 and Ozaki4 are the ~1e-6 tensor-core forms, Ozaki the FP64-class
// one; Ozaki4 reads the first four slices of the Ozaki table.
enum class Precision {
  FP64 = GSHT_FP64,
  BF16x3 = GSHT_BF16X3,
  Ozaki = GSHT_OZAKI,
  Recurrence = GSHT_RECURRENCE,
  Ozaki4 = GSHT_OZAKI4
};

template <RealFloatingPoint _Real, OrderIndexRange _MRange, IndexRange _NRange>
class GaussLegendreGrid : public GridBase<GaussLegendreGrid<_Real, _MRange, _NRange>> {
  static_assert(std::same_as<_Real, double>,
                "the GPU grid computes in double precision (Real = double)");

 public:
  using Int = std::ptrdiff_t;
  using Real = _Real;
  using Complex = std::complex<Real>;
  using MRange = _MRange;
  using NRange = _NRange;

  GaussLegendreGrid() = default;

  // The reference's third argument is an FFTW planning flag; the GPU FFT
  // keeps no planner state, so any flag value is accepted and ignored.
  template <typename Flag = int>
  GaussLegendreGrid(int lMax, int nMax, Flag = Flag{}) : GaussLegendreGrid(lMax, nMax, Precision::FP64) {}

  // Extension: also build the table form of a tensor-core precision, or
  // (Recurrence) no table at all.
  GaussLegendreGrid(int lMax, int nMax, Precision precision) : _lMax{lMax}, _nMax{nMax}, _prec{precision} {
    unsigned forms = GSHT_FORM_FP64;
    if (precision == Precision::BF16x3) forms |= GSHT_FORM_BF16X3;
    if (precision == Precision::Ozaki || precision == Precision::Ozaki4) forms |= GSHT_FORM_OZAKI;
    if (precision == Precision::Recurrence) forms = GSHT_FORM_RECURRENCE;
    gsht_grid* g = nullptr;
    Backend::Check(gsht_grid_create(lMax, nMax, Backend::RangeCode<MRange>(),
                                    Backend::RangeCode<NRange>(), forms, &g));
    _grid = Backend::GridHandle(g, Backend::GridDeleter{});
    _theta.resize(lMax + 1);
    _weight.resize(lMax + 1);
    Backend::Check(gsht_grid_nodes(g, _theta.data(), _weight.data()));
  }

  // --- GridBase interface (reference :86-103) ---
  Int MaxDegree() const { return _lMax; }
  Int MaxUpperIndex() const { return _nMax; }
  auto CoLatitudes() const { return std::views::all(_theta); }
  auto CoLatitudeWeights() const { return std::views::all(_weight); }
  auto Longitudes() const {
    const Real dPhi = std::numbers::pi_v<Real> / static_cast<Real>(_lMax);
    return std::views::iota(Int{0}, 2 * Int(_lMax)) |
           std::views::transform([dPhi](Int i) { return static_cast<Real>(i) * dPhi; });
  }
  auto LongitudeWeights() const {
    return std::views::repeat(std::numbers::pi_v<Real> / static_cast<Real>(_lMax), 2 * Int(_lMax));
  }

  Precision GetPrecision() const { return _prec; }
  void SetPrecision(Precision p) { _prec = p; }
  gsht_grid* Handle() const { return _grid.get(); }

  // --- transforms (reference :108-217 and :222-321) ---
  template <std::ranges::range InRange, std::ranges::range OutRange>
    requires((std::same_as<_MRange, All> && ComplexFloatingPoint<std::ranges::range_value_t<InRange>>) ||
             RealFloatingPoint<std::ranges::range_value_t<InRange>>) &&
            std::same_as<RemoveComplex<std::ranges::range_value_t<InRange>>, Real> &&
            std::same_as<std::ranges::range_value_t<OutRange>, Complex>
  void ForwardTransformation(Int lMax, Int n, InRange&& in, OutRange& out) const {
    using Scalar = std::ranges::range_value_t<InRange>;
    Run<Scalar>(0, lMax, n, in, out);
  }

  template <std::ranges::range InRange, std::ranges::range OutRange>
    requires((std::same_as<_MRange, All> && ComplexFloatingPoint<std::ranges::range_value_t<OutRange>>) ||
             RealFloatingPoint<std::ranges::range_value_t<OutRange>>) &&
            std::same_as<std::ranges::range_value_t<InRange>, Complex> &&
            std::same_as<RemoveComplex<std::ranges::range_value_t<OutRange>>, Real>
  void InverseTransformation(Int lMax, Int n, InRange&& in, OutRange& out) const {
    using Scalar = std::ranges::range_value_t<OutRange>;
    Run<Scalar>(1, lMax, n, in, out);
  }

 private:
  int _lMax = 0, _nMax = 0;
  Precision _prec = Precision::FP64;
  Backend::GridHandle _grid;
  std::vector<Real> _theta, _weight;

  // Contiguous ranges are passed in place; others are staged through vectors.
  template <typename Scalar, typename InRange, typename OutRange>
  void Run(int dir, Int lMax, Int n, InRange& in, OutRange& out) const {
    constexpr int isReal = RealFloatingPoint<Scalar>;
    using InV = std::remove_cv_t<std::ranges::range_value_t<InRange>>;
    using OutV = std::remove_cv_t<std::ranges::range_value_t<OutRange>>;
    const void* pin = nullptr;
    std::vector<InV> inStage;
    if constexpr (std::ranges::contiguous_range<InRange>) {
      pin = std::ranges::data(in);
    } else {
      inStage.assign(std::ranges::begin(in), std::ranges::end(in));
      pin = inStage.data();
    }
    void* pout = nullptr;
    std::vector<OutV> outStage;
    if constexpr (std::ranges::contiguous_range<OutRange>) {
      pout = std::ranges::data(out);
    } else {
      outStage.assign(std::ranges::begin(out), std::ranges::end(out));
      pout = outStage.data();
    }
    const auto sz = [&](auto& r) { return static_cast<Int>(std::ranges::distance(r)); };
    const Int coef = isReal ? this->RealCoefficientSize(lMax, n) : this->ComplexCoefficientSize(lMax, n);
    const Int field = static_cast<Int>(this->FieldSize());
    if ((dir == 0 && (sz(in) != field || sz(out) != coef)) || (dir == 1 && (sz(in) != coef || sz(out) != field)))
      throw GSHTError(GSHT_ERR_BAD_ARG, "range sizes do not match (lMax, n) and the grid");
    const int prec = static_cast<int>(_prec);
    if (dir == 0)
      Backend::Check(gsht_forward(_grid.get(), int(lMax), int(n), isReal, prec, pin, pout, nullptr));
    else
      Backend::Check(gsht_inverse(_grid.get(), int(lMax), int(n), isReal, prec, pin, pout, nullptr));
    if constexpr (!std::ranges::contiguous_range<OutRange>) std::ranges::copy(outStage, std::ranges::begin(out));
  }
};

}  // namespace GSHTrans

#endif

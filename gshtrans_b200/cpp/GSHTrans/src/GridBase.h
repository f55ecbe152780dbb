// Geometry and size helpers shared by grids (reference: GridBase.h:13-177),
// written against the CRTP interface the reference defines: the derived grid
// provides MaxDegree, MaxUpperIndex, CoLatitudes, CoLatitudeWeights,
// Longitudes and LongitudeWeights.
#ifndef GSHT_B200_GRIDBASE_H
#define GSHT_B200_GRIDBASE_H

#include <cassert>
#include <random>
#include <ranges>

#include "Indexing.h"

namespace GSHTrans {

template <typename Derived_>
class GridBase {
  using Int = std::ptrdiff_t;
  const Derived_& Self() const { return static_cast<const Derived_&>(*this); }

 public:
  // Upper indices of the NRange (All: -nMax..nMax, NonNegative: 0..nMax,
  // Single: nMax only).
  auto MinUpperIndex() const {
    using NR = typename Derived_::NRange;
    const Int nMax = Self().MaxUpperIndex();
    if constexpr (std::same_as<NR, All>) return -nMax;
    else if constexpr (std::same_as<NR, NonNegative>) return Int{0};
    else return nMax;
  }
  auto UpperIndices() const { return std::views::iota(MinUpperIndex(), Int(Self().MaxUpperIndex()) + 1); }

  auto NumberOfCoLatitudes() const { return std::ranges::size(Self().CoLatitudes()); }
  auto CoLatitudeIndices() const { return std::views::iota(Int{0}, Int(NumberOfCoLatitudes())); }
  auto NumberOfLongitudes() const { return std::ranges::size(Self().Longitudes()); }
  auto LongitudeIndices() const { return std::views::iota(Int{0}, Int(NumberOfLongitudes())); }

  auto Points() const { return std::views::cartesian_product(Self().CoLatitudes(), Self().Longitudes()); }
  auto PointIndices() const { return std::views::cartesian_product(CoLatitudeIndices(), LongitudeIndices()); }
  auto Weights() const {
    return std::views::cartesian_product(Self().CoLatitudeWeights(), Self().LongitudeWeights()) |
           std::views::transform([](auto p) { return std::get<0>(p) * std::get<1>(p); });
  }
  template <typename Function>
  auto ProjectFunction(Function f) const {
    return Points() | std::views::transform([f](auto p) { return f(std::get<0>(p), std::get<1>(p)); });
  }

  auto FieldSize() const { return NumberOfCoLatitudes() * NumberOfLongitudes(); }

  auto RealCoefficientSize(Int lMax, Int n) const { return GSHIndices<NonNegative>(lMax, lMax, n).Size(); }
  auto ComplexCoefficientSize(Int lMax, Int n) const { return GSHIndices<All>(lMax, lMax, n).Size(); }
  auto RealCoefficientSize(Int n) const { return RealCoefficientSize(Self().MaxDegree(), n); }
  auto ComplexCoefficientSize(Int n) const { return ComplexCoefficientSize(Self().MaxDegree(), n); }
  auto CoefficientSize(Int lMax, Int n) const { return ComplexCoefficientSize(lMax, n); }
  auto CoefficientSize(Int n) const { return ComplexCoefficientSize(n); }
  auto CoefficientSizeNonNegative(Int lMax, Int n) const { return RealCoefficientSize(lMax, n); }
  auto CoefficientSizeNonNegative(Int n) const { return RealCoefficientSize(n); }

  // Random coefficients with the reference's fixture semantics
  // (GridBase.h:124-172): complex N(0,1) + i N(0,1); for complex fields
  // c_{L,L} = 0 at lmax == L; for real fields Im c_{l,0} = 0 and
  // Im c_{L,L} = 0 at lmax == L.
  template <std::ranges::range Range>
    requires ComplexFloatingPoint<std::ranges::range_value_t<Range>>
  void RandomComplexCoefficient(Int lMax, Int n, Range& range) const {
    using C = std::ranges::range_value_t<Range>;
    assert(Int(std::ranges::size(range)) == ComplexCoefficientSize(lMax, n));
    std::mt19937_64 gen{std::random_device{}()};
    std::normal_distribution<RemoveComplex<C>> dist;
    for (auto& c : range) c = C{dist(gen), dist(gen)};
    if (lMax == Self().MaxDegree()) range[GSHIndices<All>(lMax, lMax, n).Index(lMax, lMax)] = 0;
  }

  template <std::ranges::range Range>
    requires ComplexFloatingPoint<std::ranges::range_value_t<Range>>
  void RandomRealCoefficient(Int lMax, Int n, Range& range) const {
    using C = std::ranges::range_value_t<Range>;
    assert(Int(std::ranges::size(range)) == RealCoefficientSize(lMax, n));
    std::mt19937_64 gen{std::random_device{}()};
    std::normal_distribution<RemoveComplex<C>> dist;
    for (auto& c : range) c = C{dist(gen), dist(gen)};
    const auto idx = GSHIndices<NonNegative>(lMax, lMax, n);
    for (auto l : idx.Degrees()) range[idx.Index(l, 0)].imag(0);
    if (lMax == Self().MaxDegree()) range[idx.Index(lMax, lMax)].imag(0);
  }
};

}  // namespace GSHTrans

#endif

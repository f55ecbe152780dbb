// Wigner d-function tables (reference: Wigner.h:99-486), computed on the GPU.
// The class keeps the reference's template parameters, constructors, index
// queries and views; the values come from gsht_wigner_compute (the same
// three-term recurrence in degree, with exponent-scaled start values, that
// builds the transform tables) and are held in host memory in the
// reference's storage order, so views index exactly as the reference's do.
//
// One deliberate difference: MaxOrder(l) returns min(l, mMax), the largest
// order stored for degree l. The reference returns max(l, mMax)
// (Wigner.h:193), which names orders outside the stored block for l < mMax
// (and so Orders(l) would run past it).
#ifndef GSHT_B200_WIGNER_H
#define GSHT_B200_WIGNER_H

#include <algorithm>
#include <cassert>
#include <cstdlib>
#include <ranges>
#include <vector>

#include "Backend.h"
#include "Views.h"

namespace GSHTrans {

template <RealFloatingPoint _Real, Normalisation _Norm = Ortho, OrderIndexRange _MRange = All,
          IndexRange _NRange = Single, AngleIndexRange _AngleRange = Single,
          WignerStorage _Storage = ColumnMajor>
class Wigner {
  static_assert(std::same_as<_Real, double>, "the GPU tables are computed in double precision");

 public:
  using Int = std::ptrdiff_t;
  using Real = _Real;
  using Norm = _Norm;
  using MRange = _MRange;
  using NRange = _NRange;
  using AngleRange = _AngleRange;
  using Storage = _Storage;

  Wigner() = default;

  template <std::ranges::range Range>
    requires RealFloatingPoint<std::ranges::range_value_t<Range>>
  Wigner(Int lMax, Int mMax, Int nMax, Range&& theta)
      : _lMax{lMax}, _mMax{mMax}, _nMax{nMax}, _nTheta(static_cast<Int>(std::ranges::distance(theta))) {
    assert(lMax >= 0 && mMax >= 0 && nMax >= 0 && nMax <= lMax);
    std::size_t size = 0;
    _offset.reserve(NumberOfUpperIndices() * NumberOfAngles());
    for (auto [n, iTheta] : Indices()) {
      _offset.push_back(size);
      size += GSHIndices<MRange>(_lMax, _mMax, n).Size();
    }
    _data.resize(size);
    ComputeAll(theta);
  }

  Wigner(Int lMax, Int mMax, Int nMax, Real theta)
    requires std::same_as<AngleRange, Single>
      : Wigner(lMax, mMax, nMax, std::vector<Real>{theta}) {}

  Wigner(const Wigner&) = default;
  Wigner(Wigner&&) = default;
  Wigner& operator=(const Wigner&) = default;
  Wigner& operator=(Wigner&&) = default;

  template <std::ranges::range Range>
    requires RealFloatingPoint<std::ranges::range_value_t<Range>>
  void ReCompute(Range&& theta) {
    assert(Int(std::ranges::distance(theta)) == NumberOfAngles());
    ComputeAll(theta);
  }
  void ReCompute(Real theta)
    requires std::same_as<AngleRange, Single>
  {
    ComputeAll(std::vector<Real>{theta});
  }

  // degrees
  auto MinDegree(Int n) const {
    assert(std::abs(n) <= _nMax);
    return std::abs(n);
  }
  auto MinDegree() const
    requires std::same_as<NRange, Single>
  {
    return std::abs(_nMax);
  }
  auto MaxDegree() const { return _lMax; }
  auto Degrees() const
    requires std::same_as<NRange, Single>
  {
    return std::views::iota(MinDegree(), MaxDegree() + 1);
  }
  auto Degrees(Int n) const { return std::views::iota(MinDegree(n), MaxDegree() + 1); }

  // orders
  auto MinOrder(Int l) const {
    assert(l >= 0 && l <= MaxDegree());
    if constexpr (std::same_as<MRange, All>) return -std::min(l, _mMax);
    else return Int{0};
  }
  auto MaxOrder() const { return _mMax; }
  auto MaxOrder(Int l) const { return std::min(l, _mMax); }
  auto Orders(Int l) const { return std::views::iota(MinOrder(l), MaxOrder(l) + 1); }

  // upper indices
  auto MinUpperIndex() const {
    if constexpr (std::same_as<NRange, All>) return -_nMax;
    else if constexpr (std::same_as<NRange, NonNegative>) return Int{0};
    else return _nMax;
  }
  auto MaxUpperIndex() const { return _nMax; }
  auto UpperIndices() const { return std::views::iota(MinUpperIndex(), MaxUpperIndex() + 1); }
  auto NumberOfUpperIndices() const { return MaxUpperIndex() - MinUpperIndex() + 1; }

  // angles
  auto NumberOfAngles() const { return _nTheta; }
  auto AngleIndices() const { return std::views::iota(Int{0}, _nTheta); }

  // (n, iTheta) pairs in storage order.
  auto Indices() const {
    if constexpr (std::same_as<Storage, ColumnMajor>) {
      return std::views::cartesian_product(UpperIndices(), AngleIndices());
    } else {
      return std::views::cartesian_product(AngleIndices(), UpperIndices()) |
             std::views::transform([](auto p) { return std::pair(std::get<1>(p), std::get<0>(p)); });
    }
  }

  // views
  auto operator[](Int n, Int iTheta) const {
    return ConstGSHView<Real, MRange>(MaxDegree(), MaxOrder(), n, &_data[Offset(n, iTheta)]);
  }
  auto operator[](Int n) const
    requires std::same_as<AngleRange, Single> && (!std::same_as<NRange, Single>)
  {
    return operator[](n, 0);
  }
  auto operator[](Int iTheta) const
    requires std::same_as<NRange, Single> && (!std::same_as<AngleRange, Single>)
  {
    return operator[](_nMax, iTheta);
  }
  auto operator[](Int l) const
    requires std::same_as<NRange, Single> && std::same_as<AngleRange, Single>
  {
    return operator[](_nMax, 0)[l];
  }

  // All values in storage order.
  const std::vector<Real>& Data() const { return _data; }

 private:
  Int _lMax = 0, _mMax = 0, _nMax = 0, _nTheta = 0;
  std::vector<Real> _data;
  std::vector<std::size_t> _offset;

  std::size_t Offset(Int n, Int iTheta) const {
    if constexpr (std::same_as<Storage, ColumnMajor>) {
      return _offset[NumberOfAngles() * (n - MinUpperIndex()) + iTheta];
    } else {
      return _offset[NumberOfUpperIndices() * iTheta + (n - MinUpperIndex())];
    }
  }

  template <typename Range>
  void ComputeAll(Range&& thetaRange) {
    std::vector<double> theta(std::ranges::begin(thetaRange), std::ranges::end(thetaRange));
    long count = 0;
    const int norm = std::same_as<Norm, Ortho> ? 0 : 1;
    const int rowMajor = std::same_as<Storage, RowMajor> ? 1 : 0;
    Backend::Check(gsht_wigner_compute(int(_lMax), int(_mMax), int(_nMax), Backend::RangeCode<MRange>(),
                                       Backend::RangeCode<NRange>(), norm, rowMajor, theta.data(),
                                       int(theta.size()), nullptr, &count));
    if (static_cast<std::size_t>(count) != _data.size())
      throw GSHTError(GSHT_ERR_BAD_ARG, "Wigner table size disagrees with the index layout");
    Backend::Check(gsht_wigner_compute(int(_lMax), int(_mMax), int(_nMax), Backend::RangeCode<MRange>(),
                                       Backend::RangeCode<NRange>(), norm, rowMajor, theta.data(),
                                       int(theta.size()), _data.data(), &count));
  }
};

}  // namespace GSHTrans

#endif

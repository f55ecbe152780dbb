// Canonical-component field holding its values on the grid points
// (reference: CanonicalComponentField.h:17-151). Values live in host memory,
// ring-major (nTheta x nPhi) as in the reference, so Data() can be passed
// straight to the grid's transforms; assignments from expressions run on the
// GPU (CanonicalComponentFieldBase).
#ifndef GSHT_B200_CANONICAL_COMPONENT_FIELD_H
#define GSHT_B200_CANONICAL_COMPONENT_FIELD_H

#include <algorithm>
#include <vector>

#include "CanonicalComponentFieldOverloads.h"

namespace GSHTrans {

template <std::ptrdiff_t _N, typename _Grid, RealOrComplexValued _Value>
  requires std::derived_from<_Grid, GridBase<_Grid>>
class CanonicalComponentField;

namespace Internal {
template <std::ptrdiff_t _N, typename _Grid, RealOrComplexValued _Value>
struct Traits<CanonicalComponentField<_N, _Grid, _Value>> {
  using Int = std::ptrdiff_t;
  using Value = _Value;
  using Real = typename _Grid::Real;
  using Complex = typename _Grid::Complex;
  using Scalar = std::conditional_t<std::same_as<Value, RealValued>, Real, Complex>;
  using Writeable = std::true_type;
};
template <std::ptrdiff_t _N, typename _Grid, RealOrComplexValued _Value>
struct IsCanonicalComponentField<CanonicalComponentField<_N, _Grid, _Value>> : std::true_type {};
}  // namespace Internal

template <std::ptrdiff_t _N, typename _Grid, RealOrComplexValued _Value>
  requires std::derived_from<_Grid, GridBase<_Grid>>
class CanonicalComponentField
    : public CanonicalComponentFieldBase<_N, CanonicalComponentField<_N, _Grid, _Value>> {
  using Base = CanonicalComponentFieldBase<_N, CanonicalComponentField<_N, _Grid, _Value>>;
  using T = Internal::Traits<CanonicalComponentField<_N, _Grid, _Value>>;

 public:
  using Value = typename T::Value;
  using Int = typename T::Int;
  using Real = typename T::Real;
  using Complex = typename T::Complex;
  using Scalar = typename T::Scalar;
  using Writeable = typename T::Writeable;

  CanonicalComponentField() = default;

  // Zero values on the grid's points.
  explicit CanonicalComponentField(_Grid& grid) : _grid{&grid}, _data(grid.FieldSize()) {}

  // Values of f(theta, phi) at the grid's points.
  template <typename Function>
    requires ScalarFunctionS2<Function, Real, Scalar>
  CanonicalComponentField(_Grid& grid, Function&& f) : CanonicalComponentField(grid) {
    std::ranges::copy(grid.ProjectFunction(f), _data.begin());
  }

  // Materialises an expression (one GPU pass).
  template <typename Derived>
    requires std::convertible_to<typename Derived::Scalar, Scalar>
  CanonicalComponentField(const CanonicalComponentFieldBase<_N, Derived>& other)
      : CanonicalComponentField(other.Grid()) {
    Base::operator=(other);
  }

  CanonicalComponentField(const CanonicalComponentField&) = default;
  CanonicalComponentField(CanonicalComponentField&&) = default;
  CanonicalComponentField& operator=(const CanonicalComponentField&) = default;
  CanonicalComponentField& operator=(CanonicalComponentField&&) = default;
  using Base::operator=;

  auto& Grid() const { return *_grid; }

  auto operator[](Int iTheta, Int iPhi) const {
    this->CheckPointIndices(iTheta, iPhi);
    return _data[Index(iTheta, iPhi)];
  }
  auto& operator[](Int iTheta, Int iPhi) {
    this->CheckPointIndices(iTheta, iPhi);
    return _data[Index(iTheta, iPhi)];
  }

  auto Data() { return std::views::all(_data); }
  auto Data() const { return std::views::all(_data); }

  // Leaf of an expression program, and the buffer an assignment writes.
  void Emit(Detail::FieldProgram& p) const { p.Load(_data.data(), std::same_as<Value, RealValued>); }
  Scalar* RawData() { return _data.data(); }

 private:
  _Grid* _grid = nullptr;
  std::vector<Scalar> _data;

  Int Index(Int iTheta, Int iPhi) const { return iTheta * Int(this->NumberOfLongitudes()) + iPhi; }
};

template <std::ptrdiff_t N, typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using RealCanonicalComponentField = CanonicalComponentField<N, Grid, RealValued>;
template <std::ptrdiff_t N, typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using ComplexCanonicalComponentField = CanonicalComponentField<N, Grid, ComplexValued>;
template <typename Grid, RealOrComplexValued Value>
  requires std::derived_from<Grid, GridBase<Grid>>
using ScalarField = CanonicalComponentField<0, Grid, Value>;
template <typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using RealScalarField = CanonicalComponentField<0, Grid, RealValued>;
template <typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using ComplexScalarField = CanonicalComponentField<0, Grid, ComplexValued>;

}  // namespace GSHTrans

#endif

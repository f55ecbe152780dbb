// Canonical-component expansion: the coefficients c_lm of one upper index N
// on a grid (reference: CanonicalComponentExpansion.h:36-105 and
// CanonicalComponentExpansionBase.h:14-160). The reference declares the
// container (GSHIndices<MRange>(L, L, N) bookkeeping, complex coefficients,
// element access, assignment and compound operators) but never connects it
// to the grid's transforms; here FromField / ToField run them on the GPU, so
// a user who holds coefficients never handles the packed layout by hand.
//
// Coefficients live in host memory in the packed order of the transforms
// (GSHIndices<All> for complex fields, GSHIndices<NonNegative> for real
// ones), always complex as in the reference.
#ifndef GSHT_B200_CANONICAL_COMPONENT_EXPANSION_H
#define GSHT_B200_CANONICAL_COMPONENT_EXPANSION_H

#include <algorithm>
#include <cassert>
#include <complex>
#include <vector>

#include "../CanonicalComponentField/CanonicalComponentField.h"
#include "../Concepts.h"
#include "../GridBase.h"
#include "../Indexing.h"

namespace GSHTrans {

template <std::ptrdiff_t _N, typename _Grid, RealOrComplexValued _Value>
  requires std::derived_from<_Grid, GridBase<_Grid>>
class CanonicalComponentExpansion
    : public GSHIndices<std::conditional_t<std::same_as<_Value, RealValued>, NonNegative, All>> {
 public:
  using Int = std::ptrdiff_t;
  using Value = _Value;
  using Real = typename _Grid::Real;
  using Complex = typename _Grid::Complex;
  using Scalar = std::conditional_t<std::same_as<Value, RealValued>, Real, Complex>;
  using MRange = std::conditional_t<std::same_as<Value, RealValued>, NonNegative, All>;
  using Field = CanonicalComponentField<_N, _Grid, _Value>;

  CanonicalComponentExpansion() = default;

  // Zero coefficients for degrees |N|..L of the grid (reference :76-79).
  explicit CanonicalComponentExpansion(_Grid& grid)
      : GSHIndices<MRange>(grid.MaxDegree(), grid.MaxDegree(), _N), _grid{&grid}, _data(this->Size()) {}

  // The expansion of a field: its forward transform.
  explicit CanonicalComponentExpansion(const Field& field)
      : CanonicalComponentExpansion(field.Grid()) {
    FromField(field);
  }

  CanonicalComponentExpansion(const CanonicalComponentExpansion&) = default;
  CanonicalComponentExpansion(CanonicalComponentExpansion&&) = default;
  CanonicalComponentExpansion& operator=(const CanonicalComponentExpansion&) = default;
  CanonicalComponentExpansion& operator=(CanonicalComponentExpansion&&) = default;

  auto UpperIndex() const { return _N; }
  auto& Grid() const { return *_grid; }

  // Element access by degree and order (reference :64-67).
  auto operator[](Int l, Int m) const { return _data[this->Index(l, m)]; }
  auto& operator[](Int l, Int m) { return _data[this->Index(l, m)]; }

  auto Data() { return std::views::all(_data); }
  auto Data() const { return std::views::all(_data); }

  // Coefficients of `field`, replacing the current ones (the grid's forward
  // transform, which adds into its output, runs on zeroed coefficients).
  CanonicalComponentExpansion& FromField(const Field& field) {
    std::fill(_data.begin(), _data.end(), Complex{});
    _grid->ForwardTransformation(this->MaxDegree(), _N, field.Data(), _data);
    return *this;
  }

  // The field with these coefficients (inverse transform).
  Field ToField() const {
    Field f(*_grid);
    auto values = f.Data();
    _grid->InverseTransformation(this->MaxDegree(), _N, _data, values);
    return f;
  }

  // Assignment and compound operators (reference Base :77-160).
  CanonicalComponentExpansion& operator+=(const CanonicalComponentExpansion& o) {
    assert(o.MaxDegree() == this->MaxDegree());
    for (Int i = 0; i < Int(_data.size()); i++) _data[i] += o._data[i];
    return *this;
  }
  CanonicalComponentExpansion& operator-=(const CanonicalComponentExpansion& o) {
    assert(o.MaxDegree() == this->MaxDegree());
    for (Int i = 0; i < Int(_data.size()); i++) _data[i] -= o._data[i];
    return *this;
  }
  CanonicalComponentExpansion& operator*=(Scalar s) {
    for (auto& c : _data) c *= s;
    return *this;
  }
  CanonicalComponentExpansion& operator/=(Scalar s) {
    for (auto& c : _data) c /= s;
    return *this;
  }

 private:
  _Grid* _grid = nullptr;
  std::vector<Complex> _data;
};

template <std::ptrdiff_t N, typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using RealCanonicalComponentExpansion = CanonicalComponentExpansion<N, Grid, RealValued>;
template <std::ptrdiff_t N, typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using ComplexCanonicalComponentExpansion = CanonicalComponentExpansion<N, Grid, ComplexValued>;
template <typename Grid, RealOrComplexValued Value>
  requires std::derived_from<Grid, GridBase<Grid>>
using ScalarExpansion = CanonicalComponentExpansion<0, Grid, Value>;
template <typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using RealScalarExpansion = CanonicalComponentExpansion<0, Grid, RealValued>;
template <typename Grid>
  requires std::derived_from<Grid, GridBase<Grid>>
using ComplexScalarExpansion = CanonicalComponentExpansion<0, Grid, ComplexValued>;

}  // namespace GSHTrans

#endif

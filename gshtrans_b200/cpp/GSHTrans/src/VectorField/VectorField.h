// Vector fields in canonical components and their expansions (reference:
// src/VectorField/, whose files the reference's GSHTrans/Field header leaves
// commented out). Component alpha = -1, 0, +1 of a vector field is a
// complex CanonicalComponentField of upper index alpha (CanonicalVector.h
// :13-22), so each one transforms with the grid's table of n = alpha, and
// every operation below runs on the components' existing GPU paths: the
// compound operators one fused pass per component, InnerProduct and
// DualityProduct (VectorFieldOverloads.h:240-288) one fused pass over all
// six components, the expansion's transforms one call per component.
// Complex-valued only: the reference's real-valued branch treats the
// components as plain reals, which has no transform counterpart.
#ifndef GSHT_B200_VECTOR_FIELD_H
#define GSHT_B200_VECTOR_FIELD_H

#include <cassert>
#include <ranges>

#include "../CanonicalComponentExpansion/CanonicalComponentExpansion.h"
#include "../CanonicalComponentField/CanonicalComponentField.h"

namespace GSHTrans {

template <typename _Grid>
  requires std::derived_from<_Grid, GridBase<_Grid>>
class ComplexVectorField {
 public:
  using Int = std::ptrdiff_t;
  using Complex = typename _Grid::Complex;
  template <int Alpha>
    requires(Alpha >= -1 && Alpha <= 1)
  using ComponentField = CanonicalComponentField<Alpha, _Grid, ComplexValued>;

  ComplexVectorField() = default;
  explicit ComplexVectorField(_Grid& grid) : _m{grid}, _z{grid}, _p{grid} {}

  static constexpr auto CanonicalIndices() { return std::ranges::views::iota(-1, 2); }
  static void CheckCanonicalIndices(Int alpha) { assert(alpha >= -1 && alpha <= 1); }

  auto& Grid() const { return _z.Grid(); }

  template <int Alpha>
  auto& Component() {
    if constexpr (Alpha == -1) return _m;
    else if constexpr (Alpha == 0) return _z;
    else return _p;
  }
  template <int Alpha>
  const auto& Component() const {
    if constexpr (Alpha == -1) return _m;
    else if constexpr (Alpha == 0) return _z;
    else return _p;
  }

  // Values (VectorFieldBase.h: operator[](alpha, iTheta, iPhi)).
  Complex operator[](Int alpha, Int iTheta, Int iPhi) const {
    CheckCanonicalIndices(alpha);
    return alpha < 0 ? _m[iTheta, iPhi] : (alpha == 0 ? _z[iTheta, iPhi] : _p[iTheta, iPhi]);
  }
  Complex& operator[](Int alpha, Int iTheta, Int iPhi) {
    CheckCanonicalIndices(alpha);
    return alpha < 0 ? _m[iTheta, iPhi] : (alpha == 0 ? _z[iTheta, iPhi] : _p[iTheta, iPhi]);
  }

  // Compound operators with vector fields, scalars and scalar fields.
  ComplexVectorField& operator+=(const ComplexVectorField& o) {
    _m += o._m;
    _z += o._z;
    _p += o._p;
    return *this;
  }
  ComplexVectorField& operator-=(const ComplexVectorField& o) {
    _m -= o._m;
    _z -= o._z;
    _p -= o._p;
    return *this;
  }
  ComplexVectorField& operator*=(Complex s) {
    _m *= s;
    _z *= s;
    _p *= s;
    return *this;
  }
  ComplexVectorField& operator/=(Complex s) {
    _m /= s;
    _z /= s;
    _p /= s;
    return *this;
  }
  template <typename D>
    requires std::convertible_to<typename D::Scalar, Complex>
  ComplexVectorField& operator*=(const CanonicalComponentFieldBase<0, D>& f) {
    _m = _m * f;
    _z = _z * f;
    _p = _p * f;
    return *this;
  }
  template <typename D>
    requires std::convertible_to<typename D::Scalar, Complex>
  ComplexVectorField& operator/=(const CanonicalComponentFieldBase<0, D>& f) {
    _m = _m / f;
    _z = _z / f;
    _p = _p / f;
    return *this;
  }

 private:
  ComponentField<-1> _m;
  ComponentField<0> _z;
  ComponentField<1> _p;
};

// sum_alpha conj(u_alpha) v_alpha, a scalar field (reference
// VectorFieldOverloads.h:240-252). conj(u_alpha) carries upper index -alpha
// here, so every term has upper index 0.
template <typename Grid>
auto InnerProduct(const ComplexVectorField<Grid>& u, const ComplexVectorField<Grid>& v) {
  using M = CanonicalComponentField<-1, Grid, ComplexValued>;
  using Z = CanonicalComponentField<0, Grid, ComplexValued>;
  using P = CanonicalComponentField<1, Grid, ComplexValued>;
  CanonicalComponentField<0, Grid, ComplexValued> w(u.Grid());
  w = CanonicalComponentFieldUnary<GSHT_OP_CONJ, 1, M>(u.template Component<-1>()) *
          v.template Component<-1>() +
      CanonicalComponentFieldUnary<GSHT_OP_CONJ, 0, Z>(u.template Component<0>()) *
          v.template Component<0>() +
      CanonicalComponentFieldUnary<GSHT_OP_CONJ, -1, P>(u.template Component<1>()) *
          v.template Component<1>();
  return w;
}

// -u_{-1} v_{+1} + u_0 v_0 - u_{+1} v_{-1}, a scalar field (reference
// VectorFieldOverloads.h:276-288).
template <typename Grid>
auto DualityProduct(const ComplexVectorField<Grid>& u, const ComplexVectorField<Grid>& v) {
  CanonicalComponentField<0, Grid, ComplexValued> w(u.Grid());
  w = u.template Component<0>() * v.template Component<0>() -
      u.template Component<-1>() * v.template Component<1>() -
      u.template Component<1>() * v.template Component<-1>();
  return w;
}

// The three canonical-component expansions of a vector field.
template <typename _Grid>
  requires std::derived_from<_Grid, GridBase<_Grid>>
class ComplexVectorExpansion {
 public:
  using Field = ComplexVectorField<_Grid>;
  template <int Alpha>
    requires(Alpha >= -1 && Alpha <= 1)
  using ComponentExpansion = CanonicalComponentExpansion<Alpha, _Grid, ComplexValued>;

  ComplexVectorExpansion() = default;
  explicit ComplexVectorExpansion(_Grid& grid) : _m{grid}, _z{grid}, _p{grid} {}
  // Forward transforms of the field's components.
  explicit ComplexVectorExpansion(const Field& u) : ComplexVectorExpansion(u.Grid()) { FromField(u); }

  static constexpr auto CanonicalIndices() { return std::ranges::views::iota(-1, 2); }

  template <int Alpha>
  auto& Component() {
    if constexpr (Alpha == -1) return _m;
    else if constexpr (Alpha == 0) return _z;
    else return _p;
  }
  template <int Alpha>
  const auto& Component() const {
    if constexpr (Alpha == -1) return _m;
    else if constexpr (Alpha == 0) return _z;
    else return _p;
  }

  ComplexVectorExpansion& FromField(const Field& u) {
    _m.FromField(u.template Component<-1>());
    _z.FromField(u.template Component<0>());
    _p.FromField(u.template Component<1>());
    return *this;
  }
  // Inverse transforms of the three components.
  Field ToField() const {
    Field u(_z.Grid());
    u.template Component<-1>() = _m.ToField();
    u.template Component<0>() = _z.ToField();
    u.template Component<1>() = _p.ToField();
    return u;
  }

 private:
  ComponentExpansion<-1> _m;
  ComponentExpansion<0> _z;
  ComponentExpansion<1> _p;
};

}  // namespace GSHTrans

#endif

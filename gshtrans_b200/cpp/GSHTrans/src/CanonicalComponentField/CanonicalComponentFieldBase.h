// Common base of canonical-component fields and their lazy expressions
// (reference: CanonicalComponentFieldBase.h:14-222). Reading one value
// (operator[]) evaluates the expression at that point on the host, as the
// reference does; assigning an expression to a field (=, +=, -=, *=, /=)
// flattens it into one postfix program that gsht_field_eval runs over every
// grid point in a single GPU kernel.
#ifndef GSHT_B200_CANONICAL_COMPONENT_FIELD_BASE_H
#define GSHT_B200_CANONICAL_COMPONENT_FIELD_BASE_H

#include <concepts>
#include <format>
#include <iostream>
#include <type_traits>

#include "../FieldBase.h"
#include "../GridBase.h"

namespace GSHTrans {

namespace Internal {
// True for fields that own their values; expression nodes hold those by
// reference and other nodes by value, so a stored expression stays valid.
template <typename T>
struct IsCanonicalComponentField : std::false_type {};
template <typename T>
using Hold = std::conditional_t<IsCanonicalComponentField<T>::value, const T&, T>;
}  // namespace Internal

template <std::ptrdiff_t _N, typename _Derived>
class CanonicalComponentFieldBase : public FieldBase<CanonicalComponentFieldBase<_N, _Derived>> {
 public:
  using Int = typename Internal::Traits<_Derived>::Int;
  using Value = typename Internal::Traits<_Derived>::Value;
  using Real = typename Internal::Traits<_Derived>::Real;
  using Complex = typename Internal::Traits<_Derived>::Complex;
  using Scalar = typename Internal::Traits<_Derived>::Scalar;
  using Writeable = typename Internal::Traits<_Derived>::Writeable;

  constexpr auto UpperIndex() const { return _N; }
  auto& Grid() const { return Derived().Grid(); }
  auto Size() const { return this->NumberOfLongitudes() * this->NumberOfCoLatitudes(); }

  auto operator[](Int iTheta, Int iPhi) const { return Derived()[iTheta, iPhi]; }
  auto& operator[](Int iTheta, Int iPhi)
    requires Writeable::value
  {
    return Derived()[iTheta, iPhi];
  }

  // Appends this expression's postfix program.
  void Emit(Detail::FieldProgram& p) const { Derived().Emit(p); }

  // Fused assignment (reference :49-67).
  template <typename D>
    requires Writeable::value && std::convertible_to<typename D::Scalar, Scalar>
  auto& operator=(const CanonicalComponentFieldBase<_N, D>& other) {
    Apply(other, -1);
    return Derived();
  }

  // Compound assignment with a field or expression of the same upper index
  // and with a scalar (reference :69-187).
  template <typename D>
    requires Writeable::value && std::convertible_to<typename D::Scalar, Scalar>
  auto& operator+=(const CanonicalComponentFieldBase<_N, D>& other) {
    Apply(other, GSHT_OP_ADD);
    return Derived();
  }
  template <typename D>
    requires Writeable::value && std::convertible_to<typename D::Scalar, Scalar>
  auto& operator-=(const CanonicalComponentFieldBase<_N, D>& other) {
    Apply(other, GSHT_OP_SUB);
    return Derived();
  }
  template <typename D>
    requires Writeable::value && std::convertible_to<typename D::Scalar, Scalar>
  auto& operator*=(const CanonicalComponentFieldBase<_N, D>& other) {
    Apply(other, GSHT_OP_MUL);
    return Derived();
  }
  template <typename D>
    requires Writeable::value && std::convertible_to<typename D::Scalar, Scalar>
  auto& operator/=(const CanonicalComponentFieldBase<_N, D>& other) {
    Apply(other, GSHT_OP_DIV);
    return Derived();
  }
  auto& operator+=(Scalar s)
    requires Writeable::value
  {
    return ApplyScalar(s, GSHT_OP_ADD);
  }
  auto& operator-=(Scalar s)
    requires Writeable::value
  {
    return ApplyScalar(s, GSHT_OP_SUB);
  }
  auto& operator*=(Scalar s)
    requires Writeable::value
  {
    return ApplyScalar(s, GSHT_OP_MUL);
  }
  auto& operator/=(Scalar s)
    requires Writeable::value
  {
    return ApplyScalar(s, GSHT_OP_DIV);
  }

  // Prints "colatitude longitude value" per point (reference :189-220).
  friend std::ostream& operator<<(std::ostream& os, const CanonicalComponentFieldBase& u) {
    const auto th = u.CoLatitudes();
    const auto ph = u.Longitudes();
    const Int nTheta = Int(u.NumberOfCoLatitudes()), nPhi = Int(u.NumberOfLongitudes());
    for (Int i = 0; i < nTheta; i++)
      for (Int j = 0; j < nPhi; j++) {
        os << std::format("{:+.8e} {:+.8e} ", th[i], ph[j]);
        if constexpr (std::same_as<Value, RealValued>) {
          os << std::format("{:+.8e}", u[i, j]);
        } else {
          const auto v = u[i, j];
          os << std::format("{:+.8e} {:+.8e}", v.real(), v.imag());
        }
        if (i != nTheta - 1 || j != nPhi - 1) os << '\n';
      }
    return os;
  }

 private:
  auto& Derived() const { return static_cast<const _Derived&>(*this); }
  auto& Derived() { return static_cast<_Derived&>(*this); }

  template <typename D>
  void Apply(const CanonicalComponentFieldBase<_N, D>& other, int op) {
    if (other.Size() != Size()) throw GSHTError(GSHT_ERR_BAD_ARG, "fields on different grids");
    Detail::FieldProgram p;
    if (op >= 0) Derived().Emit(p);
    other.Emit(p);
    if (op >= 0) p.Op(op);
    p.Evaluate(Derived().RawData(), std::same_as<Value, RealValued>, long(Size()));
  }
  auto& ApplyScalar(Scalar s, int op) {
    Detail::FieldProgram p;
    Derived().Emit(p);
    p.Constant(s);
    p.Op(op);
    p.Evaluate(Derived().RawData(), std::same_as<Value, RealValued>, long(Size()));
    return Derived();
  }
};

}  // namespace GSHTrans

#endif

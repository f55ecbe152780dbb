// Operators and functions that build field expressions (reference:
// CanonicalComponentFieldOverloads.h:22-262), with the reference's rules on
// upper indices: + and - need equal N, * adds them, / needs a divisor of
// N = 0; a scalar may be added to or subtracted from an N = 0 field only and
// may multiply or divide any field.
#ifndef GSHT_B200_CANONICAL_COMPONENT_FIELD_OVERLOADS_H
#define GSHT_B200_CANONICAL_COMPONENT_FIELD_OVERLOADS_H

#include "CanonicalComponentFieldBinary.h"
#include "CanonicalComponentFieldUnary.h"

namespace GSHTrans {

namespace Internal {
template <std::ptrdiff_t N, typename D>
const D& Cast(const CanonicalComponentFieldBase<N, D>& u) {
  return static_cast<const D&>(u);
}
}  // namespace Internal

// unary
template <std::ptrdiff_t N, typename D>
auto operator-(const CanonicalComponentFieldBase<N, D>& u) {
  return CanonicalComponentFieldUnary<GSHT_OP_NEG, N, D>(Internal::Cast(u));
}
template <std::ptrdiff_t N, typename D>
auto conj(const CanonicalComponentFieldBase<N, D>& u) {
  return CanonicalComponentFieldConj<N, D>(Internal::Cast(u));
}
template <std::ptrdiff_t N, typename D>
auto real(const CanonicalComponentFieldBase<N, D>& u) {
  return CanonicalComponentFieldReal<N, D>(Internal::Cast(u));
}
template <std::ptrdiff_t N, typename D>
auto imag(const CanonicalComponentFieldBase<N, D>& u) {
  return CanonicalComponentFieldImag<N, D>(Internal::Cast(u));
}

// with a scalar
template <std::ptrdiff_t N, typename D>
  requires(N == 0)
auto operator+(const CanonicalComponentFieldBase<N, D>& u, typename D::Scalar s) {
  return CanonicalComponentFieldUnaryWithScalar<GSHT_OP_ADD, N, D, false>(Internal::Cast(u), s);
}
template <std::ptrdiff_t N, typename D>
  requires(N == 0)
auto operator+(typename D::Scalar s, const CanonicalComponentFieldBase<N, D>& u) {
  return CanonicalComponentFieldUnaryWithScalar<GSHT_OP_ADD, N, D, true>(Internal::Cast(u), s);
}
template <std::ptrdiff_t N, typename D>
  requires(N == 0)
auto operator-(const CanonicalComponentFieldBase<N, D>& u, typename D::Scalar s) {
  return CanonicalComponentFieldUnaryWithScalar<GSHT_OP_SUB, N, D, false>(Internal::Cast(u), s);
}
template <std::ptrdiff_t N, typename D>
auto operator*(const CanonicalComponentFieldBase<N, D>& u, typename D::Scalar s) {
  return CanonicalComponentFieldUnaryWithScalar<GSHT_OP_MUL, N, D, false>(Internal::Cast(u), s);
}
template <std::ptrdiff_t N, typename D>
auto operator*(typename D::Scalar s, const CanonicalComponentFieldBase<N, D>& u) {
  return CanonicalComponentFieldUnaryWithScalar<GSHT_OP_MUL, N, D, true>(Internal::Cast(u), s);
}
template <std::ptrdiff_t N, typename D>
auto operator/(const CanonicalComponentFieldBase<N, D>& u, typename D::Scalar s) {
  return CanonicalComponentFieldUnaryWithScalar<GSHT_OP_DIV, N, D, false>(Internal::Cast(u), s);
}

// binary
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
  requires std::same_as<typename D0::Scalar, typename D1::Scalar> && (N0 == N1)
auto operator+(const CanonicalComponentFieldBase<N0, D0>& u0, const CanonicalComponentFieldBase<N1, D1>& u1) {
  return CanonicalComponentFieldAdd<N0, D0, N1, D1>(Internal::Cast(u0), Internal::Cast(u1));
}
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
  requires std::same_as<typename D0::Scalar, typename D1::Scalar> && (N0 == N1)
auto operator-(const CanonicalComponentFieldBase<N0, D0>& u0, const CanonicalComponentFieldBase<N1, D1>& u1) {
  return CanonicalComponentFieldSubtract<N0, D0, N1, D1>(Internal::Cast(u0), Internal::Cast(u1));
}
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
  requires std::same_as<typename D0::Scalar, typename D1::Scalar>
auto operator*(const CanonicalComponentFieldBase<N0, D0>& u0, const CanonicalComponentFieldBase<N1, D1>& u1) {
  return CanonicalComponentFieldMultiply<N0, D0, N1, D1>(Internal::Cast(u0), Internal::Cast(u1));
}
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
  requires std::same_as<typename D0::Scalar, typename D1::Scalar> && (N1 == 0)
auto operator/(const CanonicalComponentFieldBase<N0, D0>& u0, const CanonicalComponentFieldBase<N1, D1>& u1) {
  return CanonicalComponentFieldDivide<N0, D0, N1, D1>(Internal::Cast(u0), Internal::Cast(u1));
}

}  // namespace GSHTrans

#endif

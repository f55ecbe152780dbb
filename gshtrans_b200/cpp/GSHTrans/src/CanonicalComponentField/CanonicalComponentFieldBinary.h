// Lazy binary expressions of canonical-component fields (reference:
// CanonicalComponentFieldBinary.h:20-305): sums and differences of equal
// upper index, products (upper indices add) and quotients by an N = 0 field,
// plus the scalar forms (reference: CanonicalComponentFieldUnary.h:300-354).
#ifndef GSHT_B200_CANONICAL_COMPONENT_FIELD_BINARY_H
#define GSHT_B200_CANONICAL_COMPONENT_FIELD_BINARY_H

#include "CanonicalComponentFieldBase.h"

namespace GSHTrans {

template <int Op, std::ptrdiff_t N, typename D0, typename D1>
class CanonicalComponentFieldBinary;
template <int Op, std::ptrdiff_t N, typename D, bool ScalarLeft>
class CanonicalComponentFieldUnaryWithScalar;

namespace Internal {
template <int Op, std::ptrdiff_t N, typename D0, typename D1>
struct Traits<CanonicalComponentFieldBinary<Op, N, D0, D1>> {
  using Int = std::ptrdiff_t;
  using Value = typename Traits<D0>::Value;
  using Real = typename Traits<D0>::Real;
  using Complex = typename Traits<D0>::Complex;
  using Scalar = typename Traits<D0>::Scalar;
  using Writeable = std::false_type;
};
template <int Op, std::ptrdiff_t N, typename D, bool ScalarLeft>
struct Traits<CanonicalComponentFieldUnaryWithScalar<Op, N, D, ScalarLeft>> {
  using Int = std::ptrdiff_t;
  using Value = typename Traits<D>::Value;
  using Real = typename Traits<D>::Real;
  using Complex = typename Traits<D>::Complex;
  using Scalar = typename Traits<D>::Scalar;
  using Writeable = std::false_type;
};

template <int Op, typename S>
S Combine(S a, S b) {
  if constexpr (Op == GSHT_OP_ADD) return a + b;
  else if constexpr (Op == GSHT_OP_SUB) return a - b;
  else if constexpr (Op == GSHT_OP_MUL) return a * b;
  else return a / b;
}
}  // namespace Internal

template <int Op, std::ptrdiff_t N, typename D0, typename D1>
class CanonicalComponentFieldBinary
    : public CanonicalComponentFieldBase<N, CanonicalComponentFieldBinary<Op, N, D0, D1>> {
 public:
  using Int = std::ptrdiff_t;
  using Scalar = typename Internal::Traits<D0>::Scalar;

  CanonicalComponentFieldBinary(const D0& u0, const D1& u1) : _u0{u0}, _u1{u1} {}

  auto& Grid() const { return _u0.Grid(); }
  Scalar operator[](Int iTheta, Int iPhi) const {
    this->CheckPointIndices(iTheta, iPhi);
    return Internal::Combine<Op, Scalar>(_u0[iTheta, iPhi], _u1[iTheta, iPhi]);
  }
  void Emit(Detail::FieldProgram& p) const {
    _u0.Emit(p);
    _u1.Emit(p);
    p.Op(Op);
  }

 private:
  Internal::Hold<D0> _u0;
  Internal::Hold<D1> _u1;
};

template <int Op, std::ptrdiff_t N, typename D, bool ScalarLeft>
class CanonicalComponentFieldUnaryWithScalar
    : public CanonicalComponentFieldBase<N, CanonicalComponentFieldUnaryWithScalar<Op, N, D, ScalarLeft>> {
 public:
  using Int = std::ptrdiff_t;
  using Scalar = typename Internal::Traits<D>::Scalar;

  CanonicalComponentFieldUnaryWithScalar(const D& u, Scalar s) : _u{u}, _s{s} {}

  auto& Grid() const { return _u.Grid(); }
  Scalar operator[](Int iTheta, Int iPhi) const {
    this->CheckPointIndices(iTheta, iPhi);
    if constexpr (ScalarLeft) return Internal::Combine<Op, Scalar>(_s, _u[iTheta, iPhi]);
    else return Internal::Combine<Op, Scalar>(_u[iTheta, iPhi], _s);
  }
  void Emit(Detail::FieldProgram& p) const {
    if constexpr (ScalarLeft) {
      p.Constant(_s);
      _u.Emit(p);
    } else {
      _u.Emit(p);
      p.Constant(_s);
    }
    p.Op(Op);
  }

 private:
  Internal::Hold<D> _u;
  Scalar _s;
};

// The reference's class names for the four binary nodes.
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
using CanonicalComponentFieldAdd = CanonicalComponentFieldBinary<GSHT_OP_ADD, N0, D0, D1>;
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
using CanonicalComponentFieldSubtract = CanonicalComponentFieldBinary<GSHT_OP_SUB, N0, D0, D1>;
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
using CanonicalComponentFieldMultiply = CanonicalComponentFieldBinary<GSHT_OP_MUL, N0 + N1, D0, D1>;
template <std::ptrdiff_t N0, typename D0, std::ptrdiff_t N1, typename D1>
using CanonicalComponentFieldDivide = CanonicalComponentFieldBinary<GSHT_OP_DIV, N0, D0, D1>;

}  // namespace GSHTrans

#endif

// Lazy unary expressions of canonical-component fields (reference:
// CanonicalComponentFieldUnary.h:19-298): negation, complex conjugate, real
// and imaginary parts. Like the reference, conj keeps the upper index N
// (:104-107) and real/imag give real-valued fields of the same N.
#ifndef GSHT_B200_CANONICAL_COMPONENT_FIELD_UNARY_H
#define GSHT_B200_CANONICAL_COMPONENT_FIELD_UNARY_H

#include "CanonicalComponentFieldBase.h"

namespace GSHTrans {

template <int Op, std::ptrdiff_t N, typename D>
class CanonicalComponentFieldUnary;

namespace Internal {
template <int Op, std::ptrdiff_t N, typename D>
struct Traits<CanonicalComponentFieldUnary<Op, N, D>> {
  using Int = std::ptrdiff_t;
  static constexpr bool kToReal = Op == GSHT_OP_REAL || Op == GSHT_OP_IMAG;
  using Value = std::conditional_t<kToReal, RealValued, typename Traits<D>::Value>;
  using Real = typename Traits<D>::Real;
  using Complex = typename Traits<D>::Complex;
  using Scalar = std::conditional_t<kToReal, Real, typename Traits<D>::Scalar>;
  using Writeable = std::false_type;
};
}  // namespace Internal

template <int Op, std::ptrdiff_t N, typename D>
class CanonicalComponentFieldUnary
    : public CanonicalComponentFieldBase<N, CanonicalComponentFieldUnary<Op, N, D>> {
 public:
  using Int = std::ptrdiff_t;
  using Scalar = typename Internal::Traits<CanonicalComponentFieldUnary>::Scalar;

  explicit CanonicalComponentFieldUnary(const D& u) : _u{u} {}

  auto& Grid() const { return _u.Grid(); }
  Scalar operator[](Int iTheta, Int iPhi) const {
    this->CheckPointIndices(iTheta, iPhi);
    const auto v = _u[iTheta, iPhi];
    constexpr bool kIn = ComplexFloatingPoint<decltype(v)>;
    if constexpr (Op == GSHT_OP_NEG) {
      return -v;
    } else if constexpr (Op == GSHT_OP_CONJ) {
      if constexpr (kIn) return std::conj(v);
      else return v;
    } else if constexpr (Op == GSHT_OP_REAL) {
      if constexpr (kIn) return v.real();
      else return v;
    } else {
      if constexpr (kIn) return v.imag();
      else return Scalar{0};
    }
  }
  void Emit(Detail::FieldProgram& p) const {
    _u.Emit(p);
    p.Op(Op);
  }

 private:
  Internal::Hold<D> _u;
};

template <std::ptrdiff_t N, typename D>
using CanonicalComponentFieldConj = CanonicalComponentFieldUnary<GSHT_OP_CONJ, N, D>;
template <std::ptrdiff_t N, typename D>
using CanonicalComponentFieldReal = CanonicalComponentFieldUnary<GSHT_OP_REAL, N, D>;
template <std::ptrdiff_t N, typename D>
using CanonicalComponentFieldImag = CanonicalComponentFieldUnary<GSHT_OP_IMAG, N, D>;

}  // namespace GSHTrans

#endif

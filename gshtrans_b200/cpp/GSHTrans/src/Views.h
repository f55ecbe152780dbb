// Non-owning views of one (n, theta) block of Wigner values or of a
// coefficient vector, indexed by degree and order (reference: Views.h:11-88).
#ifndef GSHT_B200_VIEWS_H
#define GSHT_B200_VIEWS_H

#include <iterator>

#include "Indexing.h"

namespace GSHTrans {

template <RealOrComplexFloatingPoint Scalar, OrderIndexRange MRange>
class GSHSubView : public GSHSubIndices<MRange> {
 public:
  using Int = std::ptrdiff_t;
  constexpr GSHSubView(Int l, Int mMax, Scalar* start) : GSHSubIndices<MRange>(l, mMax), _p{start} {}
  constexpr Scalar* begin() { return _p; }
  constexpr Scalar* end() { return _p + this->Size(); }
  constexpr Scalar& operator[](Int m) { return _p[this->Index(m)]; }

 private:
  Scalar* _p;
};

template <RealOrComplexFloatingPoint Scalar, OrderIndexRange MRange>
class ConstGSHSubView : public GSHSubIndices<MRange> {
 public:
  using Int = std::ptrdiff_t;
  constexpr ConstGSHSubView(Int l, Int mMax, const Scalar* start)
      : GSHSubIndices<MRange>(l, mMax), _p{start} {}
  constexpr const Scalar* begin() const { return _p; }
  constexpr const Scalar* end() const { return _p + this->Size(); }
  constexpr Scalar operator[](Int m) const { return _p[this->Index(m)]; }

 private:
  const Scalar* _p;
};

template <RealOrComplexFloatingPoint Scalar, OrderIndexRange MRange>
class GSHView : public GSHIndices<MRange> {
 public:
  using Int = std::ptrdiff_t;
  constexpr GSHView(Int lMax, Int mMax, Int n, Scalar* start)
      : GSHIndices<MRange>(lMax, mMax, n), _p{start} {}
  constexpr Scalar* begin() { return _p; }
  constexpr Scalar* end() { return _p + this->Size(); }
  constexpr auto operator[](Int l) {
    return GSHSubView<Scalar, MRange>(l, this->MaxOrder(), _p + this->OffsetForDegree(l));
  }
  constexpr Scalar& operator[](Int l, Int m) { return _p[this->Index(l, m)]; }

 private:
  Scalar* _p;
};

template <RealOrComplexFloatingPoint Scalar, OrderIndexRange MRange>
class ConstGSHView : public GSHIndices<MRange> {
 public:
  using Int = std::ptrdiff_t;
  constexpr ConstGSHView(Int lMax, Int mMax, Int n, const Scalar* start)
      : GSHIndices<MRange>(lMax, mMax, n), _p{start} {}
  constexpr const Scalar* begin() const { return _p; }
  constexpr const Scalar* end() const { return _p + this->Size(); }
  constexpr auto operator[](Int l) const {
    return ConstGSHSubView<Scalar, MRange>(l, this->MaxOrder(), _p + this->OffsetForDegree(l));
  }
  constexpr Scalar operator[](Int l, Int m) const { return _p[this->Index(l, m)]; }

 private:
  const Scalar* _p;
};

}  // namespace GSHTrans

#endif

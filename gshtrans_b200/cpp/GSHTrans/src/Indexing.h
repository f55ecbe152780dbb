// Spectral index bookkeeping (reference: Indexing.h:21-156). A block for upper
// index n holds degrees l = |n|..lMax, each with orders -min(l, mMax)..
// min(l, mMax) (All) or 0..min(l, mMax) (NonNegative), degree after degree.
#ifndef GSHT_B200_INDEXING_H
#define GSHT_B200_INDEXING_H

#include <algorithm>
#include <cassert>
#include <cstddef>
#include <ranges>
#include <utility>

#include "Concepts.h"

namespace GSHTrans {

template <OrderIndexRange MRange>
class GSHSubIndices {
  using Int = std::ptrdiff_t;

 public:
  constexpr GSHSubIndices(Int l, Int mMax) : _l{l}, _top{std::min(l, mMax)} {
    assert(l >= 0 && mMax >= 0);
  }
  constexpr Int Degree() const { return _l; }
  constexpr Int MinOrder() const {
    if constexpr (std::same_as<MRange, All>) return -_top;
    return 0;
  }
  constexpr Int MaxOrder() const { return _top; }
  constexpr auto Orders() const { return std::views::iota(MinOrder(), _top + 1); }
  constexpr auto NegativeOrders() const { return std::views::iota(MinOrder(), Int{0}); }
  constexpr auto NonNegativeOrders() const { return std::views::iota(Int{0}, _top + 1); }
  constexpr Int Size() const { return _top - MinOrder() + 1; }
  constexpr Int Index(Int m) const {
    assert(m >= MinOrder() && m <= _top);
    return m - MinOrder();
  }

 private:
  Int _l, _top;
};

template <OrderIndexRange MRange>
class GSHIndices {
  using Int = std::ptrdiff_t;
  static constexpr Int Width(Int top) {
    if constexpr (std::same_as<MRange, All>) return 2 * top + 1;
    return top + 1;
  }
  // Number of entries of degrees 0..l-1 when every degree is complete up to
  // mMax (closed form of the sum of Width(min(k, mMax)), k < l).
  constexpr Int Before(Int l) const {
    const Int full = std::min(l, _mMax + 1);  // degrees with min(k, mMax) = k
    Int s;
    if constexpr (std::same_as<MRange, All>) {
      s = full * full;
    } else {
      s = full * (full + 1) / 2;
    }
    if (l > _mMax + 1) s += (l - _mMax - 1) * Width(_mMax);
    return s;
  }

 public:
  GSHIndices() = default;
  constexpr GSHIndices(Int lMax, Int mMax, Int n) : _lMax{lMax}, _mMax{std::min(lMax, mMax)}, _n{n} {
    assert(lMax >= 0 && mMax >= 0 && (n < 0 ? -n : n) <= lMax);
  }
  constexpr Int UpperIndex() const { return _n; }
  constexpr Int MaxOrder() const { return _mMax; }
  constexpr Int MinDegree() const { return _n < 0 ? -_n : _n; }
  constexpr Int MaxDegree() const { return _lMax; }
  constexpr auto Degrees() const { return std::views::iota(MinDegree(), _lMax + 1); }
  constexpr auto Indices() const {
    return Degrees() | std::views::transform([mm = _mMax](Int l) {
             return std::views::cartesian_product(std::views::single(l),
                                                  GSHSubIndices<MRange>(l, mm).Orders());
           }) |
           std::views::join;
  }
  constexpr Int OffsetForDegree(Int l) const {
    assert(l >= MinDegree() && l <= _lMax);
    return Before(l) - Before(MinDegree());
  }
  constexpr Int SizeForDegree(Int l) const { return GSHSubIndices<MRange>(l, _mMax).Size(); }
  constexpr auto Index(Int l) const {
    return std::pair(OffsetForDegree(l), GSHSubIndices<MRange>(l, _mMax));
  }
  constexpr Int Index(Int l, Int m) const {
    return OffsetForDegree(l) + GSHSubIndices<MRange>(l, _mMax).Index(m);
  }
  constexpr Int Size() const { return Before(_lMax + 1) - Before(MinDegree()); }

 private:
  Int _lMax = 0, _mMax = 0, _n = 0;
};

}  // namespace GSHTrans

#endif

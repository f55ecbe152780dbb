// Tag types and concepts of the GSHTrans interface (reference: Concepts.h:15-126).
// The names and meanings are the reference's so that code written against it
// compiles unchanged against this GPU-backed drop-in.
#ifndef GSHT_B200_CONCEPTS_H
#define GSHT_B200_CONCEPTS_H

#include <complex>
#include <concepts>
#include <iterator>
#include <ranges>
#include <type_traits>

namespace GSHTrans {

// Storage order of Wigner tables: upper index outer or angle outer.
struct ColumnMajor {};
struct RowMajor {};
template <typename T>
concept WignerStorage = std::same_as<T, ColumnMajor> || std::same_as<T, RowMajor>;

// Index ranges for orders / upper indices, and single vs many angles.
struct All {};
struct NonNegative {};
struct Single {};
struct Multiple {};
struct UpperIndexFirst {};
struct AngleFirst {};

template <typename T>
concept IndexRange = std::same_as<T, All> || std::same_as<T, NonNegative> || std::same_as<T, Single>;
template <typename T>
concept OrderIndexRange = std::same_as<T, All> || std::same_as<T, NonNegative>;
template <typename T>
concept AngleIndexRange = std::same_as<T, Multiple> || std::same_as<T, Single>;

// Normalisation of the Wigner functions.
struct Ortho {};
struct FourPi {};
template <typename T>
concept Normalisation = std::same_as<T, Ortho> || std::same_as<T, FourPi>;

// Value kind of a field.
struct RealValued {};
struct ComplexValued {};
template <typename T>
concept RealOrComplexValued = std::same_as<T, RealValued> || std::same_as<T, ComplexValued>;

namespace Detail {
template <typename T>
inline constexpr bool kIsComplexFloat = false;
template <typename T>
inline constexpr bool kIsComplexFloat<std::complex<T>> = std::is_floating_point_v<T>;
template <typename T>
struct StripComplex {
  using type = T;
};
template <typename T>
struct StripComplex<std::complex<T>> {
  using type = T;
};
}  // namespace Detail

template <typename T>
concept RealFloatingPoint = std::floating_point<T>;
template <typename T>
concept ComplexFloatingPoint = Detail::kIsComplexFloat<std::remove_const_t<T>>;
template <typename T>
concept RealOrComplexFloatingPoint = RealFloatingPoint<T> || ComplexFloatingPoint<T>;
template <typename T>
using RemoveComplex = typename Detail::StripComplex<T>::type;

template <typename T>
concept RealFloatingPointRange =
    std::ranges::common_range<T> && RealFloatingPoint<std::ranges::range_value_t<T>>;
template <typename T>
concept ComplexFloatingPointRange =
    std::ranges::common_range<T> && ComplexFloatingPoint<std::ranges::range_value_t<T>>;
template <typename T>
concept RealOrComplexFloatingPointRange =
    std::ranges::common_range<T> && RealOrComplexFloatingPoint<std::ranges::range_value_t<T>>;

template <typename Function, typename Real, typename Scalar>
concept ScalarFunctionS2 = RealFloatingPoint<Real> && RealOrComplexFloatingPoint<Scalar> &&
                           requires(Function f, Real theta, Real phi) {
                             { f(theta, phi) } -> std::convertible_to<Scalar>;
                           };
template <typename Function, typename Int, typename Scalar>
concept ScalarFunctionS2Expansion = std::integral<Int> && RealOrComplexFloatingPoint<Scalar> &&
                                    requires(Function f, Int l, Int m) {
                                      { f(l, m) } -> std::convertible_to<Scalar>;
                                    };

namespace Internal {
template <typename Derived>
struct Traits {};
}  // namespace Internal

// (-1)^m for integer m (reference: Utility.h:7-10).
template <typename Scalar = std::ptrdiff_t>
constexpr Scalar MinusOneToPower(std::ptrdiff_t m) {
  return (m & 1) ? Scalar(-1) : Scalar(1);
}

}  // namespace GSHTrans

#endif

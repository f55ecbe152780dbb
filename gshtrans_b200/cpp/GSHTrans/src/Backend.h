// Thin C++ layer over the C ABI of libgsht_cuda.so (gsht.h): status codes
// become exceptions, index-range tags become ABI constants.
#ifndef GSHT_B200_BACKEND_H
#define GSHT_B200_BACKEND_H

#include <gsht.h>

#include <memory>
#include <stdexcept>
#include <string>

#include "Concepts.h"

namespace GSHTrans {

// Raised for every non-OK status; the reference asserts where the status is
// GSHT_ERR_BAD_ARG.
class GSHTError : public std::runtime_error {
 public:
  GSHTError(gsht_status s, const std::string& what) : std::runtime_error(what), status{s} {}
  gsht_status status;
};

namespace Backend {

inline void Check(gsht_status s) {
  if (s != GSHT_OK) throw GSHTError(s, std::string("libgsht_cuda: ") + gsht_last_error());
}

template <typename R>
constexpr int RangeCode() {
  if constexpr (std::same_as<R, All>) return GSHT_RANGE_ALL;
  if constexpr (std::same_as<R, NonNegative>) return GSHT_RANGE_NONNEGATIVE;
  return GSHT_RANGE_SINGLE;
}

struct GridDeleter {
  void operator()(gsht_grid* g) const { gsht_grid_destroy(g); }
};
using GridHandle = std::shared_ptr<gsht_grid>;

}  // namespace Backend
}  // namespace GSHTrans

#endif

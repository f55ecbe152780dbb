// Grid-geometry queries shared by all fields (reference: FieldBase.h:11-42).
#ifndef GSHT_B200_FIELD_BASE_H
#define GSHT_B200_FIELD_BASE_H

#include <cassert>
#include <complex>
#include <ranges>
#include <vector>

#include "Backend.h"

namespace GSHTrans {

template <typename _Derived>
class FieldBase {
 public:
  using Int = std::ptrdiff_t;

  auto& Grid() const { return Derived().Grid(); }

  auto NumberOfCoLatitudes() const { return Grid().NumberOfCoLatitudes(); }
  auto CoLatitudes() const { return Grid().CoLatitudes(); }
  auto CoLatitudeIndices() const { return Grid().CoLatitudeIndices(); }
  auto NumberOfLongitudes() const { return Grid().NumberOfLongitudes(); }
  auto Longitudes() const { return Grid().Longitudes(); }
  auto LongitudeIndices() const { return Grid().LongitudeIndices(); }

  constexpr void CheckPointIndices([[maybe_unused]] Int iTheta, [[maybe_unused]] Int iPhi) const {
    assert(iTheta >= 0 && iTheta < Int(NumberOfCoLatitudes()));
    assert(iPhi >= 0 && iPhi < Int(NumberOfLongitudes()));
  }

  auto Points() const { return Grid().Points(); }
  auto PointIndices() const { return Grid().PointIndices(); }
  auto EnumeratePointIndices() const { return std::views::enumerate(PointIndices()); }
  auto Weights() const { return Grid().Weights(); }

 private:
  auto& Derived() const { return static_cast<const _Derived&>(*this); }
};

namespace Detail {

// A field expression flattened into the postfix program that
// gsht_field_eval runs once per grid point on the GPU. Leaves are the
// fields' value buffers (host or device); each distinct buffer is one input.
struct FieldProgram {
  std::vector<gsht_expr_op> ops;
  std::vector<const void*> inputs;
  std::vector<int> kinds;

  void Load(const void* data, bool isReal) {
    int idx = -1;
    for (int i = 0; i < int(inputs.size()); i++)
      if (inputs[i] == data) idx = i;
    if (idx < 0) {
      idx = int(inputs.size());
      inputs.push_back(data);
      kinds.push_back(isReal ? 1 : 0);
    }
    ops.push_back(gsht_expr_op{GSHT_OP_LOAD, idx, 0.0, 0.0});
  }
  template <typename S>
  void Constant(S s) {
    const std::complex<double> c(s);
    ops.push_back(gsht_expr_op{GSHT_OP_CONST, 0, c.real(), c.imag()});
  }
  void Op(int code) { ops.push_back(gsht_expr_op{code, 0, 0.0, 0.0}); }

  // Runs the program over npoints values into out (a host or device buffer
  // of npoints reals or complexes). Host buffers are staged through the
  // library; the call returns when out holds the result.
  void Evaluate(void* out, bool outReal, long npoints) const {
    Backend::Check(gsht_field_eval(ops.data(), int(ops.size()), inputs.data(), kinds.data(),
                                   int(inputs.size()), out, outReal ? 1 : 0, npoints, 1, npoints,
                                   nullptr));
  }
};

}  // namespace Detail
}  // namespace GSHTrans

#endif

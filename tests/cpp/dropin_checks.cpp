// Checks of the C++ drop-in headers (gshtrans_b200/cpp/GSHTrans), written the
// way the reference's own tests exercise its interface:
//   coefficient round trips through a grid (tests/CheckCoeff2Coeff.h),
//   n = 0 Wigner values against std::sph_legendre (tests/CheckLegendre.h),
//   the addition theorem sum_m d^l_{mn} d^l_{mn'} = delta_{nn'} for FourPi
//   tables (tests/CheckAdditionTheorem.h),
// plus field expressions evaluated on the GPU against the same expressions
// evaluated point by point on the host. Prints one line per check and exits
// with the number of failed checks.
#include <GSHTrans/All>
#include <cmath>
#include <complex>
#include <cstdio>
#include <limits>
#include <numbers>
#include <numeric>
#include <random>
#include <string>
#include <vector>

using namespace GSHTrans;
using Int = std::ptrdiff_t;

static int g_failures = 0;
static void Report(const std::string& name, bool ok, double value) {
  std::printf("%-44s %s  %.3e\n", name.c_str(), ok ? "ok  " : "FAIL", value);
  if (!ok) g_failures++;
}

static std::mt19937_64 g_gen{20241203};
static Int Uniform(Int a, Int b) { return std::uniform_int_distribution<Int>(a, b)(g_gen); }

template <typename Scalar, typename MRange, typename NRange>
double Coeff2Coeff(Int lMaxGrid, Int lMax, Precision prec = Precision::FP64) {
  using Complex = std::complex<double>;
  using Grid = GaussLegendreGrid<double, MRange, NRange>;
  const Int nMax = std::min<Int>(lMax, 4);
  Grid grid{int(lMaxGrid), int(nMax), prec};
  const Int n = std::same_as<NRange, All> ? Uniform(-nMax, nMax) : Uniform(0, nMax);
  const Int size = RealFloatingPoint<Scalar> ? grid.RealCoefficientSize(lMax, n) : grid.ComplexCoefficientSize(lMax, n);
  std::vector<Complex> flm(size), glm(size);
  if constexpr (ComplexFloatingPoint<Scalar>) grid.RandomComplexCoefficient(lMax, n, flm);
  else grid.RandomRealCoefficient(lMax, n, flm);
  std::vector<Scalar> f(grid.FieldSize());
  grid.InverseTransformation(lMax, n, flm, f);
  grid.ForwardTransformation(lMax, n, f, glm);
  double err = 0, ref = 0;
  for (Int i = 0; i < size; i++) {
    err = std::max(err, std::abs(flm[i] - glm[i]));
    ref = std::max(ref, std::abs(flm[i]));
  }
  return err / ref;
}

static double Legendre(double theta) {
  const int lMax = 300;
  auto d = Wigner(lMax, lMax, 0, theta);
  constexpr double eps = 100000 * std::numeric_limits<double>::epsilon();
  constexpr double tiny = 1000 * std::numeric_limits<double>::min();
  double worst = 0;
  for (auto l : d.Degrees(0))
    for (auto m : d[l].Orders()) {
      const double plm = d[l][m];
      // std::sph_legendre is defined for m >= 0; d^l_{-m,0} = (-1)^m d^l_{m0}.
      const double ref = MinusOneToPower<double>(m < 0 ? m : 0) * std::sph_legendre(l, std::abs(m), theta);
      // The reference divides by `norm = std::abs(ref) > tiny`, a bool, so its
      // bound is absolute; the same bound is kept here.
      if (std::abs(ref) > tiny) worst = std::max(worst, std::abs(plm - ref));
    }
  return worst / eps;  // <= 1 passes
}

static double AdditionTheorem(double theta) {
  const int lMax = 40;
  auto d = Wigner<double, FourPi, All, All>(lMax, lMax, lMax, theta);
  double worst = 0;
  for (auto n : d.UpperIndices()) {
    auto d1 = d[n];
    for (auto np : d.UpperIndices()) {
      auto d2 = d[np];
      for (Int l = std::max(std::abs(n), std::abs(np)); l <= lMax; l++) {
        double sum = std::inner_product(d1[l].begin(), d1[l].end(), d2[l].begin(), 0.0);
        if (n == np) sum -= 1;
        worst = std::max(worst, std::abs(sum));
      }
    }
  }
  return worst;
}

template <typename Field, typename Expr>
double CompareWithHost(const Field& w, const Expr& e) {
  double err = 0, ref = 0;
  for (auto [i, j] : w.PointIndices()) {
    const auto h = e[i, j];
    err = std::max(err, double(std::abs(w[i, j] - h)));
    ref = std::max(ref, double(std::abs(h)));
  }
  return err / ref;
}

static void Fields() {
  using Grid = GaussLegendreGrid<double, All, All>;
  Grid grid(48, 2);
  auto f1 = [](double th, double ph) { return std::complex<double>(std::cos(th) * std::sin(ph), std::sin(2 * th)); };
  auto f2 = [](double th, double ph) { return std::complex<double>(1.5 + std::sin(th), std::cos(3 * ph)); };
  ComplexCanonicalComponentField<1, Grid> u(grid, f1);
  ComplexCanonicalComponentField<-1, Grid> v(grid, f2);
  ComplexScalarField<Grid> s(grid, f2);
  const double tol = 8 * std::numeric_limits<double>::epsilon();

  ComplexScalarField<Grid> w = u * v + conj(u) * v;  // constructed from an expression
  Report("field u*v + conj(u)*v", CompareWithHost(w, u * v + conj(u) * v) < tol, CompareWithHost(w, u * v + conj(u) * v));

  ComplexCanonicalComponentField<1, Grid> q(grid);
  q = (u * s - u / s) * std::complex<double>(0.5, -2.0);
  const double e2 = CompareWithHost(q, (u * s - u / s) * std::complex<double>(0.5, -2.0));
  Report("field (u*s - u/s)*c", e2 < tol, e2);

  RealScalarField<Grid> r(grid);
  r = real(w) + imag(s) * 3.0;
  const double e3 = CompareWithHost(r, real(w) + imag(s) * 3.0);
  Report("field real(w) + 3 imag(s)", e3 < tol, e3);

  ComplexScalarField<Grid> a(grid, f2);
  const ComplexScalarField<Grid> a0 = a;
  a += s * s;
  a *= std::complex<double>(2.0, 1.0);
  const double e4 = CompareWithHost(a, (a0 + s * s) * std::complex<double>(2.0, 1.0));
  Report("field compound += *=", e4 < tol, e4);

  // A field's values feed the transforms directly.
  RealScalarField<Grid> g(grid, [](double th, double ph) { return std::cos(th) + std::sin(th) * std::cos(ph); });
  std::vector<std::complex<double>> glm(grid.RealCoefficientSize(0));
  grid.ForwardTransformation(grid.MaxDegree(), 0, g.Data(), glm);
  RealScalarField<Grid> h(grid);
  auto hv = h.Data();
  grid.InverseTransformation(grid.MaxDegree(), 0, glm, hv);
  double e5 = 0;
  for (auto [i, j] : g.PointIndices()) e5 = std::max(e5, std::abs(g[i, j] - h[i, j]));
  Report("field -> forward -> inverse", e5 < 1e-13, e5);
}

// Expansions (the reference's CanonicalComponentExpansion container, here
// wired to the transforms): coefficients -> field -> coefficients.
template <typename Value>
static double ExpansionRoundTrip(Int L) {
  using Grid = GaussLegendreGrid<double, All, All>;
  Grid grid(int(L), 2);
  CanonicalComponentExpansion<1, Grid, Value> e(grid);
  std::normal_distribution<double> nd;
  for (auto [l, m] : e.Indices()) {
    e[l, m] = {nd(g_gen), std::same_as<Value, RealValued> && m == 0 ? 0.0 : nd(g_gen)};
  }
  if constexpr (std::same_as<Value, ComplexValued>) e[L, L] = 0;  // alias of (L, -L)
  else e[L, L] = e[L, L].real();
  auto f = e.ToField();
  CanonicalComponentExpansion<1, Grid, Value> back(f);
  back -= e;
  double err = 0, ref = 0;
  for (auto [l, m] : e.Indices()) {
    err = std::max(err, std::abs(back[l, m]));
    ref = std::max(ref, std::abs(e[l, m]));
  }
  return err / ref;
}

// Vector fields (GSHTrans/Vector): the pointwise products and compound
// operators against the same formulas on the host, and the three-component
// expansion -> field -> expansion round trip.
static void Vectors() {
  using Grid = GaussLegendreGrid<double, All, All>;
  using Complex = std::complex<double>;
  Grid grid(40, 1);
  ComplexVectorField<Grid> u(grid), v(grid);
  std::normal_distribution<double> nd;
  for (auto alpha : u.CanonicalIndices())
    for (auto [i, j] : u.Component<0>().PointIndices()) {
      u[alpha, i, j] = {nd(g_gen), nd(g_gen)};
      v[alpha, i, j] = {nd(g_gen), nd(g_gen)};
    }
  const auto ip = InnerProduct(u, v);
  const auto dp = DualityProduct(u, v);
  double eip = 0, edp = 0, ref = 0;
  for (auto [i, j] : ip.PointIndices()) {
    Complex h = 0;
    for (auto a : u.CanonicalIndices()) h += std::conj(u[a, i, j]) * v[a, i, j];
    const Complex d = -u[-1, i, j] * v[1, i, j] + u[0, i, j] * v[0, i, j] - u[1, i, j] * v[-1, i, j];
    eip = std::max(eip, std::abs(ip[i, j] - h));
    edp = std::max(edp, std::abs(dp[i, j] - d));
    ref = std::max(ref, std::max(std::abs(h), std::abs(d)));
  }
  const double tol = 16 * std::numeric_limits<double>::epsilon();
  Report("vector InnerProduct", eip / ref < tol, eip / ref);
  Report("vector DualityProduct", edp / ref < tol, edp / ref);

  ComplexScalarField<Grid> s(grid, [](double th, double ph) { return Complex(1.5 + std::sin(th), std::cos(ph)); });
  ComplexVectorField<Grid> w = u;
  w += v;
  w *= s;
  w *= Complex(0.5, -1.0);
  double ew = 0, rw = 0;
  for (auto a : u.CanonicalIndices())
    for (auto [i, j] : s.PointIndices()) {
      const Complex h = (u[a, i, j] + v[a, i, j]) * s[i, j] * Complex(0.5, -1.0);
      ew = std::max(ew, std::abs(w[a, i, j] - h));
      rw = std::max(rw, std::abs(h));
    }
  Report("vector compound += *= (field, scalar)", ew / rw < tol, ew / rw);

  ComplexVectorExpansion<Grid> e(grid);
  const Int L = grid.MaxDegree();
  auto fill = [&](auto& c) {
    for (auto [l, m] : c.Indices()) c[l, m] = {nd(g_gen), nd(g_gen)};
    c[L, L] = 0;  // alias of (L, -L)
  };
  fill(e.Component<-1>());
  fill(e.Component<0>());
  fill(e.Component<1>());
  const auto f = e.ToField();
  ComplexVectorExpansion<Grid> back(f);
  double err = 0, rc = 0;
  auto diff = [&](const auto& a, const auto& b) {
    for (auto [l, m] : a.Indices()) {
      err = std::max(err, std::abs(a[l, m] - b[l, m]));
      rc = std::max(rc, std::abs(a[l, m]));
    }
  };
  diff(e.Component<-1>(), back.Component<-1>());
  diff(e.Component<0>(), back.Component<0>());
  diff(e.Component<1>(), back.Component<1>());
  Report("vector expansion -> field -> expansion", err / rc < 1e-12, err / rc);
}

int main() {
  for (int trial = 0; trial < 3; trial++) {
    const Int lg = Uniform(4, 256), l = Uniform(4, lg);
    const std::string tag = " L=" + std::to_string(lg) + " l=" + std::to_string(l);
    double e;
    e = Coeff2Coeff<double, All, All>(lg, l);
    Report("Coeff2Coeff R2C <All,All>" + tag, e < 1e-12, e);
    e = Coeff2Coeff<std::complex<double>, All, All>(lg, l);
    Report("Coeff2Coeff C2C <All,All>" + tag, e < 1e-12, e);
    e = Coeff2Coeff<double, NonNegative, NonNegative>(lg, l);
    Report("Coeff2Coeff R2C <NonNeg,NonNeg>" + tag, e < 1e-12, e);
    e = Coeff2Coeff<std::complex<double>, All, NonNegative>(lg, l);
    Report("Coeff2Coeff C2C <All,NonNeg>" + tag, e < 1e-12, e);
    // Extension: a grid without a stored table (l-recurrence in the kernels).
    e = Coeff2Coeff<std::complex<double>, All, All>(lg, l, Precision::Recurrence);
    Report("Coeff2Coeff C2C <All,All> recurrence" + tag, e < 1e-12, e);
    e = Coeff2Coeff<double, All, All>(lg, l, Precision::Recurrence);
    Report("Coeff2Coeff R2C <All,All> recurrence" + tag, e < 1e-12, e);
    // Extension: the tensor-core forms selected through the C++ grid
    // (max-abs error relative to the largest coefficient).
    e = Coeff2Coeff<std::complex<double>, All, All>(lg, l, Precision::Ozaki);
    Report("Coeff2Coeff C2C <All,All> Ozaki" + tag, e < 1e-12, e);
    e = Coeff2Coeff<std::complex<double>, All, All>(lg, l, Precision::Ozaki4);
    Report("Coeff2Coeff C2C <All,All> Ozaki4" + tag, e < 1e-5, e);
  }
  std::uniform_real_distribution<double> angle(0.0, std::numbers::pi);
  for (int trial = 0; trial < 3; trial++) {
    const double th = angle(g_gen);
    const double e1 = Legendre(th);
    Report("Legendre vs std::sph_legendre", e1 <= 1.0, e1);
    const double e2 = AdditionTheorem(th);
    Report("addition theorem (FourPi, All, All)", e2 <= 1000 * std::numeric_limits<double>::epsilon(), e2);
  }
  Fields();
  Vectors();
  for (Int L : {31, 96}) {
    const double ec = ExpansionRoundTrip<ComplexValued>(L);
    Report("expansion -> field -> expansion (complex) L=" + std::to_string(L), ec < 1e-12, ec);
    const double er = ExpansionRoundTrip<RealValued>(L);
    Report("expansion -> field -> expansion (real) L=" + std::to_string(L), er < 1e-12, er);
  }
  std::printf("%d failed\n", g_failures);
  return g_failures;
}

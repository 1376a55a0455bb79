// The least-squares proxy of the adaptive nest (HermiteProxy, src/nested/adaptive_nested.cpp:145-277), host side.
//
// Basis: probabilists' Hermite polynomials He_k of each standardised feature (He_{k+1} = z He_k - k He_{k-1}),
// and every product of them up to a total degree, in graded order (degree 0, then 1, ...; lexicographic within a
// degree, the first feature's exponent ascending slowest; adaptive_nested.cpp:57-75).  Fit: ridge-stabilised
// normal equations (the ridge relative to the mean diagonal, raised 1000-fold until the Cholesky factor exists)
// and the HC0 sandwich covariance of the coefficients, G^-1 (sum_i e_i^2 phi_i phi_i^T) G^-1.  Prediction: the
// value phi . beta and its estimation variance phi^T Cov phi.
//
// The layout is this file's own: the basis of all training rows is built once as a design matrix, the Gram and
// sandwich matrices are accumulated by row blocks of the triangle on several host threads, the inverse column by
// column in parallel, and predictions row-parallel.  Each entry is still summed over the same operands in the
// same order as the reference's loops (training rows in order, then k ascending, zero multipliers skipped), so
// the coefficients, values and variances keep the reference's bits whatever the thread count.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <thread>
#include <vector>

#include "zlatko_b200.h"

namespace {

// fn(begin, end) over [0, n) on up to 16 threads, at least `grain` items per thread.
template <class F>
void parallelFor(std::size_t n, std::size_t grain, F&& fn) {
  const std::size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const std::size_t workers = std::min({hw, std::size_t{16}, std::max<std::size_t>(1, n / std::max<std::size_t>(grain, 1))});
  if (workers <= 1) {
    fn(std::size_t{0}, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(workers);
  for (std::size_t w = 0; w < workers; ++w) pool.emplace_back([&, w] { fn(n * w / workers, n * (w + 1) / workers); });
  for (auto& t : pool) t.join();
}

// Row ranges [cut[w], cut[w + 1]) of a p x p lower triangle holding about the same number of entries.
std::vector<std::size_t> triangleCuts(std::size_t p, std::size_t parts) {
  std::vector<std::size_t> cut(parts + 1, p);
  cut[0] = 0;
  for (std::size_t w = 1; w < parts; ++w)
    cut[w] = std::min(p, static_cast<std::size_t>(std::ceil(static_cast<double>(p) * std::sqrt(static_cast<double>(w) / parts))));
  return cut;
}

// Exponent vectors over m features with total degree <= d, graded then lexicographic.
void gradedExponents(std::size_t m, std::size_t d, std::vector<std::vector<unsigned>>& out) {
  out.clear();
  std::vector<unsigned> e(m, 0);
  for (std::size_t g = 0; g <= d; ++g) {
    if (m == 0) {
      if (g == 0) out.push_back(e);
      continue;
    }
    // Compositions of g into m parts in lexicographic order, from (0, ..., 0, g) to (g, 0, ..., 0).  The next
    // one raises the rightmost position j < m - 1 with mass after it and puts the rest of that mass, less one,
    // in the last position.
    std::fill(e.begin(), e.end(), 0u);
    e[m - 1] = static_cast<unsigned>(g);
    for (;;) {
      out.push_back(e);
      std::size_t j = m - 1;
      unsigned rest = 0;
      while (j > 0 && rest == 0) rest += e[j--];
      if (rest == 0) break;
      ++e[j];
      std::fill(e.begin() + static_cast<std::ptrdiff_t>(j) + 1, e.end(), 0u);
      e[m - 1] = rest - 1;
    }
  }
}

// In-place lower Cholesky factor of the p x p matrix a (row-major, lower triangle read); false if a pivot is
// not positive.  Entry (i, j) is a_ij - sum_{k<j} L_ik L_jk, subtracted k ascending (src/core/matrix.cpp:49-68).
bool factor(std::vector<double>& a, std::size_t p) {
  for (std::size_t i = 0; i < p; ++i) {
    double* li = &a[i * p];
    for (std::size_t j = 0; j <= i; ++j) {
      const double* lj = &a[j * p];
      double s = li[j];
      for (std::size_t k = 0; k < j; ++k) s -= li[k] * lj[k];
      if (j < i) {
        li[j] = s / lj[j];
      } else {
        if (s <= 0.0) return false;
        li[i] = std::sqrt(s);
      }
    }
    std::fill(li + i + 1, li + p, 0.0);
  }
  return true;
}

// Solves L L^T x = b in place (forward, then backward substitution, each sum k ascending).
void substitute(const std::vector<double>& l, std::size_t p, double* x) {
  for (std::size_t i = 0; i < p; ++i) {
    double s = x[i];
    for (std::size_t k = 0; k < i; ++k) s -= l[i * p + k] * x[k];
    x[i] = s / l[i * p + i];
  }
  for (std::size_t i = p; i-- > 0;) {
    double s = x[i];
    for (std::size_t k = i + 1; k < p; ++k) s -= l[k * p + i] * x[k];
    x[i] = s / l[i * p + i];
  }
}

}  // namespace

struct zk_hermite {
  std::size_t dims = 0, degree = 0;
  std::vector<std::size_t> active;  // features with spread, in order
  std::vector<double> mean, scale;
  // Term t multiplies He_{power[j]}(z_{feature[j]}) for j in [termBegin[t], termBegin[t + 1]): its non-zero
  // exponents, feature order.
  std::vector<uint32_t> termBegin, feature, power;
  std::vector<double> beta, cov;

  std::size_t basisSize() const { return termBegin.empty() ? 0 : termBegin.size() - 1; }

  void setTerms(const std::vector<std::vector<unsigned>>& exps) {
    termBegin.assign(1, 0);
    feature.clear();
    power.clear();
    for (const auto& e : exps) {
      for (std::size_t f = 0; f < e.size(); ++f)
        if (e[f] > 0) feature.push_back(static_cast<uint32_t>(f)), power.push_back(e[f]);
      termBegin.push_back(static_cast<uint32_t>(feature.size()));
    }
  }

  // phi [p] of one feature row; he is scratch of active.size() x (degree + 1).
  void basis(const double* x, double* phi, double* he) const {
    const std::size_t w = degree + 1;
    for (std::size_t f = 0; f < active.size(); ++f) {
      const double z = (x[active[f]] - mean[active[f]]) / scale[active[f]];
      double* h = he + f * w;
      h[0] = 1.0;
      if (degree >= 1) h[1] = z;
      for (std::size_t k = 1; k < degree; ++k) h[k + 1] = z * h[k] - static_cast<double>(k) * h[k - 1];
    }
    const std::size_t p = basisSize();
    for (std::size_t t = 0; t < p; ++t) {
      double v = 1.0;
      for (uint32_t j = termBegin[t]; j < termBegin[t + 1]; ++j) v *= he[feature[j] * w + power[j]];
      phi[t] = v;
    }
  }

  // Design matrix [n][p] of the given rows, row-parallel.
  std::vector<double> design(const double* features, const uint64_t* rows, std::size_t n) const {
    const std::size_t p = basisSize();
    std::vector<double> phi(n * p);
    parallelFor(n, 256, [&](std::size_t b, std::size_t e) {
      std::vector<double> he(active.size() * (degree + 1));
      for (std::size_t k = b; k < e; ++k) basis(features + rows[k] * dims, &phi[k * p], he.data());
    });
    return phi;
  }
};

namespace {

// out[a][c] (c <= a) = sum over rows k in order of w_k phi_ka phi_kc, (w_k phi_ka) phi_kc when weighted; the
// upper triangle mirrored.  Parallel over row blocks of the triangle, each entry's sum sequential in k.
void symmetricAccumulate(const std::vector<double>& phi, std::size_t n, std::size_t p, const double* w, std::vector<double>& out) {
  out.assign(p * p, 0.0);
  const std::size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const std::size_t parts = std::min<std::size_t>({hw, 16, std::max<std::size_t>(1, n * p * p / 2000000)});
  const std::vector<std::size_t> cut = triangleCuts(p, parts);
  parallelFor(parts, 1, [&](std::size_t b, std::size_t e) {
    for (std::size_t part = b; part < e; ++part)
      for (std::size_t k = 0; k < n; ++k) {
        const double* row = &phi[k * p];
        for (std::size_t a = cut[part]; a < cut[part + 1]; ++a) {
          const double fa = w ? w[k] * row[a] : row[a];
          double* o = &out[a * p];
          for (std::size_t c = 0; c <= a; ++c) o[c] += fa * row[c];
        }
      }
  });
  for (std::size_t a = 0; a < p; ++a)
    for (std::size_t c = 0; c < a; ++c) out[c * p + a] = out[a * p + c];
}

// out = x y for p x p matrices, entry (a, c) summed over k ascending, terms with x_ak == 0 skipped.
void productSkippingZeros(const std::vector<double>& x, const std::vector<double>& y, std::size_t p, std::vector<double>& out) {
  out.assign(p * p, 0.0);
  parallelFor(p, std::max<std::size_t>(1, 4000000 / std::max<std::size_t>(p * p, 1)), [&](std::size_t b, std::size_t e) {
    for (std::size_t a = b; a < e; ++a) {
      double* o = &out[a * p];
      for (std::size_t k = 0; k < p; ++k) {
        const double v = x[a * p + k];
        if (v == 0.0) continue;
        const double* yk = &y[k * p];
        for (std::size_t c = 0; c < p; ++c) o[c] += v * yk[c];
      }
    }
  });
}

void setErr(char* err, std::size_t len, const char* what) {
  if (err && len) {
    std::strncpy(err, what, len - 1);
    err[len - 1] = 0;
  }
}

}  // namespace

extern "C" {

zk_status zk_hermite_fit(const double* features, size_t n_rows, size_t dims, const double* y, const uint64_t* rows, size_t n_train,
                         uint32_t degree, double ridge, zk_hermite** out, char* err, size_t err_len) {
  if (!features || !y || !rows || !out) return ZK_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  try {
    const std::size_t n = n_train;
    if (n < 2) throw std::invalid_argument("HermiteProxy: needs at least two training rows");
    for (std::size_t k = 0; k < n; ++k)
      if (rows[k] >= n_rows) throw std::invalid_argument("HermiteProxy: training row beyond the features");
    std::unique_ptr<zk_hermite> h(new zk_hermite());
    h->dims = dims;
    // Standardisation: the sample mean and standard deviation of each feature over the training rows.
    h->mean.assign(dims, 0.0);
    h->scale.assign(dims, 1.0);
    std::vector<double> ss(dims, 0.0);
    for (std::size_t k = 0; k < n; ++k)
      for (std::size_t j = 0; j < dims; ++j) h->mean[j] += features[rows[k] * dims + j];
    for (double& m : h->mean) m /= static_cast<double>(n);
    for (std::size_t k = 0; k < n; ++k)
      for (std::size_t j = 0; j < dims; ++j) {
        const double dv = features[rows[k] * dims + j] - h->mean[j];
        ss[j] += dv * dv;
      }
    for (std::size_t j = 0; j < dims; ++j) {
      const double sd = std::sqrt(ss[j] / static_cast<double>(n - 1));
      if (sd > 1e-12 * std::max(1.0, std::fabs(h->mean[j]))) h->scale[j] = sd, h->active.push_back(j);
    }
    // The largest degree that leaves at least two training rows per basis function.
    std::vector<std::vector<unsigned>> exps;
    std::size_t d = degree;
    for (;; --d) {
      gradedExponents(h->active.size(), d, exps);
      if (2 * exps.size() <= n || d == 0) break;
    }
    if (exps.size() > 2000) throw std::invalid_argument("HermiteProxy: more than 2000 basis functions");
    h->degree = d;
    h->setTerms(exps);
    const std::size_t p = h->basisSize();

    const std::vector<double> phi = h->design(features, rows, n);
    std::vector<double> gram, rhs(p, 0.0);
    symmetricAccumulate(phi, n, p, nullptr, gram);
    for (std::size_t k = 0; k < n; ++k)
      for (std::size_t a = 0; a < p; ++a) rhs[a] += phi[k * p + a] * y[rows[k]];
    double trace = 0.0;
    for (std::size_t a = 0; a < p; ++a) trace += gram[a * p + a];

    std::vector<double> l;
    for (double rg = ridge;; rg *= 1e3) {
      l = gram;
      const double lambda = rg * std::max(trace / static_cast<double>(p), 1e-300);
      for (std::size_t a = 0; a < p; ++a) l[a * p + a] += lambda;
      if (factor(l, p)) break;
      if (rg > 1e-2) throw std::invalid_argument("HermiteProxy: normal equations are singular");
    }
    h->beta = rhs;
    substitute(l, p, h->beta.data());

    // Squared residuals of the training rows, then the sandwich.
    std::vector<double> e2(n);
    for (std::size_t k = 0; k < n; ++k) {
      double fitted = 0.0;
      for (std::size_t a = 0; a < p; ++a) fitted += phi[k * p + a] * h->beta[a];
      const double r = y[rows[k]] - fitted;
      e2[k] = r * r;
    }
    std::vector<double> meat;
    symmetricAccumulate(phi, n, p, e2.data(), meat);
    // G^-1 column by column (column c solves the unit vector e_c), stored transposed then mirrored back.
    std::vector<double> inverseT(p * p, 0.0), inverse(p * p);
    parallelFor(p, std::max<std::size_t>(1, 2000000 / std::max<std::size_t>(p * p, 1)), [&](std::size_t b, std::size_t e) {
      for (std::size_t c = b; c < e; ++c) {
        double* col = &inverseT[c * p];
        col[c] = 1.0;
        substitute(l, p, col);
      }
    });
    for (std::size_t r = 0; r < p; ++r)
      for (std::size_t c = 0; c < p; ++c) inverse[r * p + c] = inverseT[c * p + r];
    std::vector<double> tmp;
    productSkippingZeros(inverse, meat, p, tmp);
    productSkippingZeros(tmp, inverse, p, h->cov);
    *out = h.release();
    return ZK_OK;
  } catch (const std::exception& e) {
    setErr(err, err_len, e.what());
    return ZK_ERR_INVALID_ARGUMENT;
  }
}

zk_status zk_hermite_predict(const zk_hermite* h, const double* features, size_t n_rows, size_t dims, const uint64_t* rows, size_t n,
                             double* value, double* variance) {
  if (!h || (n > 0 && (!features || !rows || !value || !variance)) || dims != h->dims) return ZK_ERR_INVALID_ARGUMENT;
  for (std::size_t k = 0; k < n; ++k)
    if (rows[k] >= n_rows) return ZK_ERR_INVALID_ARGUMENT;
  const std::size_t p = h->basisSize();
  // Four rows at a time: each row's sums keep their own order, and the four independent chains hide the
  // latency of the in-order additions.
  constexpr std::size_t kRows = 4;
  const std::size_t groups = (n + kRows - 1) / kRows;
  parallelFor(groups, std::max<std::size_t>(1, 250000 / std::max<std::size_t>(p * p, 1)), [&](std::size_t b, std::size_t e) {
    std::vector<double> phi(kRows * p), he(h->active.size() * (h->degree + 1));
    for (std::size_t g = b; g < e; ++g) {
      const std::size_t k0 = g * kRows, m = std::min(kRows, n - k0);
      for (std::size_t r = 0; r < kRows; ++r)  // short groups repeat their last row
        h->basis(features + rows[k0 + std::min(r, m - 1)] * dims, &phi[r * p], he.data());
      double v[kRows] = {}, var[kRows] = {};
      for (std::size_t a = 0; a < p; ++a) {
        const double* ca = &h->cov[a * p];
        double u[kRows] = {};
        for (std::size_t c = 0; c < p; ++c)
          for (std::size_t r = 0; r < kRows; ++r) u[r] += ca[c] * phi[r * p + c];
        for (std::size_t r = 0; r < kRows; ++r) {
          v[r] += phi[r * p + a] * h->beta[a];
          var[r] += phi[r * p + a] * u[r];
        }
      }
      for (std::size_t r = 0; r < m; ++r) value[k0 + r] = v[r], variance[k0 + r] = std::max(var[r], 0.0);
    }
  });
  return ZK_OK;
}

zk_status zk_hermite_info(const zk_hermite* h, uint64_t* degree_and_basis) {
  if (!h || !degree_and_basis) return ZK_ERR_INVALID_ARGUMENT;
  degree_and_basis[0] = h->degree;
  degree_and_basis[1] = h->basisSize();
  return ZK_OK;
}

void zk_hermite_destroy(zk_hermite* h) { delete h; }

zk_status zk_erfc_array(const double* x, size_t n, double* out) {
  if (n > 0 && (!x || !out)) return ZK_ERR_INVALID_ARGUMENT;
  for (std::size_t k = 0; k < n; ++k) out[k] = std::erfc(x[k]);
  return ZK_OK;
}

}  // extern "C"

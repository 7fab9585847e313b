// oracle/oracle_bounce.h -- TEST INFRASTRUCTURE (the oracle): the numerics of the W6 bounce passes,
// restated from riftphys-world/src/world/bounce_lcp.rs:1-330 (the contact matrix held sparse, a
// sparse Cholesky in a fixed minimum-degree order, the velocity pass's interior-point LCP solve and
// the pseudo pass's equality solve) and solver.rs:115-200 (row sides, the contact matrix, the row
// components). f64 throughout, every sum in the reference's order. Only the oracle's World::step
// uses it.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <set>
#include <utility>
#include <vector>

namespace orc {
namespace bounce {

struct D3 { double x, y, z; };
static inline D3 dadd(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline D3 dmul(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
static inline double ddot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline D3 dcross(D3 a, D3 b) { return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// DMat3 by columns; m * v = (c0 x + c1 y) + c2 z
struct DM3 { D3 c0, c1, c2; };
static inline D3 dmvec(const DM3& m, D3 v) { return dadd(dadd(dmul(m.c0, v.x), dmul(m.c1, v.y)), dmul(m.c2, v.z)); }

// One side of a contact row (solver.rs:115): the body (0xFFFFFFFF: cannot move), its Jacobian
// (linear, angular) and M^-1 J^T.
struct RowSide { uint32_t body; D3 jl, ja, mjl, mja; };
constexpr uint32_t kNone = 0xFFFFFFFFu;

// Symmetric sparse matrix, both triangles, each row's columns ascending (bounce_lcp.rs:11-60).
struct Csr {
  size_t n = 0;
  std::vector<size_t> ptr, idx;
  std::vector<double> val;
  static Csr from_rows(const std::vector<std::vector<std::pair<size_t, double>>>& rows) {
    Csr m;
    m.n = rows.size();
    m.ptr.push_back(0);
    for (auto& r : rows) {
      for (auto& e : r) { m.idx.push_back(e.first); m.val.push_back(e.second); }
      m.ptr.push_back(m.idx.size());
    }
    return m;
  }
  Csr with_compliance(double c) const {
    Csr m = *this;
    for (size_t i = 0; i < n; ++i)
      for (size_t t = m.ptr[i]; t < m.ptr[i + 1]; ++t)
        if (m.idx[t] == i) m.val[t] *= 1.0 + c;
    return m;
  }
  double diag(size_t i) const {
    for (size_t t = ptr[i]; t < ptr[i + 1]; ++t)
      if (idx[t] == i) return val[t];
    return 0.0;
  }
  double row_dot(size_t i, const std::vector<double>& x) const {
    double s = 0.0;
    for (size_t t = ptr[i]; t < ptr[i + 1]; ++t) s += val[t] * x[idx[t]];
    return s;
  }
  std::vector<double> mul(const std::vector<double>& x) const {
    std::vector<double> y(n);
    for (size_t i = 0; i < n; ++i) y[i] = row_dot(i, x);
    return y;
  }
};

// The elimination order and the factor's structure from the row graph alone
// (bounce_lcp.rs:62-148): minimum degree, the lowest row index on ties.
struct Symbolic {
  std::vector<size_t> order, pos, cp, ri, rp, re, ce;
  static Symbolic min_degree(const Csr& k) {
    const size_t n = k.n;
    std::vector<std::vector<size_t>> adj(n), nbs(n);
    for (size_t i = 0; i < n; ++i)
      for (size_t t = k.ptr[i]; t < k.ptr[i + 1]; ++t)
        if (k.idx[t] != i) adj[i].push_back(k.idx[t]);
    std::set<std::pair<size_t, size_t>> queue;
    for (size_t i = 0; i < n; ++i) queue.insert({adj[i].size(), i});
    Symbolic s;
    std::vector<size_t> merged;
    while (!queue.empty()) {
      size_t v = queue.begin()->second;
      queue.erase(queue.begin());
      s.order.push_back(v);
      std::vector<size_t> nb;
      std::swap(nb, adj[v]);
      for (size_t u : nb) {
        queue.erase({adj[u].size(), u});
        merged.clear();
        const std::vector<size_t>& a = adj[u];
        size_t x = 0, y = 0;
        while (x < a.size() || y < nb.size()) {
          size_t next;
          if (y >= nb.size() || (x < a.size() && a[x] < nb[y])) next = a[x++];
          else if (x >= a.size() || nb[y] < a[x]) next = nb[y++];
          else { next = a[x]; ++x; ++y; }
          if (next != v && next != u) merged.push_back(next);
        }
        std::swap(adj[u], merged);
        queue.insert({adj[u].size(), u});
      }
      nbs[v] = nb;
    }
    s.pos.assign(n, 0);
    for (size_t p = 0; p < n; ++p) s.pos[s.order[p]] = p;
    s.cp.push_back(0);
    for (size_t r : s.order) {
      size_t start = s.ri.size();
      for (size_t u : nbs[r]) s.ri.push_back(s.pos[u]);
      std::sort(s.ri.begin() + (long)start, s.ri.end());
      s.cp.push_back(s.ri.size());
    }
    std::vector<size_t> count(n + 1, 0);
    for (size_t p : s.ri) count[p + 1] += 1;
    for (size_t p = 0; p < n; ++p) count[p + 1] += count[p];
    s.rp = count;
    s.re.assign(s.ri.size(), 0);
    s.ce.assign(s.ri.size(), 0);
    std::vector<size_t> fill = count;
    for (size_t kc = 0; kc < n; ++kc)
      for (size_t e = s.cp[kc]; e < s.cp[kc + 1]; ++e) {
        s.re[fill[s.ri[e]]] = e;
        fill[s.ri[e]] += 1;
        s.ce[e] = s.cp[kc + 1];
      }
    return s;
  }
};

// The sparse factor of K + diag(d) (bounce_lcp.rs:157-185)
struct Factor { std::vector<double> diag, vals; };
static inline Factor factor(const Csr& k, const Symbolic& sym, const std::vector<double>& d) {
  const size_t n = k.n;
  std::vector<double> work(n, 0.0);
  Factor f;
  f.diag.assign(n, 0.0);
  f.vals.assign(sym.ri.size(), 0.0);
  for (size_t j = 0; j < n; ++j) {
    size_t r = sym.order[j];
    for (size_t t = k.ptr[r]; t < k.ptr[r + 1]; ++t) {
      size_t p = sym.pos[k.idx[t]];
      if (p >= j) work[p] += k.val[t];
    }
    work[j] += d[r];
    for (size_t q = sym.rp[j]; q < sym.rp[j + 1]; ++q) {
      size_t e = sym.re[q];
      double ljk = f.vals[e];
      size_t end = sym.ce[e];
      for (size_t t = 0; e + t < end; ++t) work[sym.ri[e + t]] -= f.vals[e + t] * ljk;
    }
    double ljj = std::sqrt(std::fmax(work[j], 1e-300));
    f.diag[j] = ljj;
    work[j] = 0.0;
    for (size_t t = sym.cp[j]; t < sym.cp[j + 1]; ++t) {
      size_t p = sym.ri[t];
      f.vals[t] = work[p] / ljj;
      work[p] = 0.0;
    }
  }
  return f;
}
// bounce_lcp.rs:195-211
static inline std::vector<double> solve(const Factor& f, const Symbolic& sym, const std::vector<double>& b) {
  const size_t n = b.size();
  std::vector<double> y(n);
  for (size_t p = 0; p < n; ++p) y[p] = b[sym.order[p]];
  for (size_t j = 0; j < n; ++j) {
    y[j] /= f.diag[j];
    double yj = y[j];
    for (size_t t = sym.cp[j]; t < sym.cp[j + 1]; ++t) y[sym.ri[t]] -= f.vals[t] * yj;
  }
  for (size_t j = n; j-- > 0;) {
    double v = y[j];
    for (size_t t = sym.cp[j]; t < sym.cp[j + 1]; ++t) v -= f.vals[t] * y[sym.ri[t]];
    y[j] = v / f.diag[j];
  }
  std::vector<double> x(n, 0.0);
  for (size_t p = 0; p < n; ++p) x[sym.order[p]] = y[p];
  return x;
}

constexpr double kCfm = 1e-12;  // CFM (bounce_lcp.rs:216)

// bounce_qp (bounce_lcp.rs:249-315): Mehrotra predictor-corrector on the LCP
// w = K (acc0 + x) - ... >= 0, y = acc0 + x >= 0, y w = 0, at most cap solves. Returns
// (x, converged, solves).
struct QpResult { std::vector<double> x; bool converged = false; size_t solves = 0; };
static inline QpResult bounce_qp(const Csr& k0, const std::vector<double>& b, const std::vector<double>& acc0, size_t cap) {
  const size_t n = k0.n;
  const Csr k = k0.with_compliance(kCfm);
  const Symbolic sym = Symbolic::min_degree(k);
  QpResult out;
  std::vector<double> kdiag(n);
  for (size_t i = 0; i < n; ++i) kdiag[i] = k0.diag(i);
  std::vector<double> ka = k.mul(acc0), q(n);
  for (size_t i = 0; i < n; ++i) q[i] = -ka[i] - b[i];
  double qmax = 0.0;
  for (size_t i = 0; i < n; ++i) qmax = std::fmax(qmax, std::fabs(q[i]));
  const double eta = std::fmax(1.0, qmax);
  std::vector<double> y(n), w(n, eta);
  for (size_t i = 0; i < n; ++i) y[i] = kdiag[i] > 0.0 ? eta / kdiag[i] : 1.0;
  auto step = [&](const std::vector<double>& dy, const std::vector<double>& dw) {
    double a = 1.0;
    for (size_t i = 0; i < n; ++i) {
      if (dy[i] < 0.0) a = std::fmin(a, -y[i] / dy[i]);
      if (dw[i] < 0.0) a = std::fmin(a, -w[i] / dw[i]);
    }
    return a;
  };
  const double nn = (double)n;
  for (size_t it = 1; it <= cap; ++it) {
    out.solves = it;
    std::vector<double> ky = k.mul(y), r(n);
    for (size_t i = 0; i < n; ++i) r[i] = (ky[i] + q[i]) - w[i];
    double mu_sum = -0.0;
    for (size_t i = 0; i < n; ++i) mu_sum += y[i] * w[i];
    const double mu = mu_sum / nn;
    double rmax = 0.0;
    for (size_t i = 0; i < n; ++i) rmax = std::fmax(rmax, std::fabs(r[i]));
    std::vector<double> x(n);
    for (size_t i = 0; i < n; ++i) x[i] = y[i] - acc0[i];
    std::vector<double> kx = k0.mul(x), wt(n);
    for (size_t i = 0; i < n; ++i) wt[i] = kx[i] - b[i];
    if (rmax < 1e-7) {
      bool ok = true;
      for (size_t i = 0; i < n && ok; ++i) {
        double tol = 1e-7 * (1.0 + std::fabs(b[i]));
        ok = wt[i] >= -tol && std::fmin(std::fabs(wt[i]), y[i] * kdiag[i]) < tol;
      }
      if (ok) {
        out.converged = true;
        out.x = x;
        return out;
      }
    }
    std::vector<double> d(n);
    for (size_t i = 0; i < n; ++i) d[i] = w[i] / y[i];
    const Factor f = factor(k, sym, d);
    auto dirs = [&](const std::vector<double>& target, std::vector<double>& dy, std::vector<double>& dw) {
      std::vector<double> rhs(n);
      for (size_t i = 0; i < n; ++i) rhs[i] = -r[i] + target[i] / y[i];
      dy = solve(f, sym, rhs);
      dw.assign(n, 0.0);
      for (size_t i = 0; i < n; ++i) dw[i] = (target[i] - w[i] * dy[i]) / y[i];
    };
    std::vector<double> aff(n), dya, dwa;
    for (size_t i = 0; i < n; ++i) aff[i] = -y[i] * w[i];
    dirs(aff, dya, dwa);
    const double aa = step(dya, dwa);
    double maff = -0.0;
    for (size_t i = 0; i < n; ++i) maff += (y[i] + aa * dya[i]) * (w[i] + aa * dwa[i]);
    const double mu_aff = maff / nn;
    const double ratio = mu_aff / std::fmax(mu, 1e-300);
    const double sigma = std::fmin(ratio * ratio * ratio, 1.0);
    std::vector<double> cor(n), dy, dw;
    for (size_t i = 0; i < n; ++i) cor[i] = (sigma * mu - y[i] * w[i]) - dya[i] * dwa[i];
    dirs(cor, dy, dw);
    const double a = std::fmin(0.995 * step(dy, dw), 1.0);
    bool finite = std::isfinite(a);
    for (size_t i = 0; i < n && finite; ++i) finite = std::isfinite(dy[i]) && std::isfinite(dw[i]);
    if (!finite) break;
    for (size_t i = 0; i < n; ++i) {
      y[i] = std::fmax(y[i] + a * dy[i], 1e-300);
      w[i] = std::fmax(w[i] + a * dw[i], 1e-300);
    }
  }
  out.x.resize(n);
  for (size_t i = 0; i < n; ++i) out.x[i] = y[i] - acc0[i];
  return out;
}

// pseudo_solve (bounce_lcp.rs:317-324): (K + CFM diag K) x = u
static inline std::vector<double> pseudo_solve(const Csr& k, const std::vector<double>& u) {
  std::vector<double> d(k.n);
  for (size_t i = 0; i < k.n; ++i) d[i] = kCfm * k.diag(i);
  const Symbolic sym = Symbolic::min_degree(k);
  return solve(factor(k, sym, d), sym, u);
}

// contact_csr (solver.rs:136-168): K = J M^-1 J^T over shared moving bodies, row i's sides first.
static inline Csr contact_csr(const std::vector<std::array<RowSide, 2>>& sides) {
  const size_t n = sides.size();
  std::map<uint32_t, std::vector<std::pair<size_t, size_t>>> by_body;
  for (size_t i = 0; i < n; ++i)
    for (size_t t = 0; t < 2; ++t)
      if (sides[i][t].body != kNone) by_body[sides[i][t].body].push_back({i, t});
  std::vector<double> acc(n, 0.0);
  std::vector<bool> seen(n, false);
  std::vector<std::vector<std::pair<size_t, double>>> rows;
  rows.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    std::vector<size_t> touched{i};
    seen[i] = true;
    for (size_t t = 0; t < 2; ++t) {
      const RowSide& si = sides[i][t];
      if (si.body == kNone) continue;
      for (auto& jt : by_body[si.body]) {
        const RowSide& sj = sides[jt.first][jt.second];
        acc[jt.first] += ddot(si.jl, sj.mjl) + ddot(si.ja, sj.mja);
        if (!seen[jt.first]) { seen[jt.first] = true; touched.push_back(jt.first); }
      }
    }
    std::sort(touched.begin(), touched.end());
    std::vector<std::pair<size_t, double>> row;
    for (size_t j : touched) { row.push_back({j, acc[j]}); acc[j] = 0.0; seen[j] = false; }
    rows.push_back(std::move(row));
  }
  return Csr::from_rows(rows);
}

// row_components (solver.rs:170-195): rows linked through a moving body; rows ascending in each,
// components ordered by their first row.
static inline std::vector<std::vector<size_t>> row_components(const std::vector<std::array<RowSide, 2>>& sides,
                                                               size_t num_bodies) {
  std::vector<uint32_t> parent(num_bodies);
  for (size_t i = 0; i < num_bodies; ++i) parent[i] = (uint32_t)i;
  auto find = [&](uint32_t x) {
    while (parent[x] != x) { uint32_t g = parent[parent[x]]; parent[x] = g; x = g; }
    return x;
  };
  for (auto& sd : sides)
    if (sd[0].body != kNone && sd[1].body != kNone) {
      uint32_t a = find(sd[0].body), b = find(sd[1].body);
      if (a != b) parent[a > b ? a : b] = a < b ? a : b;
    }
  std::vector<size_t> slot(num_bodies, (size_t)-1);
  std::vector<std::vector<size_t>> comps;
  for (size_t i = 0; i < sides.size(); ++i) {
    uint32_t body = sides[i][0].body != kNone ? sides[i][0].body : sides[i][1].body;
    if (body == kNone) { comps.push_back({i}); continue; }
    uint32_t r = find(body);
    if (slot[r] == (size_t)-1) { slot[r] = comps.size(); comps.emplace_back(); }
    comps[slot[r]].push_back(i);
  }
  return comps;
}

}  // namespace bounce
}  // namespace orc

// bounce.cuh -- the W6 bounce passes on the GPU (riftphys-world/src/world/solver.rs:1009-1241 and
// bounce_lcp.rs:1-330), included by step_solve.cu after its row helpers.
//
// Free bodies' contacts approaching faster than 1 m/s with restitution bounce at their time of
// impact: each gets its end-of-step velocity target (toi_bounce), the bounced bodies' other loaded
// contacts join as push-only supports, and every connected component of those rows is solved
// alone -- up to 250 rows by the interior-point LCP over a sparse Cholesky in minimum-degree order
// (f64, every sum in the reference's order), larger or unconverged ones by Gauss-Seidel sweeps.
// The pseudo pass then gives the bounced pairs pseudo-velocities that the integration adds to
// their motion. Bounces are rare and small, so the passes run as a few single-block kernels over
// the tick's rows (the scans and the support growth) and one thread per component for the solves;
// every kernel returns at once when no row bounces (the counter the first kernel fills).
#pragma once

// (included inside namespace rp)
namespace w6 {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kSupport = 0x80000000u;  // a W6 row list entry: contact index, | kSupport for a support
constexpr uint32_t kDirectMax = 250, kSweeps = 256, kSolves = 64;
constexpr float kTol = 1e-6f;
constexpr uint32_t kErrCapacity = 2u;  // RPHYS_STATERR_CAPACITY: a per-step buffer overflowed
constexpr double kCfm = 1e-12;
// counters: toi rows, W6 rows, components, pseudo rows, pool bytes used (low, high), pseudo on
enum : uint32_t { C_TOI = 0, C_ROWS = 1, C_COMPS = 2, C_PSEUDO = 3, C_POOL = 4, C_PON = 6, C_NTOI = 7, C_N = 8 };

struct D3 { double x, y, z; };
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 dmul(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
  return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
struct Side { uint32_t body; D3 jl, ja, mjl, mja; };

// Device view of the pass's scratch (world-owned arrays; nb per-body, nc per-contact entries).
struct W6V {
  uint32_t *rest_cnt, *rest_min, *rest_max, *parent, *slot;
  uint8_t *involved, *direct, *in_set, *has_pseudo;
  double* acc;          // 6 per body: the pseudo solve's linear and angular sums
  float4 *pl, *pa;      // pseudo-velocities (linear, angular) per body
  uint32_t* rows;       // W6 rows: toi rows first (contact order), then supports
  float *target, *sup_acc, *pseudo_u;
  uint32_t *comp_rows, *comp_start, *row_comp, *cur;
  uint32_t* ctr;
  uint8_t* pool;
  unsigned long long pool_bytes;
  const float4* toi_a;  // per contact: (s0, e, va start, va after)
  const float2* toi_b;  // per contact: (vb start, vb after)
};

__device__ __forceinline__ bool toi_set(const RowsV& R, const float* acc_jn, uint32_t c) {
  return (R.flags[c] & RF_TOI) && R.t2[c].w > 0.0f && acc_jn[c] > 0.0f;
}
__device__ __forceinline__ bool loaded_at(const float* acc_jn, const float2* acc_jt, uint32_t c) {
  float2 t = acc_jt[c];
  return acc_jn[c] > 0.0f || t.x != 0.0f || t.y != 0.0f;
}
// free_only (solver.rs:1030-1039): jointed sides immovable, the normal effective mass recomputed;
// false if neither side moves. On the GPU a row's world inverse inertias are the tick's B.Iw.
__device__ __forceinline__ bool free_only(const BodiesV& B, const uint8_t* jointed, Row& r) {
  const bool terrain = (r.flags & RF_TERRAIN) != 0;
  if (jointed && jointed[r.ai]) r.inv_a = 0.0f;
  if (terrain || (jointed && jointed[r.bi])) r.inv_b = 0.0f;
  m3 ia = r.inv_a > 0.0f ? ld_m3(B.Iw, r.ai) : mzero(), ib = r.inv_b > 0.0f ? ld_m3(B.Iw, r.bi) : mzero();
  f3 ca = cross(r.ra, r.n), cb = cross(r.rb, r.n);
  float k = ((r.inv_a + r.inv_b) + dot(ca, mvec(ia, ca))) + dot(cb, mvec(ib, cb));
  if (!(k > 1e-9f)) return false;
  r.m_n = 1.0f / k;
  return true;
}
// A W6 row: the contact's row, made free_only for a support (or for every pseudo-pass row).
__device__ __forceinline__ Row w6_row(const RowsV& R, const BodiesV& B, const uint8_t* jointed, uint32_t e, bool free) {
  Row r = ld_row(R, e & ~kSupport);
  if (free) free_only(B, jointed, r);
  return r;
}
// row_sides (solver.rs:117-134)
__device__ __forceinline__ void row_sides(const BodiesV& B, const Row& r, Side s[2]) {
  const D3 n{r.n.x, r.n.y, r.n.z};
  auto side = [&](uint32_t body, double sign, f3 rr, float inv, Side& o) {
    if (inv <= 0.0f) { o.body = kNone; o.jl = o.ja = o.mjl = o.mja = D3{0, 0, 0}; return; }
    m3 ii = ld_m3(B.Iw, body);
    o.body = body;
    o.jl = dmul(n, sign);
    o.ja = dmul(dcross(D3{rr.x, rr.y, rr.z}, n), sign);
    D3 c0{ii.c0.x, ii.c0.y, ii.c0.z}, c1{ii.c1.x, ii.c1.y, ii.c1.z}, c2{ii.c2.x, ii.c2.y, ii.c2.z};
    D3 t0{c0.x, c1.x, c2.x}, t1{c0.y, c1.y, c2.y}, t2{c0.z, c1.z, c2.z};
    D3 s0 = dmul(dadd(c0, t0), 0.5), s1 = dmul(dadd(c1, t1), 0.5), s2 = dmul(dadd(c2, t2), 0.5);
    o.mjl = dmul(o.jl, (double)inv);
    o.mja = dadd(dadd(dmul(s0, o.ja.x), dmul(s1, o.ja.y)), dmul(s2, o.ja.z));
  };
  side(r.ai, -1.0, r.ra, r.inv_a, s[0]);
  side(r.bi, 1.0, r.rb, (r.flags & RF_TERRAIN) ? 0.0f : r.inv_b, s[1]);
}
// toi_bounce (solver.rs:203-219)
__device__ __forceinline__ void toi_bounce(float s0, float v0, float a, float e, float dt, float* v_end_o, bool* has,
                                           float* u) {
  float t_c;
  if (s0 <= 0.0f) t_c = 0.0f;
  else {
    float disc = v0 * v0 - 2.0f * a * s0;
    float den = disc >= 0.0f ? -v0 + sqrtf(disc) : 0.0f;
    t_c = den > 0.0f ? rmin(2.0f * s0 / den, dt) : dt;
  }
  float v_out = rmax(-e * (v0 + a * t_c), 0.0f);
  float tau = dt - t_c;
  float rise = v_out * tau + 0.5f * a * tau * tau;
  float v_end, s_end;
  if (rise < 0.0f) { v_end = 0.0f; s_end = 0.0f; }
  else { v_end = rmax(v_out + a * tau, 0.0f); s_end = rise; }
  *v_end_o = v_end;
  *has = s0 > 0.0f;
  *u = (s_end - s0) / dt - v_end;
}

// ---- the direct solves, one thread per component, scratch carved from the pool
struct Arena {
  uint8_t* p;
  unsigned long long left;
  bool ok;
  template <class T>
  __device__ T* take(unsigned long long n) {
    unsigned long long bytes = (n * sizeof(T) + 15ull) & ~15ull;
    if (!ok || bytes > left) { ok = false; return nullptr; }
    T* r = reinterpret_cast<T*>(p);
    p += bytes;
    left -= bytes;
    return r;
  }
};
// Bytes a component of n rows may take (an upper bound of every array below).
__host__ __device__ inline unsigned long long arena_bytes(unsigned long long n) {
  return 64ull * n * n + 1024ull * n + 4096ull;
}
__device__ __forceinline__ bool arena_open(const W6V& V, unsigned long long n, Arena* a) {
  unsigned long long want = arena_bytes(n);
  unsigned long long at = atomicAdd(reinterpret_cast<unsigned long long*>(V.ctr + C_POOL), want);
  a->ok = at + want <= V.pool_bytes;
  a->p = V.pool + at;
  a->left = a->ok ? want : 0ull;
  return a->ok;
}
// CSR of a symmetric matrix, both triangles, columns ascending (bounce_lcp.rs:11-60)
struct Csr { uint32_t n; uint32_t* ptr; uint32_t* idx; double* val; };
__device__ double csr_diag(const Csr& k, uint32_t i) {
  for (uint32_t t = k.ptr[i]; t < k.ptr[i + 1]; ++t)
    if (k.idx[t] == i) return k.val[t];
  return 0.0;
}
__device__ void csr_mul(const Csr& k, const double* x, double* y) {
  for (uint32_t i = 0; i < k.n; ++i) {
    double s = 0.0;
    for (uint32_t t = k.ptr[i]; t < k.ptr[i + 1]; ++t) s += k.val[t] * x[k.idx[t]];
    y[i] = s;
  }
}
// contact_csr (solver.rs:136-168): K_ij over the moving bodies rows i and j share, row i's sides
// first; by_body lists each body's (row, side) in row order.
__device__ bool contact_csr(const Side* sides, uint32_t n, Arena& ar, Csr* out) {
  uint32_t* eb = ar.take<uint32_t>(2 * (unsigned long long)n);  // entries sorted by (body, row, side)
  uint32_t* ek = ar.take<uint32_t>(2 * (unsigned long long)n);  // 2 * row + side
  double* acc = ar.take<double>(n);
  uint8_t* seen = ar.take<uint8_t>(n);
  out->ptr = ar.take<uint32_t>(n + 1ull);
  out->idx = ar.take<uint32_t>((unsigned long long)n * n);
  out->val = ar.take<double>((unsigned long long)n * n);
  if (!ar.ok) return false;
  out->n = n;
  uint32_t m = 0;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t t = 0; t < 2; ++t)
      if (sides[2 * i + t].body != kNone) {
        // insertion in (body, row, side) order: entries arrive in (row, side) order already
        uint32_t b = sides[2 * i + t].body, q = m++;
        while (q > 0 && eb[q - 1] > b) { eb[q] = eb[q - 1]; ek[q] = ek[q - 1]; --q; }
        eb[q] = b;
        ek[q] = 2 * i + t;
      }
  for (uint32_t i = 0; i < n; ++i) { acc[i] = 0.0; seen[i] = 0; }
  uint32_t nnz = 0;
  out->ptr[0] = 0;
  for (uint32_t i = 0; i < n; ++i) {
    seen[i] = 1;
    for (uint32_t t = 0; t < 2; ++t) {
      const Side& si = sides[2 * i + t];
      if (si.body == kNone) continue;
      uint32_t lo = 0, hi = m;  // first entry of this body
      while (lo < hi) { uint32_t mid = (lo + hi) >> 1; if (eb[mid] < si.body) lo = mid + 1; else hi = mid; }
      for (uint32_t q = lo; q < m && eb[q] == si.body; ++q) {
        uint32_t j = ek[q] >> 1;
        const Side& sj = sides[ek[q]];
        acc[j] += ddot(si.jl, sj.mjl) + ddot(si.ja, sj.mja);
        seen[j] = 1;
      }
    }
    for (uint32_t j = 0; j < n; ++j)
      if (seen[j]) { out->idx[nnz] = j; out->val[nnz] = acc[j]; ++nnz; acc[j] = 0.0; seen[j] = 0; }
    out->ptr[i + 1] = nnz;
  }
  return true;
}
// Symbolic::min_degree (bounce_lcp.rs:83-148): eliminate the vertex of least (degree, index),
// merging its neighbour list into each neighbour's; then the factor's column structure.
struct Sym { uint32_t *order, *pos, *cp, *ri, *rp, *re, *ce; };
__device__ bool min_degree(const Csr& k, Arena& ar, Sym* s) {
  const uint32_t n = k.n;
  uint32_t* adj = ar.take<uint32_t>((unsigned long long)n * n);
  uint32_t* alen = ar.take<uint32_t>(n);
  uint32_t* nbs = ar.take<uint32_t>((unsigned long long)n * n);
  uint32_t* nlen = ar.take<uint32_t>(n);
  uint32_t* merged = ar.take<uint32_t>(n);
  uint8_t* done = ar.take<uint8_t>(n);
  s->order = ar.take<uint32_t>(n);
  s->pos = ar.take<uint32_t>(n);
  s->cp = ar.take<uint32_t>(n + 1ull);
  s->ri = ar.take<uint32_t>((unsigned long long)n * n);
  s->rp = ar.take<uint32_t>(n + 1ull);
  s->re = ar.take<uint32_t>((unsigned long long)n * n);
  s->ce = ar.take<uint32_t>((unsigned long long)n * n);
  uint32_t* fill = ar.take<uint32_t>(n + 1ull);
  if (!ar.ok) return false;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t c = 0;
    for (uint32_t t = k.ptr[i]; t < k.ptr[i + 1]; ++t)
      if (k.idx[t] != i) adj[(size_t)i * n + c++] = k.idx[t];
    alen[i] = c;
    done[i] = 0;
  }
  for (uint32_t step = 0; step < n; ++step) {
    uint32_t v = kNone;
    for (uint32_t i = 0; i < n; ++i)
      if (!done[i] && (v == kNone || alen[i] < alen[v])) v = i;  // ties: the lowest index
    done[v] = 1;
    s->order[step] = v;
    uint32_t* nb = nbs + (size_t)v * n;
    const uint32_t nn = alen[v];
    for (uint32_t q = 0; q < nn; ++q) nb[q] = adj[(size_t)v * n + q];
    nlen[v] = nn;
    alen[v] = 0;
    for (uint32_t q = 0; q < nn; ++q) {
      const uint32_t u = nb[q];
      const uint32_t* a = adj + (size_t)u * n;
      const uint32_t na = alen[u];
      uint32_t x = 0, y = 0, m = 0;
      while (x < na || y < nn) {
        uint32_t next;
        if (y >= nn || (x < na && a[x] < nb[y])) next = a[x++];
        else if (x >= na || nb[y] < a[x]) next = nb[y++];
        else { next = a[x]; ++x; ++y; }
        if (next != v && next != u) merged[m++] = next;
      }
      for (uint32_t t = 0; t < m; ++t) adj[(size_t)u * n + t] = merged[t];
      alen[u] = m;
    }
  }
  for (uint32_t p = 0; p < n; ++p) s->pos[s->order[p]] = p;
  uint32_t nri = 0;
  s->cp[0] = 0;
  for (uint32_t p = 0; p < n; ++p) {
    const uint32_t r = s->order[p];
    const uint32_t start = nri;
    for (uint32_t q = 0; q < nlen[r]; ++q) {
      uint32_t val = s->pos[nbs[(size_t)r * n + q]], z = nri++;
      while (z > start && s->ri[z - 1] > val) { s->ri[z] = s->ri[z - 1]; --z; }
      s->ri[z] = val;
    }
    s->cp[p + 1] = nri;
  }
  for (uint32_t p = 0; p <= n; ++p) fill[p] = 0;
  for (uint32_t e = 0; e < nri; ++e) fill[s->ri[e] + 1] += 1;
  for (uint32_t p = 0; p < n; ++p) fill[p + 1] += fill[p];
  for (uint32_t p = 0; p <= n; ++p) s->rp[p] = fill[p];
  for (uint32_t kc = 0; kc < n; ++kc)
    for (uint32_t e = s->cp[kc]; e < s->cp[kc + 1]; ++e) {
      s->re[fill[s->ri[e]]] = e;
      fill[s->ri[e]] += 1;
      s->ce[e] = s->cp[kc + 1];
    }
  return true;
}
// factor / solve (bounce_lcp.rs:157-211), the sparse path
__device__ void factor(const Csr& k, const Sym& s, const double* d, double* work, double* diag, double* vals) {
  const uint32_t n = k.n;
  for (uint32_t j = 0; j < n; ++j) work[j] = 0.0;
  for (uint32_t j = 0; j < n; ++j) {
    const uint32_t r = s.order[j];
    for (uint32_t t = k.ptr[r]; t < k.ptr[r + 1]; ++t) {
      uint32_t p = s.pos[k.idx[t]];
      if (p >= j) work[p] += k.val[t];
    }
    work[j] += d[r];
    for (uint32_t q = s.rp[j]; q < s.rp[j + 1]; ++q) {
      const uint32_t e = s.re[q];
      const double ljk = vals[e];
      const uint32_t end = s.ce[e];
      for (uint32_t t = e; t < end; ++t) work[s.ri[t]] -= vals[t] * ljk;
    }
    const double ljj = sqrt(fmax(work[j], 1e-300));
    diag[j] = ljj;
    work[j] = 0.0;
    for (uint32_t t = s.cp[j]; t < s.cp[j + 1]; ++t) {
      uint32_t p = s.ri[t];
      vals[t] = work[p] / ljj;
      work[p] = 0.0;
    }
  }
}
__device__ void fsolve(const Sym& s, uint32_t n, const double* diag, const double* vals, const double* b, double* y,
                       double* x) {
  for (uint32_t p = 0; p < n; ++p) y[p] = b[s.order[p]];
  for (uint32_t j = 0; j < n; ++j) {
    y[j] /= diag[j];
    const double yj = y[j];
    for (uint32_t t = s.cp[j]; t < s.cp[j + 1]; ++t) y[s.ri[t]] -= vals[t] * yj;
  }
  for (uint32_t j = n; j-- > 0;) {
    double v = y[j];
    for (uint32_t t = s.cp[j]; t < s.cp[j + 1]; ++t) v -= vals[t] * y[s.ri[t]];
    y[j] = v / diag[j];
  }
  for (uint32_t p = 0; p < n; ++p) x[s.order[p]] = y[p];
}
// bounce_qp (bounce_lcp.rs:249-315): x, and whether it converged within kSolves solves.
__device__ bool bounce_qp(const Csr& k0, const double* b, const double* acc0, Arena& ar, double* x_out, bool* ok) {
  const uint32_t n = k0.n;
  const unsigned long long nnz = k0.ptr[n];
  Csr k{n, k0.ptr, k0.idx, ar.take<double>(nnz)};
  double* v[20];
  for (int i = 0; i < 20; ++i) v[i] = ar.take<double>(n);
  Sym s;
  if (!ar.ok) { *ok = false; return false; }
  for (unsigned long long t = 0; t < nnz; ++t) k.val[t] = k0.val[t];
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t t = k.ptr[i]; t < k.ptr[i + 1]; ++t)
      if (k.idx[t] == i) k.val[t] *= 1.0 + kCfm;
  if (!min_degree(k, ar, &s)) { *ok = false; return false; }
  const uint32_t nri = s.cp[n];
  double* lvals = ar.take<double>(nri + 1ull);
  if (!ar.ok) { *ok = false; return false; }
  double *kdiag = v[0], *q = v[1], *y = v[2], *w = v[3], *r = v[4], *x = v[5], *wt = v[6], *d = v[7], *work = v[8],
         *ldiag = v[9], *rhs = v[10], *dya = v[11], *dwa = v[12], *dy = v[13], *dw = v[14], *tmp = v[15], *aff = v[16],
         *cor = v[17], *ysol = v[18];
  for (uint32_t i = 0; i < n; ++i) kdiag[i] = csr_diag(k0, i);
  csr_mul(k, acc0, tmp);
  for (uint32_t i = 0; i < n; ++i) q[i] = -tmp[i] - b[i];
  double qmax = 0.0;
  for (uint32_t i = 0; i < n; ++i) qmax = fmax(qmax, fabs(q[i]));
  const double eta = fmax(1.0, qmax);
  for (uint32_t i = 0; i < n; ++i) { y[i] = kdiag[i] > 0.0 ? eta / kdiag[i] : 1.0; w[i] = eta; }
  const double nn = (double)n;
  auto step = [&](const double* sdy, const double* sdw) {
    double a = 1.0;
    for (uint32_t i = 0; i < n; ++i) {
      if (sdy[i] < 0.0) a = fmin(a, -y[i] / sdy[i]);
      if (sdw[i] < 0.0) a = fmin(a, -w[i] / sdw[i]);
    }
    return a;
  };
  auto dirs = [&](const double* target, double* ody, double* odw) {
    for (uint32_t i = 0; i < n; ++i) rhs[i] = -r[i] + target[i] / y[i];
    fsolve(s, n, ldiag, lvals, rhs, ysol, ody);
    for (uint32_t i = 0; i < n; ++i) odw[i] = (target[i] - w[i] * ody[i]) / y[i];
  };
  for (uint32_t it = 1; it <= kSolves; ++it) {
    csr_mul(k, y, tmp);
    for (uint32_t i = 0; i < n; ++i) r[i] = (tmp[i] + q[i]) - w[i];
    double mu_sum = -0.0;
    for (uint32_t i = 0; i < n; ++i) mu_sum += y[i] * w[i];
    const double mu = mu_sum / nn;
    double rmx = 0.0;
    for (uint32_t i = 0; i < n; ++i) rmx = fmax(rmx, fabs(r[i]));
    for (uint32_t i = 0; i < n; ++i) x[i] = y[i] - acc0[i];
    csr_mul(k0, x, tmp);
    for (uint32_t i = 0; i < n; ++i) wt[i] = tmp[i] - b[i];
    if (rmx < 1e-7) {
      bool conv = true;
      for (uint32_t i = 0; i < n && conv; ++i) {
        double tol = 1e-7 * (1.0 + fabs(b[i]));
        conv = wt[i] >= -tol && fmin(fabs(wt[i]), y[i] * kdiag[i]) < tol;
      }
      if (conv) {
        for (uint32_t i = 0; i < n; ++i) x_out[i] = x[i];
        *ok = true;
        return true;
      }
    }
    for (uint32_t i = 0; i < n; ++i) d[i] = w[i] / y[i];
    factor(k, s, d, work, ldiag, lvals);
    for (uint32_t i = 0; i < n; ++i) aff[i] = -y[i] * w[i];
    dirs(aff, dya, dwa);
    const double aa = step(dya, dwa);
    double maff = -0.0;
    for (uint32_t i = 0; i < n; ++i) maff += (y[i] + aa * dya[i]) * (w[i] + aa * dwa[i]);
    const double mu_aff = maff / nn;
    const double ratio = mu_aff / fmax(mu, 1e-300);
    const double sigma = fmin(ratio * ratio * ratio, 1.0);
    for (uint32_t i = 0; i < n; ++i) cor[i] = (sigma * mu - y[i] * w[i]) - dya[i] * dwa[i];
    dirs(cor, dy, dw);
    const double a = fmin(0.995 * step(dy, dw), 1.0);
    bool finite = isfinite(a);
    for (uint32_t i = 0; i < n && finite; ++i) finite = isfinite(dy[i]) && isfinite(dw[i]);
    if (!finite) break;
    for (uint32_t i = 0; i < n; ++i) {
      y[i] = fmax(y[i] + a * dy[i], 1e-300);
      w[i] = fmax(w[i] + a * dw[i], 1e-300);
    }
  }
  for (uint32_t i = 0; i < n; ++i) x_out[i] = y[i] - acc0[i];
  *ok = true;
  return false;
}
// pseudo_solve (bounce_lcp.rs:317-324)
__device__ bool pseudo_solve(const Csr& k, const double* u, Arena& ar, double* x) {
  const uint32_t n = k.n;
  double* d = ar.take<double>(n);
  double* work = ar.take<double>(n);
  double* ldiag = ar.take<double>(n);
  double* ysol = ar.take<double>(n);
  Sym s;
  if (!ar.ok || !min_degree(k, ar, &s)) return false;
  double* lvals = ar.take<double>(s.cp[n] + 1ull);
  if (!ar.ok) return false;
  for (uint32_t i = 0; i < n; ++i) d[i] = kCfm * csr_diag(k, i);
  factor(k, s, d, work, ldiag, lvals);
  fsolve(s, n, ldiag, lvals, u, ysol, x);
  return true;
}

// ---- block-wide helpers (single-block kernels of 1024 threads)
constexpr int kBT = 1024;
// Appends, in index order, the entries e in [0, n) with pred(e) to out from out[base]; returns the count.
template <class Pred>
__device__ uint32_t block_compact(uint32_t n, uint32_t* out, uint32_t base, Pred pred) {
  __shared__ uint32_t warp_sum[kBT / 32];
  __shared__ uint32_t run;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) run = 0;
  __syncthreads();
  for (uint32_t c0 = 0; c0 < n; c0 += kBT) {
    const uint32_t e = c0 + tid;
    const bool f = e < n && pred(e);
    const uint32_t bal = __ballot_sync(0xffffffffu, f);
    const uint32_t below = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_sum[wid] = __popc(bal);
    __syncthreads();
    uint32_t off = 0;
    for (int q = 0; q < wid; ++q) off += warp_sum[q];
    if (f) out[base + run + off + below] = e;
    __syncthreads();
    if (tid == 0) { uint32_t t = 0; for (int q = 0; q < kBT / 32; ++q) t += warp_sum[q]; run += t; }
    __syncthreads();
  }
  return run;
}
// grow (solver.rs:1017-1029): involved spreads through rigid loaded contacts to a fixed point,
// stopping at static, sleeping and jointed bodies (the fixed point does not depend on the order).
__device__ void block_grow(uint32_t nc, const RowsV& R, const float* acc_jn, const float2* acc_jt, const uint8_t* jointed,
                           uint8_t* involved) {
  __shared__ int changed;
  for (;;) {
    if (threadIdx.x == 0) changed = 0;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < nc; c += kBT) {
      uint32_t f = R.flags[c];
      if ((f & RF_TERRAIN) || !loaded_at(acc_jn, acc_jt, c)) continue;
      uint2 ab = R.ab[c];
      float2 inv = R.inv[c];
      if (involved[ab.x] && !involved[ab.y] && inv.y > 0.0f && !(jointed && jointed[ab.y])) { involved[ab.y] = 1; changed = 1; }
      if (involved[ab.y] && !involved[ab.x] && inv.x > 0.0f && !(jointed && jointed[ab.x])) { involved[ab.x] = 1; changed = 1; }
    }
    __syncthreads();
    if (!changed) break;
    __syncthreads();
  }
}
// row_components (solver.rs:170-195), serially on one thread: components in order of their first
// row, rows ascending in each; writes comp_rows / comp_start and returns the count.
__device__ uint32_t components(const W6V& V, const RowsV& R, const BodiesV& B, const uint8_t* jointed, uint32_t nrows,
                               bool all_free) {
  auto sides_of = [&](uint32_t i, uint32_t* a, uint32_t* b) {
    const uint32_t e = V.rows[i];
    Row r = w6_row(R, B, jointed, e, all_free || (e & kSupport));
    *a = r.inv_a > 0.0f ? r.ai : kNone;
    *b = (!(r.flags & RF_TERRAIN) && r.inv_b > 0.0f) ? r.bi : kNone;
  };
  auto find = [&](uint32_t x) {
    while (V.parent[x] != x) { uint32_t g = V.parent[V.parent[x]]; V.parent[x] = g; x = g; }
    return x;
  };
  for (uint32_t i = 0; i < nrows; ++i) {
    uint32_t a, b;
    sides_of(i, &a, &b);
    if (a != kNone) { V.parent[a] = a; V.slot[a] = kNone; }
    if (b != kNone) { V.parent[b] = b; V.slot[b] = kNone; }
  }
  for (uint32_t i = 0; i < nrows; ++i) {
    uint32_t a, b;
    sides_of(i, &a, &b);
    if (a != kNone && b != kNone) {
      uint32_t x = find(a), y = find(b);
      if (x != y) V.parent[x > y ? x : y] = x < y ? x : y;
    }
  }
  uint32_t ncomp = 0;
  for (uint32_t i = 0; i < nrows; ++i) {
    uint32_t a, b;
    sides_of(i, &a, &b);
    const uint32_t body = a != kNone ? a : b;
    uint32_t c;
    if (body == kNone) {
      c = ncomp++;
      V.comp_start[c + 1] = 0;
    } else {
      const uint32_t r = find(body);
      if (V.slot[r] == kNone) { V.slot[r] = ncomp++; V.comp_start[V.slot[r] + 1] = 0; }
      c = V.slot[r];
    }
    V.row_comp[i] = c;
    V.comp_start[c + 1] += 1;
  }
  V.comp_start[0] = 0;
  for (uint32_t c = 0; c < ncomp; ++c) {
    V.comp_start[c + 1] += V.comp_start[c];
    V.cur[c] = V.comp_start[c];
  }
  for (uint32_t i = 0; i < nrows; ++i) V.comp_rows[V.cur[V.row_comp[i]]++] = i;
  return ncomp;
}

// ---- the pass's kernels (launched every tick with rows; each returns at once without a bounce)
__global__ void k_w6_count(uint32_t nc, RowsV R, const float* __restrict__ acc_jn, W6V V, uint32_t* stats) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc || !toi_set(R, acc_jn, c)) return;
  atomicAdd(V.ctr + C_TOI, 1u);
  atomicAdd(stats + STAT_BOUNCE, 1u);
}
// The velocity pass's rows (solver.rs:1049-1100): the bounces at their time-of-impact targets, then
// the push-only supports, and their components.
__global__ void __launch_bounds__(kBT) k_w6_setup(uint32_t nc, uint32_t nb, RowsV R, BodiesV B, const float* acc_jn,
                                                   const float2* acc_jt, const uint8_t* jointed, float dt, W6V V) {
  if (V.ctr[C_TOI] == 0) return;
  const int tid = threadIdx.x;
  for (uint32_t b = tid; b < nb; b += kBT) { V.rest_cnt[b] = 0; V.rest_min[b] = kNone; V.rest_max[b] = 0; V.involved[b] = 0; }
  __syncthreads();
  // loaded contacts outside the bounce, per body: with whom (partner kNone: the terrain)
  for (uint32_t c = tid; c < nc; c += kBT) {
    if (toi_set(R, acc_jn, c) || !loaded_at(acc_jn, acc_jt, c)) continue;
    const uint2 ab = R.ab[c];
    const bool terrain = (R.flags[c] & RF_TERRAIN) != 0;
    const uint32_t pa = terrain ? kNone : ab.y;
    atomicAdd(V.rest_cnt + ab.x, 1u); atomicMin(V.rest_min + ab.x, pa); atomicMax(V.rest_max + ab.x, pa);
    if (!terrain) { atomicAdd(V.rest_cnt + ab.y, 1u); atomicMin(V.rest_min + ab.y, ab.x); atomicMax(V.rest_max + ab.y, ab.x); }
  }
  __syncthreads();
  const uint32_t ntoi = block_compact(nc, V.rows, 0u, [&](uint32_t c) { return toi_set(R, acc_jn, c); });
  for (uint32_t r = tid; r < ntoi; r += kBT) {
    const uint32_t c = V.rows[r];
    const uint2 ab = R.ab[c];
    const bool terrain = (R.flags[c] & RF_TERRAIN) != 0;
    const float4 ta = V.toi_a[c];
    const float2 tb = V.toi_b[c];
    // a side resting on something other than its partner here is struck from its start velocity
    auto side = [&](uint32_t id, uint32_t other, float start, float after, float* s0, float* s1) {
      const bool rests = V.rest_cnt[id] > 0 && !(V.rest_min[id] == other && V.rest_max[id] == other);
      *s0 = start;
      *s1 = rests ? start : after;
    };
    float a0, a1, b0 = 0.0f, b1 = 0.0f;
    side(ab.x, terrain ? kNone : ab.y, ta.z, ta.w, &a0, &a1);
    if (!terrain) side(ab.y, ab.x, tb.x, tb.y, &b0, &b1);
    const float v0 = b0 - a0;
    const float acc = ((b1 - a1) - v0) / dt;
    float v_end, u;
    bool has;
    toi_bounce(ta.x, v0, acc, ta.y, dt, &v_end, &has, &u);
    V.target[r] = v_end;
    V.has_pseudo[r] = has ? 1 : 0;
    V.pseudo_u[r] = u;
    V.involved[ab.x] = 1;
    if (!terrain) V.involved[ab.y] = 1;
  }
  __syncthreads();
  block_grow(nc, R, acc_jn, acc_jt, jointed, V.involved);
  const uint32_t nsup = block_compact(nc, V.rows, ntoi, [&](uint32_t c) {
    if (toi_set(R, acc_jn, c) || acc_jn[c] <= 0.0f) return false;
    const uint2 ab = R.ab[c];
    const bool terrain = (R.flags[c] & RF_TERRAIN) != 0;
    if (!V.involved[ab.x] && (terrain || !V.involved[ab.y])) return false;
    Row r = ld_row(R, c);
    return free_only(B, jointed, r);
  });
  for (uint32_t k = tid; k < nsup; k += kBT) {
    const uint32_t c = V.rows[ntoi + k];
    V.rows[ntoi + k] = c | kSupport;
    V.target[ntoi + k] = rmin(R.t1[c].w, 0.0f);  // no approach beyond the gap (the depth bias, capped at 0)
    V.sup_acc[ntoi + k] = 0.0f;
  }
  __syncthreads();
  if (tid == 0) {
    V.ctr[C_NTOI] = ntoi;
    V.ctr[C_ROWS] = ntoi + nsup;
    V.ctr[C_COMPS] = components(V, R, B, jointed, ntoi + nsup, false);
  }
}
__device__ __forceinline__ float& w6_acc(const W6V& V, float* acc_jn, uint32_t i) {
  const uint32_t e = V.rows[i];
  return (e & kSupport) ? V.sup_acc[i] : acc_jn[e & ~kSupport];
}
// One component of the velocity pass (solver.rs:1104-1153): the direct LCP solve up to 250 rows,
// sweeps above it or when it did not converge.
__global__ void k_w6_solve(RowsV R, BodiesV B, float* acc_jn, const uint8_t* jointed, W6V V, uint32_t* stats) {
  if (V.ctr[C_TOI] == 0) return;
  const uint32_t ncomp = V.ctr[C_COMPS];
  for (uint32_t comp = blockIdx.x * blockDim.x + threadIdx.x; comp < ncomp; comp += gridDim.x * blockDim.x) {
    const uint32_t* cr = V.comp_rows + V.comp_start[comp];
    const uint32_t n = V.comp_start[comp + 1] - V.comp_start[comp];
    auto row_of = [&](uint32_t q) { return w6_row(R, B, jointed, V.rows[cr[q]], (V.rows[cr[q]] & kSupport) != 0); };
    bool sweep = n > kDirectMax;
    if (!sweep) {
      Arena ar;
      if (!arena_open(V, n, &ar)) { atomicOr(stats + STAT_ERR, kErrCapacity); sweep = true; }
      else {
        Side* sides = ar.take<Side>(2ull * n);
        double* b = ar.take<double>(n);
        double* acc0 = ar.take<double>(n);
        double* x = ar.take<double>(n);
        Csr k;
        bool ok = ar.ok;
        if (ok) {
          for (uint32_t q = 0; q < n; ++q) {
            Row r = row_of(q);
            row_sides(B, r, sides + 2 * q);
            b[q] = (double)(V.target[cr[q]] - dot(rel_vel(B, r), r.n));
            acc0[q] = (double)w6_acc(V, acc_jn, cr[q]);
          }
          ok = contact_csr(sides, n, ar, &k);
        }
        bool conv = false;
        if (ok) conv = bounce_qp(k, b, acc0, ar, x, &ok);
        if (!ok) { atomicOr(stats + STAT_ERR, kErrCapacity); sweep = true; }
        else {
          sweep = !conv;
          for (uint32_t q = 0; q < n; ++q) {
            Row r = row_of(q);
            float& a = w6_acc(V, acc_jn, cr[q]);
            const float old = a;
            const float nw = rmax((float)((double)old + x[q]), 0.0f);
            a = nw;
            contact_impulse(B, r, r.n * (nw - old));
          }
        }
      }
    }
    if (!sweep) continue;
    for (uint32_t it = 0; it < kSweeps; ++it) {
      float change = 0.0f;
      for (uint32_t m = 0; m < n; ++m) {
        const uint32_t q = it % 2 == 0 ? m : n - 1 - m;
        Row r = row_of(q);
        const float target = V.target[cr[q]];
        const float v = dot(rel_vel(B, r), r.n);
        float& a = w6_acc(V, acc_jn, cr[q]);
        const float old = a;
        const float nw = rmax(old + (target - v) * r.m_n, 0.0f);
        a = nw;
        contact_impulse(B, r, r.n * (nw - old));
        change = rmax(change, fabsf(nw - old) / r.m_n / (1.0f + fabsf(target)));
      }
      if (change < kTol) break;
    }
  }
}
// The pseudo pass's rows (solver.rs:1161-1184): the bounces that started apart, then the involved
// bodies' other loaded contacts with target 0, all with jointed sides immovable.
__global__ void __launch_bounds__(kBT) k_w6_pseudo_setup(uint32_t nc, uint32_t nb, RowsV R, BodiesV B,
                                                          const float* acc_jn, const float2* acc_jt,
                                                          const uint8_t* jointed, W6V V) {
  if (V.ctr[C_TOI] == 0) return;
  const int tid = threadIdx.x;
  const uint32_t ntoi = V.ctr[C_NTOI];
  __shared__ uint32_t npr_s, any_s;
  if (tid == 0) {
    uint32_t any = 0;
    for (uint32_t r = 0; r < ntoi; ++r) any |= V.has_pseudo[r];
    any_s = any;
  }
  __syncthreads();
  if (!any_s) return;
  for (uint32_t b = tid; b < nb; b += kBT) {
    V.involved[b] = 0;
    V.direct[b] = 0;
    V.pl[b] = make_float4(0, 0, 0, 0);
    V.pa[b] = make_float4(0, 0, 0, 0);
    for (int q = 0; q < 6; ++q) V.acc[6 * (size_t)b + q] = 0.0;
  }
  for (uint32_t c = tid; c < nc; c += kBT) V.in_set[c] = 0;
  __syncthreads();
  for (uint32_t r = tid; r < ntoi; r += kBT) {
    if (!V.has_pseudo[r]) continue;
    const uint32_t c = V.rows[r] & ~kSupport;
    const uint2 ab = R.ab[c];
    V.in_set[c] = 1;
    V.involved[ab.x] = 1;
    if (!(R.flags[c] & RF_TERRAIN)) V.involved[ab.y] = 1;
  }
  __syncthreads();
  if (tid == 0) {  // the pseudo rows that free_only keeps, in toi order, in place
    uint32_t k = 0;
    for (uint32_t r = 0; r < ntoi; ++r) {
      if (!V.has_pseudo[r]) continue;
      const uint32_t c = V.rows[r] & ~kSupport;
      Row row = ld_row(R, c);
      if (!free_only(B, jointed, row)) continue;
      const float u = V.pseudo_u[r];
      V.rows[k] = c;
      V.target[k] = u;
      ++k;
    }
    npr_s = k;
  }
  __syncthreads();
  const uint32_t npr = npr_s;
  block_grow(nc, R, acc_jn, acc_jt, jointed, V.involved);
  const uint32_t nsup = block_compact(nc, V.rows, npr, [&](uint32_t c) {
    if (V.in_set[c] || !loaded_at(acc_jn, acc_jt, c)) return false;
    const uint2 ab = R.ab[c];
    const bool terrain = (R.flags[c] & RF_TERRAIN) != 0;
    if (!V.involved[ab.x] && (terrain || !V.involved[ab.y])) return false;
    Row r = ld_row(R, c);
    return free_only(B, jointed, r);
  });
  for (uint32_t k = tid; k < nsup; k += kBT) V.target[npr + k] = 0.0f;
  __syncthreads();
  if (tid == 0) {
    V.ctr[C_PSEUDO] = npr;
    V.ctr[C_ROWS] = npr + nsup;
    V.ctr[C_COMPS] = components(V, R, B, jointed, npr + nsup, true);
    V.ctr[C_PON] = 1;
  }
}
// One component of the pseudo pass (solver.rs:1186-1234): the direct equality solve up to 250
// rows (its impulses summed per body in f64), else sweeps on the f32 pseudo-velocities.
__global__ void k_w6_pseudo_solve(RowsV R, BodiesV B, const uint8_t* jointed, W6V V, uint32_t* stats) {
  if (V.ctr[C_TOI] == 0 || V.ctr[C_PON] == 0) return;
  const uint32_t ncomp = V.ctr[C_COMPS];
  for (uint32_t comp = blockIdx.x * blockDim.x + threadIdx.x; comp < ncomp; comp += gridDim.x * blockDim.x) {
    const uint32_t* cr = V.comp_rows + V.comp_start[comp];
    const uint32_t n = V.comp_start[comp + 1] - V.comp_start[comp];
    auto row_of = [&](uint32_t q) { return w6_row(R, B, jointed, V.rows[cr[q]], true); };
    bool direct = n <= kDirectMax;
    if (direct) {
      Arena ar;
      bool ok = arena_open(V, n, &ar);
      Side* sides = ok ? ar.take<Side>(2ull * n) : nullptr;
      double* u = ok ? ar.take<double>(n) : nullptr;
      double* x = ok ? ar.take<double>(n) : nullptr;
      Csr k;
      ok = ok && ar.ok;
      if (ok) {
        for (uint32_t q = 0; q < n; ++q) {
          Row r = row_of(q);
          row_sides(B, r, sides + 2 * q);
          u[q] = (double)V.target[cr[q]];
        }
        ok = contact_csr(sides, n, ar, &k) && pseudo_solve(k, u, ar, x);
      }
      if (!ok) {
        atomicOr(stats + STAT_ERR, kErrCapacity);
        continue;
      }
      for (uint32_t q = 0; q < n; ++q)
        for (int t = 0; t < 2; ++t) {
          const Side& sd = sides[2 * q + t];
          if (sd.body == kNone) continue;
          double* e = V.acc + 6 * (size_t)sd.body;
          e[0] = e[0] + sd.mjl.x * x[q]; e[1] = e[1] + sd.mjl.y * x[q]; e[2] = e[2] + sd.mjl.z * x[q];
          e[3] = e[3] + sd.mja.x * x[q]; e[4] = e[4] + sd.mja.y * x[q]; e[5] = e[5] + sd.mja.z * x[q];
          V.direct[sd.body] = 1;
        }
      continue;
    }
    auto rel = [&](const Row& r) {
      const f3 la = xyz(V.pl[r.ai]), wa = xyz(V.pa[r.ai]);
      const bool terrain = (r.flags & RF_TERRAIN) != 0;
      const f3 lb = terrain ? mk3(0, 0, 0) : xyz(V.pl[r.bi]), wb = terrain ? mk3(0, 0, 0) : xyz(V.pa[r.bi]);
      return dot((lb + cross(wb, r.rb)) - (la + cross(wa, r.ra)), r.n);
    };
    for (uint32_t it = 0; it < kSweeps; ++it) {
      float change = 0.0f;
      for (uint32_t m = 0; m < n; ++m) {
        const uint32_t q = it % 2 == 0 ? m : n - 1 - m;
        Row r = row_of(q);
        const float u = V.target[cr[q]];
        const float d = u - rel(r);
        change = rmax(change, fabsf(d) / (1.0f + fabsf(u)));
        const f3 j = r.n * (d * r.m_n);
        if (r.inv_a > 0.0f) {
          V.pl[r.ai] = f4(xyz(V.pl[r.ai]) - j * r.inv_a);
          V.pa[r.ai] = f4(xyz(V.pa[r.ai]) - mvec(ld_m3(B.Iw, r.ai), cross(r.ra, j)));
        }
        if (r.inv_b > 0.0f) {
          V.pl[r.bi] = f4(xyz(V.pl[r.bi]) + j * r.inv_b);
          V.pa[r.bi] = f4(xyz(V.pa[r.bi]) + mvec(ld_m3(B.Iw, r.bi), cross(r.rb, j)));
        }
      }
      if (change < kTol) break;
    }
  }
}
// The directly solved bodies' pseudo-velocities, f64 sums rounded to f32 (solver.rs:1235-1237).
__global__ void k_w6_pseudo_finish(uint32_t nb, W6V V) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb || V.ctr[C_PON] == 0 || !V.direct[b]) return;
  const double* e = V.acc + 6 * (size_t)b;
  V.pl[b] = make_float4((float)e[0], (float)e[1], (float)e[2], 0.0f);
  V.pa[b] = make_float4((float)e[3], (float)e[4], (float)e[5], 0.0f);
}

}  // namespace w6

// factor.cpp — nested-dissection ordering, multifrontal supernodal Cholesky
// and the partitioned-inverse device layout.  See factor.hpp.
#include "factor.hpp"

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <stdexcept>
#include <cmath>
#include <cstdlib>
#include <numeric>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace pdfb {
namespace {

constexpr int kNdMergeLevels = 3;   // see NDBuilder
constexpr int kBlockedFront = 256;  // diagonal blocks this large use blocked_cholesky

inline double dotn(const double* a, const double* b, int n) {
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    s0 += a[k] * b[k];
    s1 += a[k + 1] * b[k + 1];
    s2 += a[k + 2] * b[k + 2];
    s3 += a[k + 3] * b[k + 3];
  }
  for (; k < n; ++k) s0 += a[k] * b[k];
  return (s0 + s1) + (s2 + s3);
}

// Nested dissection.  The separators of the top `merge` levels of the
// dissection tree are not given their own supernodes: they are deferred and
// ordered last, as one dense root supernode (top()), which removes merge - 1
// levels from the elimination tree the device sweeps walk level by level.
struct NDBuilder {
  const Model& m;
  int leaf;
  int merge;
  std::vector<int> order;           // pivot order being built
  std::vector<int> node_c0, node_n; // node columns
  std::vector<char> side;
  std::vector<int> deferred;        // separators of depth < merge, deepest first

  NDBuilder(const Model& mm, int lf, int mg) : m(mm), leaf(lf), merge(mg), side(mm.N, 0) { order.reserve(mm.N); }

  void top() {
    if (deferred.empty()) return;
    node_c0.push_back((int)order.size());
    node_n.push_back((int)deferred.size());
    order.insert(order.end(), deferred.begin(), deferred.end());
    deferred.clear();
  }

  void run(std::vector<int>& ids, int depth = 0) {
    if ((int)ids.size() <= leaf) {
      if (!ids.empty()) {
        node_c0.push_back((int)order.size());
        node_n.push_back((int)ids.size());
        order.insert(order.end(), ids.begin(), ids.end());
      }
      return;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v : ids)
      for (int c = 0; c < 3; ++c) {
        lo[c] = std::min(lo[c], m.rest[3 * (size_t)v + c]);
        hi[c] = std::max(hi[c], m.rest[3 * (size_t)v + c]);
      }
    int ax = 0;
    for (int c = 1; c < 3; ++c)
      if (hi[c] - lo[c] > hi[ax] - lo[ax]) ax = c;
    const size_t mid = ids.size() / 2;
    std::nth_element(ids.begin(), ids.begin() + mid, ids.end(), [&](int a, int b) {
      double ca = m.rest[3 * (size_t)a + ax], cb = m.rest[3 * (size_t)b + ax];
      return ca < cb || (ca == cb && a < b);
    });
    std::vector<int> s1(ids.begin(), ids.begin() + mid), s2(ids.begin() + mid, ids.end());
    ids.clear();
    ids.shrink_to_fit();
    for (int v : s1) side[v] = 1;
    std::vector<int> s2r, sep;
    for (int v : s2) {
      bool touch = false;
      for (int k = m.ata_ptr[v]; k < m.ata_ptr[v + 1] && !touch; ++k) touch = side[m.ata_col[k]] == 1;
      (touch ? sep : s2r).push_back(v);
    }
    for (int v : s1) side[v] = 0;
    s2.clear();
    s2.shrink_to_fit();
    run(s1, depth + 1);
    run(s2r, depth + 1);
    std::sort(sep.begin(), sep.end());
    if (depth < merge) {
      deferred.insert(deferred.end(), sep.begin(), sep.end());
    } else if (!sep.empty()) {
      node_c0.push_back((int)order.size());
      node_n.push_back((int)sep.size());
      order.insert(order.end(), sep.begin(), sep.end());
    }
  }
};

// Top dissection levels merged into the root supernode (PDF_ND_MERGE
// overrides it for tuning experiments).
int nd_merge_levels() {
  if (const char* e = std::getenv("PDF_ND_MERGE")) {
    const int v = std::atoi(e);
    if (v >= 0 && v <= 16) return v;
  }
  return kNdMergeLevels;
}

// In-place Cholesky of the leading ns x ns block of the row-major front F
// (leading dimension ld, lower triangle), blocked right-looking with the
// trailing updates spread over the host threads; used for large diagonal
// blocks (the merged root), where the row-by-row Crout is serial.
bool blocked_cholesky(double* F, int ns, int ld) {
  constexpr int B = 64;
  for (int kb = 0; kb < ns; kb += B) {
    const int ke = std::min(kb + B, ns);
    for (int k = kb; k < ke; ++k) {
      double* Fk = F + (size_t)k * ld;
      for (int jj = kb; jj < k; ++jj)
        Fk[jj] = (Fk[jj] - dotn(Fk + kb, F + (size_t)jj * ld + kb, jj - kb)) / F[(size_t)jj * ld + jj];
      const double d = Fk[k] - dotn(Fk + kb, Fk + kb, k - kb);
      if (!(d > 0.)) return false;
      Fk[k] = std::sqrt(d);
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = ke; i < ns; ++i) {
      double* Fi = F + (size_t)i * ld;
      for (int jj = kb; jj < ke; ++jj)
        Fi[jj] = (Fi[jj] - dotn(Fi + kb, F + (size_t)jj * ld + kb, jj - kb)) / F[(size_t)jj * ld + jj];
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = ke; i < ns; ++i) {
      double* Fi = F + (size_t)i * ld;
      for (int j = ke; j <= i; ++j) Fi[j] -= dotn(Fi + kb, F + (size_t)j * ld + kb, ke - kb);
    }
  }
  return true;
}

}  // namespace

bool factorize(const Model& m, double dt, int leaf_size, Factor& f, std::string& err) {
  auto t_start = std::chrono::steady_clock::now();
  const int N = m.N;
  f.N = N;
  // ---- ordering and supernode partition -------------------------------
  NDBuilder nd(m, std::max(8, leaf_size), nd_merge_levels());
  {
    std::vector<int> ids(N);
    std::iota(ids.begin(), ids.end(), 0);
    nd.run(ids);
    nd.top();
  }
  f.perm = nd.order;
  f.iperm.assign(N, 0);
  for (int k = 0; k < N; ++k) f.iperm[f.perm[k]] = k;
  const int S = (int)nd.node_c0.size();
  f.n_sn = S;
  f.sn_c0 = nd.node_c0;
  f.sn_ns = nd.node_n;
  std::vector<int> col_sn(N);
  for (int s = 0; s < S; ++s)
    for (int c = f.sn_c0[s]; c < f.sn_c0[s] + f.sn_ns[s]; ++c) col_sn[c] = s;
  // ---- symbolic: row sets, supernodal tree, levels ----------------------
  std::vector<std::vector<int>> R(S), children(S);
  f.sn_parent.assign(S, -1);
  f.sn_level.assign(S, 0);
  {
    std::vector<int> mark(N, -1);
    for (int s = 0; s < S; ++s) {
      const int c1 = f.sn_c0[s] + f.sn_ns[s];
      std::vector<int>& rs = R[s];
      for (int c = f.sn_c0[s]; c < c1; ++c) {
        const int v = f.perm[c];
        for (int k = m.ata_ptr[v]; k < m.ata_ptr[v + 1]; ++k) {
          int i = f.iperm[m.ata_col[k]];
          if (i >= c1 && mark[i] != s) {
            mark[i] = s;
            rs.push_back(i);
          }
        }
      }
      for (int t : children[s])
        for (int i : R[t])
          if (i >= c1 && mark[i] != s) {
            mark[i] = s;
            rs.push_back(i);
          }
      std::sort(rs.begin(), rs.end());
      int lvl = 0;
      for (int t : children[s]) lvl = std::max(lvl, f.sn_level[t] + 1);
      f.sn_level[s] = lvl;
      if (!rs.empty()) {
        int p = col_sn[rs[0]];
        f.sn_parent[s] = p;
        children[p].push_back(s);
      }
    }
  }
  f.n_levels = 0;
  for (int s = 0; s < S; ++s) f.n_levels = std::max(f.n_levels, f.sn_level[s] + 1);
  f.sn_nr.resize(S);
  f.sn_roff.assign(S + 1, 0);
  f.sn_woff.assign(S + 1, 0);
  for (int s = 0; s < S; ++s) {
    const int64_t ns = f.sn_ns[s], nr = (int64_t)R[s].size();
    f.sn_nr[s] = (int)nr;
    f.sn_roff[s + 1] = f.sn_roff[s] + nr;
    f.sn_woff[s + 1] = f.sn_woff[s] + ns * (ns + 1) / 2 + nr * ns;
  }
  f.nnz_w = f.sn_woff[S];
  f.rows.resize(f.sn_roff[S]);
  for (int s = 0; s < S; ++s) std::copy(R[s].begin(), R[s].end(), f.rows.begin() + f.sn_roff[s]);
  std::vector<double> Wr(f.nnz_w, 0.);  // packed row-major W_s (intermediate)

  // ---- numeric: multifrontal, level by level ---------------------------
  const double dt2 = std::pow(dt, 2);
  std::vector<std::vector<double>> U(S);
  std::vector<std::vector<int>> by_level(f.n_levels);
  for (int s = 0; s < S; ++s) by_level[f.sn_level[s]].push_back(s);
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  bool failed = false;
  int64_t nnz_true = 0;

  auto process = [&](int s, bool inner_parallel) {
    const int ns = f.sn_ns[s], nr = f.sn_nr[s], mdim = ns + nr;
    const int c0 = f.sn_c0[s];
    const int* rs = f.rows.data() + f.sn_roff[s];
    std::vector<double> F((size_t)mdim * mdim, 0.);
    auto loc = [&](int gi) -> int {
      if (gi < c0 + ns) return gi - c0;
      return ns + (int)(std::lower_bound(rs, rs + nr, gi) - rs);
    };
    // assemble M + dt^2 A^T A (lower triangle of the front)
    for (int jj = 0; jj < ns; ++jj) {
      const int v = f.perm[c0 + jj];
      for (int k = m.ata_ptr[v]; k < m.ata_ptr[v + 1]; ++k) {
        const int gi = f.iperm[m.ata_col[k]];
        if (gi < c0 + jj) continue;
        double a = dt2 * m.ata_val[k];
        if (gi == c0 + jj) a += m.mass[v];
        F[(size_t)loc(gi) * mdim + jj] += a;
      }
    }
    // extend-add the children's update matrices
    for (int t : children[s]) {
      const int nrt = f.sn_nr[t];
      const int* rt = f.rows.data() + f.sn_roff[t];
      std::vector<int> lt(nrt);
      for (int a = 0; a < nrt; ++a) lt[a] = loc(rt[a]);
      const std::vector<double>& Ut = U[t];
      for (int a = 0; a < nrt; ++a)
        for (int b = 0; b <= a; ++b) F[(size_t)lt[a] * mdim + lt[b]] += Ut[(size_t)a * nrt + b];
      std::vector<double>().swap(U[t]);
    }
    // Crout: L11 rows, then L21 rows (independent), then U = F22 - L21 L21^T
    if (ns >= kBlockedFront && inner_parallel) {
      if (!blocked_cholesky(F.data(), ns, mdim)) {
        failed = true;
        return;
      }
    } else {
      for (int k = 0; k < ns; ++k) {
        double* Fk = &F[(size_t)k * mdim];
        for (int jj = 0; jj < k; ++jj)
          Fk[jj] = (Fk[jj] - dotn(Fk, &F[(size_t)jj * mdim], jj)) / F[(size_t)jj * mdim + jj];
        double d = Fk[k] - dotn(Fk, Fk, k);
        if (!(d > 0.)) {
          failed = true;
          return;
        }
        Fk[k] = std::sqrt(d);
      }
    }
#pragma omp parallel for schedule(dynamic, 8) if (inner_parallel)
    for (int i = ns; i < mdim; ++i) {
      double* Fi = &F[(size_t)i * mdim];
      for (int jj = 0; jj < ns; ++jj) Fi[jj] = (Fi[jj] - dotn(Fi, &F[(size_t)jj * mdim], jj)) / F[(size_t)jj * mdim + jj];
    }
    if (nr > 0 && f.sn_parent[s] >= 0) {
      std::vector<double> Us((size_t)nr * nr, 0.);
#pragma omp parallel for schedule(dynamic, 8) if (inner_parallel)
      for (int a = 0; a < nr; ++a) {
        const double* Fa = &F[(size_t)(ns + a) * mdim];
        for (int b = 0; b <= a; ++b) Us[(size_t)a * nr + b] = Fa[ns + b] - dotn(Fa, &F[(size_t)(ns + b) * mdim], ns);
      }
      U[s].swap(Us);
    }
    // X = L11^-1 (column-major, lower), P = L21 X
    std::vector<double> X((size_t)ns * ns, 0.);
#pragma omp parallel for schedule(dynamic, 4) if (inner_parallel)
    for (int c = 0; c < ns; ++c) {
      double* Xc = &X[(size_t)c * ns];
      Xc[c] = 1.0 / F[(size_t)c * mdim + c];
      for (int i = c + 1; i < ns; ++i) {
        const double* Fi = &F[(size_t)i * mdim];
        Xc[i] = -dotn(Fi + c, Xc + c, i - c) / Fi[i];
      }
    }
    const int64_t wo = f.sn_woff[s];
    // row-major copy: rows i < ns hold X[i][0..i]; rows ns+r hold P[r][0..ns)
#pragma omp parallel for schedule(dynamic, 8) if (inner_parallel)
    for (int i = 0; i < mdim; ++i) {
      double* wr = &Wr[wo + w_rowstart(i, ns)];
      if (i < ns) {
        for (int j = 0; j <= i; ++j) wr[j] = X[(size_t)j * ns + i];
      } else {
        const double* Fi = &F[(size_t)i * mdim];
        for (int j = 0; j < ns; ++j) wr[j] = dotn(Fi + j, &X[(size_t)j * ns + j], ns - j);
      }
    }
  };

  for (int L = 0; L < f.n_levels && !failed; ++L) {
    const auto& lst = by_level[L];
    if ((int)lst.size() >= 2 * nthreads) {
#pragma omp parallel for schedule(dynamic, 1)
      for (size_t k = 0; k < lst.size(); ++k) process(lst[k], false);
    } else {
      for (int s : lst) {
        process(s, true);
        if (failed) break;
      }
    }
  }
  if (failed) {
    err = "global-step matrix M + dt^2 A^T A is not positive definite";
    return false;
  }
  // ---- tiled copies for the device sweeps (layout in factor.hpp) --------
  f.sn_btile0.assign(S + 1, 0);
  for (int s = 0; s < S; ++s) f.sn_btile0[s + 1] = f.sn_btile0[s] + (f.sn_ns[s] + kTile - 1) / kTile;
  {
    // forward tiles cover rows of W_s (ns + nr rows): more tiles than the
    // backward ones (ns columns); give every supernode both counts
    std::vector<int64_t> ft0(S + 1, 0);
    for (int s = 0; s < S; ++s) ft0[s + 1] = ft0[s] + (f.sn_ns[s] + f.sn_nr[s] + kTile - 1) / kTile;
    const int64_t nft = ft0[S], nbt = f.sn_btile0[S];
    f.ftile_off.assign(nft + 1, 0);
    f.btile_off.assign(nbt + 1, 0);
    for (int s = 0; s < S; ++s) {
      const int64_t ns = f.sn_ns[s], nr = f.sn_nr[s];
      for (int64_t t = 0; t < ft0[s + 1] - ft0[s]; ++t) {
        const int64_t w = std::min(ns, kTile * t + kTile);
        const int64_t m = std::min<int64_t>(kTile, ns + nr - kTile * t);
        f.ftile_off[ft0[s] + t + 1] = f.ftile_off[ft0[s] + t] + pad_tile(m * w);
      }
      for (int64_t t = 0; t < f.sn_btile0[s + 1] - f.sn_btile0[s]; ++t) {
        const int64_t hgt = ns - kTile * t + nr;
        const int64_t mc = std::min<int64_t>(kTile, ns - kTile * t);
        f.btile_off[f.sn_btile0[s] + t + 1] = f.btile_off[f.sn_btile0[s] + t] + pad_tile(mc * hgt);
      }
    }
    f.sn_ftile0 = ft0;
    f.Wf.assign(f.ftile_off[nft] + kTilePad, 0.);
    f.Wb.assign(f.btile_off[nbt] + kTilePad, 0.);
    f.tiled_w = std::max(f.ftile_off[nft], f.btile_off[nbt]);
#pragma omp parallel for schedule(dynamic, 4)
    for (int s = 0; s < S; ++s) {
      const int64_t ns = f.sn_ns[s], nr = f.sn_nr[s], wo = f.sn_woff[s];
      auto wval = [&](int64_t i, int64_t j) -> double {  // W_s(i, j), zero above D^-1's diagonal
        if (i < ns) return j <= i ? Wr[wo + w_rowstart(i, ns) + j] : 0.;
        if (i < ns + nr) return Wr[wo + w_rowstart(i, ns) + j];
        return 0.;
      };
      for (int64_t t = 0; t < ft0[s + 1] - ft0[s]; ++t) {
        double* T = &f.Wf[f.ftile_off[ft0[s] + t]];
        const int64_t w = std::min(ns, kTile * t + kTile);
        const int64_t m = std::min<int64_t>(kTile, ns + nr - kTile * t);
        for (int64_t j = 0; j < w; ++j)
          for (int64_t l = 0; l < m; ++l) T[m * j + l] = wval(kTile * t + l, j);
      }
      for (int64_t t = 0; t < f.sn_btile0[s + 1] - f.sn_btile0[s]; ++t) {
        double* T = &f.Wb[f.btile_off[f.sn_btile0[s] + t]];
        const int64_t j0 = kTile * t, hgt = ns - j0 + nr;
        for (int64_t i = 0; i < hgt; ++i) {
          const int64_t row = i < ns - j0 ? j0 + i : ns + (i - (ns - j0));
          const int64_t mc = std::min<int64_t>(kTile, ns - j0);
          for (int64_t l = 0; l < mc; ++l) T[mc * i + l] = wval(row, j0 + l);
        }
      }
    }
  }
  // structural nnz(L): sum over rows k of |reach of A(0:k, k) in the
  // elimination tree| plus the diagonal (row-subtree counting)
  {
    std::vector<int> parent(N, -1), anc(N, -1), mark(N, -1);
    for (int k = 0; k < N; ++k) {
      const int v = f.perm[k];
      for (int p = m.ata_ptr[v]; p < m.ata_ptr[v + 1]; ++p) {
        int i = f.iperm[m.ata_col[p]];
        while (i != -1 && i < k) {
          const int nx = anc[i];
          anc[i] = k;
          if (nx == -1) parent[i] = k;
          i = nx;
        }
      }
    }
    for (int k = 0; k < N; ++k) {
      mark[k] = k;
      const int v = f.perm[k];
      for (int p = m.ata_ptr[v]; p < m.ata_ptr[v + 1]; ++p) {
        int i = f.iperm[m.ata_col[p]];
        if (i >= k) continue;
        while (mark[i] != k) {
          mark[i] = k;
          ++nnz_true;
          i = parent[i];
        }
      }
    }
    nnz_true += N;
  }
  f.nnz_l_true = nnz_true;
  f.factor_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  return true;
}

void build_sweep_tasks(const Factor& f, int chunk, std::vector<SweepTask>& fa, std::vector<SweepTask>& ba,
                       std::vector<SnInfo>& sn) {
  std::vector<std::vector<int>> by_level(f.n_levels);
  for (int s = 0; s < f.n_sn; ++s) by_level[f.sn_level[s]].push_back(s);
  sn.assign(f.n_sn, SnInfo{});
  for (int s = 0; s < f.n_sn; ++s) {
    sn[s].c0 = f.sn_c0[s];
    sn[s].ns = f.sn_ns[s];
    sn[s].nr = f.sn_nr[s];
    sn[s].parent = f.sn_parent[s];
    sn[s].roff = f.sn_roff[s];
  }
  for (int s = 0; s < f.n_sn; ++s)
    if (f.sn_parent[s] >= 0) sn[f.sn_parent[s]].nchild++;
  fa.clear();
  ba.clear();
  for (int L = 0; L < f.n_levels; ++L)
    for (int s : by_level[L]) {
      const int ns = f.sn_ns[s];
      for (int64_t t = f.sn_ftile0[s]; t < f.sn_ftile0[s + 1]; ++t) {
        const int tl = (int)(t - f.sn_ftile0[s]);
        const int w = std::min(ns, kTile * tl + kTile);
        for (int a = 0; a < w; a += chunk) fa.push_back({s, tl, a, std::min(w, a + chunk), f.ftile_off[t]});
      }
    }
  for (int L = f.n_levels - 1; L >= 0; --L)
    for (int s : by_level[L]) {
      const int ns = f.sn_ns[s], nr = f.sn_nr[s];
      for (int64_t t = f.sn_btile0[s]; t < f.sn_btile0[s + 1]; ++t) {
        const int tl = (int)(t - f.sn_btile0[s]);
        const int hgt = ns - kTile * tl + nr;
        for (int a = 0; a < hgt; a += chunk) ba.push_back({s, tl, a, std::min(hgt, a + chunk), f.btile_off[t]});
      }
    }
  for (const auto& t : fa) sn[t.sn].ntf++;
  for (const auto& t : ba) sn[t.sn].ntb++;
}

static BlockItem block_item(int64_t off, int roff, int idx0, int c0l, int ns, int nr, int tile, int a0, int a1) {
  // the eligibility bounds of a block keep these within 16 bits
  if (c0l < 0 || c0l > INT16_MAX || ns > INT16_MAX || nr > INT16_MAX || tile > INT16_MAX || a1 > INT16_MAX)
    throw std::runtime_error("block work item field out of range");
  BlockItem I{};
  I.off = off;
  I.roff = roff;
  I.idx0 = idx0;
  I.c0l = (int16_t)c0l;
  I.ns = (int16_t)ns;
  I.nr = (int16_t)nr;
  I.tile = (int16_t)tile;
  I.a0 = (int16_t)a0;
  I.a1 = (int16_t)a1;
  return I;
}

void build_sweep_plan(const Factor& f, int chunk, int cut_level, SweepPlan& plan) {
  const int S = f.n_sn;
  plan = SweepPlan{};
  plan.cut_level = cut_level;
  plan.chunk = chunk;
  // subtree extents: supernodes are numbered in column order and every
  // parent comes after its children, so one ascending pass accumulates them
  std::vector<int> lo(S), cnt(S, 0), ftiles(S, 0), btiles(S, 0);
  auto spans = [](int len, int span) { return (len + span - 1) / span; };
  for (int s = 0; s < S; ++s) lo[s] = f.sn_c0[s];
  for (int s = 0; s < S; ++s) {
    cnt[s] += f.sn_ns[s];
    // block work items of the supernode (tiles split into spans)
    for (int tl = 0; tl < (int)(f.sn_ftile0[s + 1] - f.sn_ftile0[s]); ++tl)
      ftiles[s] += spans(std::min(f.sn_ns[s], kTile * tl + kTile), kBlockSpanF);
    for (int tl = 0; tl < (int)(f.sn_btile0[s + 1] - f.sn_btile0[s]); ++tl)
      btiles[s] += spans(f.sn_ns[s] - kTile * tl + f.sn_nr[s], kBlockSpanB);
    const int p = f.sn_parent[s];
    if (p >= 0) {
      lo[p] = std::min(lo[p], lo[s]);
      cnt[p] += cnt[s];
      ftiles[p] += ftiles[s];
      btiles[p] += btiles[s];
    }
  }
  auto eligible = [&](int s) {
    return f.sn_level[s] <= cut_level && f.sn_level[s] < kMaxBlockLevels && cnt[s] <= kMaxBlockCols &&
           f.sn_nr[s] <= kMaxBlockExt && ftiles[s] <= kMaxBlockItems && btiles[s] <= kMaxBlockItems &&
           f.sn_c0[s] + f.sn_ns[s] - lo[s] == cnt[s];
  };
  std::vector<int> blk(S, -1);
  std::vector<int> roots;
  // descending: a root's block id is set before its descendants are visited
  for (int s = S - 1; s >= 0; --s) {
    const int p = f.sn_parent[s];
    if (p >= 0 && blk[p] >= 0) {
      blk[s] = blk[p];
    } else if (eligible(s)) {
      blk[s] = (int)roots.size();
      roots.push_back(s);
    }
  }
  const int nb = (int)roots.size();
  plan.rows_loc.assign(f.rows.size(), -1);
  std::vector<std::vector<int>> members(nb);
  for (int s = 0; s < S; ++s)
    if (blk[s] >= 0) members[blk[s]].push_back(s);
  // stored elements of a supernode's tiles (either copy has the same count)
  auto sn_elems = [&](int s) {
    return f.ftile_off[f.sn_ftile0[s + 1]] - f.ftile_off[f.sn_ftile0[s]];
  };
  // largest blocks first (their CTAs start early, the small ones fill in)
  std::vector<int64_t> cost(nb, 0);
  for (int b = 0; b < nb; ++b)
    for (int s : members[b]) cost[b] += sn_elems(s);
  std::vector<int> order(nb);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  for (int b : order) {
    const int r = roots[b];
    SweepBlock fb{}, bb{};
    fb.c0 = bb.c0 = lo[r];
    fb.c1 = bb.c1 = f.sn_c0[r] + f.sn_ns[r];
    fb.parent = bb.parent = f.sn_parent[r];
    fb.nlev = bb.nlev = f.sn_level[r] + 1;
    fb.ext0 = bb.ext0 = (int)f.sn_roff[r];
    fb.next = bb.next = f.sn_nr[r];
    plan.max_block_cols = std::max(plan.max_block_cols, fb.c1 - fb.c0);
    plan.max_block_ext = std::max(plan.max_block_ext, fb.next);
    // where each row of each member lives in the block's shared vector
    const int nc = fb.c1 - fb.c0;
    const int* rr = f.rows.data() + f.sn_roff[r];
    for (int s : members[b])
      for (int k = 0; k < f.sn_nr[s]; ++k) {
        const int row = f.rows[f.sn_roff[s] + k];
        plan.rows_loc[f.sn_roff[s] + k] =
            row < fb.c1 ? row - fb.c0 : nc + (int)(std::lower_bound(rr, rr + fb.next, row) - rr);
      }
    plan.block_elems += cost[b];
    std::vector<std::vector<int>> by_lev(fb.nlev);
    for (int s : members[b]) by_lev[f.sn_level[s]].push_back(s);
    fb.item0 = (int)plan.fitem.size();
    for (int L = 0; L < fb.nlev; ++L) {
      fb.lev[L] = (int)plan.fitem.size() - fb.item0;
      for (int s : by_lev[L])
        for (int64_t t = f.sn_ftile0[s]; t < f.sn_ftile0[s + 1]; ++t) {
          const int tl = (int)(t - f.sn_ftile0[s]);
          const int w = std::min(f.sn_ns[s], kTile * tl + kTile);
          for (int a = 0; a < w; a += kBlockSpanF)
            plan.fitem.push_back(block_item(f.ftile_off[t], (int)f.sn_roff[s], 0, f.sn_c0[s] - fb.c0, f.sn_ns[s],
                                            f.sn_nr[s], tl, a, std::min(w, a + kBlockSpanF)));
        }
    }
    fb.lev[fb.nlev] = (int)plan.fitem.size() - fb.item0;
    bb.item0 = (int)plan.bitem.size();
    for (int k = 0; k < bb.nlev; ++k) {
      const int L = bb.nlev - 1 - k;
      bb.lev[k] = (int)plan.bitem.size() - bb.item0;
      for (int s : by_lev[L])
        for (int64_t t = f.sn_btile0[s]; t < f.sn_btile0[s + 1]; ++t) {
          const int tl = (int)(t - f.sn_btile0[s]);
          const int c0l = f.sn_c0[s] - bb.c0, j0t = kTile * tl, nd = f.sn_ns[s] - j0t, h = nd + f.sn_nr[s];
          for (int a = 0; a < h; a += kBlockSpanB)
            plan.bitem.push_back(block_item(f.btile_off[t], (int)f.sn_roff[s], (int)plan.bidx.size(), c0l,
                                            f.sn_ns[s], f.sn_nr[s], tl, a, std::min(h, a + kBlockSpanB)));
          for (int i = 0; i < h; ++i)
            plan.bidx.push_back(i < nd ? -1 - (c0l + j0t + i) : plan.rows_loc[f.sn_roff[s] + i - nd]);
          while (plan.bidx.size() % kSlabMax) plan.bidx.push_back(0);
        }
    }
    bb.lev[bb.nlev] = (int)plan.bitem.size() - bb.item0;
    plan.max_block_items = std::max(plan.max_block_items, std::max(fb.lev[fb.nlev], bb.lev[bb.nlev]));
    plan.fblk.push_back(fb);
    plan.bblk.push_back(bb);
  }
  // upper supernodes: the per-warp work items and their dependency records
  std::vector<SweepTask> fa, ba;
  build_sweep_tasks(f, chunk, fa, ba, plan.sn);
  for (const SweepTask& t : fa)
    if (blk[t.sn] < 0) plan.fup.push_back(t);
  for (const SweepTask& t : ba)
    if (blk[t.sn] < 0) plan.bup.push_back(t);
  for (int s = 0; s < S; ++s) {
    plan.sn[s].ntf = plan.sn[s].ntb = 0;
    if (blk[s] >= 0) continue;
    plan.upper_elems += sn_elems(s);
    for (int c = f.sn_c0[s]; c < f.sn_c0[s] + f.sn_ns[s]; ++c) plan.upper_cols.push_back(c);
  }
  for (const SweepTask& t : plan.fup) plan.sn[t.sn].ntf++;
  for (const SweepTask& t : plan.bup) plan.sn[t.sn].ntb++;
  // the blocks finish in an earlier launch than the upper items: an upper
  // supernode waits only for its upper children
  std::vector<int> upper_children(S, 0), child0(S, 0);
  std::vector<std::vector<int>> kids(S);
  for (int s = 0; s < S; ++s)
    if (blk[s] < 0 && f.sn_parent[s] >= 0) {
      upper_children[f.sn_parent[s]]++;
      kids[f.sn_parent[s]].push_back(s);
    }
  for (int s = 0; s < S; ++s) {
    child0[s] = (int)plan.child.size() / 2;
    for (int c : kids[s]) {
      plan.child.push_back(c);
      plan.child.push_back(plan.sn[c].ntf);
    }
  }
  auto upper = [&](const SweepTask& t, bool fwd) {
    const SnInfo& q = plan.sn[t.sn];
    UpperItem u{};
    u.off = t.off;
    u.sn = t.sn;
    u.tile = t.tile;
    u.a0 = t.a0;
    u.a1 = t.a1;
    u.c0 = q.c0;
    u.ns = q.ns;
    u.nr = q.nr;
    u.roff = (int)q.roff;
    u.parent = q.parent;
    u.wait = fwd ? upper_children[t.sn] : (q.parent >= 0 ? plan.sn[q.parent].ntb : 0);
    u.ntf = q.ntf;
    u.child0 = fwd ? child0[t.sn] : 0;
    return u;
  };
  for (const SweepTask& t : plan.fup) plan.fupi.push_back(upper(t, true));
  for (const SweepTask& t : plan.bup) plan.bupi.push_back(upper(t, false));
  // level boundaries (the items are in level order: ascending forward,
  // descending backward)
  auto bounds = [&](const std::vector<SweepTask>& v, std::vector<int>& lev) {
    lev.assign(1, 0);
    for (size_t k = 1; k <= v.size(); ++k)
      if (k == v.size() || f.sn_level[v[k].sn] != f.sn_level[v[k - 1].sn]) lev.push_back((int)k);
  };
  bounds(plan.fup, plan.fup_lev);
  bounds(plan.bup, plan.bup_lev);
}

bool emulate_sweeps(const Factor& f, const SweepPlan& plan, const std::vector<double>& bin,
                    std::vector<double>& xout, std::string& err) {
  const int64_t n = f.N;
  std::vector<double> b(3 * n), y(3 * n, 0.), x(3 * n, 0.);
  for (int64_t k = 0; k < n; ++k)
    for (int c = 0; c < 3; ++c) b[k + c * n] = bin[3 * (size_t)f.perm[k] + c];
  auto chk = [&](int64_t i, int64_t lim, const char* what) {
    if (i < 0 || i >= lim) {
      err = std::string("index out of range in ") + what;
      return false;
    }
    return true;
  };
  const int64_t nWf = (int64_t)f.Wf.size(), nWb = (int64_t)f.Wb.size(), nrows = (int64_t)f.rows.size();
  const int64_t nfi = (int64_t)plan.fitem.size(), nbi = (int64_t)plan.bitem.size();
  // forward, blocks: the block's slice of b and its ext rows in "shared memory"
  const int64_t nloc = (int64_t)plan.rows_loc.size();
  for (const SweepBlock& B : plan.fblk) {
    const int nc = B.c1 - B.c0, ld = nc + B.next;
    if (nc <= 0 || nc > plan.max_block_cols || B.next > plan.max_block_ext || B.nlev > kMaxBlockLevels ||
        B.lev[B.nlev] > plan.max_block_items) {
      err = "bad block extent";
      return false;
    }
    if (!chk(B.c0, n, "block columns") || !chk(B.c1 - 1, n, "block columns")) return false;
    std::vector<double> sv(3 * (size_t)ld, 0.);
    for (int k = 0; k < nc; ++k)
      for (int c = 0; c < 3; ++c) sv[k + c * ld] = b[B.c0 + k + c * n];
    for (int L = 0; L < B.nlev; ++L)
      for (int it = B.item0 + B.lev[L]; it < B.item0 + B.lev[L + 1]; ++it) {
        if (!chk(it, nfi, "forward block items")) return false;
        const BlockItem& I = plan.fitem[it];
        const int m = std::min(kTile, I.ns + I.nr - kTile * I.tile), w = std::min((int)I.ns, kTile * I.tile + (int)kTile);
        if ((I.off % kTilePad) != 0 || I.a0 % kSlabMax != 0 || I.a0 < 0 || I.a0 >= I.a1 || I.a1 > w) {
          err = "forward block item not aligned or out of its tile";
          return false;
        }
        for (int l = 0; l < m; ++l) {
          double acc[3] = {0, 0, 0};
          for (int j = I.a0; j < I.a1; ++j) {
            const int64_t wi = I.off + (int64_t)j * m + l;
            if (!chk(wi, nWf, "forward block tile") || !chk(I.c0l + j, nc, "forward block vector")) return false;
            for (int c = 0; c < 3; ++c) acc[c] += f.Wf[wi] * sv[I.c0l + j + c * ld];
          }
          const int row = kTile * I.tile + l;
          if (row < I.ns) {
            if (!chk(I.c0l + row, nc, "forward block y")) return false;
            for (int c = 0; c < 3; ++c) y[B.c0 + I.c0l + row + c * n] += acc[c];
          } else {
            if (!chk(I.roff + row - I.ns, nloc, "forward block rows")) return false;
            const int loc = plan.rows_loc[I.roff + row - I.ns];
            if (!chk(loc, ld, "forward block shared scatter")) return false;
            for (int c = 0; c < 3; ++c) sv[loc + c * ld] -= acc[c];
          }
        }
      }
    // the ext rows' accumulated updates go to b once
    for (int e = 0; e < B.next; ++e) {
      if (!chk(B.ext0 + e, nrows, "forward block ext rows")) return false;
      const int64_t r = f.rows[B.ext0 + e];
      if (!chk(r, n, "forward block ext scatter") || r < B.c1) {
        if (err.empty()) err = "ext row inside its block";
        return false;
      }
      for (int c = 0; c < 3; ++c) b[r + c * n] += sv[nc + e + c * ld];
    }
  }
  // the level launches: the items of one supernode share a level, and a
  // supernode's level comes after its children's forward and before them
  // backward (no item reads what another item of its own launch writes)
  {
    auto groups = [&](const std::vector<UpperItem>& v, const std::vector<int>& lev, std::vector<int>& grp) {
      grp.assign(f.n_sn, -1);
      if (lev.empty() || lev.front() != 0 || lev.back() != (int)v.size()) return false;
      for (size_t g = 0; g + 1 < lev.size(); ++g) {
        if (lev[g] >= lev[g + 1]) return false;
        for (int t = lev[g]; t < lev[g + 1]; ++t) {
          const int sn = v[t].sn;
          if (sn < 0 || sn >= f.n_sn || (grp[sn] >= 0 && grp[sn] != (int)g)) return false;
          grp[sn] = (int)g;
        }
      }
      return true;
    };
    std::vector<int> gf, gb;
    if (!groups(plan.fupi, plan.fup_lev, gf) || !groups(plan.bupi, plan.bup_lev, gb)) {
      err = "upper level boundaries do not partition the work items";
      return false;
    }
    for (int s = 0; s < f.n_sn; ++s) {
      const int p = f.sn_parent[s];
      if (gf[s] < 0 || p < 0 || gf[p] < 0) continue;
      if (!(gf[p] > gf[s]) || !(gb[p] < gb[s])) {
        err = "an upper supernode shares a level launch with its parent";
        return false;
      }
    }
  }
  // forward, upper work items (the records the device reads)
  const int64_t nchild = (int64_t)plan.child.size() / 2;
  for (const UpperItem& tk : plan.fupi) {
    const UpperItem& s = tk;
    for (int c = 0; c < tk.wait; ++c) {
      if (!chk(tk.child0 + c, nchild, "forward child list")) return false;
      if (!chk(plan.child[2 * (tk.child0 + c)], f.n_sn, "forward child supernode")) return false;
    }
    const int mrows = std::min(kTile, s.ns + s.nr - tk.tile * kTile);
    for (int l = 0; l < mrows; ++l) {
      const int row = tk.tile * kTile + l;
      double acc[3] = {0, 0, 0};
      for (int j = tk.a0; j < tk.a1; ++j) {
        const int64_t wi = tk.off + (int64_t)j * mrows + l;
        if (!chk(wi, nWf, "forward tile") || !chk(s.c0 + j, n, "forward vector")) return false;
        for (int c = 0; c < 3; ++c) acc[c] += f.Wf[wi] * b[s.c0 + j + c * n];
      }
      if (row < s.ns) {
        for (int c = 0; c < 3; ++c) y[s.c0 + row + c * n] += acc[c];
      } else if (row < s.ns + s.nr) {
        if (!chk(s.roff + row - s.ns, nrows, "forward rows")) return false;
        const int64_t r = f.rows[s.roff + row - s.ns];
        if (!chk(r, n, "forward scatter")) return false;
        for (int c = 0; c < 3; ++c) b[r + c * n] -= acc[c];
      }
    }
  }
  // backward, upper work items
  for (const UpperItem& tk : plan.bupi) {
    const UpperItem& s = tk;
    const int j0t = tk.tile * kTile, nd = s.ns - j0t;
    const int mc = std::min(kTile, nd);
    for (int l = 0; l < mc; ++l) {
      const int col = j0t + l;
      double acc[3] = {0, 0, 0};
      for (int i = tk.a0; i < tk.a1; ++i) {
        const int64_t wi = tk.off + (int64_t)i * mc + l;
        if (!chk(wi, nWb, "backward tile")) return false;
        double v[3];
        if (i < nd) {
          if (!chk(s.c0 + j0t + i, n, "backward y")) return false;
          for (int c = 0; c < 3; ++c) v[c] = y[s.c0 + j0t + i + c * n];
        } else {
          if (!chk(s.roff + i - nd, nrows, "backward rows")) return false;
          const int64_t r = f.rows[s.roff + i - nd];
          if (!chk(r, n, "backward gather")) return false;
          for (int c = 0; c < 3; ++c) v[c] = -x[r + c * n];
        }
        for (int c = 0; c < 3; ++c) acc[c] += f.Wb[wi] * v[c];
      }
      if (col < s.ns)
        for (int c = 0; c < 3; ++c) x[s.c0 + col + c * n] += acc[c];
    }
  }
  // backward, blocks: x of the block's columns and ext rows, and y of its
  // columns, in "shared memory"
  const int64_t nbidx = (int64_t)plan.bidx.size();
  for (const SweepBlock& B : plan.bblk) {
    const int nc = B.c1 - B.c0, ld = nc + B.next;
    std::vector<double> sx(3 * (size_t)ld, 0.), ys(3 * (size_t)nc, 0.);
    for (int e = 0; e < B.next; ++e) {
      if (!chk(B.ext0 + e, nrows, "backward block ext rows")) return false;
      const int64_t r = f.rows[B.ext0 + e];
      if (!chk(r, n, "backward block ext gather")) return false;
      for (int c = 0; c < 3; ++c) sx[nc + e + c * ld] = x[r + c * n];
    }
    for (int k = 0; k < nc; ++k)
      for (int c = 0; c < 3; ++c) ys[k + c * nc] = y[B.c0 + k + c * n];
    for (int L = 0; L < B.nlev; ++L)
      for (int it = B.item0 + B.lev[L]; it < B.item0 + B.lev[L + 1]; ++it) {
        if (!chk(it, nbi, "backward block items")) return false;
        const BlockItem& I = plan.bitem[it];
        const int j0t = kTile * I.tile, nd = I.ns - j0t, mc = std::min(kTile, nd), h = nd + I.nr;
        if ((I.off % kTilePad) != 0 || (I.idx0 % kSlabMax) != 0 || I.a0 % kSlabMax != 0 || I.a0 < 0 || I.a0 >= I.a1 ||
            I.a1 > h) {
          err = "backward block item not aligned or out of its tile";
          return false;
        }
        for (int l = 0; l < mc; ++l) {
          double acc[3] = {0, 0, 0};
          for (int i = I.a0; i < I.a1; ++i) {
            const int64_t wi = I.off + (int64_t)i * mc + l;
            if (!chk(wi, nWb, "backward block tile") || !chk(I.idx0 + i, nbidx, "backward block index")) return false;
            const int idx = plan.bidx[I.idx0 + i];
            double v[3];
            if (idx < 0) {
              if (!chk(-1 - idx, nc, "backward block y")) return false;
              for (int c = 0; c < 3; ++c) v[c] = ys[-1 - idx + c * nc];
            } else {
              if (!chk(idx, ld, "backward block shared gather")) return false;
              for (int c = 0; c < 3; ++c) v[c] = -sx[idx + c * ld];
            }
            for (int c = 0; c < 3; ++c) acc[c] += f.Wb[wi] * v[c];
          }
          for (int c = 0; c < 3; ++c) sx[I.c0l + j0t + l + c * ld] += acc[c];
        }
      }
    for (int k = 0; k < nc; ++k)
      for (int c = 0; c < 3; ++c) x[B.c0 + k + c * n] = sx[k + c * ld];
  }
  xout.assign(3 * n, 0.);
  for (int64_t k = 0; k < n; ++k)
    for (int c = 0; c < 3; ++c) xout[3 * (size_t)f.perm[k] + c] = x[k + c * n];
  return true;
}

}  // namespace pdfb

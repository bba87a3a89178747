// Host-side set-up of the multigrid hierarchy (see fb_setup.h).
#include "fb_setup.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <limits>

namespace fb
{
  std::string import_csr(HostCsr& out, uint64_t rows, uint64_t cols, uint64_t nnz, const uint64_t* rp,
                         const uint64_t* col, const double* val, bool drop_zeros)
  {
    if(rows >= (1ull << 31) || cols >= (1ull << 31) || nnz >= (1ull << 32) - 64)
      return "matrix too large for 32-bit device indices";
    if(!rp || (nnz && (!col || !val)))
      return "null CSR array";
    if(rp[0] != 0 || rp[rows] != nnz)
      return "row_ptr does not span used_elements";
    out.rows = uint32_t(rows);
    out.cols = uint32_t(cols);
    out.rp.assign(rows + 1, 0);
    out.col.clear();
    out.val.clear();
    out.col.reserve(nnz);
    out.val.reserve(nnz);
    for(uint64_t r = 0; r < rows; ++r)
    {
      if(rp[r + 1] < rp[r])
        return "row_ptr is not monotone";
      for(uint64_t j = rp[r]; j < rp[r + 1]; ++j)
      {
        if(col[j] >= cols)
          return "column index out of range";
        if(drop_zeros && val[j] == 0.0)
          continue;
        out.col.push_back(uint32_t(col[j]));
        out.val.push_back(val[j]);
      }
      out.rp[r + 1] = uint32_t(out.col.size());
    }
    return std::string();
  }

  std::vector<uint32_t> inverse_perm(const std::vector<uint32_t>& perm)
  {
    std::vector<uint32_t> inv(perm.size());
    for(uint32_t k = 0; k < perm.size(); ++k)
      inv[perm[k]] = k;
    return inv;
  }

  // BFS level structure from `root`; returns the last level's vertices and the depth.
  static uint32_t bfs_depth(const HostCsr& A, uint32_t root, std::vector<int>& level, std::vector<uint32_t>& last)
  {
    const uint32_t n = A.rows;
    level.assign(n, -1);
    std::vector<uint32_t> cur{root}, nxt;
    level[root] = 0;
    uint32_t depth = 0;
    while(true)
    {
      nxt.clear();
      for(uint32_t v : cur)
        for(uint32_t j = A.rp[v]; j < A.rp[v + 1]; ++j)
        {
          const uint32_t w = A.col[j];
          if(level[w] < 0)
          {
            level[w] = int(depth + 1);
            nxt.push_back(w);
          }
        }
      if(nxt.empty())
        break;
      ++depth;
      cur.swap(nxt);
    }
    last = cur;
    return depth;
  }

  std::vector<uint32_t> rcm_order(const HostCsr& A)
  {
    const uint32_t n = A.rows;
    std::vector<uint32_t> deg(n);
    for(uint32_t i = 0; i < n; ++i)
      deg[i] = A.rp[i + 1] - A.rp[i];
    std::vector<uint32_t> order;
    order.reserve(n);
    std::vector<char> done(n, 0);
    std::vector<int> level;
    std::vector<uint32_t> last;
    for(uint32_t start = 0; start < n; ++start)
    {
      if(done[start])
        continue;
      // pseudo-peripheral root: repeat BFS from a minimum-degree vertex of the deepest level
      uint32_t root = start;
      uint32_t depth = bfs_depth(A, root, level, last);
      for(int rep = 0; rep < 8; ++rep)
      {
        uint32_t cand = last[0];
        for(uint32_t v : last)
          if(deg[v] < deg[cand] || (deg[v] == deg[cand] && v < cand))
            cand = v;
        std::vector<uint32_t> last2;
        std::vector<int> level2;
        const uint32_t d2 = bfs_depth(A, cand, level2, last2);
        if(d2 <= depth)
          break;
        depth = d2;
        root = cand;
        level.swap(level2);
        last.swap(last2);
      }
      // Cuthill-McKee from root: neighbours in increasing degree (ties by index)
      std::deque<uint32_t> q{root};
      done[root] = 1;
      std::vector<uint32_t> nb;
      while(!q.empty())
      {
        const uint32_t v = q.front();
        q.pop_front();
        order.push_back(v);
        nb.clear();
        for(uint32_t j = A.rp[v]; j < A.rp[v + 1]; ++j)
        {
          const uint32_t w = A.col[j];
          if(!done[w])
          {
            done[w] = 1;
            nb.push_back(w);
          }
        }
        std::sort(nb.begin(), nb.end(), [&](uint32_t a, uint32_t b)
        {
          return deg[a] != deg[b] ? deg[a] < deg[b] : a < b;
        });
        for(uint32_t w : nb)
          q.push_back(w);
      }
    }
    std::reverse(order.begin(), order.end());
    return order;
  }

  HostCsr permute(const HostCsr& M, const std::vector<uint32_t>& perm_r, const std::vector<uint32_t>& inv_c)
  {
    HostCsr B;
    B.rows = M.rows;
    B.cols = M.cols;
    B.rp.assign(size_t(M.rows) + 1, 0);
    B.col.resize(M.col.size());
    B.val.resize(M.val.size());
    uint32_t pos = 0;
    for(uint32_t k = 0; k < M.rows; ++k)
    {
      const uint32_t r = perm_r.empty() ? k : perm_r[k];
      for(uint32_t j = M.rp[r]; j < M.rp[r + 1]; ++j)
      {
        B.col[pos] = inv_c.empty() ? M.col[j] : inv_c[M.col[j]];
        B.val[pos] = M.val[j];
        ++pos;
      }
      B.rp[k + 1] = pos;
    }
    return B;
  }

  std::vector<double> inv_diagonal(const HostCsr& A, double omega)
  {
    std::vector<double> d(A.rows);
    for(uint32_t r = 0; r < A.rows; ++r)
    {
      double a = 0.0;
      for(uint32_t j = A.rp[r]; j < A.rp[r + 1]; ++j)
        if(A.col[j] == r)
        {
          a = A.val[j];
          break;
        }
      d[r] = omega / a;
    }
    return d;
  }

  uint64_t HostSell::slot(uint32_t r, uint32_t j, uint32_t c) const
  {
    if(!doff.empty())
    {
      const int32_t o = int32_t(int64_t(c) - int64_t(r));
      const uint32_t k = uint32_t(std::lower_bound(doff.begin(), doff.end(), o) - doff.begin());
      return uint64_t(soff[r / 32u]) + uint64_t(k) * 32u + (r % 32u);
    }
    return uint64_t(soff[r / 32u]) + uint64_t(j) * 32u + (r % 32u);
  }

  // Diagonal storage of a square matrix (see HostSell); false when it does not qualify or would
  // store more than 12.5% padding.
  static bool build_diag(HostSell& H, const HostCsr& M, const std::vector<uint8_t>* empty)
  {
    const uint32_t n = M.rows, ns = (n + 31u) / 32u;
    std::vector<int32_t> offs;
    uint64_t nnz = 0;
    for(uint32_t r = 0; r < n; ++r)
    {
      if(empty && (*empty)[r])
        continue;
      int64_t prev = INT64_MIN;
      for(uint32_t j = M.rp[r]; j < M.rp[r + 1]; ++j)
      {
        const int64_t d = int64_t(M.col[j]) - int64_t(r);
        if(d <= prev)
          return false;
        prev = d;
        if(std::find(offs.begin(), offs.end(), int32_t(d)) == offs.end())
        {
          if(offs.size() >= DIAG_MAX)
            return false;
          offs.push_back(int32_t(d));
        }
      }
      nnz += M.rp[r + 1] - M.rp[r];
    }
    // small matrices (the coarse levels) take the diagonal form whatever their padding: the bytes
    // do not matter there, the shorter row sums do
    const uint32_t K = uint32_t(offs.size());
    if(!K || (uint64_t(K) * 32u * ns > nnz + nnz / 8 && n > DIAG_SMALL_ROWS))
      return false;
    std::sort(offs.begin(), offs.end());
    H.rows = n;
    H.cols = M.cols;
    H.kw = K;
    H.nnz = nnz;
    H.narrow = false;
    H.doff = offs;
    H.soff.assign(size_t(ns) + 1, 0u);
    for(uint32_t sl = 0; sl <= ns; ++sl)
      H.soff[sl] = sl * 32u * K;
    H.entries = H.soff[ns];
    H.val.assign(H.entries, 0.0);
    for(uint32_t r = 0; r < n; ++r)
      if(!(empty && (*empty)[r]))
        for(uint32_t j = M.rp[r]; j < M.rp[r + 1]; ++j)
          H.val[H.slot(r, j - M.rp[r], M.col[j])] = M.val[j];
    return true;
  }

  HostSell build_sell(const HostCsr& M, const std::vector<uint8_t>* empty, bool allow_narrow, bool allow_diag)
  {
    HostSell H;
    if(allow_diag && M.rows == M.cols && build_diag(H, M, empty))
      return H;
    const uint32_t n = M.rows, ns = (n + 31u) / 32u;
    H.rows = n;
    H.cols = M.cols;
    H.soff.assign(size_t(ns) + 1, 0u);
    bool narrow = allow_narrow && (M.rows == M.cols);
    auto len = [&](uint32_t r) -> uint32_t
    {
      if(r >= n || (empty && (*empty)[r]))
        return 0u;
      return M.rp[r + 1] - M.rp[r];
    };
    for(uint32_t sl = 0; sl < ns; ++sl)
    {
      uint32_t K = 0;
      for(uint32_t r = sl * 32u; r < std::min(n, sl * 32u + 32u); ++r)
      {
        const uint32_t L = len(r);
        K = std::max(K, L);
        H.nnz += L;
        for(uint32_t j = M.rp[r]; j < M.rp[r] + L; ++j)
        {
          const int64_t dlt = int64_t(M.col[j]) - int64_t(r);
          if(dlt < -32768 || dlt > 32767)
            narrow = false;
        }
      }
      H.soff[sl + 1] = H.soff[sl] + K * 32u;
    }
    uint32_t kmax = 0;
    for(uint32_t sl = 0; sl < ns; ++sl)
      kmax = std::max(kmax, (H.soff[sl + 1] - H.soff[sl]) / 32u);
    const bool uniform = uint64_t(kmax) * 32u * ns <= H.soff[ns] + H.soff[ns] / 8;
    if(uniform)
    {
      for(uint32_t sl = 0; sl <= ns; ++sl)
        H.soff[sl] = sl * 32u * kmax;
      H.kw = kmax;
    }
    H.entries = H.soff[ns];
    H.narrow = narrow;
    H.val.assign(H.entries, 0.0);
    if(narrow)
      H.dcol.assign(H.entries, 0);
    else
      H.col.assign(H.entries, M.cols);
    for(uint32_t sl = 0; sl < ns; ++sl)
    {
      const uint32_t K = (H.soff[sl + 1] - H.soff[sl]) / 32u;
      for(uint32_t lane = 0; lane < 32u; ++lane)
      {
        const uint32_t r = sl * 32u + lane;
        const uint32_t L = len(r);
        for(uint32_t k = 0; k < K && k < L; ++k)
        {
          const uint64_t e = H.soff[sl] + uint64_t(k) * 32u + lane;
          const uint32_t j = M.rp[r] + k;
          H.val[e] = M.val[j];
          if(narrow)
            H.dcol[e] = int16_t(int64_t(M.col[j]) - int64_t(r));
          else
            H.col[e] = M.col[j];
        }
      }
    }
    return H;
  }

  void coarse_inverse(const HostCsr& A, const std::vector<uint8_t>& dmask, std::vector<uint32_t>& free_dofs,
                      std::vector<double>& inv)
  {
    const uint32_t n = A.rows;
    free_dofs.clear();
    std::vector<uint32_t> pos(n, std::numeric_limits<uint32_t>::max());
    for(uint32_t i = 0; i < n; ++i)
      if(!dmask[i])
      {
        pos[i] = uint32_t(free_dofs.size());
        free_dofs.push_back(i);
      }
    const size_t m = free_dofs.size();
    std::vector<double> a(m * m, 0.0);
    inv.assign(m * m, 0.0);
    for(size_t i = 0; i < m; ++i)
    {
      const uint32_t r = free_dofs[i];
      for(uint32_t k = A.rp[r]; k < A.rp[r + 1]; ++k)
      {
        const uint32_t c = A.col[k];
        if(pos[c] != std::numeric_limits<uint32_t>::max())
          a[i * m + pos[c]] = A.val[k];
      }
      inv[i * m + i] = 1.0;
    }
    for(size_t c = 0; c < m; ++c)
    {
      size_t p = c;
      for(size_t r = c + 1; r < m; ++r)
        if(std::fabs(a[r * m + c]) > std::fabs(a[p * m + c]))
          p = r;
      if(p != c)
        for(size_t j = 0; j < m; ++j)
        {
          std::swap(a[p * m + j], a[c * m + j]);
          std::swap(inv[p * m + j], inv[c * m + j]);
        }
      const double d = a[c * m + c];
      for(size_t j = 0; j < m; ++j)
      {
        a[c * m + j] /= d;
        inv[c * m + j] /= d;
      }
      for(size_t r = 0; r < m; ++r)
      {
        if(r == c)
          continue;
        const double f = a[r * m + c];
        if(f == 0.0)
          continue;
        for(size_t j = 0; j < m; ++j)
        {
          a[r * m + j] -= f * a[c * m + j];
          inv[r * m + j] -= f * inv[c * m + j];
        }
      }
    }
  }

  SweepOrder sweep_levels(const HostCsr& A, bool backward)
  {
    const uint32_t n = A.rows;
    std::vector<uint32_t> lvl(n, 0);
    uint32_t top = 0;
    auto visit = [&](uint32_t i)
    {
      uint32_t l = 0;
      for(uint32_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      {
        const uint32_t j = A.col[k];
        if(backward ? j > i : j < i)
          l = std::max(l, lvl[j] + 1u);
      }
      lvl[i] = l;
      top = std::max(top, l);
    };
    if(backward)
      for(uint32_t i = n; i > 0; --i)
        visit(i - 1);
    else
      for(uint32_t i = 0; i < n; ++i)
        visit(i);
    SweepOrder so;
    const uint32_t nl = n ? top + 1 : 0;
    so.cofs.assign(size_t(nl) + 1, 0u);
    for(uint32_t i = 0; i < n; ++i)
      ++so.cofs[size_t(lvl[i]) + 1];
    for(uint32_t l = 0; l < nl; ++l)
      so.cofs[size_t(l) + 1] += so.cofs[l];
    so.order.resize(n);
    std::vector<uint32_t> fill(so.cofs.begin(), so.cofs.end() - 1);
    for(uint32_t i = 0; i < n; ++i)
      so.order[fill[lvl[i]]++] = i;
    return so;
  }

  SweepOrder greedy_colours(const HostCsr& A)
  {
    const uint32_t n = A.rows;
    // coupled rows of the symmetric pattern that precede row i: row i's own entries j < i and the
    // rows j < i that store an entry in column i
    std::vector<uint32_t> tp(size_t(n) + 1, 0u);
    for(uint32_t c : A.col)
      if(c < n)
        ++tp[size_t(c) + 1];
    for(uint32_t i = 0; i < n; ++i)
      tp[size_t(i) + 1] += tp[i];
    std::vector<uint32_t> tc(tp[n]), fill(tp.begin(), tp.end() - 1);
    for(uint32_t i = 0; i < n; ++i)
      for(uint32_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if(A.col[k] < n)
          tc[fill[A.col[k]]++] = i;
    std::vector<uint32_t> colour(n, 0u);
    std::vector<uint32_t> mark(size_t(n) + 1, UINT32_MAX);
    uint32_t ncol = 0;
    for(uint32_t i = 0; i < n; ++i)
    {
      for(uint32_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
        if(A.col[k] < i)
          mark[colour[A.col[k]]] = i;
      for(uint32_t k = tp[i]; k < tp[size_t(i) + 1]; ++k)
        if(tc[k] < i)
          mark[colour[tc[k]]] = i;
      uint32_t c = 0;
      while(mark[c] == i)
        ++c;
      colour[i] = c;
      ncol = std::max(ncol, c + 1u);
    }
    std::vector<uint32_t> cnt(ncol, 0u);
    for(uint32_t i = 0; i < n; ++i)
      ++cnt[colour[i]];
    std::vector<uint32_t> rank(ncol);
    for(uint32_t c = 0; c < ncol; ++c)
      rank[c] = c;
    std::stable_sort(rank.begin(), rank.end(), [&](uint32_t a, uint32_t b) { return cnt[a] < cnt[b]; });
    std::vector<uint32_t> pos(ncol);
    for(uint32_t r = 0; r < ncol; ++r)
      pos[rank[r]] = r;
    SweepOrder so;
    so.cofs.assign(size_t(ncol) + 1, 0u);
    for(uint32_t r = 0; r < ncol; ++r)
      so.cofs[size_t(r) + 1] = so.cofs[r] + cnt[rank[r]];
    so.order.resize(n);
    std::vector<uint32_t> f2(so.cofs.begin(), so.cofs.end() - 1);
    for(uint32_t i = 0; i < n; ++i)
      so.order[f2[pos[colour[i]]]++] = i;
    return so;
  }
} // namespace fb

// Host-side set-up of the nodal-block matrix structure; see setup.h.
#include "setup.h"

#include <algorithm>
#include <climits>
#include <cstdint>
#include <numeric>

namespace cfdgpu {

std::string build_topology(int nNode, int nElem, int npe, int ndof, const int32_t *conn, int nDBC,
                           const int32_t *dbc_node, const int32_t *dbc_dof, const double *dbc_value,
                           Topology &t)
{
  t = Topology();
  t.nNode = nNode; t.nElem = nElem; t.npe = npe; t.ndof = ndof;
  if (nNode <= 0 || nElem <= 0) return "empty mesh";
  for (int64_t k = 0; k < (int64_t)nElem * npe; k++)
    if (conn[k] < 0 || conn[k] >= nNode) return "connectivity refers to a node outside [0, nNode)";
  // a node listed twice in one element would make two lanes of the element
  // kernel write the same matrix block at once
  for (int e = 0; e < nElem; e++)
    for (int a = 0; a < npe; a++)
      for (int b = a + 1; b < npe; b++)
        if (conn[(int64_t)e * npe + a] == conn[(int64_t)e * npe + b]) return "element with a repeated node";

  // node -> incident elements
  std::vector<int32_t> eptr(nNode + 1, 0);
  for (int64_t k = 0; k < (int64_t)nElem * npe; k++) eptr[conn[k] + 1]++;
  for (int n = 0; n < nNode; n++) eptr[n + 1] += eptr[n];
  std::vector<int32_t> elist(eptr[nNode]);
  {
    std::vector<int32_t> fill(nNode, 0);
    for (int e = 0; e < nElem; e++)
      for (int a = 0; a < npe; a++) {
        int n = conn[(int64_t)e * npe + a];
        elist[eptr[n] + fill[n]++] = e;
      }
  }

  // node graph (block sparsity), sorted per row
  t.rowptr.assign(nNode + 1, 0);
  {
    std::vector<int32_t> mark(nNode, -1);
    for (int n = 0; n < nNode; n++) {
      int cnt = 0;
      for (int k = eptr[n]; k < eptr[n + 1]; k++) {
        const int32_t *c = conn + (int64_t)elist[k] * npe;
        for (int a = 0; a < npe; a++)
          if (mark[c[a]] != n) { mark[c[a]] = n; cnt++; }
      }
      t.rowptr[n + 1] = t.rowptr[n] + cnt;
    }
    t.colidx.resize(t.rowptr[nNode]);
    std::fill(mark.begin(), mark.end(), -1);
    for (int n = 0; n < nNode; n++) {
      int pos = t.rowptr[n];
      for (int k = eptr[n]; k < eptr[n + 1]; k++) {
        const int32_t *c = conn + (int64_t)elist[k] * npe;
        for (int a = 0; a < npe; a++)
          if (mark[c[a]] != n) { mark[c[a]] = n; t.colidx[pos++] = c[a]; }
      }
      std::sort(t.colidx.begin() + t.rowptr[n], t.colidx.begin() + t.rowptr[n + 1]);
    }
  }

  // slot map
  t.slot.resize((int64_t)nElem * npe * npe);
  for (int e = 0; e < nElem; e++) {
    const int32_t *c = conn + (int64_t)e * npe;
    for (int i = 0; i < npe; i++) {
      const int32_t *b = t.colidx.data() + t.rowptr[c[i]];
      const int32_t *en = t.colidx.data() + t.rowptr[c[i] + 1];
      for (int j = 0; j < npe; j++) {
        const int32_t *p = std::lower_bound(b, en, c[j]);
        t.slot[((int64_t)e * npe + i) * npe + j] = (int32_t)(p - t.colidx.data());
      }
    }
  }

  // greedy colouring in element order
  t.color.assign(nElem, -1);
  t.ncolors = 0;
  for (int e = 0; e < nElem; e++) {
    uint64_t used = 0;
    const int32_t *c = conn + (int64_t)e * npe;
    for (int a = 0; a < npe; a++)
      for (int k = eptr[c[a]]; k < eptr[c[a] + 1]; k++) {
        int cc = t.color[elist[k]];
        if (cc >= 0 && cc < 64) used |= (1ULL << cc);
      }
    int cc = 0;
    while (cc < 64 && (used & (1ULL << cc))) cc++;
    if (cc >= 64) return "element colouring needs more than 64 colours";
    t.color[e] = cc;
    t.ncolors = std::max(t.ncolors, cc + 1);
  }
  t.color_ptr.assign(t.ncolors + 1, 0);
  for (int e = 0; e < nElem; e++) t.color_ptr[t.color[e] + 1]++;
  for (int c = 0; c < t.ncolors; c++) t.color_ptr[c + 1] += t.color_ptr[c];
  t.color_elems.resize(nElem);
  {
    std::vector<int32_t> fill(t.ncolors, 0);
    for (int e = 0; e < nElem; e++) t.color_elems[t.color_ptr[t.color[e]] + fill[t.color[e]]++] = e;
  }

  // first writer of each block, in launch order (colour, then element id)
  {
    std::vector<uint8_t> seen(t.colidx.size(), 0);
    for (int k = 0; k < nElem; k++) {
      int e = t.color_elems[k];
      for (int p = 0; p < npe * npe; p++) {
        int32_t &s = t.slot[(int64_t)e * npe * npe + p];
        if (!seen[s]) { seen[s] = 1; s = -s - 1; }
      }
    }
  }

  // Dirichlet sets and free-dof numbering
  t.fixmask.assign(nNode, 0);
  t.dbc_index.resize(nDBC);
  t.dbc_value.resize(nDBC);
  std::vector<int32_t> mult((int64_t)nNode * ndof, 0);
  for (int k = 0; k < nDBC; k++) {
    if (dbc_node[k] < 0 || dbc_node[k] >= nNode || dbc_dof[k] < 0 || dbc_dof[k] >= ndof)
      return "Dirichlet entry outside the mesh";
    int32_t g = dbc_node[k] * ndof + dbc_dof[k];
    t.dbc_index[k] = g;
    t.dbc_value[k] = dbc_value[k];
    t.fixmask[dbc_node[k]] |= (uint8_t)(1u << dbc_dof[k]);
    mult[g]++;
  }
  t.dofmap.assign((int64_t)nNode * ndof, -1);
  t.nfree = 0;
  for (int64_t g = 0; g < (int64_t)nNode * ndof; g++) {
    if (mult[g]) {
      t.fixed_dofs.push_back((int32_t)g);
      t.dbc_mult.push_back(mult[g]);
    } else {
      t.dofmap[g] = t.nfree++;
    }
  }
  return "";
}

std::string build_ilu_pattern(const Topology &t, int levels, int nblocks, IluPattern &f)
{
  f = IluPattern();
  const int n = t.nNode;
  if (levels < -1 || levels > 16) return "ILU levels must lie in [0, 16], or -1 for a complete factorisation";
  const int nb = std::max(1, std::min(nblocks, n));
  f.levels = levels;
  f.nblocks = nb;
  if (levels < 0) levels = 1 << 29;
  f.blk.resize(nb + 1);
  {
    const int q = n / nb, r = n % nb;
    for (int b = 0; b <= nb; b++) f.blk[b] = b * q + std::min(b, r);
  }
  const uint8_t all = (uint8_t)((1u << t.ndof) - 1u);
  auto fixed_node0 = [&](int v) { return (t.fixmask[v] & all) == all; };
  if (f.levels < 0 && nb == 1) {
    // reverse Cuthill-McKee: breadth-first from a minimum-degree node of each
    // component, neighbours in increasing degree, the whole order reversed
    std::vector<int32_t> deg(n), order;
    order.reserve(n);
    for (int v = 0; v < n; v++) deg[v] = t.rowptr[v + 1] - t.rowptr[v];
    std::vector<uint8_t> seen(n, 0);
    std::vector<int32_t> nbr;
    while ((int)order.size() < n) {
      int s0 = -1;
      for (int v = 0; v < n; v++)
        if (!seen[v] && (s0 < 0 || deg[v] < deg[s0])) s0 = v;
      seen[s0] = 1;
      size_t head = order.size();
      order.push_back(s0);
      while (head < order.size()) {
        const int v = order[head++];
        nbr.clear();
        for (int k = t.rowptr[v]; k < t.rowptr[v + 1]; k++)
          if (!seen[t.colidx[k]]) { seen[t.colidx[k]] = 1; nbr.push_back(t.colidx[k]); }
        std::stable_sort(nbr.begin(), nbr.end(), [&](int a, int b) { return deg[a] < deg[b]; });
        order.insert(order.end(), nbr.begin(), nbr.end());
      }
    }
    f.perm.assign(order.rbegin(), order.rend());
    f.iperm.resize(n);
    for (int i = 0; i < n; i++) f.iperm[f.perm[i]] = i;
  }
  auto P = [&](int i) { return f.perm.empty() ? i : f.perm[i]; };    // factor row -> node
  auto IP = [&](int v) { return f.iperm.empty() ? v : f.iperm[v]; };  // node -> factor row
  auto fixed_node = [&](int i) { return fixed_node0(P(i)); };
  std::vector<int32_t> blk_of(n);
  for (int b = 0; b < nb; b++)
    for (int v = f.blk[b]; v < f.blk[b + 1]; v++) blk_of[v] = b;
  std::vector<int32_t> rowcols;
  // per-row sorted linked list over column nodes (n = end marker)
  std::vector<int32_t> next(n + 1), lv(n);
  std::vector<int32_t> ulev;       // level of every stored entry
  f.rowptr.assign(n + 1, 0);
  f.diag.assign(n, -1);
  f.colidx.reserve(t.colidx.size());
  ulev.reserve(t.colidx.size());
  for (int i = 0; i < n; i++) {
    int head = n, tail = -1;
    auto push = [&](int c) {
      lv[c] = 0;
      if (tail < 0) head = c; else next[tail] = c;
      tail = c;
    };
    if (fixed_node(i)) {
      push(i);
    } else {
      const int v = P(i);
      rowcols.clear();
      for (int k = t.rowptr[v]; k < t.rowptr[v + 1]; k++) {
        const int c = IP(t.colidx[k]);
        if (blk_of[c] != blk_of[i] || (c != i && fixed_node(c))) continue;
        rowcols.push_back(c);
      }
      std::sort(rowcols.begin(), rowcols.end());
      for (int c : rowcols) push(c);
    }
    if (tail >= 0) next[tail] = n;
    for (int p = head; p < i; p = next[p]) {
      const int lp = lv[p];
      if (lp + 1 > levels) continue;
      int ins = p;
      for (int q = f.diag[p] + 1; q < f.rowptr[p + 1]; q++) {
        const int j = f.colidx[q];
        const int l = lp + ulev[q] + 1;
        if (l > levels) continue;
        while (next[ins] < j) ins = next[ins];
        if (next[ins] == j) {
          if (l < lv[j]) lv[j] = l;
        } else {
          next[j] = next[ins];
          next[ins] = j;
          lv[j] = l;
        }
        ins = j;
      }
    }
    for (int c = head; c < n; c = next[c]) {
      if (c == i) f.diag[i] = (int32_t)f.colidx.size();
      if ((int64_t)f.colidx.size() >= INT32_MAX) return "ILU factors exceed 2^31 blocks";
      f.colidx.push_back(c);
      ulev.push_back(lv[c]);
    }
    f.rowptr[i + 1] = (int32_t)f.colidx.size();
    if (f.diag[i] < 0) return "node without a diagonal block";
  }
  // level-set orders of the lower and upper dependency DAGs
  {
    std::vector<int32_t> lev(n, 0);
    auto order_by = [&](std::vector<int32_t> &out, int &maxw) {
      int nl = 0;
      for (int i = 0; i < n; i++) nl = std::max(nl, lev[i] + 1);
      std::vector<int32_t> cnt(nl + 1, 0);
      for (int i = 0; i < n; i++) cnt[lev[i] + 1]++;
      maxw = 0;
      for (int k = 0; k < nl; k++) maxw = std::max(maxw, cnt[k + 1]);
      for (int k = 0; k < nl; k++) cnt[k + 1] += cnt[k];
      out.resize(n);
      for (int i = 0; i < n; i++) out[cnt[lev[i]]++] = i;
      return nl;
    };
    for (int i = 0; i < n; i++) {
      int d = 0;
      for (int q = f.rowptr[i]; q < f.diag[i]; q++) d = std::max(d, lev[f.colidx[q]] + 1);
      lev[i] = d;
    }
    f.nlev_l = order_by(f.lorder, f.maxw_l);
    for (int i = n - 1; i >= 0; i--) {
      int d = 0;
      for (int q = f.diag[i] + 1; q < f.rowptr[i + 1]; q++) d = std::max(d, lev[f.colidx[q]] + 1);
      lev[i] = d;
    }
    f.nlev_u = order_by(f.uorder, f.maxw_u);
  }
  // chains of the lower (ascending) and upper (descending) solves and their
  // DAG levels
  {
    auto chains = [&](bool upper, std::vector<int32_t> &ch, std::vector<int32_t> &order, int &nlev, int &maxw) {
      ch.clear();
      std::vector<int32_t> chain_of(n);
      if (!upper) {
        int start = 0;
        for (int i = 1; i <= n; i++) {
          const bool cont = i < n && i - start < ILU_CHAIN_MAX && f.diag[i] > f.rowptr[i] &&
                            f.colidx[f.diag[i] - 1] == i - 1;
          if (!cont) { ch.push_back(start); ch.push_back(i); start = i; }
        }
      } else {
        int end = n;   // current chain covers [i, end)
        for (int i = n - 2; i >= -1; i--) {
          const int r = i + 1;   // row just added
          const bool cont = i >= 0 && end - i <= ILU_CHAIN_MAX && f.diag[i] + 1 < f.rowptr[i + 1] &&
                            f.colidx[f.diag[i] + 1] == i + 1;
          if (!cont) { ch.push_back(r); ch.push_back(end); end = r; }
        }
      }
      const int nc = (int)ch.size() / 2;
      for (int c = 0; c < nc; c++)
        for (int i = ch[2 * c]; i < ch[2 * c + 1]; i++) chain_of[i] = c;
      std::vector<int32_t> lev(nc, 0);
      // chains are listed in dependency order (ascending rows for the lower
      // solve, descending for the upper one), so one pass finds the levels
      for (int c = 0; c < nc; c++) {
        int d = 0;
        for (int i = ch[2 * c]; i < ch[2 * c + 1]; i++) {
          const int q0 = upper ? f.diag[i] + 1 : f.rowptr[i], q1 = upper ? f.rowptr[i + 1] : f.diag[i];
          for (int q = q0; q < q1; q++) {
            const int oc = chain_of[f.colidx[q]];
            if (oc != c) d = std::max(d, lev[oc] + 1);
          }
        }
        lev[c] = d;
      }
      nlev = 0;
      for (int c = 0; c < nc; c++) nlev = std::max(nlev, lev[c] + 1);
      std::vector<int32_t> cnt(nlev + 1, 0);
      for (int c = 0; c < nc; c++) cnt[lev[c] + 1]++;
      maxw = 0;
      for (int k = 0; k < nlev; k++) maxw = std::max(maxw, cnt[k + 1]);
      for (int k = 0; k < nlev; k++) cnt[k + 1] += cnt[k];
      order.resize(nc);
      for (int c = 0; c < nc; c++) order[cnt[lev[c]]++] = c;
    };
    chains(false, f.lchain, f.lchain_order, f.lchain_levels, f.lchain_maxw);
    chains(true, f.uchain, f.uchain_order, f.uchain_levels, f.uchain_maxw);
  }
  // update map: positions in row i of the upper blocks of every pivot row
  {
    int64_t total = 0;
    f.uoff.assign(f.colidx.size(), -1);
    for (int i = 0; i < n; i++)
      for (int q = f.rowptr[i]; q < f.diag[i]; q++) {
        const int p = f.colidx[q];
        f.uoff[q] = total;
        total += f.rowptr[p + 1] - f.diag[p] - 1;
      }
    f.umap.resize(total);
    std::vector<int32_t> pos(n, -1);
    for (int i = 0; i < n; i++) {
      for (int k = f.rowptr[i]; k < f.rowptr[i + 1]; k++) pos[f.colidx[k]] = k;
      for (int q = f.rowptr[i]; q < f.diag[i]; q++) {
        const int p = f.colidx[q];
        int64_t o = f.uoff[q];
        for (int u = f.diag[p] + 1; u < f.rowptr[p + 1]; u++) f.umap[o++] = pos[f.colidx[u]];
      }
      for (int k = f.rowptr[i]; k < f.rowptr[i + 1]; k++) pos[f.colidx[k]] = -1;
    }
  }
  // blocks of A inside the factor pattern (A's block (v, c) lands in factor
  // row IP(v) at column IP(c))
  f.aslot.assign(t.colidx.size(), -1);
  for (int v = 0; v < n; v++) {
    const int i = IP(v);
    const int32_t *b = f.colidx.data() + f.rowptr[i], *e = f.colidx.data() + f.rowptr[i + 1];
    for (int k = t.rowptr[v]; k < t.rowptr[v + 1]; k++) {
      const int c = IP(t.colidx[k]);
      const int32_t *p = std::lower_bound(b, e, c);
      if (p != e && *p == c) f.aslot[k] = (int32_t)(p - f.colidx.data());
    }
  }
  return "";
}

}  // namespace cfdgpu

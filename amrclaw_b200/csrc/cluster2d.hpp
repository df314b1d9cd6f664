// Host-side integer algorithms of 2D regridding: flag buffering and projection,
// proper-nesting masks, point collation and Berger-Rigoutsos bisection.
//
// These consume the per-cell gradient flags computed on the device and produce
// the new patch rectangles. Each function follows the reference algorithm named
// beside it so that the resulting hierarchy (rectangles and their order) is
// identical to the reference's:
//   shift_buffer      src/2d/shiftset2.f:25-71
//   nesting masks     src/2d/setdomflags.f:22-207, griddomshrink.f:24-82,
//                     griddomup.f:16-116, setPhysBndryFlags.f:28-78
//   sort_unique       src/2d/drivesort.f:7-62 with quick_sort1.f:22-167
//   bisect            src/2d/smartbis.f:25-177, signs.f:16-71, findcut.f:7-130,
//                     moment.f:16-75
//   nest_check        src/2d/nestck2.f:37-176, baseCheck.f:19-240
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <vector>

namespace amrb {

// Box-indexed integer array over (ilo-mb .. ihi+mb) x (jlo-mb .. jhi+mb), column-major.
struct IBox {
  int ilo, ihi, jlo, jhi, mb;
  int ni() const { return ihi - ilo + 1 + 2 * mb; }
  int nj() const { return jhi - jlo + 1 + 2 * mb; }
  size_t idx(int i, int j) const { return (size_t)(i - (ilo - mb)) + (size_t)ni() * (size_t)(j - (jlo - mb)); }
};

// Non-stable quicksort of an index permutation by integer keys, with the exact
// sequence of comparisons and swaps of quick_sort1.f (ties are broken the same way).
inline void qsort_index(std::vector<int>& ord, int n, const std::vector<long long>& key /* 1-based */) {
  int pop[2][64];
  int nd = 0, u1 = n, l1 = 1, l = 0, u = 0, p = 0, q = 0, ix = 0, iz = 0, t = 0;
  long long x = 0, z = 0, xx = 0, zz = 0, y = 0;
  for (int k = 1; k <= n; ++k) ord[k] = k;
  enum { S2, S3, S4, S6, S7, S8, S9, S10, S13, S15, S16, S17, S18 } st = S2;
  while (true) {
    switch (st) {
      case S2: if (u1 <= l1) return; st = S3; break;
      case S3: l = l1; u = u1; st = S4; break;
      case S4:
        p = l; q = u; x = key[ord[p]]; z = key[ord[q]];
        if (!(x <= z)) { y = x; x = z; z = y; t = ord[p]; ord[p] = ord[q]; ord[q] = t; }
        if (u - l <= 1) { st = S15; break; }
        xx = x; ix = p; zz = z; iz = q; st = S6; break;
      case S6: p = p + 1; if (p >= q) { st = S7; break; } x = key[ord[p]]; st = (x >= xx) ? S8 : S6; break;
      case S7: p = q - 1; st = S13; break;
      case S8: q = q - 1; if (q <= p) { st = S9; break; } z = key[ord[q]]; st = (z <= zz) ? S10 : S8; break;
      case S9: q = p; p = p - 1; z = x; x = key[ord[p]]; st = S10; break;
      case S10:
        if (!(x <= z)) { y = x; x = z; z = y; t = ord[p]; ord[p] = ord[q]; ord[q] = t; }
        if (!(x <= xx)) { xx = x; ix = p; }
        if (!(z >= zz)) { zz = z; iz = q; }
        st = S6; break;
      case S13:
        if (p != ix && x != xx) { t = ord[p]; ord[p] = ord[ix]; ord[ix] = t; }
        if (q != iz && z != zz) { t = ord[q]; ord[q] = ord[iz]; ord[iz] = t; }
        st = S15; break;
      case S15: st = (u - q <= p - l) ? S16 : S17; if (st == S17) { l1 = l; u1 = p - 1; l = q + 1; } break;
      case S16: u1 = u; l1 = q + 1; u = p - 1; st = S17; break;
      case S17:
        if (u1 <= l1) { st = S18; break; }
        nd = nd + 1; pop[0][nd] = u; pop[1][nd] = l; st = S3; break;
      case S18:
        if (u > l) { st = S4; break; }
        if (nd == 0) { st = S2; break; }
        u = pop[0][nd]; l = pop[1][nd]; nd = nd - 1; st = S18; break;
    }
  }
}

// Flagged points are kept as integer cell coordinates (the reference stores
// i+0.5, j+0.5 in doubles; integer centres carry the same information).
struct Pt { int i, j; };

// drivesort.f: sort the flagged points by the key i + (isize+2*mbuff)*j and drop
// duplicates. Distinct integer keys have exactly one ascending order, so a scan of
// a byte map over the points' bounding box (j outer, i inner) gives the
// reference's result without its quicksort.
inline void sort_unique(std::vector<Pt>& pts, int isize, int mbuff) {
  (void)isize; (void)mbuff;
  const size_t n = pts.size();
  if (n == 0) return;
  int i0 = pts[0].i, i1 = i0, j0 = pts[0].j, j1 = j0;
  for (const Pt& q : pts) { i0 = std::min(i0, q.i); i1 = std::max(i1, q.i); j0 = std::min(j0, q.j); j1 = std::max(j1, q.j); }
  const size_t w = (size_t)(i1 - i0 + 1), h = (size_t)(j1 - j0 + 1);
  std::vector<Pt> out;
  if (w * h <= 16 * n + (1u << 22)) {
    std::vector<uint8_t> map(w * h, 0);
    for (const Pt& q : pts) map[(size_t)(q.j - j0) * w + (q.i - i0)] = 1;
    out.reserve(n);
    for (size_t j = 0; j < h; ++j)
      for (size_t i = 0; i < w; ++i)
        if (map[j * w + i]) out.push_back(Pt{(int)i + i0, (int)j + j0});
  } else {
    std::vector<long long> key(n);
    for (size_t k = 0; k < n; ++k) key[k] = (long long)(pts[k].i - i0) + (long long)w * (pts[k].j - j0);
    std::sort(key.begin(), key.end());
    key.erase(std::unique(key.begin(), key.end()), key.end());
    out.reserve(key.size());
    for (long long e : key) out.push_back(Pt{(int)(e % (long long)w) + i0, (int)(e / (long long)w) + j0});
  }
  pts.swap(out);
}

// Bounding box and fill ratio of a cluster of points (moment.f).
inline double bbox_usage(const Pt* p, int n, int rect[4]) {
  int i0 = p[0].i, i1 = p[0].i, j0 = p[0].j, j1 = p[0].j;
  for (int k = 0; k < n; ++k) {
    i0 = std::min(i0, p[k].i); i1 = std::max(i1, p[k].i);
    j0 = std::min(j0, p[k].j); j1 = std::max(j1, p[k].j);
  }
  rect[0] = i0; rect[1] = i1; rect[2] = j0; rect[3] = j1;
  return (double)n / (double)((i1 - i0 + 1) * (j1 - j0 + 1));
}

// Best cut of a cluster from its row/column signatures (signs.f + findcut.f).
// Returns the 1-based cut index (0: no acceptable cut) and the direction (1: x, 2: y).
inline int find_cut(const Pt* p, int n, int idim, int jdim, int& dir) {
  std::vector<int> is(idim + 2, 0), js(jdim + 2, 0);
  for (int k = 0; k < n; ++k) { is[p[k].i + 1] += 1; js[p[k].j + 1] += 1; }
  int ilo = 1, ihi = idim, jlo = 1, jhi = jdim;
  for (int t = 1; t <= idim; ++t) if (is[t] != 0) { ilo = t; break; }
  for (int t = 1; t <= idim; ++t) if (is[idim + 1 - t] != 0) { ihi = idim + 1 - t; break; }
  for (int t = 1; t <= jdim; ++t) if (js[t] != 0) { jlo = t; break; }
  for (int t = 1; t <= jdim; ++t) if (js[jdim + 1 - t] != 0) { jhi = jdim + 1 - t; break; }
  for (int i = ilo; i <= ihi; ++i) if (is[i] == 0) { dir = 1; return i; }
  for (int j = jlo; j <= jhi; ++j) if (js[j] == 0) { dir = 2; return j; }
  auto lap = [](std::vector<int>& s, int lo, int hi, int& best, int& idx) {
    int pre = s[lo];
    for (int i = lo + 1; i <= hi - 1; ++i) { const int cur = s[i]; s[i] = s[i + 1] - 2 * cur + pre; pre = cur; }
    best = 0; idx = 0;
    const int mid = (lo + hi) / 2;
    for (int i = lo + 2; i <= hi - 2 + 1; ++i) {
      const int a = s[i - 1], b = s[i], d = std::abs(a - b);
      if (a * b < 0) {
        if (d > best) { best = d; idx = i; }
        else if (d == best && std::abs(i - mid) < std::abs(idx - mid)) idx = i;
      }
    }
  };
  int bi, ii, bj, ij;
  lap(is, ilo, ihi, bi, ii);
  lap(js, jlo, jhi, bj, ij);
  int index, best;
  if (bi > bj) { index = ii; dir = 1; best = bi; }
  else if (bi < bj) { index = ij; dir = 2; best = bj; }
  else if (std::abs(ii - (ilo + ihi) / 2) < std::abs(ij - (jlo + jhi) / 2)) { index = ii; dir = 1; best = bi; }
  else { index = ij; dir = 2; best = bj; }
  if (best < 2) index = 0;
  return index;
}

// find_cut on signatures already counted (is, js: counts at 1-based positions 1..idim, 1..jdim).
inline int find_cut_sig(std::vector<int> is, std::vector<int> js, int idim, int jdim, int& dir) {
  int ilo = 1, ihi = idim, jlo = 1, jhi = jdim;
  for (int t = 1; t <= idim; ++t) if (is[t] != 0) { ilo = t; break; }
  for (int t = 1; t <= idim; ++t) if (is[idim + 1 - t] != 0) { ihi = idim + 1 - t; break; }
  for (int t = 1; t <= jdim; ++t) if (js[t] != 0) { jlo = t; break; }
  for (int t = 1; t <= jdim; ++t) if (js[jdim + 1 - t] != 0) { jhi = jdim + 1 - t; break; }
  for (int i = ilo; i <= ihi; ++i) if (is[i] == 0) { dir = 1; return i; }
  for (int j = jlo; j <= jhi; ++j) if (js[j] == 0) { dir = 2; return j; }
  auto lap = [](std::vector<int>& s, int lo, int hi, int& best, int& idx) {
    int pre = s[lo];
    for (int i = lo + 1; i <= hi - 1; ++i) { const int cur = s[i]; s[i] = s[i + 1] - 2 * cur + pre; pre = cur; }
    best = 0; idx = 0;
    const int mid = (lo + hi) / 2;
    for (int i = lo + 2; i <= hi - 2 + 1; ++i) {
      const int a = s[i - 1], b = s[i], d = std::abs(a - b);
      if (a * b < 0) {
        if (d > best) { best = d; idx = i; }
        else if (d == best && std::abs(i - mid) < std::abs(idx - mid)) idx = i;
      }
    }
  };
  int bi, ii, bj, ij;
  lap(is, ilo, ihi, bi, ii);
  lap(js, jlo, jhi, bj, ij);
  int index, best;
  if (bi > bj) { index = ii; dir = 1; best = bi; }
  else if (bi < bj) { index = ij; dir = 2; best = bj; }
  else if (std::abs(ii - (ilo + ihi) / 2) < std::abs(ij - (jlo + jhi) / 2)) { index = ii; dir = 1; best = bi; }
  else { index = ij; dir = 2; best = bj; }
  if (best < 2) index = 0;
  return index;
}

// Partition pts[a..b] (inclusive) so that points with coordinate >= cut stay at the
// front, in the in-place swap order of smartbis.f:128-154. Returns the count at the front.
inline int split_front(std::vector<Pt>& pts, int a, int b, int dir, int cut) {
  int top = a - 1, bot = b + 1, i = a;
  auto c = [&](int k) { return dir == 1 ? pts[k].i + 1 : pts[k].j + 1; };  // 1-based coordinate
  while (true) {
    if (c(i) < cut) {
      --bot;
      std::swap(pts[bot], pts[i]);
      if (top + 1 < bot) continue;
      break;
    }
    ++top;
    if (top + 1 >= bot) break;
    ++i;
  }
  return top - a + 1;
}

// Berger-Rigoutsos bisection of a sorted point list into clusters (smartbis.f).
inline void bisect(std::vector<Pt>& pts, double cutoff, int idim, int jdim, std::vector<int>& cnt) {
  cnt.assign(1, (int)pts.size());
  int icl = 0, ist = 0;
  while (icl < (int)cnt.size()) {
    const int n = cnt[icl];
    int rect[4];
    const double use = bbox_usage(&pts[ist], n, rect);
    if (use >= cutoff) { ist += n; ++icl; continue; }
    int dir = 0;
    const int cut = find_cut(&pts[ist], n, idim, jdim, dir);
    if (cut == 0) { ist += n; ++icl; continue; }
    const int front = split_front(pts, ist, ist + n - 1, dir, cut);
    cnt[icl] = front;
    cnt.insert(cnt.begin() + icl + 1, n - front);
  }
}

}  // namespace amrb

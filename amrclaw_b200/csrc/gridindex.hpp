// Uniform-bin spatial index over the patches of one level.
//
// The reference finds overlapping patches by walking the whole level list for
// every query (intfil.f90:153-260, icall.f, prepc.f:77-113, update.f:95-175,
// setdomflags.f, baseCheck.f, init_bndryList.f), which costs O(P^2) per regrid.
// This index answers the same "which patches of the level overlap this box"
// question from the bins the box touches, and returns the hits sorted by their
// position in the level list, so callers visit them in the reference's order.
#pragma once
#include <algorithm>
#include <array>
#include <vector>

namespace amrb {

class GridIndex {
 public:
  // list: patch ids in level-list order; box(id) -> {ilo, ihi, jlo, jhi, klo, khi}
  template <class BoxFn>
  void build(const std::vector<int>& list, BoxFn box, int bin = 16) {
    bs_ = bin;
    ids_ = list;
    boxes_.resize(list.size());
    lo_ = {1 << 30, 1 << 30, 1 << 30};
    std::array<int, 3> hi = {-(1 << 30), -(1 << 30), -(1 << 30)};
    for (size_t r = 0; r < list.size(); ++r) {
      boxes_[r] = box(list[r]);
      for (int d = 0; d < 3; ++d) {
        lo_[d] = std::min(lo_[d], boxes_[r][2 * d]);
        hi[d] = std::max(hi[d], boxes_[r][2 * d + 1]);
      }
    }
    if (list.empty()) { nb_ = {0, 0, 0}; start_.assign(1, 0); items_.clear(); return; }
    for (int d = 0; d < 3; ++d) nb_[d] = (hi[d] - lo_[d]) / bs_ + 1;
    const size_t nbins = (size_t)nb_[0] * nb_[1] * nb_[2];
    start_.assign(nbins + 1, 0);
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<int> fillp;
      if (pass == 1) {
        for (size_t b = 0; b < nbins; ++b) start_[b + 1] += start_[b];
        items_.assign(start_[nbins], 0);
        fillp.assign(start_.begin(), start_.end() - 1);
      }
      for (size_t r = 0; r < list.size(); ++r) {
        int b0[3], b1[3];
        for (int d = 0; d < 3; ++d) { b0[d] = (boxes_[r][2 * d] - lo_[d]) / bs_; b1[d] = (boxes_[r][2 * d + 1] - lo_[d]) / bs_; }
        for (int c = b0[2]; c <= b1[2]; ++c)
          for (int b = b0[1]; b <= b1[1]; ++b)
            for (int a = b0[0]; a <= b1[0]; ++a) {
              const size_t k = ((size_t)c * nb_[1] + b) * nb_[0] + a;
              if (pass == 0) ++start_[k + 1];
              else items_[fillp[k]++] = (int)r;
            }
      }
    }
  }

  // Ranks (positions in the level list) of the patches overlapping the box, ascending.
  // Safe to call from several threads at once.
  void query(int i0, int i1, int j0, int j1, int k0, int k1, std::vector<int>& out) const {
    out.clear();
    if (ids_.empty()) return;
    const int q0[3] = {i0, j0, k0}, q1[3] = {i1, j1, k1};
    int b0[3], b1[3];
    for (int d = 0; d < 3; ++d) {
      const int a = q0[d] - lo_[d], b = q1[d] - lo_[d];
      if (b < 0) return;
      b0[d] = std::max(0, a < 0 ? 0 : a / bs_);
      b1[d] = std::min(nb_[d] - 1, b / bs_);
      if (b0[d] > b1[d]) return;
    }
    for (int c = b0[2]; c <= b1[2]; ++c)
      for (int b = b0[1]; b <= b1[1]; ++b)
        for (int a = b0[0]; a <= b1[0]; ++a) {
          const size_t k = ((size_t)c * nb_[1] + b) * nb_[0] + a;
          for (int t = start_[k]; t < start_[k + 1]; ++t) {
            const int r = items_[t];
            const auto& x = boxes_[r];
            if (x[0] <= i1 && x[1] >= i0 && x[2] <= j1 && x[3] >= j0 && x[4] <= k1 && x[5] >= k0) out.push_back(r);
          }
        }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
  }
  void query2(int i0, int i1, int j0, int j1, std::vector<int>& out) const { query(i0, i1, j0, j1, 0, 0, out); }

  int id(int rank) const { return ids_[rank]; }
  const std::vector<int>& ids() const { return ids_; }
  size_t size() const { return ids_.size(); }

 private:
  int bs_ = 16;
  std::array<int, 3> lo_{}, nb_{};
  std::vector<int> ids_;
  std::vector<std::array<int, 6>> boxes_;
  std::vector<int> start_, items_;
};

}  // namespace amrb

// Oracle trim loops in a face's parameter domain: crossing parity over pieces monotone
// in both parameters, answered through a quadtree of cells with reference points.
// Restates crates/icam-core/src/trim2.rs (Trim2, 79-94 and 1105-1658). The reference
// fits polynomial cubics to each edge and certifies them within the model tolerance;
// the descriptions here carry each use's exact curve as rational cubic pieces
// (u w, v w, w), so a piece is rational and every routine below evaluates it as such.
// TEST INFRASTRUCTURE ONLY.
#pragma once

#include <array>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

namespace oracle {

using P2 = std::array<double, 2>;

struct TPiece {
  std::array<std::array<double, 3>, 4> c;  // (u w, v w, w)
};

class Trim2 {
 public:
  // pieces: each use's curves in traversal order (already monotone or not);
  // inside_left: the face lies left of its loops (trim2.rs:88-91).
  bool build(const std::vector<TPiece>& raw, P2 lo, P2 hi, P2 period, bool inside_left, std::string* err);
  bool inside(double u, double v) const;
  // -1 straddles, 0 wholly outside, 1 wholly inside (trim2.rs:1570-1612)
  int box_class(P2 lo, P2 hi) const;
  size_t piece_count() const { return pieces_.size(); }

 private:
  struct Cell {
    P2 lo, hi, r;
    bool inside;
    int kind;  // 0 leaf, 1 crossed, 2 split
    std::vector<uint32_t> among;
    std::array<uint32_t, 4> kids;
  };
  std::vector<TPiece> pieces_;
  std::vector<std::pair<uint32_t, P2>> instances_;
  std::vector<Cell> cells_;
  P2 lo_{}, hi_{};
  double period_[2] = {0, 0};
  bool inside_left_ = true;

  TPiece shifted(uint32_t inst) const;
  bool parity(P2 a, P2 b, const std::vector<uint32_t>& among) const;
  void build_cell(size_t id, const std::vector<uint32_t>& cand, const std::vector<std::pair<P2, P2>>& boxes,
                  int depth);
  bool offset_from(const TPiece& p, const std::vector<uint32_t>& all, bool left, P2* out) const;
  double dist2_to(uint32_t inst, P2 q) const;
  int class_in(size_t id, P2 lo, P2 hi) const;
};

// helpers shared with the tests of this directory
double tp_eval(const TPiece& p, int k, double t);
P2 tp_at(const TPiece& p, double t);
bool tp_crossing(const TPiece& p, int k, double x, double* t);

}  // namespace oracle

// Oracle C API for the tests and the CPU baseline of bench.py: the exact signed
// distance of points, candidate lists, and the brick-cache bake of a level
// (crates/icam-sim/src/partcache.rs: decide 226-331, exact_brick 979-1058).
// TEST INFRASTRUCTURE ONLY.
#include <atomic>
#include <cstring>
#include <string>
#include <thread>

#include "exact.hpp"
#include "oracle.h"

using namespace oracle;

namespace {

template <class F>
void parallel_for(int64_t n, int threads, F&& f) {
  if (threads <= 1 || n < 2) {
    for (int64_t i = 0; i < n; i++) f(i);
    return;
  }
  std::atomic<int64_t> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++)
    pool.emplace_back([&]() {
      for (;;) {
        int64_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

void* oracle_new(const IcamSolidDesc* d, char* err, int errlen) {
  auto* ex = new Exact();
  std::string e;
  if (!ex->init(d, &e)) {
    if (err && errlen > 0) {
      std::strncpy(err, e.c_str(), errlen - 1);
      err[errlen - 1] = 0;
    }
    delete ex;
    return nullptr;
  }
  return ex;
}

void oracle_free(void* h) { delete static_cast<Exact*>(h); }

void oracle_bbox(void* h, double* lo, double* hi) {
  auto* ex = static_cast<Exact*>(h);
  lo[0] = ex->bbox.first.x;
  lo[1] = ex->bbox.first.y;
  lo[2] = ex->bbox.first.z;
  hi[0] = ex->bbox.second.x;
  hi[1] = ex->bbox.second.y;
  hi[2] = ex->bbox.second.z;
}

int oracle_counts(void* h, int* nf, int* ne, int* nv) {
  auto* ex = static_cast<Exact*>(h);
  *nf = int(ex->nf());
  *ne = int(ex->ne());
  *nv = int(ex->nv());
  return 0;
}

void oracle_sdf(void* h, const double* pts, int64_t n, double bound, double* d_out, double* q_out,
                int32_t* kind_out, int32_t* id_out, uint8_t* unsure_out, int32_t* pops_out, int threads) {
  auto* ex = static_cast<Exact*>(h);
  parallel_for(n, threads, [&](int64_t i) {
    ExactStats st;
    Sd s = ex->sdf_within(V3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), bound, &st);
    d_out[i] = s.d;
    if (q_out) {
      q_out[3 * i] = s.q.x;
      q_out[3 * i + 1] = s.q.y;
      q_out[3 * i + 2] = s.q.z;
    }
    if (kind_out) kind_out[i] = s.kind;
    if (id_out) id_out[i] = s.id;
    if (unsure_out) unsure_out[i] = s.unsure;
    if (pops_out) pops_out[i] = st.pops;
  });
}

int oracle_candidates(void* h, const double* c, double r, double d, int32_t* out, int cap, int32_t* kinds) {
  auto* ex = static_cast<Exact*>(h);
  auto v = ex->candidates(V3(c[0], c[1], c[2]), r, d);
  int n = int(v.size());
  for (int i = 0; i < n && i < cap; i++) {
    out[i] = int32_t(v[i]);
    if (kinds) kinds[i] = ex->kind_of(v[i]);
  }
  return n;
}

// partcache.rs:226-331 decide, with every box centre read on the CPU (box_bounds'
// all_cpu, 341-367). Bricks are named by their index within the level (x fastest);
// the box grid is aligned on `origin` as the reference aligns it on the stock's
// corner. Returns the number of bricks to read (written to read_idx / read_d up to
// cap), and the map (nb[0]*nb[1]*nb[2] entries) with AIR/SOLID decided and
// ORACLE_READ at bricks to read.
// With tight != 0 a box's radius is the half diagonal of its own nodes' box instead of
// the box grown by the clamp: every node still lies within it of the centre, so a box
// it decides AIR (SOLID) holds only nodes past the clamp, which the reference's rule
// reads and packs as an AIR (SOLID) brick. The map after the bricks are read is the same.
int64_t oracle_decide_rule(void* h, double hcell, const double* lo3, const int64_t* nb, double clamp,
                           const double* origin, int threads, int tight, uint32_t* map, int64_t* read_idx,
                           double* read_d, int64_t cap) {
  auto* ex = static_cast<Exact*>(h);
  V3 lo(lo3[0], lo3[1], lo3[2]);
  double side = 8.0 * hcell;
  auto first = [&](const int64_t* b) { return lo + V3(side * b[0], side * b[1], side * b[2]); };
  struct Bx {
    int64_t a[3];
  };
  int64_t nbmax = std::max(nb[0], std::max(nb[1], nb[2]));
  int64_t size = 1;
  while (size < nbmax) size *= 2;
  V3 o(origin[0] - hcell, origin[1] - hcell, origin[2] - hcell);
  int64_t g0[3] = {int64_t(std::llround((lo.x - o.x) / side)), int64_t(std::llround((lo.y - o.y) / side)),
                   int64_t(std::llround((lo.z - o.z) / side))};
  auto start = [&](int k) {
    int64_t q = g0[k] >= 0 ? g0[k] / size : -((-g0[k] + size - 1) / size);
    return q * size - g0[k];
  };
  int64_t total = nb[0] * nb[1] * nb[2];
  for (int64_t i = 0; i < total; i++) map[i] = ORACLE_AIR;
  std::vector<Bx> boxes;
  for (int64_t z = start(2); z < nb[2]; z += size)
    for (int64_t y = start(1); y < nb[1]; y += size)
      for (int64_t x = start(0); x < nb[0]; x += size) boxes.push_back({{x, y, z}});
  int64_t nread = 0;
  while (!boxes.empty()) {
    // grown(a, n): the box of bricks [a, a + n) grown by the clamp; its centre and half diagonal
    std::vector<double> lo_f(boxes.size()), hi_f(boxes.size()), dc(boxes.size());
    parallel_for(int64_t(boxes.size()), threads, [&](int64_t i) {
      const int64_t* a = boxes[i].a;
      int64_t b2[3] = {a[0] + size, a[1] + size, a[2] + size};
      V3 p = first(a) - V3(clamp, clamp, clamp), q = first(b2) + V3(clamp, clamp, clamp);
      V3 c((p.x + q.x) * 0.5, (p.y + q.y) * 0.5, (p.z + q.z) * 0.5);
      double r = tight ? 0.5 * (first(b2) - first(a)).len() : 0.5 * (q - p).len();
      ExactStats st;
      Sd s = ex->sdf(c, &st);
      if (s.unsure) {
        lo_f[i] = -INF;
        hi_f[i] = INF;
        dc[i] = NAN;
      } else {
        lo_f[i] = s.d - r;
        hi_f[i] = s.d + r;
        dc[i] = s.d;
      }
    });
    std::vector<Bx> next;
    for (size_t i = 0; i < boxes.size(); i++) {
      const int64_t* a = boxes[i].a;
      if (lo_f[i] > clamp || hi_f[i] < -clamp) {
        uint32_t v = lo_f[i] > clamp ? ORACLE_AIR : ORACLE_SOLID;
        for (int64_t z = std::max<int64_t>(a[2], 0); z < std::min(a[2] + size, nb[2]); z++)
          for (int64_t y = std::max<int64_t>(a[1], 0); y < std::min(a[1] + size, nb[1]); y++)
            for (int64_t x = std::max<int64_t>(a[0], 0); x < std::min(a[0] + size, nb[0]); x++)
              map[x + nb[0] * (y + nb[1] * z)] = v;
      } else if (size == 1) {
        int64_t idx = a[0] + nb[0] * (a[1] + nb[1] * a[2]);
        map[idx] = ORACLE_READ;
        if (nread < cap) {
          read_idx[nread] = idx;
          read_d[nread] = dc[i];
        }
        nread++;
      } else {
        int64_t half = size / 2;
        for (int q = 0; q < 8; q++) {
          Bx k{{a[0] + half * (q & 1), a[1] + half * ((q >> 1) & 1), a[2] + half * ((q >> 2) & 1)}};
          bool in = true;
          for (int j = 0; j < 3; j++)
            if (!(k.a[j] < nb[j] && k.a[j] + half > 0)) in = false;
          if (in) next.push_back(k);
        }
      }
    }
    boxes.swap(next);
    size /= 2;
  }
  return nread;
}

int64_t oracle_decide(void* h, double hcell, const double* lo3, const int64_t* nb, double clamp, const double* origin,
                      int threads, uint32_t* map, int64_t* read_idx, double* read_d, int64_t cap) {
  return oracle_decide_rule(h, hcell, lo3, nb, clamp, origin, threads, 0, map, read_idx, read_d, cap);
}

// partcache.rs:979-1058 exact_brick: the 729 nodes of each brick whose first node is
// firsts[i], read coarse to fine with the bound the brick's centre gives, each reading
// past the clamp settling the nodes within its empty ball. Writes the values before
// quantisation (f_out, n x 729; the clamp with its sign where a node was settled, not
// read), the stored i16 values (q_out) and the packed kind (0 words, 1 air, 2 solid).
void oracle_bricks(void* h, const double* firsts, int64_t n, double hcell, double clamp, int threads, double* f_out,
                   int16_t* q_out, int32_t* kind_out, uint32_t* words_out) {
  auto* ex = static_cast<Exact*>(h);
  parallel_for(n, threads, [&](int64_t bi) {
    V3 p(firsts[3 * bi], firsts[3 * bi + 1], firsts[3 * bi + 2]);
    double half = 4.0 * hcell;
    V3 c = p + V3(half, half, half);
    double d0 = std::fabs(ex->sdf(c, nullptr).d);
    auto at = [&](int nn) { return p + V3(hcell * (nn % 9), hcell * ((nn / 9) % 9), hcell * (nn / 81)); };
    double v[729];
    bool have[729] = {false};
    for (int step : {8, 4, 2, 1})
      for (int k = 0; k < 9; k += step)
        for (int j = 0; j < 9; j += step)
          for (int i = 0; i < 9; i += step) {
            int nn = i + 9 * j + 81 * k;
            if (have[nn]) continue;
            V3 x = at(nn);
            double f = ex->sdf_within(x, d0 + (x - c).len() + 1e-9, nullptr).d;
            v[nn] = f;
            have[nn] = true;
            double r = std::fabs(f) - clamp;
            if (r > 0.0) {
              int cells = int(std::floor(r / hcell));
              for (int kk = std::max(k - cells, 0); kk <= std::min(k + cells, 8); kk++)
                for (int jj = std::max(j - cells, 0); jj <= std::min(j + cells, 8); jj++)
                  for (int ii = std::max(i - cells, 0); ii <= std::min(i + cells, 8); ii++) {
                    int m = ii + 9 * jj + 81 * kk;
                    if (!have[m] && (at(m) - x).len() < r) {
                      v[m] = std::copysign(clamp, f);
                      have[m] = true;
                    }
                  }
            }
          }
    int16_t q[729];
    for (int nn = 0; nn < 729; nn++) {
      double f = have[nn] ? v[nn] : clamp;
      if (f_out) f_out[bi * 729 + nn] = f;
      double x = std::min(std::max(f / clamp, -1.0), 1.0) * 32767.0;
      q[nn] = int16_t(std::round(x));
      if (q_out) q_out[bi * 729 + nn] = q[nn];
    }
    if (kind_out) kind_out[bi] = packed_kind(q);
    if (words_out) pack_words(q, words_out + bi * 365);
  });
}

}  // extern "C"

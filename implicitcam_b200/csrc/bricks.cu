// The brick kernel of the exact part field on sm_100a: one warp a brick, from the
// brick's candidate list to its packed words (the reference's per-brick list, read and
// post-processing, partcache.rs:759-970).
#include <type_traits>

#include "field.cuh"
#include "kernels.h"

namespace icam {

constexpr int WARPS = 4;    // bricks a block works on at once, one a warp
constexpr int MAXC = 128;   // candidates a brick may list
constexpr int MAXSUB = 32;  // sub-patches a brick seeds from its centre
constexpr int FR = 64;      // tree nodes one level of the list's walk may hold
constexpr unsigned FULL = 0xffffffffu;

// The 26 neighbours of node n inside the brick, in the reference's order (dk, dj, di
// from -1 to 1, partcache.rs:829-839).
__device__ __forceinline__ int nb_of(int n, int k, double* dist) {
  int i = n % 9, j = (n / 9) % 9, kk = n / 81;
  int o = k < 13 ? k : k + 1;  // skip (0,0,0)
  int di = o % 3 - 1, dj = (o / 3) % 3 - 1, dk = o / 9 - 1;
  int a = i + di, b = j + dj, c = kk + dk;
  if (a < 0 || a > 8 || b < 0 || b > 8 || c < 0 || c > 8) return -1;
  *dist = sqrt(double(di * di + dj * dj + dk * dk));
  return a + 9 * b + 81 * c;
}

// A node the candidate list could not settle (more candidates than the list holds, or a
// feature whose certificate fails there): the whole tree walk with every fallback, out
// of line so the common path keeps its registers.
__device__ __noinline__ void node_fallback(const DPack& P, double3 p, double clamp, double* value, int* flag) {
  Acc A;
  point_query(P, p, clamp, A);
  finish(A, clamp, value, flag);
}

// Edges, pieces and vertices: eval_item out of line (faces and sub-patches, the common
// candidates, are evaluated in the kernel's own loop).
__device__ __noinline__ void eval_item_cold(const DPack& P, uint32_t code, double3 p, Acc& A) {
  eval_item(P, code, p, A, 0, 0.5, 0.5);
}

// A node's features whose certificate failed there (at most two), searched by
// subdivision after every other candidate has tightened the bound, nearest bound
// first (the deferral of the tree walk, restated for the list). Out of line too.
__device__ __noinline__ void node_resolve(const DPack& P, double3 p, uint32_t c0, double l0, uint32_t c1, double l1,
                                         int nd, double* best, double* sd, double* und) {
  Acc B;
  B.best = *best;
  B.sd = *sd;
  B.und = INFINITY;
  B.why = 0;
  B.ub = INFINITY;
  B.nd = 0;
  B.record = false;
  if (nd == 2 && l1 < l0) {
    uint32_t tc = c0;
    c0 = c1, c1 = tc;
    double tl = l0;
    l0 = l1, l1 = tl;
  }
  if (l0 < B.best) subdivide(P, c0, p, B);
  if (nd == 2 && l1 < B.best) subdivide(P, c1, p, B);
  *best = B.best;
  *sd = B.sd;
  *und = B.und;
}

// A seeded sub-patch's solution at the brick's centre, for first-order seeds at the
// nodes: (s, t) there, the inverse Hessian of |S - c|^2 and the tangents, so that
// (s, t)(p) ~ (s, t) + H^-1 [S_s.(p - c), S_t.(p - c)].
struct Seed {
  double s, t, i00, i01, i11;
  double ss[3], st[3];
};

// A warp's shared memory for its brick. The list before its ranking and the walk's
// frontier share room with the node values, which come later.
struct BrickSmem {
  union {
    double f[729];  // node values: exact, signed far, bridged; NaN while unknown
    struct {
      uint32_t code[MAXC];
      double lb[MAXC];
      int32_t fr[2][FR];
    } list;
  } u;
  double lb[MAXC];  // ranked candidates: lower bound at the centre, code
  uint32_t code[MAXC];
  double4 net[16];  // the control net of the sub-patch the warp is on
  float4 net32[16];
  union {
    Seed seed[MAXSUB];
    // after the nodes: node masks by row (row j + 9 k, bit i of node i + 9 j + 81 k)
    struct {
      uint32_t m0[81], m1[81], m2[81];
    } mk;
  } v;
  int8_t flag[729];
  int8_t cert[MAXC];
  int8_t slot[MAXC];
  int n;
};
static_assert(sizeof(BrickSmem) * WARPS <= 48 * 1024, "static shared memory of a block");

__device__ __forceinline__ uint32_t spread(uint32_t m) { return m | (m << 1) | (m >> 1); }

// Row masks grown by one node in every direction (the 26-neighbourhood and the node):
// rows r of this lane, up to three.
__device__ __forceinline__ uint32_t dilate_row(const uint32_t* m, int r) {
  int j = r % 9, k = r / 9;
  uint32_t d = 0;
#pragma unroll
  for (int dk = -1; dk <= 1; dk++) {
    int kk = k + dk;
    if (kk < 0 || kk > 8) continue;
#pragma unroll
    for (int dj = -1; dj <= 1; dj++) {
      int jj = j + dj;
      if (jj < 0 || jj > 8) continue;
      d |= spread(m[jj + 9 * kk]);
    }
  }
  return d & 0x1ffu;
}

// Far nodes signed by a signed neighbour, until nothing changes (partcache.rs:845-858):
// m0 / m1 the nodes of positive / negative value, m2 the far nodes not yet signed. A
// far node lies farther than the clamp from the surface, so its neighbours within a
// cell diagonal all share its sign when the clamp is at least that diagonal; a node
// offered both signs takes the positive one.
__device__ void flood(BrickSmem& S, int lane) {
  for (;;) {
    uint32_t np[3], nq[3];
    bool any = false;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      int r = lane + 32 * q;
      np[q] = nq[q] = 0;
      if (r < 81) {
        uint32_t o = S.v.mk.m2[r];
        if (o) {
          np[q] = dilate_row(S.v.mk.m0, r) & o;
          nq[q] = dilate_row(S.v.mk.m1, r) & o & ~np[q];
          any |= (np[q] | nq[q]) != 0;
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 3; q++) {
      int r = lane + 32 * q;
      if (r < 81 && (np[q] | nq[q])) {
        S.v.mk.m0[r] |= np[q];
        S.v.mk.m1[r] |= nq[q];
        S.v.mk.m2[r] &= ~(np[q] | nq[q]);
      }
    }
    __syncwarp();
    if (!__any_sync(FULL, any)) break;
  }
}

// One brick a warp:
//  0. a brick whose centre distance puts every node past the clamp is written at once;
//  1. list: the tree walked a level at a time by the warp, every leaf within half
//     sqrt(3) + clamp of the brick's centre giving its features within that bound
//     (GpuPack::list with r = 0, partcache.rs:767), ranked by the bound;
//  2. each of the first MAXSUB sub-patches: its convexity certified for the whole brick
//     and its Newton solution at the centre kept for seeds, a lane each;
//  3. 23 passes of 32 nodes: candidate by candidate, every lane on its node at once (the
//     warp leaves when all its nodes are nearer than the next bound), each node capped at
//     the clamp; a feature uncertified at a node sends that node to the tree walk;
//  4. far nodes signed, undecided ones bridged, quantised and packed.
// MIXED: sub-patches run Newton in floats on the rebased nets and are polished in
// doubles (with the critical-point test and the trim) only when their float distance
// can beat the node's answer.
template <bool MIXED>
// Two blocks a SM: the evaluators' register need (255 a thread) left unspilled beats
// more warps with spills (measured: 8 warps a SM 240 ms, 16 warps 280 ms a bake).
__global__ void __launch_bounds__(WARPS * 32, 2) k_bricks_t(BrickArgs a) {
  __shared__ BrickSmem smem[WARPS];
  const DPack& P = a.P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BrickSmem& S = smem[warp];
  unsigned long long* work = a.stats ? a.stats + 15 : nullptr;
  auto next_brick = [&](int64_t cur) -> int64_t {
    if (work) {
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(work, 1ull);
      return int64_t(__shfl_sync(FULL, b, 0));
    }
    return cur < 0 ? int64_t(blockIdx.x) * WARPS + warp : cur + int64_t(gridDim.x) * WARPS;
  };
  const double h = a.h, clamp = a.clamp;
  for (int64_t bi = next_brick(-1); bi < a.n; bi = next_brick(bi)) {
    double3 first = mk(a.firsts[3 * bi], a.firsts[3 * bi + 1], a.firsts[3 * bi + 2]);
    const double half = 4.0 * h;
    const double3 c = first + mk(half, half, half);
    const double reach = half * SQRT3 + clamp;
    const double dc = a.dcs ? a.dcs[bi] : NAN;
    // ---- 0. every node past the clamp, known from the centre alone: the field is
    // 1-Lipschitz, so |d(node)| >= |dc| - half sqrt(3), and with a margin far above the
    // rounding of both every node would come out a bound (flag 1) and the whole brick
    // the centre's sign (partcache.rs:876-892). Same outputs as reading it.
    if (isfinite(dc) && fabs(dc) - half * SQRT3 > clamp + 1e-6 * (1.0 + clamp)) {
      for (int nn = lane; nn < 729; nn += 32) {
        if (a.d_out) a.d_out[bi * 729 + nn] = clamp;
        if (a.flag_out) a.flag_out[bi * 729 + nn] = 1;
      }
      const uint32_t q = dc > 0 ? 32767u : uint32_t(uint16_t(int16_t(-32767)));
      if (a.words_out)
        for (int w = lane; w < 365; w += 32) a.words_out[bi * 365 + w] = w < 364 ? q | (q << 16) : q;
      if (lane == 0) {
        if (a.kind_out) a.kind_out[bi] = dc > 0 ? 1 : 2;
        if (a.stats) atomicAdd(&a.stats[1], 729ull);
      }
      continue;
    }
    // ---- 1. list
    if (lane == 0) {
      S.n = 0;
      S.u.list.fr[0][0] = 0;
    }
    __syncwarp();
    bool walked = true;
    {
      int cur = 0, ncur = 1;
      while (ncur > 0) {
        int nnext = 0;
        for (int base = 0; base < ncur; base += 32) {
          const int i = base + lane;
          bool inner = false;
          int32_t kid = 0;
          if (i < ncur) {
            const DBvh& nd = P.bvh[S.u.list.fr[cur][i]];
            if (box_dist_f(c, nd.lo, nd.hi) <= reach) {
              if (nd.count > 0) {
                for (int k = 0; k < nd.count; k++) {
                  uint32_t code = P.items[nd.first + k];
                  double lb = item_lb(P, code, c);
                  if (lb <= reach) {
                    int slot = atomicAdd(&S.n, 1);
                    if (slot < MAXC) {
                      S.u.list.code[slot] = code;
                      S.u.list.lb[slot] = lb;
                    }
                  }
                }
              } else {
                inner = true;
                kid = nd.first;
              }
            }
          }
          const unsigned m = __ballot_sync(FULL, inner);
          const int off = nnext + 2 * __popc(m & ((1u << lane) - 1u));
          if (inner && off + 1 < FR) {
            S.u.list.fr[cur ^ 1][off] = kid;
            S.u.list.fr[cur ^ 1][off + 1] = kid + 1;
          }
          nnext += 2 * __popc(m);
        }
        __syncwarp();
        if (nnext > FR) {  // a level wider than the frontier: every leaf instead
          walked = false;
          break;
        }
        cur ^= 1;
        ncur = nnext;
      }
    }
    if (!walked) {
      if (lane == 0) S.n = 0;
      __syncwarp();
      for (int leaf = lane; leaf < a.n_leaves; leaf += 32) {
        const DBvh& nd = P.bvh[a.leaves[leaf]];
        if (box_dist_f(c, nd.lo, nd.hi) > reach) continue;
        for (int k = 0; k < nd.count; k++) {
          uint32_t code = P.items[nd.first + k];
          double lb = item_lb(P, code, c);
          if (lb <= reach) {
            int slot = atomicAdd(&S.n, 1);
            if (slot < MAXC) {
              S.u.list.code[slot] = code;
              S.u.list.lb[slot] = lb;
            }
          }
        }
      }
    }
    __syncwarp();
    int n = S.n;
    const bool overflow = n > MAXC;
    if (overflow) n = MAXC;
    // rank sort: ties by code so the order does not depend on the list's arrival order
    for (int k = lane; k < n; k += 32) {
      double lb = S.u.list.lb[k];
      uint32_t code = S.u.list.code[k];
      int rank = 0;
      for (int j = 0; j < n; j++) {
        double l2 = S.u.list.lb[j];
        rank += (l2 < lb) || (l2 == lb && S.u.list.code[j] < code);
      }
      S.code[rank] = code;
      S.lb[rank] = lb;
    }
    __syncwarp();
    // ---- 2. certify and seed the first MAXSUB sub-patches, a lane each
    {
      int subs_before = 0;
      for (int base = 0; base < n; base += 32) {
        const int k = base + lane;
        const bool is_sub = k < n && (S.code[k] >> IK_SHIFT) == IK_SUB;
        const unsigned m = __ballot_sync(FULL, is_sub);
        const int before = subs_before + __popc(m & ((1u << lane) - 1u));
        subs_before += __popc(m);
        if (k >= n) continue;
        int slot = -1;
        int8_t cert = 0;
        if (is_sub) {
          const uint32_t idx = S.code[k] & IK_MASK;
          const DSub& s = P.subs[idx];
          cert = sub_convex(s, first, first + mk(8 * h, 8 * h, 8 * h)) ? 1 : 0;
          if (before < MAXSUB) {
            slot = before;
            const double4* cp = P.sub_cp + 16 * size_t(idx);
            double ss = 0.5, tt = 0.5;
            bool conv;
            newton_bicubic(cp, c, &ss, &tt, 12, &conv);
            SE e = eval_bicubic(cp, ss, tt);
            double3 r = e.p - c;
            double h0 = dot(e.ps, e.ps) + dot(e.pss, r), h1 = dot(e.ps, e.pt) + dot(e.pst, r),
                   h2 = dot(e.pt, e.pt) + dot(e.ptt, r);
            if (!(h0 > 0.0 && h0 * h2 - h1 * h1 > 0.0)) h0 = dot(e.ps, e.ps), h1 = dot(e.ps, e.pt), h2 = dot(e.pt, e.pt);
            double det = h0 * h2 - h1 * h1;
            Seed sd;
            sd.s = ss, sd.t = tt;
            if (fabs(det) > 1e-300) {
              sd.i00 = h2 / det, sd.i01 = -h1 / det, sd.i11 = h0 / det;
            } else {
              sd.i00 = sd.i01 = sd.i11 = 0.0;
            }
            sd.ss[0] = e.ps.x, sd.ss[1] = e.ps.y, sd.ss[2] = e.ps.z;
            sd.st[0] = e.pt.x, sd.st[1] = e.pt.y, sd.st[2] = e.pt.z;
            S.v.seed[slot] = sd;
          }
        } else if ((S.code[k] >> IK_SHIFT) == IK_FACE) {
          // a plane's trim over the feet of the whole brick (the box's corners projected,
          // with a margin over their rounding): 1 all inside, 2 all outside, 0 ask a node
          const DFace& f = P.faces[S.code[k] & IK_MASK];
          if (f.kind == S_PLANE) {
            double blo[2] = {INFINITY, INFINITY}, bhi[2] = {-INFINITY, -INFINITY};
            const double3 z = ld3(f.z), o = ld3(f.o), fx = ld3(f.x), fy = ld3(f.y);
            for (int q = 0; q < 8; q++) {
              double3 x = first + mk(q & 1 ? 8 * h : 0.0, q & 2 ? 8 * h : 0.0, q & 4 ? 8 * h : 0.0);
              double3 e = (x - z * dot(x - o, z)) - o;
              double u = dot(e, fx), v = dot(e, fy);
              blo[0] = fmin(blo[0], u), bhi[0] = fmax(bhi[0], u);
              blo[1] = fmin(blo[1], v), bhi[1] = fmax(bhi[1], v);
            }
            double m = 1e-9 * (1.0 + fmax(fmax(fabs(blo[0]), fabs(bhi[0])), fmax(fabs(blo[1]), fabs(bhi[1]))));
            blo[0] -= m, blo[1] -= m, bhi[0] += m, bhi[1] += m;
            int cls = trim_box_class(P, f, blo, bhi);
            cert = cls == 1 ? 1 : (cls == 0 ? 2 : 0);
          }
        }
        S.cert[k] = cert;
        S.slot[k] = int8_t(slot);
      }
    }
    __syncwarp();
    // ---- 3. every node: the warp's lanes walk the same ranked candidates together
    int cnt[3] = {0, 0, 0};
    for (int nn0 = 0; nn0 < 729; nn0 += 32) {
      const int nn = nn0 + lane;
      const bool live = nn < 729;
      double3 p = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
      double rr = len(p - c);
      double best = live ? clamp : -1.0;  // a lane past the last node is done
      double sdv = NAN, und = INFINITY;
      // features left for subdivision: the first two, and how many
      uint32_t dc0 = 0, dc1 = 0;
      double dl0 = 0.0, dl1 = 0.0;
      int nd = 0;
      auto defer_item = [&](uint32_t code, double lb) {
        und = fmin(und, lb);
        if (nd == 0)
          dc0 = code, dl0 = lb;
        else if (nd == 1)
          dc1 = code, dl1 = lb;
        nd++;
      };
      if (!overflow) {
        for (int k = 0; k < n; k++) {
          double lbc = S.lb[k];
          if (__all_sync(FULL, lbc - rr >= best)) break;  // ranked: nothing later is nearer
          uint32_t code = S.code[k];
          uint32_t kind = code >> IK_SHIFT, idx = code & IK_MASK;
          if (kind == IK_SUB) {  // the control net to shared memory, by the whole warp
            __syncwarp();
            if (lane < 16)
              S.net[lane] = P.sub_cp[16 * size_t(idx) + lane];
            else if (MIXED)
              S.net32[lane - 16] = P.sub_cp32[16 * size_t(idx) + lane - 16];
            __syncwarp();
          }
          if (lbc - rr >= best) continue;
          if (kind == IK_FACE) {  // eval_item's analytic face, inline
            if (S.cert[k] == 2) continue;  // no node's foot is within the trim
            const DFace& f = P.faces[idx];
            if (box_dist(p, f.box) >= best) continue;
            double3 q, fn;
            double u, v;
            if (!analytic_foot(f, p, &q, &fn, &u, &v)) continue;
            double d = len(p - q);
            if (!(d < best) || (S.cert[k] != 1 && !trim_inside(P, f, u, v))) continue;
            best = d;
            sdv = d * sgn(dot(p - q, fn));
            continue;
          }
          if (kind != IK_SUB) {
            Acc A;
            A.best = best;
            A.sd = sdv;
            A.und = INFINITY;
            A.why = 0;
            A.ub = INFINITY;
            A.nd = 0;
            A.record = true;  // an uncertified piece records its bound in und
            eval_item_cold(P, code, p, A);
            best = A.best;
            sdv = A.sd;
            if (A.und < INFINITY) defer_item(code, A.und);
            continue;
          }
          const DSub& s = P.subs[idx];
          double lb = box_dist(p, s.box);
          if (lb >= best) continue;
          if (!S.cert[k] && !sub_convex(s, p, p)) {
            defer_item(code, lb);
            continue;
          }
          int slot = S.slot[k];
          double ss = 0.5, tt = 0.5;
          if (slot >= 0) {
            const Seed& sd = S.v.seed[slot];
            double3 dp = p - c;
            double gs = sd.ss[0] * dp.x + sd.ss[1] * dp.y + sd.ss[2] * dp.z;
            double gt = sd.st[0] * dp.x + sd.st[1] * dp.y + sd.st[2] * dp.z;
            ss = fmin(fmax(sd.s + sd.i00 * gs + sd.i01 * gt, 0.0), 1.0);
            tt = fmin(fmax(sd.t + sd.i01 * gs + sd.i11 * gt, 0.0), 1.0);
          }
          const double4* cp64 = S.net;
          bool conv;
          if (MIXED) {
            const float4* cp32 = S.net32;
            float3 p32 = f3(float(p.x - s.c[0]), float(p.y - s.c[1]), float(p.z - s.c[2]));
            float sf = float(ss), tf = float(tt);
            newton_bicubic_f(cp32, p32, &sf, &tf, 8);
            SEf ef = eval_bicubic_f(cp32, sf, tf);
            float3 rf = f3(ef.p.x - p32.x, ef.p.y - p32.y, ef.p.z - p32.z);
            double d32 = sqrt(double(dotf(rf, rf)));
            // a float distance past the answer by more than its error cannot win
            if (d32 > best + 1e-4 * (1.0 + best)) continue;
            ss = sf, tt = tf;
            newton_bicubic(cp64, p, &ss, &tt, 3, &conv);
            if (!conv) newton_bicubic(cp64, p, &ss, &tt, 16, &conv);
          } else {
            newton_bicubic(cp64, p, &ss, &tt, 16, &conv);
          }
          if (!conv) {
            defer_item(code, lb);
            continue;
          }
          SE e = eval_bicubic(cp64, ss, tt);
          double d = len(e.p - p);
          if (!(d < best) || !is_critical(p, e)) continue;
          double3 nrm = cross(e.ps, e.pt);
          if (!(len(nrm) > 0.0)) continue;
          if (s.klass != 1 &&
              !trim_inside(P, P.faces[s.face], s.u0 + ss * (s.u1 - s.u0), s.v0 + tt * (s.v1 - s.v0)))
            continue;
          best = d;
          sdv = d * sgn(dot(p - e.p, unit(nrm) * P.faces[s.face].sense));
        }
      }
      if (!live) continue;
      if (nd > 0 && nd <= 2 && und < best && und <= clamp)
        node_resolve(P, p, dc0, dl0, dc1, dl1, nd, &best, &sdv, &und);
      double v;
      int f;
      if (overflow || (und < best && und <= clamp)) {
        node_fallback(P, p, clamp, &v, &f);
      } else if (!isnan(sdv) && best <= clamp) {
        v = sdv, f = 0;
      } else {
        v = clamp, f = 1;
      }
      if (a.d_out) a.d_out[bi * 729 + nn] = v;
      if (a.flag_out) a.flag_out[bi * 729 + nn] = int8_t(f);
      S.flag[nn] = int8_t(f);
      S.u.f[nn] = f == 0 ? v : NAN;
      cnt[f]++;
    }
    __syncwarp();
    const int n_exact = __reduce_add_sync(FULL, cnt[0]), n_far = __reduce_add_sync(FULL, cnt[1]),
              n_und = __reduce_add_sync(FULL, cnt[2]);
    int provisional = 0;
    if (a.words_out || a.kind_out) {
      // every node far with the centre's sign known: the last rule decides them all
      // (partcache.rs:876-892), whatever the fill and the ball would have given
      const bool all_far = n_far == 729 && isfinite(dc) && dc != 0.0;
      if (all_far) {
        for (int nn = lane; nn < 729; nn += 32) S.u.f[nn] = copysign(clamp, dc);
      } else {
        // ---- far nodes signed by a neighbour within a cell diagonal (partcache.rs:845-858)
        for (int r = lane; r < 81; r += 32) {
          uint32_t pm = 0, qm = 0, om = 0;
          for (int i = 0; i < 9; i++) {
            double v = S.u.f[9 * r + i];
            if (v > 0.0)
              pm |= 1u << i;
            else if (v < 0.0)
              qm |= 1u << i;
            else if (isnan(v) && S.flag[9 * r + i] == 1)
              om |= 1u << i;
          }
          S.v.mk.m0[r] = pm, S.v.mk.m1[r] = qm, S.v.mk.m2[r] = om;
        }
        __syncwarp();
        flood(S, lane);
        // ---- far nodes in the centre's empty ball, or the centre in theirs (partcache.rs:860-875)
        if (isfinite(dc) && dc != 0.0) {
          double rch = 0.999 * fmax(clamp, fabs(dc));
          for (int r = lane; r < 81; r += 32) {
            uint32_t om = S.v.mk.m2[r], hit = 0;
            for (int i = 0; i < 9; i++) {
              if (!((om >> i) & 1u)) continue;
              int nn = 9 * r + i;
              double3 x = first + mk(h * (nn % 9), h * ((nn / 9) % 9), h * (nn / 81));
              if (len(x - c) < rch) hit |= 1u << i;
            }
            if (hit) {
              S.v.mk.m2[r] = om & ~hit;
              if (dc > 0)
                S.v.mk.m0[r] |= hit;
              else
                S.v.mk.m1[r] |= hit;
            }
          }
          __syncwarp();
          flood(S, lane);
        }
        for (int r = lane; r < 81; r += 32) {
          uint32_t pm = S.v.mk.m0[r], qm = S.v.mk.m1[r];
          for (int i = 0; i < 9; i++) {
            int nn = 9 * r + i;
            if (!isnan(S.u.f[nn])) continue;
            if ((pm >> i) & 1u)
              S.u.f[nn] = clamp;
            else if ((qm >> i) & 1u)
              S.u.f[nn] = -clamp;
          }
        }
      }
      __syncwarp();
      // ---- bridging: the mean of the known neighbours, held in the brackets the exact
      // ones give (partcache.rs:893-916), pass after pass; m0 the nodes known when the
      // pass began, m1 the nodes it sets
      for (int r = lane; r < 81; r += 32) {
        uint32_t km = 0;
        for (int i = 0; i < 9; i++)
          if (!isnan(S.u.f[9 * r + i])) km |= 1u << i;
        S.v.mk.m0[r] = km;
      }
      __syncwarp();
      for (int pass = 0; pass < 729; pass++) {
        bool any = false;
        for (int r = lane; r < 81; r += 32) {
          uint32_t sm = dilate_row(S.v.mk.m0, r) & ~S.v.mk.m0[r] & 0x1ffu;
          S.v.mk.m1[r] = sm;
          any |= sm != 0;
        }
        if (!__any_sync(FULL, any)) break;
        __syncwarp();
        for (int nn = lane; nn < 729; nn += 32) {
          if (!((S.v.mk.m1[nn / 9] >> (nn % 9)) & 1u)) continue;
          double sum = 0.0, lo = -clamp, hi = clamp;
          int cn = 0;
          for (int k = 0; k < 26; k++) {
            double dd;
            int m = nb_of(nn, k, &dd);
            if (m < 0) continue;
            if ((S.v.mk.m0[m / 9] >> (m % 9)) & 1u) {
              sum += S.u.f[m];
              cn++;
              if (S.flag[m] == 0) {
                lo = fmax(lo, S.u.f[m] - dd * h);
                hi = fmin(hi, S.u.f[m] + dd * h);
              }
            }
          }
          double vm = sum / cn;
          S.u.f[nn] = lo <= hi ? fmin(fmax(vm, lo), hi) : 0.5 * (lo + hi);
          provisional++;
        }
        __syncwarp();
        for (int r = lane; r < 81; r += 32) S.v.mk.m0[r] |= S.v.mk.m1[r];
        __syncwarp();
      }
      // nothing around them known: the brick's far side, taken as air
      for (int nn = lane; nn < 729; nn += 32)
        if (isnan(S.u.f[nn])) {
          S.u.f[nn] = clamp;
          provisional++;
        }
      __syncwarp();
      // ---- quantise and pack
      bool pos = true, nonpos = true;
      for (int w = lane; w < 365; w += 32) {
        double q0 = round(fmin(fmax(S.u.f[2 * w] / clamp, -1.0), 1.0) * 32767.0);
        pos = pos && q0 > 0;
        nonpos = nonpos && q0 <= 0;
        uint32_t word = uint32_t(uint16_t(int16_t(q0)));
        if (2 * w + 1 < 729) {
          double q1 = round(fmin(fmax(S.u.f[2 * w + 1] / clamp, -1.0), 1.0) * 32767.0);
          pos = pos && q1 > 0;
          nonpos = nonpos && q1 <= 0;
          word |= uint32_t(uint16_t(int16_t(q1))) << 16;
        }
        if (a.words_out) a.words_out[bi * 365 + w] = word;
      }
      const bool all_pos = __all_sync(FULL, pos), all_nonpos = __all_sync(FULL, nonpos);
      if (a.kind_out && lane == 0) a.kind_out[bi] = all_pos ? 1 : (all_nonpos ? 2 : 0);
    }
    if (a.stats) {
      provisional = __reduce_add_sync(FULL, provisional);
      // the census by kind, B-spline sub-patches counted by their distinct spans
      unsigned kinds[5] = {0, 0, 0, 0, 0};
      for (int k = lane; k < n; k += 32) {
        uint32_t kind = S.code[k] >> IK_SHIFT;
        if (kind == IK_SUB) {
          const DSub& s = P.subs[S.code[k] & IK_MASK];
          bool seen = false;
          for (int j = 0; j < k && !seen; j++)
            if ((S.code[j] >> IK_SHIFT) == IK_SUB) {
              const DSub& o = P.subs[S.code[j] & IK_MASK];
              seen = o.nurbs == s.nurbs && o.span_a == s.span_a && o.span_b == s.span_b;
            }
          if (!seen) kinds[1]++;
        } else {
          kinds[kind == IK_FACE ? 0 : kind == IK_EDGE ? 2 : kind == IK_PIECE ? 3 : 4]++;
        }
      }
      for (int k = 0; k < 5; k++) kinds[k] = __reduce_add_sync(FULL, kinds[k]);
      if (lane == 0) {
        atomicAdd(&a.stats[0], (unsigned long long)n_exact);
        atomicAdd(&a.stats[1], (unsigned long long)n_far);
        atomicAdd(&a.stats[2], (unsigned long long)n_und);
        if (provisional) atomicAdd(&a.stats[3], (unsigned long long)provisional);
        atomicAdd(&a.stats[4], (unsigned long long)n);
        for (int k = 0; k < 5; k++)
          if (kinds[k]) atomicAdd(&a.stats[6 + k], (unsigned long long)kinds[k]);
        if (overflow) atomicAdd(&a.stats[5], 1ull);
      }
    }
    __syncwarp();
  }
}

void launch_bricks(const BrickArgs& a, cudaStream_t s) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (a.n + WARPS - 1) / WARPS;
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sms) * 2)));
  if (a.mixed)
    k_bricks_t<true><<<grid, WARPS * 32, 0, s>>>(a);
  else
    k_bricks_t<false><<<grid, WARPS * 32, 0, s>>>(a);
}

}  // namespace icam

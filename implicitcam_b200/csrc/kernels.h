// Launch arguments of the field kernels (kernels.cu) and their declarations.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pack.h"

namespace icam {

constexpr int kStatCount = 24;  // counters of the brick kernel (BrickArgs::stats)
// A brick's packed words in the brick kernels' output (BrickArgs::words_out): the 365 of
// the layout padded to 368, so that every brick starts on a 16-byte boundary and a lane
// stores four words (eight nodes) at once, 128-bit and coalesced.
constexpr int WORD_STRIDE = 368;

// A box of bricks being decided: its first brick, its parent's signed distance at the
// parent's centre (NaN when not known) and how far that centre is from its own.
struct Box4 {
  long long x, y, z;
  double parent_sd;
  double reach;
};

// One part of a batch (batch.cu): its pack, its level's cell side and clamp, its tree's
// leaves and its seed network (null: centre starts).
struct PartParams {
  DPack P;
  const int32_t* leaves;
  int32_t n_leaves;
  int32_t pad;
  double h, clamp;
  const float* net_feat;
  const void* net_w;
};

struct BrickArgs {
  const PartParams* parts;  // a batch: every brick's part in part_of; else null and
  const int32_t* part_of;   //   the single part's fields below
  DPack P;
  const double* firsts;  // n x 3 first nodes
  const double* dcs;     // n centre distances (NaN when not known), or null
  double dc_err;         // the centre distances' error bound (0: exact; the mixed decision's float reading)
  int64_t n;
  double h, clamp;
  const int32_t* leaves;  // the tree's leaf nodes
  int32_t n_leaves;
  int32_t mixed;          // 1: single-precision bulk with double polish
  int32_t kind_only;      // 1 (a level bake): a brick whose every node lies on one side of
                          //   the surface by more than an i16 step gets its kind alone
  const float* net_feat;  // the seed network's sub-patch features and weights
  const void* net_w;      //   (seednet.cuh), or null: centre starts
  double* d_out;          // optional n x 729 values
  int8_t* flag_out;       // optional n x 729 flags
  uint32_t* words_out;    // optional n x WORD_STRIDE packed words (365 used)
  int32_t* kind_out;      // optional n kinds (0 words, 1 air, 2 solid)
  // exact, far, undecided, bridged, pairs, overflows, census [6..10], bricks given their
  // kind from the centre alone [11], nodes the mixed kernel read in double precision [12],
  // a bulk copy that timed out [13]; [15] the kernel's brick counter; the mixed kernel's
  // float Newton iterations [16] and solves [17]. kStatCount counters, zeroed before each
  // launch; null for none (bricks then taken in a fixed order).
  unsigned long long* stats;
};

struct DecideArgs {
  DPack P;
  const int32_t* leaves;  // the tree's leaf nodes
  int32_t n_leaves;
  const Box4* boxes;
  int64_t n;  // the boxes; with n_in, the most the list holds
  // when set, the count of boxes the previous size appended (read on the device, capped
  // at n), so that sizes follow one another without the host reading counts back; the
  // launch then spans the whole GPU (sms multiprocessors) and groups are sized on it
  const unsigned long long* n_in;
  int32_t sms;
  long long size;
  double h, clamp;
  double lo[3];
  long long nb[3];
  uint32_t* map;
  Box4* next;
  int64_t next_cap;
  unsigned long long* n_next;
  int64_t* read_idx;
  double* read_dc;
  int64_t read_cap;
  unsigned long long* n_read;
  // The first round's boxes lie on a grid of first_dims boxes (x fastest, in list
  // order): their centres' values (NaN unless exact) and signs for k_first_signs.
  double* first_sd;
  int8_t* first_sign;
  long long first_dims[3];
  // the mixed form: centres the float walk left to the double walk (counted; or null)
  unsigned long long* n_double;
  // 0: the reference's rule (a box's radius is that of the box grown by the clamp,
  // partcache.rs:341-423); 1: a level bake's, the box's own radius: a box whose centre
  // lies farther than that plus the clamp from the surface has every node past the
  // clamp, so each of its bricks would be read into air or material. The map and words
  // are the same; fewer boxes and bricks are read, with shorter cuts.
  int32_t tight;
};

__global__ void k_points(DPack P, const double* xyz, int64_t n, double cap, double* value, int8_t* flag);

// The brick kernel (bricks.cu) in the arithmetic a.mixed names, one warp a brick, `warps`
// (1, 2 or 4) a block, over a grid sized for the current device.
void launch_bricks(const BrickArgs& a, cudaStream_t s, int warps = 4);
// The mixed form's brick kernel (bricks_mixed.cu): float bulk, the nodes it cannot settle
// read by the double walk afterwards; launch_bricks sends a.mixed here.
void launch_bricks_mixed(const BrickArgs& a, cudaStream_t s, int warps = 4);
// Map entries and atlas words of a batch's read bricks (batch.cu).
__global__ void k_assemble_batch(const int64_t* idx, const int32_t* part_of, const int64_t* part_off,
                                 uint32_t* const* maps, const int32_t* kind, const int64_t* slot, int64_t n,
                                 const uint32_t* words, uint32_t* atlas);
// The decision of one box size of a level (decide.cu), 32 boxes a warp; `first`: the
// level's first boxes, whose far ones then take their sign from a neighbour.
// mixed: the float reading (decide.cu decide_group_f), the same map.
void launch_decide(const DecideArgs& a, cudaStream_t s, bool first = false, bool mixed = false);

// Many parts' decisions together (decide.cu), one round a box size. Part p's fields are
// args[2p + (round & 1)]: `size` its first boxes' size (round r decides size >> r),
// boxes / next its two box regions (swapped between the pair), n_next its next count
// (cnt[2p + ((round + 1) & 1)]), n_read its read count. cnt[2p] holds the first boxes'
// count at the start; groups (n_parts + 2 values) is k_decide_prep's numbering and the
// round's boxes a group.
struct DecideBatchArgs {
  const DecideArgs* args;
  int n_parts;
  int sms;  // the device's SMs (set by launch_decide_batch)
  unsigned long long* cnt;
  int64_t* groups;
  unsigned long long* boxes_read;
  int* err;  // set when a part's box list would overflow
  int mixed;  // the float reading (decide_group_f)
};
// `rounds` rounds (the largest first box size's log2 + 1), no host synchronisation.
void launch_decide_batch(const DecideBatchArgs& b, int rounds, cudaStream_t s);
__global__ void k_gather_firsts(const int64_t* idx, int64_t n, int64_t nb0, int64_t nb1, double h, double lo0,
                                double lo1, double lo2, double* firsts);
__global__ void k_assemble(const int64_t* idx, const int32_t* kind, const int64_t* slot, int64_t n,
                           const uint32_t* words, uint32_t* map, uint32_t* atlas);
__global__ void k_is_words(const int32_t* kind, int64_t n, int64_t* flag);
__global__ void k_warm(float* out, int iters);
// Independent FMA chains in doubles (fp64) or floats: the throughput probe.
void launch_fma(bool fp64, void* out, int blocks, int threads, int iters, cudaStream_t s);

}  // namespace icam

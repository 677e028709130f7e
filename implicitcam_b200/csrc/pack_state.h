// What an IcamPack holds (include/icam_cuda.h keeps it opaque): the packed solid on the
// device, its stream, scratch grown on demand, and the seed network's state.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "pack_build.h"

// The learned seeds (seednet.cu): per sub-patch features, the network's FP32 master
// weights and Adam moments for training, the BF16 copy the kernels read, and the
// training batch. All device arrays, allocated on first use and kept in `owned`.
struct SeedNetState {
  float* feat = nullptr;    // SN_FEAT floats a sub-patch
  float* params = nullptr;  // SN_PARAMS, FP32 master
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  void* wbf = nullptr;      // BF16 transposed weights (SN_TBF) then FP32 biases
  float* x = nullptr;       // batch inputs (SN_INP a sample) and targets (4 a sample)
  float* y = nullptr;
  int64_t batch_cap = 0;
  unsigned long long* step = nullptr;  // the step the device-side training is on
  float* loss = nullptr;               // loss per step
  int64_t loss_cap = 0;
  bool ready = false;       // weights set (trained or loaded)
};

// One level of the brick cache to bake: cell side h, first node lo, nb bricks a side,
// the clamp, and the box grid's origin (the stock's low corner) when there is one.
struct LevelDesc {
  double h = 0.0, clamp = 0.0;
  double lo[3] = {0, 0, 0}, origin[3] = {0, 0, 0};
  int64_t nb[3] = {0, 0, 0};
  bool has_origin = false;
  int precision = 0;  // ICAM_FP64, ICAM_MIXED or ICAM_MIXED_LEARNED
  bool tight = false;  // the decision's tight rule (DecideArgs::tight): a level bake's
};

// The box decision of a level, left on the device in the pack's scratch: the map (read
// bricks marked), the read bricks' indices in brick order and their centre distances.
struct DecideOut {
  uint32_t* map = nullptr;
  int64_t* read_idx = nullptr;
  double* read_dc = nullptr;
  int64_t n_read = 0, boxes_read = 0, launches = 0;
  int64_t h2d_bytes = 0, d2h_bytes = 0;  // host copies the decision made
  int64_t centres_double = 0;            // the mixed form: box centres read again in double
};

namespace icam {
struct Box4;
}
// api.cu: the first boxes of a level's decision (their size in bricks returned).
long long first_boxes(const LevelDesc& L, std::vector<icam::Box4>* out, long long dims[3] = nullptr);

struct IcamPack;
// api.cu: the decision (partcache.rs:226-331) through the sort of the read bricks.
int decide_level(IcamPack* pk, const LevelDesc& L, DecideOut* out);

struct IcamPack {
  int device = 0;
  cudaStream_t stream = nullptr;
  icam::HostPack host;
  icam::DPack dev{};
  std::vector<void*> owned;  // the pack's device arrays
  std::vector<int32_t> leaves_host;
  int32_t* leaves = nullptr;
  // scratch, grown on demand
  struct Buf {
    void* p = nullptr;
    size_t n = 0;
  };
  Buf scratch[24];
  std::string err;
  unsigned long long* d_stats = nullptr;
  // the last level bake's results (scratch 3 and 17), for icam_level_read
  const uint32_t* last_map = nullptr;
  const uint32_t* last_atlas = nullptr;
  size_t last_map_entries = 0, last_slots = 0;
  SeedNetState net;
};

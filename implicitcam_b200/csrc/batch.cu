// Many parts baked together: every part's box decision in one launch a box size (warps
// take groups of 32 boxes of one part across all parts; no host synchronisation between
// sizes), one sort of all parts' read bricks, then every part's read bricks through ONE
// launch of the brick kernel fed by a device work queue (an atomic brick counter over all
// parts), one scan numbering the stored bricks and one assembly into every part's map and
// a shared atlas.
// The part after the decisions is captured as a CUDA graph and replayed while the batch's
// levels and sizes stay the same; the brick kernel's tiling (warps a block) is picked by
// timing each choice on the batch's first bake. No counterpart in the reference, which
// bakes one part at a time.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "../../include/icam_cuda.h"
#include "kernels.h"
#include "pack_state.h"

using namespace icam;

namespace icam {

constexpr int PART_SHIFT = 34;  // a read brick's sort key: part << PART_SHIFT | brick index

// Every part's read bricks (part p's n_read[p] at read_off[p]) as dense sort keys and
// centre distances: dense position j of part p is off[p] + its rank in the part's list.
__global__ void k_batch_keys(const int64_t* read_idx, const double* read_dc, const int64_t* read_off,
                             const int64_t* off, int n_parts, int64_t R, uint64_t* keys, double* dcs) {
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < R; j += int64_t(gridDim.x) * blockDim.x) {
    int lo = 0, hi = n_parts;  // off[lo] <= j < off[lo + 1]
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (off[mid] <= j) lo = mid;
      else hi = mid;
    }
    const int64_t src = read_off[lo] + (j - off[lo]);
    keys[j] = (uint64_t(lo) << PART_SHIFT) | uint64_t(read_idx[src]);
    dcs[j] = read_dc[src];
  }
}

// The sorted keys split into brick indices, parts and first nodes (as k_gather_firsts).
__global__ void k_batch_split(const uint64_t* keys, int64_t R, const DecideArgs* args, int64_t* idx, int32_t* part_of,
                              double* firsts) {
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < R; j += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t k = keys[j];
    const int p = int(k >> PART_SHIFT);
    const int64_t b = int64_t(k & ((uint64_t(1) << PART_SHIFT) - 1));
    const DecideArgs& a = args[2 * p];
    const int64_t nb0 = a.nb[0], nb1 = a.nb[1];
    const int64_t x = b % nb0, y = (b / nb0) % nb1, z = b / (nb0 * nb1);
    const double side = 8.0 * a.h;
    idx[j] = b;
    part_of[j] = p;
    firsts[3 * j] = a.lo[0] + side * x;
    firsts[3 * j + 1] = a.lo[1] + side * y;
    firsts[3 * j + 2] = a.lo[2] + side * z;
  }
}

// The stored-brick number of each part's first brick (slot at its offset), n + 1 values.
__global__ void k_part_slots(const int64_t* slot, const int64_t* off, int n, int64_t* out) {
  for (int i = threadIdx.x; i <= n; i += blockDim.x) out[i] = slot[off[i]];
}

__global__ void k_assemble_batch(const int64_t* idx, const int32_t* part_of, const int64_t* part_off,
                                 uint32_t* const* maps, const int32_t* kind, const int64_t* slot, int64_t n,
                                 const uint32_t* words, uint32_t* atlas) {
  for (int64_t i = blockIdx.x; i < n; i += gridDim.x) {
    const int k = kind[i];
    const int part = part_of[i];
    if (threadIdx.x == 0) {
      const int64_t local = slot[i] - slot[part_off[part]];
      maps[part][idx[i]] = k == 1 ? 0xffffffffu : (k == 2 ? 0xfffffffeu : uint32_t(local));
    }
    if (k == 0)
      for (int w = threadIdx.x; w < 365; w += blockDim.x) atlas[slot[i] * 365 + w] = words[i * WORD_STRIDE + w];
  }
}

}  // namespace icam

struct IcamBatch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<IcamPack*> packs;
  std::vector<void*> owned;
  struct Buf {
    void* p = nullptr;
    size_t n = 0;
  };
  Buf buf[25];
  PartParams* d_parts = nullptr;
  unsigned long long* d_stats = nullptr;
  int warps = 0;  // the tuned tiling (0: not tuned yet)
  double tune_ms[3] = {0, 0, 0};
  cudaGraphExec_t exec = nullptr;
  std::vector<int64_t> graph_key;
  std::string err;
};

namespace {

int bfail(IcamBatch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

#define BCK(call)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return bfail(bt, ICAM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int bbuf(IcamBatch* bt, int k, size_t bytes, void** out) {
  auto& b = bt->buf[k];
  if (b.n < bytes) {
    if (b.p) BCK(cudaFree(b.p));
    b.p = nullptr;
    b.n = 0;
    size_t want = std::max(bytes, size_t(1) << 16);
    BCK(cudaMalloc(&b.p, want));
    b.n = want;
  }
  *out = b.p;
  return ICAM_OK;
}

int grid_of(int64_t n, int threads) {
  return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 32)));
}

}  // namespace

extern "C" {

int icam_batch_create(IcamPack* const* packs, size_t n, IcamBatch** out, char* err, size_t errlen) {
  auto report = [&](const char* m) {
    if (err && errlen) std::snprintf(err, errlen, "%s", m);
  };
  if (!packs || !out || n == 0) {
    report("null argument");
    return ICAM_ERR_ARG;
  }
  *out = nullptr;
  for (size_t i = 0; i < n; i++) {
    if (!packs[i] || packs[i]->device != packs[0]->device) {
      report("every pack of a batch must exist and be on one device");
      return ICAM_ERR_ARG;
    }
  }
  IcamBatch* bt = new IcamBatch();
  bt->device = packs[0]->device;
  bt->packs.assign(packs, packs + n);
  auto done = [&](int rc, const char* m) -> int {
    if (rc != ICAM_OK) {
      report(m);
      icam_batch_destroy(bt);
      return rc;
    }
    *out = bt;
    return ICAM_OK;
  };
  if (cudaSetDevice(bt->device) != cudaSuccess || cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking) != cudaSuccess)
    return done(ICAM_ERR_CUDA, "cannot create the batch's stream");
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(PartParams)) != cudaSuccess) return done(ICAM_ERR_CUDA, "cudaMalloc");
  bt->owned.push_back(p);
  bt->d_parts = static_cast<PartParams*>(p);
  if (cudaMalloc(&p, kStatCount * sizeof(unsigned long long)) != cudaSuccess) return done(ICAM_ERR_CUDA, "cudaMalloc");
  bt->owned.push_back(p);
  bt->d_stats = static_cast<unsigned long long*>(p);
  return done(ICAM_OK, "");
}

void icam_batch_destroy(IcamBatch* bt) {
  if (!bt) return;
  cudaSetDevice(bt->device);
  if (bt->stream) cudaStreamSynchronize(bt->stream);
  if (bt->exec) cudaGraphExecDestroy(bt->exec);
  for (void* p : bt->owned) cudaFree(p);
  for (auto& b : bt->buf)
    if (b.p) cudaFree(b.p);
  if (bt->stream) cudaStreamDestroy(bt->stream);
  delete bt;
}

const char* icam_batch_last_error(const IcamBatch* bt) { return bt ? bt->err.c_str() : "null batch"; }

int icam_batch_read(IcamBatch* bt, const IcamBatchPart* part, size_t map_entries, uint32_t* map_out,
                    uint32_t* atlas_out, size_t atlas_cap_words) {
  if (!bt || !part || (map_entries && !map_out)) return bfail(bt, ICAM_ERR_ARG, "null argument");
  if (atlas_out && atlas_cap_words < part->n_slots * 365) return bfail(bt, ICAM_ERR_ARG, "atlas_out too small");
  BCK(cudaSetDevice(bt->device));
  if (map_entries)
    BCK(cudaMemcpyAsync(map_out, part->d_map, map_entries * sizeof(uint32_t), cudaMemcpyDeviceToHost, bt->stream));
  if (atlas_out && part->n_slots)
    BCK(cudaMemcpyAsync(atlas_out, part->d_atlas, part->n_slots * 365 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        bt->stream));
  BCK(cudaStreamSynchronize(bt->stream));
  return ICAM_OK;
}

int icam_batch_bake(IcamBatch* bt, const IcamBatchLevel* levels, int precision, IcamBatchPart* parts_out,
                    IcamBatchStats* stats) {
  if (!bt || !levels || !parts_out) return bfail(bt, ICAM_ERR_ARG, "null argument");
  if (precision < ICAM_FP64 || precision > ICAM_MIXED_LEARNED) return bfail(bt, ICAM_ERR_ARG, "unknown precision");
  BCK(cudaSetDevice(bt->device));
  const int n = int(bt->packs.size());
  cudaStream_t s = bt->stream;
  cudaEvent_t ev[4];
  for (auto& e : ev) BCK(cudaEventCreate(&e));
  auto cleanup = [&]() {
    for (auto& e : ev) cudaEventDestroy(e);
  };
  BCK(cudaEventRecord(ev[0], s));
  // every part's decision together: first boxes, regions of the box lists, maps and read
  // lists at per-part offsets, then one launch pair a box size
  std::vector<DecideArgs> args(2 * n);
  std::vector<std::vector<Box4>> first(n);
  std::vector<int64_t> box_off(n + 1, 0), lvl_off(n + 1, 0);
  int rounds = 0;
  for (int i = 0; i < n; i++) {
    IcamPack* pk = bt->packs[i];
    const IcamBatchLevel& lv = levels[i];
    if (!(lv.h > 0) || !(lv.clamp > 0) || lv.nb[0] <= 0 || lv.nb[1] <= 0 || lv.nb[2] <= 0) {
      cleanup();
      return bfail(bt, ICAM_ERR_ARG, "part " + std::to_string(i) + ": h, clamp and nb must be positive");
    }
    const int64_t total = lv.nb[0] * lv.nb[1] * lv.nb[2];
    if (total > (int64_t(1) << PART_SHIFT)) {
      cleanup();
      return bfail(bt, ICAM_ERR_ARG, "part " + std::to_string(i) + ": level too large");
    }
    if (precision == ICAM_MIXED_LEARNED && !pk->net.ready && pk->dev.n_subs > 0) {
      cleanup();
      return bfail(bt, ICAM_ERR_ARG, "ICAM_MIXED_LEARNED: part " + std::to_string(i) + " has no trained seed network");
    }
    BCK(cudaStreamSynchronize(pk->stream));  // the pack's uploads and training done
    LevelDesc L;
    L.h = lv.h, L.clamp = lv.clamp;
    for (int k = 0; k < 3; k++) L.lo[k] = lv.lo[k], L.nb[k] = lv.nb[k], L.origin[k] = lv.origin[k];
    L.has_origin = lv.has_origin != 0;
    const long long size = first_boxes(L, &first[i], args[2 * i].first_dims);
    int lg = 0;
    while ((1LL << lg) < size) lg++;
    rounds = std::max(rounds, lg + 1);
    // box lists: boxes of one size are disjoint and each holds a brick of the level
    box_off[i + 1] = box_off[i] + std::max<int64_t>(total + 64, 1 << 12);
    lvl_off[i + 1] = lvl_off[i] + total;
    DecideArgs& a = args[2 * i];
    a.P = pk->dev;
    a.leaves = pk->leaves;
    a.n_leaves = int32_t(pk->leaves_host.size());
    a.size = size;
    a.h = lv.h;
    a.clamp = lv.clamp;
    a.tight = 1;  // a bake: the decision's tight rule (same maps and words, fewer reads)
    for (int k = 0; k < 3; k++) a.lo[k] = lv.lo[k], a.nb[k] = lv.nb[k];
    a.next_cap = box_off[i + 1] - box_off[i];
    a.read_cap = total;
  }
  void *boxes[2], *maps_all, *ridx, *rdc, *cnt, *groups, *d_args, *d_roff, *keys[2], *firsts_sd;
  const int64_t BX = box_off[n], LV = lvl_off[n];
  std::vector<int64_t> first_off(n + 1, 0);  // the first boxes' values, then their signs
  for (int i = 0; i < n; i++) first_off[i + 1] = first_off[i] + int64_t(first[i].size());
  int r;
  if ((r = bbuf(bt, 24, first_off[n] * (sizeof(double) + 1) + 16, &firsts_sd))) {
    cleanup();
    return r;
  }
  if ((r = bbuf(bt, 12, BX * sizeof(Box4), &boxes[0])) || (r = bbuf(bt, 13, BX * sizeof(Box4), &boxes[1])) ||
      (r = bbuf(bt, 14, LV * sizeof(uint32_t), &maps_all)) || (r = bbuf(bt, 15, LV * sizeof(int64_t), &ridx)) ||
      (r = bbuf(bt, 16, LV * sizeof(double), &rdc)) ||
      (r = bbuf(bt, 17, (3 * n + 2) * sizeof(unsigned long long), &cnt)) ||
      (r = bbuf(bt, 18, (n + 2) * sizeof(int64_t), &groups)) || (r = bbuf(bt, 19, 2 * n * sizeof(DecideArgs), &d_args)) ||
      (r = bbuf(bt, 20, (n + 1) * sizeof(int64_t), &d_roff))) {
    cleanup();
    return r;
  }
  unsigned long long* c = static_cast<unsigned long long*>(cnt);  // 2n box counts, n read counts, boxes, error
  std::vector<unsigned long long> c0(3 * n + 2, 0);
  std::vector<uint32_t*> maps(n);
  for (int i = 0; i < n; i++) {
    DecideArgs& a = args[2 * i];
    maps[i] = static_cast<uint32_t*>(maps_all) + lvl_off[i];
    a.map = maps[i];
    a.read_idx = static_cast<int64_t*>(ridx) + lvl_off[i];
    a.read_dc = static_cast<double*>(rdc) + lvl_off[i];
    a.n_read = c + 2 * n + i;
    DecideArgs& b = args[2 * i + 1];
    b = a;
    a.boxes = static_cast<Box4*>(boxes[0]) + box_off[i];
    a.next = static_cast<Box4*>(boxes[1]) + box_off[i];
    a.n_next = c + 2 * i + 1;
    b.boxes = static_cast<Box4*>(boxes[1]) + box_off[i];
    b.next = static_cast<Box4*>(boxes[0]) + box_off[i];
    b.n_next = c + 2 * i;
    a.first_sd = static_cast<double*>(firsts_sd) + first_off[i];
    a.first_sign = reinterpret_cast<int8_t*>(static_cast<double*>(firsts_sd) + first_off[n]) + first_off[i];
    c0[2 * i] = first[i].size();
    if (!first[i].empty())
      BCK(cudaMemcpyAsync(static_cast<Box4*>(boxes[0]) + box_off[i], first[i].data(), first[i].size() * sizeof(Box4),
                          cudaMemcpyHostToDevice, s));
  }
  BCK(cudaMemcpyAsync(c, c0.data(), c0.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
  BCK(cudaMemcpyAsync(d_args, args.data(), args.size() * sizeof(DecideArgs), cudaMemcpyHostToDevice, s));
  BCK(cudaMemcpyAsync(d_roff, lvl_off.data(), (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  DecideBatchArgs db{};
  db.mixed = precision != ICAM_FP64;
  db.args = static_cast<const DecideArgs*>(d_args);
  db.n_parts = n;
  db.cnt = c;
  db.groups = static_cast<int64_t*>(groups);
  db.boxes_read = c + 3 * n;
  db.err = reinterpret_cast<int*>(c + 3 * n + 1);
  launch_decide_batch(db, rounds, s);
  BCK(cudaGetLastError());
  int64_t launches = 2 * rounds + 1;
  BCK(cudaMemcpyAsync(c0.data(), c, c0.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  BCK(cudaStreamSynchronize(s));
  if (c0[3 * n + 1] != 0) {
    cleanup();
    return bfail(bt, ICAM_ERR_ROOM, "box list overflow");
  }
  std::vector<int64_t> off(n + 1, 0), n_read(n);
  for (int i = 0; i < n; i++) {
    n_read[i] = int64_t(c0[2 * n + i]);
    if (n_read[i] > lvl_off[i + 1] - lvl_off[i]) {
      cleanup();
      return bfail(bt, ICAM_ERR_ROOM, "read list overflow");
    }
    off[i + 1] = off[i] + n_read[i];
  }
  const int64_t boxes_n = int64_t(c0[3 * n]);
  const int64_t R = off[n];
  const size_t Rb = size_t(std::max<int64_t>(R, 1));
  // the batch's arrays: first nodes, centre distances, brick indices and parts, words,
  // kinds, stored flags and slots, scan room, the atlas (room for every brick stored, so
  // that the whole of what follows can be one graph), part offsets and map pointers
  void *firsts, *dcs, *idx, *part_of, *words, *kind, *flags, *tmp, *atlas, *d_off, *d_maps, *d_pslot, *stmp;
  size_t tmp_bytes = 0, sort_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (int64_t*)nullptr, (int64_t*)nullptr, R + 1, s);
  int end_bit = PART_SHIFT;
  while ((int64_t(1) << (end_bit - PART_SHIFT)) < n) end_bit++;
  cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint64_t*)nullptr, (uint64_t*)nullptr, (double*)nullptr,
                                  (double*)nullptr, R, 0, end_bit, s);
  if ((r = bbuf(bt, 0, Rb * 3 * sizeof(double), &firsts)) || (r = bbuf(bt, 1, Rb * sizeof(double), &dcs)) ||
      (r = bbuf(bt, 2, Rb * sizeof(int64_t), &idx)) || (r = bbuf(bt, 3, Rb * sizeof(int32_t), &part_of)) ||
      (r = bbuf(bt, 4, Rb * WORD_STRIDE * sizeof(uint32_t), &words)) || (r = bbuf(bt, 5, Rb * sizeof(int32_t), &kind)) ||
      (r = bbuf(bt, 6, (Rb + 1) * 2 * sizeof(int64_t), &flags)) || (r = bbuf(bt, 7, tmp_bytes + 16, &tmp)) ||
      (r = bbuf(bt, 8, Rb * 365 * sizeof(uint32_t), &atlas)) || (r = bbuf(bt, 9, (n + 1) * sizeof(int64_t), &d_off)) ||
      (r = bbuf(bt, 10, n * sizeof(uint32_t*), &d_maps)) || (r = bbuf(bt, 11, (n + 1) * sizeof(int64_t), &d_pslot)) ||
      (r = bbuf(bt, 21, Rb * sizeof(uint64_t), &keys[0])) || (r = bbuf(bt, 22, Rb * sizeof(uint64_t), &keys[1])) ||
      (r = bbuf(bt, 23, sort_bytes + 16, &stmp))) {
    cleanup();
    return r;
  }
  int64_t* slot = static_cast<int64_t*>(flags) + (Rb + 1);
  BCK(cudaMemcpyAsync(d_off, off.data(), (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  if (R > 0) {
    // the read bricks of all parts in (part, brick) order: each part's in brick order
    // (partcache.rs:486), the parts one after another
    // gathered dense into keys[0] and dcs, the distances then moved to the read lists'
    // room (free once gathered, and at least as long) as the sort's input
    double* dc_tmp = static_cast<double*>(rdc);
    k_batch_keys<<<grid_of(R, 256), 256, 0, s>>>(static_cast<const int64_t*>(ridx), static_cast<const double*>(rdc),
                                                  static_cast<const int64_t*>(d_roff), static_cast<const int64_t*>(d_off),
                                                  n, R, static_cast<uint64_t*>(keys[0]), static_cast<double*>(dcs));
    BCK(cudaMemcpyAsync(dc_tmp, dcs, R * sizeof(double), cudaMemcpyDeviceToDevice, s));
    BCK(cub::DeviceRadixSort::SortPairs(stmp, sort_bytes, static_cast<const uint64_t*>(keys[0]),
                                        static_cast<uint64_t*>(keys[1]), static_cast<const double*>(dc_tmp),
                                        static_cast<double*>(dcs), R, 0, end_bit, s));
    k_batch_split<<<grid_of(R, 256), 256, 0, s>>>(static_cast<const uint64_t*>(keys[1]), R,
                                                   static_cast<const DecideArgs*>(d_args), static_cast<int64_t*>(idx),
                                                   static_cast<int32_t*>(part_of), static_cast<double*>(firsts));
    launches += 4;
  }
  BCK(cudaEventRecord(ev[1], s));
  std::vector<PartParams> hp(n);
  for (int i = 0; i < n; i++) {
    IcamPack* pk = bt->packs[i];
    const IcamBatchLevel& lv = levels[i];
    PartParams& q = hp[i];
    std::memset(&q, 0, sizeof(q));
    q.P = pk->dev;
    q.leaves = pk->leaves;
    q.n_leaves = int32_t(pk->leaves_host.size());
    q.h = lv.h;
    q.clamp = lv.clamp;
    if (precision == ICAM_MIXED_LEARNED && pk->dev.n_subs > 0) q.net_feat = pk->net.feat, q.net_w = pk->net.wbf;
  }
  BCK(cudaMemcpyAsync(bt->d_parts, hp.data(), n * sizeof(PartParams), cudaMemcpyHostToDevice, s));
  BCK(cudaMemcpyAsync(d_maps, maps.data(), n * sizeof(uint32_t*), cudaMemcpyHostToDevice, s));
  BrickArgs a{};
  a.parts = bt->d_parts;
  a.part_of = static_cast<const int32_t*>(part_of);
  a.firsts = static_cast<const double*>(firsts);
  a.dcs = static_cast<const double*>(dcs);
  a.n = R;
  a.mixed = precision != ICAM_FP64;
  a.kind_only = 1;
  a.words_out = static_cast<uint32_t*>(words);
  a.kind_out = static_cast<int32_t*>(kind);
  a.stats = bt->d_stats;
  // the tiling: warps a block, each choice timed once on the batch's first bake (on up
  // to 65,536 of its bricks) and the fastest kept
  if (bt->warps == 0 && R > 0) {
    const int choices[3] = {1, 2, 4};
    BrickArgs t = a;
    t.n = std::min<int64_t>(R, 65536);
    float best = 1e30f;
    for (int c = 0; c < 3; c++) {
      BCK(cudaMemsetAsync(bt->d_stats, 0, kStatCount * sizeof(unsigned long long), s));
      BCK(cudaEventRecord(ev[2], s));
      launch_bricks(t, s, choices[c]);
      BCK(cudaGetLastError());
      BCK(cudaEventRecord(ev[3], s));
      BCK(cudaEventSynchronize(ev[3]));
      float ms = 0.f;
      BCK(cudaEventElapsedTime(&ms, ev[2], ev[3]));
      bt->tune_ms[c] = ms;
      if (ms < best) best = ms, bt->warps = choices[c];
    }
  }
  // everything after the decisions as one graph, replayed while the key holds
  std::vector<int64_t> key = {R, precision, bt->warps, int64_t(reinterpret_cast<intptr_t>(words)),
                              int64_t(reinterpret_cast<intptr_t>(atlas)), int64_t(reinterpret_cast<intptr_t>(tmp))};
  for (int i = 0; i < n; i++) key.push_back(int64_t(reinterpret_cast<intptr_t>(maps[i])));
  bool replayed = bt->exec && key == bt->graph_key;
  BCK(cudaEventRecord(ev[2], s));
  if (R > 0) {
    if (!replayed) {
      if (bt->exec) cudaGraphExecDestroy(bt->exec);
      bt->exec = nullptr;
      cudaGraph_t graph = nullptr;
      BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaMemsetAsync(bt->d_stats, 0, kStatCount * sizeof(unsigned long long), s);
      launch_bricks(a, s, bt->warps);
      k_is_words<<<grid_of(R, 256), 256, 0, s>>>(static_cast<const int32_t*>(kind), R, static_cast<int64_t*>(flags));
      cudaMemsetAsync(static_cast<int64_t*>(flags) + R, 0, sizeof(int64_t), s);
      cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, static_cast<const int64_t*>(flags), slot, R + 1, s);
      k_part_slots<<<1, 256, 0, s>>>(slot, static_cast<const int64_t*>(d_off), n, static_cast<int64_t*>(d_pslot));
      k_assemble_batch<<<grid_of(R, 1), 128, 0, s>>>(static_cast<const int64_t*>(idx), static_cast<const int32_t*>(part_of),
                                                     static_cast<const int64_t*>(d_off),
                                                     static_cast<uint32_t* const*>(d_maps), static_cast<const int32_t*>(kind),
                                                     slot, R, static_cast<const uint32_t*>(words),
                                                     static_cast<uint32_t*>(atlas));
      cudaError_t ce = cudaStreamEndCapture(s, &graph);
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&bt->exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (ce != cudaSuccess) {
        cleanup();
        bt->exec = nullptr;
        return bfail(bt, ICAM_ERR_CUDA, std::string("the batch's graph: ") + cudaGetErrorString(ce));
      }
      bt->graph_key = key;
    }
    BCK(cudaGraphLaunch(bt->exec, s));
    launches += 6;
  }
  BCK(cudaEventRecord(ev[3], s));
  std::vector<int64_t> pslot(n + 1, 0);
  if (R > 0) BCK(cudaMemcpyAsync(pslot.data(), d_pslot, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  unsigned long long st[kStatCount] = {0};
  BCK(cudaMemcpyAsync(st, bt->d_stats, sizeof(st), cudaMemcpyDeviceToHost, s));
  BCK(cudaStreamSynchronize(s));
  for (int i = 0; i < n; i++) {
    parts_out[i].d_map = maps[i];
    parts_out[i].d_atlas = static_cast<const uint32_t*>(atlas) + size_t(pslot[i]) * 365;
    parts_out[i].n_slots = size_t(pslot[i + 1] - pslot[i]);
    parts_out[i].bricks_read = n_read[i];
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->parts = n;
    stats->boxes_read = boxes_n;
    stats->bricks_read = R;
    stats->bricks_words = pslot[n];
    stats->nodes_exact = int64_t(st[0]);
    stats->nodes_undecided = int64_t(st[2]);
    stats->bricks_settled = int64_t(st[11]);
    stats->kernel_launches = launches;
    stats->warps = bt->warps;
    stats->graph_replayed = replayed ? 1 : 0;
    for (int c = 0; c < 3; c++) stats->tune_ms[c] = bt->tune_ms[c];
    float ms;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    stats->ms_decide = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    stats->ms_bricks = ms;
  }
  cleanup();
  return ICAM_OK;
}

}  // extern "C"
